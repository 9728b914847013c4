// Host mesh processing: MSH 4.1 input, faces, geometry, P1 gradients, P2 edge numbering,
// boundary tagging. Behaviour follows src/Mesh/Mesh.cpp of the reference (line numbers cited
// per function); the face and edge builds are bucket+sort based instead of std::map based and
// produce the same orders.
#include "Mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <unordered_map>

namespace {

constexpr int kLocalFaces[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
constexpr int kEdgePairs[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

// Stable counting sort of record indices by an integer key in [0, nkeys).
template <class KeyFn>
std::vector<int64_t> bucket_by(size_t n, size_t nkeys, KeyFn key, std::vector<int64_t> &offsets) {
  offsets.assign(nkeys + 1, 0);
  for (size_t r = 0; r < n; ++r) offsets[key(r) + 1]++;
  for (size_t k = 0; k < nkeys; ++k) offsets[k + 1] += offsets[k];
  std::vector<int64_t> order(n);
  std::vector<int64_t> fill(offsets.begin(), offsets.end() - 1);
  for (size_t r = 0; r < n; ++r) order[fill[key(r)]++] = (int64_t)r;
  return order;
}

}  // namespace

// src/Mesh/Mesh.cpp:16-144 (reader semantics: entity blocks list all tags, then all
// coordinates; only element type 4 is kept; unknown node ids are an error).
void Mesh::generateFromMshFile(const std::string &filename) {
  std::ifstream ifs(filename);
  if (!ifs.is_open()) {
    throw std::runtime_error("[Mesh] Could not open msh file: " + filename);
  }
  std::vector<Vec3> verts;
  std::vector<std::array<int, 4>> tets;
  std::unordered_map<long long, int> node_index;

  std::string line;
  while (std::getline(ifs, line)) {
    if (line.empty()) continue;
    if (line == "$Nodes") {
      if (!std::getline(ifs, line)) break;
      long long nblocks = 0, nnodes = 0, mintag = 0, maxtag = 0;
      std::sscanf(line.c_str(), "%lld %lld %lld %lld", &nblocks, &nnodes, &mintag, &maxtag);
      verts.reserve((size_t)std::max<long long>(nnodes, 0));
      node_index.reserve((size_t)std::max<long long>(nnodes, 0) * 2);
      for (long long b = 0; b < nblocks; ++b) {
        if (!std::getline(ifs, line)) break;
        long long edim = 0, etag = 0, param = 0, nin = 0;
        std::sscanf(line.c_str(), "%lld %lld %lld %lld", &edim, &etag, &param, &nin);
        std::vector<long long> tags((size_t)nin);
        for (long long i = 0; i < nin; ++i) {
          if (!std::getline(ifs, line)) throw std::runtime_error("Unexpected EOF in Node Tags");
          tags[(size_t)i] = std::stoll(line);
        }
        for (long long i = 0; i < nin; ++i) {
          if (!std::getline(ifs, line)) throw std::runtime_error("Unexpected EOF in Node Coords");
          const char *s = line.c_str();
          char *end = nullptr;
          double x = std::strtod(s, &end);
          double y = std::strtod(end, &end);
          double z = std::strtod(end, &end);
          node_index[tags[(size_t)i]] = (int)verts.size();
          verts.emplace_back(x, y, z);
        }
      }
    } else if (line == "$Elements") {
      if (!std::getline(ifs, line)) break;
      long long nblocks = 0, nel = 0, mintag = 0, maxtag = 0;
      std::sscanf(line.c_str(), "%lld %lld %lld %lld", &nblocks, &nel, &mintag, &maxtag);
      for (long long b = 0; b < nblocks; ++b) {
        if (!std::getline(ifs, line)) break;
        long long edim = 0, etag = 0, etype = 0, nin = 0;
        std::sscanf(line.c_str(), "%lld %lld %lld %lld", &edim, &etag, &etype, &nin);
        if (etype == 4) {
          tets.reserve(tets.size() + (size_t)nin);
          for (long long i = 0; i < nin; ++i) {
            if (!std::getline(ifs, line)) break;
            long long tag = 0, n[4] = {0, 0, 0, 0};
            std::sscanf(line.c_str(), "%lld %lld %lld %lld %lld", &tag, &n[0], &n[1], &n[2], &n[3]);
            std::array<int, 4> t{};
            for (int k = 0; k < 4; ++k) {
              auto it = node_index.find(n[k]);
              if (it == node_index.end()) {
                throw std::runtime_error("[Mesh] Element references unknown node id: " +
                                         std::to_string(n[0]));
              }
              t[k] = it->second;
            }
            tets.push_back(t);
          }
        } else {
          for (long long i = 0; i < nin; ++i) std::getline(ifs, line);
        }
      }
    }
  }
  if (verts.empty() || tets.empty()) {
    throw std::runtime_error("[Mesh] Failed to read vertices or tets from msh.");
  }
  vertices_ = std::move(verts);
  tets_.clear();
  tets_.resize(tets.size());
  for (size_t t = 0; t < tets.size(); ++t) tets_[t].vertids = tets[t];
  finalizeFromArrays(true);
}

void Mesh::generateFromArrays(const std::vector<Vec3> &vertices,
                              const std::vector<std::array<int, 4>> &tets) {
  if (vertices.empty() || tets.empty()) {
    throw std::runtime_error("[Mesh] empty vertex or tet array.");
  }
  for (const auto &t : tets) {
    for (int k = 0; k < 4; ++k) {
      if (t[k] < 0 || (size_t)t[k] >= vertices.size()) {
        throw std::runtime_error("[Mesh] Element references unknown node id: " +
                                 std::to_string(t[k]));
      }
    }
  }
  vertices_ = vertices;
  tets_.clear();
  tets_.resize(tets.size());
  for (size_t t = 0; t < tets.size(); ++t) tets_[t].vertids = tets[t];
  finalizeFromArrays(true);
}

// Post-load pipeline of the MSH reader (src/Mesh/Mesh.cpp:130-143).
void Mesh::finalizeFromArrays(bool check_degenerate) {
  buildConnectivity();
  computeGeometry();
  ensureConsistentFaceNormals();
  computeShapeFunctionGradients();
  buildP2EdgeNodes();
  computeMinEdgeLength();
  solid_vert_bc_types_.resize(vertices_.size(), SolidBCType::Undefined);
  p1_fluid_vert_bc_types_.resize(vertices_.size(), FluidBCType::Undefined);
  if (check_degenerate && hasDegenerateTet()) {
    throw std::runtime_error("[Mesh] degenerate tetrahedral elements found.\n");
  }
}

// src/Mesh/Mesh.cpp:146-225 (vertex order i fastest, 6 tets per cell around the v0-v7
// diagonal).
void Mesh::generateStructuredRectangularPrism(double length, double width, double height, int nx,
                                              int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) {
    throw std::invalid_argument("nx, ny, nz must be >= 1");
  }
  const int nxp = nx + 1, nyp = ny + 1, nzp = nz + 1;
  const double dx = length / static_cast<double>(nx);
  const double dy = width / static_cast<double>(ny);
  const double dz = height / static_cast<double>(nz);
  auto idx = [nxp, nyp](int i, int j, int k) { return i + nxp * (j + nyp * k); };
  vertices_.clear();
  tets_.clear();
  vertices_.reserve((size_t)nxp * nyp * nzp);
  for (int k = 0; k < nzp; ++k)
    for (int j = 0; j < nyp; ++j)
      for (int i = 0; i < nxp; ++i)
        vertices_.emplace_back(static_cast<double>(i) * dx, static_cast<double>(j) * dy,
                               static_cast<double>(k) * dz);
  tets_.reserve((size_t)nx * ny * nz * 6);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int v0 = idx(i, j, k), v1 = idx(i + 1, j, k), v2 = idx(i, j + 1, k),
                  v3 = idx(i + 1, j + 1, k), v4 = idx(i, j, k + 1), v5 = idx(i + 1, j, k + 1),
                  v6 = idx(i, j + 1, k + 1), v7 = idx(i + 1, j + 1, k + 1);
        const int cells[6][4] = {{v0, v1, v3, v7}, {v0, v3, v2, v7}, {v0, v2, v6, v7},
                                 {v0, v6, v4, v7}, {v0, v4, v5, v7}, {v0, v5, v1, v7}};
        for (auto &c : cells) {
          Tet t;
          t.vertids = {c[0], c[1], c[2], c[3]};
          tets_.push_back(t);
        }
      }
  finalizeFromArrays(false);
}

// Procedural cylinder (replaces the TetGen path for synthetic inputs). Disk: ring 0 is the
// centre, ring k (1..rings) has 6k points at radius R*k/rings; consecutive rings are stitched by
// an angular merge walk. Axis: `layers` equal prism layers from x=0 to x=L. Each prism is split
// into 3 tets with the minimum-global-index rule (Dompierre et al. 1999), which makes the
// diagonals of shared quad faces agree, so the tet mesh is conforming. Tets are oriented with
// positive signed volume.
void Mesh::generateCylinder(double length, double radius, int rings, int layers) {
  if (rings < 1 || layers < 1 || !(length > 0.0) || !(radius > 0.0)) {
    throw std::invalid_argument("cylinder: rings, layers >= 1 and positive length/radius required");
  }
  const double two_pi = 2.0 * M_PI;
  std::vector<std::pair<double, double>> disk;  // (y, z)
  std::vector<int> ring_start(rings + 2, 0), ring_size(rings + 1, 0);
  disk.emplace_back(0.0, 0.0);
  ring_size[0] = 1;
  for (int k = 1; k <= rings; ++k) {
    ring_start[k] = (int)disk.size();
    const int m = 6 * k;
    ring_size[k] = m;
    const double r = radius * (double)k / (double)rings;
    for (int j = 0; j < m; ++j) {
      const double th = two_pi * (double)j / (double)m;
      disk.emplace_back(r * std::cos(th), r * std::sin(th));
    }
  }
  std::vector<std::array<int, 3>> tris;
  for (int k = 1; k <= rings; ++k) {
    const int ma = ring_size[k - 1], mb = ring_size[k];
    const int sa = ring_start[k - 1], sb = ring_start[k];
    int i = 0, j = 0;
    while (i < ma || j < mb) {
      const double next_a = (k == 1) ? 2.0 : (double)(i + 1) / (double)ma;  // centre never advances
      const double next_b = (double)(j + 1) / (double)mb;
      const bool advance_inner = (j >= mb) || (i < ma && k > 1 && next_a < next_b);
      const int in_i = sa + (i % ma), out_j = sb + (j % mb);
      if (advance_inner) {
        tris.push_back({in_i, out_j, sa + ((i + 1) % ma)});
        ++i;
      } else {
        tris.push_back({in_i, out_j, sb + ((j + 1) % mb)});
        ++j;
      }
      if (k == 1 && j >= mb) break;
    }
  }
  const int np = (int)disk.size();
  vertices_.clear();
  vertices_.reserve((size_t)np * (layers + 1));
  for (int l = 0; l <= layers; ++l) {
    const double x = length * (double)l / (double)layers;
    for (int q = 0; q < np; ++q) vertices_.emplace_back(x, disk[q].first, disk[q].second);
  }
  static const int perm[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 2, 0, 4, 5, 3}, {2, 0, 1, 5, 3, 4},
                                 {3, 5, 4, 0, 2, 1}, {4, 3, 5, 1, 0, 2}, {5, 4, 3, 2, 1, 0}};
  tets_.clear();
  tets_.reserve(tris.size() * (size_t)layers * 3);
  for (int l = 0; l < layers; ++l) {
    for (const auto &tr : tris) {
      int P[6];
      for (int a = 0; a < 3; ++a) {
        P[a] = l * np + tr[a];
        P[a + 3] = (l + 1) * np + tr[a];
      }
      int imin = 0;
      for (int a = 1; a < 6; ++a)
        if (P[a] < P[imin]) imin = a;
      int V[6];
      for (int a = 0; a < 6; ++a) V[a] = P[perm[imin][a]];
      int out[3][4];
      if (std::min(V[1], V[5]) < std::min(V[2], V[4])) {
        const int o[3][4] = {{V[0], V[1], V[2], V[5]}, {V[0], V[1], V[5], V[4]}, {V[0], V[4], V[5], V[3]}};
        std::memcpy(out, o, sizeof(out));
      } else {
        const int o[3][4] = {{V[0], V[1], V[2], V[4]}, {V[0], V[4], V[2], V[5]}, {V[0], V[4], V[5], V[3]}};
        std::memcpy(out, o, sizeof(out));
      }
      for (auto &c : out) {
        const Vec3 &a = vertices_[c[0]], &b = vertices_[c[1]], &cc = vertices_[c[2]], &d = vertices_[c[3]];
        const double det = (b - a).cross(cc - a).dot(d - a);
        Tet t;
        if (det < 0.0)
          t.vertids = {c[0], c[1], c[3], c[2]};
        else
          t.vertids = {c[0], c[1], c[2], c[3]};
        tets_.push_back(t);
      }
    }
  }
  finalizeFromArrays(true);
}

namespace {

struct YGeom {
  Vec3 a[3], b[3], d[3];
  double r[3];
  double k;
  // signed distance to the capsule union (smooth, quadratic polynomial min), cut by the inlet
  // plane x = 0 and the two daughter end planes
  double sdf(const Vec3 &p) const {
    double f = 0.0;
    for (int s = 0; s < 3; ++s) {
      const Vec3 ab = b[s] - a[s];
      double t = (p - a[s]).dot(ab) / ab.dot(ab);
      t = std::min(1.0, std::max(0.0, t));
      const double di = (p - (a[s] + ab * t)).norm() - r[s];
      if (s == 0) {
        f = di;
      } else {
        const double h = std::max(k - std::fabs(f - di), 0.0) / k;
        f = std::min(f, di) - h * h * k * 0.25;
      }
    }
    f = std::max(f, -p.x());
    for (int s = 1; s < 3; ++s) f = std::max(f, (p - b[s]).dot(d[s]));
    return f;
  }
  Vec3 grad(const Vec3 &p, double h) const {
    Vec3 g;
    for (int c = 0; c < 3; ++c) {
      Vec3 e(0, 0, 0);
      e[c] = h;
      g[c] = (sdf(p + e) - sdf(p - e)) / (2.0 * h);
    }
    return g;
  }
};

double signed_volume(const Vec3 &a, const Vec3 &b, const Vec3 &c, const Vec3 &d) {
  return (b - a).cross(c - a).dot(d - a) / 6.0;
}

}  // namespace

void Mesh::generateYBifurcation(const YBifurcation &sp) {
  if (!(sp.cell > 0.0) || !(sp.parent_radius > 0.0) || !(sp.daughter_radius > 0.0) ||
      !(sp.parent_length > 0.0) || !(sp.daughter_length > 0.0) || !(sp.blend > 0.0))
    throw std::invalid_argument("yBifurcation: positive sizes required");
  YGeom G;
  const double ang = sp.angle_deg * M_PI / 180.0;
  G.a[0] = Vec3(0, 0, 0);
  G.b[0] = Vec3(sp.parent_length, 0, 0);
  G.r[0] = sp.parent_radius;
  for (int s = 1; s < 3; ++s) {
    const double sg = (s == 1) ? 1.0 : -1.0;
    G.d[s] = Vec3(std::cos(ang), sg * std::sin(ang), 0.0);
    G.a[s] = G.b[0];
    G.b[s] = G.a[s] + G.d[s] * sp.daughter_length;
    G.r[s] = sp.daughter_radius;
  }
  G.k = sp.blend;
  const double a = sp.cell;
  // lattice: x from 0 (the inlet plane is a lattice plane), y and z symmetric about 0
  double xmax = sp.parent_length + sp.parent_radius, ymax = sp.parent_radius;
  for (int s = 1; s < 3; ++s) {
    xmax = std::max(xmax, G.b[s].x() + sp.daughter_radius);
    ymax = std::max(ymax, std::fabs(G.b[s].y()) + sp.daughter_radius);
  }
  const double zmax = std::max(sp.parent_radius, sp.daughter_radius) + sp.blend;
  const int nx = (int)std::ceil(xmax / a) + 1;
  const int ny = 2 * ((int)std::ceil(ymax / a) + 1), nz = 2 * ((int)std::ceil(zmax / a) + 1);
  const double y0 = -0.5 * ny * a, z0 = -0.5 * nz * a;
  if ((double)nx * ny * nz > 2.0e9) throw std::invalid_argument("yBifurcation: lattice too large");
  auto node_id = [&](int i, int j, int k) -> int64_t { return ((int64_t)k * (ny + 1) + j) * (nx + 1) + i; };
  auto node_pos = [&](int i, int j, int k) { return Vec3(i * a, y0 + j * a, z0 + k * a); };
  // Kuhn subdivision: the 6 monotone lattice paths from corner 000 to 111
  static const int paths[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
  std::vector<int64_t> used_nodes;
  std::vector<std::array<int64_t, 4>> ltets;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const Vec3 cc = node_pos(i, j, k) + Vec3(0.5 * a, 0.5 * a, 0.5 * a);
        if (G.sdf(cc) > 1.0 * a) continue;  // no tet of this cube can be inside
        for (const auto &pth : paths) {
          int c[3] = {0, 0, 0};
          std::array<int64_t, 4> t;
          Vec3 cen(0, 0, 0);
          t[0] = node_id(i, j, k);
          cen = cen + node_pos(i, j, k);
          for (int q = 0; q < 3; ++q) {
            c[pth[q]] = 1;
            t[q + 1] = node_id(i + c[0], j + c[1], k + c[2]);
            cen = cen + node_pos(i + c[0], j + c[1], k + c[2]);
          }
          if (G.sdf(cen * 0.25) < 0.0) ltets.push_back(t);
        }
      }
  if (ltets.empty()) throw std::invalid_argument("yBifurcation: empty mesh");
  // compact numbering in lattice order
  for (const auto &t : ltets)
    for (int q = 0; q < 4; ++q) used_nodes.push_back(t[q]);
  std::sort(used_nodes.begin(), used_nodes.end());
  used_nodes.erase(std::unique(used_nodes.begin(), used_nodes.end()), used_nodes.end());
  std::vector<Vec3> verts(used_nodes.size());
  for (size_t v = 0; v < used_nodes.size(); ++v) {
    const int64_t id = used_nodes[v];
    const int i = (int)(id % (nx + 1)), j = (int)((id / (nx + 1)) % (ny + 1)), k = (int)(id / ((int64_t)(nx + 1) * (ny + 1)));
    verts[v] = node_pos(i, j, k);
  }
  std::vector<std::array<int, 4>> tets(ltets.size());
  for (size_t t = 0; t < ltets.size(); ++t) {
    for (int q = 0; q < 4; ++q)
      tets[t][q] = (int)(std::lower_bound(used_nodes.begin(), used_nodes.end(), ltets[t][q]) - used_nodes.begin());
    if (signed_volume(verts[tets[t][0]], verts[tets[t][1]], verts[tets[t][2]], verts[tets[t][3]]) < 0.0)
      std::swap(tets[t][2], tets[t][3]);
  }
  ltets.clear();
  // classify the lattice boundary faces: inlet (on x = 0), outlet s (outward normal along the
  // daughter axis, within 1.5 cells of its end plane), wall (the rest)
  Mesh lat;
  lat.generateFromArrays(verts, tets);
  const size_t nv = verts.size();
  std::vector<unsigned char> is_wall(nv, 0), is_in(nv, 0), out_of(nv, 0);
  std::vector<int> face_kind(lat.faces_.size(), -1);  // 0 wall, 1 inlet, 2/3 outlet
  for (size_t fi = 0; fi < lat.faces_.size(); ++fi) {
    const Face &f = lat.faces_[fi];
    if (f.tet_b != -1) continue;
    const auto &fv = f.vertids;
    Vec3 n = f.normal;
    const Vec3 tc = lat.tets_[f.tet_a].centroid;
    if (n.dot(f.center - tc) < 0.0) n = -n;
    int kind = 0;
    if (verts[fv[0]].x() == 0.0 && verts[fv[1]].x() == 0.0 && verts[fv[2]].x() == 0.0) {
      kind = 1;
    } else {
      for (int s = 1; s < 3; ++s) {
        bool near = n.dot(G.d[s]) > 0.3;
        for (int q = 0; q < 3 && near; ++q) near = (verts[fv[q]] - G.b[s]).dot(G.d[s]) > -1.5 * a;
        if (near) kind = 1 + s;
      }
    }
    face_kind[fi] = kind;
    for (int q = 0; q < 3; ++q) {
      if (kind == 0) is_wall[fv[q]] = 1;
      if (kind == 1) is_in[fv[q]] = 1;
      if (kind >= 2) out_of[fv[q]] = (unsigned char)kind;
    }
  }
  // vertex -> tets
  std::vector<int> vt_ptr(nv + 1, 0), vt(tets.size() * 4);
  for (const auto &t : tets)
    for (int q = 0; q < 4; ++q) vt_ptr[t[q] + 1]++;
  for (size_t v = 0; v < nv; ++v) vt_ptr[v + 1] += vt_ptr[v];
  {
    std::vector<int> fill(vt_ptr.begin(), vt_ptr.end() - 1);
    for (size_t t = 0; t < tets.size(); ++t)
      for (int q = 0; q < 4; ++q) vt[fill[tets[t][q]]++] = (int)t;
  }
  const double vmin = 0.3 * a * a * a / 6.0;  // keep moved tets at >= 30% of the lattice tet volume
  auto try_move = [&](size_t v, const Vec3 &target, double max_step) {
    const Vec3 orig = verts[v];
    Vec3 step = target - orig;
    if (step.norm() > max_step) step = step * (max_step / step.norm());
    for (int attempt = 0; attempt < 4; ++attempt) {
      verts[v] = orig + step;
      bool ok = true;
      for (int q = vt_ptr[v]; q < vt_ptr[v + 1] && ok; ++q) {
        const auto &t = tets[vt[q]];
        ok = signed_volume(verts[t[0]], verts[t[1]], verts[t[2]], verts[t[3]]) > vmin;
      }
      if (ok) return;
      step = step * 0.5;
    }
    verts[v] = orig;
  };
  for (size_t v = 0; v < nv; ++v) {
    if (!is_wall[v]) continue;
    Vec3 p = verts[v];
    for (int it = 0; it < 3; ++it) {
      const Vec3 g = G.grad(p, 1e-4 * a);
      const double g2 = g.dot(g);
      if (g2 < 1e-12) break;
      p = p - g * (G.sdf(p) / g2);
    }
    if (is_in[v]) p[0] = 0.0;  // inlet rim vertices stay on the inlet plane
    try_move(v, p, 0.5 * a);
  }
  for (size_t v = 0; v < nv; ++v) {
    if (!out_of[v]) continue;
    const int s = out_of[v] - 1;
    const Vec3 p = verts[v] - G.d[s] * (verts[v] - G.b[s]).dot(G.d[s]);
    try_move(v, p, 1.6 * a);
  }
  generateFromArrays(verts, tets);
  // tags: boundary faces in their sorted order tag their vertices Wall, inlet/outlet faces then
  // overwrite with Inlet/Outlet (the write order of setupBoundaryConditions)
  for (size_t v = 0; v < vertices_.size(); ++v) setFluidVertexBC(v, FluidBCType::Internal);
  for (size_t fi = 0; fi < faces_.size(); ++fi) {
    const Face &f = faces_[fi];
    if (f.tet_b != -1) continue;
    const auto &fv = f.vertids;
    for (const int vi : fv) setFluidVertexBC(vi, FluidBCType::Wall);
    if (is_in[fv[0]] && is_in[fv[1]] && is_in[fv[2]] && vertices_[fv[0]].x() == 0.0 &&
        vertices_[fv[1]].x() == 0.0 && vertices_[fv[2]].x() == 0.0) {
      for (const int vi : fv) setFluidVertexBC(vi, FluidBCType::Inlet);
    } else if (out_of[fv[0]] && out_of[fv[0]] == out_of[fv[1]] && out_of[fv[0]] == out_of[fv[2]]) {
      for (const int vi : fv) setFluidVertexBC(vi, FluidBCType::Outlet);
    }
  }
  setP2BoundariesFromP1Boundaries();
}

void Mesh::writeMshFile(const std::string &filename) const {
  FILE *f = std::fopen(filename.c_str(), "w");
  if (!f) throw std::runtime_error("[Mesh] Could not write msh file: " + filename);
  const size_t nv = vertices_.size(), nt = tets_.size();
  std::fprintf(f, "$MeshFormat\n4.1 0 8\n$EndMeshFormat\n");
  std::fprintf(f, "$Nodes\n1 %zu 1 %zu\n3 1 0 %zu\n", nv, nv, nv);
  for (size_t i = 0; i < nv; ++i) std::fprintf(f, "%zu\n", i + 1);
  for (size_t i = 0; i < nv; ++i)
    std::fprintf(f, "%.17g %.17g %.17g\n", vertices_[i].x(), vertices_[i].y(), vertices_[i].z());
  std::fprintf(f, "$EndNodes\n$Elements\n1 %zu 1 %zu\n3 1 4 %zu\n", nt, nt, nt);
  for (size_t t = 0; t < nt; ++t) {
    const auto &v = tets_[t].vertids;
    std::fprintf(f, "%zu %d %d %d %d\n", t + 1, v[0] + 1, v[1] + 1, v[2] + 1, v[3] + 1);
  }
  std::fprintf(f, "$EndElements\n");
  std::fclose(f);
}

// src/Mesh/Mesh.cpp:325-417. Faces are visited in their sorted order; every boundary face
// first tags its vertices Wall, then Inlet/Outlet when its centre lies within
// 0.01*extent*coverage of the inlet/outlet plane along the longest axis. Later faces overwrite.
void Mesh::setupBoundaryConditions(const Vec3 &inlet_to_outlet_direction, double percent_coverage,
                                   Mesh &mesh) {
  if (mesh.nFaces() == 0 || mesh.nVertices() < 3) return;
  Vec3 min_bounds = mesh.getVertexPositon(0);
  Vec3 max_bounds = mesh.getVertexPositon(0);
  for (size_t vi = 0; vi < mesh.nVertices(); vi++) {
    min_bounds = min_bounds.cwiseMin(mesh.getVertexPositon(vi));
    max_bounds = max_bounds.cwiseMax(mesh.getVertexPositon(vi));
  }
  const Vec3 mesh_size = max_bounds - min_bounds;
  int primary_axis = 0;
  if (mesh_size.y() > mesh_size.x() && mesh_size.y() > mesh_size.z())
    primary_axis = 1;
  else if (mesh_size.z() > mesh_size.x() && mesh_size.z() > mesh_size.y())
    primary_axis = 2;
  const double tolerance = mesh_size[primary_axis] * 0.01 * percent_coverage;
  const double inlet_pos = inlet_to_outlet_direction[primary_axis] > 0 ? min_bounds[primary_axis]
                                                                       : max_bounds[primary_axis];
  const double outlet_pos = inlet_to_outlet_direction[primary_axis] > 0 ? max_bounds[primary_axis]
                                                                        : min_bounds[primary_axis];
  for (size_t vi = 0; vi < mesh.nVertices(); vi++) {
    mesh.setFluidVertexBC(vi, FluidBCType::Internal);
    mesh.setSolidVertexBC(vi, SolidBCType::Free);
  }
  for (size_t fi = 0; fi < mesh.nFaces(); fi++) {
    Face &face = mesh.faces_[fi];
    if (mesh.isFaceInternal(fi)) {
      face.is_ecm = false;
      continue;
    }
    face.is_ecm = true;
    for (const int vi : face.vertids) mesh.setFluidVertexBC(vi, FluidBCType::Wall);
    const double dist_to_inlet = std::abs(face.center[primary_axis] - inlet_pos);
    const double dist_to_outlet = std::abs(face.center[primary_axis] - outlet_pos);
    if (dist_to_inlet < tolerance) {
      face.is_ecm = false;
      for (const int vi : face.vertids) {
        mesh.setFluidVertexBC(vi, FluidBCType::Inlet);
        mesh.setSolidVertexBC(vi, SolidBCType::Fixed);
      }
    } else if (dist_to_outlet < tolerance) {
      face.is_ecm = false;
      for (const int vi : face.vertids) {
        mesh.setFluidVertexBC(vi, FluidBCType::Outlet);
        mesh.setSolidVertexBC(vi, SolidBCType::Fixed);
      }
    }
  }
  mesh.setP2BoundariesFromP1Boundaries();
}

void Mesh::setP2BoundariesFromP1Boundaries() {
  if (p2_fluid_vert_bc_types_.empty()) buildP2EdgeNodes();
  if (p1_fluid_vert_bc_types_.size() != vertices_.size())
    p1_fluid_vert_bc_types_.resize(vertices_.size(), FluidBCType::Undefined);
  for (const auto &edge : edge_to_node_id_) {
    const int p2_idx = edge.second;
    const FluidBCType b1 = p1_fluid_vert_bc_types_[edge.first.first];
    const FluidBCType b2 = p1_fluid_vert_bc_types_[edge.first.second];
    p2_fluid_vert_bc_types_[p2_idx] =
        (b1 == b2 && b1 != FluidBCType::Internal) ? b1 : FluidBCType::Internal;
  }
}

// src/Mesh/Mesh.cpp:419-446
void Mesh::computeMinEdgeLength() {
  double min_len_sq = std::numeric_limits<double>::max();
  for (const auto &tet : tets_) {
    for (int i = 0; i < 4; ++i)
      for (int j = i + 1; j < 4; ++j) {
        const Vec3 diff = vertices_[tet.vertids[i]] - vertices_[tet.vertids[j]];
        const double len_sq = diff.dot(diff);
        if (len_sq < min_len_sq) min_len_sq = len_sq;
      }
  }
  min_edge_length_ =
      (min_len_sq == std::numeric_limits<double>::max()) ? 0.0 : std::sqrt(min_len_sq);
}

// src/Mesh/Mesh.cpp:448-471
void Mesh::computeGeometry() {
  size_t n_degenerate = 0;
  for (auto &tet : tets_) {
    const Vec3 &a = vertices_[tet.vertids[0]];
    const Vec3 &b = vertices_[tet.vertids[1]];
    const Vec3 &c = vertices_[tet.vertids[2]];
    const Vec3 &d = vertices_[tet.vertids[3]];
    tet.centroid = (((a + b) + c) + d) / 4.0;
    tet.volume = std::fabs((b - a).cross(c - a).dot(d - a) / 6.0);
    if (tet.volume <= 0.0) ++n_degenerate;
  }
  if (n_degenerate) {
    std::cerr << "[Mesh][Warning] " << n_degenerate << " degenerate tets found." << std::endl;
  }
  for (auto &face : faces_) {
    const Vec3 &a = vertices_[face.vertids[0]];
    const Vec3 &b = vertices_[face.vertids[1]];
    const Vec3 &c = vertices_[face.vertids[2]];
    const Vec3 ab = b - a;
    const Vec3 ac = c - a;
    face.normal = ac.cross(ab).normalized();
    face.area = 0.5 * ab.cross(ac).norm();
    face.center = ((a + b) + c) / 3.0;
  }
  computeShapeFunctionGradients();
}

// src/Mesh/Mesh.cpp:472-493 (neighbour lists in first-encounter order)
void Mesh::buildVertexNeighbors() {
  vertex_neighbors_.assign(vertices_.size(), {});
  for (const auto &tet : tets_) {
    for (int i = 0; i < 4; i++) {
      const int vi = tet.vertids[i];
      for (int j = 0; j < 4; j++) {
        if (i == j) continue;
        const int vj = tet.vertids[j];
        auto &nb = vertex_neighbors_[vi];
        if (std::find(nb.begin(), nb.end(), vj) == nb.end()) nb.push_back(vj);
      }
    }
  }
}

// src/Mesh/Mesh.cpp:494-588. Faces in sorted-triple order; tet_a = first tet (lowest index)
// holding the face, tet_b = the last further one; vertids in tet_a's local face order.
void Mesh::buildConnectivity() {
  faces_.clear();
  const size_t nt = tets_.size();
  const size_t nrec = nt * 4;
  std::vector<std::array<int, 3>> key(nrec);
  for (size_t t = 0; t < nt; ++t) {
    const auto &vid = tets_[t].vertids;
    for (int f = 0; f < 4; ++f) {
      std::array<int, 3> s = {vid[kLocalFaces[f][0]], vid[kLocalFaces[f][1]], vid[kLocalFaces[f][2]]};
      std::sort(s.begin(), s.end());
      key[t * 4 + f] = s;
    }
  }
  std::vector<int64_t> offs;
  std::vector<int64_t> order =
      bucket_by(nrec, vertices_.size(), [&](size_t r) { return (size_t)key[r][0]; }, offs);
  for (size_t b = 0; b < vertices_.size(); ++b) {
    std::sort(order.begin() + offs[b], order.begin() + offs[b + 1], [&](int64_t x, int64_t y) {
      if (key[x][1] != key[y][1]) return key[x][1] < key[y][1];
      if (key[x][2] != key[y][2]) return key[x][2] < key[y][2];
      return x < y;
    });
  }
  for (auto &t : tets_) {
    t.faceids = {-1, -1, -1, -1};
    t.neighbors = {-1, -1, -1, -1};
  }
  size_t r = 0;
  while (r < nrec) {
    size_t e = r + 1;
    while (e < nrec && key[order[e]] == key[order[r]]) ++e;
    const int64_t first = order[r], last = order[e - 1];
    Face face{};
    const int ta = (int)(first / 4), fa = (int)(first % 4);
    const auto &vid = tets_[ta].vertids;
    face.vertids = {vid[kLocalFaces[fa][0]], vid[kLocalFaces[fa][1]], vid[kLocalFaces[fa][2]]};
    face.tet_a = ta;
    face.face_id_a = fa;
    if (e - r >= 2) {
      face.tet_b = (int)(last / 4);
      face.face_id_b = (int)(last % 4);
    }
    const int fidx = (int)faces_.size();
    for (size_t q = r; q < e; ++q) tets_[order[q] / 4].faceids[order[q] % 4] = fidx;
    faces_.push_back(face);
    r = e;
  }
  for (const auto &face : faces_) {
    if (face.tet_a >= 0 && face.tet_b >= 0) {
      if (face.face_id_a >= 0 && face.face_id_a < 4 && face.face_id_b >= 0 && face.face_id_b < 4) {
        tets_[face.tet_a].neighbors[face.face_id_a] = face.tet_b;
        tets_[face.tet_b].neighbors[face.face_id_b] = face.tet_a;
      }
    }
  }
  buildVertexNeighbors();
}

// src/Mesh/Mesh.cpp:590-614 (exact P1 gradients from the signed 6V)
void Mesh::computeShapeFunctionGradients() {
  tet_gradients_.resize(tets_.size());
  for (size_t ti = 0; ti < tets_.size(); ti++) {
    const auto &tet = tets_[ti];
    const Vec3 &p0 = vertices_[tet.vertids[0]];
    const Vec3 &p1 = vertices_[tet.vertids[1]];
    const Vec3 &p2 = vertices_[tet.vertids[2]];
    const Vec3 &p3 = vertices_[tet.vertids[3]];
    const Vec3 e1 = p1 - p0, e2 = p2 - p0, e3 = p3 - p0;
    const double sixv = e1.dot(e2.cross(e3));
    const double invsixv = 1.0 / sixv;
    std::array<Vec3, 4> g;
    g[0] = invsixv * (p3 - p1).cross(p2 - p1);
    g[1] = invsixv * (p2 - p0).cross(p3 - p0);
    g[2] = invsixv * (p3 - p0).cross(p1 - p0);
    g[3] = invsixv * (p1 - p0).cross(p2 - p0);
    tet_gradients_[ti] = g;
  }
}

// src/Mesh/Mesh.cpp:615-639 (only internal faces are re-oriented)
void Mesh::ensureConsistentFaceNormals() {
  const double eps = 1e-12;
  for (auto &face : faces_) {
    if (face.tet_a >= 0 && face.tet_b >= 0) {
      const Vec3 &ca = tets_[face.tet_a].centroid;
      const Vec3 &cb = tets_[face.tet_b].centroid;
      const Vec3 desired = (cb - ca).normalized();
      if (face.normal.dot(desired) <= eps) {
        face.normal = -face.normal;
        std::swap(face.vertids[1], face.vertids[2]);
      } else {
        const Vec3 outward = (face.center - ca).normalized();
        if (face.normal.dot(outward) <= eps) {
          face.normal = -face.normal;
          std::swap(face.vertids[1], face.vertids[2]);
        }
      }
    }
  }
}

// src/Mesh/Mesh.cpp:641-677. Edge ids follow the first occurrence of each (min,max) pair in
// (tet, local edge) order.
void Mesh::buildP2EdgeNodes() {
  edge_nodes_.clear();
  edge_to_node_id_.clear();
  tet_edge_nodes_.assign(tets_.size(), {});
  const size_t nrec = tets_.size() * 6;
  std::vector<int> lo(nrec), hi(nrec);
  for (size_t t = 0; t < tets_.size(); ++t) {
    const auto &v = tets_[t].vertids;
    for (int e = 0; e < 6; ++e) {
      int a = v[kEdgePairs[e][0]], b = v[kEdgePairs[e][1]];
      if (a > b) std::swap(a, b);
      lo[t * 6 + e] = a;
      hi[t * 6 + e] = b;
    }
  }
  std::vector<int64_t> offs;
  std::vector<int64_t> order =
      bucket_by(nrec, vertices_.size(), [&](size_t r) { return (size_t)lo[r]; }, offs);
  for (size_t b = 0; b < vertices_.size(); ++b) {
    std::sort(order.begin() + offs[b], order.begin() + offs[b + 1], [&](int64_t x, int64_t y) {
      if (hi[x] != hi[y]) return hi[x] < hi[y];
      return x < y;
    });
  }
  // group id per record; first occurrence position per group
  std::vector<int> group_of(nrec);
  std::vector<int64_t> group_first;
  std::vector<std::pair<int, int>> group_key;
  size_t r = 0;
  while (r < nrec) {
    size_t e = r + 1;
    while (e < nrec && lo[order[e]] == lo[order[r]] && hi[order[e]] == hi[order[r]]) ++e;
    const int g = (int)group_first.size();
    group_first.push_back(order[r]);  // smallest record index in the group
    group_key.emplace_back(lo[order[r]], hi[order[r]]);
    for (size_t q = r; q < e; ++q) group_of[order[q]] = g;
    r = e;
  }
  const size_t ngroups = group_first.size();
  std::vector<int> first_mark(nrec, -1);
  for (size_t g = 0; g < ngroups; ++g) first_mark[group_first[g]] = (int)g;
  std::vector<int> group_id(ngroups, -1);
  int next_id = 0;
  for (size_t p = 0; p < nrec; ++p)
    if (first_mark[p] >= 0) group_id[first_mark[p]] = next_id++;
  edge_nodes_.resize(ngroups);
  edge_to_node_id_.resize(ngroups);
  for (size_t g = 0; g < ngroups; ++g) {
    const int id = group_id[g];
    const auto &k = group_key[g];
    edge_nodes_[id] = 0.5 * (vertices_[k.first] + vertices_[k.second]);
    edge_to_node_id_[g] = {k, id};  // groups are already in (lo,hi) order
  }
  for (size_t p = 0; p < nrec; ++p) tet_edge_nodes_[p / 6][p % 6] = group_id[group_of[p]];
  p2_fluid_vert_bc_types_.resize(edge_nodes_.size(), FluidBCType::Undefined);
}

int Mesh::getEdgeNodeId(int vi, int vj) const {
  const std::pair<int, int> key(std::min(vi, vj), std::max(vi, vj));
  auto it = std::lower_bound(
      edge_to_node_id_.begin(), edge_to_node_id_.end(), key,
      [](const std::pair<std::pair<int, int>, int> &a, const std::pair<int, int> &k) {
        return a.first < k;
      });
  if (it == edge_to_node_id_.end() || it->first != key) return -1;
  return it->second;
}

const Vec3 &Mesh::getP2NodesAtEdge(size_t vi, size_t vj) const {
  const int id = getEdgeNodeId((int)vi, (int)vj);
  assert(id >= 0);
  return edge_nodes_[(size_t)id];
}

bool Mesh::hasDegenerateTet() const {
  for (const auto &tet : tets_)
    if (tet.volume <= 0.0) return true;
  return false;
}
