// C ABI over the host Mesh class (declarations and reference citations in include/cfsa_mesh.h).
#include "cfsa_mesh.h"
#include "cfsa_ns.h"
#include "Mesh.hpp"

#include <cstring>
#include <exception>
#include <string>

struct cfsa_mesh {
  Mesh mesh;
};

namespace {
thread_local std::string g_mesh_error;

int fail(int code, const std::string &msg) {
  g_mesh_error = msg;
  return code;
}

template <class F>
int guarded(F &&f) {
  try {
    return f();
  } catch (const std::exception &e) {
    return fail(CFSA_BAD_ARG, e.what());
  } catch (...) {
    return fail(CFSA_BAD_ARG, "unknown error");
  }
}
}  // namespace

extern "C" {

int cfsa_mesh_from_msh(const char *path, cfsa_mesh **out) {
  if (!path || !out) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    auto *m = new cfsa_mesh();
    try {
      m->mesh.generateFromMshFile(path);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return CFSA_OK;
  });
}

int cfsa_mesh_from_arrays(int64_t nv, const double *xyz, int64_t nt, const int32_t *tets,
                          cfsa_mesh **out) {
  if (!xyz || !tets || !out || nv <= 0 || nt <= 0) return fail(CFSA_BAD_ARG, "bad arrays");
  return guarded([&] {
    std::vector<Vec3> v((size_t)nv);
    for (int64_t i = 0; i < nv; ++i) v[i] = Vec3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    std::vector<std::array<int, 4>> t((size_t)nt);
    for (int64_t i = 0; i < nt; ++i)
      t[i] = {tets[4 * i], tets[4 * i + 1], tets[4 * i + 2], tets[4 * i + 3]};
    auto *m = new cfsa_mesh();
    try {
      m->mesh.generateFromArrays(v, t);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return CFSA_OK;
  });
}

int cfsa_mesh_structured_prism(double length, double width, double height, int nx, int ny, int nz,
                               cfsa_mesh **out) {
  if (!out) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    auto *m = new cfsa_mesh();
    try {
      m->mesh.generateStructuredRectangularPrism(length, width, height, nx, ny, nz);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return CFSA_OK;
  });
}

int cfsa_mesh_cylinder(double length, double radius, int rings, int layers, cfsa_mesh **out) {
  if (!out) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    auto *m = new cfsa_mesh();
    try {
      m->mesh.generateCylinder(length, radius, rings, layers);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return CFSA_OK;
  });
}

int cfsa_mesh_y_bifurcation(const double spec[7], cfsa_mesh **out) {
  if (!out || !spec) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    YBifurcation y;
    y.parent_radius = spec[0];
    y.parent_length = spec[1];
    y.daughter_radius = spec[2];
    y.daughter_length = spec[3];
    y.angle_deg = spec[4];
    y.blend = spec[5];
    y.cell = spec[6];
    auto *m = new cfsa_mesh();
    try {
      m->mesh.generateYBifurcation(y);
    } catch (...) {
      delete m;
      throw;
    }
    *out = m;
    return CFSA_OK;
  });
}

int cfsa_mesh_setup_boundary_conditions(cfsa_mesh *m, const double dir[3], double coverage) {
  if (!m || !dir) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    Mesh::setupBoundaryConditions(Vec3(dir[0], dir[1], dir[2]), coverage, m->mesh);
    return CFSA_OK;
  });
}

int cfsa_mesh_set_fluid_bc(cfsa_mesh *m, const int8_t *p1_bc, const int8_t *p2_bc) {
  if (!m) return fail(CFSA_BAD_ARG, "null mesh");
  if (p1_bc)
    for (size_t i = 0; i < m->mesh.nVertices(); ++i) {
      if (p1_bc[i] < 0 || p1_bc[i] > CFSA_BC_UNDEFINED) return fail(CFSA_BAD_ARG, "bad P1 tag");
      m->mesh.setFluidVertexBC(i, (FluidBCType)p1_bc[i]);
    }
  if (p2_bc)
    for (size_t k = 0; k < m->mesh.getNumberOfEdgeNodes(); ++k) {
      if (p2_bc[k] < 0 || p2_bc[k] > CFSA_BC_UNDEFINED) return fail(CFSA_BAD_ARG, "bad P2 tag");
      m->mesh.setFluidP2vertexBC(k, (FluidBCType)p2_bc[k]);
    }
  return CFSA_OK;
}

int cfsa_mesh_write_msh(const cfsa_mesh *m, const char *path) {
  if (!m || !path) return fail(CFSA_BAD_ARG, "null argument");
  return guarded([&] {
    m->mesh.writeMshFile(path);
    return CFSA_OK;
  });
}

int cfsa_mesh_sizes(const cfsa_mesh *m, int64_t sizes[5]) {
  if (!m || !sizes) return fail(CFSA_BAD_ARG, "null argument");
  const Mesh &M = m->mesh;
  int64_t nb = 0;
  for (size_t f = 0; f < M.nFaces(); ++f) nb += !M.isFaceInternal(f);
  sizes[0] = (int64_t)M.nVertices();
  sizes[1] = (int64_t)M.nTets();
  sizes[2] = (int64_t)M.getNumberOfEdgeNodes();
  sizes[3] = (int64_t)M.nFaces();
  sizes[4] = nb;
  return CFSA_OK;
}

int cfsa_mesh_get_vertices(const cfsa_mesh *m, double *xyz) {
  if (!m || !xyz) return fail(CFSA_BAD_ARG, "null argument");
  const auto &v = m->mesh.getVertPositions();
  for (size_t i = 0; i < v.size(); ++i)
    for (int c = 0; c < 3; ++c) xyz[3 * i + c] = v[i][c];
  return CFSA_OK;
}

int cfsa_mesh_get_tets(const cfsa_mesh *m, int32_t *tets) {
  if (!m || !tets) return fail(CFSA_BAD_ARG, "null argument");
  const auto &T = m->mesh.getTets();
  for (size_t t = 0; t < T.size(); ++t)
    for (int k = 0; k < 4; ++k) tets[4 * t + k] = T[t].vertids[k];
  return CFSA_OK;
}

int cfsa_mesh_get_tet_edges(const cfsa_mesh *m, int32_t *edges) {
  if (!m || !edges) return fail(CFSA_BAD_ARG, "null argument");
  const auto &E = m->mesh.getAllTetEdgeNodes();
  for (size_t t = 0; t < E.size(); ++t)
    for (int k = 0; k < 6; ++k) edges[6 * t + k] = E[t][k];
  return CFSA_OK;
}

int cfsa_mesh_get_edge_nodes(const cfsa_mesh *m, double *xyz) {
  if (!m || !xyz) return fail(CFSA_BAD_ARG, "null argument");
  const auto &v = m->mesh.getEdgeNodePositions();
  for (size_t i = 0; i < v.size(); ++i)
    for (int c = 0; c < 3; ++c) xyz[3 * i + c] = v[i][c];
  return CFSA_OK;
}

int cfsa_mesh_get_fluid_bc(const cfsa_mesh *m, int8_t *p1_bc, int8_t *p2_bc) {
  if (!m) return fail(CFSA_BAD_ARG, "null argument");
  if (p1_bc)
    for (size_t i = 0; i < m->mesh.nVertices(); ++i) p1_bc[i] = (int8_t)m->mesh.getFluidVertexBC(i);
  if (p2_bc)
    for (size_t k = 0; k < m->mesh.getNumberOfEdgeNodes(); ++k)
      p2_bc[k] = (int8_t)m->mesh.getP2FluidVertexBC(k);
  return CFSA_OK;
}

int cfsa_mesh_get_faces(const cfsa_mesh *m, int32_t *vertids, int32_t *tets, double *geom) {
  if (!m) return fail(CFSA_BAD_ARG, "null argument");
  const auto &F = m->mesh.getFaces();
  for (size_t f = 0; f < F.size(); ++f) {
    if (vertids)
      for (int k = 0; k < 3; ++k) vertids[3 * f + k] = F[f].vertids[k];
    if (tets) {
      tets[2 * f] = F[f].tet_a;
      tets[2 * f + 1] = F[f].tet_b;
    }
    if (geom) {
      double *g = geom + 7 * f;
      g[0] = F[f].normal.x();
      g[1] = F[f].normal.y();
      g[2] = F[f].normal.z();
      g[3] = F[f].area;
      g[4] = F[f].center.x();
      g[5] = F[f].center.y();
      g[6] = F[f].center.z();
    }
  }
  return CFSA_OK;
}

int cfsa_mesh_get_tet_geometry(const cfsa_mesh *m, double *volumes, double *grads) {
  if (!m) return fail(CFSA_BAD_ARG, "null argument");
  for (size_t t = 0; t < m->mesh.nTets(); ++t) {
    if (volumes) volumes[t] = m->mesh.tetAt(t).volume;
    if (grads) {
      const auto &g = m->mesh.getTetGradients(t);
      for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 3; ++c) grads[12 * t + 3 * a + c] = g[a][c];
    }
  }
  return CFSA_OK;
}

void cfsa_mesh_destroy(cfsa_mesh *m) { delete m; }

const char *cfsa_mesh_last_error(void) { return g_mesh_error.c_str(); }

}  // extern "C"
