// ============================================================================================
// ORACLE — TEST INFRASTRUCTURE ONLY. Not part of the product path.
//
// A plain FP64 CPU restatement of the reference's Taylor-Hood P2/P1 PISO Navier-Stokes path
// (sudo-shaka/Cell-Fluid-Structure-Analysis):
//   * mesh processing: src/Mesh/Mesh.cpp:448-677 (geometry, faces in std::map order, P1
//     gradients, P2 edge numbering with std::map) and the boundary tagging of
//     src/Mesh/Mesh.cpp:325-417 with include/Mesh/Mesh.hpp:198-215;
//   * assembly of M, K, Gx/Gy/Gz, L: src/FEM/NavierStokes.cpp:70-356 (triplets summed in
//     insertion order, as Eigen::SparseMatrix::setFromTriplets does);
//   * pisoStep / simpleStep and their phases: src/FEM/NavierStokes.cpp:374-771, 804-839,
//     968-1024; boundary forces: src/FEM/NavierStokes.cpp:841-965.
// The Krylov solvers restate the published algorithms (BiCGSTAB: van der Vorst 1992, right
// Jacobi preconditioning; CG: Hestenes-Stiefel with Jacobi preconditioning) with the stopping
// rule ||r|| <= tol*||b||, zero initial guess and an iteration cap; Eigen's sources were not
// consulted (Eigen is not installed here).
//
// PARITY UNPINNED: the reference cannot be compiled in this environment (Eigen, yaml-cpp and
// TetGen are absent) and it ships no tests, fixtures or golden vectors, so this restatement
// could not be checked against outputs of the reference itself. It is cross-checked against an
// independent numpy restatement and against analytic element identities in tests/.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library.
// Extensions relative to the reference (each documented in the C API below): per-node inlet
// profile, routing of the Krylov tolerances and iteration caps, CG for the pressure solve.
// ============================================================================================
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x = 0, y = 0, z = 0;
  V3() = default;
  V3(double a, double b, double c) : x(a), y(b), z(c) {}
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  double &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  V3 operator+(const V3 &o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(const V3 &o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator-() const { return {-x, -y, -z}; }
  V3 operator*(double s) const { return {x * s, y * s, z * s}; }
  V3 operator/(double s) const { return {x / s, y / s, z / s}; }
  double dot(const V3 &o) const { return (x * o.x + y * o.y) + z * o.z; }
  V3 cross(const V3 &o) const { return {y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x}; }
  double norm() const { return std::sqrt(dot(*this)); }
  V3 normalized() const {
    double n = norm();
    return n > 0 ? (*this) / n : *this;
  }
};
inline V3 operator*(double s, const V3 &a) { return a * s; }

enum BC { kWall = 0, kInlet = 1, kOutlet = 2, kInternal = 3, kUndefined = 4 };
enum Outlet { kDirichlet = 0, kNeumann = 1, kOutletUndefined = 2 };

constexpr int kLocalFaces[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
constexpr int kEdgeVerts[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};

struct OTet {
  double volume = 0;
  int v[4] = {0, 0, 0, 0};
  V3 centroid;
};
struct OFace {
  int tet_a = -1, tet_b = -1, fa = -1, fb = -1;
  double area = 0;
  int v[3] = {0, 0, 0};
  V3 normal, center;
};

struct Triplet {
  int r, c;
  double v;
};

struct CSR {
  int64_t n = 0;
  std::vector<int64_t> rowptr;
  std::vector<int> col;
  std::vector<double> val;
  int64_t nnz() const { return (int64_t)col.size(); }
};

// setFromTriplets semantics: entries (r,c) summed in triplet insertion order; row-major CSR
// with ascending columns.
CSR from_triplets(int64_t n, const std::vector<Triplet> &trips) {
  CSR A;
  A.n = n;
  std::vector<int64_t> cnt(n + 1, 0);
  for (const auto &t : trips) cnt[t.r + 1]++;
  for (int64_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  std::vector<int64_t> order(trips.size());
  {
    std::vector<int64_t> fill(cnt.begin(), cnt.end() - 1);
    for (size_t k = 0; k < trips.size(); ++k) order[fill[trips[k].r]++] = (int64_t)k;
  }
  A.rowptr.assign(n + 1, 0);
  std::vector<int> cols;
  std::vector<double> vals;
  cols.reserve(trips.size() / 2);
  vals.reserve(trips.size() / 2);
  std::vector<int64_t> seg;
  for (int64_t i = 0; i < n; ++i) {
    seg.assign(order.begin() + cnt[i], order.begin() + cnt[i + 1]);
    std::stable_sort(seg.begin(), seg.end(),
                     [&](int64_t a, int64_t b) { return trips[a].c < trips[b].c; });
    size_t k = 0;
    while (k < seg.size()) {
      const int c = trips[seg[k]].c;
      double s = trips[seg[k]].v;
      size_t e = k + 1;
      while (e < seg.size() && trips[seg[e]].c == c) {
        s += trips[seg[e]].v;
        ++e;
      }
      cols.push_back(c);
      vals.push_back(s);
      k = e;
    }
    A.rowptr[i + 1] = (int64_t)cols.size();
  }
  A.col.swap(cols);
  A.val.swap(vals);
  return A;
}

void spmv(const CSR &A, const double *x, double *y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.n; ++i) {
    double s = 0.0;
    for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) s += A.val[k] * x[A.col[k]];
    y[i] = s;
  }
}

// ---------------------------------------------------------------------------------------------
// Reductions. Krylov dot products are summed in one fixed tree, the one the CUDA solver uses, so
// that the two FP64 trajectories can be compared bit for bit (the reference's Eigen order depends
// on its SIMD build and cannot be reproduced here in any case). Tree: the products are laid out
// by "position"; positions are cut into blocks of 256 = 8 warps of 32; a warp sums its 32 values
// by a butterfly (v_l + v_{l^o} for o = 16, 8, 4, 2, 1); a block adds its 8 warp sums in order;
// 256 accumulators then take block b into accumulator b mod 256 in increasing b, and these 256
// accumulators are combined by the same warp butterflies and in-order warp sum.
// A position is either a row index ("natural" order) or a slot of the SELL-32 layout of the
// operator (rows sorted by decreasing length inside windows of 256 rows, stable), for the
// reductions that the device fuses into its sparse products.
struct RedOrder {
  std::vector<int> pos2row;  // row of each position, -1 for padding
  int64_t nblocks = 0;
};

RedOrder natural_order(int64_t n) {
  RedOrder o;
  o.nblocks = (n + 255) / 256;
  o.pos2row.resize(o.nblocks * 256);
  for (int64_t r = 0; r < (int64_t)o.pos2row.size(); ++r) o.pos2row[r] = r < n ? (int)r : -1;
  return o;
}

RedOrder sell_order(const CSR &A) {
  const int64_t n = A.n;
  const int64_t npad = (n + 31) / 32 * 32;
  RedOrder o;
  o.nblocks = (npad + 255) / 256;
  o.pos2row.assign(o.nblocks * 256, -1);
  std::vector<int> idx;
  for (int64_t w0 = 0; w0 < n; w0 += 256) {
    const int64_t w1 = std::min(n, w0 + 256);
    idx.resize(w1 - w0);
    std::iota(idx.begin(), idx.end(), (int)w0);
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
      return (A.rowptr[a + 1] - A.rowptr[a]) > (A.rowptr[b + 1] - A.rowptr[b]);
    });
    for (int64_t k = 0; k < w1 - w0; ++k) o.pos2row[w0 + k] = idx[k];
  }
  return o;
}

inline double warp_butterfly(double *x) {
  double y[32];
  for (int off = 16; off > 0; off >>= 1) {
    for (int l = 0; l < 32; ++l) y[l] = x[l] + x[l ^ off];
    for (int l = 0; l < 32; ++l) x[l] = y[l];
  }
  return x[0];
}

inline double block_sum(double *v /*256 values*/) {
  double s = 0.0;
  for (int w = 0; w < 8; ++w) s += warp_butterfly(v + 32 * w);
  return s;
}

// sum over positions of f(row) (0 for padding) in the device tree
template <class F>
double tree_sum(const RedOrder &o, F f) {
  const int64_t G = o.nblocks;
  std::vector<double> part(G);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < G; ++b) {
    double v[256];
    for (int k = 0; k < 256; ++k) {
      const int row = o.pos2row[b * 256 + k];
      v[k] = row >= 0 ? f(row) : 0.0;
    }
    part[b] = block_sum(v);
  }
  double acc[256];
  for (int t = 0; t < 256; ++t) {
    double a = 0.0;
    for (int64_t b = t; b < G; b += 256) a += part[b];
    acc[t] = a;
  }
  return block_sum(acc);
}

double odot(const RedOrder &o, const double *a, const double *b) {
  return tree_sum(o, [&](int i) { return a[i] * b[i]; });
}

struct SolveInfo {
  int iters = 0;
  double rel_res = 0;
  bool converged = false;
};

std::vector<double> inverse_diagonal(const CSR &A, std::vector<double> *diag = nullptr) {
  std::vector<double> inv(A.n, 1.0);
  if (diag) diag->assign(A.n, 0.0);
  for (int64_t i = 0; i < A.n; ++i)
    for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k)
      if (A.col[k] == i) {
        inv[i] = (A.val[k] != 0.0) ? 1.0 / A.val[k] : 1.0;
        if (diag) (*diag)[i] = A.val[k];
      }
  return inv;
}

// Right-Jacobi-preconditioned BiCGSTAB (van der Vorst 1992), zero initial guess, stop when
// ||r||^2 <= tol^2 ||b||^2 or after maxit iterations. The preconditioned operator is applied as
// the column-scaled matrix At = A diag(1/a_jj); x is kept in original variables
// (x += alpha D^-1 p + omega D^-1 s). A zero denominator (r0.v or, when unconverged, omega) or a
// NaN residual ends the solve unconverged. Near-breakdown (|rho| < eps^2 ||r0||^2) restarts from
// the true residual with r0 = r, p = r. `init` orders the ||b||^2 reduction, `sell` the products
// fused into the sparse products, `nat` the rest.
// `scaled`: convergence norm ||D^-1/2 r|| (sum of (r_i r_i) / a_ii) instead of ||r||.
SolveInfo bicgstab(const CSR &A, const std::vector<double> &b, std::vector<double> &x, double tol,
                   int maxit, const RedOrder &init, const RedOrder &sell, const RedOrder &nat,
                   bool scaled) {
  const int64_t n = A.n;
  SolveInfo info;
  std::vector<double> diag;
  const std::vector<double> invdiag = inverse_diagonal(A, &diag);
  CSR At = A;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) At.val[k] = A.val[k] * invdiag[A.col[k]];
  x.assign(n, 0.0);
  auto crit_of = [&](const RedOrder &o, const std::vector<double> &v) {
    return scaled ? tree_sum(o, [&](int i) { return (v[i] * v[i]) * invdiag[i]; })
                  : odot(o, v.data(), v.data());
  };
  const double b2 = odot(init, b.data(), b.data());
  const double bnorm2 = crit_of(init, b);
  const double tol2 = tol * tol * bnorm2;
  if (std::isnan(bnorm2) || std::isnan(b2)) return info;
  if (bnorm2 == 0.0 || bnorm2 <= tol2) {
    info.converged = true;
    return info;
  }
  std::vector<double> r(b), r0(b), p(n, 0.0), v(n, 0.0), s(n), t(n), dx(n);
  double r0norm2 = b2, rho = b2, alpha = 1.0, w = 1.0, beta = 0.0;
  const double eps = std::numeric_limits<double>::epsilon();
  bool restart = false;
  double rn2 = bnorm2;
  int i = 0;
  while (true) {
    if (restart) {
      for (int64_t k = 0; k < n; ++k) dx[k] = diag[k] * x[k];
      spmv(At, dx.data(), t.data());
      for (int64_t k = 0; k < n; ++k) {
        r[k] = b[k] - t[k];
        r0[k] = r[k];
        p[k] = r[k];
      }
      rho = r0norm2 = odot(sell, r.data(), r.data());
      restart = false;
    } else {
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; ++k) p[k] = r[k] + beta * (p[k] - w * v[k]);
    }
    spmv(At, p.data(), v.data());
    const double r0v = odot(sell, r0.data(), v.data());
    if (r0v == 0.0) break;
    alpha = rho / r0v;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) s[k] = r[k] - alpha * v[k];
    spmv(At, s.data(), t.data());
    const double tt = odot(sell, t.data(), t.data());
    const double ts = odot(sell, t.data(), s.data());
    w = (tt > 0.0) ? ts / tt : 0.0;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < n; ++k) {
      const double y = invdiag[k] * p[k];
      const double z = invdiag[k] * s[k];
      x[k] += alpha * y + w * z;
      r[k] = s[k] - w * t[k];
    }
    rn2 = crit_of(nat, r);
    const double rho_new = odot(nat, r0.data(), r.data());
    ++i;
    if (std::isnan(rn2) || std::isnan(rho_new)) break;
    if (rn2 <= tol2) break;
    if (i >= maxit) break;
    if (w == 0.0) break;
    if (std::fabs(rho_new) < eps * eps * r0norm2) {
      restart = true;
    } else {
      beta = (rho_new / rho) * (alpha / w);
      rho = rho_new;
    }
  }
  info.iters = i;
  info.rel_res = std::sqrt(rn2 / bnorm2);
  info.converged = rn2 <= tol2;
  return info;
}

// Jacobi-preconditioned CG (Hestenes-Stiefel), zero initial guess, same stopping rule; p.q is
// fused into the sparse product (`sell` order), the other reductions use `nat`.
// `scaled`: convergence norm r.z = ||D^-1/2 r||^2 instead of r.r.
SolveInfo cg(const CSR &A, const std::vector<double> &b, std::vector<double> &x, double tol,
             int maxit, const RedOrder &sell, const RedOrder &nat, bool scaled) {
  const int64_t n = A.n;
  SolveInfo info;
  const std::vector<double> invdiag = inverse_diagonal(A);
  x.assign(n, 0.0);
  std::vector<double> r(b), z(n), p(n), q(n);
  for (int64_t k = 0; k < n; ++k) z[k] = invdiag[k] * r[k];
  const double b2 = odot(nat, b.data(), b.data());
  double absnew = odot(nat, b.data(), z.data());
  const double bnorm2 = scaled ? absnew : b2;
  const double thr = tol * tol * bnorm2;
  if (std::isnan(bnorm2)) return info;
  double rn2 = bnorm2;
  int i = 0;
  if (!(bnorm2 == 0.0 || bnorm2 <= thr)) {
    p = z;
    while (true) {
      spmv(A, p.data(), q.data());
      const double pq = odot(sell, p.data(), q.data());
      if (pq == 0.0) break;
      const double alpha = absnew / pq;
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; ++k) {
        x[k] += alpha * p[k];
        r[k] = r[k] - alpha * q[k];
        z[k] = invdiag[k] * r[k];
      }
      const double rr = odot(nat, r.data(), r.data());
      const double rz = odot(nat, r.data(), z.data());
      rn2 = scaled ? rz : rr;
      ++i;
      if (std::isnan(rr) || std::isnan(rz)) break;
      if (rn2 <= thr) break;
      if (i >= maxit) break;
      const double beta = rz / absnew;
      absnew = rz;
#pragma omp parallel for schedule(static)
      for (int64_t k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
    }
  }
  info.iters = i;
  info.rel_res = std::sqrt(rn2 / bnorm2);
  info.converged = rn2 <= thr;
  return info;
}

// Jacobi-preconditioned CG with one reduction per iteration (Chronopoulos & Gear, J. Comput.
// Appl. Math. 25 (1989)): the same iterates as cg() in exact arithmetic. s = A p is carried by a
// recurrence, so one fused product-and-reduction pass per iteration suffices:
//   p = u + beta p;  s = w + beta s;  x += alpha p;  r -= alpha s;  u = M r;  w = A u;
//   gamma = r.u, delta = w.u, rr = r.r;
//   beta' = gamma'/gamma, alpha' = gamma' / (delta' - beta' gamma' / alpha).
// Start: u = M b, w = A u, gamma = b.u (natural order), delta = w.u (product order), alpha =
// gamma/delta, beta = 0. The three dots of an iteration are summed in `sell` order (they are fused
// into the product); the stopping rule is cg()'s.
SolveInfo cg1(const CSR &A, const std::vector<double> &b, std::vector<double> &x, double tol,
              int maxit, const RedOrder &sell, const RedOrder &nat, bool scaled) {
  const int64_t n = A.n;
  SolveInfo info;
  const std::vector<double> invdiag = inverse_diagonal(A);
  x.assign(n, 0.0);
  std::vector<double> r(b), u(n), w(n), p(n, 0.0), s(n, 0.0);
  for (int64_t k = 0; k < n; ++k) u[k] = invdiag[k] * r[k];
  const double b2 = odot(nat, b.data(), b.data());
  double gamma = odot(nat, b.data(), u.data());
  const double bnorm2 = scaled ? gamma : b2;
  const double thr = tol * tol * bnorm2;
  if (std::isnan(bnorm2)) return info;
  double rn2 = bnorm2;
  int it = 0;
  if (!(bnorm2 == 0.0 || bnorm2 <= thr)) {
    spmv(A, u.data(), w.data());
    const double delta0 = odot(sell, w.data(), u.data());
    if (delta0 == 0.0) {
      info.rel_res = 1.0;
      return info;
    }
    double alpha = gamma / delta0, beta = 0.0;
    while (true) {
      for (int64_t k = 0; k < n; ++k) {
        p[k] = u[k] + beta * p[k];
        s[k] = w[k] + beta * s[k];
        x[k] += alpha * p[k];
        r[k] = r[k] - alpha * s[k];
        u[k] = invdiag[k] * r[k];
      }
      spmv(A, u.data(), w.data());
      const double g_new = odot(sell, r.data(), u.data());
      const double delta = odot(sell, w.data(), u.data());
      const double rr = odot(sell, r.data(), r.data());
      rn2 = scaled ? g_new : rr;
      ++it;
      if (std::isnan(g_new) || std::isnan(delta) || std::isnan(rr)) break;
      if (rn2 <= thr) break;
      if (it >= maxit) break;
      const double beta_new = g_new / gamma;
      const double den = delta - beta_new * g_new / alpha;
      if (den == 0.0) break;
      alpha = g_new / den;
      beta = beta_new;
      gamma = g_new;
    }
  }
  info.iters = it;
  info.rel_res = std::sqrt(rn2 / bnorm2);
  info.converged = rn2 <= thr;
  return info;
}

// ---------------------------------------------------------------------------------------------
// Two-level preconditioner of the pressure CG (pressure_solver 3). Not in the reference, which
// solves the Poisson problem with Jacobi-preconditioned BiCGSTAB; this is a faster solver of the
// same system (the CUDA solver's CFSA_KRYLOV_CG2L), restated here so that the device iterates can
// be checked bit for bit.
//   M r = D^-1 r + P Z P^T r,   Z = (P^T A P)^-1,
// P the indicator matrix of geometric aggregates (boxes of a uniform grid over the vertices) on the
// rows without a penalty (Dirichlet outlet rows, or the Neumann reference row, belong to no
// aggregate). Additive two-level Schwarz with a piecewise-constant coarse space: the coarse solve
// removes the smooth error components that Jacobi-CG converges slowly on (684 -> 134 CG iterations
// on the 1M-tet cylinder with ~256 aggregates).
//
// Aggregation: box edge h_k = e * c^k (e = largest extent of the vertex bounding box,
// c = 2^-1/4, k the smallest exponent in [0, 64] for which the number of occupied boxes reaches
// `target`, found by bisection); boxes are numbered in order of their first vertex.
// Z from the Cholesky factor G of A_c (row-wise Cholesky-Banachiewicz, then the lower-triangular
// inverse by columns, then Z = G^-T G^-1 summed over ascending rows); A_c entries summed over the
// CSR in row-major order. A non-SPD A_c (a pivot <= 0) disables the coarse part (nc = 0).
// Aggregate sums are exact fixed-point sums: x -> floor(x 2^S) as a 128-bit integer (x 2^S
// clamped to +-2^100, NaN -> 0), S = 80 - floor(log2(b.b) / 2) for the solve's right-hand side b,
// summed exactly and converted back as (hi 2^64 + lo) 2^-S with hi the upper 64 bits (signed) and
// lo the lower 64 bits (unsigned). Coarse values c[m] = butterfly over lanes l of
// (sum over k = l, l+32, ... of Z[m][k] t[k]).
struct CoarseSpace {
  int nc = 0;
  std::vector<int> agg;                // [n], nc for rows without aggregate
  std::vector<double> Z;               // [nc*nc], symmetric
};

constexpr double kBoxShrink = 0.8408964152537145;  // 2^-1/4

int count_boxes(const std::vector<V3> &xyz, const std::vector<char> &pen, int64_t n, double h,
                const V3 &lo, std::vector<int64_t> *keys_out = nullptr) {
  std::vector<int64_t> keys;
  keys.reserve(n);
  for (int64_t i = 0; i < n; ++i) {
    if (pen[i]) continue;
    const int64_t ix = (int64_t)std::floor((xyz[i].x - lo.x) / h);
    const int64_t iy = (int64_t)std::floor((xyz[i].y - lo.y) / h);
    const int64_t iz = (int64_t)std::floor((xyz[i].z - lo.z) / h);
    keys.push_back((ix * 2097152 + iy) * 2097152 + iz);
  }
  if (keys_out) *keys_out = keys;
  std::sort(keys.begin(), keys.end());
  return (int)(std::unique(keys.begin(), keys.end()) - keys.begin());
}

CoarseSpace build_coarse(const CSR &A, const std::vector<V3> &xyz, const std::vector<char> &pen,
                         int target) {
  CoarseSpace cs;
  const int64_t n = A.n;
  cs.agg.assign(n, 0);
  V3 lo{0, 0, 0}, hi{0, 0, 0};
  bool any = false;
  for (int64_t i = 0; i < n; ++i) {
    if (pen[i]) continue;
    if (!any) {
      lo = hi = xyz[i];
      any = true;
    }
    lo.x = std::min(lo.x, xyz[i].x), lo.y = std::min(lo.y, xyz[i].y), lo.z = std::min(lo.z, xyz[i].z);
    hi.x = std::max(hi.x, xyz[i].x), hi.y = std::max(hi.y, xyz[i].y), hi.z = std::max(hi.z, xyz[i].z);
  }
  const double e = std::max(hi.x - lo.x, std::max(hi.y - lo.y, hi.z - lo.z));
  if (!any || !(e > 0.0) || target < 1) {
    cs.nc = 0;  // no coarse space: every row maps to the zero coarse value
  } else {
    auto h_of = [&](int k) {
      double h = e;
      for (int q = 0; q < k; ++q) h = h * kBoxShrink;
      return h;
    };
    int klo = 0, khi = 64;  // count(h_klo) < target unless klo == 0; count(h_khi) >= target assumed
    while (klo < khi) {
      const int km = (klo + khi) / 2;
      if (count_boxes(xyz, pen, n, h_of(km), lo) >= target)
        khi = km;
      else
        klo = km + 1;
    }
    std::vector<int64_t> keys;
    count_boxes(xyz, pen, n, h_of(klo), lo, &keys);
    // number boxes by first vertex
    std::vector<std::pair<int64_t, int>> kv(keys.size());
    for (size_t q = 0; q < keys.size(); ++q) kv[q] = {keys[q], (int)q};
    std::stable_sort(kv.begin(), kv.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    std::vector<int> first_of(keys.size());  // box rank by first vertex
    std::vector<std::pair<int, int>> firsts;  // (first q, group start)
    for (size_t q = 0; q < kv.size();) {
      size_t r = q;
      while (r < kv.size() && kv[r].first == kv[q].first) ++r;
      firsts.push_back({kv[q].second, (int)q});
      q = r;
    }
    std::sort(firsts.begin(), firsts.end());
    std::vector<int> id_of_sorted(kv.size());
    for (size_t g = 0; g < firsts.size(); ++g) {
      size_t q = firsts[g].second;
      const int64_t key = kv[q].first;
      while (q < kv.size() && kv[q].first == key) id_of_sorted[q++] = (int)g;
    }
    std::vector<int> id_of_q(keys.size());
    for (size_t q = 0; q < kv.size(); ++q) id_of_q[kv[q].second] = id_of_sorted[q];
    cs.nc = (int)firsts.size();
    size_t q = 0;
    for (int64_t i = 0; i < n; ++i) cs.agg[i] = pen[i] ? cs.nc : id_of_q[q++];
  }
  const int nc = cs.nc;
  if (nc > 0) {
    std::vector<double> Ac((size_t)nc * nc, 0.0), G((size_t)nc * nc, 0.0), Gi((size_t)nc * nc, 0.0);
    for (int64_t i = 0; i < n; ++i) {
      if (cs.agg[i] >= nc) continue;
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
        const int j = A.col[k];
        if (cs.agg[j] >= nc) continue;
        double &a = Ac[(size_t)cs.agg[i] * nc + cs.agg[j]];
        a = a + A.val[k];
      }
    }
    bool spd = true;
    for (int i = 0; i < nc && spd; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = Ac[(size_t)i * nc + j];
        for (int k = 0; k < j; ++k) s = s - G[(size_t)i * nc + k] * G[(size_t)j * nc + k];
        if (i == j) {
          if (!(s > 0.0)) {
            spd = false;
            break;
          }
          G[(size_t)i * nc + i] = std::sqrt(s);
        } else {
          G[(size_t)i * nc + j] = s / G[(size_t)j * nc + j];
        }
      }
    if (!spd) {
      cs.nc = 0;
      for (auto &a : cs.agg) a = 0;
    } else {
      for (int j = 0; j < nc; ++j) {
        Gi[(size_t)j * nc + j] = 1.0 / G[(size_t)j * nc + j];
        for (int i = j + 1; i < nc; ++i) {
          double s = 0.0;
          for (int k = j; k < i; ++k) s = s - G[(size_t)i * nc + k] * Gi[(size_t)k * nc + j];
          Gi[(size_t)i * nc + j] = s / G[(size_t)i * nc + i];
        }
      }
      cs.Z.assign((size_t)nc * nc, 0.0);
      for (int m = 0; m < nc; ++m)
        for (int k = 0; k < nc; ++k) {
          double s = 0.0;
          for (int q = std::max(m, k); q < nc; ++q) s = s + Gi[(size_t)q * nc + m] * Gi[(size_t)q * nc + k];
          cs.Z[(size_t)m * nc + k] = s;
        }
    }
  }
  return cs;
}

// fixed-point scale exponent of a solve with right-hand side norm^2 b2
int fixed_scale(double b2) {
  if (!(b2 > 0.0) || !(b2 <= std::numeric_limits<double>::max())) return 80;
  const int e2 = std::ilogb(b2);
  return 80 - ((e2 >= 0) ? e2 / 2 : -((1 - e2) / 2));
}

__int128 fixed128(double x, double scale) {
  double y = x * scale;
  if (!(y == y)) y = 0.0;
  y = std::fmin(std::fmax(y, -0x1p100), 0x1p100);
  const double t = std::floor(y);
  if (std::fabs(t) < 0x1p63) return (__int128)(long long)t;
  const double hd = std::floor(t * 0x1p-64);
  const unsigned long long hi = (unsigned long long)(long long)hd;
  const unsigned long long lo = (unsigned long long)(t - hd * 0x1p64);
  return (__int128)(((unsigned __int128)hi << 64) | (unsigned __int128)lo);
}

double unfixed128(__int128 v, double iscale) {
  const long long hi = (long long)(v >> 64);
  const unsigned long long lo = (unsigned long long)v;
  return ((double)hi * 0x1p64 + (double)lo) * iscale;
}

// aggregate sums of v (size nc)
std::vector<double> aggregate_sums(const CoarseSpace &cs, const std::vector<double> &v, int S) {
  const double scale = std::scalbn(1.0, S), iscale = std::scalbn(1.0, -S);
  std::vector<__int128> acc(cs.nc, 0);
  for (size_t i = 0; i < v.size(); ++i)
    if (cs.agg[i] < cs.nc) acc[cs.agg[i]] += fixed128(v[i], scale);
  std::vector<double> T(cs.nc);
  for (int m = 0; m < cs.nc; ++m) T[m] = unfixed128(acc[m], iscale);
  return T;
}

// c = Z t (size nc + 1, c[nc] = 0 for rows without aggregate)
std::vector<double> coarse_values(const CoarseSpace &cs, const std::vector<double> &t) {
  const int nc = cs.nc;
  std::vector<double> c(nc + 1, 0.0);
  for (int m = 0; m < nc; ++m) {
    double lanes[32];
    for (int l = 0; l < 32; ++l) {
      double s = 0.0;
      for (int k = l; k < nc; k += 32) s += cs.Z[(size_t)m * nc + k] * t[k];
      lanes[l] = s;
    }
    c[m] = warp_butterfly(lanes);
  }
  return c;
}

// Single-reduction CG (the recurrences of cg1) preconditioned by M r = D^-1 r + P Z P^T r.
// t = P^T r of the new residual comes from the previous iteration's aggregate sums of r and w and
// the aggregate-level recurrence T(s) <- T(w) + beta T(s), t = T(r) - alpha T(s), so the device
// needs one grid barrier per iteration.
// Start: u = M b, w = A u, gamma = b.u and delta = w.u in product order. The stopping rule is
// cg1's: ||r||^2 or, scaled, sum r_i (r_i / a_ii) (the Jacobi-scaled norm, not r.u).
SolveInfo cg2l(const CSR &A, const std::vector<double> &b, std::vector<double> &x, double tol,
               int maxit, const RedOrder &sell, const RedOrder &nat, bool scaled,
               const CoarseSpace &cs) {
  const int64_t n = A.n;
  SolveInfo info;
  const std::vector<double> invdiag = inverse_diagonal(A);
  x.assign(n, 0.0);
  std::vector<double> r(b), u(n), w(n), p(n, 0.0), s(n, 0.0);
  const double b2 = odot(nat, b.data(), b.data());
  const double bz = tree_sum(nat, [&](int i) { return b[i] * (invdiag[i] * b[i]); });
  const double bnorm2 = scaled ? bz : b2;
  const double thr = tol * tol * bnorm2;
  if (std::isnan(bnorm2) || std::isnan(b2)) return info;
  double rn2 = bnorm2;
  int it = 0;
  if (!(bnorm2 == 0.0 || bnorm2 <= thr)) {
    const int sc = fixed_scale(b2);
    std::vector<double> R = aggregate_sums(cs, r, sc), S(cs.nc, 0.0);
    std::vector<double> c = coarse_values(cs, R);
    for (int64_t k = 0; k < n; ++k) u[k] = invdiag[k] * r[k] + c[cs.agg[k]];
    spmv(A, u.data(), w.data());
    const double delta0 = odot(sell, w.data(), u.data());
    double gamma = odot(sell, r.data(), u.data());
    std::vector<double> W = aggregate_sums(cs, w, sc);
    if (delta0 == 0.0 || std::isnan(delta0) || std::isnan(gamma)) {
      info.rel_res = 1.0;
      return info;
    }
    double alpha = gamma / delta0, beta = 0.0;
    std::vector<double> t(cs.nc);
    while (true) {
      for (int m = 0; m < cs.nc; ++m) {
        const double sm = W[m] + beta * S[m];  // T(s) of the new s, by recurrence
        S[m] = sm;
        t[m] = R[m] - alpha * sm;
      }
      c = coarse_values(cs, t);
      for (int64_t k = 0; k < n; ++k) {
        p[k] = u[k] + beta * p[k];
        s[k] = w[k] + beta * s[k];
        x[k] += alpha * p[k];
        r[k] = r[k] - alpha * s[k];
        u[k] = invdiag[k] * r[k] + c[cs.agg[k]];
      }
      spmv(A, u.data(), w.data());
      const double g_new = odot(sell, r.data(), u.data());
      const double delta = odot(sell, w.data(), u.data());
      const double rr = odot(sell, r.data(), r.data());
      const double rz = tree_sum(sell, [&](int i) { return r[i] * (invdiag[i] * r[i]); });
      R = aggregate_sums(cs, r, sc);
      W = aggregate_sums(cs, w, sc);
      rn2 = scaled ? rz : rr;
      ++it;
      if (std::isnan(g_new) || std::isnan(delta) || std::isnan(rr) || std::isnan(rz)) break;
      if (rn2 <= thr) break;
      if (it >= maxit) break;
      const double beta_new = g_new / gamma;
      const double den = delta - beta_new * g_new / alpha;
      if (den == 0.0) break;
      alpha = g_new / den;
      beta = beta_new;
      gamma = g_new;
    }
  }
  info.iters = it;
  info.rel_res = std::sqrt(rn2 / bnorm2);
  info.converged = rn2 <= thr;
  return info;
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Oracle {
  // ---- mesh (src/Mesh/Mesh.cpp restatement) ----
  std::vector<V3> vertices, edge_nodes;
  std::vector<OTet> tets;
  std::vector<OFace> faces;
  std::vector<std::array<V3, 4>> grads;
  std::map<std::pair<int, int>, int> edge_map;
  std::vector<std::array<int, 6>> tet_edges;
  std::vector<int> p1bc, p2bc;
  size_t nv = 0, ne = 0, nt = 0, N2 = 0;

  // ---- solver (src/FEM/NavierStokes.cpp restatement) ----
  double density = 1000, viscosity = 0.001;
  double dt = 1e-4, time = 0.0;
  double tol_mom = 1e-6, tol_p = 1e-8;  // values hard-coded at NavierStokes.cpp:500,635
  int maxit_mom = 1000, maxit_p = 1000;
  int n_corr = 1;
  double relax_u = 1.0, relax_p = 1.0;
  int outlet_type = kDirichlet;
  double outlet_pressure = 0.0;
  int reference_node = -1;
  int pressure_solver = 0;  // 0 = BiCGSTAB (reference), 1 = CG, 2 = CG with one reduction,
                            // 3 = the latter with the two-level preconditioner
  int conv_norm = 0;        // 0 = ||r|| (reference), 1 = ||D^-1/2 r||
  int momentum_solver = 0;  // 0 = BiCGSTAB (reference), 1 = Jacobi CG on the same SPD system
  std::vector<V3> inlet;    // per P2-node inlet velocity (the reference: one mean vector)
  std::vector<V3> u, ustar;
  std::vector<double> p, pcorr, inv_lumped;
  CSR M, K, Gx, Gy, Gz, L;
  RedOrder order_p2, order_p1, order_n2, order_nv;  // reduction orders (see tree_sum)
  bool initialized = false;

  // stats of the last step
  int it_mom[3] = {0, 0, 0}, it_p = 0;
  double res_mom[3] = {0, 0, 0}, res_p = 0;
  double t_conv = 0, t_mom = 0, t_press = 0, t_corr = 0, t_assembly = 0;

  // ---------------------------------------------------------------- mesh processing
  void build_mesh(const double *xyz, const int *tv) {
    for (size_t i = 0; i < nv; ++i) vertices[i] = V3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    for (size_t t = 0; t < nt; ++t)
      for (int k = 0; k < 4; ++k) tets[t].v[k] = tv[4 * t + k];
    // buildConnectivity (Mesh.cpp:494-530)
    std::map<std::array<int, 3>, OFace> face_map;
    for (int t = 0; t < (int)nt; ++t) {
      for (int f = 0; f < 4; ++f) {
        std::array<int, 3> fv = {tets[t].v[kLocalFaces[f][0]], tets[t].v[kLocalFaces[f][1]],
                                 tets[t].v[kLocalFaces[f][2]]};
        std::array<int, 3> sv = fv;
        std::sort(sv.begin(), sv.end());
        auto it = face_map.find(sv);
        if (it == face_map.end()) {
          OFace face;
          face.v[0] = fv[0];
          face.v[1] = fv[1];
          face.v[2] = fv[2];
          face.tet_a = t;
          face.fa = f;
          face_map[sv] = face;
        } else {
          it->second.tet_b = t;
          it->second.fb = f;
        }
      }
    }
    faces.clear();
    for (auto &kv : face_map) faces.push_back(kv.second);
    // computeGeometry (Mesh.cpp:448-471)
    for (auto &tet : tets) {
      const V3 &a = vertices[tet.v[0]], &b = vertices[tet.v[1]], &c = vertices[tet.v[2]],
               &d = vertices[tet.v[3]];
      tet.centroid = (((a + b) + c) + d) / 4.0;
      tet.volume = std::fabs((b - a).cross(c - a).dot(d - a) / 6.0);
    }
    for (auto &face : faces) {
      const V3 &a = vertices[face.v[0]], &b = vertices[face.v[1]], &c = vertices[face.v[2]];
      const V3 ab = b - a, ac = c - a;
      face.normal = ac.cross(ab).normalized();
      face.area = 0.5 * ab.cross(ac).norm();
      face.center = ((a + b) + c) / 3.0;
    }
    // ensureConsistentFaceNormals (Mesh.cpp:615-639)
    for (auto &face : faces) {
      if (face.tet_a >= 0 && face.tet_b >= 0) {
        const V3 &ca = tets[face.tet_a].centroid, &cb = tets[face.tet_b].centroid;
        const V3 desired = (cb - ca).normalized();
        if (face.normal.dot(desired) <= 1e-12) {
          face.normal = -face.normal;
          std::swap(face.v[1], face.v[2]);
        } else {
          const V3 out = (face.center - ca).normalized();
          if (face.normal.dot(out) <= 1e-12) {
            face.normal = -face.normal;
            std::swap(face.v[1], face.v[2]);
          }
        }
      }
    }
    // computeShapeFunctionGradients (Mesh.cpp:590-614)
    grads.resize(nt);
    for (size_t t = 0; t < nt; ++t) {
      const V3 &p0 = vertices[tets[t].v[0]], &p1 = vertices[tets[t].v[1]],
               &p2 = vertices[tets[t].v[2]], &p3 = vertices[tets[t].v[3]];
      const V3 e1 = p1 - p0, e2 = p2 - p0, e3 = p3 - p0;
      const double inv6v = 1.0 / e1.dot(e2.cross(e3));
      grads[t][0] = inv6v * (p3 - p1).cross(p2 - p1);
      grads[t][1] = inv6v * (p2 - p0).cross(p3 - p0);
      grads[t][2] = inv6v * (p3 - p0).cross(p1 - p0);
      grads[t][3] = inv6v * (p1 - p0).cross(p2 - p0);
    }
    // buildP2EdgeNodes (Mesh.cpp:641-677)
    edge_map.clear();
    tet_edges.assign(nt, {});
    edge_nodes.clear();
    int id = 0;
    for (size_t t = 0; t < nt; ++t) {
      for (int e = 0; e < 6; ++e) {
        int a = tets[t].v[kEdgeVerts[e][0]], b = tets[t].v[kEdgeVerts[e][1]];
        if (a > b) std::swap(a, b);
        auto key = std::make_pair(a, b);
        auto it = edge_map.find(key);
        if (it == edge_map.end()) {
          edge_nodes.push_back(0.5 * (vertices[a] + vertices[b]));
          edge_map[key] = id;
          tet_edges[t][e] = id++;
        } else {
          tet_edges[t][e] = it->second;
        }
      }
    }
    ne = edge_nodes.size();
    N2 = nv + ne;
    p1bc.assign(nv, kUndefined);
    p2bc.assign(ne, kUndefined);
  }

  // Mesh::setupBoundaryConditions (Mesh.cpp:325-417) + setP2BoundariesFromP1Boundaries
  // (Mesh.hpp:198-215)
  void setup_bc(const double dir[3], double coverage) {
    V3 mn = vertices[0], mx = vertices[0];
    for (const auto &v : vertices)
      for (int k = 0; k < 3; ++k) {
        mn[k] = std::min(mn[k], v[k]);
        mx[k] = std::max(mx[k], v[k]);
      }
    const V3 size = mx - mn;
    int ax = 0;
    if (size.y > size.x && size.y > size.z)
      ax = 1;
    else if (size.z > size.x && size.z > size.y)
      ax = 2;
    const double tol = size[ax] * 0.01 * coverage;
    const double inlet_pos = dir[ax] > 0 ? mn[ax] : mx[ax];
    const double outlet_pos = dir[ax] > 0 ? mx[ax] : mn[ax];
    p1bc.assign(nv, kInternal);
    for (const auto &f : faces) {
      if (f.tet_b != -1) continue;
      for (int k = 0; k < 3; ++k) p1bc[f.v[k]] = kWall;
      const double di = std::abs(f.center[ax] - inlet_pos);
      const double dout = std::abs(f.center[ax] - outlet_pos);
      if (di < tol) {
        for (int k = 0; k < 3; ++k) p1bc[f.v[k]] = kInlet;
      } else if (dout < tol) {
        for (int k = 0; k < 3; ++k) p1bc[f.v[k]] = kOutlet;
      }
    }
    set_p2_bc();
  }
  void set_p2_bc() {
    for (const auto &kv : edge_map) {
      const int a = p1bc[kv.first.first], b = p1bc[kv.first.second];
      p2bc[kv.second] = (a == b && a != kInternal) ? a : kInternal;
    }
  }
  int bc_of(size_t i) const { return i < nv ? p1bc[i] : p2bc[i - nv]; }

  // ---------------------------------------------------------------- assembly
  // buildGradientMatrices (NavierStokes.cpp:70-133)
  void build_gradient() {
    std::vector<Triplet> tx, ty, tz;
    tx.reserve(nt * 16);
    ty.reserve(nt * 16);
    tz.reserve(nt * 16);
    for (size_t t = 0; t < nt; ++t) {
      const double vol = tets[t].volume;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          const double c = vol / 4.0;
          const V3 &g = grads[t][j];
          tx.push_back({tets[t].v[i], tets[t].v[j], c * g.x});
          ty.push_back({tets[t].v[i], tets[t].v[j], c * g.y});
          tz.push_back({tets[t].v[i], tets[t].v[j], c * g.z});
        }
    }
    Gx = from_triplets(nv, tx);
    Gy = from_triplets(nv, ty);
    Gz = from_triplets(nv, tz);
  }
  // buildStiffnessMatrix (NavierStokes.cpp:135-225); note mu = 1/viscosity
  void build_stiffness() {
    std::vector<Triplet> tr;
    tr.reserve(nt * 100);
    const double mu = 1.0 / viscosity;
    for (size_t t = 0; t < nt; ++t) {
      const double vol = tets[t].volume;
      const auto &g = grads[t];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          tr.push_back({tets[t].v[i], tets[t].v[j], mu * vol * g[i].dot(g[j])});
      for (int e = 0; e < 6; ++e) {
        const int ei = (int)nv + tet_edges[t][e];
        const V3 ge = g[kEdgeVerts[e][0]] + g[kEdgeVerts[e][1]];
        for (int j = 0; j < 4; ++j) {
          const double kev = mu * vol * ge.dot(g[j]);
          tr.push_back({ei, tets[t].v[j], kev});
          tr.push_back({tets[t].v[j], ei, kev});
        }
        for (int f = 0; f < 6; ++f) {
          const int ej = (int)nv + tet_edges[t][f];
          const V3 gf = g[kEdgeVerts[f][0]] + g[kEdgeVerts[f][1]];
          tr.push_back({ei, ej, mu * vol * ge.dot(gf)});
        }
      }
    }
    K = from_triplets(N2, tr);
  }
  // buildMassMatrix (NavierStokes.cpp:227-310)
  void build_mass() {
    std::vector<Triplet> tr;
    tr.reserve(nt * 100);
    for (size_t t = 0; t < nt; ++t) {
      const double mass = density * tets[t].volume;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          tr.push_back({tets[t].v[i], tets[t].v[j], (i == j) ? mass / 10.0 : mass / 20.0});
      for (int e = 0; e < 6; ++e) {
        const int ei = (int)nv + tet_edges[t][e];
        for (int i = 0; i < 4; ++i) {
          tr.push_back({ei, tets[t].v[i], mass / 30.0});
          tr.push_back({tets[t].v[i], ei, mass / 30.0});
        }
        for (int f = 0; f < 6; ++f) {
          const int ej = (int)nv + tet_edges[t][f];
          tr.push_back({ei, ej, (e == f) ? mass / 15.0 : mass / 60.0});
        }
      }
    }
    M = from_triplets(N2, tr);
    std::vector<double> ones(N2, 1.0), rs(N2);
    spmv(M, ones.data(), rs.data());
    inv_lumped.assign(N2, 0.0);
    for (size_t i = 0; i < N2; ++i) inv_lumped[i] = (std::abs(rs[i]) > 1e-14) ? 1.0 / rs[i] : 1.0;
  }
  // buildPoissonMatrix (NavierStokes.cpp:316-356)
  void build_poisson() {
    std::vector<Triplet> tr;
    tr.reserve(nt * 16);
    for (size_t t = 0; t < nt; ++t) {
      const double vol = tets[t].volume;
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j)
          tr.push_back({tets[t].v[i], tets[t].v[j], vol * grads[t][i].dot(grads[t][j])});
    }
    L = from_triplets(nv, tr);
  }

  // initialize (NavierStokes.cpp:10-68): matrices, zero fields, inlet nodes set from the inlet
  // value current at this call, reference node for Neumann outlets.
  void initialize() {
    const double t0 = now_s();
    u.assign(N2, V3());
    ustar.assign(N2, V3());
    p.assign(nv, 0.0);
    pcorr.assign(nv, 0.0);
    if (inlet.size() != N2) inlet.assign(N2, V3());
    build_mass();
    build_stiffness();
    build_gradient();
    build_poisson();
    order_p2 = sell_order(M);
    order_p1 = sell_order(L);
    order_n2 = natural_order((int64_t)N2);
    order_nv = natural_order((int64_t)nv);
    for (size_t i = 0; i < N2; ++i)
      if (bc_of(i) == kInlet) u[i] = inlet[i];
    if (reference_node < 0 && outlet_type == kNeumann) {
      for (size_t i = 0; i < nv; ++i)
        if (p1bc[i] == kInternal) {
          reference_node = (int)i;
          break;
        }
      if (reference_node < 0 && nv > 0) reference_node = 0;
    }
    initialized = true;
    t_assembly = now_s() - t0;
  }

  // ---------------------------------------------------------------- step phases
  // computeAdvectionRHS (NavierStokes.cpp:526-584)
  std::vector<V3> advection() const {
    std::vector<V3> conv(N2, V3());
    for (size_t t = 0; t < nt; ++t) {
      const double vol = tets[t].volume;
      V3 ue;
      for (int i = 0; i < 4; ++i) ue = ue + 0.25 * u[tets[t].v[i]];
      double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int j = 0; j < 4; ++j) {
        const V3 &uj = u[tets[t].v[j]];
        const V3 &gj = grads[t][j];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) gu[a][b] += uj[a] * gj[b];
      }
      V3 c;
      for (int a = 0; a < 3; ++a) c[a] = (gu[a][0] * ue.x + gu[a][1] * ue.y) + gu[a][2] * ue.z;
      for (int i = 0; i < 4; ++i) {
        V3 &o = conv[tets[t].v[i]];
        const double w = vol / 4.0;
        o = o - w * c;
      }
      for (int e = 0; e < 6; ++e) {
        V3 &o = conv[nv + tet_edges[t][e]];
        const double w = vol / 24.0;
        o = o - w * c;
      }
    }
    return conv;
  }

  // The momentum Krylov solve of one component: the reference's Jacobi BiCGSTAB
  // (NavierStokes.cpp:498-515), or Jacobi CG on the same symmetric positive definite system. The
  // device batches the three components; its reductions run over the SELL runs of the P2 pattern
  // (order_p2: products, and the BiCGSTAB initialisation fused into the right-hand side) and over
  // natural 256-position blocks (order_n2: vector updates, and the CG initialisation).
  SolveInfo momentum_solve(const CSR &lhs, const std::vector<double> &rhs, std::vector<double> &x) const {
    if (momentum_solver == 1) return cg(lhs, rhs, x, tol_mom, maxit_mom, order_p2, order_n2, conv_norm == 1);
    return bicgstab(lhs, rhs, x, tol_mom, maxit_mom, order_p2, order_p2, order_n2, conv_norm == 1);
  }

  // solveMomentumPredictor (NavierStokes.cpp:416-524)
  bool momentum() {
    const double t0 = now_s();
    std::vector<V3> conv = advection();
    t_conv = now_s() - t0;
    std::vector<double> uc(N2), rhs(N2), mu(N2), gp(nv), x;
    for (int comp = 0; comp < 3; ++comp) {
      for (size_t i = 0; i < N2; ++i) uc[i] = u[i][comp];
      spmv(M, uc.data(), mu.data());
      for (size_t i = 0; i < N2; ++i) rhs[i] = 0.0 + mu[i] / dt;
      const CSR &G = comp == 0 ? Gx : (comp == 1 ? Gy : Gz);
      spmv(G, p.data(), gp.data());
      for (size_t i = 0; i < nv; ++i) rhs[i] -= gp[i];
      for (size_t i = 0; i < N2; ++i) rhs[i] += conv[i][comp];
      CSR lhs = M;  // same pattern as K
      for (int64_t k = 0; k < lhs.nnz(); ++k) lhs.val[k] = M.val[k] / dt + K.val[k];
      const double penalty = 1e10;
      for (size_t i = 0; i < N2; ++i) {
        const int bc = bc_of(i);
        if (bc == kInlet || bc == kWall) {
          const double up = (bc == kInlet) ? inlet[i][comp] : 0.0;
          for (int64_t k = lhs.rowptr[i]; k < lhs.rowptr[i + 1]; ++k)
            if (lhs.col[k] == (int)i) lhs.val[k] += penalty;
          rhs[i] += penalty * up;
        }
      }
      SolveInfo si = momentum_solve(lhs, rhs, x);
      it_mom[comp] = si.iters;
      res_mom[comp] = si.rel_res;
      if (!si.converged) {
        t_mom = now_s() - t0;
        return false;
      }
      for (size_t i = 0; i < N2; ++i) ustar[i][comp] = x[i];
    }
    t_mom = now_s() - t0;
    return true;
  }

  // computeDivergence (NavierStokes.cpp:670-700)
  void divergence(const std::vector<V3> &uu, std::vector<double> &div) const {
    div.assign(nv, 0.0);
    for (size_t t = 0; t < nt; ++t) {
      const double vol = tets[t].volume;
      double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int j = 0; j < 4; ++j) {
        const V3 &uj = uu[tets[t].v[j]];
        const V3 &gj = grads[t][j];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) gu[a][b] += uj[a] * gj[b];
      }
      const double d = (gu[0][0] + gu[1][1]) + gu[2][2];
      for (int i = 0; i < 4; ++i) div[tets[t].v[i]] += (vol / 4.0) * d;
    }
  }

  void reinforce_pressure_bcs() {
    if (outlet_type == kDirichlet)
      for (size_t i = 0; i < nv; ++i)
        if (p1bc[i] == kOutlet) p[i] = outlet_pressure;
  }
  void normalize_pressure() {
    if (reference_node >= 0 && reference_node < (int)p.size()) {
      const double ref = p[reference_node];
      for (auto &v : p) v -= ref;
    }
  }

  // Pressure Krylov solve with the selected method (0 BiCGSTAB as the reference, 1 CG, 2 CG with
  // one reduction, 3 the same with the two-level preconditioner). The coarse space depends on the
  // penalised rows only through the boundary setup, so it is built once.
  CoarseSpace coarse;
  bool coarse_built = false;
  int coarse_target = 256;
  SolveInfo solve_pressure(const CSR &Lbc, const std::vector<double> &rhs, std::vector<double> &x) {
    if (pressure_solver == 1) return cg(Lbc, rhs, x, tol_p, maxit_p, order_p1, order_nv, conv_norm == 1);
    if (pressure_solver == 2) return cg1(Lbc, rhs, x, tol_p, maxit_p, order_p1, order_nv, conv_norm == 1);
    if (pressure_solver == 3) {
      if (!coarse_built) {
        std::vector<char> pen(nv, 0);
        if (outlet_type == kNeumann) {
          if (reference_node >= 0 && reference_node < (int)nv) pen[reference_node] = 1;
        } else if (outlet_type == kDirichlet) {
          for (size_t i = 0; i < nv; ++i) pen[i] = p1bc[i] == kOutlet;
        }
        coarse = build_coarse(Lbc, vertices, pen, coarse_target);
        coarse_built = true;
      }
      return cg2l(Lbc, rhs, x, tol_p, maxit_p, order_p1, order_nv, conv_norm == 1, coarse);
    }
    return bicgstab(Lbc, rhs, x, tol_p, maxit_p, order_nv, order_p1, order_nv, conv_norm == 1);
  }

  // solvePressurePoisson (NavierStokes.cpp:586-668)
  bool pressure() {
    const double t0 = now_s();
    std::vector<double> div, rhs(nv), x;
    divergence(ustar, div);
    for (size_t i = 0; i < nv; ++i) rhs[i] = -div[i] / dt;
    CSR Lbc = L;
    const double penalty = 1e12;
    auto add_diag = [&](size_t i, double v) {
      for (int64_t k = Lbc.rowptr[i]; k < Lbc.rowptr[i + 1]; ++k)
        if (Lbc.col[k] == (int)i) Lbc.val[k] += v;
    };
    if (outlet_type == kNeumann) {
      if (reference_node >= 0 && reference_node < (int)nv) {
        add_diag(reference_node, penalty);
        rhs[reference_node] += penalty * 0.0;
      }
    } else if (outlet_type == kDirichlet) {
      for (size_t i = 0; i < nv; ++i)
        if (p1bc[i] == kOutlet) {
          add_diag(i, penalty);
          rhs[i] += penalty * outlet_pressure;
        }
    }
    SolveInfo si = solve_pressure(Lbc, rhs, x);
    it_p = si.iters;
    res_p = si.rel_res;
    if (!si.converged) {
      t_press += now_s() - t0;
      return false;
    }
    for (size_t i = 0; i < nv; ++i) pcorr[i] = x[i];
    for (size_t i = 0; i < nv; ++i) p[i] += relax_p * pcorr[i];
    reinforce_pressure_bcs();
    normalize_pressure();
    t_press += now_s() - t0;
    return true;
  }

  // correctVelocity (NavierStokes.cpp:702-771)
  bool correct() {
    const double t0 = now_s();
    std::vector<double> gx(nv), gy(nv), gz(nv);
    spmv(Gx, pcorr.data(), gx.data());
    spmv(Gy, pcorr.data(), gy.data());
    spmv(Gz, pcorr.data(), gz.data());
    for (size_t i = 0; i < nv; ++i) {
      const int bc = p1bc[i];
      if (bc == kInlet) {
        u[i] = inlet[i];
        continue;
      } else if (bc == kWall) {
        u[i] = V3();
        continue;
      }
      if (inv_lumped[i] > 1e-14) {
        const double f = -dt * inv_lumped[i];
        const V3 corr(f * gx[i], f * gy[i], f * gz[i]);
        u[i] = ustar[i] + relax_u * corr;
      } else {
        u[i] = ustar[i];
      }
    }
    for (size_t k = 0; k < ne; ++k) {
      const int bc = p2bc[k];
      const size_t idx = nv + k;
      if (bc == kInlet) {
        u[idx] = inlet[idx];
        continue;
      } else if (bc == kWall) {
        u[idx] = V3();
        continue;
      }
      u[idx] = ustar[idx];
    }
    t_corr += now_s() - t0;
    return true;
  }

  // reenforceVelocityBCs (NavierStokes.cpp:815-839)
  void reenforce_velocity_bcs() {
    for (size_t i = 0; i < N2; ++i) {
      const int bc = bc_of(i);
      if (bc == kInlet)
        u[i] = inlet[i];
      else if (bc == kWall)
        u[i] = V3();
    }
  }

  bool has_nans() const {
    for (const auto &v : u)
      if (std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z)) return true;
    for (const auto &v : ustar)
      if (std::isnan(v.x) || std::isnan(v.y) || std::isnan(v.z)) return true;
    for (double v : p)
      if (std::isnan(v)) return true;
    for (double v : pcorr)
      if (std::isnan(v)) return true;
    return false;
  }

  // pisoStep (NavierStokes.cpp:374-414)
  int piso_step() {
    if (!initialized) return 6;
    t_press = t_corr = 0;
    if (!momentum()) return 1;
    for (int c = 0; c < n_corr; ++c) {
      if (!pressure()) return 1;
      if (!correct()) return 1;
    }
    reenforce_velocity_bcs();
    time += dt;
    return has_nans() ? 3 : 0;
  }
  // simpleStep (NavierStokes.cpp:968-1009)
  int simple_step() {
    if (!initialized) return 6;
    t_press = t_corr = 0;
    if (!momentum()) return 1;
    if (!pressure()) return 1;
    reinforce_pressure_bcs();
    if (!correct()) return 1;
    reenforce_velocity_bcs();
    time += dt;
    return has_nans() ? 3 : 0;
  }

  // computePressureForces / computeShearStress (NavierStokes.cpp:841-944)
  void pressure_forces(double *out) const {
    std::fill(out, out + 3 * nv, 0.0);
    for (const auto &f : faces) {
      if (f.tet_b != -1) continue;
      double fp = 0.0;
      for (int k = 0; k < 3; ++k) fp += p[f.v[k]];
      fp /= 3.0;
      const V3 ff = -fp * f.normal * f.area;
      for (int k = 0; k < 3; ++k) {
        const V3 c = ff * (1.0 / 3.0);
        out[3 * f.v[k]] += c.x;
        out[3 * f.v[k] + 1] += c.y;
        out[3 * f.v[k] + 2] += c.z;
      }
    }
  }
  void shear_stress(double *out) const {
    std::fill(out, out + 3 * nv, 0.0);
    const double mu = viscosity;
    for (const auto &f : faces) {
      if (f.tet_b != -1) continue;
      const int t = f.tet_a;
      double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      for (int i = 0; i < 4; ++i) {
        const V3 &uu = u[tets[t].v[i]];
        const V3 &g = grads[t][i];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) gu[a][b] += uu[a] * g[b];
      }
      double tau[3][3];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) tau[a][b] = 2.0 * mu * (0.5 * (gu[a][b] + gu[b][a]));
      V3 tr;
      for (int a = 0; a < 3; ++a)
        tr[a] = (tau[a][0] * f.normal.x + tau[a][1] * f.normal.y) + tau[a][2] * f.normal.z;
      const V3 ff = tr * f.area;
      for (int k = 0; k < 3; ++k) {
        const V3 c = ff * (1.0 / 3.0);
        out[3 * f.v[k]] += c.x;
        out[3 * f.v[k] + 1] += c.y;
        out[3 * f.v[k] + 2] += c.z;
      }
    }
  }

  // ---------------------------------------------------------------- discrete adjoint
  // Reverse mode through the PISO steps exactly as implemented above (each Krylov solve taken
  // as the exact linear solve it converges to). The differentiated map is
  //   (inlet values g, viscosity) -> J(u^N, p^N)
  // with the state (u^0, p^0) at the start of recording held fixed. Operators: M, K, L are
  // symmetric, so the adjoint solves reuse the forward operators; G needs its transpose.
  struct AdjRecord {
    std::vector<V3> u, us;  // u^n (step input) and u* of step n
  };
  std::vector<AdjRecord> adj_rec;
  std::vector<V3> adj_u0;
  std::vector<double> adj_p0;
  int adj_it_mom = 0, adj_it_p = 0;

  // Forward half: nsteps PISO steps from the current state, recording step inputs and u*.
  int adjoint_forward(int nsteps) {
    adj_rec.clear();
    adj_u0 = u;
    adj_p0 = p;
    for (int n = 0; n < nsteps; ++n) {
      adj_rec.push_back({u, {}});
      const int rc = piso_step();
      adj_rec.back().us = ustar;
      if (rc) return rc;
    }
    return 0;
  }

  static CSR transpose(const CSR &A, int64_t ncols) {
    CSR T;
    T.n = ncols;
    T.rowptr.assign(ncols + 1, 0);
    for (int c : A.col) T.rowptr[c + 1]++;
    for (int64_t i = 0; i < ncols; ++i) T.rowptr[i + 1] += T.rowptr[i];
    T.col.resize(A.col.size());
    T.val.resize(A.val.size());
    std::vector<int64_t> fill(T.rowptr.begin(), T.rowptr.end() - 1);
    for (int64_t i = 0; i < A.n; ++i)
      for (int64_t k = A.rowptr[i]; k < A.rowptr[i + 1]; ++k) {
        const int64_t q = fill[A.col[k]]++;
        T.col[q] = (int)i;
        T.val[q] = A.val[k];
      }
    return T;
  }

  CSR momentum_lhs() const {
    CSR lhs = M;
    for (int64_t k = 0; k < lhs.nnz(); ++k) lhs.val[k] = M.val[k] / dt + K.val[k];
    for (size_t i = 0; i < N2; ++i) {
      const int bc = bc_of(i);
      if (bc == kInlet || bc == kWall)
        for (int64_t k = lhs.rowptr[i]; k < lhs.rowptr[i + 1]; ++k)
          if (lhs.col[k] == (int)i) lhs.val[k] += 1e10;
    }
    return lhs;
  }
  CSR poisson_lhs() const {
    CSR Lbc = L;
    auto add_diag = [&](size_t i, double v) {
      for (int64_t k = Lbc.rowptr[i]; k < Lbc.rowptr[i + 1]; ++k)
        if (Lbc.col[k] == (int)i) Lbc.val[k] += v;
    };
    if (outlet_type == kNeumann) {
      if (reference_node >= 0 && reference_node < (int)nv) add_diag(reference_node, 1e12);
    } else if (outlet_type == kDirichlet) {
      for (size_t i = 0; i < nv; ++i)
        if (p1bc[i] == kOutlet) add_diag(i, 1e12);
    }
    return Lbc;
  }

  // Objectives on the current state. kind 0: mean over wall vertices with
  // lo <= x[axis] <= hi of |s_v|^2, s = computeShearStress (NavierStokes.cpp:874-944);
  // kind 1: mean p over inlet vertices minus mean p over outlet vertices. Returns J and the
  // seeds dJ/du [N2], dJ/dp [nv] and the explicit dJ/dviscosity; -1 if the vertex set is empty.
  int objective(int kind, int axis, double lo, double hi, double *J, std::vector<V3> &su,
                std::vector<double> &sp, double *dnu) const {
    su.assign(N2, V3());
    sp.assign(nv, 0.0);
    *dnu = 0.0;
    if (kind == 0) {
      std::vector<double> s(3 * nv);
      shear_stress(s.data());
      std::vector<char> in(nv, 0);
      int64_t np = 0;
      for (size_t v = 0; v < nv; ++v)
        if (p1bc[v] == kWall && vertices[v][axis] >= lo && vertices[v][axis] <= hi) {
          in[v] = 1;
          ++np;
        }
      if (np == 0) return -1;
      const double inv = 1.0 / (double)np;
      const double acc = tree_sum(order_nv, [&](int v) {
        return in[v] ? (s[3 * v] * s[3 * v] + s[3 * v + 1] * s[3 * v + 1]) + s[3 * v + 2] * s[3 * v + 2]
                     : 0.0;
      });
      *J = acc * inv;
      const double c = 2.0 * inv;
      std::vector<V3> w(nv);
      for (size_t v = 0; v < nv; ++v)
        if (in[v]) w[v] = V3(c * s[3 * v], c * s[3 * v + 1], c * s[3 * v + 2]);
      const double mu = viscosity;
      for (const auto &f : faces) {
        if (f.tet_b != -1) continue;
        const V3 ws = (w[f.v[0]] + w[f.v[1]]) + w[f.v[2]];
        const V3 W = ws * (f.area * (1.0 / 3.0));
        const int t = f.tet_a;
        for (int l = 0; l < 4; ++l) {
          const V3 &g = grads[t][l];
          const double ng = f.normal.dot(g), wg = W.dot(g);
          V3 &o = su[tets[t].v[l]];
          for (int a = 0; a < 3; ++a) o[a] = o[a] + mu * (W[a] * ng + f.normal[a] * wg);
        }
      }
      *dnu = 2.0 * (*J) / viscosity;
      return 0;
    }
    int64_t nin = 0, nout = 0;
    for (size_t v = 0; v < nv; ++v) {
      nin += p1bc[v] == kInlet;
      nout += p1bc[v] == kOutlet;
    }
    if (nin == 0 || nout == 0) return -1;
    const double ii = 1.0 / (double)nin, io = 1.0 / (double)nout;
    const double si = tree_sum(order_nv, [&](int v) { return p1bc[v] == kInlet ? p[v] : 0.0; });
    const double so = tree_sum(order_nv, [&](int v) { return p1bc[v] == kOutlet ? p[v] : 0.0; });
    *J = si * ii - so * io;
    for (size_t v = 0; v < nv; ++v) {
      if (p1bc[v] == kInlet) sp[v] = ii;
      if (p1bc[v] == kOutlet) sp[v] = -io;
    }
    return 0;
  }

  // Backward half. lu/lp: dJ/du^N, dJ/dp^N on entry, dJ/du^0, dJ/dp^0 on exit. gin: dJ/dg per
  // node [N2] (zero off inlet nodes); gnu: dJ/dviscosity (dnu_explicit included).
  int adjoint_backward(std::vector<V3> &lu, std::vector<double> &lp, double dnu_explicit,
                       std::vector<V3> &gin, double *gnu) {
    const CSR A = momentum_lhs();
    const CSR Lbc = poisson_lhs();
    const CSR GT[3] = {transpose(Gx, nv), transpose(Gy, nv), transpose(Gz, nv)};
    gin.assign(N2, V3());
    double gn = dnu_explicit;
    adj_it_mom = adj_it_p = 0;
    const bool normalize = reference_node >= 0 && reference_node < (int)nv;
    const int ncorr = std::max(n_corr, 0);
    std::vector<double> q[3], lam(N2), x, lpp(nv), chain(nv), rhs(nv), mu_p, t0(nv), t1(nv), t2(nv);
    std::vector<V3> lus(N2), nu(N2), cadj(N2);
    for (int a = 0; a < 3; ++a) q[a].assign(nv, 0.0);
    for (int n = (int)adj_rec.size() - 1; n >= 0; --n) {
      const AdjRecord &R = adj_rec[n];
      // correctVelocity + reenforceVelocityBCs (NavierStokes.cpp:702-771, 815-839)
      for (size_t i = 0; i < N2; ++i) {
        const int bc = bc_of(i);
        lus[i] = V3();
        if (i < nv)
          for (int a = 0; a < 3; ++a) q[a][i] = 0.0;
        if (bc == kInlet) {
          gin[i] = gin[i] + lu[i];
          continue;
        }
        if (bc == kWall) continue;
        lus[i] = lu[i];
        if (i < nv && inv_lumped[i] > 1e-14) {
          const double f = -dt * inv_lumped[i];
          for (int a = 0; a < 3; ++a) q[a][i] = relax_u * (f * lu[i][a]);
        }
      }
      // p += relax_p p', reinforcePressureBCs, normalizePressire, once per corrector
      chain = lp;
      std::fill(lpp.begin(), lpp.end(), 0.0);
      for (int c = ncorr - 1; c >= 0; --c) {
        double S = 0.0;
        if (normalize) S = tree_sum(order_nv, [&](int i) { return chain[i]; });
        for (size_t i = 0; i < nv; ++i) {
          double w = chain[i];
          if (normalize && (int)i == reference_node) w = w - S;
          if (outlet_type == kDirichlet && p1bc[i] == kOutlet) w = 0.0;
          lpp[i] = lpp[i] + relax_p * w;
          chain[i] = w;
        }
      }
      // velocity correction u -= relax_u dt m^-1 G p'
      spmv(GT[0], q[0].data(), t0.data());
      spmv(GT[1], q[1].data(), t1.data());
      spmv(GT[2], q[2].data(), t2.data());
      for (size_t i = 0; i < nv; ++i) rhs[i] = ((t0[i] + t1[i]) + t2[i]) + lpp[i];
      // pressure Poisson solve (L symmetric)
      {
        SolveInfo si = solve_pressure(Lbc, rhs, mu_p);
        adj_it_p += si.iters;
        if (!si.converged) return 1;
      }
      // b = -div(u*)/dt = -(1/dt) sum_a G_a u*_a|P1
      spmv(GT[0], mu_p.data(), t0.data());
      spmv(GT[1], mu_p.data(), t1.data());
      spmv(GT[2], mu_p.data(), t2.data());
      for (size_t i = 0; i < nv; ++i) {
        lus[i].x = lus[i].x - t0[i] / dt;
        lus[i].y = lus[i].y - t1[i] / dt;
        lus[i].z = lus[i].z - t2[i] / dt;
      }
      // momentum solves (A symmetric)
      for (int a = 0; a < 3; ++a) {
        for (size_t i = 0; i < N2; ++i) lam[i] = lus[i][a];
        SolveInfo si = momentum_solve(A, lam, x);
        adj_it_mom = std::max(adj_it_mom, si.iters);
        if (!si.converged) return 1;
        for (size_t i = 0; i < N2; ++i) nu[i][a] = x[i];
      }
      // viscosity: dA/dnu = -K/nu  ->  dJ/dnu += sum_a nu_a . K u*_a / nu
      {
        std::vector<double> ku[3], na[3], usa(N2);
        for (int a = 0; a < 3; ++a) {
          for (size_t i = 0; i < N2; ++i) usa[i] = R.us[i][a];
          ku[a].resize(N2);
          spmv(K, usa.data(), ku[a].data());
        }
        const double tot = tree_sum(order_p2, [&](int i) {
          return (nu[i].x * ku[0][i] + nu[i].y * ku[1][i]) + nu[i].z * ku[2][i];
        });
        gn += tot / viscosity;
      }
      // convection adjoint (computeAdvectionRHS, NavierStokes.cpp:550-580) over u^n
      std::fill(cadj.begin(), cadj.end(), V3());
      for (size_t t = 0; t < nt; ++t) {
        const double vol = tets[t].volume;
        V3 s1, s2;
        for (int l = 0; l < 4; ++l) s1 = s1 + nu[tets[t].v[l]];
        for (int e = 0; e < 6; ++e) s2 = s2 + nu[nv + tet_edges[t][e]];
        double ch[3];
        for (int a = 0; a < 3; ++a) ch[a] = -((vol / 4.0) * s1[a] + (vol / 24.0) * s2[a]);
        V3 ue;
        for (int l = 0; l < 4; ++l) ue = ue + 0.25 * R.u[tets[t].v[l]];
        double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int j = 0; j < 4; ++j) {
          const V3 &uj = R.u[tets[t].v[j]];
          const V3 &gj = grads[t][j];
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) gu[a][b] += uj[a] * gj[b];
        }
        double h[3];
        for (int b = 0; b < 3; ++b) h[b] = 0.25 * ((gu[0][b] * ch[0] + gu[1][b] * ch[1]) + gu[2][b] * ch[2]);
        for (int l = 0; l < 4; ++l) {
          const double d = grads[t][l].dot(ue);
          V3 &o = cadj[tets[t].v[l]];
          for (int a = 0; a < 3; ++a) o[a] = o[a] + (ch[a] * d + h[a]);
        }
      }
      // momentum right-hand side: M u^n / dt - G p^n + conv(u^n) + penalty g
      std::vector<double> mv[3], na(N2);
      for (int a = 0; a < 3; ++a) {
        for (size_t i = 0; i < N2; ++i) na[i] = nu[i][a];
        mv[a].resize(N2);
        spmv(M, na.data(), mv[a].data());
      }
      for (int a = 0; a < 3; ++a) {
        std::vector<double> nP(nv);
        for (size_t i = 0; i < nv; ++i) nP[i] = nu[i][a];
        spmv(GT[a], nP.data(), a == 0 ? t0.data() : (a == 1 ? t1.data() : t2.data()));
      }
      for (size_t i = 0; i < N2; ++i) {
        for (int a = 0; a < 3; ++a) {
          double v = mv[a][i] / dt;
          if (i < nv) v = v + cadj[i][a];
          lu[i][a] = v;
        }
        if (bc_of(i) == kInlet)
          for (int a = 0; a < 3; ++a) gin[i][a] = gin[i][a] + 1e10 * nu[i][a];
      }
      for (size_t i = 0; i < nv; ++i) lp[i] = chain[i] - ((t0[i] + t1[i]) + t2[i]);
    }
    *gnu = gn;
    return 0;
  }
};

const CSR *matrix_of(const Oracle *o, int which) {
  switch (which) {
    case 0: return &o->M;
    case 1: return &o->K;
    case 2: return &o->Gx;
    case 3: return &o->Gy;
    case 4: return &o->Gz;
    case 5: return &o->L;
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

// Builds the oracle mesh from raw vertices [nv][3] and tets [nt][4] (0-based) and, when
// apply_bc != 0, tags boundaries with Mesh::setupBoundaryConditions(dir, coverage).
void *orc_create(int64_t nv, const double *xyz, int64_t nt, const int *tets, int apply_bc,
                 const double *dir, double coverage) {
  Oracle *o = new Oracle();
  o->nv = (size_t)nv;
  o->nt = (size_t)nt;
  o->vertices.resize(o->nv);
  o->tets.resize(o->nt);
  o->build_mesh(xyz, tets);
  if (apply_bc) o->setup_bc(dir, coverage);
  return o;
}
void orc_destroy(void *h) { delete static_cast<Oracle *>(h); }

// sizes: nv, nt, ne, nfaces, n boundary faces
void orc_sizes(void *h, int64_t *out) {
  Oracle *o = static_cast<Oracle *>(h);
  int64_t nb = 0;
  for (const auto &f : o->faces) nb += (f.tet_b == -1);
  out[0] = (int64_t)o->nv;
  out[1] = (int64_t)o->nt;
  out[2] = (int64_t)o->ne;
  out[3] = (int64_t)o->faces.size();
  out[4] = nb;
}
void orc_get_mesh(void *h, int *tet_edges, int *p1bc, int *p2bc, int *face_verts, int *face_tets,
                  double *face_geom, double *vol, double *grads, double *edge_xyz) {
  Oracle *o = static_cast<Oracle *>(h);
  for (size_t t = 0; t < o->nt; ++t) {
    for (int e = 0; e < 6; ++e) tet_edges[6 * t + e] = o->tet_edges[t][e];
    vol[t] = o->tets[t].volume;
    for (int a = 0; a < 4; ++a)
      for (int c = 0; c < 3; ++c) grads[12 * t + 3 * a + c] = o->grads[t][a][c];
  }
  for (size_t i = 0; i < o->nv; ++i) p1bc[i] = o->p1bc[i];
  for (size_t k = 0; k < o->ne; ++k) {
    p2bc[k] = o->p2bc[k];
    for (int c = 0; c < 3; ++c) edge_xyz[3 * k + c] = o->edge_nodes[k][c];
  }
  for (size_t f = 0; f < o->faces.size(); ++f) {
    const auto &F = o->faces[f];
    for (int k = 0; k < 3; ++k) face_verts[3 * f + k] = F.v[k];
    face_tets[2 * f] = F.tet_a;
    face_tets[2 * f + 1] = F.tet_b;
    double *g = face_geom + 7 * f;
    g[0] = F.normal.x;
    g[1] = F.normal.y;
    g[2] = F.normal.z;
    g[3] = F.area;
    g[4] = F.center.x;
    g[5] = F.center.y;
    g[6] = F.center.z;
  }
}
// Overrides the boundary tags (FluidBCType integers) before initialize.
void orc_set_bc(void *h, const int *p1bc, const int *p2bc) {
  Oracle *o = static_cast<Oracle *>(h);
  for (size_t i = 0; i < o->nv; ++i) o->p1bc[i] = p1bc[i];
  for (size_t k = 0; k < o->ne; ++k) o->p2bc[k] = p2bc[k];
}

void orc_set_fluid(void *h, double density, double viscosity) {
  Oracle *o = static_cast<Oracle *>(h);
  o->density = density;
  o->viscosity = viscosity;
}
// Parameters: dt, momentum tol, pressure tol, momentum maxit, pressure maxit, corrections,
// relax_u, relax_p, outlet type, outlet pressure, reference node, pressure solver (0 BiCGSTAB,
// 1 CG, 2 single-reduction CG, 3 single-reduction CG with the two-level preconditioner),
// convergence norm (0 ||r||, 1 ||D^-1/2 r||).
void orc_set_params(void *h, double dt, double tol_mom, double tol_p, int maxit_mom, int maxit_p,
                    int n_corr, double relax_u, double relax_p, int outlet_type,
                    double outlet_pressure, int reference_node, int pressure_solver, int conv_norm) {
  Oracle *o = static_cast<Oracle *>(h);
  o->conv_norm = conv_norm;
  o->dt = dt;
  o->tol_mom = tol_mom;
  o->tol_p = tol_p;
  o->maxit_mom = maxit_mom;
  o->maxit_p = maxit_p;
  o->n_corr = n_corr;
  o->relax_u = relax_u;
  o->relax_p = relax_p;
  o->outlet_type = outlet_type;
  o->outlet_pressure = outlet_pressure;
  o->reference_node = reference_node;
  o->pressure_solver = pressure_solver;
  o->coarse_built = false;
}
// NavierStokesSolver::solvePressureBiCGSTAB (src/FEM/NavierStokes.cpp:773-802): BiCGSTAB with
// Jacobi on the raw Poisson matrix L (no boundary penalty), zero initial guess (Eigen's solve),
// stopping at tol / maxit; x [nv] receives the iterate. Returns 0 when converged, 1 otherwise.
int orc_solve_poisson_raw(void *h, const double *rhs, double *x, double tol, int maxit, int *iters) {
  Oracle *o = static_cast<Oracle *>(h);
  std::vector<double> b(rhs, rhs + o->nv), xv;
  SolveInfo si = bicgstab(o->L, b, xv, tol, maxit, o->order_nv, o->order_p1, o->order_nv, false);
  std::copy(xv.begin(), xv.end(), x);
  if (iters) *iters = si.iters;
  return si.converged ? 0 : 1;
}

// Target number of aggregates of the two-level pressure preconditioner (default 256). Returns 0,
// or 1 (target unchanged) outside [1, 1024], the range the device solver accepts.
// Momentum Krylov method: 0 BiCGSTAB (the reference's), 1 Jacobi CG.
int orc_set_momentum_solver(void *h, int solver) {
  if (solver != 0 && solver != 1) return 1;
  static_cast<Oracle *>(h)->momentum_solver = solver;
  return 0;
}

int orc_set_coarse_target(void *h, int target) {
  if (target < 1 || target > 1024) return 1;
  Oracle *o = static_cast<Oracle *>(h);
  o->coarse_target = target;
  o->coarse_built = false;
  return 0;
}
// Aggregates of the coarse space last built (0 before the first two-level solve).
int orc_coarse_size(void *h) { return static_cast<Oracle *>(h)->coarse.nc; }
// Per-node inlet velocity [N2][3] (P1 nodes first, then P2 edge nodes).
void orc_set_inlet(void *h, const double *vals) {
  Oracle *o = static_cast<Oracle *>(h);
  o->inlet.resize(o->N2);
  for (size_t i = 0; i < o->N2; ++i) o->inlet[i] = V3(vals[3 * i], vals[3 * i + 1], vals[3 * i + 2]);
}
void orc_initialize(void *h) { static_cast<Oracle *>(h)->initialize(); }
int orc_reference_node(void *h) { return static_cast<Oracle *>(h)->reference_node; }
int orc_piso_step(void *h) { return static_cast<Oracle *>(h)->piso_step(); }
int orc_simple_step(void *h) { return static_cast<Oracle *>(h)->simple_step(); }
int orc_momentum(void *h) { return static_cast<Oracle *>(h)->momentum() ? 0 : 1; }
int orc_pressure(void *h) { return static_cast<Oracle *>(h)->pressure() ? 0 : 1; }
int orc_correct(void *h) { return static_cast<Oracle *>(h)->correct() ? 0 : 1; }

void orc_get_state(void *h, double *u, double *ustar, double *p, double *pcorr, double *time) {
  Oracle *o = static_cast<Oracle *>(h);
  for (size_t i = 0; i < o->N2; ++i)
    for (int c = 0; c < 3; ++c) {
      u[3 * i + c] = o->u[i][c];
      ustar[3 * i + c] = o->ustar[i][c];
    }
  for (size_t i = 0; i < o->nv; ++i) {
    p[i] = o->p[i];
    pcorr[i] = o->pcorr[i];
  }
  *time = o->time;
}
void orc_set_state(void *h, const double *u, const double *p) {
  Oracle *o = static_cast<Oracle *>(h);
  for (size_t i = 0; i < o->N2; ++i) o->u[i] = V3(u[3 * i], u[3 * i + 1], u[3 * i + 2]);
  for (size_t i = 0; i < o->nv; ++i) o->p[i] = p[i];
}
// which: 0 M, 1 K, 2 Gx, 3 Gy, 4 Gz, 5 L. Returns nnz (rows in *nrows).
int64_t orc_matrix_nnz(void *h, int which, int64_t *nrows) {
  const CSR *A = matrix_of(static_cast<Oracle *>(h), which);
  if (!A) return -1;
  *nrows = A->n;
  return A->nnz();
}
void orc_get_matrix(void *h, int which, int64_t *rowptr, int *cols, double *vals) {
  const CSR *A = matrix_of(static_cast<Oracle *>(h), which);
  std::copy(A->rowptr.begin(), A->rowptr.end(), rowptr);
  std::copy(A->col.begin(), A->col.end(), cols);
  std::copy(A->val.begin(), A->val.end(), vals);
}
void orc_get_inv_lumped_mass(void *h, double *out) {
  Oracle *o = static_cast<Oracle *>(h);
  std::copy(o->inv_lumped.begin(), o->inv_lumped.end(), out);
}
void orc_advection(void *h, double *out) {
  Oracle *o = static_cast<Oracle *>(h);
  std::vector<V3> c = o->advection();
  for (size_t i = 0; i < o->N2; ++i)
    for (int k = 0; k < 3; ++k) out[3 * i + k] = c[i][k];
}
void orc_divergence(void *h, const double *u, double *out) {
  Oracle *o = static_cast<Oracle *>(h);
  std::vector<V3> uu(o->N2);
  for (size_t i = 0; i < o->N2; ++i) uu[i] = V3(u[3 * i], u[3 * i + 1], u[3 * i + 2]);
  std::vector<double> d;
  o->divergence(uu, d);
  std::copy(d.begin(), d.end(), out);
}
void orc_pressure_forces(void *h, double *out) { static_cast<Oracle *>(h)->pressure_forces(out); }
void orc_shear_stress(void *h, double *out) { static_cast<Oracle *>(h)->shear_stress(out); }
// stats: it_mom[3], it_p, res_mom[3], res_p, t_assembly, t_conv, t_mom, t_press, t_corr
void orc_stats(void *h, int *iters, double *res, double *times) {
  Oracle *o = static_cast<Oracle *>(h);
  for (int c = 0; c < 3; ++c) {
    iters[c] = o->it_mom[c];
    res[c] = o->res_mom[c];
  }
  iters[3] = o->it_p;
  res[3] = o->res_p;
  times[0] = o->t_assembly;
  times[1] = o->t_conv;
  times[2] = o->t_mom;
  times[3] = o->t_press;
  times[4] = o->t_corr;
}
// ---- discrete adjoint ----
// Runs nsteps PISO steps from the current state, recording what the backward pass needs.
int orc_adjoint_forward(void *h, int nsteps) { return static_cast<Oracle *>(h)->adjoint_forward(nsteps); }
// Objective on the current state (kind 0: wall-shear patch over [lo,hi] along axis; 1: pressure
// drop inlet-outlet); seeds returned as dJ/du [N2][3], dJ/dp [nv] and explicit dJ/dviscosity.
int orc_objective(void *h, int kind, int axis, double lo, double hi, double *J, double *su,
                  double *sp, double *dnu) {
  Oracle *o = static_cast<Oracle *>(h);
  std::vector<V3> u_s;
  std::vector<double> p_s;
  const int rc = o->objective(kind, axis, lo, hi, J, u_s, p_s, dnu);
  if (rc) return rc;
  for (size_t i = 0; i < o->N2; ++i)
    for (int c = 0; c < 3; ++c) su[3 * i + c] = u_s[i][c];
  std::copy(p_s.begin(), p_s.end(), sp);
  return 0;
}
// Backward pass from seeds (lu [N2][3], lp [nv] are overwritten by dJ/du^0, dJ/dp^0);
// gin [N2][3] = dJ/d(inlet values), *gnu = dJ/dviscosity (dnu_explicit included).
int orc_adjoint_backward(void *h, double *lu, double *lp, double dnu_explicit, double *gin,
                         double *gnu, int *iters) {
  Oracle *o = static_cast<Oracle *>(h);
  std::vector<V3> L(o->N2), G;
  for (size_t i = 0; i < o->N2; ++i) L[i] = V3(lu[3 * i], lu[3 * i + 1], lu[3 * i + 2]);
  std::vector<double> P(lp, lp + o->nv);
  const int rc = o->adjoint_backward(L, P, dnu_explicit, G, gnu);
  iters[0] = o->adj_it_mom;
  iters[1] = o->adj_it_p;
  if (rc) return rc;
  for (size_t i = 0; i < o->N2; ++i)
    for (int c = 0; c < 3; ++c) {
      lu[3 * i + c] = L[i][c];
      gin[3 * i + c] = G[i][c];
    }
  std::copy(P.begin(), P.end(), lp);
  return 0;
}
// Synthetic cylinder input (the reference meshes with TetGen, absent here): the same vertex and
// tet arrays as the product's procedural mesher, produced here so that a CPU run of the oracle
// needs no product library. Disk: centre point, then ring k = 1..rings of 6k points at radius
// R k / rings; rings k-1 and k are stitched by a merge walk over their angular positions. Axis x:
// `layers` equal prism layers on [0, L]. Each prism splits into 3 tets around its minimum-index
// vertex (Dompierre et al. 1999, so shared quad faces get the same diagonal); tets are oriented
// to positive signed volume. Sizes: nv = (1 + 3 rings (rings+1)) (layers+1), nt = 3 * 6 rings^2
// * layers. Returns 0, or 1 for invalid sizes.
int orc_cylinder(double length, double radius, int rings, int layers, double *xyz, int *tets) {
  if (rings < 1 || layers < 1 || !(length > 0.0) || !(radius > 0.0)) return 1;
  std::vector<double> dy{0.0}, dz{0.0};
  std::vector<int> first(rings + 1, 0), count(rings + 1, 1);
  for (int k = 1; k <= rings; ++k) {
    first[k] = (int)dy.size();
    count[k] = 6 * k;
    const double rad = radius * (double)k / (double)rings;
    for (int j = 0; j < count[k]; ++j) {
      const double th = 2.0 * M_PI * (double)j / (double)count[k];
      dy.push_back(rad * std::cos(th));
      dz.push_back(rad * std::sin(th));
    }
  }
  std::vector<std::array<int, 3>> tri;
  for (int k = 1; k <= rings; ++k) {
    const int na = count[k - 1], nb = count[k], fa = first[k - 1], fb = first[k];
    int i = 0, j = 0;
    while (i < na || j < nb) {
      // position of the next point on each ring as a fraction of a turn; the centre never moves
      const double ta = (k == 1) ? 2.0 : (double)(i + 1) / (double)na;
      const double tb = (double)(j + 1) / (double)nb;
      const bool inner = (j >= nb) || (i < na && k > 1 && ta < tb);
      if (inner) {
        tri.push_back({fa + i % na, fb + j % nb, fa + (i + 1) % na});
        ++i;
      } else {
        tri.push_back({fa + i % na, fb + j % nb, fb + (j + 1) % nb});
        ++j;
      }
      if (k == 1 && j >= nb) break;
    }
  }
  const int np = (int)dy.size();
  for (int l = 0; l <= layers; ++l) {
    const double x = length * (double)l / (double)layers;
    for (int q = 0; q < np; ++q) {
      double *v = xyz + 3 * ((size_t)l * np + q);
      v[0] = x;
      v[1] = dy[q];
      v[2] = dz[q];
    }
  }
  // vertex order of the prism (bottom 0,1,2 / top 3,4,5) rotated so the smallest index comes first
  static const int rot[6][6] = {{0, 1, 2, 3, 4, 5}, {1, 2, 0, 4, 5, 3}, {2, 0, 1, 5, 3, 4},
                                {3, 5, 4, 0, 2, 1}, {4, 3, 5, 1, 0, 2}, {5, 4, 3, 2, 1, 0}};
  size_t t = 0;
  for (int l = 0; l < layers; ++l)
    for (const auto &tr : tri) {
      int P[6];
      for (int a = 0; a < 3; ++a) {
        P[a] = l * np + tr[a];
        P[a + 3] = (l + 1) * np + tr[a];
      }
      int m = 0;
      for (int a = 1; a < 6; ++a)
        if (P[a] < P[m]) m = a;
      int V[6];
      for (int a = 0; a < 6; ++a) V[a] = P[rot[m][a]];
      int T[3][4];
      if (std::min(V[1], V[5]) < std::min(V[2], V[4])) {
        const int c[3][4] = {{V[0], V[1], V[2], V[5]}, {V[0], V[1], V[5], V[4]}, {V[0], V[4], V[5], V[3]}};
        std::memcpy(T, c, sizeof(T));
      } else {
        const int c[3][4] = {{V[0], V[1], V[2], V[4]}, {V[0], V[4], V[2], V[5]}, {V[0], V[4], V[5], V[3]}};
        std::memcpy(T, c, sizeof(T));
      }
      for (auto &c : T) {
        const double *a = xyz + 3 * (size_t)c[0], *b = xyz + 3 * (size_t)c[1], *e = xyz + 3 * (size_t)c[2],
                     *d = xyz + 3 * (size_t)c[3];
        const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const double w[3] = {e[0] - a[0], e[1] - a[1], e[2] - a[2]};
        const double s[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
        const double det = (u[1] * w[2] - u[2] * w[1]) * s[0] + (u[2] * w[0] - u[0] * w[2]) * s[1] +
                           (u[0] * w[1] - u[1] * w[0]) * s[2];
        int *o = tets + 4 * t++;
        o[0] = c[0];
        o[1] = c[1];
        o[2] = det < 0.0 ? c[3] : c[2];
        o[3] = det < 0.0 ? c[2] : c[3];
      }
    }
  return 0;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

}  // extern "C"
