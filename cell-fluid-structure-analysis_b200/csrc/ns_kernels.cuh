// CUDA kernels of the P2/P1 PISO step (sm_100a, FP64 path).
//
// Every kernel that mirrors an element loop of the reference keeps the reference's arithmetic
// order (this translation unit is compiled with -fmad=false, so a*b+c rounds twice as on the
// host) and replaces the scatter "out[node] += contribution, tets in order" with a gather over
// the node's incident tets in ascending tet order. The sums therefore come out bit-identical to
// the reference's element loops while needing no atomics.
#pragma once

#include <type_traits>

#include "ns_common.cuh"

namespace cfsa {

// ------------------------------------------------------------------------------------------
// Geometry: Mesh::computeGeometry volume and Mesh::computeShapeFunctionGradients
// (src/Mesh/Mesh.cpp:455, 590-614).
__global__ void k_geometry(int nt, const double *__restrict__ xyz, const int *__restrict__ tnode,
                           double *__restrict__ vol, double *__restrict__ grad) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double P[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int v = tnode[(size_t)a * nt + t];
#pragma unroll
    for (int c = 0; c < 3; ++c) P[a][c] = xyz[3 * (size_t)v + c];
  }
  auto sub = [](const double *x, const double *y, double *o) {
    o[0] = x[0] - y[0];
    o[1] = x[1] - y[1];
    o[2] = x[2] - y[2];
  };
  auto cross = [](const double *x, const double *y, double *o) {
    o[0] = x[1] * y[2] - x[2] * y[1];
    o[1] = x[2] * y[0] - x[0] * y[2];
    o[2] = x[0] * y[1] - x[1] * y[0];
  };
  auto dot = [](const double *x, const double *y) { return (x[0] * y[0] + x[1] * y[1]) + x[2] * y[2]; };
  double ba[3], ca[3], da[3], cr[3];
  sub(P[1], P[0], ba);
  sub(P[2], P[0], ca);
  sub(P[3], P[0], da);
  cross(ba, ca, cr);
  vol[t] = fabs(dot(cr, da) / 6.0);
  double e23[3];
  cross(ca, da, e23);
  const double inv6v = 1.0 / dot(ba, e23);
  double g[4][3], x1[3], x2[3];
  sub(P[3], P[1], x1);
  sub(P[2], P[1], x2);
  cross(x1, x2, g[0]);
  cross(ca, da, g[1]);  // (p2-p0) x (p3-p0)
  sub(P[3], P[0], x1);
  sub(P[1], P[0], x2);
  cross(x1, x2, g[2]);
  cross(ba, ca, g[3]);  // (p1-p0) x (p2-p0)
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) grad[(size_t)(3 * a + c) * nt + t] = inv6v * g[a][c];
}

// ------------------------------------------------------------------------------------------
// Sparsity patterns. One warp per row: candidates are the nodes of the row's incident tets
// (all 10 for the P2 pattern, the 4 vertices for the P1 pattern); duplicates are dropped and
// the survivors are ranked to produce ascending column indices.
constexpr int kPatternCap = 1024;  // candidates per row held in shared memory

template <bool P2>
__global__ void k_pattern(int nrows, int nt, const int *__restrict__ adj_ptr,
                          const int *__restrict__ adj, const int *__restrict__ tnode,
                          int *__restrict__ counts, const int *__restrict__ rp,
                          int *__restrict__ ci, int *__restrict__ err) {
  __shared__ int cand[kBlock / 32][kPatternCap];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row = blockIdx.x * (blockDim.x >> 5) + warp;
  if (row >= nrows) return;
  const int nloc = P2 ? 10 : 4;
  const int beg = adj_ptr[row], end = adj_ptr[row + 1];
  const int ncand = (end - beg) * nloc;
  if (ncand > kPatternCap) {
    if (lane == 0) atomicExch(err, row + 1);
    return;
  }
  int *cw = cand[warp];
  for (int q = lane; q < ncand; q += 32) {
    const int e = adj[beg + q / nloc] >> 4;  // tet id
    cw[q] = tnode[(size_t)(q % nloc) * nt + e];
  }
  __syncwarp();
  // pass 1: bit j of `dup` marks candidate lane + 32*j as a repeat of an earlier candidate
  unsigned int dup = 0u;
  for (int j = 0; j * 32 < ncand; ++j) {
    const int q = j * 32 + lane;
    if (q < ncand) {
      const int c = cw[q];
      for (int k = 0; k < q; ++k)
        if (cw[k] == c) {
          dup |= 1u << j;
          break;
        }
    }
  }
  __syncwarp();
  // pass 2: repeats are replaced by INT_MAX so that only distinct values remain comparable
  for (int j = 0; j * 32 < ncand; ++j) {
    const int q = j * 32 + lane;
    if (q < ncand && ((dup >> j) & 1u)) cw[q] = 0x7fffffff;
  }
  __syncwarp();
  int nuniq = 0;
  for (int j = 0; j * 32 < ncand; ++j) {
    const int q = j * 32 + lane;
    const bool first = (q < ncand) && !((dup >> j) & 1u);
    if (counts == nullptr && first) {
      const int c = cw[q];
      int rank = 0;  // number of distinct candidates smaller than c
      for (int k = 0; k < ncand; ++k) rank += (cw[k] < c);
      ci[rp[row] + rank] = c;
    }
    nuniq += __popc(__ballot_sync(0xffffffffu, first));
  }
  if (counts != nullptr && lane == 0) counts[row] = nuniq;
}

__device__ __forceinline__ int find_col(const int *__restrict__ ci, int beg, int end, int c) {
  int lo = beg, hi = end - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (ci[mid] < c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void node_grad(const double *__restrict__ grad, int nt, int t, int l,
                                          double g[3]) {
  // P1: grad phi_l; P2 edge node: grad phi_a + grad phi_b (NavierStokes.cpp:194)
  constexpr int ev[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  if (l < 4) {
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c] = grad[(size_t)(3 * l + c) * nt + t];
  } else {
    const int a = ev[l - 4][0], b = ev[l - 4][1];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      g[c] = grad[(size_t)(3 * a + c) * nt + t] + grad[(size_t)(3 * b + c) * nt + t];
  }
}

// P2 mass and stiffness, one thread per row, incident tets in ascending order
// (buildMassMatrix NavierStokes.cpp:247-285, buildStiffnessMatrix :159-218).
__global__ void k_assemble_p2(int nrows, int nt, double density, double mu,
                              const int *__restrict__ adj_ptr, const int *__restrict__ adj,
                              const int *__restrict__ tnode, const double *__restrict__ vol,
                              const double *__restrict__ grad, const int *__restrict__ rp,
                              const int *__restrict__ ci, double *__restrict__ Mv,
                              double *__restrict__ Kv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int beg = rp[row], end = rp[row + 1];
  for (int k = beg; k < end; ++k) {
    Mv[k] = 0.0;
    Kv[k] = 0.0;
  }
  for (int q = adj_ptr[row]; q < adj_ptr[row + 1]; ++q) {
    const int t = adj[q] >> 4, li = adj[q] & 15;
    const double V = vol[t];
    const double mass = density * V;
    double gi[3];
    node_grad(grad, nt, t, li, gi);
    for (int lj = 0; lj < 10; ++lj) {
      const int col = tnode[(size_t)lj * nt + t];
      const int slot = find_col(ci, beg, end, col);
      double m;
      if (li < 4 && lj < 4)
        m = (li == lj) ? mass / 10.0 : mass / 20.0;
      else if (li >= 4 && lj >= 4)
        m = (li == lj) ? mass / 15.0 : mass / 60.0;
      else
        m = mass / 30.0;
      double gj[3];
      node_grad(grad, nt, t, lj, gj);
      const double d = (gi[0] * gj[0] + gi[1] * gj[1]) + gi[2] * gj[2];
      Mv[slot] += m;
      Kv[slot] += mu * V * d;
    }
  }
}

// P1 gradient and Poisson matrices (buildGradientMatrices NavierStokes.cpp:91-120,
// buildPoissonMatrix :331-349). G is stored as three consecutive nnz1 blocks (x, y, z).
__global__ void k_assemble_p1(int nrows, int nt, int64_t nnz1, const int *__restrict__ adj_ptr,
                              const int *__restrict__ adj, const int *__restrict__ tnode,
                              const double *__restrict__ vol, const double *__restrict__ grad,
                              const int *__restrict__ rp, const int *__restrict__ ci,
                              double *__restrict__ Gv, double *__restrict__ Lv) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int beg = rp[row], end = rp[row + 1];
  for (int k = beg; k < end; ++k) {
    Gv[k] = 0.0;
    Gv[nnz1 + k] = 0.0;
    Gv[2 * nnz1 + k] = 0.0;
    Lv[k] = 0.0;
  }
  for (int q = adj_ptr[row]; q < adj_ptr[row + 1]; ++q) {
    const int t = adj[q] >> 4, li = adj[q] & 15;
    if (li >= 4) continue;
    const double V = vol[t];
    double gi[3];
    node_grad(grad, nt, t, li, gi);
    for (int lj = 0; lj < 4; ++lj) {
      const int col = tnode[(size_t)lj * nt + t];
      const int slot = find_col(ci, beg, end, col);
      double gj[3];
      node_grad(grad, nt, t, lj, gj);
      const double contrib = V / 4.0;
      Gv[slot] += contrib * gj[0];
      Gv[nnz1 + slot] += contrib * gj[1];
      Gv[2 * nnz1 + slot] += contrib * gj[2];
      Lv[slot] += V * ((gi[0] * gj[0] + gi[1] * gj[1]) + gi[2] * gj[2]);
    }
  }
}

// 1/rowsum(M) with the reference's 1e-14 guard (NavierStokes.cpp:293-306).
__global__ void k_lumped_mass(int n, const int *__restrict__ rp, const double *__restrict__ Mv,
                              double *__restrict__ invm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) s += Mv[k] * 1.0;
  invm[i] = (fabs(s) > 1e-14) ? 1.0 / s : 1.0;
}

__global__ void k_diag_pos(int n, const int *__restrict__ rp, const int *__restrict__ ci,
                           int *__restrict__ dpos) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int pos = -1;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) pos = k;
  dpos[i] = pos;
}

// SELL layout: column indices and the CSR slot -> SELL position map.
__global__ void k_sell_fill(int nrows_pad, const int *__restrict__ sptr, const int *__restrict__ perm,
                            const int *__restrict__ len, const int *__restrict__ rp,
                            const int *__restrict__ ci, int *__restrict__ scol,
                            int *__restrict__ posmap) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrows_pad) return;
  const int i = perm[r];
  if (i < 0) return;
  const int base = sptr[r >> 5] + (r & 31);
  const int b = rp[i];
  for (int k = 0; k < len[r]; ++k) {
    scol[base + k * kSellC] = ci[b + k];
    posmap[b + k] = base + k * kSellC;
  }
}

__global__ void k_scatter_vals(int64_t nnz, const int *__restrict__ posmap,
                               const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) dst[posmap[k]] = src[k];
}

// Momentum operator A = M/dt + K + 1e10 on Inlet/Wall diagonals (NavierStokes.cpp:460-495).
__global__ void k_momentum_diag(int n, double dt, const int *__restrict__ dpos,
                                const double *__restrict__ Mv, const double *__restrict__ Kv,
                                const signed char *__restrict__ bc, double *__restrict__ diagA,
                                double *__restrict__ invA) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = dpos[i];
  double d = Mv[k] / dt + Kv[k];
  if (bc[i] == BC_INLET || bc[i] == BC_WALL) d += kMomentumPenalty;
  diagA[i] = d;
  invA[i] = (d != 0.0) ? 1.0 / d : 1.0;
}

// Momentum operator in SELL layout: right-preconditioned At = A * diag(invA) for BiCGSTAB
// (scale != 0) or A itself for CG; and M in SELL.
__global__ void k_momentum_sell(int64_t nnz, double dt, const int *__restrict__ posmap,
                                const int *__restrict__ rows, const int *__restrict__ ci,
                                const double *__restrict__ Mv, const double *__restrict__ Kv,
                                const signed char *__restrict__ bc,
                                const double *__restrict__ invA, double *__restrict__ At,
                                double *__restrict__ Ms, int scale) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = rows[k], j = ci[k];
  double a = Mv[k] / dt + Kv[k];
  if (i == j && (bc[i] == BC_INLET || bc[i] == BC_WALL)) a += kMomentumPenalty;
  const int pos = posmap[k];
  At[pos] = scale ? a * invA[j] : a;
  Ms[pos] = Mv[k];
}

__global__ void k_row_of_slot(int n, const int *__restrict__ rp, int *__restrict__ rows) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) rows[k] = i;
}

// Poisson operator with the outlet / reference penalty (NavierStokes.cpp:604-626) in SELL
// layout: Ls = Lbc (for CG), Lt = Lbc * diag(invL) (for BiCGSTAB); diagonal inverse invL.
// outlet_type -1 adds no penalty (the raw operator of solvePressureBiCGSTAB, :773-802).
__global__ void k_poisson_diag(int n, int outlet_type, int ref_node, const int *__restrict__ dpos,
                               const double *__restrict__ Lv, const signed char *__restrict__ bc,
                               double *__restrict__ diagL, double *__restrict__ invL) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double d = Lv[dpos[i]];
  if ((outlet_type == 1 && i == ref_node) || (outlet_type == 0 && bc[i] == BC_OUTLET))
    d += kPoissonPenalty;
  diagL[i] = d;
  invL[i] = (d != 0.0) ? 1.0 / d : 1.0;
}

__global__ void k_poisson_sell(int64_t nnz, int outlet_type, int ref_node,
                               const int *__restrict__ posmap, const int *__restrict__ rows,
                               const int *__restrict__ ci, const double *__restrict__ Lv,
                               const signed char *__restrict__ bc,
                               const double *__restrict__ invL, double *__restrict__ Ls,
                               double *__restrict__ Lt) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = rows[k], j = ci[k];
  double a = Lv[k];
  if (i == j && ((outlet_type == 1 && i == ref_node) || (outlet_type == 0 && bc[i] == BC_OUTLET)))
    a += kPoissonPenalty;
  const int pos = posmap[k];
  if (Ls) Ls[pos] = a;
  Lt[pos] = a * invL[j];
}

// ------------------------------------------------------------------------------------------
// Per-tet convection vector c_t = grad(u) * u_mean over P1 vertex velocities
// (computeAdvectionRHS NavierStokes.cpp:550-567).
__global__ void k_tet_conv(int nt, int64_t n2, const int *__restrict__ tnode,
                           const double *__restrict__ grad, const double *__restrict__ u,
                           double *__restrict__ ct, const DevStatus *__restrict__ st) {
  if (st->halt) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double uv[4][3];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int v = tnode[(size_t)a * nt + t];
#pragma unroll
    for (int c = 0; c < 3; ++c) uv[a][c] = u[c * n2 + v];
  }
  double ue[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[c] = ue[c] + 0.25 * uv[a][c];
  double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double g[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) g[b] = grad[(size_t)(3 * j + b) * nt + t];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) gu[a][b] += uv[j][a] * g[b];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a)
    ct[(size_t)a * nt + t] = (gu[a][0] * ue[0] + gu[a][1] * ue[1]) + gu[a][2] * ue[2];
}

// Per-tet divergence tr(grad u) over P1 vertex velocities (computeDivergence
// NavierStokes.cpp:684-693).
__global__ void k_tet_div(int nt, int64_t n2, const int *__restrict__ tnode,
                          const double *__restrict__ grad, const double *__restrict__ u,
                          double *__restrict__ divt, const DevStatus *__restrict__ st) {
  if (st && st->halt) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double d[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int v = tnode[(size_t)j * nt + t];
#pragma unroll
    for (int a = 0; a < 3; ++a) d[a] += u[a * n2 + v] * grad[(size_t)(3 * j + a) * nt + t];
  }
  divt[t] = (d[0] + d[1]) + d[2];
}

// Convection gather: conv_i = -sum_t w_t c_t, w = V/4 (vertex) or V/24 (edge node)
// (NavierStokes.cpp:571-580), tets ascending.
__device__ __forceinline__ void gather_conv(int i, int nt, const int *__restrict__ adj_ptr,
                                            const int *__restrict__ adj,
                                            const double *__restrict__ vol,
                                            const double *__restrict__ ct, double acc[3]) {
  acc[0] = acc[1] = acc[2] = 0.0;
  for (int q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
    const int t = adj[q] >> 4, l = adj[q] & 15;
    const double w = (l < 4) ? vol[t] / 4.0 : vol[t] / 24.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = acc[c] - w * ct[(size_t)c * nt + t];
  }
}

// Divergence gather onto P1 vertices: div_i = sum_t (V/4) d_t (NavierStokes.cpp:696-698).
__device__ __forceinline__ double gather_div(int i, const int *__restrict__ adj_ptr,
                                             const int *__restrict__ adj,
                                             const double *__restrict__ vol,
                                             const double *__restrict__ divt) {
  double s = 0.0;
  for (int q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
    const int t = adj[q] >> 4;
    s += (vol[t] / 4.0) * divt[t];
  }
  return s;
}

__global__ void k_gather_conv(int n, int nt, const int *__restrict__ adj_ptr,
                              const int *__restrict__ adj, const double *__restrict__ vol,
                              const double *__restrict__ ct, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double acc[3];
  gather_conv(i, nt, adj_ptr, adj, vol, ct, acc);
  for (int c = 0; c < 3; ++c) out[(size_t)c * n + i] = acc[c];
}

__global__ void k_gather_div(int nv, const int *__restrict__ adj_ptr, const int *__restrict__ adj,
                             const double *__restrict__ vol, const double *__restrict__ divt,
                             double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  out[i] = gather_div(i, adj_ptr, adj, vol, divt);
}

// One SELL row, NC right-hand sides sharing the matrix. Entries are fetched in chunks of U
// (all column indices and values of a chunk first, then the U*NC gathers) so that many loads are
// in flight per thread. The last len % U entries form one predicated chunk, so a row costs
// ceil(len / U) dependent round trips (index and value, then gather) instead of one per leftover
// entry: 82% of the P2 momentum rows have len % 4 == 3. The products are still accumulated in
// ascending column order, so the result is bit-identical to the sequential CSR row sum. Matrix
// entries are streamed once per product (evict-first), the gathered vector stays cacheable.
template <int NC, int U = 8, int MASK = (1 << NC) - 1>
__device__ __forceinline__ void sell_spmv_row(const SellView &S, const double *__restrict__ val,
                                              const double *__restrict__ x, int64_t n, int r,
                                              double acc[NC]) {
  const int base = S.sptr[r >> 5] + (r & 31), len = S.len[r];
#pragma unroll
  for (int c = 0; c < NC; ++c) acc[c] = 0.0;
  int k = 0;
  for (; k + U <= len; k += U) {
    int j[U];
    double a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int pos = base + (k + u) * kSellC;
      j[u] = __ldcs(S.col + pos);
      a[u] = __ldcs(val + pos);
    }
    double xv[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if ((MASK >> c) & 1) xv[u][c] = __ldg(x + c * n + j[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if ((MASK >> c) & 1) acc[c] += a[u] * xv[u][c];
  }
  if (k < len) {  // the last len % U entries as one predicated chunk: one memory round trip
    int j[U];
    double a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int pos = base + (k + u) * kSellC;
      const bool in = k + u < len;
      j[u] = in ? __ldcs(S.col + pos) : 0;
      a[u] = in ? __ldcs(val + pos) : 0.0;
    }
    double xv[U][NC];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if ((MASK >> c) & 1) xv[u][c] = (k + u < len) ? __ldg(x + c * n + j[u]) : 0.0;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < NC; ++c)
        if (((MASK >> c) & 1) && k + u < len) acc[c] += a[u] * xv[u][c];
  }
}

// Compile-time variants of a product loop for the right-hand sides still active in `mask`: f is
// called with std::integral_constant<int, MASK> for every non-empty subset of three components
// (the penalty-dominated streamwise component converges first), so that a converged component
// costs no gathers and each variant's whole loop is compiled for its mask (a dispatch per row
// inside the loop measured 6% slower on the FP32 product). Active components get the same sums in
// the same order in every variant.
template <int NC, class F>
__device__ __forceinline__ void with_mask(int mask, F &&f) {
  if constexpr (NC == 3) {
    switch (mask) {
      case 1: f(std::integral_constant<int, 1>{}); break;
      case 2: f(std::integral_constant<int, 2>{}); break;
      case 4: f(std::integral_constant<int, 4>{}); break;
      case 3: f(std::integral_constant<int, 3>{}); break;
      case 5: f(std::integral_constant<int, 5>{}); break;
      case 6: f(std::integral_constant<int, 6>{}); break;
      default: f(std::integral_constant<int, 7>{}); break;
    }
  } else {
    f(std::integral_constant<int, (1 << NC) - 1>{});
  }
}

// Entries per chunk of a row in the FP64 Krylov products (4 measured faster than 8 on the
// 1M-tet momentum operator: 135.8 vs 142.9 us; 12 or 16 with fewer threads per SM were slower).
constexpr int kU64 = 4;

// Row i of the transposed P1 operators G_a^T (a = 0..2) applied to x_a. The P1 pattern is
// structurally symmetric: the entry (i, j) of G_a^T is G_a(j, i), stored at the transposed slot
// tpos[k] of the entry k = (i, j); entries are summed in ascending column order.
__device__ __forceinline__ void gt_row3(int i, const int *__restrict__ rp, const int *__restrict__ ci,
                                        const int *__restrict__ tpos, const double *__restrict__ Gv,
                                        int64_t nnz1, const double *__restrict__ x0,
                                        const double *__restrict__ x1,
                                        const double *__restrict__ x2, double out[3]) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int k = rp[i]; k < rp[i + 1]; ++k) {
    const int j = ci[k], t = tpos[k];
    s0 += Gv[t] * x0[j];
    s1 += Gv[nnz1 + t] * x1[j];
    s2 += Gv[2 * nnz1 + t] * x2[j];
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
}

// ------------------------------------------------------------------------------------------
// Momentum right-hand side (NavierStokes.cpp:429-495) for the three components, fused with the
// initialisation of the batched BiCGSTAB (x0 = 0, r = r0 = b, p = v = 0).
struct MomentumRhsArgs {
  SellView S;
  const double *Ms;  // M in SELL layout
  CsrView G;         // P1 pattern
  const double *Gv;  // [3][nnz1]
  int64_t nnz1;
  const int *adj_ptr, *adj;
  const double *vol, *ct;
  const signed char *bc;
  const double *inlet;  // [3][N2]
  const double *u, *p;
  double dt, tol;
  int n, nv, nt, maxit;
  double *b, *x, *r, *r0, *pk, *v;
  const double *cw;  // convergence-norm weights (diag(A)^-1), nullptr: unscaled ||r||
  BicgState *bs;
  DevStatus *st;
  Reduce red;
  // Adjoint mode (adj_mu != nullptr): b holds the adjoint right-hand side on entry and its P1
  // rows receive -G_a^T mu / dt (transposed slots tpos); the forward terms are not formed.
  const double *adj_mu;
  const int *tpos;
};

__global__ void k_momentum_rhs(MomentumRhsArgs A) {
  if (A.st->halt) return;
  // one resident wave; each CTA visits 256-position blocks blockIdx.x, blockIdx.x + gridDim.x, ...
  // (the reduction tree is that of one CTA per block, with one ticket per CTA instead of per block)
  __shared__ WarpSums<6> S;
  const int nblk = (A.S.nrows_pad + kBlock - 1) / kBlock;
  int slot = 0;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x, ++slot) {
    const int r = blk * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
    if (i >= 0) {
      const int64_t n = A.n;
      const double w = A.cw ? A.cw[i] : 1.0;
      double b[3];
      if (A.adj_mu) {
#pragma unroll
        for (int c = 0; c < 3; ++c) b[c] = A.b[c * n + i];
        if (i < A.nv) {
          double g[3];
          gt_row3(i, A.G.rp, A.G.ci, A.tpos, A.Gv, A.nnz1, A.adj_mu, A.adj_mu, A.adj_mu, g);
#pragma unroll
          for (int c = 0; c < 3; ++c) b[c] = b[c] - g[c] / A.dt;
        }
      } else {
      double mu[3];
      sell_spmv_row<3>(A.S, A.Ms, A.u, n, r, mu);
#pragma unroll
      for (int c = 0; c < 3; ++c) b[c] = 0.0 + mu[c] / A.dt;
      if (i < A.nv) {
        double gp[3] = {0.0, 0.0, 0.0};
        for (int k = A.G.rp[i]; k < A.G.rp[i + 1]; ++k) {
          const double pj = A.p[A.G.ci[k]];
          gp[0] += A.Gv[k] * pj;
          gp[1] += A.Gv[A.nnz1 + k] * pj;
          gp[2] += A.Gv[2 * A.nnz1 + k] * pj;
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) b[c] -= gp[c];
      }
      double conv[3];
      gather_conv(i, A.nt, A.adj_ptr, A.adj, A.vol, A.ct, conv);
#pragma unroll
      for (int c = 0; c < 3; ++c) b[c] += conv[c];
      const int bcv = A.bc[i];
      if (bcv == BC_INLET || bcv == BC_WALL) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double up = (bcv == BC_INLET) ? A.inlet[c * n + i] : 0.0;
          b[c] += kMomentumPenalty * up;
        }
      }
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t o = c * n + i;
        A.b[o] = b[c];
        A.x[o] = 0.0;
        A.r[o] = b[c];
        A.r0[o] = b[c];
        A.pk[o] = 0.0;
        A.v[o] = 0.0;
        part[c] = b[c] * b[c];
        part[3 + c] = (b[c] * b[c]) * w;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    BicgState *s = A.bs;
    s->active = 0;
    s->restart = 0;
    s->maxit = A.maxit;
    s->ncomp = 3;
    for (int c = 0; c < 3; ++c) {
      s->bnorm2[c] = tot[3 + c];  // convergence norm of b
      s->r0norm2[c] = tot[c];     // r0 . r0 (restart threshold)
      s->rnorm2[c] = tot[3 + c];
      s->tol2[c] = A.tol * A.tol * tot[3 + c];
      s->rho[c] = tot[c];  // r0 . r with r = r0 = b
      s->alpha[c] = s->omega[c] = 1.0;
      s->beta[c] = 0.0;
      s->iters[c] = 0;
      if (isnan(tot[c]) || isnan(tot[3 + c])) {
        s->status[c] = KS_BREAKDOWN;
      } else if (tot[3 + c] == 0.0 || tot[3 + c] <= s->tol2[c]) {
        s->status[c] = KS_CONVERGED;
      } else {
        s->status[c] = KS_RUNNING;
        s->active |= 1 << c;
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// Batched right-Jacobi-preconditioned BiCGSTAB on At = A diag(1/diag(A)); x is kept in the
// original variables (x += alpha*D^-1 p + omega*D^-1 s). NC right-hand sides share At.
struct BicgArgs {
  SellView S;
  const double *At;
  const double *diagA;  // diag(A), for the restart residual
  const double *invA;
  const double *b;
  double *x, *r, *r0, *pk, *v, *s, *t;
  int n;
  BicgState *bs;
  Reduce red;
  cudaGraphConditionalHandle cond;
  int use_cond;
  DevStatus *st;  // launch counters
  int slot;       // 0 momentum, 1 pressure
  const double *cw;  // convergence-norm weights, nullptr: unscaled ||r||
  double tol;        // relative tolerance (read by the momentum CG's initialisation)
};

// K1: p = r + beta (p - omega v); on restart: r = b - A x, r0 = r, p = r, rho = |r|^2.
template <int NC>
__global__ void k_bicg_p(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int restart = A.bs->restart;
  // the scalars are read once, before any store the compiler could not prove disjoint from them
  double beta_c[NC], omega_c[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) beta_c[c] = A.bs->beta[c], omega_c[c] = A.bs->omega[c];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
  const int64_t n = A.n;
  double part[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) part[c] = 0.0;
  if (i >= 0) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      const int64_t o = c * n + i;
      if ((restart >> c) & 1) {
        const int base = A.S.sptr[r >> 5] + (r & 31), len = A.S.len[r];
        double acc = 0.0;
        for (int k = 0; k < len; ++k) {
          const int pos = base + k * kSellC;
          const int j = A.S.col[pos];
          acc += A.At[pos] * (A.diagA[j] * A.x[c * n + j]);
        }
        const double ri = A.b[o] - acc;
        A.r[o] = ri;
        A.r0[o] = ri;
        A.pk[o] = ri;
        part[c] = ri * ri;
      } else {
        A.pk[o] = A.r[o] + beta_c[c] * (A.pk[o] - omega_c[c] * A.v[o]);
      }
    }
  }
  if (restart) {
    double tot[NC];
    if (grid_reduce<NC>(part, A.red, tot) && threadIdx.x == 0) {
      for (int c = 0; c < NC; ++c)
        if ((restart >> c) & 1) {
          A.bs->rho[c] = tot[c];
          A.bs->r0norm2[c] = tot[c];
        }
      A.bs->restart = 0;
    }
  }
}

// K2: v = At p, alpha = rho / (r0 . v)
template <int NC>
__global__ void __launch_bounds__(kRunThreads, 1) k_bicg_v(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<NC>(active, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) part[c] = 0.0;
      if (i >= 0) {
        double acc[NC];
        sell_spmv_row<NC, kU64, MASK>(A.S, A.At, A.pk, n, r, acc);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if (!((MASK >> c) & 1)) continue;
          const int64_t o = c * n + i;
          A.v[o] = acc[c];
          part[c] = A.r0[o] * acc[c];
        }
      }
      slice_partial<NC>(part, A.S, sl);
    }
  });
  double tot[NC];
  if (grid_reduce_runs<NC>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      if (tot[c] == 0.0) {
        A.bs->status[c] = KS_BREAKDOWN;
        A.bs->active &= ~(1 << c);
      } else {
        A.bs->alpha[c] = A.bs->rho[c] / tot[c];
      }
    }
  }
}

// K3: s = r - alpha v
template <int NC>
__global__ void k_bicg_s(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  double alpha[NC], rv[NC], vv[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    alpha[c] = A.bs->alpha[c];
    if ((active >> c) & 1) rv[c] = A.r[c * n + i], vv[c] = A.v[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < NC; ++c)
    if ((active >> c) & 1) A.s[c * n + i] = rv[c] - alpha[c] * vv[c];
}

// K4: t = At s, omega = (t . s) / (t . t) (0 when t . t == 0)
template <int NC>
__global__ void __launch_bounds__(kRunThreads, 1) k_bicg_t(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<NC>(active, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[2 * NC];
#pragma unroll
      for (int c = 0; c < 2 * NC; ++c) part[c] = 0.0;
      if (i >= 0) {
        double acc[NC];
        sell_spmv_row<NC, kU64, MASK>(A.S, A.At, A.s, n, r, acc);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if (!((MASK >> c) & 1)) continue;
          const int64_t o = c * n + i;
          A.t[o] = acc[c];
          part[c] = acc[c] * acc[c];
          part[NC + c] = acc[c] * A.s[o];
        }
      }
      slice_partial<2 * NC>(part, A.S, sl);
    }
  });
  double tot[2 * NC];
  if (grid_reduce_runs<2 * NC>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      A.bs->omega[c] = (tot[c] > 0.0) ? tot[NC + c] / tot[c] : 0.0;
    }
  }
}

// K5: x += alpha D^-1 p + omega D^-1 s, r = s - omega t; convergence test and next beta.
template <int NC>
__global__ void k_bicg_xr(BicgArgs A) {
  const int active = A.bs->active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[A.slot] += 1;
  if (!active) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  __shared__ WarpSums<2 * NC> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  const int64_t n = A.n;
  double alpha_c[NC], omega_c[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) alpha_c[c] = A.bs->alpha[c], omega_c[c] = A.bs->omega[c];
  int slot = 0;
  for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++slot) {
    const int i = b * kBlock + threadIdx.x;
    double part[2 * NC];
#pragma unroll
    for (int c = 0; c < 2 * NC; ++c) part[c] = 0.0;
    if (i < A.n) {
      const double dinv = A.invA[i];
      const double w = A.cw ? A.cw[i] : 1.0;
      double pv[NC], sv[NC], tv[NC], xv[NC], r0v[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (!((active >> c) & 1)) continue;
        const int64_t o = c * n + i;
        pv[c] = A.pk[o], sv[c] = A.s[o], tv[c] = A.t[o], xv[c] = A.x[o], r0v[c] = A.r0[o];
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (!((active >> c) & 1)) continue;
        const int64_t o = c * n + i;
        const double y = dinv * pv[c];
        const double z = dinv * sv[c];
        A.x[o] = xv[c] + (alpha_c[c] * y + omega_c[c] * z);
        const double ri = sv[c] - omega_c[c] * tv[c];
        A.r[o] = ri;
        part[c] = (ri * ri) * w;
        part[NC + c] = r0v[c] * ri;
      }
    }
    warp_partial<2 * NC>(part, S, slot);
  }
  double tot[2 * NC];
  if (grid_reduce_strided<2 * NC>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    BicgState *s = A.bs;
    const double eps = 2.220446049250313e-16;
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      s->iters[c] += 1;
      s->rnorm2[c] = tot[c];
      if (isnan(tot[c]) || isnan(tot[NC + c])) {
        s->status[c] = KS_BREAKDOWN;
        s->active &= ~(1 << c);
      } else if (tot[c] <= s->tol2[c]) {
        s->status[c] = KS_CONVERGED;
        s->active &= ~(1 << c);
      } else if (s->iters[c] >= s->maxit) {
        s->status[c] = KS_MAXIT;
        s->active &= ~(1 << c);
      } else if (s->omega[c] == 0.0) {
        s->status[c] = KS_BREAKDOWN;
        s->active &= ~(1 << c);
      } else {
        const double rho_new = tot[NC + c];
        if (fabs(rho_new) < eps * eps * s->r0norm2[c]) {
          s->restart |= 1 << c;
        } else {
          s->beta[c] = (rho_new / s->rho[c]) * (s->alpha[c] / s->omega[c]);
          s->rho[c] = rho_new;
        }
      }
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, s->active ? 1u : 0u);
  }
}

// ------------------------------------------------------------------------------------------
// Batched Jacobi-preconditioned CG for the momentum system (selectable; the reference solves it
// with BiCGSTAB, NavierStokes.cpp:498-515). A = M/dt + K + 1e10 I_D is symmetric positive
// definite (the convection term is explicit), so CG solves the same system with one product per
// iteration instead of two. With this method the SELL values hold A itself, not A D^-1. Each
// component keeps its own scalars and stops on its own, as in the BiCGSTAB batch:
//   G0: z = D^-1 b, p = z, absnew = b.z; ||b|| in the convergence norm (r.r, or r.z)
//   G1: q = A p, alpha = absnew / (p.q)
//   G2: x += alpha p, r -= alpha q, z = D^-1 r; convergence test; beta = r.z / absnew
//   G3: p = z + beta p
// z is recomputed from r where it is needed (the same product, one stored vector less). The
// reductions of G0 and G2 run over natural 256-position blocks, the one of G1 over the SELL runs.

// G0, after k_momentum_rhs has written b, x = 0 and r = b.
template <int NC>
__global__ void k_mcg_init(BicgArgs A) {
  if (A.st && A.st->halt) return;
  __shared__ WarpSums<2 * NC> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  const int64_t n = A.n;
  int slot = 0;
  for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++slot) {
    const int i = b * kBlock + threadIdx.x;
    double part[2 * NC];
#pragma unroll
    for (int c = 0; c < 2 * NC; ++c) part[c] = 0.0;
    if (i < A.n) {
      const double dinv = A.invA[i];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const int64_t o = c * n + i;
        const double bi = A.b[o];
        const double zi = dinv * bi;
        A.pk[o] = zi;
        part[c] = bi * bi;
        part[NC + c] = bi * zi;
      }
    }
    warp_partial<2 * NC>(part, S, slot);
  }
  double tot[2 * NC];
  if (grid_reduce_strided<2 * NC>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    BicgState *s = A.bs;
    s->active = 0;
    s->restart = 0;
    s->ncomp = NC;
    for (int c = 0; c < NC; ++c) {
      const double bn = A.cw ? tot[NC + c] : tot[c];
      s->bnorm2[c] = bn;
      s->rnorm2[c] = bn;
      s->tol2[c] = A.tol * A.tol * bn;
      s->rho[c] = tot[NC + c];
      s->alpha[c] = 0.0;
      s->beta[c] = 0.0;
      s->iters[c] = 0;
      if (isnan(bn)) {
        s->status[c] = KS_BREAKDOWN;
      } else if (bn == 0.0 || bn <= s->tol2[c]) {
        s->status[c] = KS_CONVERGED;
      } else {
        s->status[c] = KS_RUNNING;
        s->active |= 1 << c;
      }
    }
  }
}

// G1: q = A p (into v), alpha = absnew / (p . q)
template <int NC>
__global__ void __launch_bounds__(kRunThreads, 1) k_mcg_q(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<NC>(active, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) part[c] = 0.0;
      if (i >= 0) {
        double acc[NC];
        sell_spmv_row<NC, kU64, MASK>(A.S, A.At, A.pk, n, r, acc);
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          if (!((MASK >> c) & 1)) continue;
          const int64_t o = c * n + i;
          A.v[o] = acc[c];
          part[c] = A.pk[o] * acc[c];
        }
      }
      slice_partial<NC>(part, A.S, sl);
    }
  });
  double tot[NC];
  if (grid_reduce_runs<NC>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      if (tot[c] == 0.0) {
        A.bs->status[c] = KS_BREAKDOWN;
        A.bs->active &= ~(1 << c);
      } else {
        A.bs->alpha[c] = A.bs->rho[c] / tot[c];
      }
    }
  }
}

// G2: x += alpha p, r -= alpha q, z = D^-1 r; r.r and r.z; convergence test and next beta.
template <int NC>
__global__ void k_mcg_xr(BicgArgs A) {
  const int active = A.bs->active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[A.slot] += 1;
  if (!active) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  __shared__ WarpSums<2 * NC> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  const int64_t n = A.n;
  double alpha_c[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) alpha_c[c] = A.bs->alpha[c];
  int slot = 0;
  for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++slot) {
    const int i = b * kBlock + threadIdx.x;
    double part[2 * NC];
#pragma unroll
    for (int c = 0; c < 2 * NC; ++c) part[c] = 0.0;
    if (i < A.n) {
      const double dinv = A.invA[i];
      double xv[NC], pv[NC], rv[NC], qv[NC];
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (!((active >> c) & 1)) continue;
        const int64_t o = c * n + i;
        xv[c] = A.x[o], pv[c] = A.pk[o], rv[c] = A.r[o], qv[c] = A.v[o];
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (!((active >> c) & 1)) continue;
        const int64_t o = c * n + i;
        A.x[o] = xv[c] + alpha_c[c] * pv[c];
        const double ri = rv[c] - alpha_c[c] * qv[c];
        A.r[o] = ri;
        const double zi = dinv * ri;
        part[c] = ri * ri;
        part[NC + c] = ri * zi;
      }
    }
    warp_partial<2 * NC>(part, S, slot);
  }
  double tot[2 * NC];
  if (grid_reduce_strided<2 * NC>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    BicgState *s = A.bs;
    for (int c = 0; c < NC; ++c) {
      if (!((active >> c) & 1)) continue;
      s->iters[c] += 1;
      const double rr = tot[c], rz = tot[NC + c];
      const double crit = A.cw ? rz : rr;
      s->rnorm2[c] = crit;
      if (isnan(rr) || isnan(rz)) {
        s->status[c] = KS_BREAKDOWN;
        s->active &= ~(1 << c);
      } else if (crit <= s->tol2[c]) {
        s->status[c] = KS_CONVERGED;
        s->active &= ~(1 << c);
      } else if (s->iters[c] >= s->maxit) {
        s->status[c] = KS_MAXIT;
        s->active &= ~(1 << c);
      } else {
        s->beta[c] = rz / s->rho[c];
        s->rho[c] = rz;
      }
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, s->active ? 1u : 0u);
  }
}

// G3: p = z + beta p with z = D^-1 r
template <int NC>
__global__ void k_mcg_p(BicgArgs A) {
  const int active = A.bs->active;
  if (!active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  const double dinv = A.invA[i];
  double beta[NC], rv[NC], pv[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) {
    beta[c] = A.bs->beta[c];
    if ((active >> c) & 1) rv[c] = A.r[c * n + i], pv[c] = A.pk[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < NC; ++c)
    if ((active >> c) & 1) A.pk[c * n + i] = dinv * rv[c] + beta[c] * pv[c];
}

// After a Krylov loop: record a failure and halt the rest of the batch (pisoStep returns false
// right after a failed solve, NavierStokes.cpp:387-398).
__global__ void k_check_bicg(const BicgState *__restrict__ bs, int ncomp, int slot, DevStatus *st) {
  if (st->halt) return;
  int code = 0, it = 0;
  for (int c = 0; c < ncomp; ++c) it = max(it, bs->iters[c]);
  st->iters[slot] += (unsigned long long)it;
  for (int c = 0; c < ncomp; ++c) {
    if (bs->status[c] == KS_MAXIT && code == 0) code = 1;
    if (bs->status[c] == KS_BREAKDOWN && code == 0) code = 2;
  }
  if (code) {
    st->code = code;
    st->halt = 1;
  }
}

__global__ void k_check_cg(const CgState *__restrict__ cs, DevStatus *st, const int *__restrict__ barrier_err) {
  if (st->halt) return;
  st->iters[1] += (unsigned long long)cs->iters;
  int code = 0;
  if (cs->status == KS_MAXIT) code = 1;
  if (cs->status == KS_BREAKDOWN) code = 2;
  if (barrier_err && *barrier_err) code = 4;  // persistent solve gave up waiting at a grid barrier
  if (code) {
    st->code = code;
    st->halt = 1;
  }
}

// ------------------------------------------------------------------------------------------
// Pressure Poisson right-hand side b = -div(u*)/dt + penalty * p_out on Dirichlet outlet nodes
// (NavierStokes.cpp:590-626), fused with the Krylov initialisation (CG or BiCGSTAB, x0 = 0).
struct PressureRhsArgs {
  const int *adj_ptr, *adj;
  const double *vol, *divt;
  const signed char *bc;
  const double *invL;
  double dt, tol, outlet_pressure;
  int nv, outlet_type, ref_node, maxit, krylov;  // krylov: 0 CG, 1 BiCGSTAB
  int scaled;  // convergence norm: 0 ||r||, 1 ||D^-1/2 r||
  double *b, *x, *r, *z_or_r0, *pk, *v;
  CgState *cs;
  BicgState *bs;
  DevStatus *st;
  Reduce red;
  // Adjoint mode (adj_q != nullptr): b = sum_a G_a^T q_a + adj_lpp (q_a = adj_q + a*nv).
  const double *adj_q, *adj_lpp;
  // Given right-hand side (given_b != nullptr): b = given_b, no divergence and no penalty term
  // (the raw Poisson solve of solvePressureBiCGSTAB).
  const double *given_b;
  CsrView G;
  const int *tpos;
  const double *Gv;
  int64_t nnz1;
};

__global__ void k_pressure_rhs(PressureRhsArgs A) {
  if (A.st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part[2] = {0.0, 0.0};
  if (i < A.nv) {
    double b;
    if (A.given_b) {
      b = A.given_b[i];
    } else if (A.adj_q) {
      double g[3];
      gt_row3(i, A.G.rp, A.G.ci, A.tpos, A.Gv, A.nnz1, A.adj_q, A.adj_q + A.nv,
              A.adj_q + 2 * (int64_t)A.nv, g);
      b = ((g[0] + g[1]) + g[2]) + A.adj_lpp[i];
    } else {
      const double d = gather_div(i, A.adj_ptr, A.adj, A.vol, A.divt);
      b = -d / A.dt;
      if (A.outlet_type == 1) {
        if (i == A.ref_node) b += kPoissonPenalty * 0.0;
      } else if (A.outlet_type == 0) {
        if (A.bc[i] == BC_OUTLET) b += kPoissonPenalty * A.outlet_pressure;
      }
    }
    A.b[i] = b;
    A.x[i] = 0.0;
    A.r[i] = b;
    const double z = A.invL[i] * b;
    if (A.krylov == 0) {
      A.z_or_r0[i] = z;
      A.pk[i] = z;
    } else {
      A.z_or_r0[i] = b;
      A.pk[i] = 0.0;
      A.v[i] = 0.0;
    }
    part[0] = b * b;
    // scaled convergence norm of b in the form each method's iterations use: CG r.z, BiCGSTAB (r.r) w
    part[1] = (A.krylov == 0) ? b * z : (b * b) * A.invL[i];
  }
  double tot[2];
  if (grid_reduce<2>(part, A.red, tot) && threadIdx.x == 0) {
    const double crit = A.scaled ? tot[1] : tot[0];  // convergence norm of b
    const double tol2 = A.tol * A.tol * crit;
    const bool bad = isnan(tot[0]) || isnan(tot[1]);
    const bool done = bad || (crit == 0.0 || crit <= tol2);
    const int final_status = bad ? KS_BREAKDOWN : KS_CONVERGED;
    if (A.krylov == 0) {
      CgState *c = A.cs;
      c->bnorm2 = crit;
      c->rnorm2 = crit;
      c->tol2 = tol2;
      c->absnew = tot[1];
      c->bb = tot[0];
      c->iters = 0;
      c->maxit = A.maxit;
      c->status = done ? final_status : KS_RUNNING;
      c->active = done ? 0 : 1;
    } else {
      BicgState *s = A.bs;
      s->ncomp = 1;
      s->maxit = A.maxit;
      s->restart = 0;
      s->bnorm2[0] = s->rnorm2[0] = crit;
      s->r0norm2[0] = tot[0];
      s->tol2[0] = tol2;
      s->rho[0] = tot[0];  // r0 . r with r = r0 = b
      s->alpha[0] = s->omega[0] = 1.0;
      s->beta[0] = 0.0;
      s->iters[0] = 0;
      s->status[0] = done ? final_status : KS_RUNNING;
      s->active = done ? 0 : 1;
    }
  }
}

// Jacobi-preconditioned CG (Hestenes-Stiefel) on the SPD Poisson operator.
struct CgArgs {
  SellView S;
  const double *Ls;
  const double *invL;
  double *x, *r, *z, *pk, *q;
  int n;
  CgState *cs;
  Reduce red;
  cudaGraphConditionalHandle cond;
  int use_cond;
  DevStatus *st;  // launch counters
  int scaled;     // convergence norm: 0 r.r, 1 r.z = ||D^-1/2 r||^2
};

// C1: q = L p, alpha = absnew / (p . q)
__global__ void k_cg_q(CgArgs A) {
  if (!A.cs->active) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
  double part[1] = {0.0};
  if (i >= 0) {
    double acc[1];
    sell_spmv_row<1>(A.S, A.Ls, A.pk, A.n, r, acc);
    A.q[i] = acc[0];
    part[0] = A.pk[i] * acc[0];
  }
  double tot[1];
  if (grid_reduce<1>(part, A.red, tot) && threadIdx.x == 0) {
    if (tot[0] == 0.0) {
      A.cs->status = KS_BREAKDOWN;
      A.cs->active = 0;
    } else {
      A.cs->alpha = A.cs->absnew / tot[0];
    }
  }
}

// C2: x += alpha p, r -= alpha q, z = D^-1 r; convergence test, beta = (r.z)_new / (r.z)_old
__global__ void k_cg_xr(CgArgs A) {
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[1] += 1;
  if (!A.cs->active) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part[2] = {0.0, 0.0};
  if (i < A.n) {
    const double alpha = A.cs->alpha;
    A.x[i] += alpha * A.pk[i];
    const double ri = A.r[i] - alpha * A.q[i];
    A.r[i] = ri;
    const double zi = A.invL[i] * ri;
    A.z[i] = zi;
    part[0] = ri * ri;
    part[1] = ri * zi;
  }
  double tot[2];
  if (grid_reduce<2>(part, A.red, tot) && threadIdx.x == 0) {
    CgState *c = A.cs;
    const double crit = A.scaled ? tot[1] : tot[0];
    c->iters += 1;
    c->rnorm2 = crit;
    if (isnan(tot[0]) || isnan(tot[1])) {
      c->status = KS_BREAKDOWN;
      c->active = 0;
    } else if (crit <= c->tol2) {
      c->status = KS_CONVERGED;
      c->active = 0;
    } else if (c->iters >= c->maxit) {
      c->status = KS_MAXIT;
      c->active = 0;
    } else {
      c->beta = tot[1] / c->absnew;
      c->absnew = tot[1];
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, c->active ? 1u : 0u);
  }
}

// C3: p = z + beta p
__global__ void k_cg_p(CgArgs A) {
  if (!A.cs->active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  A.pk[i] = A.z[i] + A.cs->beta * A.pk[i];
}

// ------------------------------------------------------------------------------------------
// Persistent CG: the whole pressure solve in one cooperative launch. Per iteration:
//   A  (SELL blocks)    p_new = z + beta p (on the fly, double-buffered), q = L p_new, p.q partials
//   -- grid barrier --
//   B  (natural blocks) alpha = absnew / (p.q); x += alpha p; r -= alpha q; z = D^-1 r; r.r, r.z
//   -- grid barrier --
//   C  (every CTA)      totals, convergence test, beta
// Every CTA recomputes the totals from the block partials with the same tree as grid_reduce, so
// all CTAs take the same decisions and the iterates equal those of k_cg_q / k_cg_xr / k_cg_p bit
// for bit. Data written by other CTAs inside the launch is read with L1-bypassing loads.
// Barriers spin with a bound; on expiry the kernel records an error and every CTA returns.
// The bound is a launch argument (default kBarrierSpinLimit polls, over a second), so that a
// test can make a wait run out on purpose and check that the step reports it.
constexpr long long kBarrierSpinLimit = 1LL << 25;

struct GridBarrier {
  unsigned int *count;  // [1 + kBarrierGroups]: top counter, then one counter per group of CTAs
  unsigned int *gen;
  int *err;
  long long spin_limit;  // polls of the generation word before a waiting CTA gives up
};
constexpr int kBarrierGroupSize = 32;  // CTAs per first-level counter
constexpr int kBarrierGroups = 64;     // supports grids of up to 2048 CTAs

// Two-level arrival: a CTA increments its group's counter; the last CTA of a group increments
// the top counter; the last group releases everyone by bumping the generation word.
__device__ __forceinline__ bool grid_sync(const GridBarrier &B) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *vgen = B.gen;
    volatile int *verr = B.err;
    const unsigned int g = *vgen;
    __threadfence();
    int ok = 1;
    const unsigned int grp = blockIdx.x / kBarrierGroupSize;
    const unsigned int ngroups = (gridDim.x + kBarrierGroupSize - 1) / kBarrierGroupSize;
    const unsigned int in_grp = min((unsigned int)kBarrierGroupSize, gridDim.x - grp * kBarrierGroupSize);
    bool releaser = false;
    if (atomicAdd(B.count + 1 + grp, 1u) == in_grp - 1) {
      B.count[1 + grp] = 0u;
      __threadfence();
      if (atomicAdd(B.count, 1u) == ngroups - 1) {
        *B.count = 0u;
        __threadfence();
        atomicAdd(B.gen, 1u);
        releaser = true;
      }
    }
    if (!releaser) {
      long long spins = 0;
      while (*vgen == g) {
        if (*verr) {
          ok = 0;
          break;
        }
        if (++spins > B.spin_limit) {
          atomicExch(B.err, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok && (*verr == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

// Same tree as the last block of grid_reduce: thread t sums partials t, t+256, ... in order,
// then warp butterflies and an in-order sum over the 8 warps. All threads get the totals.
template <int NV>
__device__ __forceinline__ void tree_total(const double *__restrict__ partials, int nblk,
                                           double (&out)[NV]) {
  __shared__ double sm[NV][kBlock / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double s = 0.0;
    int b = threadIdx.x;
    for (; b + 3 * (int)blockDim.x < nblk; b += 4 * blockDim.x) {  // four independent loads in flight
      const double v0 = __ldcg(&partials[(size_t)b * kMaxRed + j]);
      const double v1 = __ldcg(&partials[(size_t)(b + blockDim.x) * kMaxRed + j]);
      const double v2 = __ldcg(&partials[(size_t)(b + 2 * blockDim.x) * kMaxRed + j]);
      const double v3 = __ldcg(&partials[(size_t)(b + 3 * blockDim.x) * kMaxRed + j]);
      s += v0;
      s += v1;
      s += v2;
      s += v3;
    }
    for (; b < nblk; b += blockDim.x) s += __ldcg(&partials[(size_t)b * kMaxRed + j]);
    s = warp_sum(s);
    if (lane == 0) sm[j][warp] = s;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[j][w];
    out[j] = s;
  }
  __syncthreads();
}

// First stage of grid_reduce for one block of 256 positions: the block partial.
template <int NV>
__device__ __forceinline__ void block_partial(double (&v)[NV], double *__restrict__ partials, int b) {
  __shared__ double sm[NV][kBlock / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double w = warp_sum(v[j]);
    if (lane == 0) sm[j][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sm[j][w];
      partials[(size_t)b * kMaxRed + j] = s;
    }
  }
  __syncthreads();
}

struct CgPersistentArgs {
  SellView S;
  const double *Ls, *invL;
  double *x, *r, *z, *q;
  double *p[2];  // search direction, double-buffered
  int n;
  int nblk_sell, nblk_nat;
  double *part_a, *part_b;  // block partials of phases A and B
  CgState *cs;
  DevStatus *st;
  GridBarrier bar;
  int scaled;  // convergence norm: 0 r.r, 1 r.z
};

// Entries fetched per chunk of a row in the fused SpMV (4 measured fastest against 8, and against
// a variant that stores p in a third phase behind one more grid barrier).
constexpr int kCgChunk = 4;

__global__ void __launch_bounds__(kBlock, 4) k_cg_persistent(CgPersistentArgs A) {
  if (A.st && A.st->halt) return;
  if (!A.cs->active) return;
  const double tol2 = A.cs->tol2;
  const int maxit = A.cs->maxit;
  double absnew = A.cs->absnew, beta = 0.0, alpha = 0.0, rr = 0.0;
  int it = 0, status = KS_RUNNING, cur = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[1] += 1;
  while (true) {
    const bool fly = it > 0;  // p_new = z + beta p_old formed on the fly from both
    const double *pold = A.p[cur];
    double *pnew = A.p[cur ^ 1];
    // phase A: q = L p on SELL blocks
    for (int b = blockIdx.x; b < A.nblk_sell; b += gridDim.x) {
      const int r = b * kBlock + threadIdx.x;
      const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
      double v[1] = {0.0};
      if (i >= 0) {
        const int base = A.S.sptr[r >> 5] + (r & 31), len = A.S.len[r];
        double acc = 0.0;
        int k = 0;
        for (; k + kCgChunk <= len; k += kCgChunk) {  // indices and values, gathers, then the sum
          int jj[kCgChunk];
          double a[kCgChunk], po[kCgChunk], zz[kCgChunk];
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const int pos = base + (k + u) * kSellC;
            jj[u] = __ldg(A.S.col + pos);
            a[u] = __ldg(A.Ls + pos);
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            po[u] = __ldcg(pold + jj[u]);
            zz[u] = fly ? __ldcg(A.z + jj[u]) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) acc += a[u] * (fly ? zz[u] + beta * po[u] : po[u]);
        }
        if (k < len) {  // the last len % kCgChunk entries as one predicated chunk
          int jj[kCgChunk];
          double a[kCgChunk], po[kCgChunk], zz[kCgChunk];
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const int pos = base + (k + u) * kSellC;
            const bool in = k + u < len;
            jj[u] = in ? __ldg(A.S.col + pos) : 0;
            a[u] = in ? __ldg(A.Ls + pos) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const bool in = k + u < len;
            po[u] = in ? __ldcg(pold + jj[u]) : 0.0;
            zz[u] = (in && fly) ? __ldcg(A.z + jj[u]) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u)
            if (k + u < len) acc += a[u] * (fly ? zz[u] + beta * po[u] : po[u]);
        }
        const double pi = fly ? __ldcg(A.z + i) + beta * __ldcg(pold + i) : __ldcg(pold + i);
        __stcg(pnew + i, pi);
        __stcg(A.q + i, acc);
        v[0] = pi * acc;
      }
      block_partial<1>(v, A.part_a, b);
    }
    if (!grid_sync(A.bar)) return;
    double pq[1];
    tree_total<1>(A.part_a, A.nblk_sell, pq);
    if (pq[0] == 0.0) {
      status = KS_BREAKDOWN;
      break;
    }
    alpha = absnew / pq[0];
    // phase B: vector updates on natural blocks
    for (int b = blockIdx.x; b < A.nblk_nat; b += gridDim.x) {
      const int i = b * kBlock + threadIdx.x;
      double v[2] = {0.0, 0.0};
      if (i < A.n) {
        const double xi = __ldcg(A.x + i) + alpha * __ldcg(pnew + i);
        const double ri = __ldcg(A.r + i) - alpha * __ldcg(A.q + i);
        const double zi = __ldg(A.invL + i) * ri;
        __stcg(A.x + i, xi);
        __stcg(A.r + i, ri);
        __stcg(A.z + i, zi);
        v[0] = ri * ri;
        v[1] = ri * zi;
      }
      block_partial<2>(v, A.part_b, b);
    }
    if (!grid_sync(A.bar)) return;
    double tb[2];
    tree_total<2>(A.part_b, A.nblk_nat, tb);
    ++it;
    rr = A.scaled ? tb[1] : tb[0];
    if (isnan(tb[0]) || isnan(tb[1])) {
      status = KS_BREAKDOWN;
      break;
    }
    if (rr <= tol2) {
      status = KS_CONVERGED;
      break;
    }
    if (it >= maxit) {
      status = KS_MAXIT;
      break;
    }
    beta = tb[1] / absnew;
    absnew = tb[1];
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    CgState *c = A.cs;
    c->iters = it;
    c->rnorm2 = rr;
    c->alpha = alpha;
    c->beta = beta;
    c->absnew = absnew;
    c->status = status;
    c->active = 0;
  }
}

// ------------------------------------------------------------------------------------------
// SMEM-resident persistent CG: one CTA of 1024 threads per SM for the whole solve. Each CTA owns
// a contiguous run of 256-position blocks (SELL blocks for the product, natural blocks for the
// vector updates) and keeps, in shared memory for the whole solve, the row id, length and entry
// base of each of its SELL positions and the column indices of as many of its slices as fit
// (the rest are read from global memory). Inside an iteration the column indices then cost a
// shared-memory read instead of an L2 round trip before the gathers can be issued. The
// arithmetic, the per-block partial sums and the 256-accumulator tree are those of
// k_cg_persistent, so both kernels produce the same bits.
constexpr int kCgResThreads = 1024;
constexpr int kCgResGroups = kCgResThreads / kBlock;  // 256-thread groups per CTA

struct CgResidentArgs {
  CgPersistentArgs P;
  int nslices;
  int bpc_sell, bpc_nat;  // blocks per CTA
  int col_cap;            // column indices that fit in shared memory per CTA
};

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, %1;" ::"r"(1 + g), "r"(kBlock) : "memory");
}

// block_partial for one 256-thread group of a larger CTA (named barrier 1 + g); the values go to
// slots j0, j0 + 1, ... of the block's partials.
template <int NV, int NS>
__device__ __forceinline__ void group_partial(double (&v)[NV], double *__restrict__ partials, int b,
                                              int g, double (*sm)[NS][kBlock / 32], int j0 = 0) {
  const int lt = threadIdx.x & (kBlock - 1), warp = lt >> 5, lane = lt & 31;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double w = warp_sum(v[j]);
    if (lane == 0) sm[g][j][warp] = w;
  }
  group_sync(g);
  if (lt == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0.0;
      for (int w = 0; w < kBlock / 32; ++w) s += sm[g][j][w];
      partials[(size_t)b * kMaxRed + j0 + j] = s;
    }
  }
  group_sync(g);
}

// tree_total for a 1024-thread CTA: the 256-thread quarter j forms the 256 accumulators of value
// j (same sums in the same order as tree_total), so the values are reduced side by side with eight
// loads in flight per thread instead of one value after another.
template <int NV>
__device__ __forceinline__ void tree_total_cta(const double *__restrict__ partials, int nblk,
                                               double (&out)[NV], double (*sm)[kBlock / 32]) {
  static_assert(NV * kBlock <= kCgResThreads, "one 256-thread quarter per value");
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = threadIdx.x / kBlock, t = threadIdx.x & (kBlock - 1);
  if (j < NV) {
    // accumulator t of value j: blocks t, t + 256, ... in order, eight loads in flight
    constexpr int kB = 8;
    double s = 0.0;
    int b = t;
    for (; b + (kB - 1) * kBlock < nblk; b += kB * kBlock) {
      double v[kB];
#pragma unroll
      for (int q = 0; q < kB; ++q) v[q] = __ldcg(&partials[(size_t)(b + q * kBlock) * kMaxRed + j]);
#pragma unroll
      for (int q = 0; q < kB; ++q) s += v[q];
    }
    double v[kB];
#pragma unroll
    for (int q = 0; q < kB; ++q)
      v[q] = (b + q * kBlock < nblk) ? __ldcg(&partials[(size_t)(b + q * kBlock) * kMaxRed + j]) : 0.0;
#pragma unroll
    for (int q = 0; q < kB; ++q)
      if (b + q * kBlock < nblk) s += v[q];
    s = warp_sum(s);
    if (lane == 0) sm[j][warp & (kBlock / 32 - 1)] = s;
  }
  __syncthreads();
#pragma unroll
  for (int j2 = 0; j2 < NV; ++j2) {
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += sm[j2][w];
    out[j2] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kCgResThreads, 1) k_cg_resident(CgResidentArgs R) {
  extern __shared__ int s_dyn[];
  __shared__ double s_grp[kCgResGroups][3][kBlock / 32];
  __shared__ double s_tree[3][kBlock / 32];
  const CgPersistentArgs &A = R.P;
  if (A.st && A.st->halt) return;
  if (!A.cs->active) return;
  const int g = threadIdx.x / kBlock, lt = threadIdx.x & (kBlock - 1);
  // owned blocks
  const int b0 = min(A.nblk_sell, (int)blockIdx.x * R.bpc_sell);
  const int b1 = min(A.nblk_sell, b0 + R.bpc_sell);
  const int c0 = min(A.nblk_nat, (int)blockIdx.x * R.bpc_nat);
  const int c1 = min(A.nblk_nat, c0 + R.bpc_nat);
  int *s_row = s_dyn;                          // [bpc_sell * 256]
  int *s_len = s_row + R.bpc_sell * kBlock;    // [bpc_sell * 256]
  int *s_base = s_len + R.bpc_sell * kBlock;   // [bpc_sell * 256]
  int *s_col = s_base + R.bpc_sell * kBlock;   // [col_cap]
  const int e0 = (b0 < b1) ? A.S.sptr[8 * b0] : 0;
  int bs = b0;  // blocks [b0, bs) have their column indices in shared memory
  while (bs < b1 && A.S.sptr[min(8 * (bs + 1), R.nslices)] - e0 <= R.col_cap) ++bs;
  const int e1 = (bs > b0) ? A.S.sptr[min(8 * bs, R.nslices)] : e0;
  for (int e = e0 + (int)threadIdx.x; e < e1; e += kCgResThreads) s_col[e - e0] = A.S.col[e];
  for (int q = threadIdx.x; q < (b1 - b0) * kBlock; q += kCgResThreads) {
    const int r = b0 * kBlock + q;
    const bool in = r < A.S.nrows_pad;
    s_row[q] = in ? A.S.perm[r] : -1;
    s_len[q] = in ? A.S.len[r] : 0;
    s_base[q] = in ? A.S.sptr[r >> 5] + (r & 31) : 0;
  }
  __syncthreads();
  const double tol2 = A.cs->tol2;
  const int maxit = A.cs->maxit;
  double absnew = A.cs->absnew, beta = 0.0, alpha = 0.0, rr = 0.0;
  int it = 0, status = KS_RUNNING, cur = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[1] += 1;
  while (true) {
    const bool fly = it > 0;
    const double *pold = A.p[cur];
    double *pnew = A.p[cur ^ 1];
    // phase A: q = L p on the owned SELL blocks, one group per block
    for (int b = b0 + g; b < b1; b += kCgResGroups) {
      const int lp = (b - b0) * kBlock + lt;
      const int i = s_row[lp];
      double v[1] = {0.0};
      if (i >= 0) {
        const int base = s_base[lp], len = s_len[lp];
        const bool staged = b < bs;
        double acc = 0.0;
        int k = 0;
        for (; k + kCgChunk <= len; k += kCgChunk) {
          int jj[kCgChunk];
          double a[kCgChunk], po[kCgChunk], zz[kCgChunk];
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const int pos = base + (k + u) * kSellC;
            jj[u] = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
            a[u] = __ldg(A.Ls + pos);
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            po[u] = __ldcg(pold + jj[u]);
            zz[u] = fly ? __ldcg(A.z + jj[u]) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) acc += a[u] * (fly ? zz[u] + beta * po[u] : po[u]);
        }
        if (k < len) {  // the last len % kCgChunk entries as one predicated chunk
          int jj[kCgChunk];
          double a[kCgChunk], po[kCgChunk], zz[kCgChunk];
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const int pos = base + (k + u) * kSellC;
            const bool in = k + u < len;
            jj[u] = !in ? 0 : staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
            a[u] = in ? __ldg(A.Ls + pos) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u) {
            const bool in = k + u < len;
            po[u] = in ? __ldcg(pold + jj[u]) : 0.0;
            zz[u] = (in && fly) ? __ldcg(A.z + jj[u]) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kCgChunk; ++u)
            if (k + u < len) acc += a[u] * (fly ? zz[u] + beta * po[u] : po[u]);
        }
        const double pi = fly ? __ldcg(A.z + i) + beta * __ldcg(pold + i) : __ldcg(pold + i);
        __stcg(pnew + i, pi);
        __stcg(A.q + i, acc);
        v[0] = pi * acc;
      }
      group_partial<1>(v, A.part_a, b, g, s_grp);
    }
    if (!grid_sync(A.bar)) return;
    double pq[1];
    tree_total_cta<1>(A.part_a, A.nblk_sell, pq, s_tree);
    if (pq[0] == 0.0) {
      status = KS_BREAKDOWN;
      break;
    }
    alpha = absnew / pq[0];
    // phase B: vector updates on the owned natural blocks
    for (int b = c0 + g; b < c1; b += kCgResGroups) {
      const int i = b * kBlock + lt;
      double v[2] = {0.0, 0.0};
      if (i < A.n) {
        const double xi = __ldcg(A.x + i) + alpha * __ldcg(pnew + i);
        const double ri = __ldcg(A.r + i) - alpha * __ldcg(A.q + i);
        const double zi = __ldg(A.invL + i) * ri;
        __stcg(A.x + i, xi);
        __stcg(A.r + i, ri);
        __stcg(A.z + i, zi);
        v[0] = ri * ri;
        v[1] = ri * zi;
      }
      group_partial<2>(v, A.part_b, b, g, s_grp);
    }
    if (!grid_sync(A.bar)) return;
    double tb[2];
    tree_total_cta<2>(A.part_b, A.nblk_nat, tb, s_tree);
    ++it;
    rr = A.scaled ? tb[1] : tb[0];
    if (isnan(tb[0]) || isnan(tb[1])) {
      status = KS_BREAKDOWN;
      break;
    }
    if (rr <= tol2) {
      status = KS_CONVERGED;
      break;
    }
    if (it >= maxit) {
      status = KS_MAXIT;
      break;
    }
    beta = tb[1] / absnew;
    absnew = tb[1];
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    CgState *c = A.cs;
    c->iters = it;
    c->rnorm2 = rr;
    c->alpha = alpha;
    c->beta = beta;
    c->absnew = absnew;
    c->status = status;
    c->active = 0;
  }
}

// Jacobi-preconditioned CG with one reduction per iteration (Chronopoulos & Gear 1989), the same
// iterates as CG in exact arithmetic: s = A p is carried by a recurrence, so an iteration is ONE
// fused pass (vector updates, product, three dot products) and ONE grid barrier instead of two:
//   p = u + b p;  s = w + b s;  x += a p;  r -= a s;  u = M r;  w = A u;
//   gamma = r.u, delta = w.u, rr = r.r;   b' = gamma'/gamma,  a' = gamma' / (delta' - b' gamma' / a).
// The product needs the new u of neighbouring rows: each gathering thread forms it from that row's
// previous r, w and s (the expression its owner evaluates, so the same bits). r, w and s are
// double-buffered; p and x are only read by their own row. Layout, staging and reduction tree
// are those of k_cg_resident.
struct Cg1Args {
  CgResidentArgs R;
  double *r[2], *w[2], *s[2];  // r[0] = b on entry; s[0] zero on entry
  const double *u0;            // M b (from the right-hand-side kernel)
  double *p;                   // zero on entry
};

__global__ void __launch_bounds__(kCgResThreads, 1) k_cg1_resident(Cg1Args C) {
  extern __shared__ int s_dyn[];
  __shared__ double s_grp[kCgResGroups][3][kBlock / 32];
  __shared__ double s_tree[3][kBlock / 32];
  const CgResidentArgs &R = C.R;
  const CgPersistentArgs &A = R.P;
  if (A.st && A.st->halt) return;
  if (!A.cs->active) return;
  const int g = threadIdx.x / kBlock, lt = threadIdx.x & (kBlock - 1);
  const int b0 = min(A.nblk_sell, (int)blockIdx.x * R.bpc_sell);
  const int b1 = min(A.nblk_sell, b0 + R.bpc_sell);
  int *s_row = s_dyn;
  int *s_len = s_row + R.bpc_sell * kBlock;
  int *s_base = s_len + R.bpc_sell * kBlock;
  int *s_col = s_base + R.bpc_sell * kBlock;
  const int e0 = (b0 < b1) ? A.S.sptr[8 * b0] : 0;
  int bs = b0;
  while (bs < b1 && A.S.sptr[min(8 * (bs + 1), R.nslices)] - e0 <= R.col_cap) ++bs;
  const int e1 = (bs > b0) ? A.S.sptr[min(8 * bs, R.nslices)] : e0;
  for (int e = e0 + (int)threadIdx.x; e < e1; e += kCgResThreads) s_col[e - e0] = A.S.col[e];
  for (int q = threadIdx.x; q < (b1 - b0) * kBlock; q += kCgResThreads) {
    const int r = b0 * kBlock + q;
    const bool in = r < A.S.nrows_pad;
    s_row[q] = in ? A.S.perm[r] : -1;
    s_len[q] = in ? A.S.len[r] : 0;
    s_base[q] = in ? A.S.sptr[r >> 5] + (r & 31) : 0;
  }
  __syncthreads();
  const double tol2 = A.cs->tol2;
  const int maxit = A.cs->maxit;
  double gamma = A.cs->absnew, alpha = 0.0, beta = 0.0, rn2 = A.cs->bnorm2;
  int it = 0, status = KS_RUNNING, cur = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[1] += 1;
  // start: w = A u0, delta = w.u0
  for (int b = b0 + g; b < b1; b += kCgResGroups) {
    const int lp = (b - b0) * kBlock + lt;
    const int i = s_row[lp];
    double v[1] = {0.0};
    if (i >= 0) {
      const int base = s_base[lp], len = s_len[lp];
      const bool staged = b < bs;
      double acc = 0.0;
      for (int k = 0; k < len; ++k) {
        const int pos = base + k * kSellC;
        const int jj = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
        acc += __ldg(A.Ls + pos) * __ldcg(C.u0 + jj);
      }
      __stcg(C.w[0] + i, acc);
      v[0] = acc * __ldcg(C.u0 + i);
    }
    group_partial<1>(v, A.part_a, b, g, s_grp);
  }
  if (!grid_sync(A.bar)) return;
  {
    double d0[1];
    tree_total_cta<1>(A.part_a, A.nblk_sell, d0, s_tree);
    if (d0[0] == 0.0)
      status = KS_BREAKDOWN;
    else
      alpha = gamma / d0[0];
  }
  while (status == KS_RUNNING) {
    // partials alternate between the two buffers: with one barrier per iteration a CTA may write
    // this iteration's partials while another still reads the previous iteration's
    double *part = (it & 1) ? A.part_a : A.part_b;
    const double *ro = C.r[cur], *wo = C.w[cur], *so = C.s[cur];
    double *rn = C.r[cur ^ 1], *wn = C.w[cur ^ 1], *sn = C.s[cur ^ 1];
    for (int b = b0 + g; b < b1; b += kCgResGroups) {
      const int lp = (b - b0) * kBlock + lt;
      const int i = s_row[lp];
      double v[3] = {0.0, 0.0, 0.0};
      if (i >= 0) {
        const int base = s_base[lp], len = s_len[lp];
        const bool staged = b < bs;
        double acc = 0.0;
        int k = 0;
        for (; k + kCgChunk <= len; k += kCgChunk) {
          int jj[kCgChunk];
          double a[kCgChunk], rr_[kCgChunk], ww[kCgChunk], ss[kCgChunk], mm[kCgChunk];
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            const int pos = base + (k + q) * kSellC;
            jj[q] = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
            a[q] = __ldg(A.Ls + pos);
          }
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            rr_[q] = __ldcg(ro + jj[q]);
            ww[q] = __ldcg(wo + jj[q]);
            ss[q] = __ldcg(so + jj[q]);
            mm[q] = __ldg(A.invL + jj[q]);
          }
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            const double sj = ww[q] + beta * ss[q];
            const double rj = rr_[q] - alpha * sj;
            acc += a[q] * (mm[q] * rj);
          }
        }
        if (k < len) {  // the last len % kCgChunk entries as one predicated chunk
          int jj[kCgChunk];
          double a[kCgChunk], rr_[kCgChunk], ww[kCgChunk], ss[kCgChunk], mm[kCgChunk];
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            const int pos = base + (k + q) * kSellC;
            const bool in = k + q < len;
            jj[q] = !in ? 0 : staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
            a[q] = in ? __ldg(A.Ls + pos) : 0.0;
          }
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            const bool in = k + q < len;
            rr_[q] = in ? __ldcg(ro + jj[q]) : 0.0;
            ww[q] = in ? __ldcg(wo + jj[q]) : 0.0;
            ss[q] = in ? __ldcg(so + jj[q]) : 0.0;
            mm[q] = in ? __ldg(A.invL + jj[q]) : 0.0;
          }
#pragma unroll
          for (int q = 0; q < kCgChunk; ++q) {
            const double sj = ww[q] + beta * ss[q];
            const double rj = rr_[q] - alpha * sj;
            if (k + q < len) acc += a[q] * (mm[q] * rj);
          }
        }
        // own row
        const double mi = __ldg(A.invL + i);
        const double roi = __ldcg(ro + i);
        const double uoi = (it == 0) ? __ldcg(C.u0 + i) : mi * roi;
        const double pi = uoi + beta * __ldcg(C.p + i);
        const double si = __ldcg(wo + i) + beta * __ldcg(so + i);
        const double xi = __ldcg(A.x + i) + alpha * pi;
        const double ri = roi - alpha * si;
        const double ui = mi * ri;
        __stcg(C.p + i, pi);
        __stcg(sn + i, si);
        __stcg(A.x + i, xi);
        __stcg(rn + i, ri);
        __stcg(wn + i, acc);
        v[0] = ri * ui;
        v[1] = acc * ui;
        v[2] = ri * ri;
      }
      group_partial<3>(v, part, b, g, s_grp);
    }
    if (!grid_sync(A.bar)) return;
    double t[3];
    tree_total_cta<3>(part, A.nblk_sell, t, s_tree);
    ++it;
    rn2 = A.scaled ? t[0] : t[2];
    cur ^= 1;
    if (isnan(t[0]) || isnan(t[1]) || isnan(t[2])) {
      status = KS_BREAKDOWN;
      break;
    }
    if (rn2 <= tol2) {
      status = KS_CONVERGED;
      break;
    }
    if (it >= maxit) {
      status = KS_MAXIT;
      break;
    }
    const double beta_new = t[0] / gamma;
    const double den = t[1] - beta_new * t[0] / alpha;
    if (den == 0.0) {
      status = KS_BREAKDOWN;
      break;
    }
    alpha = t[0] / den;
    beta = beta_new;
    gamma = t[0];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    CgState *c = A.cs;
    c->iters = it;
    c->rnorm2 = rn2;
    c->alpha = alpha;
    c->beta = beta;
    c->absnew = gamma;
    c->status = status;
    c->active = 0;
  }
}

// ------------------------------------------------------------------------------------------
// Two-level single-reduction CG (CFSA_KRYLOV_CG2L): the recurrences of k_cg1_resident with the
// preconditioner M r = D^-1 r + P Z P^T r, where P is the indicator matrix of geometric aggregates
// (boxes of a uniform grid over the vertices, rows without a penalty only) and Z = (P^T A P)^-1 is
// a dense nc x nc matrix built on the host. The coarse correction removes the smooth error
// components that make Jacobi-CG slow on the Poisson operator (681 -> 127 iterations on the
// 1M-tet cylinder with ~256 aggregates requested).
//
// One grid barrier per iteration is kept: the coarse input t = P^T r of the new residual is
// formed after the barrier from the previous iteration's aggregate sums of r and w and the
// aggregate-level recurrence for s,
//   T(s) <- T(w) + beta T(s),   t = T(r) - alpha T(s),   c = Z t,
// and each neighbour's new u = D^-1 r_new + c[agg] is then formed on the fly in the fused product,
// as k_cg1_resident does for the Jacobi part.
//
// Aggregate sums are exact fixed-point sums, so their order does not matter and they cost a few
// atomics instead of a reduction tree: each value x becomes the 128-bit integer floor(x 2^S)
// (S = 80 - floor(log2(b.b) / 2), clamped to +-2^100). A CTA stages its rows' values in shared
// memory sorted by aggregate, one warp per 64-position piece of a segment sums it exactly and adds
// it into a global accumulator (three carry-free 64-bit words, red128), and after the barrier a
// sum converts back as (hi 2^64 + lo) 2^-S.
// Global accumulators rotate over three buffers; the buffer of the next phase is cleared while no
// CTA can still read it. c[m] is a warp butterfly over lanes l of sum_{k = l mod 32} Z[m][k]
// t[k]. Each CTA forms c only for the aggregates its rows and their neighbours belong to. The
// oracle's cg2l() restates the same arithmetic, so GPU and oracle agree bit for bit.
constexpr int kSegPiece = 64;  // staging positions per piece of an aggregate sum

struct CoarseView {
  int nc;                       // aggregates (0: Jacobi only)
  const int *agg;               // [n] aggregate of each row; nc for rows without one
  const double *Z;              // [nc*nc] (P^T A P)^-1, symmetric
  const int *row_pos;           // [n] position of the row in its CTA's aggregate-sorted staging
                                // order, -1 for rows without aggregate
  const int *own_ptr, *own;     // aggregates of each CTA's rows (ascending)
  const int *seg_lo, *seg_hi;   // staging positions of each own aggregate's rows
  const int *own_pfirst;        // [own entries + 1] first piece of each own aggregate's segment
  const int4 *pieces;           // (first, end staging position, aggregate, 0) per piece
  const int *need_ptr, *need;   // aggregates whose coarse value each CTA reads
  unsigned long long *gacc;     // [3 buffers][3 vectors][nc][3 words] fixed-point sums (red128)
  int npos_max;                 // largest staging list (shared-memory doubles per vector)
};

struct Cg2lArgs {
  CgResidentArgs R;
  CoarseView V;
  double *r[2], *w[2], *s[2];  // r[0] = b on entry
  double *p;                   // zero on entry
  // float storage of the mixed-precision inner solve (k_cg2l_resident<float>): operator values,
  // inverse diagonal, solution and the same vectors (r32[0] = b, p32 = s32[0] = 0 on entry)
  const float *Ls32, *invL32;
  float *x32, *r32[2], *w32[2], *s32[2], *p32;
  // u = D^-1 r + c[agg] of the current residual, stored by the split form (k_cg2l_resident with
  // SPLIT) between its two passes
  double *u;
  float *u32;
};

// floor(x 2^S) as a two's-complement 128-bit integer (lo, hi); x 2^S is clamped to +-2^100 and a
// NaN counts as 0.
__device__ __forceinline__ void fixed128(double x, double scale, unsigned long long &lo,
                                         unsigned long long &hi) {
  double y = x * scale;
  if (!(y == y)) y = 0.0;
  y = fmin(fmax(y, -0x1p100), 0x1p100);
  const double t = floor(y);
  if (fabs(t) < 0x1p63) {
    const long long v = (long long)t;
    lo = (unsigned long long)v;
    hi = (v < 0) ? ~0ull : 0ull;
  } else {
    const double hd = floor(t * 0x1p-64);
    hi = (unsigned long long)(long long)hd;
    lo = (unsigned long long)(t - hd * 0x1p64);
  }
}

// Exact 128-bit sums held in three 64-bit words of 42, 42 and 44 bits: every term adds its chunk
// to each word with an atomic whose result is not used (a reduction the thread does not wait
// for; no carry passes between the words, so no atomic depends on another). The two low words
// stay exact for fewer than 2^22 terms, far above the pieces of one phase (at most 148 CTAs x a
// few hundred); the top word only matters modulo 2^44.
constexpr unsigned long long kMask42 = (1ull << 42) - 1ull;

__device__ __forceinline__ void red128(unsigned long long *p, unsigned long long lo, unsigned long long hi) {
  atomicAdd(p, lo & kMask42);
  atomicAdd(p + 1, ((lo >> 42) | (hi << 22)) & kMask42);
  atomicAdd(p + 2, hi >> 20);
}

// The 128-bit total (lo, hi) of three accumulated words: w0 + w1 2^42 + w2 2^84 modulo 2^128.
__device__ __forceinline__ void words128(const unsigned long long *a, unsigned long long &lo,
                                         unsigned long long &hi) {
  const unsigned long long w0 = __ldcg(a), w1 = __ldcg(a + 1), w2 = __ldcg(a + 2);
  const unsigned long long s = w1 << 42;
  lo = w0 + s;
  hi = (w1 >> 22) + (w2 << 20) + ((lo < s) ? 1ull : 0ull);
}

__device__ __forceinline__ double unfixed128(unsigned long long lo, unsigned long long hi, double iscale) {
  return ((double)(long long)hi * 0x1p64 + (double)lo) * iscale;
}

// Sums of this CTA's staged values per own aggregate into global buffer `buf`. Each own
// aggregate's segment of the staging is cut into pieces of kSegPiece positions (listed per CTA
// on the host) and the warps take the CTA's pieces round robin, so a CTA whose rows fall into a
// few large aggregates still spreads the work over all its warps. In a piece each lane adds its
// values exactly as 128-bit integers offset by 2^100 (so that they are non-negative); the lane sums
// are cut into five 26-bit limbs, each limb summed by a warp reduction (32 x 2^26 < 2^32), and
// lane 0 re-assembles the piece's total, removes count x 2^100 and adds it to the global
// accumulator (red128). The sums are exact, so how a segment is cut does not change the result.
template <int NV>
__device__ __forceinline__ void seg_sums(const CoarseView &V, const double *__restrict__ stage,
                                         int buf, const int (&vi)[NV], double scale) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int g0 = __ldg(V.own_pfirst + __ldg(V.own_ptr + blockIdx.x));
  const int g1 = __ldg(V.own_pfirst + __ldg(V.own_ptr + blockIdx.x + 1));
  for (int gp = g0 + warp; gp < g1; gp += nw) {
    const int4 pc = __ldg(V.pieces + gp);  // x = first, y = end position, z = aggregate
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double *sv = stage + (size_t)v * V.npos_max;
      unsigned long long al = 0ull, ah = 0ull;
      for (int p = pc.x + lane; p < pc.y; p += 32) {
        unsigned long long l, h;
        fixed128(sv[p], scale, l, h);
        h += 1ull << 36;  // + 2^100
        al += l;
        ah += h + ((al < l) ? 1ull : 0ull);
      }
      const unsigned m26 = (1u << 26) - 1u;
      const unsigned long long s0 = __reduce_add_sync(0xffffffffu, (unsigned)(al & m26));
      const unsigned long long s1 = __reduce_add_sync(0xffffffffu, (unsigned)((al >> 26) & m26));
      const unsigned long long s2 = __reduce_add_sync(0xffffffffu, (unsigned)(((al >> 52) | (ah << 12)) & m26));
      const unsigned long long s3 = __reduce_add_sync(0xffffffffu, (unsigned)((ah >> 14) & m26));
      const unsigned long long s4 = __reduce_add_sync(0xffffffffu, (unsigned)((ah >> 40) & m26));
      if (lane == 0) {
        const unsigned long long l1 = s0 + (s1 << 26);
        const unsigned long long l2 = l1 + (s2 << 52);
        const unsigned long long h = (s2 >> 12) + (s3 << 14) + (s4 << 40) + ((l2 < l1) ? 1ull : 0ull) -
                                     ((unsigned long long)(pc.y - pc.x) << 36);
        red128(V.gacc + 3 * ((size_t)(3 * buf + vi[v]) * V.nc + pc.z), l2, h);
      }
    }
  }
}

// Clears global buffer `buf` (every CTA a share).
__device__ __forceinline__ void clear_acc(const CoarseView &V, int buf) {
  unsigned long long *g = V.gacc + (size_t)9 * V.nc * buf;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 9 * V.nc; k += gridDim.x * blockDim.x) g[k] = 0ull;
}

// Aggregate sums of vectors [v0, v0 + NV) from global buffer `buf`.
template <int NV>
__device__ __forceinline__ void read_sums(const CoarseView &V, int buf, int v0, double iscale,
                                          double *const (&dst)[NV]) {
  for (int idx = threadIdx.x; idx < NV * V.nc; idx += blockDim.x) {
    const int v = idx / V.nc, m = idx - v * V.nc;
    unsigned long long lo, hi;
    words128(V.gacc + 3 * ((size_t)(3 * buf + v0 + v) * V.nc + m), lo, hi);
    dst[v][m] = unfixed128(lo, hi, iscale);
  }
}

// c[m] = Z[m] . t for the aggregates this CTA reads: one warp per aggregate, lane l adding
// k = l, l + 32, ... in order, then a warp butterfly. ZB entries of the Z row are loaded per lane
// at a time (16: one round trip for up to 512 aggregates); the batch does not change the sums.
template <int ZB>
__device__ __forceinline__ void coarse_values(const CoarseView &V, const double *__restrict__ t,
                                              double *__restrict__ c) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  const int q0 = __ldg(V.need_ptr + blockIdx.x), q1 = __ldg(V.need_ptr + blockIdx.x + 1);
  const int nc = V.nc;
  for (int q = q0 + warp; q < q1; q += nw) {
    const int m = __ldg(V.need + q);
    const double *zr = V.Z + (size_t)m * nc;
    double sum = 0.0;
    for (int k0 = lane; k0 < nc; k0 += 32 * ZB) {
      double z[ZB];
#pragma unroll
      for (int u = 0; u < ZB; ++u) z[u] = (k0 + 32 * u < nc) ? __ldg(zr + k0 + 32 * u) : 0.0;
#pragma unroll
      for (int u = 0; u < ZB; ++u)
        if (k0 + 32 * u < nc) sum += z[u] * t[k0 + 32 * u];
    }
    sum = warp_sum(sum);
    if (lane == 0) c[m] = sum;
  }
}

// Entries per chunk of the split form's product (one gather per entry, so twice the fused
// form's chunk fits in the registers).
constexpr int kCg2lChunk = 8;

// TS: storage type of the operator values, inverse diagonal, solution and Krylov vectors. double:
// the FP64 solve (bit-identical to the oracle's cg2l); float: the inner solve of the mixed-precision
// pressure solve (half the bytes per entry). Arithmetic, dot products, aggregate sums and scalars
// are FP64 in both; in the float form each updated vector entry is rounded to float once and the
// rounded value is the one used in the dot products and aggregate sums, so they describe the
// stored vectors.
template <class TS, bool SPLIT>
__global__ void __launch_bounds__(kCgResThreads, 1) k_cg2l_resident(Cg2lArgs C) {
  extern __shared__ double s_dbl[];
  __shared__ double s_grp[kCgResGroups][4][kBlock / 32];
  __shared__ double s_tree[4][kBlock / 32];
  const CgResidentArgs &R = C.R;
  const CgPersistentArgs &A = R.P;
  const CoarseView &V = C.V;
  constexpr bool f32 = std::is_same<TS, float>::value;
  constexpr int kZB = f32 ? 8 : 16;  // 16 spills in the float form
  const TS *Lsv, *invLv;
  TS *xv, *pv, *uv, *rv0, *rv1, *wv0, *wv1, *sv0, *sv1;
  if constexpr (f32) {
    Lsv = C.Ls32, invLv = C.invL32, xv = C.x32, pv = C.p32, uv = C.u32;
    rv0 = C.r32[0], rv1 = C.r32[1], wv0 = C.w32[0], wv1 = C.w32[1], sv0 = C.s32[0], sv1 = C.s32[1];
  } else {
    Lsv = A.Ls, invLv = A.invL, xv = A.x, pv = C.p, uv = C.u;
    rv0 = C.r[0], rv1 = C.r[1], wv0 = C.w[0], wv1 = C.w[1], sv0 = C.s[0], sv1 = C.s[1];
  }
  auto rnd = [](double v) { return (double)(TS)v; };  // storage rounding (identity for double)
  if (A.st && A.st->halt) return;
  if (!A.cs->active) return;
  const int g = threadIdx.x / kBlock, lt = threadIdx.x & (kBlock - 1);
  const int b0 = min(A.nblk_sell, (int)blockIdx.x * R.bpc_sell);
  const int b1 = min(A.nblk_sell, b0 + R.bpc_sell);
  const int nc = V.nc, n = A.n;
  // shared memory: aggregate sums of r, w, s, the coarse input t, coarse values (two
  // generations, entry nc = 0 for rows without aggregate), the aggregate-sorted staging of two
  // row vectors, then the row staging of k_cg1_resident
  double *cR = s_dbl, *cW = cR + nc, *cS = cW + nc, *ct = cS + nc;
  double *cc[2] = {ct + nc, ct + 2 * nc + 1};
  double *s_stage = ct + 3 * nc + 2;
  int *s_row = reinterpret_cast<int *>(s_stage + 2 * V.npos_max);
  int *s_len = s_row + R.bpc_sell * kBlock;
  int *s_base = s_len + R.bpc_sell * kBlock;
  int *s_col = s_base + R.bpc_sell * kBlock;
  const int e0 = (b0 < b1) ? A.S.sptr[8 * b0] : 0;
  int bs = b0;
  while (bs < b1 && A.S.sptr[min(8 * (bs + 1), R.nslices)] - e0 <= R.col_cap) ++bs;
  const int e1 = (bs > b0) ? A.S.sptr[min(8 * bs, R.nslices)] : e0;
  for (int e = e0 + (int)threadIdx.x; e < e1; e += kCgResThreads) s_col[e - e0] = A.S.col[e];
  for (int q = threadIdx.x; q < (b1 - b0) * kBlock; q += kCgResThreads) {
    const int r = b0 * kBlock + q;
    const bool in = r < A.S.nrows_pad;
    s_row[q] = in ? A.S.perm[r] : -1;
    s_len[q] = in ? A.S.len[r] : 0;
    s_base[q] = in ? A.S.sptr[r >> 5] + (r & 31) : 0;
  }
  for (int m = threadIdx.x; m <= nc; m += kCgResThreads) {
    cc[0][m] = 0.0;
    cc[1][m] = 0.0;
    if (m < nc) cS[m] = 0.0;
  }
  __syncthreads();
  const double tol2 = A.cs->tol2;
  const int maxit = A.cs->maxit;
  // fixed-point scale of the aggregate sums: 2^S with S = 80 - floor(log2(b.b) / 2)
  int S = 80;
  {
    const double bb = A.cs->bb;
    if (bb > 0.0 && bb <= 1.7976931348623157e308) {
      const int e2 = ilogb(bb);
      S = 80 - ((e2 >= 0) ? e2 / 2 : -((1 - e2) / 2));
    }
  }
  const double scale = scalbn(1.0, S), iscale = scalbn(1.0, -S);
  double gamma = 0.0, alpha = 0.0, beta = 0.0, rn2 = A.cs->bnorm2;
  int it = 0, status = KS_RUNNING, cur = 0, pc = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[1] += 1;
  const TS *bvec = rv0;
  const int v_r[1] = {0}, v_w[1] = {1}, v_rw[2] = {0, 1};
  // start: c0 = Z T(b) (phase 0, buffer 0)
  if (nc > 0) {
    for (int i = b0 * kBlock + (int)threadIdx.x; i < min(n, b1 * kBlock); i += kCgResThreads) {
      const int ps = __ldg(V.row_pos + i);
      if (ps >= 0) s_stage[ps] = (double)__ldcg(bvec + i);
    }
    __syncthreads();
    seg_sums<1>(V, s_stage, 0, v_r, scale);
    if (!grid_sync(A.bar)) return;
    double *const dR[1] = {cR};
    read_sums<1>(V, 0, 0, iscale, dR);
    __syncthreads();
    coarse_values<kZB>(V, cR, cc[0]);
    __syncthreads();
  }
  // phase 1 (buffer 1): w0 = A u0 with u0 = D^-1 b + c0[agg]; delta0 = w0.u0, gamma0 = b.u0
  for (int b = b0 + g; b < b1; b += kCgResGroups) {
    const int lp = (b - b0) * kBlock + lt;
    const int i = s_row[lp];
    double v[2] = {0.0, 0.0};
    if (i >= 0) {
      const int base = s_base[lp], len = s_len[lp];
      const bool staged = b < bs;
      double acc = 0.0;
      for (int k = 0; k < len; ++k) {
        const int pos = base + k * kSellC;
        const int jj = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
        const double uj = (double)__ldg(invLv + jj) * (double)__ldcg(bvec + jj) + cc[0][__ldg(V.agg + jj)];
        acc += (double)__ldg(Lsv + pos) * uj;
      }
      acc = rnd(acc);
      const double bi = (double)__ldcg(bvec + i);
      const double ui = (double)__ldg(invLv + i) * bi + cc[0][__ldg(V.agg + i)];
      __stcg(wv0 + i, (TS)acc);
      v[0] = acc * ui;
      v[1] = bi * ui;
      if (nc > 0) {
        const int ps = __ldg(V.row_pos + i);
        if (ps >= 0) s_stage[ps] = acc;
      }
    }
    group_partial<2>(v, A.part_a, b, g, s_grp);
  }
  if (nc > 0) {
    __syncthreads();
    seg_sums<1>(V, s_stage, 1, v_w, scale);
  }
  if (!grid_sync(A.bar)) return;
  {
    double d0[2];
    tree_total_cta<2>(A.part_a, A.nblk_sell, d0, s_tree);
    if (d0[0] == 0.0 || isnan(d0[0]) || isnan(d0[1]))
      status = KS_BREAKDOWN;
    else
      alpha = d0[1] / d0[0];
    gamma = d0[1];
    if (nc > 0) {
      double *const dW[1] = {cW};
      read_sums<1>(V, 1, 1, iscale, dW);
      __syncthreads();
    }
  }
  while (status == KS_RUNNING) {
    double *part = (it & 1) ? A.part_a : A.part_b;
    const int buf = (it + 2) % 3;  // phase it + 2
    const TS *ro = cur ? rv1 : rv0, *wo = cur ? wv1 : wv0, *so = cur ? sv1 : sv0;
    TS *rn = cur ? rv0 : rv1, *wn = cur ? wv0 : wv1, *sn = cur ? sv0 : sv1;
    // coarse input of the new residual and its coarse values
    if (nc > 0) {
      clear_acc(V, (it + 3) % 3);  // buffer of the next phase; last read before the previous barrier
      for (int m = threadIdx.x; m < nc; m += kCgResThreads) {
        const double sm = cW[m] + beta * cS[m];  // T(s) of the new s, by recurrence
        cS[m] = sm;
        ct[m] = cR[m] - alpha * sm;
      }
      __syncthreads();
      coarse_values<kZB>(V, ct, cc[pc ^ 1]);
      __syncthreads();
    }
    const double *cold = cc[pc], *cnew = cc[pc ^ 1];
    if constexpr (SPLIT) {
      // pass 1: own-row updates and u = D^-1 r_new + c_new[agg]; slots 0-2 take r.u, r.r, r.D^-1 r
      for (int b = b0 + g; b < b1; b += kCgResGroups) {
        const int lp = (b - b0) * kBlock + lt;
        const int i = s_row[lp];
        double v[3] = {0.0, 0.0, 0.0};
        if (i >= 0) {
          const int ai = __ldg(V.agg + i);
          const double mi = (double)__ldg(invLv + i);
          const double roi = (double)__ldcg(ro + i);
          const double woi = (double)__ldcg(wo + i), soi = (double)__ldcg(so + i);
          const double poi = (double)__ldcg(pv + i), xoi = (double)__ldcg(xv + i);
          const double uoi = mi * roi + cold[ai];
          const double pi = rnd(uoi + beta * poi);
          const double si = rnd(woi + beta * soi);
          const double xi = xoi + alpha * pi;
          const double ri = rnd(roi - alpha * si);
          const double ui = rnd(mi * ri + cnew[ai]);
          __stcg(pv + i, (TS)pi);
          __stcg(sn + i, (TS)si);
          __stcg(xv + i, (TS)xi);
          __stcg(rn + i, (TS)ri);
          __stcg(uv + i, (TS)ui);
          v[0] = ri * ui;
          v[1] = ri * ri;
          v[2] = ri * (mi * ri);
          if (nc > 0) {
            const int ps = __ldg(V.row_pos + i);
            if (ps >= 0) s_stage[ps] = ri;
          }
        }
        group_partial<3>(v, part, b, g, s_grp);
      }
      if (!grid_sync(A.bar)) return;
      // pass 2: w = A u (one gather per entry); slot 3 takes w.u
      for (int b = b0 + g; b < b1; b += kCgResGroups) {
        const int lp = (b - b0) * kBlock + lt;
        const int i = s_row[lp];
        double v[1] = {0.0};
        if (i >= 0) {
          const int base = s_base[lp], len = s_len[lp];
          const bool staged = b < bs;
          double acc = 0.0;
          int k = 0;
          for (; k + kCg2lChunk <= len; k += kCg2lChunk) {
            int jj[kCg2lChunk];
            double a[kCg2lChunk], uu[kCg2lChunk];
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q) {
              const int pos = base + (k + q) * kSellC;
              jj[q] = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
              a[q] = (double)__ldg(Lsv + pos);
            }
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q) uu[q] = (double)__ldcg(uv + jj[q]);
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q) acc += a[q] * uu[q];
          }
          if (k < len) {  // the last len % kCg2lChunk entries as one predicated chunk
            int jj[kCg2lChunk];
            double a[kCg2lChunk], uu[kCg2lChunk];
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q) {
              const int pos = base + (k + q) * kSellC;
              const bool in = k + q < len;
              jj[q] = !in ? 0 : staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
              a[q] = in ? (double)__ldg(Lsv + pos) : 0.0;
            }
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q) uu[q] = (k + q < len) ? (double)__ldcg(uv + jj[q]) : 0.0;
#pragma unroll
            for (int q = 0; q < kCg2lChunk; ++q)
              if (k + q < len) acc += a[q] * uu[q];
          }
          acc = rnd(acc);
          __stcg(wn + i, (TS)acc);
          v[0] = acc * (double)__ldcg(uv + i);
          if (nc > 0) {
            const int ps = __ldg(V.row_pos + i);
            if (ps >= 0) s_stage[V.npos_max + ps] = acc;
          }
        }
        group_partial<1>(v, part, b, g, s_grp, 3);
      }
    } else {
      for (int b = b0 + g; b < b1; b += kCgResGroups) {
        const int lp = (b - b0) * kBlock + lt;
        const int i = s_row[lp];
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        if (i >= 0) {
          const int base = s_base[lp], len = s_len[lp];
          const bool staged = b < bs;
          double acc = 0.0;
          int k = 0;
          for (; k + kCgChunk <= len; k += kCgChunk) {
            int jj[kCgChunk], aj[kCgChunk];
            double a[kCgChunk], rr_[kCgChunk], ww[kCgChunk], ss[kCgChunk], mm[kCgChunk];
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              const int pos = base + (k + q) * kSellC;
              jj[q] = staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
              a[q] = (double)__ldg(Lsv + pos);
            }
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              rr_[q] = (double)__ldcg(ro + jj[q]);
              ww[q] = (double)__ldcg(wo + jj[q]);
              ss[q] = (double)__ldcg(so + jj[q]);
              mm[q] = (double)__ldg(invLv + jj[q]);
              aj[q] = __ldg(V.agg + jj[q]);
            }
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              const double sj = ww[q] + beta * ss[q];
              const double rj = rr_[q] - alpha * sj;
              acc += a[q] * (mm[q] * rj + cnew[aj[q]]);
            }
          }
          if (k < len) {  // the last len % kCgChunk entries as one predicated chunk
            int jj[kCgChunk], aj[kCgChunk];
            double a[kCgChunk], rr_[kCgChunk], ww[kCgChunk], ss[kCgChunk], mm[kCgChunk];
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              const int pos = base + (k + q) * kSellC;
              const bool in = k + q < len;
              jj[q] = !in ? 0 : staged ? s_col[pos - e0] : __ldg(A.S.col + pos);
              a[q] = in ? (double)__ldg(Lsv + pos) : 0.0;
            }
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              const bool in = k + q < len;
              rr_[q] = in ? (double)__ldcg(ro + jj[q]) : 0.0;
              ww[q] = in ? (double)__ldcg(wo + jj[q]) : 0.0;
              ss[q] = in ? (double)__ldcg(so + jj[q]) : 0.0;
              mm[q] = in ? (double)__ldg(invLv + jj[q]) : 0.0;
              aj[q] = in ? __ldg(V.agg + jj[q]) : 0;
            }
  #pragma unroll
            for (int q = 0; q < kCgChunk; ++q) {
              const double sj = ww[q] + beta * ss[q];
              const double rj = rr_[q] - alpha * sj;
              if (k + q < len) acc += a[q] * (mm[q] * rj + cnew[aj[q]]);
            }
          }
          acc = rnd(acc);
          // own row
          const int ai = __ldg(V.agg + i);
          const double mi = (double)__ldg(invLv + i);
          const double roi = (double)__ldcg(ro + i);
          const double uoi = mi * roi + cold[ai];
          const double pi = rnd(uoi + beta * (double)__ldcg(pv + i));
          const double si = rnd((double)__ldcg(wo + i) + beta * (double)__ldcg(so + i));
          const double xi = (double)__ldcg(xv + i) + alpha * pi;
          const double ri = rnd(roi - alpha * si);
          const double ui = mi * ri + cnew[ai];
          __stcg(pv + i, (TS)pi);
          __stcg(sn + i, (TS)si);
          __stcg(xv + i, (TS)xi);
          __stcg(rn + i, (TS)ri);
          __stcg(wn + i, (TS)acc);
          v[0] = ri * ui;
          v[1] = acc * ui;
          v[2] = ri * ri;
          v[3] = ri * (mi * ri);
          if (nc > 0) {
            const int ps = __ldg(V.row_pos + i);
            if (ps >= 0) {
              s_stage[ps] = ri;
              s_stage[V.npos_max + ps] = acc;
            }
          }
        }
        group_partial<4>(v, part, b, g, s_grp);
      }
    }
    if (nc > 0) {
      __syncthreads();
      seg_sums<2>(V, s_stage, buf, v_rw, scale);
    }
    if (!grid_sync(A.bar)) return;
    double t[4];
    tree_total_cta<4>(part, A.nblk_sell, t, s_tree);
    if constexpr (SPLIT) {  // slots r.u, r.r, r.D^-1 r, w.u -> r.u, w.u, r.r, r.D^-1 r
      const double wu = t[3];
      t[3] = t[2];
      t[2] = t[1];
      t[1] = wu;
    }
    if (nc > 0) {
      double *const d2[2] = {cR, cW};
      read_sums<2>(V, buf, 0, iscale, d2);
      __syncthreads();
    }
    ++it;
    pc ^= 1;
    rn2 = A.scaled ? t[3] : t[2];
    cur ^= 1;
    if (isnan(t[0]) || isnan(t[1]) || isnan(t[2]) || isnan(t[3])) {
      status = KS_BREAKDOWN;
      break;
    }
    if (rn2 <= tol2) {
      status = KS_CONVERGED;
      break;
    }
    if (it >= maxit) {
      status = KS_MAXIT;
      break;
    }
    const double beta_new = t[0] / gamma;
    const double den = t[1] - beta_new * t[0] / alpha;
    if (den == 0.0) {
      status = KS_BREAKDOWN;
      break;
    }
    alpha = t[0] / den;
    beta = beta_new;
    gamma = t[0];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    CgState *c = A.cs;
    c->iters = it;
    c->rnorm2 = rn2;
    c->alpha = alpha;
    c->beta = beta;
    c->absnew = gamma;
    c->status = status;
    c->active = 0;
  }
}

// ------------------------------------------------------------------------------------------
// Host transfers of vector fields: the API's [N][3] node-major layout <-> the device's
// component-major [3][N], converted on the device so that the host side is one straight copy.
__global__ void k_vec3_interleave(int64_t n, const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * n) return;
  const int64_t i = k / 3, c = k - 3 * i;
  dst[k] = src[c * n + i];
}

__global__ void k_vec3_split(int64_t n, const double *__restrict__ src, double *__restrict__ dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 3 * n) return;
  const int64_t c = k / n, i = k - c * n;
  dst[k] = src[3 * i + c];
}

// ------------------------------------------------------------------------------------------
// p += relax_p p'; Dirichlet outlet reset (NavierStokes.cpp:652-662, reinforcePressureBCs
// :1011-1024). The pressure correction p' is the Krylov solution.
__global__ void k_pressure_update(int nv, double relax_p, int outlet_type, double outlet_pressure,
                                  const signed char *__restrict__ bc, const double *__restrict__ pc,
                                  double *__restrict__ p, const DevStatus *__restrict__ st) {
  if (st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double v = p[i] + relax_p * pc[i];
  if (outlet_type == 0 && bc[i] == BC_OUTLET) v = outlet_pressure;
  p[i] = v;
}

// normalizePressire (NavierStokes.cpp:804-813): p -= p[ref] (ref value stashed first).
__global__ void k_pressure_stash(int ref, const double *__restrict__ p, double *__restrict__ stash,
                                 const DevStatus *__restrict__ st) {
  if (st->halt) return;
  *stash = p[ref];
}
__global__ void k_pressure_normalize(int nv, const double *__restrict__ stash,
                                     double *__restrict__ p, const DevStatus *__restrict__ st) {
  if (st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  p[i] -= *stash;
}

// correctVelocity (NavierStokes.cpp:702-771).
struct CorrectArgs {
  CsrView G;
  const double *Gv;
  int64_t nnz1;
  const double *invm, *pc, *ustar, *inlet;
  const signed char *bc;
  double dt, relax_u;
  int n, nv;
  double *u;
  const DevStatus *st;
};

__global__ void k_correct_velocity(CorrectArgs A) {
  if (A.st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  const int bcv = A.bc[i];
  double out[3];
  if (bcv == BC_INLET) {
    for (int c = 0; c < 3; ++c) out[c] = A.inlet[c * n + i];
  } else if (bcv == BC_WALL) {
    out[0] = out[1] = out[2] = 0.0;
  } else if (i < A.nv && A.invm[i] > 1e-14) {
    double g[3] = {0.0, 0.0, 0.0};
    for (int k = A.G.rp[i]; k < A.G.rp[i + 1]; ++k) {
      const double pj = A.pc[A.G.ci[k]];
      g[0] += A.Gv[k] * pj;
      g[1] += A.Gv[A.nnz1 + k] * pj;
      g[2] += A.Gv[2 * A.nnz1 + k] * pj;
    }
    const double f = -A.dt * A.invm[i];
    for (int c = 0; c < 3; ++c) out[c] = A.ustar[c * n + i] + A.relax_u * (f * g[c]);
  } else {
    for (int c = 0; c < 3; ++c) out[c] = A.ustar[c * n + i];
  }
  for (int c = 0; c < 3; ++c) A.u[c * n + i] = out[c];
}

// End of step: reenforceVelocityBCs (NavierStokes.cpp:815-839) and hasNans
// (NavierStokes.hpp:116-138) over u, u*, p, p'; records the step in the status.
struct FinishArgs {
  const signed char *bc;
  const double *inlet;
  double *u;
  const double *ustar, *p, *pc;
  int n, nv;
  DevStatus *st;
  Reduce red;
};

__global__ void k_finish_step(FinishArgs A) {
  if (A.st->halt) return;
  // one resident wave visiting 256-position blocks (one reduction ticket per CTA)
  __shared__ WarpSums<1> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x, ++slot) {
    const int i = blk * kBlock + threadIdx.x;
    double part[1] = {0.0};
    if (i < A.n) {
      const int64_t n = A.n;
      const int bcv = A.bc[i];
      bool nan = false;
      for (int c = 0; c < 3; ++c) {
        double ui = A.u[c * n + i];
        if (bcv == BC_INLET) {
          ui = A.inlet[c * n + i];
          A.u[c * n + i] = ui;
        } else if (bcv == BC_WALL) {
          ui = 0.0;
          A.u[c * n + i] = ui;
        }
        nan |= isnan(ui) || isnan(A.ustar[c * n + i]);
      }
      if (i < A.nv) nan |= isnan(A.p[i]) || isnan(A.pc[i]);
      part[0] = nan ? 1.0 : 0.0;
    }
    warp_partial<1>(part, S, slot);
  }
  double tot[1];
  if (grid_reduce_strided<1>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    A.st->steps_done += 1;
    if (tot[0] > 0.0) {
      A.st->nan = 1;
      if (A.st->code == 0) A.st->code = 3;
      A.st->halt = 1;
    }
  }
}

// ------------------------------------------------------------------------------------------
// Boundary-face forces (computePressureForces / computeShearStress, NavierStokes.cpp:841-944):
// per-face force, then a per-vertex gather over the vertex's boundary faces in face order.
__global__ void k_face_forces(int nbf, int nt, int64_t n2, double mu, const int *__restrict__ fverts,
                              const int *__restrict__ ftet, const double *__restrict__ fnormal,
                              const double *__restrict__ farea, const int *__restrict__ tnode,
                              const double *__restrict__ grad, const double *__restrict__ u,
                              const double *__restrict__ p, double *__restrict__ fshear,
                              double *__restrict__ fpress) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nbf) return;
  const double nx = fnormal[3 * f], ny = fnormal[3 * f + 1], nz = fnormal[3 * f + 2];
  const double area = farea[f];
  double fp = 0.0;
  for (int k = 0; k < 3; ++k) fp += p[fverts[3 * f + k]];
  fp /= 3.0;
  fpress[3 * f] = -fp * nx * area;
  fpress[3 * f + 1] = -fp * ny * area;
  fpress[3 * f + 2] = -fp * nz * area;
  const int t = ftet[f];
  double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (int a = 0; a < 4; ++a) {
    const int v = tnode[(size_t)a * nt + t];
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y) gu[x][y] += u[x * n2 + v] * grad[(size_t)(3 * a + y) * nt + t];
  }
  const double nrm[3] = {nx, ny, nz};
  for (int x = 0; x < 3; ++x) {
    double tr = 0.0;
    double tau[3];
    for (int y = 0; y < 3; ++y) tau[y] = 2.0 * mu * (0.5 * (gu[x][y] + gu[y][x]));
    tr = (tau[0] * nrm[0] + tau[1] * nrm[1]) + tau[2] * nrm[2];
    fshear[3 * f + x] = tr * area;
  }
}

__global__ void k_face_gather(int nv, const int *__restrict__ vf_ptr, const int *__restrict__ vf,
                              const double *__restrict__ fval, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  double a[3] = {0.0, 0.0, 0.0};
  for (int q = vf_ptr[i]; q < vf_ptr[i + 1]; ++q) {
    const int f = vf[q];
    for (int c = 0; c < 3; ++c) a[c] += fval[3 * f + c] * (1.0 / 3.0);
  }
  for (int c = 0; c < 3; ++c) out[3 * i + c] = a[c];
}

}  // namespace cfsa
