// Discrete adjoint of the PISO step (pisoStep, NavierStokes.cpp:374-414, as implemented by the
// forward kernels): reverse-mode kernels, objective seeds and the transposed-slot map.
//
// One forward step n maps (u^n, p^n; g, nu) to (u^{n+1}, p^{n+1}), g the inlet values and nu
// the viscosity (stiffness K = K_hat / nu, NavierStokes.cpp:153):
//   conv = C(u^n)                                   (per-tet c_t = grad(u) u_mean, P1 velocities)
//   A u*_a = M u^n_a / dt - E G_a p^n + conv_a + P g_a,   A = M/dt + K + P (penalty rows P)
//   L_bc p' = -(1/dt) sum_a G_a u*_a|P1 + const
//   p^{n+1} = Pi(p^n + relax_p p')   once per corrector (Pi: outlet reset, reference shift)
//   u^{n+1} = F u* - relax_u dt F m^-1 E G p' + chi_in g   (F: rows that are not inlet/wall)
// The reverse step takes (lambda_u, lambda_p) = dJ/d(u^{n+1}, p^{n+1}) to dJ/d(u^n, p^n) and
// accumulates dJ/dg and dJ/dnu; every Krylov solve is taken as the exact linear solve it
// converges to. M, K and L_bc are symmetric, so the adjoint solves run the forward Krylov
// kernels on the forward operators; G_a^T is applied through the transposed-slot map.
// All kernels are gathers with fixed summation orders: the reverse pass is deterministic.
#pragma once

#include "ns_kernels.cuh"

namespace cfsa {

// Transposed slot of each entry of a structurally symmetric CSR pattern. err is set when a
// transposed entry is missing.
__global__ void k_transpose_slots(int64_t nnz, const int *__restrict__ rows, const int *__restrict__ rp,
                                  const int *__restrict__ ci, int *__restrict__ tpos,
                                  int *__restrict__ err) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  const int i = rows[k], j = ci[k];
  const int beg = rp[j], end = rp[j + 1];
  const int q = (end > beg) ? find_col(ci, beg, end, i) : beg;
  if (end > beg && ci[q] == i) {
    tpos[k] = q;
  } else {
    tpos[k] = (int)k;
    atomicExch(err, 1);
  }
}

// Reverse of correctVelocity + reenforceVelocityBCs (NavierStokes.cpp:702-771, 815-839):
// lus = F lambda_u (the momentum adjoint right-hand side before the divergence term),
// gin += lambda_u on inlet rows, q_a = relax_u (-dt m^-1) lambda_u,a on free P1 rows.
struct AdjCorrectArgs {
  const double *lu;
  const signed char *bc;
  const double *invm;
  double dt, relax_u;
  int n, nv;
  double *lus, *gin, *q;
  const DevStatus *st;
};

__global__ void k_adj_correct(AdjCorrectArgs A) {
  if (A.st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n, nv = A.nv;
  const int bcv = A.bc[i];
  double l[3], ls[3] = {0.0, 0.0, 0.0}, q[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int c = 0; c < 3; ++c) l[c] = A.lu[c * n + i];
  if (bcv == BC_INLET) {
#pragma unroll
    for (int c = 0; c < 3; ++c) A.gin[c * n + i] = A.gin[c * n + i] + l[c];
  } else if (bcv != BC_WALL) {
#pragma unroll
    for (int c = 0; c < 3; ++c) ls[c] = l[c];
    if (i < A.nv && A.invm[i] > 1e-14) {
      const double f = -A.dt * A.invm[i];
#pragma unroll
      for (int c = 0; c < 3; ++c) q[c] = A.relax_u * (f * l[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) A.lus[c * n + i] = ls[c];
  if (i < A.nv)
#pragma unroll
    for (int c = 0; c < 3; ++c) A.q[c * nv + i] = q[c];
}

// Deterministic sum of x[0..n) into *out (the reference-node shift of normalizePressire).
__global__ void k_adj_sum(int n, const double *__restrict__ x, double *__restrict__ out, Reduce red,
                          const DevStatus *__restrict__ st) {
  if (st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part[1] = {i < n ? x[i] : 0.0};
  double tot[1];
  if (grid_reduce<1>(part, red, tot) && threadIdx.x == 0) *out = tot[0];
}

// Reverse of one corrector's pressure update p = Pi(p + relax_p p') (NavierStokes.cpp:652-666,
// 804-813, 1011-1024): w = Pi^T chain; lpp += relax_p w; chain = w. Pi^T applies the
// reference-shift transpose (chain_ref -= sum(chain), S from k_adj_sum) and then zeroes the
// Dirichlet outlet rows.
struct AdjChainArgs {
  double *chain, *lpp;
  const double *S;  // nullptr: no reference-node normalisation
  const signed char *bc;
  double relax_p;
  int nv, ref_node, dirichlet, first;
  const DevStatus *st;
};

__global__ void k_adj_pchain(AdjChainArgs A) {
  if (A.st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nv) return;
  double w = A.chain[i];
  if (A.S && i == A.ref_node) w = w - *A.S;
  if (A.dirichlet && A.bc[i] == BC_OUTLET) w = 0.0;
  A.lpp[i] = (A.first ? 0.0 : A.lpp[i]) + A.relax_p * w;
  A.chain[i] = w;
}

// Per-tet data of the convection adjoint (computeAdvectionRHS, NavierStokes.cpp:550-580) with
// nu the momentum adjoint: c_hat = -(V/4 sum_vertices nu + V/24 sum_edge_nodes nu), the mean
// vertex velocity u_mean and h = (1/4) grad(u)^T c_hat. A vertex j of the tet then receives
// c_hat (grad phi_j . u_mean) + h. tsc layout [9][nt]: c_hat, u_mean, h.
__global__ void k_adj_conv_tet(int nt, int64_t n2, int64_t nv, const int *__restrict__ tnode,
                               const double *__restrict__ grad, const double *__restrict__ vol,
                               const double *__restrict__ nu, const double *__restrict__ un,
                               double *__restrict__ tsc, const DevStatus *__restrict__ st) {
  if (st->halt) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double s1[3] = {0.0, 0.0, 0.0}, s2[3] = {0.0, 0.0, 0.0};
  double uv[4][3];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const int v = tnode[(size_t)l * nt + t];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      s1[c] = s1[c] + nu[c * n2 + v];
      uv[l][c] = un[c * nv + v];
    }
  }
#pragma unroll
  for (int e = 0; e < 6; ++e) {
    const int v = tnode[(size_t)(4 + e) * nt + t];
#pragma unroll
    for (int c = 0; c < 3; ++c) s2[c] = s2[c] + nu[c * n2 + v];
  }
  const double V = vol[t];
  double ch[3], ue[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int c = 0; c < 3; ++c) ch[c] = -((V / 4.0) * s1[c] + (V / 24.0) * s2[c]);
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int c = 0; c < 3; ++c) ue[c] = ue[c] + 0.25 * uv[l][c];
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
  for (int c = 0; c < 3; ++c) {
    tsc[(size_t)c * nt + t] = ch[c];
    tsc[(size_t)(3 + c) * nt + t] = ue[c];
    tsc[(size_t)(6 + c) * nt + t] =
        0.25 * ((gu[0][c] * ch[0] + gu[1][c] * ch[1]) + gu[2][c] * ch[2]);
  }
}

// Reverse of the momentum right-hand side (NavierStokes.cpp:429-495) on SELL rows of the P2
// pattern, given nu = A^-1 lus:
//   lambda_u^n = M nu / dt + (convection adjoint on P1 rows)
//   lambda_p^n = chain - sum_a G_a^T nu_a|P1       (chain: Pi^T-propagated lambda_p)
//   gin += penalty * nu on inlet rows
//   dJ/dnu += sum_a nu_a . K u*_a / nu              (dA/dnu = -K/nu)
struct AdjMomOutArgs {
  SellView S;
  const double *Ms;
  CsrView K;  // P2 CSR pattern
  const double *Kv;
  CsrView G;
  const int *tpos;
  const double *Gv;
  int64_t nnz1;
  const int *adj_ptr, *adj;
  const double *grad;
  const double *tsc;
  const signed char *bc;
  const double *nu, *us;
  double dt, viscosity;
  int n, nv, nt;
  double *lu, *lp, *gin, *gnu;
  Reduce red;
  const DevStatus *st;
};

__global__ void k_adj_mom_out(AdjMomOutArgs A) {
  if (A.st->halt) return;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
  double part[1] = {0.0};
  if (i >= 0) {
    const int64_t n = A.n;
    double mv[3];
    sell_spmv_row<3>(A.S, A.Ms, A.nu, n, r, mv);
    double ca[3] = {0.0, 0.0, 0.0};
    if (i < A.nv) {
      for (int q = A.adj_ptr[i]; q < A.adj_ptr[i + 1]; ++q) {
        const int t = A.adj[q] >> 4, l = A.adj[q] & 15;
        double d = 0.0;
        {
          const double g0 = A.grad[(size_t)(3 * l) * A.nt + t];
          const double g1 = A.grad[(size_t)(3 * l + 1) * A.nt + t];
          const double g2 = A.grad[(size_t)(3 * l + 2) * A.nt + t];
          d = (g0 * A.tsc[(size_t)3 * A.nt + t] + g1 * A.tsc[(size_t)4 * A.nt + t]) +
              g2 * A.tsc[(size_t)5 * A.nt + t];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c)
          ca[c] = ca[c] + (A.tsc[(size_t)c * A.nt + t] * d + A.tsc[(size_t)(6 + c) * A.nt + t]);
      }
    }
    double nv3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      nv3[c] = A.nu[c * n + i];
      double v = mv[c] / A.dt;
      if (i < A.nv) v = v + ca[c];
      A.lu[c * n + i] = v;
    }
    if (A.bc[i] == BC_INLET)
#pragma unroll
      for (int c = 0; c < 3; ++c) A.gin[c * n + i] = A.gin[c * n + i] + kMomentumPenalty * nv3[c];
    double ku[3] = {0.0, 0.0, 0.0};
    for (int k = A.K.rp[i]; k < A.K.rp[i + 1]; ++k) {
      const int j = A.K.ci[k];
      const double kv = A.Kv[k];
#pragma unroll
      for (int c = 0; c < 3; ++c) ku[c] += kv * A.us[c * n + j];
    }
    part[0] = (nv3[0] * ku[0] + nv3[1] * ku[1]) + nv3[2] * ku[2];
    if (i < A.nv) {
      double g[3];
      gt_row3(i, A.G.rp, A.G.ci, A.tpos, A.Gv, A.nnz1, A.nu, A.nu + n, A.nu + 2 * n, g);
      A.lp[i] = A.lp[i] - ((g[0] + g[1]) + g[2]);
    }
  }
  double tot[1];
  if (grid_reduce<1>(part, A.red, tot) && threadIdx.x == 0) *A.gnu = *A.gnu + tot[0] / A.viscosity;
}

// ------------------------------------------------------------------------------------------
// Objectives on the current state.
//
// Wall-shear patch: J = (1/|P|) sum_{v in P} |s_v|^2 with s the per-vertex wall traction of
// computeShearStress (NavierStokes.cpp:874-944, mu = viscosity) and P the wall vertices inside
// the patch mask. Seed: w_v = (2/|P|) s_v; a boundary face f with tet t carries
// W_f = (w_0 + w_1 + w_2) A_f / 3, and vertex j of t receives mu((n_f . grad phi_j) W_f +
// (W_f . grad phi_j) n_f). Explicit dJ/dnu = 2 J / nu.
__global__ void k_obj_wss_value(int nv, const double *__restrict__ s, const signed char *__restrict__ mask,
                                double inv_np, double viscosity, double *__restrict__ w,
                                double *__restrict__ J, double *__restrict__ gnu, Reduce red) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part[1] = {0.0};
  if (i < nv) {
    double wv[3] = {0.0, 0.0, 0.0};
    if (mask[i]) {
      const double s0 = s[3 * i], s1 = s[3 * i + 1], s2 = s[3 * i + 2];
      part[0] = (s0 * s0 + s1 * s1) + s2 * s2;
      const double c = 2.0 * inv_np;
      wv[0] = c * s0;
      wv[1] = c * s1;
      wv[2] = c * s2;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) w[3 * i + c] = wv[c];
  }
  double tot[1];
  if (grid_reduce<1>(part, red, tot) && threadIdx.x == 0) {
    const double j = tot[0] * inv_np;
    *J = j;
    *gnu = 2.0 * j / viscosity;
  }
}

__global__ void k_obj_wss_face(int nbf, const int *__restrict__ fverts, const double *__restrict__ farea,
                               const double *__restrict__ w, double *__restrict__ W) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nbf) return;
  const int v0 = fverts[3 * f], v1 = fverts[3 * f + 1], v2 = fverts[3 * f + 2];
  const double s = farea[f] * (1.0 / 3.0);
#pragma unroll
  for (int c = 0; c < 3; ++c) W[3 * f + c] = ((w[3 * v0 + c] + w[3 * v1 + c]) + w[3 * v2 + c]) * s;
}

// Seed gather: vertex v over the (boundary face, local index in the face's tet) pairs of the
// faces whose tet contains v, ascending face order (vbf entry = face * 4 + local index).
__global__ void k_obj_wss_seed(int nv, int64_t n2, int nt, const int *__restrict__ vbf_ptr,
                               const int *__restrict__ vbf, const int *__restrict__ ftet,
                               const double *__restrict__ fnormal, const double *__restrict__ grad,
                               const double *__restrict__ W, double mu, double *__restrict__ lu) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n2) return;
  double acc[3] = {0.0, 0.0, 0.0};
  if (i < nv) {
    for (int q = vbf_ptr[i]; q < vbf_ptr[i + 1]; ++q) {
      const int f = vbf[q] >> 2, l = vbf[q] & 3, t = ftet[f];
      const double g0 = grad[(size_t)(3 * l) * nt + t], g1 = grad[(size_t)(3 * l + 1) * nt + t],
                   g2 = grad[(size_t)(3 * l + 2) * nt + t];
      const double n0 = fnormal[3 * f], n1 = fnormal[3 * f + 1], n2v = fnormal[3 * f + 2];
      const double W0 = W[3 * f], W1 = W[3 * f + 1], W2 = W[3 * f + 2];
      const double ng = (n0 * g0 + n1 * g1) + n2v * g2;
      const double wg = (W0 * g0 + W1 * g1) + W2 * g2;
      acc[0] = acc[0] + mu * (W0 * ng + n0 * wg);
      acc[1] = acc[1] + mu * (W1 * ng + n1 * wg);
      acc[2] = acc[2] + mu * (W2 * ng + n2v * wg);
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) lu[c * n2 + i] = acc[c];
}

// Pressure drop: J = mean p over inlet vertices - mean p over outlet vertices; seed
// lambda_p = chi_in / n_in - chi_out / n_out.
__global__ void k_obj_pdrop(int nv, const double *__restrict__ p, const signed char *__restrict__ bc,
                            double inv_in, double inv_out, double *__restrict__ lp,
                            double *__restrict__ J, Reduce red) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part[2] = {0.0, 0.0};
  if (i < nv) {
    const int b = bc[i];
    double s = 0.0;
    if (b == BC_INLET) {
      part[0] = p[i];
      s = inv_in;
    }
    if (b == BC_OUTLET) {
      part[1] = p[i];
      s = -inv_out;
    }
    lp[i] = s;
  }
  double tot[2];
  if (grid_reduce<2>(part, red, tot) && threadIdx.x == 0) *J = tot[0] * inv_in - tot[1] * inv_out;
}

}  // namespace cfsa
