// Mixed-precision momentum solve: one batched BiCGSTAB sequence in FP32 with reliable updates
// of the solution and the residual in FP64 (residual replacement: van der Vorst & Ye, SIAM J. Sci.
// Comput. 22(5), 2000; group-wise solution updates: Sleijpen & van der Vorst, Computing 56, 1996;
// their mixed-precision GPU form: Clark et al., Comput. Phys. Commun. 181, 2010).
//
//   FP64: b, x (solution), r64 (true residual), xs = diag(A) x
//   FP32: r, r0, p, v, s, t (Krylov vectors), dx (correction accumulated since the last update)
//   every iteration (FP32 operator At32 = FP32 copy of A D^-1, FP64 dot products and scalars):
//     p = r + beta (p - omega v); v = At32 p; alpha = rho / (r0.v); s = r - alpha v;
//     t = At32 s; omega = (t.s) / (t.t); dx += alpha D^-1 p + omega D^-1 s; r = s - omega t
//   reliable update of component c when its iterated residual has dropped below delta times the
//   largest one since its last update, meets the tolerance, hits the iteration cap or nears a
//   breakdown:  x += dx; dx = 0; r64 = b - A x (FP64 operator); r = (float) r64
// The Krylov space is kept across updates (p, r0 and the scalars carry on), so the iteration
// count stays that of the FP64 solve instead of restarting with every correction. Convergence is
// decided on the FP64 true residual only, with the FP64 solve's criterion. In a CUDA graph the
// update is a conditional IF node inside the iteration's WHILE body, so iterations without an
// update launch nothing extra. The penalty rows (diagonal 1e10) have unit diagonal in A D^-1, so
// FP32 holds them without overflow or loss. Components are independent (per-component scalars,
// masks and updates).
#pragma once

#include "ns_kernels.cuh"

namespace cfsa {

constexpr double kMixedDrift2 = 100.0;  // true / iterated residual (squared) that restarts the space

struct MixedState {
  double bnorm2[3], tol2[3], rnorm2[3];  // FP64 criterion; rnorm2: true residual at the last update
  double rho[3], alpha[3], omega[3], beta[3], r0norm2[3];
  double rin2[3];   // iterated FP32 residual, same norm
  double rmax2[3];  // largest iterated residual since the last update
  int iters[3], status[3], updates[3];
  int active;   // components iterating
  int upd;      // components updated at the end of this iteration
  int restart;  // components whose Krylov space restarts at that update (near-breakdown)
  int restart_next;  // components restarting at the next iteration (the FP32 recurrence drifted)
  int force;         // components whose r0 . v vanished: update and restart at this iteration's end
  int maxit;
  double delta2;  // update trigger: rin2 < delta2 * rmax2
  int restarts[3];  // Krylov-space restarts (drift or a growing true residual)
};

struct MixedArgs {
  SellView S;
  const float *At32;
  const double *At64, *diagA, *invA;
  const float *invA32;
  const double *b;
  double *x, *r64, *xs;  // FP64 solution, true residual, scaled solution D x
  float *r, *r0, *p, *v, *s, *t, *dx;
  int n;
  MixedState *ms;
  DevStatus *st;
  Reduce red;
  cudaGraphConditionalHandle cond;      // WHILE node of the iteration
  cudaGraphConditionalHandle cond_upd;  // IF node of the reliable update
  int use_cond;
  int use_if;  // cond_upd is a live IF node (otherwise the update kernels run every iteration)
  const double *cw;   // convergence-norm weights (diag(A)^-1), nullptr: unscaled ||r||
  const float *cw32;  // the same for the FP32 residual
};

template <int U = 8, int MASK = 7>
__device__ __forceinline__ void sell_spmv_row_f32x3(const SellView &S, const float *__restrict__ val,
                                                    const float *__restrict__ x, int64_t n, int r,
                                                    float acc[3]) {
  const int base = S.sptr[r >> 5] + (r & 31), len = S.len[r];
  acc[0] = acc[1] = acc[2] = 0.f;
  int k = 0;
  for (; k + U <= len; k += U) {
    int j[U];
    float a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int pos = base + (k + u) * kSellC;
      j[u] = __ldcs(S.col + pos);
      a[u] = __ldcs(val + pos);
    }
    float xv[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if ((MASK >> c) & 1) xv[u][c] = __ldg(x + c * n + j[u]);
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if ((MASK >> c) & 1) acc[c] += a[u] * xv[u][c];
  }
  if (k < len) {  // the last len % U entries as one predicated chunk: one memory round trip
    int j[U];
    float a[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int pos = base + (k + u) * kSellC;
      const bool in = k + u < len;
      j[u] = in ? __ldcs(S.col + pos) : 0;
      a[u] = in ? __ldcs(val + pos) : 0.f;
    }
    float xv[U][3];
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if ((MASK >> c) & 1) xv[u][c] = (k + u < len) ? __ldg(x + c * n + j[u]) : 0.f;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (((MASK >> c) & 1) && k + u < len) acc[c] += a[u] * xv[u][c];
  }
}


// Init (after k_momentum_rhs wrote b and x = 0): r = r0 = (float) b, p = v = dx = 0;
// FP64 ||b|| in the convergence norm, rho = r0 . r.
__global__ void k_mp_init(MixedArgs A, double tol, int maxit, double delta) {
  if (A.st->halt) return;
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int bk = blockIdx.x; bk < nblk; bk += gridDim.x, ++slot) {
    const int i = bk * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const double w = A.cw ? A.cw[i] : 1.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t o = c * n + i;
        const double bi = A.b[o];
        const float ri = (float)bi;
        A.r[o] = ri;
        A.r0[o] = ri;
        A.p[o] = 0.f;
        A.v[o] = 0.f;
        A.dx[o] = 0.f;
        part[c] = (bi * bi) * w;
        part[3 + c] = (double)ri * (double)ri;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    m->active = 0;
    m->upd = 0;
    m->restart = 0;
    m->restart_next = 0;
    m->force = 0;
    m->maxit = maxit;
    m->delta2 = delta * delta;
    for (int c = 0; c < 3; ++c) {
      m->bnorm2[c] = tot[c];
      m->rnorm2[c] = tot[c];
      m->rin2[c] = tot[c];
      m->rmax2[c] = tot[c];
      m->tol2[c] = tol * tol * tot[c];
      m->rho[c] = tot[3 + c];
      m->r0norm2[c] = tot[3 + c];
      m->alpha[c] = m->omega[c] = 1.0;
      m->beta[c] = 0.0;
      m->iters[c] = 0;
      m->updates[c] = 0;
      m->restarts[c] = 0;
      if (isnan(tot[c]) || isnan(tot[3 + c])) {
        m->status[c] = KS_BREAKDOWN;
      } else if (tot[c] == 0.0 || tot[c] <= m->tol2[c]) {
        m->status[c] = KS_CONVERGED;
      } else {
        m->status[c] = KS_RUNNING;
        m->active |= 1 << c;
      }
    }
  }
}

// K1: p = r + beta (p - omega v)  (beta = 0 after a restart: p = r). Components whose FP32
// recurrence drifted from the true residual (flagged by the last update) restart here instead:
// r0 = p = r and rho = r0 . r, the one reduction of this kernel (taken only when a restart is due).
__global__ void k_mp_p(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int rs = A.ms->restart_next & act;
  float beta[3], omega[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) beta[c] = (float)A.ms->beta[c], omega[c] = (float)A.ms->omega[c];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = A.n;
  double part[3] = {0.0, 0.0, 0.0};
  if (i < A.n) {
    float rv[3], pv[3], vv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((act >> c) & 1) rv[c] = A.r[c * n + i], pv[c] = A.p[c * n + i], vv[c] = A.v[c * n + i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      const int64_t o = c * n + i;
      if ((rs >> c) & 1) {
        A.p[o] = rv[c];
        A.r0[o] = rv[c];
        part[c] = (double)rv[c] * (double)rv[c];
      } else {
        A.p[o] = rv[c] + beta[c] * (pv[c] - omega[c] * vv[c]);
      }
    }
  }
  if (!rs) return;
  double tot[3];
  if (grid_reduce<3>(part, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    for (int c = 0; c < 3; ++c)
      if ((rs >> c) & 1) {
        m->rho[c] = tot[c];
        m->r0norm2[c] = tot[c];
        m->restarts[c] += 1;
      }
    m->restart_next = 0;
  }
}

// K2: v = At32 p, alpha = rho / (r0 . v)
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_v(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<3>(act, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[3] = {0.0, 0.0, 0.0};
      if (i >= 0) {
        float acc[3];
        sell_spmv_row_f32x3<8, MASK>(A.S, A.At32, A.p, n, r, acc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!((MASK >> c) & 1)) continue;
          A.v[c * n + i] = acc[c];
          part[c] = (double)A.r0[c * n + i] * (double)acc[c];
        }
      }
      slice_partial<3>(part, A.S, sl);
    }
  });
  double tot[3];
  if (grid_reduce_runs<3>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      if (isnan(tot[c])) {
        A.ms->status[c] = KS_BREAKDOWN;
        A.ms->active &= ~(1 << c);
      } else if (tot[c] == 0.0) {
        // r0 . v vanished: no step along p; the iteration ends in an update and a restart
        A.ms->alpha[c] = 0.0;
        A.ms->force |= 1 << c;
      } else {
        A.ms->alpha[c] = A.ms->rho[c] / tot[c];
      }
    }
  }
}

// K3: s = r - alpha v
__global__ void k_mp_s(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  float alpha[3], rv[3], vv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    alpha[c] = (float)A.ms->alpha[c];
    if ((act >> c) & 1) rv[c] = A.r[c * n + i], vv[c] = A.v[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if ((act >> c) & 1) A.s[c * n + i] = rv[c] - alpha[c] * vv[c];
}

// K4: t = At32 s, omega = (t . s) / (t . t)
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_t(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<3>(act, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (i >= 0) {
        float acc[3];
        sell_spmv_row_f32x3<8, MASK>(A.S, A.At32, A.s, n, r, acc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!((MASK >> c) & 1)) continue;
          A.t[c * n + i] = acc[c];
          part[c] = (double)acc[c] * (double)acc[c];
          part[3 + c] = (double)acc[c] * (double)A.s[c * n + i];
        }
      }
      slice_partial<6>(part, A.S, sl);
    }
  });
  double tot[6];
  if (grid_reduce_runs<6>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      A.ms->omega[c] = (tot[c] > 0.0) ? tot[3 + c] / tot[c] : 0.0;
    }
  }
}

// K5: dx += alpha D^-1 p + omega D^-1 s, r = s - omega t; ||r||, r0 . r; which components take a
// reliable update at the end of this iteration (IF node), next beta for the others.
__global__ void k_mp_xr(MixedArgs A) {
  const int act = A.ms->active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[0] += 1;
  if (!act) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) {
      if (A.use_if) cudaGraphSetConditional(A.cond_upd, 0);
      cudaGraphSetConditional(A.cond, 0);
    }
    return;
  }
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  float alpha_c[3], omega_c[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) alpha_c[c] = (float)A.ms->alpha[c], omega_c[c] = (float)A.ms->omega[c];
  int slot = 0;
  for (int bk = blockIdx.x; bk < nblk; bk += gridDim.x, ++slot) {
    const int i = bk * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const float dinv = A.invA32[i];
      const double w = A.cw32 ? (double)A.cw32[i] : 1.0;
      float pv[3], sv[3], tv[3], dxv[3], r0v[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        const int64_t o = c * n + i;
        pv[c] = A.p[o], sv[c] = A.s[o], tv[c] = A.t[o], dxv[c] = A.dx[o], r0v[c] = A.r0[o];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        const int64_t o = c * n + i;
        A.dx[o] = dxv[c] + (alpha_c[c] * (dinv * pv[c]) + omega_c[c] * (dinv * sv[c]));
        const float ri = sv[c] - omega_c[c] * tv[c];
        A.r[o] = ri;
        part[c] = ((double)ri * (double)ri) * w;
        part[3 + c] = (double)r0v[c] * (double)ri;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    const double eps = 2.220446049250313e-16;
    int upd = 0, rst = 0, live = 0;
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      m->iters[c] += 1;
      m->rin2[c] = tot[c];
      const double rho_new = tot[3 + c];
      if (isnan(tot[c]) || isnan(rho_new)) {
        m->status[c] = KS_BREAKDOWN;
        m->active &= ~(1 << c);
        continue;
      }
      live |= 1 << c;
      // near-breakdown, a vanished omega or r0 . v: the FP32 space is exhausted; the update
      // replaces the residual and the Krylov space restarts from it
      const bool restart = fabs(rho_new) < eps * eps * m->r0norm2[c] || m->omega[c] == 0.0 ||
                           ((m->force >> c) & 1);
      if (tot[c] <= m->tol2[c] || m->iters[c] >= m->maxit || tot[c] < m->delta2 * m->rmax2[c] || restart) {
        upd |= 1 << c;
        if (restart) rst |= 1 << c;
      }
    }
    // Components update on their own triggers only: replacing a residual before it has dropped by
    // delta perturbs BiCGSTAB's recurrences, and on the 4M-tet Y-bifurcation updates brought
    // forward to share one FP64 product made the iteration erratic until it hit the cap.
    for (int c = 0; c < 3; ++c) {
      if (!(((live & ~upd) >> c) & 1)) continue;
      const double rho_new = tot[3 + c];
      m->beta[c] = (rho_new / m->rho[c]) * (m->alpha[c] / m->omega[c]);
      m->rho[c] = rho_new;
      m->rmax2[c] = fmax(m->rmax2[c], tot[c]);
    }
    m->upd = upd;
    m->restart = rst;
    m->force = 0;
    if (A.use_cond) {
      if (A.use_if) cudaGraphSetConditional(A.cond_upd, upd ? 1u : 0u);
      cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
    }
  }
}

// Reliable update, part 1: x += dx (FP64), dx = 0, xs = diag(A) x for the updated components.
__global__ void k_mp_xupdate(MixedArgs A) {
  const int upd = A.ms->upd;
  if (!upd) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  const double d = A.diagA[i];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((upd >> c) & 1)) continue;
    const int64_t o = c * n + i;
    const double xi = A.x[o] + (double)A.dx[o];
    A.x[o] = xi;
    A.dx[o] = 0.f;
    A.xs[o] = d * xi;
  }
}

// Reliable update, part 2: r64 = b - At64 (D x) (FP64 true residual), r = (float) r64 (and r0 = r
// for a restart); convergence on the true residual, next beta from the replaced residual.
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_residual(MixedArgs A) {
  const int upd = A.ms->upd;
  if (!upd) return;
  const int rst = A.ms->restart;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[2] += 1;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<3>(upd, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (i >= 0) {
        double acc[3];
        sell_spmv_row<3, kU64, MASK>(A.S, A.At64, A.xs, n, r, acc);
        const double w = A.cw ? A.cw[i] : 1.0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!((MASK >> c) & 1)) continue;
          const int64_t o = c * n + i;
          const double ri = A.b[o] - acc[c];
          A.r64[o] = ri;
          const float rf = (float)ri;
          A.r[o] = rf;
          float r0 = A.r0[o];
          if ((rst >> c) & 1) {
            r0 = rf;
            A.r0[o] = rf;
          }
          part[c] = (ri * ri) * w;
          part[3 + c] = (double)r0 * (double)rf;
        }
      }
      slice_partial<6>(part, A.S, sl);
    }
  });
  double tot[6];
  if (grid_reduce_runs<6>(A.S, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    for (int c = 0; c < 3; ++c) {
      if (!((upd >> c) & 1)) continue;
      m->updates[c] += 1;
      const double prev2 = m->rnorm2[c];  // true residual at the previous update
      m->rnorm2[c] = tot[c];
      const double rho_new = tot[3 + c];
      if (isnan(tot[c]) || isnan(rho_new)) {
        m->status[c] = KS_BREAKDOWN;
        m->active &= ~(1 << c);
      } else if (tot[c] <= m->tol2[c]) {
        m->status[c] = KS_CONVERGED;
        m->active &= ~(1 << c);
      } else if (m->iters[c] >= m->maxit) {
        m->status[c] = KS_MAXIT;
        m->active &= ~(1 << c);
      } else {
        if ((rst >> c) & 1) {
          m->r0norm2[c] = rho_new;
          m->beta[c] = 0.0;
        } else {
          m->beta[c] = (rho_new / m->rho[c]) * (m->alpha[c] / m->omega[c]);
          // the true residual is more than 10x (in norm) the FP32 recurrence's (its Krylov space
          // has drifted), or it grew since the previous update (erratic convergence): the next
          // iteration restarts the space from the replaced residual
          if (tot[c] > kMixedDrift2 * m->rin2[c] || tot[c] > prev2) m->restart_next |= 1 << c;
        }
        m->rho[c] = rho_new;
        m->rin2[c] = tot[c];
        m->rmax2[c] = tot[c];
      }
    }
    m->upd = 0;
    m->restart = 0;
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
  }
}

__global__ void k_mp_check(const MixedState *__restrict__ m, DevStatus *st) {
  if (st->halt) return;
  int code = 0, it = 0;
  for (int c = 0; c < 3; ++c) {
    it = max(it, m->iters[c]);
    if (m->status[c] == KS_MAXIT && code == 0) code = 1;
    if (m->status[c] == KS_BREAKDOWN && code == 0) code = 2;
  }
  st->iters[0] += (unsigned long long)it;
  if (code) {
    st->code = code;
    st->halt = 1;
  }
}

// ------------------------------------------------------------------------------------------
// Mixed-precision momentum CG (the CFSA_KRYLOV_CG momentum method with a mixed precision): one
// batched Jacobi CG sequence in FP32 with FP64 reliable updates, the scheme of the BiCGSTAB above
// applied to CG (residual replacement with group-wise solution updates, van der Vorst & Ye 2000).
//   FP64: b, x (solution), r64 (true residual); FP32: r, p, q, dx; FP32 copy A32 of A
//   every iteration (FP64 dot products and scalars):
//     q = A32 p; alpha = rho / (p.q); dx += alpha p; r -= alpha q; z = D^-1 r; rho' = r.z
//   reliable update of component c when its iterated residual has dropped below delta times the
//   largest one since its last update, meets the tolerance or hits the cap:
//     x += dx; dx = 0; r64 = b - A x (FP64 operator); r = (float) r64; rho' = r.z
//   then p = z + (rho'/rho) p: the search direction carries on across updates. Convergence is
//   decided on the FP64 true residual with the FP64 solve's criterion. An update that finds the
//   true residual more than 10x the iterated one, or larger than at the previous update, restarts
//   the direction (p = z).

// Init (after k_momentum_rhs wrote b and x = 0): r = (float) b, p = z = D^-1 r, dx = 0; the FP64
// ||b|| in the convergence norm and rho = r.z.
__global__ void k_mpc_init(MixedArgs A, double tol, int maxit, double delta) {
  if (A.st->halt) return;
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int bk = blockIdx.x; bk < nblk; bk += gridDim.x, ++slot) {
    const int i = bk * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const double w = A.cw ? A.cw[i] : 1.0;
      const float dinv = A.invA32[i];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t o = c * n + i;
        const double bi = A.b[o];
        const float ri = (float)bi;
        const float zi = dinv * ri;
        A.r[o] = ri;
        A.p[o] = zi;
        A.dx[o] = 0.f;
        part[c] = (bi * bi) * w;
        part[3 + c] = (double)ri * (double)zi;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    m->active = 0;
    m->upd = 0;
    m->restart = 0;
    m->restart_next = 0;
    m->force = 0;
    m->maxit = maxit;
    m->delta2 = delta * delta;
    for (int c = 0; c < 3; ++c) {
      m->bnorm2[c] = tot[c];
      m->rnorm2[c] = tot[c];
      m->rin2[c] = tot[c];
      m->rmax2[c] = tot[c];
      m->tol2[c] = tol * tol * tot[c];
      m->rho[c] = tot[3 + c];
      m->alpha[c] = 0.0;
      m->beta[c] = 0.0;
      m->iters[c] = 0;
      m->updates[c] = 0;
      m->restarts[c] = 0;
      if (isnan(tot[c]) || isnan(tot[3 + c])) {
        m->status[c] = KS_BREAKDOWN;
      } else if (tot[c] == 0.0 || tot[c] <= m->tol2[c]) {
        m->status[c] = KS_CONVERGED;
      } else {
        m->status[c] = KS_RUNNING;
        m->active |= 1 << c;
      }
    }
  }
}

// C1: q = A32 p (into v), alpha = rho / (p . q)
__global__ void __launch_bounds__(kRunThreads, 1) k_mpc_q(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<3>(act, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[3] = {0.0, 0.0, 0.0};
      if (i >= 0) {
        float acc[3];
        sell_spmv_row_f32x3<8, MASK>(A.S, A.At32, A.p, n, r, acc);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!((MASK >> c) & 1)) continue;
          A.v[c * n + i] = acc[c];
          part[c] = (double)A.p[c * n + i] * (double)acc[c];
        }
      }
      slice_partial<3>(part, A.S, sl);
    }
  });
  double tot[3];
  if (grid_reduce_runs<3>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      if (isnan(tot[c]) || tot[c] == 0.0) {
        A.ms->status[c] = KS_BREAKDOWN;
        A.ms->active &= ~(1 << c);
      } else {
        A.ms->alpha[c] = A.ms->rho[c] / tot[c];
      }
    }
  }
}

// C2: dx += alpha p, r -= alpha q, z = D^-1 r; the iterated residual (convergence norm) and r.z;
// which components take a reliable update at the end of this iteration (IF node); next beta for
// the others.
__global__ void k_mpc_xr(MixedArgs A) {
  const int act = A.ms->active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[0] += 1;
  if (!act) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) {
      if (A.use_if) cudaGraphSetConditional(A.cond_upd, 0);
      cudaGraphSetConditional(A.cond, 0);
    }
    return;
  }
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  float alpha_c[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) alpha_c[c] = (float)A.ms->alpha[c];
  int slot = 0;
  for (int bk = blockIdx.x; bk < nblk; bk += gridDim.x, ++slot) {
    const int i = bk * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const float dinv = A.invA32[i];
      const double w = A.cw32 ? (double)A.cw32[i] : 1.0;
      float pv[3], qv[3], rv[3], dxv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        const int64_t o = c * n + i;
        pv[c] = A.p[o], qv[c] = A.v[o], rv[c] = A.r[o], dxv[c] = A.dx[o];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        const int64_t o = c * n + i;
        A.dx[o] = dxv[c] + alpha_c[c] * pv[c];
        const float ri = rv[c] - alpha_c[c] * qv[c];
        A.r[o] = ri;
        const float zi = dinv * ri;
        part[c] = ((double)ri * (double)ri) * w;
        part[3 + c] = (double)ri * (double)zi;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    int upd = 0;
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      m->iters[c] += 1;
      m->rin2[c] = tot[c];
      if (isnan(tot[c]) || isnan(tot[3 + c])) {
        m->status[c] = KS_BREAKDOWN;
        m->active &= ~(1 << c);
        continue;
      }
      if (tot[c] <= m->tol2[c] || m->iters[c] >= m->maxit || tot[c] < m->delta2 * m->rmax2[c]) {
        upd |= 1 << c;  // the update replaces rho and beta from the true residual
      } else {
        m->beta[c] = tot[3 + c] / m->rho[c];
        m->rho[c] = tot[3 + c];
        m->rmax2[c] = fmax(m->rmax2[c], tot[c]);
      }
    }
    m->upd = upd;
    if (A.use_cond) {
      if (A.use_if) cudaGraphSetConditional(A.cond_upd, upd ? 1u : 0u);
      cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
    }
  }
}

// Reliable update, part 1: x += dx (FP64) and dx = 0 for the updated components.
__global__ void k_mpc_xupdate(MixedArgs A) {
  const int upd = A.ms->upd;
  if (!upd) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((upd >> c) & 1)) continue;
    const int64_t o = c * n + i;
    A.x[o] = A.x[o] + (double)A.dx[o];
    A.dx[o] = 0.f;
  }
}

// Reliable update, part 2: r64 = b - A x (FP64 operator, rows in SELL order), r = (float) r64;
// convergence on the true residual; rho = r.z and the next beta from the replaced residual (0 when
// the direction restarts).
__global__ void __launch_bounds__(kRunThreads, 1) k_mpc_residual(MixedArgs A) {
  const int upd = A.ms->upd;
  if (!upd) return;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[2] += 1;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  __shared__ int s_next;
  const int sl0 = run_first_slice(&s_next, A.S.rfirst[blockIdx.x]);
  with_mask<3>(upd, [&](auto mk) {
    constexpr int MASK = decltype(mk)::value;
    for (int sl = sl0; sl < s1; sl = run_next_slice(&s_next)) {
      const int r = sl * kSellC + (threadIdx.x & 31);
      const int i = A.S.perm[r];
      double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (i >= 0) {
        double acc[3];
        sell_spmv_row<3, kU64, MASK>(A.S, A.At64, A.x, n, r, acc);
        const double w = A.cw ? A.cw[i] : 1.0;
        const float dinv = A.invA32[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (!((MASK >> c) & 1)) continue;
          const int64_t o = c * n + i;
          const double ri = A.b[o] - acc[c];
          A.r64[o] = ri;
          const float rf = (float)ri;
          A.r[o] = rf;
          part[c] = (ri * ri) * w;
          part[3 + c] = (double)rf * (double)(dinv * rf);
        }
      }
      slice_partial<6>(part, A.S, sl);
    }
  });
  double tot[6];
  if (grid_reduce_runs<6>(A.S, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    for (int c = 0; c < 3; ++c) {
      if (!((upd >> c) & 1)) continue;
      m->updates[c] += 1;
      const double prev2 = m->rnorm2[c];  // true residual at the previous update
      m->rnorm2[c] = tot[c];
      const double rz = tot[3 + c];
      if (isnan(tot[c]) || isnan(rz)) {
        m->status[c] = KS_BREAKDOWN;
        m->active &= ~(1 << c);
      } else if (tot[c] <= m->tol2[c]) {
        m->status[c] = KS_CONVERGED;
        m->active &= ~(1 << c);
      } else if (m->iters[c] >= m->maxit) {
        m->status[c] = KS_MAXIT;
        m->active &= ~(1 << c);
      } else {
        // the FP32 recurrence drifted from the true residual, or convergence turned erratic:
        // restart the direction from the replaced residual
        const bool restart = tot[c] > kMixedDrift2 * m->rin2[c] || tot[c] > prev2;
        m->beta[c] = restart ? 0.0 : rz / m->rho[c];
        if (restart) m->restarts[c] += 1;
        m->rho[c] = rz;
        m->rin2[c] = tot[c];
        m->rmax2[c] = tot[c];
      }
    }
    m->upd = 0;
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
  }
}

// C3: p = z + beta p with z = D^-1 r (after the update, which may have replaced r and beta)
__global__ void k_mpc_p(MixedArgs A) {
  const int act = A.ms->active;
  if (!act) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  const float dinv = A.invA32[i];
  float beta[3], rv[3], pv[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    beta[c] = (float)A.ms->beta[c];
    if ((act >> c) & 1) rv[c] = A.r[c * n + i], pv[c] = A.p[c * n + i];
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
    if ((act >> c) & 1) A.p[c * n + i] = dinv * rv[c] + beta[c] * pv[c];
}

// ------------------------------------------------------------------------------------------
// Mixed-precision pressure solve: FP64 defect correction around the two-level CG with float
// storage (k_cg2l_resident<float>: operator values, inverse diagonal and Krylov vectors in float,
// arithmetic and reductions in FP64).
//   x = 0, r = b                                  (FP64, from k_pressure_rhs)
//   while ||r|| > tol ||b|| (the FP64 solve's criterion, on the FP64 true residual):
//     solve Lbc d = r in float to tol_in relative  (k_cg2l_resident<float>, one cooperative launch)
//     x += d;  r = b - Lbc x                       (FP64)
// The operator is L2-resident at the benchmark sizes and the solve is bound by the latency of its
// grid barriers, so float storage shortens the body of an iteration (half the bytes gathered per
// entry) but not its barrier; the sweeps add one FP64 product each.
struct PMixState {
  double bnorm2, tol2, rnorm2;  // outer criterion on the FP64 true residual
  int sweeps, status, active;
  int iters;       // inner iterations over all sweeps
  int bar_failed;  // an inner solve gave up at a grid barrier
  int max_sweeps;
  double tol_in;
};

struct PMixArgs {
  SellView S;
  const double *Ls, *invL;  // FP64 penalised operator (SELL) and its inverse diagonal
  const float *invL32;
  const double *b;
  double *x, *r;            // FP64 solution and true residual (x = 0, r = b on entry)
  float *r32, *x32, *p32, *s32;  // inner right-hand side, solution, and the two zero-on-entry vectors
  int n, scaled, maxit;
  CgState *cs;     // the FP64 solve's state (criterion of b from k_pressure_rhs; totals at the end)
  CgState *cs_in;  // the inner float solve
  PMixState *pm;
  DevStatus *st;
  Reduce red;
  const int *bar_err;
  cudaGraphConditionalHandle cond;
  int use_cond;
};

__global__ void k_pmx_init(PMixArgs A, double tol_in, int max_sweeps) {
  PMixState *m = A.pm;
  const bool halted = A.st && A.st->halt;
  m->bnorm2 = A.cs->bnorm2;
  m->tol2 = A.cs->tol2;
  m->rnorm2 = A.cs->bnorm2;
  m->sweeps = 0;
  m->iters = 0;
  m->bar_failed = 0;
  m->status = A.cs->status;
  m->active = halted ? 0 : A.cs->active;
  m->max_sweeps = max_sweeps;
  m->tol_in = tol_in;
}

// Sweep start: inner right-hand side r32 = (float) r, x32 = p32 = s32 = 0, inner criterion.
__global__ void k_pmx_prep(PMixArgs A) {
  if (!A.pm->active) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      A.cs_in->active = 0;
      if (A.use_cond) cudaGraphSetConditional(A.cond, 0);
    }
    return;
  }
  __shared__ WarpSums<2> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int bk = blockIdx.x; bk < nblk; bk += gridDim.x, ++slot) {
    const int i = bk * kBlock + threadIdx.x;
    double part[2] = {0.0, 0.0};
    if (i < A.n) {
      const float rf = (float)A.r[i];
      A.r32[i] = rf;
      A.x32[i] = 0.f;
      A.p32[i] = 0.f;
      A.s32[i] = 0.f;
      const double rd = (double)rf;
      part[0] = rd * rd;
      part[1] = A.scaled ? rd * ((double)A.invL32[i] * rd) : rd * rd;
    }
    warp_partial<2>(part, S, slot);
  }
  double tot[2];
  if (grid_reduce_strided<2>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    CgState *c = A.cs_in;
    c->bb = tot[0];
    c->bnorm2 = tot[1];
    c->rnorm2 = tot[1];
    c->tol2 = A.pm->tol_in * A.pm->tol_in * tot[1];
    c->iters = 0;
    c->maxit = A.maxit;
    const bool run = tot[1] > 0.0 && !isnan(tot[1]);
    c->status = run ? KS_RUNNING : KS_BREAKDOWN;
    c->active = run ? 1 : 0;
  }
}

// x += d (FP64)
__global__ void k_pmx_xupdate(PMixArgs A) {
  if (!A.pm->active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < A.n) A.x[i] += (double)A.x32[i];
}

// r = b - Lbc x (FP64 true residual, rows in SELL order, one thread per row); outer criterion,
// sweep count and loop condition.
__global__ void k_pmx_residual(PMixArgs A) {
  if (!A.pm->active) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (r < A.S.nrows_pad) ? A.S.perm[r] : -1;
  double part[1] = {0.0};
  if (i >= 0) {
    const int base = A.S.sptr[r >> 5] + (r & 31), len = A.S.len[r];
    double acc = 0.0;
    for (int k = 0; k < len; ++k) {
      const int pos = base + k * kSellC;
      acc += A.Ls[pos] * A.x[A.S.col[pos]];
    }
    const double ri = A.b[i] - acc;
    A.r[i] = ri;
    part[0] = A.scaled ? ri * (A.invL[i] * ri) : ri * ri;
  }
  double tot[1];
  if (grid_reduce<1>(part, A.red, tot) && threadIdx.x == 0) {
    PMixState *m = A.pm;
    m->sweeps += 1;
    m->iters += A.cs_in->iters;
    m->rnorm2 = tot[0];
    if (A.bar_err && *A.bar_err) {
      m->bar_failed = 1;
      m->status = KS_BREAKDOWN;
      m->active = 0;
    } else if (isnan(tot[0])) {
      m->status = KS_BREAKDOWN;
      m->active = 0;
    } else if (tot[0] <= m->tol2) {
      m->status = KS_CONVERGED;
      m->active = 0;
    } else if (A.cs_in->status == KS_BREAKDOWN) {
      m->status = KS_BREAKDOWN;
      m->active = 0;
    } else if (m->sweeps >= m->max_sweeps) {
      m->status = KS_MAXIT;
      m->active = 0;
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
  }
}

// After the sweeps: totals into the FP64 solve's state (for the statistics) and, on failure, the
// step's status word (as k_check_cg does for the FP64 solve).
__global__ void k_pmx_check(PMixArgs A, DevStatus *st) {
  const PMixState *m = A.pm;
  if (st->halt) return;
  A.cs->iters = m->iters;
  A.cs->rnorm2 = m->rnorm2;
  A.cs->status = m->status;
  A.cs->active = 0;
  st->iters[1] += (unsigned long long)m->iters;
  int code = 0;
  if (m->status == KS_MAXIT) code = 1;
  if (m->status == KS_BREAKDOWN) code = 2;
  if (m->bar_failed) code = 4;
  if (code) {
    st->code = code;
    st->halt = 1;
  }
}

__global__ void k_to_f32(int64_t n, const double *__restrict__ src, float *__restrict__ dst) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) dst[k] = (float)src[k];
}

}  // namespace cfsa
