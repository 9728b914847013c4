// Mixed-precision momentum solve: FP32 batched BiCGSTAB inside FP64 defect correction.
//
//   x = 0, r = b                                       (FP64, from k_momentum_rhs)
//   repeat (outer sweep) while some component has ||r||^2 > tol^2 ||b||^2:
//     solve At d = r approximately in FP32            (inner: FP32 operator values and vectors,
//                                                      FP64 dot products and scalars, stop at
//                                                      ||r_in|| <= tol_in ||r||, a cap or near-breakdown)
//     x += D^-1 d                                     (FP64)
//     r = b - A x                                     (FP64 operator, true residual)
// At = A D^-1 is the right-Jacobi-scaled momentum operator (At32 is its FP32 copy); the penalty
// rows (diagonal 1e10) have unit diagonal in At, so FP32 holds them without overflow or loss.
// The convergence test is on the true FP64 residual, so the result meets the same tolerance as
// the FP64 solve. Components are independent (per-component scalars and masks).
#pragma once

#include "ns_kernels.cuh"

namespace cfsa {

struct MixedState {
  // outer (FP64)
  double bnorm2[3], tol2[3], rnorm2[3];
  int outer[3], status[3];
  int active;  // components still sweeping
  int max_outer;
  // inner (FP32 vectors, FP64 scalars)
  double rho[3], alpha[3], omega[3], beta[3], r0norm2[3], tol_in2[3], rin2[3];
  int iters[3], total_iters[3];
  int in_active;  // components iterating in the current sweep
  int in_maxit;
  double tol_in;
};

struct MixedArgs {
  SellView S;
  const float *At32;
  const double *At64, *diagA, *invA;
  const float *invA32;
  const double *b;
  double *x, *r64, *xs;  // FP64 solution, residual, scaled solution D x
  float *r, *r0, *p, *v, *s, *t, *dx;
  int n;
  MixedState *ms;
  DevStatus *st;
  Reduce red;
  cudaGraphConditionalHandle cond;
  int use_cond;
  const double *cw;   // convergence-norm weights (diag(A)^-1), nullptr: unscaled ||r||
  const float *cw32;  // the same for the inner solve
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
  for (; k < len; ++k) {
    const int pos = base + k * kSellC;
    const int j = __ldcs(S.col + pos);
    const float a = __ldcs(val + pos);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      if ((MASK >> c) & 1) acc[c] += a * __ldg(x + c * n + j);
  }
}

// sell_spmv_row_f32x3 for the components still active in `mask` (see sell_spmv_row_active).
__device__ __forceinline__ void sell_spmv_row_f32x3_active(const SellView &S, const float *__restrict__ val,
                                                           const float *__restrict__ x, int64_t n, int r,
                                                           float acc[3], int mask) {
  if (mask == 6)
    sell_spmv_row_f32x3<8, 6>(S, val, x, n, r, acc);
  else if (mask == 5)
    sell_spmv_row_f32x3<8, 5>(S, val, x, n, r, acc);
  else if (mask == 3)
    sell_spmv_row_f32x3<8, 3>(S, val, x, n, r, acc);
  else
    sell_spmv_row_f32x3(S, val, x, n, r, acc);
}

// Outer init (after k_momentum_rhs wrote b and x = 0): r64 = b, ||b||^2 per component.
__global__ void k_mp_outer_init(MixedArgs A, double tol, int max_outer, double tol_in, int in_maxit) {
  if (A.st->halt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t n = A.n;
  double part[3] = {0.0, 0.0, 0.0};
  if (i < A.n) {
    const double w = A.cw ? A.cw[i] : 1.0;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double bi = A.b[c * n + i];
      A.r64[c * n + i] = bi;
      part[c] = (bi * bi) * w;
    }
  }
  double tot[3];
  if (grid_reduce<3>(part, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    m->active = 0;
    m->max_outer = max_outer;
    m->tol_in = tol_in;
    m->in_maxit = in_maxit;
    for (int c = 0; c < 3; ++c) {
      m->bnorm2[c] = tot[c];
      m->rnorm2[c] = tot[c];
      m->tol2[c] = tol * tol * tot[c];
      m->outer[c] = 0;
      m->total_iters[c] = 0;
      m->iters[c] = 0;
      if (isnan(tot[c])) {
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

// Inner init: r = r0 = (float) r64, p = v = dx = 0; rho = ||r||^2. When captured it also sets
// the inner loop's condition (a nested loop is not re-armed by its handle's default value).
__global__ void k_mp_inner_init(MixedArgs A) {
  const int active = A.ms->active;
  if (!active) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      A.ms->in_active = 0;
      if (A.use_cond) cudaGraphSetConditional(A.cond, 0);
    }
    return;
  }
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++slot) {
    const int i = b * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const double w = A.cw32 ? (double)A.cw32[i] : 1.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t o = c * n + i;
        const float ri = (float)A.r64[o];
        A.r[o] = ri;
        A.r0[o] = ri;
        A.p[o] = 0.f;
        A.v[o] = 0.f;
        A.dx[o] = 0.f;
        if ((active >> c) & 1) {
          part[c] = (double)ri * (double)ri;
          part[3 + c] = ((double)ri * (double)ri) * w;
        }
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    m->in_active = 0;
    for (int c = 0; c < 3; ++c) {
      m->iters[c] = 0;
      if (!((active >> c) & 1)) continue;
      m->rho[c] = tot[c];
      m->r0norm2[c] = tot[c];
      m->rin2[c] = tot[3 + c];
      m->tol_in2[c] = m->tol_in * m->tol_in * tot[3 + c];
      m->alpha[c] = m->omega[c] = 1.0;
      m->beta[c] = 0.0;
      if (tot[c] > 0.0 && !isnan(tot[c])) m->in_active |= 1 << c;
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->in_active ? 1u : 0u);
  }
}

// K1: p = r + beta (p - omega v)
__global__ void k_mp_p(MixedArgs A) {
  const int act = A.ms->in_active;
  if (!act) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((act >> c) & 1)) continue;
    const int64_t o = c * n + i;
    const float beta = (float)A.ms->beta[c], omega = (float)A.ms->omega[c];
    A.p[o] = A.r[o] + beta * (A.p[o] - omega * A.v[o]);
  }
}

// K2: v = At32 p, alpha = rho / (r0 . v)
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_v(MixedArgs A) {
  const int act = A.ms->in_active;
  if (!act) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  for (int sl = A.S.rfirst[blockIdx.x] + (threadIdx.x >> 5); sl < s1; sl += kRunWarps) {
    const int r = sl * kSellC + (threadIdx.x & 31);
    const int i = A.S.perm[r];
    double part[3] = {0.0, 0.0, 0.0};
    if (i >= 0) {
      float acc[3];
      sell_spmv_row_f32x3_active(A.S, A.At32, A.p, n, r, acc, act);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        A.v[c * n + i] = acc[c];
        part[c] = (double)A.r0[c * n + i] * (double)acc[c];
      }
    }
    slice_partial<3>(part, A.S, sl);
  }
  double tot[3];
  if (grid_reduce_runs<3>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      if (tot[c] == 0.0 || isnan(tot[c]))
        A.ms->in_active &= ~(1 << c);  // sweep ends; the outer residual restarts it
      else
        A.ms->alpha[c] = A.ms->rho[c] / tot[c];
    }
  }
}

// K3: s = r - alpha v
__global__ void k_mp_s(MixedArgs A) {
  const int act = A.ms->in_active;
  if (!act) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (!((act >> c) & 1)) continue;
    const int64_t o = c * n + i;
    A.s[o] = A.r[o] - (float)A.ms->alpha[c] * A.v[o];
  }
}

// K4: t = At32 s, omega = (t . s) / (t . t)
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_t(MixedArgs A) {
  const int act = A.ms->in_active;
  if (!act) return;
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  for (int sl = A.S.rfirst[blockIdx.x] + (threadIdx.x >> 5); sl < s1; sl += kRunWarps) {
    const int r = sl * kSellC + (threadIdx.x & 31);
    const int i = A.S.perm[r];
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i >= 0) {
      float acc[3];
      sell_spmv_row_f32x3_active(A.S, A.At32, A.s, n, r, acc, act);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        A.t[c * n + i] = acc[c];
        part[c] = (double)acc[c] * (double)acc[c];
        part[3 + c] = (double)acc[c] * (double)A.s[c * n + i];
      }
    }
    slice_partial<6>(part, A.S, sl);
  }
  double tot[6];
  if (grid_reduce_runs<6>(A.S, A.red, tot) && threadIdx.x == 0) {
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      A.ms->omega[c] = (tot[c] > 0.0) ? tot[3 + c] / tot[c] : 0.0;
    }
  }
}

// K5: dx += alpha D^-1 p + omega D^-1 s, r = s - omega t; inner convergence, next beta.
__global__ void k_mp_xr(MixedArgs A) {
  const int act = A.ms->in_active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[0] += 1;
  if (!act) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  const int64_t n = A.n;
  __shared__ WarpSums<6> S;
  const int nblk = (A.n + kBlock - 1) / kBlock;
  int slot = 0;
  for (int b = blockIdx.x; b < nblk; b += gridDim.x, ++slot) {
    const int i = b * kBlock + threadIdx.x;
    double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < A.n) {
      const float dinv = A.invA32[i];
      const double w = A.cw32 ? (double)A.cw32[i] : 1.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((act >> c) & 1)) continue;
        const int64_t o = c * n + i;
        const float alpha = (float)A.ms->alpha[c], omega = (float)A.ms->omega[c];
        A.dx[o] += alpha * (dinv * A.p[o]) + omega * (dinv * A.s[o]);
        const float ri = A.s[o] - omega * A.t[o];
        A.r[o] = ri;
        part[c] = ((double)ri * (double)ri) * w;
        part[3 + c] = (double)A.r0[o] * (double)ri;
      }
    }
    warp_partial<6>(part, S, slot);
  }
  double tot[6];
  if (grid_reduce_strided<6>(S, slot, nblk, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    const double eps = 2.220446049250313e-16;
    for (int c = 0; c < 3; ++c) {
      if (!((act >> c) & 1)) continue;
      m->iters[c] += 1;
      m->total_iters[c] += 1;
      m->rin2[c] = tot[c];
      const double rho_new = tot[3 + c];
      if (isnan(tot[c]) || tot[c] <= m->tol_in2[c] || m->iters[c] >= m->in_maxit || m->omega[c] == 0.0 ||
          fabs(rho_new) < eps * eps * m->r0norm2[c]) {
        m->in_active &= ~(1 << c);
      } else {
        m->beta[c] = (rho_new / m->rho[c]) * (m->alpha[c] / m->omega[c]);
        m->rho[c] = rho_new;
      }
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->in_active ? 1u : 0u);
  }
}

// x += D^-1-scaled correction (FP64); xs = diag(A) x for the residual product.
__global__ void k_mp_xupdate(MixedArgs A) {
  const int active = A.ms->active;
  if (!active) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int64_t n = A.n;
  const double d = A.diagA[i];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t o = c * n + i;
    double xi = A.x[o];
    if ((active >> c) & 1) {
      xi += (double)A.dx[o];
      A.x[o] = xi;
    }
    A.xs[o] = d * xi;
  }
}

// r64 = b - At64 (D x) (FP64 true residual); outer convergence and loop condition.
__global__ void __launch_bounds__(kRunThreads, 1) k_mp_residual(MixedArgs A) {
  const int active = A.ms->active;
  if (blockIdx.x == 0 && threadIdx.x == 0 && A.st) A.st->body_runs[2] += 1;
  if (!active) {
    if (A.use_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(A.cond, 0);
    return;
  }
  const int64_t n = A.n;
  const int s1 = A.S.rfirst[blockIdx.x + 1];
  for (int sl = A.S.rfirst[blockIdx.x] + (threadIdx.x >> 5); sl < s1; sl += kRunWarps) {
    const int r = sl * kSellC + (threadIdx.x & 31);
    const int i = A.S.perm[r];
    double part[3] = {0.0, 0.0, 0.0};
    if (i >= 0) {
      double acc[3];
      sell_spmv_row_active<3>(A.S, A.At64, A.xs, n, r, acc, active);
      const double w = A.cw ? A.cw[i] : 1.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (!((active >> c) & 1)) continue;
        const double ri = A.b[c * n + i] - acc[c];
        A.r64[c * n + i] = ri;
        part[c] = (ri * ri) * w;
      }
    }
    slice_partial<3>(part, A.S, sl);
  }
  double tot[3];
  if (grid_reduce_runs<3>(A.S, A.red, tot) && threadIdx.x == 0) {
    MixedState *m = A.ms;
    for (int c = 0; c < 3; ++c) {
      if (!((active >> c) & 1)) continue;
      m->outer[c] += 1;
      m->rnorm2[c] = tot[c];
      if (isnan(tot[c])) {
        m->status[c] = KS_BREAKDOWN;
        m->active &= ~(1 << c);
      } else if (tot[c] <= m->tol2[c]) {
        m->status[c] = KS_CONVERGED;
        m->active &= ~(1 << c);
      } else if (m->outer[c] >= m->max_outer) {
        m->status[c] = KS_MAXIT;
        m->active &= ~(1 << c);
      }
    }
    if (A.use_cond) cudaGraphSetConditional(A.cond, m->active ? 1u : 0u);
  }
}

__global__ void k_mp_check(const MixedState *__restrict__ m, DevStatus *st) {
  if (st->halt) return;
  int code = 0, it = 0;
  for (int c = 0; c < 3; ++c) {
    it = max(it, m->total_iters[c]);
    if (m->status[c] == KS_MAXIT && code == 0) code = 1;
    if (m->status[c] == KS_BREAKDOWN && code == 0) code = 2;
  }
  st->iters[0] += (unsigned long long)it;
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
