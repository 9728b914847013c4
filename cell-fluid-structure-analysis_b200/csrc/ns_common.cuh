// Device-side data structures and helpers shared by the Navier-Stokes kernels.
//
// Layouts in HBM (all device arrays are owned by the solver handle):
//   * tet data is structure-of-arrays so that per-tet kernels load with unit stride:
//     tet_node[l*nt + t] (l = 0..3 vertices, 4..9 P2 nodes nv+edge_id), vol[t],
//     grad[k*nt + t] (k = 3*a + c: component c of the gradient of vertex a);
//   * vector fields are component-major: u[c*N2 + i];
//   * every operator is held in CSR (ascending columns, the assembly format) and, for the
//     operators used inside Krylov loops, in SELL-32 (slices of 32 rows, entries of a slice
//     stored column-major, rows sorted by length inside windows of 256 rows). One thread owns
//     one row and sums its entries in ascending column order, which is the summation order of
//     the CSR (and of the reference's Eigen products), so SELL and CSR products agree bit for bit.
#pragma once

#include <cstdint>
#include <cuda/atomic>
#include <cuda_runtime.h>

namespace cfsa {

constexpr int kBlock = 256;
constexpr int kSellC = 32;
constexpr int kSellSigma = 256;
constexpr int kMaxRed = 8;  // values per block partial
constexpr double kMomentumPenalty = 1e10;  // NavierStokes.cpp:463
constexpr double kPoissonPenalty = 1e12;   // NavierStokes.cpp:611,619

enum : int { BC_WALL = 0, BC_INLET = 1, BC_OUTLET = 2, BC_INTERNAL = 3, BC_UNDEFINED = 4 };

// Krylov per-component status
enum : int { KS_RUNNING = 0, KS_CONVERGED = 1, KS_MAXIT = 2, KS_BREAKDOWN = 3 };

struct SellView {
  const int *sptr;  // [nslices+1] entry offset of each slice
  const int *col;   // [nentries]
  const int *len;   // [nrows_pad] row length
  const int *perm;  // [nrows_pad] original row, -1 for padding rows
  int nrows_pad;
  // Slice runs of the run-walking product kernels: CTA c owns slices [rfirst[c], rfirst[c+1]),
  // runs balanced by entries and split on 256-row block boundaries (multiples of 8 slices).
  const int *rfirst;  // [nruns+1]
  double *spart;      // [nslices * kMaxRed] warp sums of each slice (reduction scratch)
};

struct CsrView {
  const int *rp;
  const int *ci;
};

// Batched BiCGSTAB state (up to 3 right-hand sides sharing one matrix).
struct BicgState {
  double rho[3], alpha[3], omega[3], beta[3];
  double bnorm2[3], tol2[3], r0norm2[3], rnorm2[3];
  int iters[3], status[3];
  int active;   // bit c: component c still iterating
  int restart;  // bit c: component c restarts next iteration
  int maxit;
  int ncomp;
};

struct CgState {
  double absnew, alpha, beta, bnorm2, tol2, rnorm2;
  double bb;  // b.b of the solve's right-hand side (scale of the two-level CG's fixed-point sums)
  int iters, status, active, maxit;
};

struct DevStatus {
  int halt;        // nonzero: remaining work of this batch is skipped
  int code;        // first failure (CFSA_* code), 0 if none
  int steps_done;  // completed steps in this batch
  int nan;         // NaN flag of the current step
  unsigned long long body_runs[3];  // loop bodies executed: [0] momentum Krylov, [1] pressure,
                                    // [2] mixed-precision reliable updates
  unsigned long long iters[2];      // Krylov iterations completed: [0] momentum (max over rhs), [1] pressure
};

struct Reduce {
  double *partials;       // [gridDim.x * kMaxRed]
  unsigned int *counter;  // one ticket counter
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Second stage of the reduction tree, run by one block of 256 threads: the 256 accumulators
// (accumulator t sums block partials t, t+256, ... in order) are combined by warp butterflies and an
// in-order sum over the 8 warps; every thread gets the totals.
template <int NV>
__device__ __forceinline__ void combine_partials(const Reduce &red, unsigned int G, double (&out)[NV]) {
  __shared__ double sm[NV][kBlock / 32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int nwarps = kBlock / 32;
  // Thread t adds partials t, t+blockDim, ... in increasing order. Loads are issued in batches
  // before their additions so that the L2 latency is paid once per batch instead of once per
  // load; the order of the additions is unchanged. Few values: four blocks x all values per
  // batch; many values: one value at a time, eight blocks per batch (measured faster for 6).
  // The tree has kBlock accumulators whatever the block size: in a larger block the threads past
  // kBlock hold zeros and only take part in the barriers.
  double acc[NV];
#pragma unroll
  for (int j = 0; j < NV; ++j) acc[j] = 0.0;
  constexpr unsigned int T = kBlock;
  if (threadIdx.x >= T) {
  } else if (NV <= 3) {
    unsigned int b = threadIdx.x;
    for (; b + 3 * T < G; b += 4 * T) {
      double v[4][NV];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int j = 0; j < NV; ++j) v[q][j] = __ldcg(&red.partials[(size_t)(b + q * T) * kMaxRed + j]);
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int j = 0; j < NV; ++j) acc[j] += v[q][j];
    }
    for (; b < G; b += T)
#pragma unroll
      for (int j = 0; j < NV; ++j) acc[j] += __ldcg(&red.partials[(size_t)b * kMaxRed + j]);
  } else {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0.0;
      for (unsigned int b0 = threadIdx.x; b0 < G; b0 += 8 * T) {
        double x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const unsigned int b = b0 + q * T;
          x[q] = (b < G) ? __ldcg(&red.partials[(size_t)b * kMaxRed + j]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
          if (b0 + q * T < G) s += x[q];
      }
      acc[j] = s;
    }
  }
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double s = warp_sum(acc[j]);
    if (lane == 0 && warp < nwarps) sm[j][warp] = s;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double s = 0.0;
    for (int w = 0; w < nwarps; ++w) s += sm[j][w];
    out[j] = s;
  }
  __syncthreads();
}

// Deterministic grid reduction of NV doubles per thread. Every block writes its partial;
// the last block to arrive (ticket counter) sums the partials in block order and returns true
// with the totals in `out` (valid in all threads of that block). Other blocks return false.
template <int NV>
__device__ bool grid_reduce(double (&v)[NV], const Reduce &red, double (&out)[NV]) {
  __shared__ double sm[NV][kBlock / 32];
  __shared__ bool last;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    double w = warp_sum(v[j]);
    if (lane == 0) sm[j][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double s = 0.0;
      for (int w = 0; w < nwarps; ++w) s += sm[j][w];
      red.partials[(size_t)blockIdx.x * kMaxRed + j] = s;
    }
    // release: this block's partials are visible to the block that takes the last ticket
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ctr(*red.counter);
    const unsigned int ticket = ctr.fetch_add(1u, cuda::memory_order_acq_rel);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  combine_partials<NV>(red, gridDim.x, out);
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

// Grid-stride form of grid_reduce for kernels whose CTAs each visit up to kMaxStride blocks of
// 256 positions (blocks blockIdx.x, blockIdx.x + gridDim.x, ...). Each visited block leaves its 8
// warp sums in shared memory (no block-wide synchronisation per block); at the end the CTA forms
// the block partials (warp sums added in warp order, as grid_reduce does), writes them at their
// block index, and the last CTA to take a ticket combines all nblk partials in the same tree.
// Same tree, same bits as grid_reduce over one block per position block; fewer CTA-wide barriers
// and nblk / kMaxStride tickets instead of nblk.
constexpr int kMaxStride = 16;

template <int NV>
struct WarpSums {
  double v[kMaxStride][NV][kBlock / 32];
};

template <int NV>
__device__ __forceinline__ void warp_partial(const double (&v)[NV], WarpSums<NV> &S, int slot) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double w = warp_sum(v[j]);
    if (lane == 0) S.v[slot][j][warp] = w;
  }
}

template <int NV>
__device__ bool grid_reduce_strided(WarpSums<NV> &S, int nslots, unsigned int nblk, const Reduce &red,
                                    double (&out)[NV]) {
  __shared__ bool last;
  __syncthreads();
  if ((int)threadIdx.x < nslots * NV) {
    const int slot = threadIdx.x / NV, j = threadIdx.x % NV;
    double s = 0.0;
    for (int w = 0; w < kBlock / 32; ++w) s += S.v[slot][j][w];
    red.partials[(size_t)(blockIdx.x + slot * gridDim.x) * kMaxRed + j] = s;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ctr(*red.counter);
    const unsigned int ticket = ctr.fetch_add(1u, cuda::memory_order_acq_rel);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  combine_partials<NV>(red, nblk, out);
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

// Run-walking form for the SELL products of the Krylov loops: one CTA of kRunThreads per SM walks
// a contiguous run of slices (SellView::rfirst), warp w taking slices s0 + w, s0 + w + 32, ...
// Neighbouring rows gather from neighbouring parts of x, so the window of x that a CTA reads
// slides through the SM's L1 instead of being spread over the whole vector (one CTA per 256-row
// block puts blocks far apart in the row order on the same SM): 115 vs 137 us for the FP64
// 3-right-hand-side momentum product at 1M tets.
// Reduction: the warp that computes slice sl leaves its warp sums at spart[sl]; at the end each CTA
// forms the partials of the 256-row blocks of its run (the 8 slice sums in slice order, which is
// the warp order of grid_reduce) and the last CTA to take a ticket combines all block partials with
// the tree of grid_reduce. Same tree, same bits as grid_reduce over one block per 256 rows.
constexpr int kRunThreads = 1024;
constexpr int kRunWarps = kRunThreads / 32;
constexpr int kSlicesPerBlock = kBlock / kSellC;

// Slice scheduling inside a run: warp w starts with slice s0 + w and then takes the next slice
// nobody has claimed from a shared-memory counter. A static stride (w, w + 32, ...) gave a warp
// the same position in every 256-row window (rows are sorted by length inside a window, so warps
// 0, 8, 16, 24 always got the longest rows) and left the other warps waiting at the run's closing
// barrier (ncu, 415k tets: 7.8 barrier stalls per issued instruction). Which warp computes a slice
// does not matter for the results: each slice's sums go to its own slot of spart.
__device__ __forceinline__ int run_first_slice(int *next, int s0) {
  if (threadIdx.x == 0) *next = s0 + (int)(blockDim.x >> 5);
  __syncthreads();
  return s0 + (int)(threadIdx.x >> 5);
}
__device__ __forceinline__ int run_next_slice(int *next) {
  int v = 0;
  if ((threadIdx.x & 31) == 0) v = atomicAdd(next, 1);
  return __shfl_sync(0xffffffffu, v, 0);
}

template <int NV>
__device__ __forceinline__ void slice_partial(const double (&v)[NV], const SellView &S, int sl) {
#pragma unroll
  for (int j = 0; j < NV; ++j) {
    const double w = warp_sum(v[j]);
    if ((threadIdx.x & 31) == 0) __stcg(&S.spart[(size_t)sl * kMaxRed + j], w);
  }
}

template <int NV>
__device__ bool grid_reduce_runs(const SellView &S, const Reduce &red, double (&out)[NV]) {
  __shared__ bool last;
  __syncthreads();  // every slice sum of this run is written
  const int nsl = S.nrows_pad / kSellC;
  const int s0 = S.rfirst[blockIdx.x], s1 = S.rfirst[blockIdx.x + 1];
  const int b0 = s0 / kSlicesPerBlock, b1 = (s1 + kSlicesPerBlock - 1) / kSlicesPerBlock;
  for (int t = threadIdx.x; t < (b1 - b0) * NV; t += blockDim.x) {
    const int b = b0 + t / NV, j = t % NV;
    double s = 0.0;
    for (int w = 0; w < kSlicesPerBlock && kSlicesPerBlock * b + w < nsl; ++w)
      s += __ldcg(&S.spart[(size_t)(kSlicesPerBlock * b + w) * kMaxRed + j]);
    red.partials[(size_t)b * kMaxRed + j] = s;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    cuda::atomic_ref<unsigned int, cuda::thread_scope_device> ctr(*red.counter);
    const unsigned int ticket = ctr.fetch_add(1u, cuda::memory_order_acq_rel);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  combine_partials<NV>(red, (unsigned int)((nsl + kSlicesPerBlock - 1) / kSlicesPerBlock), out);
  if (threadIdx.x == 0) *red.counter = 0u;
  return true;
}

}  // namespace cfsa
