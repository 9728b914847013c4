// Host side of the C ABI declared in include/cfsa_ns.h: device memory, set-up (adjacency,
// patterns, SELL layout, assembly), the step sequence and its CUDA-graph capture.
//
// One PISO step is captured once into a CUDA graph whose two Krylov loops are conditional
// WHILE nodes: the last reduction kernel of each iteration decides on the device whether the
// loop continues, so a step (or a batch of steps) runs with no host round trip.
#include "cfsa_ns.h"
#include "ns_adjoint.cuh"
#include "ns_kernels.cuh"
#include "ns_mixed.cuh"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <exception>
#include <fstream>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <vector>

using namespace cfsa;

namespace {

// NVTX range over a host-side phase (set-up, a batch of steps, an adjoint pass); free unless a
// profiler is attached.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

struct Sell {
  int *sptr = nullptr, *col = nullptr, *len = nullptr, *perm = nullptr, *posmap = nullptr;
  int nrows = 0, nrows_pad = 0, nslices = 0;
  int64_t nentries = 0;
  std::vector<int> h_sptr;  // host copy of sptr
  int *rfirst = nullptr;    // slice runs of the run-walking kernels (one per SM)
  double *spart = nullptr;  // their per-slice warp sums
  int nruns = 0;
  SellView view() const { return SellView{sptr, col, len, perm, nrows_pad, rfirst, spart}; }
};

// Entry-balanced runs of slices, one per CTA of a run-walking kernel, split on 256-row block
// boundaries: run c starts at the first block boundary at or after c/nruns of the entries.
std::vector<int> slice_runs(const std::vector<int> &sptr, int nslices, int nruns) {
  std::vector<int> f(nruns + 1, 0);
  const int64_t ne = sptr[nslices];
  for (int c = 1; c < nruns; ++c) {
    const int64_t target = ne * c / nruns;
    int sl = (int)(std::lower_bound(sptr.begin(), sptr.begin() + nslices + 1, target,
                                    [](int a, int64_t t) { return (int64_t)a < t; }) -
                   sptr.begin());
    sl = (sl + kSlicesPerBlock - 1) / kSlicesPerBlock * kSlicesPerBlock;
    f[c] = std::max(f[c - 1], std::min(sl, nslices));
  }
  f[nruns] = nslices;
  return f;
}

struct CudaError {
  std::string msg;
};

#define CK(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      throw CudaError{std::string(#call) + ": " + cudaGetErrorString(e_)};                     \
  } while (0)

inline unsigned int blocks_for(int64_t n) { return (unsigned int)((n + kBlock - 1) / kBlock); }

// Pinned host buffers released together (staging of one export call).
struct PinnedSet {
  std::vector<void *> p;
  ~PinnedSet() {
    for (void *q : p) cudaFreeHost(q);
  }
  template <class T>
  T *get(size_t count) {
    void *q = nullptr;
    CK(cudaMallocHost(&q, std::max<size_t>(count, 1) * sizeof(T)));
    p.push_back(q);
    return static_cast<T *>(q);
  }
};

}  // namespace

struct cfsa_ns {
  int device = 0;
  cudaStream_t stream = nullptr, body_stream = nullptr, body_stream2 = nullptr;
  // stream-ordered field read-back (cfsa_ns_get_*_async): device staging copies of u (node-major)
  // and p taken on `stream`, copied to the caller's host arrays on copy_stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_u_ready = nullptr, ev_u_done = nullptr, ev_p_ready = nullptr, ev_p_done = nullptr;
  double *out_u = nullptr, *out_p = nullptr;
  std::string err;
  std::vector<void *> allocs;

  int64_t nv = 0, ne = 0, N2 = 0, nt = 0, nbf = 0;
  double density = 1000, viscosity = 0.001;
  double dt = 1e-4, tol_mom = 1e-6, tol_p = 1e-8;
  int maxit_mom = 1000, maxit_p = 1000, ncorr = 1;
  double relax_u = 1.0, relax_p = 1.0;
  int outlet_type = CFSA_OUTLET_DIRICHLET;
  double outlet_pressure = 0.0;
  int ref_node = -1;
  int krylov = CFSA_KRYLOV_BICGSTAB;  // the reference's pressure method (NavierStokes.cpp:633)
  int mom_krylov = CFSA_KRYLOV_BICGSTAB;  // the reference's momentum method (NavierStokes.cpp:498)
  int precision = CFSA_PRECISION_FP64;
  int conv_norm = CFSA_NORM_REFERENCE;
  double time = 0.0;
  int64_t steps = 0;
  float last_ms = 0.f;

  std::vector<signed char> h_bc;  // [N2]
  std::vector<double> h_inlet;    // [3][N2]
  std::vector<int> h_rp2, h_rp1;

  // mesh
  double *xyz = nullptr, *vol = nullptr, *grad = nullptr;
  int *tnode = nullptr;
  signed char *bc = nullptr;
  int *adj_ptr = nullptr, *adj = nullptr;
  // P2 operators
  int *rp2 = nullptr, *ci2 = nullptr, *rows2 = nullptr, *dpos2 = nullptr;
  int64_t nnz2 = 0;
  double *Mv = nullptr, *Kv = nullptr, *Ms = nullptr, *At = nullptr, *diagA = nullptr, *invA = nullptr;
  Sell s2;
  // P1 operators
  int *rp1 = nullptr, *ci1 = nullptr, *rows1 = nullptr, *dpos1 = nullptr;
  int64_t nnz1 = 0;
  double *Gv = nullptr, *Lv = nullptr, *Ls = nullptr, *Lt = nullptr, *diagL = nullptr, *invL = nullptr;
  Sell s1;
  double *invm = nullptr;
  // fields
  double *u = nullptr, *ustar = nullptr, *p = nullptr, *pc = nullptr, *inlet = nullptr;
  // work
  double *ct = nullptr, *divt = nullptr;
  double *wb = nullptr, *wr = nullptr, *wr0 = nullptr, *wp = nullptr, *wv = nullptr, *ws = nullptr,
         *wt = nullptr;  // [3][N2]
  double *pb = nullptr, *pr = nullptr, *pz = nullptr, *pp = nullptr, *pq = nullptr, *ps = nullptr,
         *pt = nullptr, *pv = nullptr, *pu = nullptr;  // [nv]
  double *stash = nullptr;
  // boundary faces
  int *fverts = nullptr, *ftet = nullptr, *vf_ptr = nullptr, *vf = nullptr;
  double *fnormal = nullptr, *farea = nullptr, *fshear = nullptr, *fpress = nullptr, *fout = nullptr;
  // solver states
  BicgState *bs_mom = nullptr, *bs_p = nullptr;
  CgState *cs = nullptr;
  DevStatus *st = nullptr, *st_free = nullptr;
  Reduce red{};
  DevStatus *h_st = nullptr;
  BicgState *h_bs = nullptr;
  CgState *h_cs = nullptr;
  double *h_stage = nullptr;  // pinned [3][N2] staging for host transfers
  double *d_vec3 = nullptr;   // device [N2][3] staging of vector-field transfers
  bool h_inlet_stale = false;  // h_inlet behind the device inlet (set from a device-side split)
  BicgState *bs_prof = nullptr;
  CgState *cs_prof = nullptr;
  MixedState *ms_prof = nullptr;
  // persistent CG
  bool cg_persistent = true;
  int cg_grid = 0;
  std::map<const void *, int> stride_ctas_of;  // one resident wave of each grid-stride kernel
  // SMEM-resident variant of the persistent CG (k_cg_resident): one 1024-thread CTA per SM
  bool cg_resident = false;
  double *cg1_vec[3] = {nullptr, nullptr, nullptr};  // second r, w, s buffers of k_cg1_resident
  int cg_res_grid = 0, cg_res_bpc_sell = 0, cg_res_bpc_nat = 0, cg_res_col_cap = 0;
  size_t cg_res_smem = 0;
  unsigned int *bar_count = nullptr, *bar_gen = nullptr;
  int *bar_err = nullptr;
  long long bar_spin_limit = kBarrierSpinLimit;
  // raw Poisson operator of solvePressureBiCGSTAB (no penalty rows), column-scaled by its inverse
  // diagonal like Lt; built on first use and again after the geometry changed
  double *Lraw_t = nullptr, *diag_raw = nullptr, *inv_raw = nullptr;
  int64_t raw_gen = -1;
  // two-level pressure preconditioner of k_cg2l_resident (rebuilt with the Poisson operator)
  int coarse_target = 256;
  bool coarse_dirty = true;
  int coarse_nc = 0;
  std::vector<void *> coarse_allocs;
  CoarseView coarse_view{};
  int cg2l_col_cap = 0;
  size_t cg2l_smem = 0;
  double *cg_part_a = nullptr, *cg_part_b = nullptr;
  // mixed precision (FP32 BiCGSTAB with FP64 reliable updates)
  float *At32 = nullptr, *invA32 = nullptr;
  float *fr = nullptr, *fr0 = nullptr, *fp = nullptr, *fv = nullptr, *fs = nullptr, *ft = nullptr,
        *fdx = nullptr;  // [3][N2]
  MixedState *ms = nullptr;
  MixedState *h_ms = nullptr;
  // mixed-precision pressure (two-level CG in float storage inside FP64 defect correction)
  float *Ls32 = nullptr, *invL32 = nullptr, *px32 = nullptr, *pp32 = nullptr, *pu32 = nullptr;
  float *pr32[2] = {nullptr, nullptr}, *pw32[2] = {nullptr, nullptr}, *ps32[2] = {nullptr, nullptr};
  CgState *cs_in = nullptr;
  PMixState *pmx = nullptr;
  PMixState *h_pmx = nullptr;
  double mixed_p_tol_in = 1e-5;  // inner reduction per sweep
  int mixed_p_max_sweeps = 30;
  // reliable-update threshold of the mixed-precision momentum solve: the FP64 residual replaces the
  // FP32 one when the latter has dropped by this factor since the previous update (0: the method's
  // default). BiCGSTAB 1e-2: a larger drop between updates costs it extra iterations. CG 1e-4: its FP32
  // iterations follow the FP64 ones whatever the threshold (1.4% faster than 1e-2 at 1M tets,
  // mixed vs FP64 3.5e-8 after 85 steps), so fewer FP64 residual products are pure savings.
  double mixed_delta = 0.0;
  double mixed_delta_of_method() const {
    if (mixed_delta > 0.0) return mixed_delta;
    return mom_krylov == CFSA_KRYLOV_CG ? 1e-4 : 1e-2;
  }
  bool cg2l_split = false;  // two-level CG iteration in two passes (u stored, one gather per entry)

  // discrete adjoint (ns_adjoint.cuh): transposed P1 slots, vertex -> (boundary face, local
  // index in the face's tet) incidence, host vertex coordinates for objective patches
  int *tpos1 = nullptr, *vbf_ptr = nullptr, *vbf = nullptr;
  std::vector<double> h_xyz;
  int64_t geom_gen = 0;
  bool adj_work = false;
  double *a_lu = nullptr, *a_lp = nullptr, *a_x = nullptr, *a_px = nullptr, *a_q = nullptr,
         *a_lpp = nullptr, *a_tsc = nullptr, *a_gin = nullptr, *a_scal = nullptr, *a_un = nullptr,
         *a_us = nullptr, *a_w = nullptr, *a_W = nullptr;  // a_scal: dJ/dnu, J, chain sum
  signed char *a_mask = nullptr;
  DevStatus *st_adj = nullptr;
  std::vector<void *> rec_allocs;  // checkpoints and step records (re-planned per forward pass)
  double *a_rec = nullptr, *a_ck = nullptr, *a_fin = nullptr;
  int64_t a_rec_slots = 0, a_ck_slots = 0;
  int adj_steps = 0, adj_C = 0, adj_nseg = 0;
  bool adj_valid = false, adj_last_valid = false;
  double adj_time_end = 0.0;
  int64_t adj_steps_end = 0;
  uint64_t adj_fp = 0;
  cfsa_adjoint_stats adj_stats{};
  cudaGraphExec_t adj_exec = nullptr;
  int64_t adj_launches_fixed = 0;
  int64_t batch_launches = 0;
  int64_t batch_iters[2] = {0, 0};
  int launches_per_step = 0;  // kernels of one step outside the Krylov loop bodies

  bool mom_dirty = true, poisson_dirty = true, graph_dirty = true;
  bool use_graph = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ph[4] = {nullptr, nullptr, nullptr, nullptr};  // step phase boundaries

  template <class T>
  T *dalloc(size_t count) {
    void *ptr = nullptr;
    if (count == 0) count = 1;
    CK(cudaMalloc(&ptr, count * sizeof(T)));
    allocs.push_back(ptr);
    return static_cast<T *>(ptr);
  }
  template <class T>
  T *dupload(const std::vector<T> &h) {
    T *d = dalloc<T>(h.size());
    if (!h.empty()) CK(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return d;
  }

  ~cfsa_ns() {
    if (copy_stream) {
      cudaStreamSynchronize(copy_stream);  // async read-backs still in flight
      cudaStreamDestroy(copy_stream);
    }
    for (cudaEvent_t e : {ev_u_ready, ev_u_done, ev_p_ready, ev_p_done})
      if (e) cudaEventDestroy(e);
    if (adj_exec) cudaGraphExecDestroy(adj_exec);
    for (void *ptr : rec_allocs) cudaFree(ptr);
    for (void *ptr : coarse_allocs) cudaFree(ptr);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    for (void *ptr : allocs) cudaFree(ptr);
    if (h_st) cudaFreeHost(h_st);
    if (h_bs) cudaFreeHost(h_bs);
    if (h_cs) cudaFreeHost(h_cs);
    if (h_stage) cudaFreeHost(h_stage);
    if (h_ms) cudaFreeHost(h_ms);
    if (h_pmx) cudaFreeHost(h_pmx);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    for (cudaEvent_t e : ph)
      if (e) cudaEventDestroy(e);
    if (body_stream) cudaStreamDestroy(body_stream);
    if (body_stream2) cudaStreamDestroy(body_stream2);
    if (stream) cudaStreamDestroy(stream);
  }

  // ------------------------------------------------------------------ set-up
  void build_sell(int n, const std::vector<int> &rp, Sell &S, const int *d_rp, const int *d_ci) {
    S.nrows = n;
    S.nrows_pad = (n + kSellC - 1) / kSellC * kSellC;
    S.nslices = S.nrows_pad / kSellC;
    std::vector<int> perm(S.nrows_pad, -1), len(S.nrows_pad, 0);
    std::vector<int> idx;
    for (int w0 = 0; w0 < n; w0 += kSellSigma) {
      const int w1 = std::min(n, w0 + kSellSigma);
      idx.resize(w1 - w0);
      std::iota(idx.begin(), idx.end(), w0);
      std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
        return (rp[a + 1] - rp[a]) > (rp[b + 1] - rp[b]);
      });
      for (int k = 0; k < w1 - w0; ++k) {
        perm[w0 + k] = idx[k];
        len[w0 + k] = rp[idx[k] + 1] - rp[idx[k]];
      }
    }
    std::vector<int> sptr(S.nslices + 1, 0);
    for (int s = 0; s < S.nslices; ++s) {
      int w = 0;
      for (int k = 0; k < kSellC; ++k) w = std::max(w, len[s * kSellC + k]);
      sptr[s + 1] = sptr[s] + w * kSellC;
    }
    S.nentries = sptr[S.nslices];
    S.h_sptr = sptr;
    {
      int nsm = 0;
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
      S.nruns = std::max(1, nsm);
      S.rfirst = dupload(slice_runs(sptr, S.nslices, S.nruns));
      S.spart = dalloc<double>((size_t)S.nslices * kMaxRed);
    }
    S.perm = dupload(perm);
    S.len = dupload(len);
    S.sptr = dupload(sptr);
    S.col = dalloc<int>((size_t)S.nentries);
    CK(cudaMemsetAsync(S.col, 0, (size_t)S.nentries * sizeof(int), stream));
    S.posmap = dalloc<int>((size_t)rp[n]);
    k_sell_fill<<<blocks_for(S.nrows_pad), kBlock, 0, stream>>>(S.nrows_pad, S.sptr, S.perm, S.len,
                                                                d_rp, d_ci, S.col, S.posmap);
    CK(cudaGetLastError());
  }

  void build_pattern(bool p2, int nrows, std::vector<int> &h_rp, int *&d_rp, int *&d_ci,
                     int64_t &nnz, int *d_err) {
    int *counts = dalloc<int>(nrows);
    const unsigned int g = (unsigned int)((nrows + 7) / 8);
    if (p2)
      k_pattern<true><<<g, kBlock, 0, stream>>>(nrows, (int)nt, adj_ptr, adj, tnode, counts, nullptr,
                                                nullptr, d_err);
    else
      k_pattern<false><<<g, kBlock, 0, stream>>>(nrows, (int)nt, adj_ptr, adj, tnode, counts,
                                                 nullptr, nullptr, d_err);
    CK(cudaGetLastError());
    std::vector<int> hc(nrows);
    CK(cudaMemcpyAsync(hc.data(), counts, nrows * sizeof(int), cudaMemcpyDeviceToHost, stream));
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    if (herr) throw CudaError{"sparsity pattern: node " + std::to_string(herr - 1) +
                              " has more than " + std::to_string(kPatternCap) + " candidate columns"};
    h_rp.assign(nrows + 1, 0);
    int64_t acc = 0;
    for (int i = 0; i < nrows; ++i) {
      acc += hc[i];
      if (acc > 0x7fffffffLL) throw CudaError{"matrix has more than 2^31 nonzeros"};
      h_rp[i + 1] = (int)acc;
    }
    nnz = acc;
    d_rp = dupload(h_rp);
    d_ci = dalloc<int>((size_t)nnz);
    if (p2)
      k_pattern<true><<<g, kBlock, 0, stream>>>(nrows, (int)nt, adj_ptr, adj, tnode, nullptr, d_rp,
                                                d_ci, d_err);
    else
      k_pattern<false><<<g, kBlock, 0, stream>>>(nrows, (int)nt, adj_ptr, adj, tnode, nullptr, d_rp,
                                                 d_ci, d_err);
    CK(cudaGetLastError());
  }

  void setup(const cfsa_mesh_view *m, const cfsa_fluid *f) {
    CK(cudaGetDevice(&device));
    CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&body_stream2, cudaStreamNonBlocking));
    CK(cudaEventCreate(&ev0));
    CK(cudaEventCreate(&ev1));
    for (cudaEvent_t &e : ph) CK(cudaEventCreate(&e));
    nv = m->nv;
    nt = m->nt;
    ne = m->ne;
    N2 = nv + ne;
    density = f->density;
    viscosity = f->viscosity;
    if (N2 > 0x7fffffffLL / 3 || nt * 16 > 0x7fffffffLL) throw CudaError{"mesh too large for 32-bit indices"};
    // host-side node table (SoA) and boundary tags
    std::vector<int> h_tnode((size_t)nt * 10);
    for (int64_t t = 0; t < nt; ++t) {
      for (int a = 0; a < 4; ++a) {
        const int v = m->tets[4 * t + a];
        if (v < 0 || v >= nv) throw CudaError{"tet references a vertex out of range"};
        h_tnode[(size_t)a * nt + t] = v;
      }
      for (int e = 0; e < 6; ++e) {
        const int id = m->tet_edges[6 * t + e];
        if (id < 0 || id >= ne) throw CudaError{"tet references an edge node out of range"};
        h_tnode[(size_t)(4 + e) * nt + t] = (int)nv + id;
      }
    }
    h_bc.assign((size_t)N2, (signed char)BC_UNDEFINED);
    for (int64_t i = 0; i < nv; ++i) h_bc[i] = m->p1_bc ? m->p1_bc[i] : BC_UNDEFINED;
    for (int64_t k = 0; k < ne; ++k) h_bc[nv + k] = m->p2_bc ? m->p2_bc[k] : BC_UNDEFINED;
    // node -> incident tets, ascending tet order; entry = tet*16 + local node index
    std::vector<int> h_adj_ptr((size_t)N2 + 1, 0), h_adj((size_t)nt * 10);
    for (int64_t t = 0; t < nt; ++t)
      for (int l = 0; l < 10; ++l) h_adj_ptr[h_tnode[(size_t)l * nt + t] + 1]++;
    for (int64_t i = 0; i < N2; ++i) h_adj_ptr[i + 1] += h_adj_ptr[i];
    {
      std::vector<int> fill(h_adj_ptr.begin(), h_adj_ptr.end() - 1);
      for (int64_t t = 0; t < nt; ++t)
        for (int l = 0; l < 10; ++l) h_adj[fill[h_tnode[(size_t)l * nt + t]]++] = (int)(t * 16 + l);
    }
    h_xyz.assign(m->vertices, m->vertices + 3 * nv);
    xyz = dupload(h_xyz);
    tnode = dupload(h_tnode);
    bc = dupload(h_bc);
    adj_ptr = dupload(h_adj_ptr);
    adj = dupload(h_adj);
    vol = dalloc<double>(nt);
    grad = dalloc<double>((size_t)nt * 12);
    k_geometry<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, xyz, tnode, vol, grad);
    CK(cudaGetLastError());
    int *d_err = dalloc<int>(1);
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
    build_pattern(true, (int)N2, h_rp2, rp2, ci2, nnz2, d_err);
    build_pattern(false, (int)nv, h_rp1, rp1, ci1, nnz1, d_err);
    rows2 = dalloc<int>((size_t)nnz2);
    rows1 = dalloc<int>((size_t)nnz1);
    dpos2 = dalloc<int>((size_t)N2);
    dpos1 = dalloc<int>((size_t)nv);
    k_row_of_slot<<<blocks_for(N2), kBlock, 0, stream>>>((int)N2, rp2, rows2);
    k_row_of_slot<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, rp1, rows1);
    k_diag_pos<<<blocks_for(N2), kBlock, 0, stream>>>((int)N2, rp2, ci2, dpos2);
    k_diag_pos<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, rp1, ci1, dpos1);
    CK(cudaGetLastError());
    build_sell((int)N2, h_rp2, s2, rp2, ci2);
    build_sell((int)nv, h_rp1, s1, rp1, ci1);
    tpos1 = dalloc<int>((size_t)nnz1);
    k_transpose_slots<<<blocks_for(nnz1), kBlock, 0, stream>>>(nnz1, rows1, rp1, ci1, tpos1, d_err);
    CK(cudaGetLastError());
    {
      int herr = 0;
      CK(cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      if (herr) throw CudaError{"P1 sparsity pattern is not structurally symmetric"};
    }
    Mv = dalloc<double>((size_t)nnz2);
    Kv = dalloc<double>((size_t)nnz2);
    Ms = dalloc<double>((size_t)s2.nentries);
    At = dalloc<double>((size_t)s2.nentries);
    CK(cudaMemsetAsync(Ms, 0, (size_t)s2.nentries * sizeof(double), stream));
    CK(cudaMemsetAsync(At, 0, (size_t)s2.nentries * sizeof(double), stream));
    diagA = dalloc<double>(N2);
    invA = dalloc<double>(N2);
    Gv = dalloc<double>((size_t)nnz1 * 3);
    Lv = dalloc<double>((size_t)nnz1);
    Ls = dalloc<double>((size_t)s1.nentries);
    Lt = dalloc<double>((size_t)s1.nentries);
    CK(cudaMemsetAsync(Ls, 0, (size_t)s1.nentries * sizeof(double), stream));
    CK(cudaMemsetAsync(Lt, 0, (size_t)s1.nentries * sizeof(double), stream));
    diagL = dalloc<double>(nv);
    invL = dalloc<double>(nv);
    invm = dalloc<double>(N2);
    // fields and work
    const size_t n3 = (size_t)3 * N2;
    u = dalloc<double>(n3);
    ustar = dalloc<double>(n3);
    inlet = dalloc<double>(n3);
    p = dalloc<double>(nv);
    pc = dalloc<double>(nv);
    for (double **w : {&wb, &wr, &wr0, &wp, &wv, &ws, &wt}) *w = dalloc<double>(n3);
    for (double **w : {&pb, &pr, &pz, &pp, &pq, &ps, &pt, &pv, &pu}) *w = dalloc<double>(nv);
    ct = dalloc<double>((size_t)nt * 3);
    divt = dalloc<double>(nt);
    stash = dalloc<double>(1);
    for (double *w : {u, ustar, inlet}) CK(cudaMemsetAsync(w, 0, n3 * sizeof(double), stream));
    CK(cudaMemsetAsync(p, 0, nv * sizeof(double), stream));
    CK(cudaMemsetAsync(pc, 0, nv * sizeof(double), stream));
    h_inlet.assign(n3, 0.0);
    // reductions and states
    const int64_t maxrows = std::max<int64_t>({(int64_t)s2.nrows_pad, nt, N2});
    red.partials = dalloc<double>((size_t)(blocks_for(maxrows) + 1) * kMaxRed);
    red.counter = dalloc<unsigned int>(1);
    CK(cudaMemsetAsync(red.counter, 0, sizeof(unsigned int), stream));
    bs_mom = dalloc<BicgState>(1);
    bs_p = dalloc<BicgState>(1);
    cs = dalloc<CgState>(1);
    st = dalloc<DevStatus>(1);
    st_free = dalloc<DevStatus>(1);
    CK(cudaMemsetAsync(bs_mom, 0, sizeof(BicgState), stream));
    CK(cudaMemsetAsync(bs_p, 0, sizeof(BicgState), stream));
    CK(cudaMemsetAsync(cs, 0, sizeof(CgState), stream));
    CK(cudaMemsetAsync(st, 0, sizeof(DevStatus), stream));
    CK(cudaMemsetAsync(st_free, 0, sizeof(DevStatus), stream));
    CK(cudaMallocHost(&h_st, sizeof(DevStatus)));
    CK(cudaMallocHost(&h_bs, 2 * sizeof(BicgState)));
    CK(cudaMallocHost(&h_cs, sizeof(CgState)));
    CK(cudaMallocHost(&h_stage, n3 * sizeof(double)));
    d_vec3 = dalloc<double>(n3);
    CK(cudaMallocHost(&h_ms, sizeof(MixedState)));
    At32 = dalloc<float>((size_t)s2.nentries);
    invA32 = dalloc<float>((size_t)N2);
    CK(cudaMemsetAsync(At32, 0, (size_t)s2.nentries * sizeof(float), stream));
    for (float **w : {&fr, &fr0, &fp, &fv, &fs, &ft, &fdx}) *w = dalloc<float>(n3);
    ms = dalloc<MixedState>(1);
    CK(cudaMemsetAsync(ms, 0, sizeof(MixedState), stream));
    Ls32 = dalloc<float>((size_t)s1.nentries);
    CK(cudaMemsetAsync(Ls32, 0, (size_t)s1.nentries * sizeof(float), stream));
    for (float **w : {&invL32, &px32, &pp32, &pu32, &pr32[0], &pr32[1], &pw32[0], &pw32[1], &ps32[0], &ps32[1]})
      *w = dalloc<float>((size_t)nv);
    cs_in = dalloc<CgState>(1);
    pmx = dalloc<PMixState>(1);
    CK(cudaMemsetAsync(cs_in, 0, sizeof(CgState), stream));
    CK(cudaMemsetAsync(pmx, 0, sizeof(PMixState), stream));
    CK(cudaMallocHost(&h_pmx, sizeof(PMixState)));
    if (const char *e = std::getenv("CFSA_MIXED_P_TOL_IN")) mixed_p_tol_in = std::atof(e);
    if (const char *e = std::getenv("CFSA_MIXED_DELTA")) mixed_delta = std::atof(e);
    if (const char *e = std::getenv("CFSA_CG2L_SPLIT")) cg2l_split = std::atoi(e) != 0;

    bs_prof = dalloc<BicgState>(1);
    cs_prof = dalloc<CgState>(1);
    ms_prof = dalloc<MixedState>(1);
    // boundary faces
    nbf = m->nbf;
    if (nbf > 0) {
      std::vector<int> hv(m->bface_verts, m->bface_verts + 3 * nbf), ht(m->bface_tet, m->bface_tet + nbf);
      std::vector<double> hn(m->bface_normal, m->bface_normal + 3 * nbf), ha(m->bface_area, m->bface_area + nbf);
      std::vector<int> hvp((size_t)nv + 1, 0), hvf((size_t)nbf * 3);
      for (int64_t fi = 0; fi < nbf; ++fi)
        for (int k = 0; k < 3; ++k) {
          if (hv[3 * fi + k] < 0 || hv[3 * fi + k] >= nv) throw CudaError{"boundary face vertex out of range"};
          hvp[hv[3 * fi + k] + 1]++;
        }
      for (int64_t i = 0; i < nv; ++i) hvp[i + 1] += hvp[i];
      std::vector<int> fill(hvp.begin(), hvp.end() - 1);
      for (int64_t fi = 0; fi < nbf; ++fi)
        for (int k = 0; k < 3; ++k) hvf[fill[hv[3 * fi + k]]++] = (int)fi;
      fverts = dupload(hv);
      ftet = dupload(ht);
      fnormal = dupload(hn);
      farea = dupload(ha);
      vf_ptr = dupload(hvp);
      vf = dupload(hvf);
      fshear = dalloc<double>((size_t)nbf * 3);
      fpress = dalloc<double>((size_t)nbf * 3);
      // vertex -> (face, local index of the vertex in the face's tet), ascending face order
      std::vector<int> hbp((size_t)nv + 1, 0), hb((size_t)nbf * 4);
      for (int64_t fi = 0; fi < nbf; ++fi) {
        if (ht[fi] < 0 || ht[fi] >= nt) throw CudaError{"boundary face tet out of range"};
        for (int l = 0; l < 4; ++l) hbp[h_tnode[(size_t)l * nt + ht[fi]] + 1]++;
      }
      for (int64_t i = 0; i < nv; ++i) hbp[i + 1] += hbp[i];
      std::vector<int> fb(hbp.begin(), hbp.end() - 1);
      for (int64_t fi = 0; fi < nbf; ++fi)
        for (int l = 0; l < 4; ++l) hb[fb[h_tnode[(size_t)l * nt + ht[fi]]]++] = (int)(fi * 4 + l);
      vbf_ptr = dupload(hbp);
      vbf = dupload(hb);
    }
    fout = dalloc<double>((size_t)nv * 3);
    // persistent CG: co-resident grid, barrier words, partial buffers
    {
      int nsm = 0, per_sm = 0;
      CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
      {  // one resident wave per grid-stride reduction kernel
        auto q = [&](const void *fn) {
          int o = 0;
          CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, kBlock, 0));
          stride_ctas_of[fn] = std::max(o, 1) * nsm;
        };
        q((const void *)k_bicg_xr<3>);
        q((const void *)k_bicg_xr<1>);
        q((const void *)k_mcg_xr<3>);
        q((const void *)k_momentum_rhs);
        q((const void *)k_finish_step);
        q((const void *)k_mpc_xr);
        q((const void *)k_mpc_init);
        q((const void *)k_mcg_init<3>);
        q((const void *)k_mp_xr);
        q((const void *)k_mp_init);
        q((const void *)k_pmx_prep);
      }
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_persistent, kBlock, 0));
      const int nblk_sell = (int)blocks_for(s1.nrows_pad), nblk_nat = (int)blocks_for(nv);
      cg_grid = std::min(nsm * per_sm, std::max(nblk_sell, nblk_nat));
      cg_grid = std::min(cg_grid, kBarrierGroupSize * kBarrierGroups);
      bar_count = dalloc<unsigned int>(1 + kBarrierGroups);
      bar_gen = dalloc<unsigned int>(1);
      bar_err = dalloc<int>(1);
      CK(cudaMemsetAsync(bar_count, 0, (1 + kBarrierGroups) * sizeof(unsigned int), stream));
      CK(cudaMemsetAsync(bar_gen, 0, sizeof(unsigned int), stream));
      CK(cudaMemsetAsync(bar_err, 0, sizeof(int), stream));
      cg_part_a = dalloc<double>((size_t)std::max(nblk_sell, nblk_nat) * kMaxRed);
      cg_part_b = dalloc<double>((size_t)std::max(nblk_sell, nblk_nat) * kMaxRed);
      for (double *&v : cg1_vec) v = dalloc<double>((size_t)nv);
      if (cg_grid < 1) cg_persistent = false;
      // resident variant: blocks split into contiguous runs, one run per SM
      int optin = 0;
      CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
      const int grid = std::max(1, std::min(nsm, std::max(nblk_sell, nblk_nat)));
      const int bpc_s = (nblk_sell + grid - 1) / grid, bpc_n = (nblk_nat + grid - 1) / grid;
      int max_entries = 0;
      for (int c = 0; c < grid; ++c) {
        const int b0 = std::min(nblk_sell, c * bpc_s), b1 = std::min(nblk_sell, b0 + bpc_s);
        if (b1 > b0)
          max_entries = std::max(max_entries, s1.h_sptr[std::min(8 * b1, s1.nslices)] - s1.h_sptr[8 * b0]);
      }
      const int64_t row_bytes = (int64_t)3 * bpc_s * kBlock * (int64_t)sizeof(int);
      const int64_t avail = (int64_t)optin - 2048 - row_bytes;  // 2 KiB for static shared memory
      if (avail > 0) {
        cg_res_col_cap = (int)std::min<int64_t>(max_entries, avail / (int64_t)sizeof(int));
        cg_res_smem = (size_t)(row_bytes + (int64_t)cg_res_col_cap * (int64_t)sizeof(int));
        int per_sm_res = 0;
        int per_sm_res1 = 0;
        if (cudaFuncSetAttribute(k_cg_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cg_res_smem) == cudaSuccess &&
            cudaFuncSetAttribute(k_cg1_resident, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)cg_res_smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_res, k_cg_resident, kCgResThreads,
                                                          cg_res_smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_res1, k_cg1_resident, kCgResThreads,
                                                          cg_res_smem) == cudaSuccess &&
            per_sm_res >= 1 && per_sm_res1 >= 1) {
          cg_resident = true;
          cg_res_grid = grid;
          cg_res_bpc_sell = bpc_s;
          cg_res_bpc_nat = bpc_n;
        }
        cudaGetLastError();
      }
    }
    if (const char *e = std::getenv("CFSA_CG_LOOP")) cg_persistent = cg_persistent && (std::atoi(e) == 0);
    // CFSA_CG_KERNEL=persistent selects the 256-thread persistent kernel over the resident one
    if (const char *e = std::getenv("CFSA_CG_KERNEL"))
      if (std::string(e) == "persistent") cg_resident = false;
    assemble();
    if (const char *e = std::getenv("CFSA_NO_GRAPH")) use_graph = (std::atoi(e) == 0);
    CK(cudaStreamSynchronize(stream));
  }

  // buildMassMatrix + buildStiffnessMatrix + buildGradientMatrices + buildPoissonMatrix
  void assemble() {
    NvtxRange nvtx_("cfsa assemble");
    ++geom_gen;
    k_geometry<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, xyz, tnode, vol, grad);
    k_assemble_p2<<<blocks_for(N2), kBlock, 0, stream>>>((int)N2, (int)nt, density, 1.0 / viscosity,
                                                         adj_ptr, adj, tnode, vol, grad, rp2, ci2, Mv, Kv);
    k_assemble_p1<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, (int)nt, nnz1, adj_ptr, adj, tnode,
                                                         vol, grad, rp1, ci1, Gv, Lv);
    k_lumped_mass<<<blocks_for(N2), kBlock, 0, stream>>>((int)N2, rp2, Mv, invm);
    CK(cudaGetLastError());
    mom_dirty = poisson_dirty = true;
  }

  void ensure_operators() {
    if (mom_dirty) {
      k_momentum_diag<<<blocks_for(N2), kBlock, 0, stream>>>((int)N2, dt, dpos2, Mv, Kv, bc, diagA, invA);
      k_momentum_sell<<<blocks_for(nnz2), kBlock, 0, stream>>>(nnz2, dt, s2.posmap, rows2, ci2, Mv, Kv,
                                                               bc, invA, At, Ms,
                                                               mom_krylov == CFSA_KRYLOV_BICGSTAB ? 1 : 0);
      k_to_f32<<<blocks_for(s2.nentries), kBlock, 0, stream>>>(s2.nentries, At, At32);
      k_to_f32<<<blocks_for(N2), kBlock, 0, stream>>>(N2, invA, invA32);
      CK(cudaGetLastError());
      mom_dirty = false;
    }
    if (poisson_dirty) {
      k_poisson_diag<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, outlet_type, ref_node, dpos1, Lv,
                                                            bc, diagL, invL);
      k_poisson_sell<<<blocks_for(nnz1), kBlock, 0, stream>>>(nnz1, outlet_type, ref_node, s1.posmap,
                                                              rows1, ci1, Lv, bc, invL, Ls, Lt);
      k_to_f32<<<blocks_for(s1.nentries), kBlock, 0, stream>>>(s1.nentries, Ls, Ls32);
      k_to_f32<<<blocks_for(nv), kBlock, 0, stream>>>(nv, invL, invL32);
      CK(cudaGetLastError());
      poisson_dirty = false;
      coarse_dirty = true;
    }
    if (krylov == CFSA_KRYLOV_CG2L && coarse_dirty) build_coarse();
  }

  // ------------------------------------------------------------------ two-level preconditioner
  // Coarse space of k_cg2l_resident: geometric aggregates over the vertices without a penalty
  // row, Z = (P^T L P)^-1 by Cholesky, and the index lists of the aggregate sums. Every step of
  // the construction is fixed in order (the oracle's build_coarse follows the same steps), so the
  // device and oracle solves agree bit for bit.
  //   box edge h_k = e c^k, e the largest extent of the bounding box of the unpenalised vertices,
  //   c = 2^-1/4, k in [0, 64] the smallest exponent (bisection) with >= coarse_target occupied
  //   boxes; boxes numbered by first vertex; an A_c that is not SPD disables the coarse part.
  template <class T>
  T *cupload(const std::vector<T> &h) {
    void *ptr = nullptr;
    CK(cudaMalloc(&ptr, std::max<size_t>(h.size(), 1) * sizeof(T)));
    coarse_allocs.push_back(ptr);
    if (!h.empty()) CK(cudaMemcpyAsync(ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return static_cast<T *>(ptr);
  }

  static int count_boxes(const std::vector<double> &xyz, const std::vector<char> &pen, int64_t n,
                         double h, const double lo[3], std::vector<int64_t> *keys_out) {
    std::vector<int64_t> keys;
    keys.reserve(n);
    for (int64_t i = 0; i < n; ++i) {
      if (pen[i]) continue;
      const int64_t ix = (int64_t)std::floor((xyz[3 * i] - lo[0]) / h);
      const int64_t iy = (int64_t)std::floor((xyz[3 * i + 1] - lo[1]) / h);
      const int64_t iz = (int64_t)std::floor((xyz[3 * i + 2] - lo[2]) / h);
      keys.push_back((ix * 2097152 + iy) * 2097152 + iz);
    }
    if (keys_out) *keys_out = keys;
    std::sort(keys.begin(), keys.end());
    return (int)(std::unique(keys.begin(), keys.end()) - keys.begin());
  }

  void build_coarse() {
    NvtxRange nvtx_("cfsa two-level coarse space");
    CK(cudaStreamSynchronize(stream));
    for (void *q : coarse_allocs) CK(cudaFree(q));
    coarse_allocs.clear();
    const int64_t n = nv;
    std::vector<char> pen(n, 0);
    if (outlet_type == CFSA_OUTLET_NEUMANN) {
      if (ref_node >= 0 && ref_node < n) pen[ref_node] = 1;
    } else if (outlet_type == CFSA_OUTLET_DIRICHLET) {
      for (int64_t i = 0; i < n; ++i) pen[i] = h_bc[i] == BC_OUTLET;
    }
    std::vector<int> agg(n, 0);
    int nc = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    bool any = false;
    for (int64_t i = 0; i < n; ++i) {
      if (pen[i]) continue;
      for (int d = 0; d < 3; ++d) {
        const double x = h_xyz[3 * i + d];
        if (!any) lo[d] = hi[d] = x;
        lo[d] = std::min(lo[d], x);
        hi[d] = std::max(hi[d], x);
      }
      any = true;
    }
    const double e = std::max(hi[0] - lo[0], std::max(hi[1] - lo[1], hi[2] - lo[2]));
    if (any && e > 0.0 && coarse_target >= 1) {
      auto h_of = [&](int k) {
        double h = e;
        for (int q = 0; q < k; ++q) h = h * 0.8408964152537145;  // 2^-1/4
        return h;
      };
      int klo = 0, khi = 64;
      while (klo < khi) {
        const int km = (klo + khi) / 2;
        if (count_boxes(h_xyz, pen, n, h_of(km), lo, nullptr) >= coarse_target)
          khi = km;
        else
          klo = km + 1;
      }
      std::vector<int64_t> keys;
      count_boxes(h_xyz, pen, n, h_of(klo), lo, &keys);
      // number the boxes by their first vertex
      std::vector<std::pair<int64_t, int>> kv(keys.size());
      for (size_t q = 0; q < keys.size(); ++q) kv[q] = {keys[q], (int)q};
      std::stable_sort(kv.begin(), kv.end(), [](const std::pair<int64_t, int> &a, const std::pair<int64_t, int> &b) {
        return a.first < b.first;
      });
      std::vector<std::pair<int, int>> firsts;  // (first vertex rank, start in kv)
      for (size_t q = 0; q < kv.size();) {
        size_t r = q;
        while (r < kv.size() && kv[r].first == kv[q].first) ++r;
        firsts.push_back({kv[q].second, (int)q});
        q = r;
      }
      std::sort(firsts.begin(), firsts.end());
      std::vector<int> id_sorted(kv.size()), id_of(keys.size());
      for (size_t gq = 0; gq < firsts.size(); ++gq) {
        size_t q = firsts[gq].second;
        const int64_t key = kv[q].first;
        while (q < kv.size() && kv[q].first == key) id_sorted[q++] = (int)gq;
      }
      for (size_t q = 0; q < kv.size(); ++q) id_of[kv[q].second] = id_sorted[q];
      nc = (int)firsts.size();
      size_t q = 0;
      for (int64_t i = 0; i < n; ++i) agg[i] = pen[i] ? nc : id_of[q++];
    }
    std::vector<double> Z;
    if (nc > 0) {
      // A_c = P^T L P over the unpenalised rows (the penalties sit on penalised rows only)
      std::vector<int> ci((size_t)nnz1);
      std::vector<double> lv((size_t)nnz1);
      CK(cudaMemcpyAsync(ci.data(), ci1, (size_t)nnz1 * sizeof(int), cudaMemcpyDeviceToHost, stream));
      CK(cudaMemcpyAsync(lv.data(), Lv, (size_t)nnz1 * sizeof(double), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      std::vector<double> Ac((size_t)nc * nc, 0.0), G((size_t)nc * nc, 0.0), Gi((size_t)nc * nc, 0.0);
      for (int64_t i = 0; i < n; ++i) {
        if (agg[i] >= nc) continue;
        for (int k = h_rp1[i]; k < h_rp1[i + 1]; ++k) {
          const int j = ci[k];
          if (agg[j] >= nc) continue;
          double &a = Ac[(size_t)agg[i] * nc + agg[j]];
          a = a + lv[k];
        }
      }
      bool spd = true;
      for (int i = 0; i < nc && spd; ++i)
        for (int j = 0; j <= i; ++j) {
          double sum = Ac[(size_t)i * nc + j];
          for (int k = 0; k < j; ++k) sum = sum - G[(size_t)i * nc + k] * G[(size_t)j * nc + k];
          if (i == j) {
            if (!(sum > 0.0)) {
              spd = false;
              break;
            }
            G[(size_t)i * nc + i] = std::sqrt(sum);
          } else {
            G[(size_t)i * nc + j] = sum / G[(size_t)j * nc + j];
          }
        }
      if (!spd) {
        nc = 0;
        std::fill(agg.begin(), agg.end(), 0);
      } else {
        for (int j = 0; j < nc; ++j) {
          Gi[(size_t)j * nc + j] = 1.0 / G[(size_t)j * nc + j];
          for (int i = j + 1; i < nc; ++i) {
            double sum = 0.0;
            for (int k = j; k < i; ++k) sum = sum - G[(size_t)i * nc + k] * Gi[(size_t)k * nc + j];
            Gi[(size_t)i * nc + j] = sum / G[(size_t)i * nc + i];
          }
        }
        Z.assign((size_t)nc * nc, 0.0);
        for (int m = 0; m < nc; ++m)
          for (int k = 0; k < nc; ++k) {
            double sum = 0.0;
            for (int q = std::max(m, k); q < nc; ++q) sum = sum + Gi[(size_t)q * nc + m] * Gi[(size_t)q * nc + k];
            Z[(size_t)m * nc + k] = sum;
          }
      }
    }
    // per CTA: its rows sorted by aggregate (staging positions, one segment per aggregate) and
    // the aggregates of its rows' columns (coarse values it reads)
    const int nblk_sell = (int)blocks_for(s1.nrows_pad);
    std::vector<int> row_pos(n, -1), own_ptr(cg_res_grid + 1, 0), own, seg_lo, seg_hi,
        need_ptr(cg_res_grid + 1, 0), need;
    int npos_max = 0;
    if (nc > 0) {
      std::vector<int> ci((size_t)nnz1);
      CK(cudaMemcpyAsync(ci.data(), ci1, (size_t)nnz1 * sizeof(int), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      for (int c = 0; c < cg_res_grid; ++c) {
        const int b0 = std::min(nblk_sell, c * cg_res_bpc_sell), b1 = std::min(nblk_sell, b0 + cg_res_bpc_sell);
        const int64_t r0 = (int64_t)kBlock * b0, r1 = std::min<int64_t>(n, (int64_t)kBlock * b1);
        std::vector<std::pair<int, int>> rows;  // (aggregate, row)
        std::vector<int> mn;
        for (int64_t i = r0; i < r1; ++i) {
          if (agg[i] < nc) rows.push_back({agg[i], (int)i});
          for (int k = h_rp1[i]; k < h_rp1[i + 1]; ++k)
            if (agg[ci[k]] < nc) mn.push_back(agg[ci[k]]);
        }
        std::sort(rows.begin(), rows.end());
        for (size_t q = 0; q < rows.size(); ++q) {
          row_pos[rows[q].second] = (int)q;
          if (q == 0 || rows[q].first != rows[q - 1].first) {
            own.push_back(rows[q].first);
            seg_lo.push_back((int)q);
            seg_hi.push_back((int)q);
            mn.push_back(rows[q].first);
          }
          seg_hi.back() = (int)q + 1;
        }
        own_ptr[c + 1] = (int)own.size();
        std::sort(mn.begin(), mn.end());
        mn.erase(std::unique(mn.begin(), mn.end()), mn.end());
        need.insert(need.end(), mn.begin(), mn.end());
        need_ptr[c + 1] = (int)need.size();
        npos_max = std::max(npos_max, (int)rows.size());
      }
    }
    // pieces of kSegPiece staging positions per segment, in segment order (seg_sums)
    std::vector<int> own_pfirst(own.size() + 1, 0);
    std::vector<int4> pieces;
    for (size_t q = 0; q < own.size(); ++q) {
      own_pfirst[q] = (int)pieces.size();
      for (int a0 = seg_lo[q]; a0 < seg_hi[q]; a0 += kSegPiece)
        pieces.push_back(make_int4(a0, std::min(seg_hi[q], a0 + kSegPiece), own[q], 0));
    }
    own_pfirst[own.size()] = (int)pieces.size();
    CoarseView V{};
    V.nc = nc;
    V.agg = cupload(agg);
    V.Z = cupload(Z);
    V.row_pos = cupload(row_pos);
    V.own_ptr = cupload(own_ptr);
    V.own = cupload(own);
    V.seg_lo = cupload(seg_lo);
    V.seg_hi = cupload(seg_hi);
    V.own_pfirst = cupload(own_pfirst);
    V.pieces = cupload(pieces);
    V.need_ptr = cupload(need_ptr);
    V.need = cupload(need);
    V.gacc = cupload(std::vector<unsigned long long>((size_t)27 * std::max(nc, 1), 0ull));
    V.npos_max = npos_max;
    // shared memory: coarse arrays, row staging, then as many column indices as fit
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, k_cg2l_resident<double, false>));
    const int64_t coarse_bytes = (int64_t)(6 * nc + 2 + 2 * npos_max) * (int64_t)sizeof(double);
    const int64_t row_bytes = (int64_t)3 * cg_res_bpc_sell * kBlock * (int64_t)sizeof(int);
    const int64_t avail = (int64_t)optin - (int64_t)fa.sharedSizeBytes - coarse_bytes - row_bytes;
    if (avail < 0) throw CudaError{"two-level pressure preconditioner: coarse space too large for shared memory"};
    int max_entries = 0;
    for (int c = 0; c < cg_res_grid; ++c) {
      const int b0 = std::min(nblk_sell, c * cg_res_bpc_sell), b1 = std::min(nblk_sell, b0 + cg_res_bpc_sell);
      if (b1 > b0) max_entries = std::max(max_entries, s1.h_sptr[std::min(8 * b1, s1.nslices)] - s1.h_sptr[8 * b0]);
    }
    cg2l_col_cap = (int)std::min<int64_t>(max_entries, avail / (int64_t)sizeof(int));
    cg2l_smem = (size_t)(coarse_bytes + row_bytes + (int64_t)cg2l_col_cap * (int64_t)sizeof(int));
    int per_sm = 1;
    for (const void *fn : {(const void *)k_cg2l_resident<double, false>, (const void *)k_cg2l_resident<float, false>,
                           (const void *)k_cg2l_resident<double, true>, (const void *)k_cg2l_resident<float, true>}) {
      cudaFuncAttributes fb{};
      CK(cudaFuncGetAttributes(&fb, fn));
      if (fb.sharedSizeBytes > fa.sharedSizeBytes)
        throw CudaError{"two-level pressure preconditioner: float form needs more static shared memory"};
      CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cg2l_smem));
      int o = 0;
      CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, fn, kCgResThreads, cg2l_smem));
      per_sm = std::min(per_sm, o);
    }
    if (per_sm < 1) throw CudaError{"two-level pressure preconditioner: kernel does not fit on an SM"};
    CK(cudaStreamSynchronize(stream));
    coarse_view = V;
    coarse_nc = nc;
    coarse_dirty = false;
    graph_dirty = true;
  }

  // ------------------------------------------------------------------ Krylov loops
  // Appends a WHILE conditional node to the graph being captured on `stream`; its body (one
  // Krylov iteration) is captured from `body` on body_stream. Returns the handle.
  template <class Body>
  void capture_while(Body body) {
    capture_while_on(stream, body_stream, body);
  }

  // WHILE node appended to the graph being captured on `cap`; the body is captured on `sub`.
  template <class Body>
  void capture_while_on(cudaStream_t cap, cudaStream_t sub, Body body) {
    capture_while_with(cap, sub, new_cond_handle(cap), body);
  }

  // Handle of a conditional node of the graph being captured on `cap`. Its default is applied
  // when the top-level graph is launched; a node nested in a loop body must be set by a kernel
  // upstream of it in the same body (k_mp_xr sets the reliable-update IF node every iteration).
  cudaGraphConditionalHandle new_cond_handle(cudaStream_t cap, unsigned int dflt = 1) {
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    CK(cudaStreamGetCaptureInfo(cap, &cst, nullptr, &g, nullptr, nullptr));
    if (cst != cudaStreamCaptureStatusActive) throw CudaError{"stream is not capturing"};
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, dflt, cudaGraphCondAssignDefault));
    return h;
  }

  template <class Body>
  void capture_while_with(cudaStream_t cap, cudaStream_t sub, cudaGraphConditionalHandle h, Body body) {
    capture_cond_with(cap, sub, h, cudaGraphCondTypeWhile, body);
  }

  // Conditional node (WHILE or IF) appended to the graph being captured on `cap`; its body is
  // captured from `body` on `sub`.
  template <class Body>
  void capture_cond_with(cudaStream_t cap, cudaStream_t sub, cudaGraphConditionalHandle h,
                         cudaGraphConditionalNodeType type, Body body) {
    cudaStreamCaptureStatus cst;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(cudaStreamGetCaptureInfo(cap, &cst, nullptr, &g, &deps, &ndeps));
    if (cst != cudaStreamCaptureStatusActive) throw CudaError{"stream is not capturing"};
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = h;
    cp.conditional.type = type;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    CK(cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
    CK(cudaStreamBeginCaptureToGraph(sub, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    body(sub, h, 1);
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(sub, &out));
  }

  // Eager loop: enqueue iterations in growing chunks and poll the active flag in between.
  template <class Body, class ActiveFn>
  void eager_while(Body body, ActiveFn active_of, int maxit) {
    int done = 0, chunk = 2;
    while (done <= maxit) {
      for (int k = 0; k < chunk; ++k) body(stream, (cudaGraphConditionalHandle)0, 0);
      done += chunk;
      if (!active_of()) break;
      chunk = std::min(chunk * 2, 64);
    }
  }

  // Grid of a grid-stride reduction kernel over nblk blocks of 256 positions. The FP32 mixed-
  // precision x/r update and the FP64 x/r update run one resident wave of CTAs that each visit
  // several blocks (fewer CTA-wide barriers and tickets: 325 vs 355 us per FP32 inner iteration,
  // 438 vs 448 us per FP64 iteration at 1M tets). The SELL products of the Krylov loops are
  // run-walking kernels instead (one kRunThreads CTA per SM over a contiguous run of slices).
  template <class K>
  unsigned int strided(K kernel, unsigned int nblk) const {
    auto it = stride_ctas_of.find((const void *)kernel);
    if (it == stride_ctas_of.end()) return nblk;
    const unsigned int need = (nblk + kMaxStride - 1) / kMaxStride;
    return std::min(nblk, std::max(need, (unsigned int)it->second));
  }

  template <int NC>
  void bicg_body(BicgArgs a, cudaStream_t s, const Sell &S, int n) {
    const unsigned int gs = blocks_for(S.nrows_pad), gp = blocks_for(n);
    k_bicg_p<NC><<<gs, kBlock, 0, s>>>(a);
    k_bicg_v<NC><<<S.nruns, kRunThreads, 0, s>>>(a);
    k_bicg_s<NC><<<gp, kBlock, 0, s>>>(a);
    k_bicg_t<NC><<<S.nruns, kRunThreads, 0, s>>>(a);
    k_bicg_xr<NC><<<strided(k_bicg_xr<NC>, gp), kBlock, 0, s>>>(a);
  }

  bool poll_bicg(const BicgState *d) {
    CK(cudaMemcpyAsync(h_bs, d, sizeof(BicgState), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_bs->active != 0;
  }
  bool poll_cg() {
    CK(cudaMemcpyAsync(h_cs, cs, sizeof(CgState), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_cs->active != 0;
  }

  BicgArgs momentum_args(double *x_out = nullptr, DevStatus *s_out = nullptr) {
    BicgArgs a{};
    a.S = s2.view();
    a.At = At;
    a.diagA = diagA;
    a.invA = invA;
    a.b = wb;
    a.x = x_out ? x_out : ustar;
    a.r = wr;
    a.r0 = wr0;
    a.pk = wp;
    a.v = wv;
    a.s = ws;
    a.t = wt;
    a.n = (int)N2;
    a.bs = bs_mom;
    a.red = red;
    a.st = s_out ? s_out : st;
    a.slot = 0;
    a.cw = (conv_norm == CFSA_NORM_JACOBI) ? invA : nullptr;
    a.tol = tol_mom;
    return a;
  }

  // ------------------------------------------------------------------ step phases
  void enqueue_momentum(bool capture) {
    k_tet_conv<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, N2, tnode, grad, u, ct, st);
    MomentumRhsArgs m{};
    m.S = s2.view();
    m.Ms = Ms;
    m.G = CsrView{rp1, ci1};
    m.Gv = Gv;
    m.nnz1 = nnz1;
    m.adj_ptr = adj_ptr;
    m.adj = adj;
    m.vol = vol;
    m.ct = ct;
    m.bc = bc;
    m.inlet = inlet;
    m.u = u;
    m.p = p;
    m.dt = dt;
    m.tol = tol_mom;
    m.n = (int)N2;
    m.nv = (int)nv;
    m.nt = (int)nt;
    m.maxit = maxit_mom;
    m.b = wb;
    m.x = ustar;
    m.r = wr;
    m.r0 = wr0;
    m.pk = wp;
    m.v = wv;
    m.bs = bs_mom;
    m.st = st;
    m.red = red;
    m.cw = (conv_norm == CFSA_NORM_JACOBI) ? invA : nullptr;
    k_momentum_rhs<<<strided(k_momentum_rhs, blocks_for(s2.nrows_pad)), kBlock, 0, stream>>>(m);
    CK(cudaGetLastError());
    enqueue_momentum_krylov(capture, ustar, st);
  }

  // Batched momentum Krylov solve (x = 0, r = b in wb set up by k_momentum_rhs) into x; the
  // check kernel records failures and iteration counts in `s`.
  void enqueue_momentum_krylov(bool capture, double *x, DevStatus *s_out) {
    if (momentum_mixed()) {
      enqueue_momentum_mixed(capture, x, s_out);
      return;
    }
    BicgArgs a = momentum_args(x, s_out);
    const bool cg = (mom_krylov == CFSA_KRYLOV_CG);
    const unsigned int gp = blocks_for(N2);
    if (cg) {
      k_mcg_init<3><<<strided(k_mcg_init<3>, gp), kBlock, 0, stream>>>(a);
      CK(cudaGetLastError());
    }
    auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
      BicgArgs b = a;
      b.cond = h;
      b.use_cond = use;
      if (cg) {
        k_mcg_q<3><<<s2.nruns, kRunThreads, 0, s>>>(b);
        k_mcg_xr<3><<<strided(k_mcg_xr<3>, gp), kBlock, 0, s>>>(b);
        k_mcg_p<3><<<gp, kBlock, 0, s>>>(b);
      } else {
        bicg_body<3>(b, s, s2, (int)N2);
      }
    };
    if (capture)
      capture_while(body);
    else
      eager_while(body, [&] { return poll_bicg(bs_mom); }, maxit_mom);
    k_check_bicg<<<1, 1, 0, stream>>>(bs_mom, 3, 0, s_out);
    CK(cudaGetLastError());
  }

  MixedArgs mixed_args(double *x_out, DevStatus *s_out) {
    MixedArgs a{};
    a.S = s2.view();
    a.At32 = At32;
    a.At64 = At;
    a.diagA = diagA;
    a.invA = invA;
    a.invA32 = invA32;
    a.b = wb;
    a.x = x_out;
    a.r64 = wr;
    a.xs = wv;
    a.r = fr;
    a.r0 = fr0;
    a.p = fp;
    a.v = fv;
    a.s = fs;
    a.t = ft;
    a.dx = fdx;
    a.n = (int)N2;
    a.ms = ms;
    a.st = s_out;
    a.red = red;
    a.cw = (conv_norm == CFSA_NORM_JACOBI) ? invA : nullptr;
    a.cw32 = (conv_norm == CFSA_NORM_JACOBI) ? invA32 : nullptr;
    return a;
  }

  // FP32 BiCGSTAB with FP64 reliable updates (ns_mixed.cuh). Captured: a WHILE node whose body
  // is one iteration followed by an IF node holding the reliable update; eager: the update
  // kernels run after every iteration and return at once when no component asked for one.
  void enqueue_momentum_mixed(bool capture, double *x, DevStatus *s_out) {
    if (mom_krylov == CFSA_KRYLOV_CG) {
      enqueue_momentum_mixed_cg(capture, x, s_out);
      return;
    }
    const MixedArgs a = mixed_args(x, s_out);
    const unsigned int gp = blocks_for(N2);
    k_mp_init<<<strided(k_mp_init, gp), kBlock, 0, stream>>>(a, tol_mom, maxit_mom, mixed_delta_of_method());
    CK(cudaGetLastError());
    auto update_body = [&](cudaStream_t s, MixedArgs b) {
      k_mp_xupdate<<<gp, kBlock, 0, s>>>(b);
      k_mp_residual<<<s2.nruns, kRunThreads, 0, s>>>(b);
    };
    auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
      MixedArgs b = a;
      b.cond = h;
      b.use_cond = use;
      b.use_if = use;
      if (b.use_if) b.cond_upd = new_cond_handle(s, 0);
      k_mp_p<<<gp, kBlock, 0, s>>>(b);
      k_mp_v<<<s2.nruns, kRunThreads, 0, s>>>(b);
      k_mp_s<<<gp, kBlock, 0, s>>>(b);
      k_mp_t<<<s2.nruns, kRunThreads, 0, s>>>(b);
      k_mp_xr<<<strided(k_mp_xr, gp), kBlock, 0, s>>>(b);
      if (b.use_if)
        capture_cond_with(s, body_stream2, b.cond_upd, cudaGraphCondTypeIf,
                          [&](cudaStream_t ss, cudaGraphConditionalHandle, int) { update_body(ss, b); });
      else
        update_body(s, b);
    };
    if (capture)
      capture_while(body);
    else
      eager_while(body, [&] { return poll_mixed(); }, maxit_mom);
    k_mp_check<<<1, 1, 0, stream>>>(ms, s_out);
    CK(cudaGetLastError());
  }

  // FP32 CG with FP64 reliable updates (ns_mixed.cuh, k_mpc_*): per iteration the product, the
  // x/r update and, after the reliable-update IF node, the direction update.
  void enqueue_momentum_mixed_cg(bool capture, double *x, DevStatus *s_out) {
    const MixedArgs a = mixed_args(x, s_out);
    const unsigned int gp = blocks_for(N2);
    k_mpc_init<<<strided(k_mpc_init, gp), kBlock, 0, stream>>>(a, tol_mom, maxit_mom, mixed_delta_of_method());
    CK(cudaGetLastError());
    auto update_body = [&](cudaStream_t s, MixedArgs b) {
      k_mpc_xupdate<<<gp, kBlock, 0, s>>>(b);
      k_mpc_residual<<<s2.nruns, kRunThreads, 0, s>>>(b);
    };
    auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
      MixedArgs b = a;
      b.cond = h;
      b.use_cond = use;
      b.use_if = use;
      if (b.use_if) b.cond_upd = new_cond_handle(s, 0);
      k_mpc_q<<<s2.nruns, kRunThreads, 0, s>>>(b);
      k_mpc_xr<<<strided(k_mpc_xr, gp), kBlock, 0, s>>>(b);
      if (b.use_if)
        capture_cond_with(s, body_stream2, b.cond_upd, cudaGraphCondTypeIf,
                          [&](cudaStream_t ss, cudaGraphConditionalHandle, int) { update_body(ss, b); });
      else
        update_body(s, b);
      k_mpc_p<<<gp, kBlock, 0, s>>>(b);
    };
    if (capture)
      capture_while(body);
    else
      eager_while(body, [&] { return poll_mixed(); }, maxit_mom);
    k_mp_check<<<1, 1, 0, stream>>>(ms, s_out);
    CK(cudaGetLastError());
  }

  bool poll_mixed() {
    CK(cudaMemcpyAsync(h_ms, ms, sizeof(MixedState), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_ms->active != 0;
  }

  void enqueue_pressure_solve(bool capture) {
    k_tet_div<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, N2, tnode, grad, ustar, divt, st);
    const PressureRhsArgs a = pressure_rhs_args(pc, st);
    k_pressure_rhs<<<blocks_for(nv), kBlock, 0, stream>>>(a);
    CK(cudaGetLastError());
    enqueue_pressure_krylov(capture, pc, st);
  }

  PressureRhsArgs pressure_rhs_args(double *x, DevStatus *s_out) {
    PressureRhsArgs a{};
    a.adj_ptr = adj_ptr;
    a.adj = adj;
    a.vol = vol;
    a.divt = divt;
    a.bc = bc;
    a.invL = invL;
    a.dt = dt;
    a.tol = tol_p;
    a.outlet_pressure = outlet_pressure;
    a.nv = (int)nv;
    a.outlet_type = outlet_type;
    a.ref_node = ref_node;
    a.maxit = maxit_p;
    a.krylov = (krylov == CFSA_KRYLOV_BICGSTAB) ? 1 : 0;
    a.scaled = (conv_norm == CFSA_NORM_JACOBI) ? 1 : 0;
    a.b = pb;
    a.x = x;
    a.r = pr;
    a.z_or_r0 = pz;
    a.pk = pp;
    a.v = pv;
    a.cs = cs;
    a.bs = bs_p;
    a.st = s_out;
    a.red = red;
    return a;
  }

  // Arguments of the resident two-level CG (FP64 form into x; the float form's vectors are the
  // handle's FP32 pressure buffers).
  Cg2lArgs cg2l_args(double *x, DevStatus *s_out, CgState *state) {
    CgPersistentArgs c{};
    c.S = s1.view();
    c.Ls = Ls;
    c.invL = invL;
    c.x = x;
    c.r = pr;
    c.z = pz;
    c.q = pq;
    c.p[0] = pp;
    c.p[1] = ps;
    c.n = (int)nv;
    c.nblk_sell = (int)blocks_for(s1.nrows_pad);
    c.nblk_nat = (int)blocks_for(nv);
    c.part_a = cg_part_a;
    c.part_b = cg_part_b;
    c.cs = state;
    c.st = s_out;
    c.bar = GridBarrier{bar_count, bar_gen, bar_err, bar_spin_limit};
    c.scaled = (conv_norm == CFSA_NORM_JACOBI) ? 1 : 0;
    CgResidentArgs rz{};
    rz.P = c;
    rz.nslices = s1.nslices;
    rz.bpc_sell = cg_res_bpc_sell;
    rz.bpc_nat = cg_res_bpc_nat;
    rz.col_cap = cg2l_col_cap;
    Cg2lArgs c2{};
    c2.R = rz;
    c2.V = coarse_view;
    c2.r[0] = pr;
    c2.r[1] = cg1_vec[0];
    c2.w[0] = pq;
    c2.w[1] = cg1_vec[1];
    c2.s[0] = ps;
    c2.s[1] = cg1_vec[2];
    c2.p = pp;
    c2.Ls32 = Ls32;
    c2.invL32 = invL32;
    c2.x32 = px32;
    c2.p32 = pp32;
    c2.u = pu;
    c2.u32 = pu32;
    for (int q = 0; q < 2; ++q) {
      c2.r32[q] = pr32[q];
      c2.w32[q] = pw32[q];
      c2.s32[q] = ps32[q];
    }
    return c2;
  }

  // One cooperative launch of the two-level CG on `s` (barrier words and coarse accumulators
  // cleared first; the caller zeroes p and s[0] of the form it launches).
  void launch_cg2l(const Cg2lArgs &c2, bool f32, cudaStream_t s) {
    CK(cudaMemsetAsync(bar_count, 0, (1 + kBarrierGroups) * sizeof(unsigned int), s));
    CK(cudaMemsetAsync(bar_err, 0, sizeof(int), s));
    if (coarse_view.nc > 0)
      CK(cudaMemsetAsync(coarse_view.gacc, 0, (size_t)27 * coarse_view.nc * sizeof(unsigned long long), s));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned int)cg_res_grid);
    cfg.blockDim = dim3(kCgResThreads);
    cfg.dynamicSmemBytes = cg2l_smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (f32)
      CK(cudaLaunchKernelEx(&cfg, cg2l_split ? k_cg2l_resident<float, true> : k_cg2l_resident<float, false>, c2));
    else
      CK(cudaLaunchKernelEx(&cfg, cg2l_split ? k_cg2l_resident<double, true> : k_cg2l_resident<double, false>, c2));
  }

  // Mixed-precision pressure solve (ns_mixed.cuh): FP64 defect correction around the float
  // two-level CG; the sweeps are a WHILE node when captured.
  void enqueue_pressure_mixed(bool capture, double *x, DevStatus *s_out) {
    PMixArgs a{};
    a.S = s1.view();
    a.Ls = Ls;
    a.invL = invL;
    a.invL32 = invL32;
    a.b = pb;
    a.x = x;
    a.r = pr;
    a.r32 = pr32[0];
    a.x32 = px32;
    a.p32 = pp32;
    a.s32 = ps32[0];
    a.n = (int)nv;
    a.scaled = (conv_norm == CFSA_NORM_JACOBI) ? 1 : 0;
    a.maxit = maxit_p;
    a.cs = cs;
    a.cs_in = cs_in;
    a.pm = pmx;
    a.st = s_out;
    a.red = red;
    a.bar_err = bar_err;
    k_pmx_init<<<1, 1, 0, stream>>>(a, mixed_p_tol_in, mixed_p_max_sweeps);
    CK(cudaGetLastError());
    const Cg2lArgs c2 = cg2l_args(x, s_out, cs_in);
    const unsigned int gp = blocks_for(nv);
    auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
      PMixArgs b = a;
      b.cond = h;
      b.use_cond = use;
      k_pmx_prep<<<strided(k_pmx_prep, gp), kBlock, 0, s>>>(b);
      launch_cg2l(c2, true, s);
      k_pmx_xupdate<<<gp, kBlock, 0, s>>>(b);
      k_pmx_residual<<<blocks_for(s1.nrows_pad), kBlock, 0, s>>>(b);
    };
    if (capture)
      capture_while(body);
    else
      eager_while(body, [&] { return poll_pmx(); }, mixed_p_max_sweeps);
    k_pmx_check<<<1, 1, 0, stream>>>(a, s_out);
    CK(cudaGetLastError());
  }

  bool poll_pmx() {
    CK(cudaMemcpyAsync(h_pmx, pmx, sizeof(PMixState), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_pmx->active != 0;
  }

  // Pressure Krylov solve (state set up by k_pressure_rhs) into x; failures and iteration
  // counts go to `s_out`. Mixed precision applies to the two-level CG (the other methods solve
  // in FP64 in both precisions).
  void enqueue_pressure_krylov(bool capture, double *x, DevStatus *s_out) {
    if (pressure_mixed()) {
      enqueue_pressure_mixed(capture, x, s_out);
      return;
    }
    if (krylov == CFSA_KRYLOV_BICGSTAB) {
      BicgArgs b{};
      b.S = s1.view();
      b.At = Lt;
      b.diagA = diagL;
      b.invA = invL;
      b.b = pb;
      b.x = x;
      b.r = pr;
      b.r0 = pz;
      b.pk = pp;
      b.v = pv;
      b.s = ps;
      b.t = pt;
      b.n = (int)nv;
      b.bs = bs_p;
      b.red = red;
      b.st = s_out;
      b.slot = 1;
      b.cw = (conv_norm == CFSA_NORM_JACOBI) ? invL : nullptr;
      auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
        BicgArgs c = b;
        c.cond = h;
        c.use_cond = use;
        bicg_body<1>(c, s, s1, (int)nv);
      };
      if (capture)
        capture_while(body);
      else
        eager_while(body, [&] { return poll_bicg(bs_p); }, maxit_p);
      k_check_bicg<<<1, 1, 0, stream>>>(bs_p, 1, 1, s_out);
    } else if (cg_persistent || krylov == CFSA_KRYLOV_CG1 || krylov == CFSA_KRYLOV_CG2L) {
      CgPersistentArgs c{};
      c.S = s1.view();
      c.Ls = Ls;
      c.invL = invL;
      c.x = x;
      c.r = pr;
      c.z = pz;
      c.q = pq;
      c.p[0] = pp;
      c.p[1] = ps;
      c.n = (int)nv;
      c.nblk_sell = (int)blocks_for(s1.nrows_pad);
      c.nblk_nat = (int)blocks_for(nv);
      c.part_a = cg_part_a;
      c.part_b = cg_part_b;
      c.cs = cs;
      c.st = s_out;
      c.bar = GridBarrier{bar_count, bar_gen, bar_err, bar_spin_limit};
      c.scaled = (conv_norm == CFSA_NORM_JACOBI) ? 1 : 0;
      CK(cudaMemsetAsync(bar_count, 0, (1 + kBarrierGroups) * sizeof(unsigned int), stream));
      CK(cudaMemsetAsync(bar_err, 0, sizeof(int), stream));
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned int)cg_grid);
      cfg.blockDim = dim3(kBlock);
      cfg.stream = stream;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeCooperative;
      attr[0].val.cooperative = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if (krylov == CFSA_KRYLOV_CG2L) {
        CK(cudaMemsetAsync(pp, 0, (size_t)nv * sizeof(double), stream));
        CK(cudaMemsetAsync(ps, 0, (size_t)nv * sizeof(double), stream));
        launch_cg2l(cg2l_args(x, s_out, cs), false, stream);
      } else if (krylov == CFSA_KRYLOV_CG1) {
        CgResidentArgs rz{};
        rz.P = c;
        rz.nslices = s1.nslices;
        rz.bpc_sell = cg_res_bpc_sell;
        rz.bpc_nat = cg_res_bpc_nat;
        rz.col_cap = cg_res_col_cap;
        Cg1Args c1{};
        c1.R = rz;
        c1.r[0] = pr;
        c1.r[1] = cg1_vec[0];
        c1.w[0] = pq;
        c1.w[1] = cg1_vec[1];
        c1.s[0] = ps;
        c1.s[1] = cg1_vec[2];
        c1.u0 = pz;
        c1.p = pp;
        CK(cudaMemsetAsync(pp, 0, (size_t)nv * sizeof(double), stream));
        CK(cudaMemsetAsync(ps, 0, (size_t)nv * sizeof(double), stream));
        cfg.gridDim = dim3((unsigned int)cg_res_grid);
        cfg.blockDim = dim3(kCgResThreads);
        cfg.dynamicSmemBytes = cg_res_smem;
        CK(cudaLaunchKernelEx(&cfg, k_cg1_resident, c1));
      } else if (cg_resident) {
        CgResidentArgs rz{};
        rz.P = c;
        rz.nslices = s1.nslices;
        rz.bpc_sell = cg_res_bpc_sell;
        rz.bpc_nat = cg_res_bpc_nat;
        rz.col_cap = cg_res_col_cap;
        cfg.gridDim = dim3((unsigned int)cg_res_grid);
        cfg.blockDim = dim3(kCgResThreads);
        cfg.dynamicSmemBytes = cg_res_smem;
        CK(cudaLaunchKernelEx(&cfg, k_cg_resident, rz));
      } else {
        CK(cudaLaunchKernelEx(&cfg, k_cg_persistent, c));
      }
      k_check_cg<<<1, 1, 0, stream>>>(cs, s_out, bar_err);
    } else {
      CgArgs c{};
      c.S = s1.view();
      c.Ls = Ls;
      c.invL = invL;
      c.x = x;
      c.r = pr;
      c.z = pz;
      c.pk = pp;
      c.q = pq;
      c.n = (int)nv;
      c.cs = cs;
      c.red = red;
      c.st = s_out;
      c.scaled = (conv_norm == CFSA_NORM_JACOBI) ? 1 : 0;
      auto body = [&](cudaStream_t s, cudaGraphConditionalHandle h, int use) {
        CgArgs d = c;
        d.cond = h;
        d.use_cond = use;
        k_cg_q<<<blocks_for(s1.nrows_pad), kBlock, 0, s>>>(d);
        k_cg_xr<<<blocks_for(nv), kBlock, 0, s>>>(d);
        k_cg_p<<<blocks_for(nv), kBlock, 0, s>>>(d);
      };
      if (capture)
        capture_while(body);
      else
        eager_while(body, [&] { return poll_cg(); }, maxit_p);
      k_check_cg<<<1, 1, 0, stream>>>(cs, s_out, nullptr);
    }
    CK(cudaGetLastError());
  }

  // NavierStokesSolver::solvePressureBiCGSTAB (src/FEM/NavierStokes.cpp:773-802): Jacobi
  // BiCGSTAB on the raw Poisson matrix, zero initial guess, stopping rule ||r|| <= tol ||b||.
  // Uses the pressure solve's work vectors and leaves the solver's fields untouched.
  int solve_poisson_raw(const double *rhs, double *x_host, double tol, int maxit) {
    ensure_operators();
    if (!Lraw_t) {
      Lraw_t = dalloc<double>((size_t)s1.nentries);
      diag_raw = dalloc<double>((size_t)nv);
      inv_raw = dalloc<double>((size_t)nv);
      CK(cudaMemsetAsync(Lraw_t, 0, (size_t)s1.nentries * sizeof(double), stream));
    }
    if (raw_gen != geom_gen) {
      k_poisson_diag<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, -1, -1, dpos1, Lv, bc, diag_raw, inv_raw);
      k_poisson_sell<<<blocks_for(nnz1), kBlock, 0, stream>>>(nnz1, -1, -1, s1.posmap, rows1, ci1, Lv, bc,
                                                              inv_raw, nullptr, Lraw_t);
      CK(cudaGetLastError());
      raw_gen = geom_gen;
    }
    double *d_b = d_vec3, *d_x = d_vec3 + nv;  // staging buffer, 3 N2 >= 2 nv doubles
    CK(cudaMemcpyAsync(d_b, rhs, (size_t)nv * sizeof(double), cudaMemcpyHostToDevice, stream));
    reset_status();
    PressureRhsArgs a = pressure_rhs_args(d_x, st);
    a.given_b = d_b;
    a.invL = inv_raw;
    a.tol = tol;
    a.maxit = maxit;
    a.krylov = 1;
    a.scaled = 0;
    k_pressure_rhs<<<blocks_for(nv), kBlock, 0, stream>>>(a);
    CK(cudaGetLastError());
    BicgArgs b{};
    b.S = s1.view();
    b.At = Lraw_t;
    b.diagA = diag_raw;
    b.invA = inv_raw;
    b.b = pb;
    b.x = d_x;
    b.r = pr;
    b.r0 = pz;
    b.pk = pp;
    b.v = pv;
    b.s = ps;
    b.t = pt;
    b.n = (int)nv;
    b.bs = bs_p;
    b.red = red;
    b.st = st;
    b.slot = 1;
    b.cw = nullptr;
    auto body = [&](cudaStream_t s, cudaGraphConditionalHandle hc, int use) {
      BicgArgs c = b;
      c.cond = hc;
      c.use_cond = use;
      bicg_body<1>(c, s, s1, (int)nv);
    };
    eager_while(body, [&] { return poll_bicg(bs_p); }, maxit);
    k_check_bicg<<<1, 1, 0, stream>>>(bs_p, 1, 1, st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(x_host, d_x, (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    return h_st->code;
  }

  void enqueue_pressure_update() {
    k_pressure_update<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, relax_p, outlet_type,
                                                             outlet_pressure, bc, pc, p, st);
    if (ref_node >= 0 && ref_node < nv) {
      k_pressure_stash<<<1, 1, 0, stream>>>(ref_node, p, stash, st);
      k_pressure_normalize<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, stash, p, st);
    }
    CK(cudaGetLastError());
  }

  void enqueue_correct() {
    CorrectArgs c{};
    c.G = CsrView{rp1, ci1};
    c.Gv = Gv;
    c.nnz1 = nnz1;
    c.invm = invm;
    c.pc = pc;
    c.ustar = ustar;
    c.inlet = inlet;
    c.bc = bc;
    c.dt = dt;
    c.relax_u = relax_u;
    c.n = (int)N2;
    c.nv = (int)nv;
    c.u = u;
    c.st = st;
    k_correct_velocity<<<blocks_for(N2), kBlock, 0, stream>>>(c);
    CK(cudaGetLastError());
  }

  void enqueue_finish() {
    FinishArgs f{};
    f.bc = bc;
    f.inlet = inlet;
    f.u = u;
    f.ustar = ustar;
    f.p = p;
    f.pc = pc;
    f.n = (int)N2;
    f.nv = (int)nv;
    f.st = st;
    f.red = red;
    k_finish_step<<<strided(k_finish_step, blocks_for(N2)), kBlock, 0, stream>>>(f);
    CK(cudaGetLastError());
  }

  // pisoStep (ncorr correctors) or simpleStep (one corrector). The 2nd and later correctors of
  // the reference solve the identical system again (the divergence is always that of u*), so
  // their pressure correction is the first one's; only the p update and u correction repeat.
  // Phase boundary; inside stream capture it must become an event-record node of the graph.
  void mark_phase(int k, bool capture) {
    if (capture)
      CK(cudaEventRecordWithFlags(ph[k], stream, cudaEventRecordExternal));
    else
      CK(cudaEventRecord(ph[k], stream));
  }

  void enqueue_step(bool capture, bool simple) {
    mark_phase(0, capture);
    enqueue_momentum(capture);
    mark_phase(1, capture);
    const int nc = simple ? 1 : ncorr;
    const bool normalize = (ref_node >= 0 && ref_node < nv);
    for (int c = 0; c < nc; ++c) {
      if (c == 0) {
        enqueue_pressure_solve(capture);
        mark_phase(2, capture);
      }
      enqueue_pressure_update();
      enqueue_correct();
    }
    if (nc == 0) mark_phase(2, capture);
    enqueue_finish();
    mark_phase(3, capture);
    // tet_conv, momentum_rhs, check, [tet_div, pressure_rhs, check], per corrector
    // update (+ stash + normalize) and correct, finish
    launches_per_step = 3 + (nc > 0 ? 3 : 0) + nc * (2 + (normalize ? 2 : 0)) + 1;
  }

  void ensure_graph() {
    if (!graph_dirty && graph_exec) return;
    if (graph_exec) {
      CK(cudaGraphExecDestroy(graph_exec));
      graph_exec = nullptr;
    }
    if (graph) {
      CK(cudaGraphDestroy(graph));
      graph = nullptr;
    }
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
      enqueue_step(true, false);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(stream, &graph));
    CK(cudaGraphInstantiate(&graph_exec, graph, 0));
    graph_dirty = false;
  }

  void reset_status() { CK(cudaMemsetAsync(st, 0, sizeof(DevStatus), stream)); }

  // Kernels of one pressure-solve body run (counted by DevStatus::body_runs[1]) and the extra
  // fixed kernels of a mixed-precision step, for the launch counts.
  bool momentum_mixed() const { return precision != CFSA_PRECISION_FP64; }
  bool pressure_mixed() const { return precision == CFSA_PRECISION_MIXED_FULL && krylov == CFSA_KRYLOV_CG2L; }
  int pressure_body_kernels() const {
    if (pressure_mixed()) return 4;  // prep, float two-level CG, x update, FP64 residual
    if (krylov == CFSA_KRYLOV_BICGSTAB) return 5;
    return (cg_persistent || krylov == CFSA_KRYLOV_CG1 || krylov == CFSA_KRYLOV_CG2L) ? 1 : 3;
  }
  // Kernels of one momentum-solve body run (DevStatus::body_runs[0]): BiCGSTAB 5, CG 3.
  bool momentum_cg() const { return !momentum_mixed() && mom_krylov == CFSA_KRYLOV_CG; }
  int momentum_body_kernels() const { return mom_krylov == CFSA_KRYLOV_CG ? 3 : 5; }
  int mixed_fixed_kernels() const {
    return (momentum_mixed() ? 1 : 0) + (pressure_mixed() ? 1 : 0) + (momentum_cg() ? 1 : 0);
  }

  int finish_batch(int launched_steps) {
    CK(cudaMemcpyAsync(h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    CK(cudaEventSynchronize(ev1));
    CK(cudaStreamSynchronize(stream));
    CK(cudaEventElapsedTime(&last_ms, ev0, ev1));
    const int pressure_body = pressure_body_kernels();
    // momentum: 5 kernels per BiCGSTAB iteration, 3 per CG iteration; mixed momentum: 2 more per
    // reliable update (x update, residual) and an init kernel per solve, as has FP64 CG; mixed
    // two-level CG pressure: 4 kernels per sweep plus its init
    batch_launches = (int64_t)launched_steps * (launches_per_step + mixed_fixed_kernels()) +
                     momentum_body_kernels() * (int64_t)h_st->body_runs[0] +
                     pressure_body * (int64_t)h_st->body_runs[1] +
                     2 * (int64_t)h_st->body_runs[2];
    batch_iters[0] = (int64_t)h_st->iters[0];
    batch_iters[1] = (int64_t)h_st->iters[1];
    for (int64_t k = 0; k < h_st->steps_done; ++k) time += dt;
    steps += h_st->steps_done;
    return h_st->code;
  }

  int run_steps(int n, int *n_done, bool simple) {
    NvtxRange nvtx_("cfsa steps");
    ensure_operators();
    reset_status();
    int launched = 0;
    if (use_graph && !simple) {
      ensure_graph();
      CK(cudaEventRecord(ev0, stream));
      for (int k = 0; k < n; ++k) CK(cudaGraphLaunch(graph_exec, stream));
      launched = n;
      CK(cudaEventRecord(ev1, stream));
    } else {
      CK(cudaEventRecord(ev0, stream));
      for (int k = 0; k < n; ++k) {
        enqueue_step(false, simple);
        ++launched;
        CK(cudaMemcpyAsync(h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (h_st->halt) break;
      }
      CK(cudaEventRecord(ev1, stream));
    }
    const int code = finish_batch(launched);
    if (n_done) *n_done = h_st->steps_done;
    return code;
  }

  // [N2][3] host layout <-> component-major device layout through pinned staging.
  // [3][N2] device field -> caller's [N2][3] host array (one copy; fast when the caller's memory
  // is pinned, staged by the driver otherwise)
  void download_vec3(const double *d, double *out) {
    k_vec3_interleave<<<blocks_for(3 * N2), kBlock, 0, stream>>>(N2, d, d_vec3);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d_vec3, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  // Stream-ordered read-back of u (node-major [N2][3]) or p into a host array: the staging copy is
  // taken on `stream` after the work enqueued so far, then copied to `out` on copy_stream. The
  // next read-back of the same field first waits for this copy to finish with the staging buffer.
  void readback_async(bool velocity, double *out) {
    if (!copy_stream) {
      CK(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
      for (cudaEvent_t *e : {&ev_u_ready, &ev_u_done, &ev_p_ready, &ev_p_done})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
      out_u = dalloc<double>((size_t)3 * N2);
      out_p = dalloc<double>((size_t)nv);
    }
    cudaEvent_t ready = velocity ? ev_u_ready : ev_p_ready, done = velocity ? ev_u_done : ev_p_done;
    CK(cudaStreamWaitEvent(stream, done, 0));
    size_t bytes;
    if (velocity) {
      k_vec3_interleave<<<blocks_for(3 * N2), kBlock, 0, stream>>>(N2, u, out_u);
      CK(cudaGetLastError());
      bytes = (size_t)3 * N2 * sizeof(double);
    } else {
      CK(cudaMemcpyAsync(out_p, p, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      bytes = (size_t)nv * sizeof(double);
    }
    CK(cudaEventRecord(ready, stream));
    CK(cudaStreamWaitEvent(copy_stream, ready, 0));
    CK(cudaMemcpyAsync(out, velocity ? out_u : out_p, bytes, cudaMemcpyDeviceToHost, copy_stream));
    CK(cudaEventRecord(done, copy_stream));
  }

  void upload_vec3(const double *in, double *d) {
    CK(cudaMemcpyAsync(d_vec3, in, (size_t)3 * N2 * sizeof(double), cudaMemcpyHostToDevice, stream));
    k_vec3_split<<<blocks_for(3 * N2), kBlock, 0, stream>>>(N2, d_vec3, d);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(stream));
  }
  // the host mirror of the inlet values (fingerprint, field initialisation)
  const std::vector<double> &host_inlet() {
    if (h_inlet_stale) {
      CK(cudaMemcpyAsync(h_inlet.data(), inlet, h_inlet.size() * sizeof(double), cudaMemcpyDeviceToHost, stream));
      CK(cudaStreamSynchronize(stream));
      h_inlet_stale = false;
    }
    return h_inlet;
  }

  // ------------------------------------------------------------------ discrete adjoint
  // Everything the recorded forward pass depends on besides the state: parameters, inlet
  // values, boundary tags and the geometry generation. The backward pass refuses to run when
  // it differs from the value taken at recording time.
  uint64_t adjoint_fingerprint() {
    uint64_t hsh = 1469598103934665603ull;
    auto mix = [&](const void *ptr, size_t nb) {
      const unsigned char *b = static_cast<const unsigned char *>(ptr);
      for (size_t k = 0; k < nb; ++k) hsh = (hsh ^ b[k]) * 1099511628211ull;
    };
    const double d[] = {dt, tol_mom, tol_p, relax_u, relax_p, outlet_pressure, viscosity, density,
                        mixed_delta};
    const int64_t k[] = {maxit_mom, maxit_p, ncorr, outlet_type, ref_node, krylov, precision,
                         conv_norm, geom_gen, (int64_t)cg_persistent, mom_krylov};
    mix(d, sizeof(d));
    mix(k, sizeof(k));
    const std::vector<double> &hin = host_inlet();
    mix(hin.data(), hin.size() * sizeof(double));
    mix(h_bc.data(), h_bc.size());
    return hsh;
  }

  void ensure_adjoint_work() {
    if (adj_work) return;
    const size_t n3 = (size_t)3 * N2;
    a_lu = dalloc<double>(n3);
    a_x = dalloc<double>(n3);
    a_gin = dalloc<double>(n3);
    a_us = dalloc<double>(n3);
    a_lp = dalloc<double>(nv);
    a_px = dalloc<double>(nv);
    a_lpp = dalloc<double>(nv);
    a_q = dalloc<double>((size_t)3 * nv);
    a_un = dalloc<double>((size_t)3 * nv);
    a_w = dalloc<double>((size_t)3 * nv);
    a_W = dalloc<double>((size_t)3 * std::max<int64_t>(nbf, 1));
    a_tsc = dalloc<double>((size_t)9 * nt);
    a_scal = dalloc<double>(4);
    a_mask = dalloc<signed char>(nv);
    st_adj = dalloc<DevStatus>(1);
    CK(cudaMemsetAsync(a_scal, 0, 4 * sizeof(double), stream));
    adj_work = true;
  }

  int64_t rec_slot_doubles() const { return 3 * nv + 3 * N2; }
  int64_t ck_slot_doubles() const { return 3 * N2 + nv; }

  // Checkpoint and record storage for nsteps steps in segments of C (C <= 0: automatic).
  void plan_records(int nsteps, int C) {
    for (void *ptr : rec_allocs) CK(cudaFree(ptr));
    rec_allocs.clear();
    a_rec = a_ck = a_fin = nullptr;
    const int64_t slot_b = rec_slot_doubles() * (int64_t)sizeof(double);
    if (C <= 0) {
      size_t freeb = 0, totb = 0;
      CK(cudaMemGetInfo(&freeb, &totb));
      const int64_t fit = (int64_t)(freeb / 2) / std::max<int64_t>(slot_b, 1);
      C = (int)std::max<int64_t>(1, std::min<int64_t>(fit, nsteps));
    }
    C = std::max(1, std::min(C, std::max(nsteps, 1)));
    adj_C = C;
    adj_nseg = (nsteps + C - 1) / C;
    a_rec_slots = C;
    a_ck_slots = std::max(adj_nseg, 1);
    auto alloc = [&](int64_t count) {
      void *ptr = nullptr;
      CK(cudaMalloc(&ptr, (size_t)std::max<int64_t>(count, 1) * sizeof(double)));
      rec_allocs.push_back(ptr);
      return static_cast<double *>(ptr);
    };
    a_rec = alloc(a_rec_slots * rec_slot_doubles());
    a_ck = alloc(a_ck_slots * ck_slot_doubles());
    a_fin = alloc((int64_t)6 * N2 + 2 * nv);
  }

  double *rec_u1(int slot) const { return a_rec + (int64_t)slot * rec_slot_doubles(); }
  double *rec_us(int slot) const { return rec_u1(slot) + 3 * nv; }

  void save_state(double *dst_u, double *dst_p) {
    CK(cudaMemcpyAsync(dst_u, u, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(dst_p, p, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  }
  void load_state(const double *src_u, const double *src_p) {
    CK(cudaMemcpyAsync(u, src_u, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(p, src_p, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, stream));
  }

  // Steps n0..n1-1 of the recording: before each step u on the P1 vertices, after it u*, into
  // the record slot n - n0. Eager stepping polls the status between steps.
  void enqueue_recorded_steps(int n0, int n1) {
    for (int n = n0; n < n1; ++n) {
      const int slot = n - n0;
      CK(cudaMemcpy2DAsync(rec_u1(slot), (size_t)nv * sizeof(double), u, (size_t)N2 * sizeof(double),
                           (size_t)nv * sizeof(double), 3, cudaMemcpyDeviceToDevice, stream));
      if (use_graph) {
        CK(cudaGraphLaunch(graph_exec, stream));
      } else {
        enqueue_step(false, false);
      }
      CK(cudaMemcpyAsync(rec_us(slot), ustar, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice,
                         stream));
      if (!use_graph) {
        CK(cudaMemcpyAsync(h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
        CK(cudaStreamSynchronize(stream));
        if (h_st->halt) break;
      }
    }
  }

  int adjoint_forward(int nsteps, int C, int *n_done) {
    NvtxRange nvtx_("cfsa adjoint forward");
    if (ncorr < 1) throw CudaError{"the adjoint needs at least one pressure corrector"};
    ensure_operators();
    ensure_adjoint_work();
    adj_valid = false;
    plan_records(nsteps, C);
    if (use_graph) ensure_graph();
    reset_status();
    CK(cudaEventRecord(ev0, stream));
    for (int seg = 0; seg < adj_nseg; ++seg) {
      const int n0 = seg * adj_C, n1 = std::min(nsteps, n0 + adj_C);
      double *ck = a_ck + (int64_t)seg * ck_slot_doubles();
      save_state(ck, ck + 3 * N2);
      enqueue_recorded_steps(n0, n1);
    }
    if (adj_nseg == 0) save_state(a_ck, a_ck + 3 * N2);
    CK(cudaEventRecord(ev1, stream));
    const int code = finish_batch(nsteps);
    if (n_done) *n_done = h_st->steps_done;
    // final snapshot: u, u*, p, p'
    CK(cudaMemcpyAsync(a_fin, u, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(a_fin + 3 * N2, ustar, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice,
                       stream));
    CK(cudaMemcpyAsync(a_fin + 6 * N2, p, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(a_fin + 6 * N2 + nv, pc, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice,
                       stream));
    CK(cudaStreamSynchronize(stream));
    adj_stats = cfsa_adjoint_stats{};
    adj_stats.steps = nsteps;
    adj_stats.checkpoint_every = adj_C;
    adj_stats.checkpoints = adj_nseg;
    adj_stats.forward_ms = last_ms;
    adj_stats.record_bytes =
        (int64_t)sizeof(double) * (a_rec_slots * rec_slot_doubles() + a_ck_slots * ck_slot_doubles() +
                                   6 * N2 + 2 * nv);
    if (code != CFSA_OK) return code;
    adj_steps = nsteps;
    adj_last_valid = true;  // the last segment's records are the ones just written
    adj_time_end = time;
    adj_steps_end = steps;
    adj_fp = adjoint_fingerprint();
    adj_valid = true;
    return CFSA_OK;
  }

  void restore_final_state() {
    CK(cudaMemcpyAsync(u, a_fin, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(ustar, a_fin + 3 * N2, (size_t)3 * N2 * sizeof(double), cudaMemcpyDeviceToDevice,
                       stream));
    CK(cudaMemcpyAsync(p, a_fin + 6 * N2, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    CK(cudaMemcpyAsync(pc, a_fin + 6 * N2 + nv, (size_t)nv * sizeof(double), cudaMemcpyDeviceToDevice,
                       stream));
  }

  // Objective on the current fields: J -> a_scal[1]; with seed, dJ/du -> a_lu, dJ/dp -> a_lp,
  // explicit dJ/dnu -> a_scal[0]. Returns false when the objective's vertex set is empty.
  bool enqueue_objective(const cfsa_objective &o, bool seed) {
    ensure_adjoint_work();
    const size_t n3 = (size_t)3 * N2;
    if (o.kind == CFSA_OBJECTIVE_WALL_SHEAR) {
      if (nbf <= 0) throw CudaError{"wall-shear objective needs boundary faces"};
      if (o.axis < 0 || o.axis > 2) throw CudaError{"objective axis must be 0, 1 or 2"};
      std::vector<signed char> mask((size_t)nv, 0);
      int64_t np = 0;
      for (int64_t v = 0; v < nv; ++v) {
        const double x = h_xyz[3 * v + o.axis];
        if (h_bc[v] == BC_WALL && x >= o.lo && x <= o.hi) {
          mask[v] = 1;
          ++np;
        }
      }
      if (np == 0) return false;
      CK(cudaMemcpyAsync(a_mask, mask.data(), (size_t)nv, cudaMemcpyHostToDevice, stream));
      k_face_forces<<<blocks_for(nbf), kBlock, 0, stream>>>((int)nbf, (int)nt, N2, viscosity, fverts, ftet,
                                                           fnormal, farea, tnode, grad, u, p, fshear, fpress);
      k_face_gather<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, vf_ptr, vf, fshear, fout);
      k_obj_wss_value<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, fout, a_mask, 1.0 / (double)np,
                                                             viscosity, a_w, a_scal + 1, a_scal, red);
      if (seed) {
        k_obj_wss_face<<<blocks_for(nbf), kBlock, 0, stream>>>((int)nbf, fverts, farea, a_w, a_W);
        k_obj_wss_seed<<<blocks_for(N2), kBlock, 0, stream>>>((int)nv, N2, (int)nt, vbf_ptr, vbf, ftet,
                                                              fnormal, grad, a_W, viscosity, a_lu);
        CK(cudaMemsetAsync(a_lp, 0, (size_t)nv * sizeof(double), stream));
      }
      CK(cudaGetLastError());
      // the mask upload reads host memory that goes out of scope
      CK(cudaStreamSynchronize(stream));
      return true;
    }
    if (o.kind == CFSA_OBJECTIVE_PRESSURE_DROP) {
      int64_t nin = 0, nout = 0;
      for (int64_t v = 0; v < nv; ++v) {
        nin += h_bc[v] == BC_INLET;
        nout += h_bc[v] == BC_OUTLET;
      }
      if (nin == 0 || nout == 0) return false;
      k_obj_pdrop<<<blocks_for(nv), kBlock, 0, stream>>>((int)nv, p, bc, 1.0 / (double)nin,
                                                         1.0 / (double)nout, a_lp, a_scal + 1, red);
      if (seed) {
        CK(cudaMemsetAsync(a_lu, 0, n3 * sizeof(double), stream));
        CK(cudaMemsetAsync(a_scal, 0, sizeof(double), stream));
      }
      CK(cudaGetLastError());
      return true;
    }
    throw CudaError{"unknown objective kind"};
  }

  // One reverse step on (a_lu, a_lp) with the step's records in a_un (u^n on P1) and a_us (u*).
  void enqueue_adj_step(bool capture) {
    const unsigned int gN2 = blocks_for(N2), gnv = blocks_for(nv);
    AdjCorrectArgs c{};
    c.lu = a_lu;
    c.bc = bc;
    c.invm = invm;
    c.dt = dt;
    c.relax_u = relax_u;
    c.n = (int)N2;
    c.nv = (int)nv;
    c.lus = wb;
    c.gin = a_gin;
    c.q = a_q;
    c.st = st_adj;
    k_adj_correct<<<gN2, kBlock, 0, stream>>>(c);
    const bool normalize = (ref_node >= 0 && ref_node < nv);
    for (int k = ncorr - 1; k >= 0; --k) {
      if (normalize) k_adj_sum<<<gnv, kBlock, 0, stream>>>((int)nv, a_lp, a_scal + 2, red, st_adj);
      AdjChainArgs ch{};
      ch.chain = a_lp;
      ch.lpp = a_lpp;
      ch.S = normalize ? a_scal + 2 : nullptr;
      ch.bc = bc;
      ch.relax_p = relax_p;
      ch.nv = (int)nv;
      ch.ref_node = ref_node;
      ch.dirichlet = (outlet_type == CFSA_OUTLET_DIRICHLET) ? 1 : 0;
      ch.first = (k == ncorr - 1) ? 1 : 0;
      ch.st = st_adj;
      k_adj_pchain<<<gnv, kBlock, 0, stream>>>(ch);
    }
    PressureRhsArgs pa = pressure_rhs_args(a_px, st_adj);
    pa.adj_q = a_q;
    pa.adj_lpp = a_lpp;
    pa.G = CsrView{rp1, ci1};
    pa.tpos = tpos1;
    pa.Gv = Gv;
    pa.nnz1 = nnz1;
    k_pressure_rhs<<<gnv, kBlock, 0, stream>>>(pa);
    CK(cudaGetLastError());
    enqueue_pressure_krylov(capture, a_px, st_adj);
    MomentumRhsArgs m{};
    m.S = s2.view();
    m.G = CsrView{rp1, ci1};
    m.Gv = Gv;
    m.nnz1 = nnz1;
    m.bc = bc;
    m.dt = dt;
    m.tol = tol_mom;
    m.n = (int)N2;
    m.nv = (int)nv;
    m.nt = (int)nt;
    m.maxit = maxit_mom;
    m.b = wb;
    m.x = a_x;
    m.r = wr;
    m.r0 = wr0;
    m.pk = wp;
    m.v = wv;
    m.bs = bs_mom;
    m.st = st_adj;
    m.red = red;
    m.cw = (conv_norm == CFSA_NORM_JACOBI) ? invA : nullptr;
    m.adj_mu = a_px;
    m.tpos = tpos1;
    k_momentum_rhs<<<strided(k_momentum_rhs, blocks_for(s2.nrows_pad)), kBlock, 0, stream>>>(m);
    CK(cudaGetLastError());
    enqueue_momentum_krylov(capture, a_x, st_adj);
    k_adj_conv_tet<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, N2, nv, tnode, grad, vol, a_x, a_un,
                                                          a_tsc, st_adj);
    AdjMomOutArgs o{};
    o.S = s2.view();
    o.Ms = Ms;
    o.K = CsrView{rp2, ci2};
    o.Kv = Kv;
    o.G = CsrView{rp1, ci1};
    o.tpos = tpos1;
    o.Gv = Gv;
    o.nnz1 = nnz1;
    o.adj_ptr = adj_ptr;
    o.adj = adj;
    o.grad = grad;
    o.tsc = a_tsc;
    o.bc = bc;
    o.nu = a_x;
    o.us = a_us;
    o.dt = dt;
    o.viscosity = viscosity;
    o.n = (int)N2;
    o.nv = (int)nv;
    o.nt = (int)nt;
    o.lu = a_lu;
    o.lp = a_lp;
    o.gin = a_gin;
    o.gnu = a_scal;
    o.red = red;
    o.st = st_adj;
    k_adj_mom_out<<<blocks_for(s2.nrows_pad), kBlock, 0, stream>>>(o);
    CK(cudaGetLastError());
    // correct, [sum,] chain per corrector, pressure rhs + check, momentum rhs + check,
    // conv_tet, mom_out (Krylov loop bodies counted from the status)
    adj_launches_fixed = 1 + ncorr * (normalize ? 2 : 1) + 2 + 2 + 2 + mixed_fixed_kernels();
  }

  void ensure_adj_graph() {
    if (adj_exec) {
      CK(cudaGraphExecDestroy(adj_exec));
      adj_exec = nullptr;
    }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
    try {
      enqueue_adj_step(true);
    } catch (...) {
      cudaGraph_t gg = nullptr;
      cudaStreamEndCapture(stream, &gg);
      if (gg) cudaGraphDestroy(gg);
      throw;
    }
    CK(cudaStreamEndCapture(stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&adj_exec, g, 0);
    cudaGraphDestroy(g);
    CK(e);
  }

  // Backward pass. The seed is already in a_lu / a_lp / a_scal[0].
  int adjoint_backward_core(double *grad_inlet, double *grad_viscosity, double *grad_u0, double *grad_p0) {
    NvtxRange nvtx_("cfsa adjoint backward");
    const size_t n3 = (size_t)3 * N2;
    CK(cudaMemsetAsync(a_gin, 0, n3 * sizeof(double), stream));
    CK(cudaMemsetAsync(st_adj, 0, sizeof(DevStatus), stream));
    reset_status();
    if (use_graph) {
      ensure_graph();
      ensure_adj_graph();
    }
    const double time_save = time;
    const int64_t steps_save = steps;
    int64_t recomputed = 0;
    CK(cudaEventRecord(ev0, stream));
    for (int seg = adj_nseg - 1; seg >= 0; --seg) {
      const int n0 = seg * adj_C, n1 = std::min(adj_steps, n0 + adj_C);
      if (!(seg == adj_nseg - 1 && adj_last_valid)) {
        const double *ck = a_ck + (int64_t)seg * ck_slot_doubles();
        load_state(ck, ck + 3 * N2);
        enqueue_recorded_steps(n0, n1);
        recomputed += n1 - n0;
      }
      for (int n = n1 - 1; n >= n0; --n) {
        const int slot = n - n0;
        CK(cudaMemcpyAsync(a_un, rec_u1(slot), (size_t)3 * nv * sizeof(double), cudaMemcpyDeviceToDevice,
                           stream));
        CK(cudaMemcpyAsync(a_us, rec_us(slot), n3 * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        if (use_graph) {
          CK(cudaGraphLaunch(adj_exec, stream));
        } else {
          enqueue_adj_step(false);
        }
      }
    }
    CK(cudaEventRecord(ev1, stream));
    restore_final_state();
    // the last segment's records now hold its own steps again only if it was not recomputed
    adj_last_valid = (adj_nseg <= 1);
    DevStatus hs_adj{};
    CK(cudaMemcpyAsync(h_st, st, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    CK(cudaMemcpyAsync(&hs_adj, st_adj, sizeof(DevStatus), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    time = time_save;
    steps = steps_save;
    adj_stats.recomputed_steps = recomputed;
    adj_stats.momentum_iters = (int64_t)hs_adj.iters[0];
    adj_stats.pressure_iters = (int64_t)hs_adj.iters[1];
    adj_stats.backward_ms = ms;
    const int pressure_body = pressure_body_kernels();
    adj_stats.kernel_launches = (int64_t)adj_steps * adj_launches_fixed +
                                momentum_body_kernels() * (int64_t)hs_adj.body_runs[0] +
                                pressure_body * (int64_t)hs_adj.body_runs[1] +
                                2 * (int64_t)hs_adj.body_runs[2];
    if (h_st->code != CFSA_OK) {
      err = "forward recomputation failed with status " + std::to_string(h_st->code);
      return h_st->code;
    }
    if (hs_adj.code != CFSA_OK) {
      err = "adjoint solve failed with status " + std::to_string(hs_adj.code);
      return hs_adj.code;
    }
    std::vector<double> tmp(n3);
    if (grad_inlet) download_vec3(a_gin, grad_inlet);
    if (grad_u0) download_vec3(a_lu, grad_u0);
    if (grad_p0) CK(cudaMemcpy(grad_p0, a_lp, (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost));
    if (grad_viscosity) CK(cudaMemcpy(grad_viscosity, a_scal, sizeof(double), cudaMemcpyDeviceToHost));
    return CFSA_OK;
  }

  int check_adjoint_ready() {
    if (!adj_valid) {
      err = "no recorded forward pass (cfsa_ns_adjoint_forward) for the backward pass";
      return CFSA_NOT_INITIALIZED;
    }
    if (mom_dirty || poisson_dirty || adjoint_fingerprint() != adj_fp) {
      adj_valid = false;
      err = "parameters, inlet values, tags or geometry changed since the recorded forward pass";
      return CFSA_BAD_ARG;
    }
    return CFSA_OK;
  }

  // Kernel timing on the live data with private Krylov states (solver state untouched).
  void profile_kernel(int which, int iters, double *avg_ms, double *alg_bytes) {
    NvtxRange nvtx_("cfsa profile kernel");  // lets a profiler select these launches
    ensure_operators();
    CK(cudaStreamSynchronize(stream));
    if (which == CFSA_KERNEL_MOMENTUM_SPMV_F32) {
      MixedState hm{};
      hm.active = 7;
      CK(cudaMemcpyAsync(ms_prof, &hm, sizeof(hm), cudaMemcpyHostToDevice, stream));
      MixedArgs a = mixed_args(ustar, nullptr);
      a.ms = ms_prof;
      // input: the velocity rounded to float (nonzero wherever the flow is, so neither method's
      // dot product vanishes; a zero p.q would end the CG product early); fs and ft are FP32 Krylov
      // scratch that every mixed solve rewrites before reading
      k_to_f32<<<blocks_for(3 * N2), kBlock, 0, stream>>>(3 * N2, u, fs);
      a.p = fs;
      a.r0 = fs;
      a.v = ft;   // scratch output
      auto *kern = (mom_krylov == CFSA_KRYLOV_CG) ? k_mpc_q : k_mp_v;  // the method's FP32 product
      kern<<<s2.nruns, kRunThreads, 0, stream>>>(a);  // warm-up
      CK(cudaEventRecord(ev0, stream));
      for (int k = 0; k < iters; ++k) kern<<<s2.nruns, kRunThreads, 0, stream>>>(a);
      CK(cudaEventRecord(ev1, stream));
      *alg_bytes = 8.0 * (double)nnz2 + 8.0 * s2.nrows_pad + 4.0 * (s2.nslices + 1) + 36.0 * (double)N2;
    } else if (which == CFSA_KERNEL_MOMENTUM_SPMV) {
      BicgState hs{};
      hs.active = 7;
      hs.ncomp = 3;
      for (int c = 0; c < 3; ++c) hs.rho[c] = 1.0;
      CK(cudaMemcpyAsync(bs_prof, &hs, sizeof(hs), cudaMemcpyHostToDevice, stream));
      BicgArgs a = momentum_args();
      a.bs = bs_prof;
      a.st = nullptr;
      a.v = ws;  // scratch output
      // the product kernel of the selected momentum method (BiCGSTAB: v = At p with r0.v; CG:
      // q = A p with p.q); same matrix stream, gathers and algorithmic bytes
      auto *kern = (mom_krylov == CFSA_KRYLOV_CG) ? k_mcg_q<3> : k_bicg_v<3>;
      kern<<<s2.nruns, kRunThreads, 0, stream>>>(a);  // warm-up
      CK(cudaEventRecord(ev0, stream));
      for (int k = 0; k < iters; ++k) kern<<<s2.nruns, kRunThreads, 0, stream>>>(a);
      CK(cudaEventRecord(ev1, stream));
      *alg_bytes = 12.0 * (double)nnz2 + 8.0 * s2.nrows_pad + 4.0 * (s2.nslices + 1) + 72.0 * (double)N2;
    } else if (which == CFSA_KERNEL_PRESSURE_SPMV) {
      CgState hc{};
      hc.active = 1;
      hc.absnew = 1.0;
      CK(cudaMemcpyAsync(cs_prof, &hc, sizeof(hc), cudaMemcpyHostToDevice, stream));
      CgArgs c{};
      c.S = s1.view();
      c.Ls = Ls;
      c.invL = invL;
      c.x = pc;
      c.r = pr;
      c.z = pz;
      c.pk = pp;
      c.q = ps;  // scratch output
      c.n = (int)nv;
      c.cs = cs_prof;
      c.red = red;
      c.st = nullptr;
      const unsigned int g = blocks_for(s1.nrows_pad);
      k_cg_q<<<g, kBlock, 0, stream>>>(c);
      CK(cudaEventRecord(ev0, stream));
      for (int k = 0; k < iters; ++k) k_cg_q<<<g, kBlock, 0, stream>>>(c);
      CK(cudaEventRecord(ev1, stream));
      *alg_bytes = 12.0 * (double)nnz1 + 8.0 * s1.nrows_pad + 4.0 * (s1.nslices + 1) + 16.0 * (double)nv;
    } else if (which == CFSA_KERNEL_PRESSURE_SOLVE) {
      // the whole resident pressure solve on the divergence of the current u* (the system of the
      // last step), into scratch: the solver's fields and status are not touched
      if (krylov != CFSA_KRYLOV_CG2L && krylov != CFSA_KRYLOV_CG1)
        throw CudaError{"pressure-solve profile needs the resident CG solvers (CG1 or CG2L)"};
      CK(cudaMemsetAsync(st_free, 0, sizeof(DevStatus), stream));
      float total = 0.f;
      int64_t its = 0;
      for (int k = 0; k < iters; ++k) {
        k_tet_div<<<blocks_for(nt), kBlock, 0, stream>>>((int)nt, N2, tnode, grad, ustar, divt, st_free);
        const PressureRhsArgs a = pressure_rhs_args(pv, st_free);
        k_pressure_rhs<<<blocks_for(nv), kBlock, 0, stream>>>(a);
        CK(cudaEventRecord(ev0, stream));
        enqueue_pressure_krylov(false, pv, st_free);
        CK(cudaEventRecord(ev1, stream));
        CK(cudaMemcpyAsync(h_cs, cs, sizeof(CgState), cudaMemcpyDeviceToHost, stream));
        CK(cudaEventSynchronize(ev1));
        CK(cudaStreamSynchronize(stream));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, ev0, ev1));
        total += ms;
        its += h_cs->iters;
      }
      *avg_ms = (double)total / (double)iters;
      // per iteration: operator values and columns, row metadata, the vectors each read or
      // written once (r, w, s, p, x, D^-1 read; r, w, s, p, x written; aggregate ids and staging
      // positions) and, with the coarse space, the dense coarse inverse once
      const double per_it = 12.0 * (double)nnz1 + 8.0 * s1.nrows_pad + 4.0 * (s1.nslices + 1) +
                            96.0 * (double)nv +
                            (krylov == CFSA_KRYLOV_CG2L ? 8.0 * (double)coarse_nc * coarse_nc : 0.0);
      *alg_bytes = per_it * (double)its / (double)iters;
      return;
    } else {
      throw CudaError{"unknown kernel id"};
    }
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(ev1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    *avg_ms = (double)ms / (double)std::max(1, iters);
  }
};

namespace {

int fail(cfsa_ns *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  return code;
}

// Runs one C-ABI operation. The thread's CUDA last-error state is cleared first, so that the
// launch checks inside report this operation's own failures only.
template <class F>
int guarded(cfsa_ns *h, F &&f) {
  (void)cudaGetLastError();
  try {
    return f();
  } catch (const CudaError &e) {
    return fail(h, CFSA_CUDA_ERROR, e.msg);
  } catch (const std::bad_alloc &) {
    return fail(h, CFSA_CUDA_ERROR, "host allocation failed");
  } catch (const std::exception &e) {
    return fail(h, CFSA_BAD_ARG, e.what());
  }
}

std::string g_create_error;

}  // namespace

extern "C" {

int cfsa_ns_create(const cfsa_mesh_view *mesh, const cfsa_fluid *fluid, cfsa_ns **out) {
  if (!mesh || !fluid || !out || mesh->nv <= 0 || mesh->nt <= 0 || mesh->ne < 0 || !mesh->vertices ||
      !mesh->tets || !mesh->tet_edges) {
    g_create_error = "cfsa_ns_create: bad arguments";
    return CFSA_BAD_ARG;
  }
  if (!(fluid->viscosity > 0.0) || !(fluid->density > 0.0)) {
    g_create_error = "cfsa_ns_create: density and viscosity must be positive";
    return CFSA_BAD_ARG;
  }
  cfsa_ns *h = new (std::nothrow) cfsa_ns();
  if (!h) return CFSA_CUDA_ERROR;
  int code = guarded(h, [&] {
    h->setup(mesh, fluid);
    return CFSA_OK;
  });
  if (code != CFSA_OK) {
    g_create_error = h->err;
    delete h;
    *out = nullptr;
    return code;
  }
  *out = h;
  return CFSA_OK;
}

void cfsa_ns_destroy(cfsa_ns *h) { delete h; }

const char *cfsa_ns_last_error(const cfsa_ns *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int cfsa_ns_sizes(const cfsa_ns *h, int64_t out[4]) {
  if (!h || !out) return CFSA_BAD_ARG;
  out[0] = h->nv;
  out[1] = h->ne;
  out[2] = h->N2;
  out[3] = h->nt;
  return CFSA_OK;
}

int cfsa_ns_set_dt(cfsa_ns *h, double dt) {
  if (!h) return CFSA_BAD_ARG;
  if (!(dt > 0.0)) return fail(h, CFSA_BAD_ARG, "dt must be positive");
  if (dt != h->dt) h->mom_dirty = h->graph_dirty = true;
  h->dt = dt;
  return CFSA_OK;
}

int cfsa_ns_set_tolerances(cfsa_ns *h, double momentum, double pressure) {
  if (!h) return CFSA_BAD_ARG;
  if (!(momentum > 0.0) || !(pressure > 0.0)) return fail(h, CFSA_BAD_ARG, "tolerances must be positive");
  h->tol_mom = momentum;
  h->tol_p = pressure;
  h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_max_iterations(cfsa_ns *h, int momentum, int pressure) {
  if (!h) return CFSA_BAD_ARG;
  if (momentum < 1 || pressure < 1) return fail(h, CFSA_BAD_ARG, "iteration caps must be >= 1");
  h->maxit_mom = momentum;
  h->maxit_p = pressure;
  h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_num_corrections(cfsa_ns *h, int n) {
  if (!h) return CFSA_BAD_ARG;
  if (n < 0) return fail(h, CFSA_BAD_ARG, "number of corrections must be >= 0");
  h->ncorr = n;
  h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_relaxation(cfsa_ns *h, double relax_u, double relax_p) {
  if (!h) return CFSA_BAD_ARG;
  h->relax_u = relax_u;
  h->relax_p = relax_p;
  h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_outlet(cfsa_ns *h, int outlet_type, double outlet_pressure) {
  if (!h) return CFSA_BAD_ARG;
  if (outlet_type < 0 || outlet_type > 2) return fail(h, CFSA_BAD_ARG, "bad outlet type");
  h->outlet_type = outlet_type;
  h->outlet_pressure = outlet_pressure;
  h->poisson_dirty = h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_reference_node(cfsa_ns *h, int node) {
  if (!h) return CFSA_BAD_ARG;
  h->ref_node = node;
  h->poisson_dirty = h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_inlet_uniform(cfsa_ns *h, const double u[3]) {
  if (!h || !u) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    for (int c = 0; c < 3; ++c)
      std::fill(h->h_inlet.begin() + (size_t)c * h->N2, h->h_inlet.begin() + (size_t)(c + 1) * h->N2, u[c]);
    h->h_inlet_stale = false;
    CK(cudaMemcpyAsync(h->inlet, h->h_inlet.data(), h->h_inlet.size() * sizeof(double),
                       cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_set_inlet_profile(cfsa_ns *h, const double *u) {
  if (!h || !u) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->upload_vec3(u, h->inlet);
    h->h_inlet_stale = true;
    return CFSA_OK;
  });
}

int cfsa_ns_set_pressure_solver(cfsa_ns *h, int krylov) {
  if (!h) return CFSA_BAD_ARG;
  if (krylov != CFSA_KRYLOV_CG && krylov != CFSA_KRYLOV_BICGSTAB && krylov != CFSA_KRYLOV_CG1 &&
      krylov != CFSA_KRYLOV_CG2L)
    return fail(h, CFSA_BAD_ARG, "unknown Krylov method");
  if ((krylov == CFSA_KRYLOV_CG1 || krylov == CFSA_KRYLOV_CG2L) && !h->cg_resident)
    return fail(h, CFSA_UNSUPPORTED, "single-reduction CG needs the shared-memory-resident grid on this device");
  h->krylov = krylov;
  h->graph_dirty = true;
  return CFSA_OK;
}

int cfsa_ns_set_momentum_solver(cfsa_ns *h, int krylov) {
  if (!h) return CFSA_BAD_ARG;
  if (krylov != CFSA_KRYLOV_CG && krylov != CFSA_KRYLOV_BICGSTAB)
    return fail(h, CFSA_BAD_ARG, "momentum Krylov method must be CFSA_KRYLOV_BICGSTAB or CFSA_KRYLOV_CG");
  if (krylov != h->mom_krylov) {
    h->mom_dirty = true;  // the SELL values change between A D^-1 and A
    h->graph_dirty = true;
  }
  h->mom_krylov = krylov;
  return CFSA_OK;
}

int cfsa_ns_set_coarse_target(cfsa_ns *h, int target) {
  if (!h) return CFSA_BAD_ARG;
  if (target < 1 || target > 1024) return fail(h, CFSA_BAD_ARG, "coarse target outside [1, 1024]");
  if (target != h->coarse_target) h->coarse_dirty = h->graph_dirty = true;
  h->coarse_target = target;
  return CFSA_OK;
}

int cfsa_ns_get_coarse_size(cfsa_ns *h, int *nc) {
  if (!h || !nc) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    if (h->krylov == CFSA_KRYLOV_CG2L) h->ensure_operators();
    *nc = (h->krylov == CFSA_KRYLOV_CG2L) ? h->coarse_nc : 0;
    return CFSA_OK;
  });
}

int cfsa_ns_set_precision(cfsa_ns *h, int precision) {
  if (!h) return CFSA_BAD_ARG;
  if (precision != CFSA_PRECISION_FP64 && precision != CFSA_PRECISION_MIXED &&
      precision != CFSA_PRECISION_MIXED_FULL)
    return fail(h, CFSA_BAD_ARG, "unknown precision");
  if (precision != h->precision) h->graph_dirty = true;
  h->precision = precision;
  return CFSA_OK;
}

int cfsa_ns_set_convergence_norm(cfsa_ns *h, int norm) {
  if (!h) return CFSA_BAD_ARG;
  if (norm != CFSA_NORM_REFERENCE && norm != CFSA_NORM_JACOBI)
    return fail(h, CFSA_BAD_ARG, "unknown convergence norm");
  if (norm != h->conv_norm) h->graph_dirty = true;
  h->conv_norm = norm;
  return CFSA_OK;
}

int cfsa_ns_set_viscosity(cfsa_ns *h, double viscosity) {
  if (!h) return CFSA_BAD_ARG;
  if (!(viscosity > 0.0)) return fail(h, CFSA_BAD_ARG, "viscosity must be positive");
  return guarded(h, [&] {
    h->viscosity = viscosity;
    h->assemble();
    h->graph_dirty = true;
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_initialize_fields(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    const size_t n3 = (size_t)3 * h->N2;
    std::vector<double> u0(n3, 0.0);
    const std::vector<double> &hin = h->host_inlet();
    for (int64_t i = 0; i < h->N2; ++i)
      if (h->h_bc[i] == BC_INLET)
        for (int c = 0; c < 3; ++c) u0[(size_t)c * h->N2 + i] = hin[(size_t)c * h->N2 + i];
    CK(cudaMemcpyAsync(h->u, u0.data(), n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->ustar, 0, n3 * sizeof(double), h->stream));
    CK(cudaMemsetAsync(h->p, 0, h->nv * sizeof(double), h->stream));
    CK(cudaMemsetAsync(h->pc, 0, h->nv * sizeof(double), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->time = 0.0;
    return CFSA_OK;
  });
}

int cfsa_ns_assemble(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->assemble();
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_update_vertices(cfsa_ns *h, const double *xyz) {
  if (!h || !xyz) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    CK(cudaMemcpyAsync(h->xyz, xyz, (size_t)3 * h->nv * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    h->h_xyz.assign(xyz, xyz + 3 * h->nv);
    h->assemble();
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_update_boundary_tags(cfsa_ns *h, const int8_t *p1_bc, const int8_t *p2_bc) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    if (p1_bc)
      for (int64_t i = 0; i < h->nv; ++i) h->h_bc[i] = p1_bc[i];
    if (p2_bc)
      for (int64_t k = 0; k < h->ne; ++k) h->h_bc[h->nv + k] = p2_bc[k];
    CK(cudaMemcpyAsync(h->bc, h->h_bc.data(), h->h_bc.size(), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->mom_dirty = h->poisson_dirty = h->graph_dirty = true;
    return CFSA_OK;
  });
}

// Message of a failed stepping call (status from the device status word).
static std::string step_failure(int code) {
  std::string m = "step failed with status " + std::to_string(code);
  if (code == CFSA_CUDA_ERROR) m += ": the pressure solve gave up waiting at a grid barrier";
  return m;
}

int cfsa_ns_piso_steps(cfsa_ns *h, int n, int *n_done) {
  if (!h) return CFSA_BAD_ARG;
  if (n < 0) return fail(h, CFSA_BAD_ARG, "negative step count");
  return guarded(h, [&] {
    const int code = h->run_steps(n, n_done, false);
    if (code != CFSA_OK) h->err = step_failure(code);
    return code;
  });
}

int cfsa_ns_piso_step(cfsa_ns *h) { return cfsa_ns_piso_steps(h, 1, nullptr); }

int cfsa_ns_simple_step(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    const int code = h->run_steps(1, nullptr, true);
    if (code != CFSA_OK) h->err = step_failure(code);
    return code;
  });
}

int cfsa_ns_momentum_predictor(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->ensure_operators();
    h->reset_status();
    h->enqueue_momentum(false);
    CK(cudaMemcpyAsync(h->h_st, h->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return h->h_st->code;
  });
}

int cfsa_ns_pressure_poisson(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->ensure_operators();
    h->reset_status();
    h->enqueue_pressure_solve(false);
    h->enqueue_pressure_update();
    CK(cudaMemcpyAsync(h->h_st, h->st, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return h->h_st->code;
  });
}

int cfsa_ns_solve_pressure_bicgstab(cfsa_ns *h, const double *rhs, double *x, double tol, int maxit) {
  if (!h || !rhs || !x) return CFSA_BAD_ARG;
  if (!(tol >= 0.0) || maxit < 1) return fail(h, CFSA_BAD_ARG, "solvePressureBiCGSTAB: tol >= 0 and maxit >= 1 required");
  return guarded(h, [&] {
    const int code = h->solve_poisson_raw(rhs, x, tol, maxit);
    if (code == CFSA_NOT_CONVERGED) h->err = "BiCGSTAB failed: no convergence within the iteration cap";
    if (code == CFSA_BREAKDOWN) h->err = "BiCGSTAB failed: breakdown";
    return code;
  });
}

int cfsa_ns_correct_velocity(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->reset_status();
    h->enqueue_correct();
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_get_velocity(cfsa_ns *h, double *u) {
  if (!h || !u) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->download_vec3(h->u, u);
    return CFSA_OK;
  });
}

int cfsa_ns_get_velocity_async(cfsa_ns *h, double *u) {
  if (!h || !u) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->readback_async(true, u);
    return CFSA_OK;
  });
}

int cfsa_ns_get_pressure_async(cfsa_ns *h, double *p) {
  if (!h || !p) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->readback_async(false, p);
    return CFSA_OK;
  });
}

int cfsa_ns_wait_outputs(cfsa_ns *h) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    if (h->copy_stream) CK(cudaStreamSynchronize(h->copy_stream));
    return CFSA_OK;
  });
}

int cfsa_ns_get_velocity_star(cfsa_ns *h, double *u) {
  if (!h || !u) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->download_vec3(h->ustar, u);
    return CFSA_OK;
  });
}

int cfsa_ns_get_pressure(cfsa_ns *h, double *p) {
  if (!h || !p) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    CK(cudaMemcpyAsync(p, h->p, h->nv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_get_pressure_correction(cfsa_ns *h, double *p) {
  if (!h || !p) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    CK(cudaMemcpyAsync(p, h->pc, h->nv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_set_fields(cfsa_ns *h, const double *u, const double *p) {
  if (!h) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    if (u) h->upload_vec3(u, h->u);
    if (p) {
      CK(cudaMemcpyAsync(h->p, p, h->nv * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
    return CFSA_OK;
  });
}

namespace {
constexpr char kStateTag[8] = {'C', 'F', 'S', 'A', 'S', 'T', '0', '1'};
}

int cfsa_ns_save_state(cfsa_ns *h, const char *path) {
  if (!h || !path) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    std::vector<double> u((size_t)3 * h->N2), p((size_t)h->nv);
    h->download_vec3(h->u, u.data());
    CK(cudaMemcpyAsync(p.data(), h->p, p.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(h, CFSA_BAD_ARG, std::string("cannot open ") + path + " for writing");
    const int64_t sizes[2] = {h->N2, h->nv};
    const int64_t steps = h->steps;
    bool ok = std::fwrite(kStateTag, 1, 8, f) == 8 && std::fwrite(sizes, sizeof(int64_t), 2, f) == 2 &&
              std::fwrite(&h->time, sizeof(double), 1, f) == 1 && std::fwrite(&steps, sizeof(int64_t), 1, f) == 1 &&
              std::fwrite(u.data(), sizeof(double), u.size(), f) == u.size() &&
              std::fwrite(p.data(), sizeof(double), p.size(), f) == p.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? CFSA_OK : fail(h, CFSA_BAD_ARG, std::string("write error on ") + path);
  });
}

int cfsa_ns_load_state(cfsa_ns *h, const char *path) {
  if (!h || !path) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(h, CFSA_BAD_ARG, std::string("cannot open ") + path);
    char tag[8];
    int64_t sizes[2] = {0, 0}, steps = 0;
    double t = 0.0;
    bool ok = std::fread(tag, 1, 8, f) == 8 && std::memcmp(tag, kStateTag, 8) == 0 &&
              std::fread(sizes, sizeof(int64_t), 2, f) == 2 && std::fread(&t, sizeof(double), 1, f) == 1 &&
              std::fread(&steps, sizeof(int64_t), 1, f) == 1;
    if (!ok || sizes[0] != h->N2 || sizes[1] != h->nv) {
      std::fclose(f);
      return fail(h, CFSA_BAD_ARG, std::string(path) + ": not a state file of this mesh (N2/nv differ or bad header)");
    }
    std::vector<double> u((size_t)3 * h->N2), p((size_t)h->nv);
    ok = std::fread(u.data(), sizeof(double), u.size(), f) == u.size() &&
         std::fread(p.data(), sizeof(double), p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) return fail(h, CFSA_BAD_ARG, std::string(path) + ": truncated state file");
    h->upload_vec3(u.data(), h->u);
    CK(cudaMemcpyAsync(h->p, p.data(), p.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->time = t;
    h->steps = steps;
    return CFSA_OK;
  });
}

int cfsa_ns_get_time(const cfsa_ns *h, double *t) {
  if (!h || !t) return CFSA_BAD_ARG;
  *t = h->time;
  return CFSA_OK;
}

int cfsa_ns_get_stats(const cfsa_ns *hc, cfsa_ns_stats *s) {
  if (!hc || !s) return CFSA_BAD_ARG;
  cfsa_ns *h = const_cast<cfsa_ns *>(hc);
  return guarded(h, [&] {
    CK(cudaMemcpyAsync(h->h_bs, h->bs_mom, sizeof(BicgState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_bs + 1, h->bs_p, sizeof(BicgState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->h_cs, h->cs, sizeof(CgState), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    std::memset(s, 0, sizeof(*s));
    if (h->momentum_mixed()) {
      CK(cudaMemcpyAsync(h->h_ms, h->ms, sizeof(MixedState), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
      for (int c = 0; c < 3; ++c) {
        s->momentum_iters[c] = h->h_ms->iters[c];
        s->momentum_outer[c] = h->h_ms->updates[c];
        const double b2 = h->h_ms->bnorm2[c];
        s->momentum_residual[c] = b2 > 0 ? std::sqrt(h->h_ms->rnorm2[c] / b2) : 0.0;
      }
    } else {
      for (int c = 0; c < 3; ++c) {
        s->momentum_iters[c] = h->h_bs[0].iters[c];
        const double b2 = h->h_bs[0].bnorm2[c];
        s->momentum_residual[c] = b2 > 0 ? std::sqrt(h->h_bs[0].rnorm2[c] / b2) : 0.0;
      }
    }
    if (h->krylov == CFSA_KRYLOV_BICGSTAB) {
      s->pressure_iters = h->h_bs[1].iters[0];
      const double b2 = h->h_bs[1].bnorm2[0];
      s->pressure_residual = b2 > 0 ? std::sqrt(h->h_bs[1].rnorm2[0] / b2) : 0.0;
    } else {
      s->pressure_iters = h->h_cs->iters;
      const double b2 = h->h_cs->bnorm2;
      s->pressure_residual = b2 > 0 ? std::sqrt(h->h_cs->rnorm2 / b2) : 0.0;
      if (h->pressure_mixed()) {
        CK(cudaMemcpyAsync(h->h_pmx, h->pmx, sizeof(PMixState), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        s->pressure_outer = h->h_pmx->sweeps;
      }
    }
    s->steps = h->steps;
    s->time = h->time;
    s->last_step_ms = h->last_ms;
    s->nnz_p2 = h->nnz2;
    s->nnz_p1 = h->nnz1;
    s->kernel_launches = h->batch_launches;
    if (h->steps > 0) {
      float a = 0.f, b = 0.f, c = 0.f;
      if (cudaEventElapsedTime(&a, h->ph[0], h->ph[1]) == cudaSuccess &&
          cudaEventElapsedTime(&b, h->ph[1], h->ph[2]) == cudaSuccess &&
          cudaEventElapsedTime(&c, h->ph[2], h->ph[3]) == cudaSuccess) {
        s->phase_ms[0] = a;
        s->phase_ms[1] = b;
        s->phase_ms[2] = c;
      } else {
        (void)cudaGetLastError();  // phases not recorded (no full step yet): leave zeros
      }
    }
    s->krylov_iters[0] = h->batch_iters[0];
    s->krylov_iters[1] = h->batch_iters[1];
    return CFSA_OK;
  });
}

int cfsa_ns_compute_divergence(cfsa_ns *h, const double *u, double *div) {
  if (!h || !u || !div) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->upload_vec3(u, h->wb);
    k_tet_div<<<blocks_for(h->nt), kBlock, 0, h->stream>>>((int)h->nt, h->N2, h->tnode, h->grad, h->wb,
                                                           h->divt, h->st_free);
    k_gather_div<<<blocks_for(h->nv), kBlock, 0, h->stream>>>((int)h->nv, h->adj_ptr, h->adj, h->vol,
                                                              h->divt, h->pb);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(div, h->pb, h->nv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_compute_advection(cfsa_ns *h, double *conv) {
  if (!h || !conv) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    k_tet_conv<<<blocks_for(h->nt), kBlock, 0, h->stream>>>((int)h->nt, h->N2, h->tnode, h->grad, h->u,
                                                            h->ct, h->st_free);
    k_gather_conv<<<blocks_for(h->N2), kBlock, 0, h->stream>>>((int)h->N2, (int)h->nt, h->adj_ptr, h->adj,
                                                               h->vol, h->ct, h->wb);
    CK(cudaGetLastError());
    h->download_vec3(h->wb, conv);
    return CFSA_OK;
  });
}

static int face_forces(cfsa_ns *h, double *out, int which) {
  if (!h || !out) return CFSA_BAD_ARG;
  if (h->nbf <= 0) return fail(h, CFSA_BAD_ARG, "mesh view carried no boundary faces");
  return guarded(h, [&] {
    k_face_forces<<<blocks_for(h->nbf), kBlock, 0, h->stream>>>(
        (int)h->nbf, (int)h->nt, h->N2, h->viscosity, h->fverts, h->ftet, h->fnormal, h->farea, h->tnode,
        h->grad, h->u, h->p, h->fshear, h->fpress);
    std::vector<double> a((size_t)3 * h->nv), b((size_t)3 * h->nv);
    if (which == 0 || which == 2) {
      k_face_gather<<<blocks_for(h->nv), kBlock, 0, h->stream>>>((int)h->nv, h->vf_ptr, h->vf, h->fpress,
                                                                 h->fout);
      CK(cudaMemcpyAsync(a.data(), h->fout, a.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
    if (which == 1 || which == 2) {
      k_face_gather<<<blocks_for(h->nv), kBlock, 0, h->stream>>>((int)h->nv, h->vf_ptr, h->vf, h->fshear,
                                                                 h->fout);
      CK(cudaMemcpyAsync(b.data(), h->fout, b.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaGetLastError());
    for (size_t k = 0; k < a.size(); ++k)
      out[k] = (which == 0) ? a[k] : (which == 1) ? b[k] : a[k] + b[k];
    return CFSA_OK;
  });
}

int cfsa_ns_compute_pressure_forces(cfsa_ns *h, double *out) { return face_forces(h, out, 0); }
int cfsa_ns_compute_shear_stress(cfsa_ns *h, double *out) { return face_forces(h, out, 1); }
int cfsa_ns_compute_total_fluid_forces(cfsa_ns *h, double *out) { return face_forces(h, out, 2); }

int cfsa_ns_get_matrix_size(cfsa_ns *h, int which, int64_t *nrows, int64_t *nnz) {
  if (!h || !nrows || !nnz) return CFSA_BAD_ARG;
  if (which < 0 || which > 7) return fail(h, CFSA_BAD_ARG, "unknown matrix id");
  const bool p2 = (which == CFSA_MAT_MASS || which == CFSA_MAT_STIFFNESS || which == CFSA_MAT_MOMENTUM);
  *nrows = p2 ? h->N2 : h->nv;
  *nnz = p2 ? h->nnz2 : h->nnz1;
  return CFSA_OK;
}

int cfsa_ns_get_matrix(cfsa_ns *h, int which, int64_t *rowptr, int32_t *cols, double *vals) {
  if (!h || !rowptr || !cols || !vals) return CFSA_BAD_ARG;
  if (which < 0 || which > 7) return fail(h, CFSA_BAD_ARG, "unknown matrix id");
  return guarded(h, [&] {
    const bool p2 = (which == CFSA_MAT_MASS || which == CFSA_MAT_STIFFNESS || which == CFSA_MAT_MOMENTUM);
    const int64_t n = p2 ? h->N2 : h->nv, nnz = p2 ? h->nnz2 : h->nnz1;
    const std::vector<int> &rp = p2 ? h->h_rp2 : h->h_rp1;
    for (int64_t i = 0; i <= n; ++i) rowptr[i] = rp[i];
    CK(cudaMemcpyAsync(cols, p2 ? h->ci2 : h->ci1, nnz * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    auto get = [&](const double *d, double *o) {
      CK(cudaMemcpyAsync(o, d, nnz * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    };
    std::vector<double> tmp;
    switch (which) {
      case CFSA_MAT_MASS: get(h->Mv, vals); break;
      case CFSA_MAT_STIFFNESS: get(h->Kv, vals); break;
      case CFSA_MAT_GRAD_X: get(h->Gv, vals); break;
      case CFSA_MAT_GRAD_Y: get(h->Gv + h->nnz1, vals); break;
      case CFSA_MAT_GRAD_Z: get(h->Gv + 2 * h->nnz1, vals); break;
      case CFSA_MAT_POISSON: get(h->Lv, vals); break;
      case CFSA_MAT_MOMENTUM:
        tmp.resize(nnz);
        get(h->Mv, vals);
        get(h->Kv, tmp.data());
        break;
      case CFSA_MAT_POISSON_BC: get(h->Lv, vals); break;
    }
    CK(cudaStreamSynchronize(h->stream));
    if (which == CFSA_MAT_MOMENTUM) {
      for (int64_t i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
          double a = vals[k] / h->dt + tmp[k];
          if (cols[k] == i && (h->h_bc[i] == BC_INLET || h->h_bc[i] == BC_WALL)) a += kMomentumPenalty;
          vals[k] = a;
        }
    } else if (which == CFSA_MAT_POISSON_BC) {
      for (int64_t i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k)
          if (cols[k] == i && ((h->outlet_type == 1 && i == h->ref_node) ||
                               (h->outlet_type == 0 && h->h_bc[i] == BC_OUTLET)))
            vals[k] += kPoissonPenalty;
    }
    return CFSA_OK;
  });
}

int cfsa_ns_get_inv_lumped_mass(cfsa_ns *h, double *out) {
  if (!h || !out) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    CK(cudaMemcpyAsync(out, h->invm, h->N2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

// ---- VTK export (io::exportToVtk(filename, const NavierStokesSolver&, scale),
// src/IO/VtkExport.cpp:49-84, 238-268) ----
int cfsa_ns_write_vtk(cfsa_ns *h, const char *path, double scale, int fields) {
  if (!h || !path) return CFSA_BAD_ARG;
  if ((fields & (CFSA_VTK_SHEAR_STRESS | CFSA_VTK_PRESSURE_FORCES)) && h->nbf <= 0)
    return fail(h, CFSA_BAD_ARG, "boundary-force fields need boundary faces in the mesh view");
  return guarded(h, [&] {
    const int64_t nv = h->nv, nt = h->nt, N2 = h->N2;
    // pinned staging; the geometry copies are waited for first, the field copies (and the
    // force kernels) keep running while the points and cells are formatted
    double *hx = nullptr, *hp = nullptr, *hu = nullptr, *hf = nullptr;
    int *ht = nullptr;
    signed char *hb = nullptr;
    const int nforce = ((fields & CFSA_VTK_SHEAR_STRESS) ? 1 : 0) + ((fields & CFSA_VTK_PRESSURE_FORCES) ? 1 : 0);
    PinnedSet pin;
    hx = pin.get<double>((size_t)3 * nv);
    ht = pin.get<int>((size_t)4 * nt);
    hb = pin.get<signed char>((size_t)nv);
    hp = pin.get<double>((size_t)nv);
    hu = pin.get<double>((size_t)3 * nv);
    if (nforce) hf = pin.get<double>((size_t)3 * nv * nforce);
    cudaEvent_t geo = nullptr;
    CK(cudaEventCreateWithFlags(&geo, cudaEventDisableTiming));
    CK(cudaMemcpyAsync(hx, h->xyz, (size_t)3 * nv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(ht, h->tnode, (size_t)4 * nt * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(hb, h->bc, (size_t)nv, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaEventRecord(geo, h->stream));
    CK(cudaMemcpyAsync(hp, h->p, (size_t)nv * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpy2DAsync(hu, (size_t)nv * sizeof(double), h->u, (size_t)N2 * sizeof(double),
                         (size_t)nv * sizeof(double), 3, cudaMemcpyDeviceToHost, h->stream));
    int slot = 0;
    for (int which : {CFSA_VTK_SHEAR_STRESS, CFSA_VTK_PRESSURE_FORCES}) {
      if (!(fields & which)) continue;
      k_face_forces<<<blocks_for(h->nbf), kBlock, 0, h->stream>>>((int)h->nbf, (int)nt, N2, h->viscosity,
                                                                    h->fverts, h->ftet, h->fnormal, h->farea,
                                                                    h->tnode, h->grad, h->u, h->p, h->fshear,
                                                                    h->fpress);
      k_face_gather<<<blocks_for(nv), kBlock, 0, h->stream>>>(
          (int)nv, h->vf_ptr, h->vf, which == CFSA_VTK_SHEAR_STRESS ? h->fshear : h->fpress, h->fout);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(hf + (size_t)3 * nv * slot, h->fout, (size_t)3 * nv * sizeof(double),
                         cudaMemcpyDeviceToHost, h->stream));
      ++slot;
    }
    const cudaError_t eg = cudaEventSynchronize(geo);
    cudaEventDestroy(geo);
    CK(eg);
    std::ofstream out(path);
    if (!out.is_open()) {
      CK(cudaStreamSynchronize(h->stream));
      return fail(h, CFSA_BAD_ARG, std::string("cannot open ") + path);
    }
    out << "# vtk DataFile Version 3.0\nShape export\nASCII\nDATASET UNSTRUCTURED_GRID\n";
    out << "POINTS " << nv << " double\n";
    for (int64_t i = 0; i < nv; ++i)
      out << hx[3 * i] * scale << " " << hx[3 * i + 1] * scale << " " << hx[3 * i + 2] * scale << "\n";
    out << "CELLS " << nt << " " << nt * 5 << "\n";
    for (int64_t t = 0; t < nt; ++t)
      out << "4 " << ht[t] << " " << ht[nt + t] << " " << ht[2 * nt + t] << " " << ht[3 * nt + t] << "\n";
    out << "CELL_TYPES " << nt << "\n";
    for (int64_t t = 0; t < nt; ++t) out << "10\n";
    out << "\nPOINT_DATA " << nv << "\n";
    out << "SCALARS FluidBoundaryType int 1\nLOOKUP_TABLE default\n";
    for (int64_t i = 0; i < nv; ++i) out << (int)hb[i] << "\n";
    CK(cudaStreamSynchronize(h->stream));
    out << "\nSCALARS pressure double 1\nLOOKUP_TABLE default\n";
    for (int64_t i = 0; i < nv; ++i) out << hp[i] << "\n";
    out << "\nVECTORS velocity double\n";
    for (int64_t i = 0; i < nv; ++i)
      out << hu[i] * scale << " " << hu[nv + i] * scale << " " << hu[2 * nv + i] * scale << "\n";
    slot = 0;
    for (int which : {CFSA_VTK_SHEAR_STRESS, CFSA_VTK_PRESSURE_FORCES}) {
      if (!(fields & which)) continue;
      out << "\nVECTORS " << (which == CFSA_VTK_SHEAR_STRESS ? "shear_stress" : "pressure_forces") << " double\n";
      const double *f = hf + (size_t)3 * nv * slot;
      for (int64_t i = 0; i < nv; ++i) out << f[3 * i] << " " << f[3 * i + 1] << " " << f[3 * i + 2] << "\n";
      ++slot;
    }
    out.close();
    if (!out) return fail(h, CFSA_BAD_ARG, std::string("write failed: ") + path);
    return CFSA_OK;
  });
}

// ---- discrete adjoint ----
int cfsa_ns_objective(cfsa_ns *h, const cfsa_objective *obj, double *J) {
  if (!h || !obj || !J) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    if (!h->enqueue_objective(*obj, false)) return fail(h, CFSA_BAD_ARG, "objective vertex set is empty");
    CK(cudaMemcpyAsync(J, h->a_scal + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}

int cfsa_ns_adjoint_forward(cfsa_ns *h, int nsteps, int checkpoint_every, int *n_done) {
  if (!h) return CFSA_BAD_ARG;
  if (nsteps < 1) return fail(h, CFSA_BAD_ARG, "the forward pass needs at least one step");
  if (h->ncorr < 1) return fail(h, CFSA_UNSUPPORTED, "the adjoint needs at least one pressure corrector");
  return guarded(h, [&] {
    const int code = h->adjoint_forward(nsteps, checkpoint_every, n_done);
    if (code != CFSA_OK) h->err = "forward pass failed with status " + std::to_string(code);
    return code;
  });
}

int cfsa_ns_adjoint_backward(cfsa_ns *h, const cfsa_objective *obj, double *J, double *grad_inlet,
                             double *grad_viscosity, double *grad_u0, double *grad_p0) {
  if (!h || !obj) return CFSA_BAD_ARG;
  const int ready = h->check_adjoint_ready();
  if (ready != CFSA_OK) return ready;
  return guarded(h, [&] {
    h->restore_final_state();
    if (!h->enqueue_objective(*obj, true)) return fail(h, CFSA_BAD_ARG, "objective vertex set is empty");
    if (J) {
      CK(cudaMemcpyAsync(J, h->a_scal + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      CK(cudaStreamSynchronize(h->stream));
    }
    return h->adjoint_backward_core(grad_inlet, grad_viscosity, grad_u0, grad_p0);
  });
}

int cfsa_ns_adjoint_backward_seed(cfsa_ns *h, const double *dJ_du, const double *dJ_dp,
                                  double dJ_dviscosity, double *grad_inlet, double *grad_viscosity,
                                  double *grad_u0, double *grad_p0) {
  if (!h) return CFSA_BAD_ARG;
  const int ready = h->check_adjoint_ready();
  if (ready != CFSA_OK) return ready;
  return guarded(h, [&] {
    h->ensure_adjoint_work();
    h->restore_final_state();
    if (dJ_du)
      h->upload_vec3(dJ_du, h->a_lu);
    else
      CK(cudaMemsetAsync(h->a_lu, 0, (size_t)3 * h->N2 * sizeof(double), h->stream));
    if (dJ_dp)
      CK(cudaMemcpyAsync(h->a_lp, dJ_dp, (size_t)h->nv * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    else
      CK(cudaMemsetAsync(h->a_lp, 0, (size_t)h->nv * sizeof(double), h->stream));
    CK(cudaMemcpyAsync(h->a_scal, &dJ_dviscosity, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return h->adjoint_backward_core(grad_inlet, grad_viscosity, grad_u0, grad_p0);
  });
}

int cfsa_ns_get_adjoint_stats(cfsa_ns *h, cfsa_adjoint_stats *out) {
  if (!h || !out) return CFSA_BAD_ARG;
  *out = h->adj_stats;
  return CFSA_OK;
}

}  // extern "C"

extern "C" int cfsa_ns_set_barrier_spin_limit(cfsa_ns *h, int64_t polls) {
  if (!h) return CFSA_BAD_ARG;
  const long long lim = polls < 0 ? kBarrierSpinLimit : (long long)polls;
  if (lim != h->bar_spin_limit) h->graph_dirty = true;  // the limit is a captured launch argument
  h->bar_spin_limit = lim;
  return CFSA_OK;
}

extern "C" int cfsa_ns_profile_kernel(cfsa_ns *h, int which, int iters, double *avg_ms,
                                      double *alg_bytes) {
  if (!h || !avg_ms || !alg_bytes || iters < 1) return CFSA_BAD_ARG;
  return guarded(h, [&] {
    h->profile_kernel(which, iters, avg_ms, alg_bytes);
    return CFSA_OK;
  });
}

// ---------------------------------------------------------------------------------------------
// Allocation-free divergence. Its per-tet scratch is a static device array instead of handle
// memory; callers pass device inputs and outputs.
namespace {
constexpr int64_t kNoAllocMaxTets = int64_t(1) << 20;  // 8 MiB per GPU that loads the library
__device__ __align__(256) double g_noalloc_divt[kNoAllocMaxTets];

std::mutex g_noalloc_mutex;
constexpr int kNoAllocMaxDevices = 256;
double *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of g_noalloc_divt for the current device (host code cannot use the symbol
// itself as a device address). Looked up once per device, under a lock.
int noalloc_scratch(cfsa_ns *h, double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(h, CFSA_CUDA_ERROR, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(h, CFSA_BAD_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_noalloc_divt);
    if (e != cudaSuccess || !ptr)
      return fail(h, CFSA_CUDA_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = static_cast<double *>(ptr);
  }
  *out = g_noalloc_ptr[dev];
  return CFSA_OK;
}

// Makes `dev` current for the lifetime of the guard and puts the caller's device back on every
// return path, so a multi-GPU caller's later CUDA calls run where it expects.
struct DeviceGuard {
  int prev = -1;
  bool switched = false;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) {
      ok = (cudaSetDevice(dev) == cudaSuccess);
      switched = ok && prev >= 0;
    }
  }
  ~DeviceGuard() {
    if (switched) cudaSetDevice(prev);
  }
};
}  // namespace

extern "C" int cfsa_ns_compute_divergence_noalloc(cfsa_ns *h, const double *u_dev, double *div_dev) {
  if (!h || !u_dev || !div_dev) return CFSA_BAD_ARG;
  if (h->nt > kNoAllocMaxTets)
    return fail(h, CFSA_BAD_ARG,
                "cfsa_ns_compute_divergence_noalloc: mesh has " + std::to_string(h->nt) +
                    " tets, the static scratch holds at most " + std::to_string(kNoAllocMaxTets));
  DeviceGuard guard(h->device);
  if (!guard.ok) return fail(h, CFSA_CUDA_ERROR, "cannot select the handle's device");
  double *scratch = nullptr;
  const int code = noalloc_scratch(h, &scratch);
  if (code != CFSA_OK) return code;
  return guarded(h, [&] {
    k_tet_div<<<blocks_for(h->nt), kBlock, 0, h->stream>>>((int)h->nt, h->N2, h->tnode, h->grad, u_dev,
                                                           scratch, nullptr);
    k_gather_div<<<blocks_for(h->nv), kBlock, 0, h->stream>>>((int)h->nv, h->adj_ptr, h->adj, h->vol,
                                                              scratch, div_dev);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return CFSA_OK;
  });
}
