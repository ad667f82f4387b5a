// planc_gpu.cu -- context, orchestration and C ABI of the B200 NTF library.
//
// One context = one device-resident tensor + CP factors + one stream. The
// AUNTF outer iteration (ntf/auntf.hpp:128-177) is issued as a fixed launch
// sequence per mode: [MTTKRP] -> [update] -> [normalise + Gram + next
// leave-one-out Gram], then the Gram-form error; it is captured once into a
// CUDA graph and replayed for every iteration.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/planc_gpu.h"
#include "bpp.cuh"
#include "common.cuh"
#include "kernels_f64.cuh"
#include "tc_mttkrp.cuh"
#include "nmf.cuh"
#include "updates_iter.cuh"
#include "batch_group.cuh"
#include "tc_group.cuh"

using namespace pg;

namespace {

thread_local std::string g_last_error;

struct Fail {
  int code;
};

[[noreturn]] void fail(int code, const std::string& msg) {
  g_last_error = msg;
  throw Fail{code};
}

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    fail(e == cudaErrorMemoryAllocation ? PLANC_GPU_ERR_OOM : PLANC_GPU_ERR_CUDA,
         std::string(what) + ": " + cudaGetErrorString(e));
  }
}
#define CK(x) cuda_check((x), #x)

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return PLANC_GPU_OK;
  } catch (const Fail& e) {
    return e.code;
  } catch (...) {
    g_last_error = "unexpected host exception";
    return PLANC_GPU_ERR_CUDA;
  }
}

int kpad(int k) { return k <= 8 ? 8 : k <= 16 ? 16 : k <= 32 ? 32 : 64; }

// Longest Khatri-Rao operand (rows) of the balanced 4-way tree: at rank 64
// its hi|lo image is 256 B a row, 32 MiB at this bound, small enough to stay
// in L2 while every CTA of the long-K contraction streams it.
constexpr int64_t kBal4MaxK = int64_t(1) << 17;

}  // namespace

// Host tensors are uploaded through a staging buffer of this size, in chunks
// of the natural element order; the sum of squares takes this many per-chunk
// partials.
constexpr int64_t kStageBytes = 64ll << 20;
constexpr int kNormBlocks = 1184;

struct planc_gpu_ctx {
  int device = 0;
  int precision = PLANC_GPU_PREC_FP64;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int sm_count = 148;
  size_t smem_optin = 0;     // dynamic shared memory the cooperative W sweep may use
  int ngc_ctas = 0;          // largest cluster of k_normgram_cluster (0: not used)
  int nes_max_steps = NES_MAX_STEPS;  // step cap of the Nesterov inner loop
  bool coop_launch = false;  // device takes cooperative launches

  int N = 0;
  int64_t dims[kMaxModes] = {0};
  int64_t numel = 0;
  int s = 0;
  int64_t L = 0, R = 0;
  // 4-way tensor on the tensor-core paths: balanced tree {0,1} | {2,3} (see
  // mttkrp_bal4) instead of the reference's {0,1,2} | {3}.
  bool bal4 = false;
  int k = 0;
  bool have_tensor = false, have_factors = false;

  double* X64 = nullptr;         // FP64 tensor (plain path)
  int64_t x64_elems = 0;
  void* stage = nullptr;         // host-upload staging buffer (kStageBytes), made on first use
  double* cp_part = nullptr;     // CP-loss Gram partials (N x CPG_BLOCKS x k x k)
  unsigned* cp_ctr = nullptr;    // their per-factor completion counters
  double* norm_part = nullptr;   // per-block partial sums of squares of one chunk
  TcTensor tct;                  // tensor-core operand copy (BF16 paths)
  // copies with mode n moved last for the direct (non-tree) MTTKRP on the
  // tensor cores, made on first use; the last mode uses tct when its view
  // already splits before the last mode
  TcTensor tcd[kMaxModes];
  // the direct views' Khatri-Rao generators take two or three factors: a
  // lone listed mode runs against a row of ones, four or more against the
  // first listed factor and an image of the product of the others
  double* ones_k = nullptr;      // kMaxRank ones
  int ones_cap = 0;
  double* krp_tail = nullptr;    // tail image, rows x k
  size_t krp_tail_elems = 0;
  double* normX2 = nullptr;      // device scalar ||X||^2
  double* F[kMaxModes] = {nullptr};
  double* M[kMaxModes] = {nullptr};
  double* Gall = nullptr;
  double* Gloo = nullptr;
  double* lambda = nullptr;
  double* P = nullptr;           // right-contracted partial MTTKRP, row-major L x k
  float* P32 = nullptr;          // same, FP32, for the tensor-core paths
  double* Q = nullptr;           // N = 4: P contracted with F_0, row-major (I1*I2) x k;
                                 // balanced 4-way tree: X^T KRP(F_0, F_1), (I2*I3) x k
  double* scratch = nullptr;
  size_t scratch_elems = 0;
  double* lam_tmp = nullptr;    // lambda of a normalisation whose lambda is not kept
  double* gram_part = nullptr;  // per-row-block partial Grams
  size_t gram_part_elems = 0;
  double* errs_dev = nullptr;
  int errs_cap = 0;
  int* counter_dev = nullptr;
  int* status_dev = nullptr;
  int64_t factor_cap[kMaxModes] = {0};

  // Per-mode state of the iterative updates, kept between runs like the
  // members of the reference's solver objects; allocated zeroed on the first
  // run of the algorithm (planc_gpu_reset_update_state zeroes it again).
  //   AO-ADMM (NTFAOADMM, ntf/ntfaoadmm.hpp:13-21): the dual variable aux[n].
  //   Nesterov (NTFNES, ntf/ntfnes.hpp:11-24): proximal and previous iterates
  //   prox[n] / prev[n] and their lambdas, the acceleration counters (NesDev).
  bool admm_ready = false, nes_ready = false;
  double* aux[kMaxModes] = {nullptr};
  double* admm_L = nullptr;     // k x k Cholesky factor of G + alpha I
  double* admm_scal = nullptr;  // alpha
  int* admm_flag = nullptr;     // [0] stop flag, [1] CTA counter
  double* admm_part = nullptr;  // partial norms (ADMM_MAX_BLOCKS x 4) / column sums
  size_t admm_part_elems = 0;
  double* prox[kMaxModes] = {nullptr};
  double* prev[kMaxModes] = {nullptr};
  double* nes_acc = nullptr;    // maxI x k scratch of the inner loop
  double* nes_grad = nullptr;
  double* nes_modM = nullptr;
  double* nes_lam = nullptr;    // [0,k) proximal, [k,2k) previous, [2k,3k) backup lambda
  double* nes_gbak = nullptr;   // N x k x k backup Grams
  NesDev* nes = nullptr;
  int cl_ctas = NES_CTAS;       // CTAs of the register-resident update clusters

  // Shared-memory NMF of the context's 2-way tensor A ~ W H^T (W = F[0],
  // H = F[1], A H -> M[0], A^T W -> M[1]); buffers allocated on the first run.
  bool nmf_have = false;        // W and H set by planc_gpu_nmf_set_factors
  bool nmf_ready = false;
  double* nmf_G = nullptr;      // regularised Gram of the fixed factor, k x k
  double* nmf_GW = nullptr;     // W^T W and H^T H of the objective, k x k each
  double* nmf_GH = nullptr;
  double* nmf_norms = nullptr;  // column norms of the HALS W sweep, k
  double* nmf_part = nullptr;   // Gram / column-sum / norm partials
  size_t nmf_part_elems = 0;
  int* nmf_ctr = nullptr;       // [0] objective index, [1] CTA ticket, [4] W sweep error flag
  double* nmf_obj = nullptr;    // objective and relative error per iteration
  double* nmf_rel = nullptr;
  int nmf_cap = 0;
  double nmf_reg[5] = {0, 0, 0, 0, 0};  // regW L2, L1, regH L2, L1, symm_reg
  cudaGraphExec_t nmf_gexec = nullptr;
  int nmf_galgo = -1;
  int64_t nmf_gepoch = -1;

  // cached iteration graphs: [0] the plain iteration, [1] iteration +
  // Nesterov acceleration
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int g_algo[2] = {-1, -1}, g_dimtree[2] = {-1, -1}, g_err[2] = {-1, -1};

  bool timing = false;
  bool capturing = false;
  struct Pending {
    int cls;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> ev_pool;
  double kms[KC_COUNT] = {0};
  int64_t klaunch[KC_COUNT] = {0};
  int64_t launch_count = 0;
  int bpp_max_iter = 0;  // 0: the reference's 5k cap
  bool bpp_warm = true;  // ANLS/BPP rows start from the replaced factor's passive set
  int bpp_kernel = 0;    // 0: by size, 1: a warp per right-hand side, 2: a CTA per right-hand side
  // Fraction of the GPU one launch of this context aims to fill (split-K and
  // grid sizing). 1 for a context alone on the GPU; the batch autotuner lowers
  // it when many contexts run concurrently.
  double par_scale = 1.0;
  // fewest chunks per split-K partial of the tensor-core left contraction
  // (0: the default plan); the batch autotuner raises it for small members
  int left_chunks = 0;
  // parts per run of I0 of the factored left contraction's work units
  // (PLANC_GPU_LEFT_PARTS; 0: the default)
  int left_parts = 0;
  // 3-way tensor-core left contraction without the factored form (I_0 not a
  // multiple of 64): against a Khatri-Rao image with the long-K kernel
  // (default) or with Khatri-Rao producer warps (PLANC_GPU_LEFT_FORM=producers)
  bool left_long = true;
  // tensor tiles of the tensor-core right and factored left contractions
  // through cp.async producer warps (default) or TMA (PLANC_GPU_TC_LOADS=tma)
  bool tc_cpa = true;
  // Incremented whenever a device buffer that a captured graph may reference
  // is (re)allocated; cached graphs are rebuilt when it changes.
  int64_t buf_epoch = 0;
  size_t gall_elems = 0;  // capacity of Gall
  int kvec = 0;           // rank the k-sized buffers (Gloo, lambda, lam_tmp) hold
  int64_t g_epoch = -1;
};

namespace {

void set_device(planc_gpu_ctx* c) { CK(cudaSetDevice(c->device)); }

// SMs one launch of this context is sized for
int eff_sm(const planc_gpu_ctx* c) {
  int v = (int)(c->sm_count * c->par_scale);
  return v < 1 ? 1 : v;
}

// Batched BPP of ncols right-hand sides with the k x k matrix AtA (k_bpp: a
// warp per right-hand side; k_bpp_cta: a CTA per right-hand side, for k > 16
// while the right-hand sides are too few to give every SM several warps).
// Launched on the context's stream; the caller times it.
void launch_bpp(planc_gpu_ctx* c, const double* AtA, const double* B, int n, int64_t ncols,
                double* X, int* P, int* I, const double* warm) {
  if (ncols <= 0) return;
  const int kp = kpad(n);
  bool cta = kp >= 32 && ncols <= 4 * (int64_t)c->sm_count;
  if (c->bpp_kernel == 1) cta = false;
  if (c->bpp_kernel == 2) cta = kp >= 32;
  if (cta) {
    const unsigned grid = (unsigned)std::min<int64_t>(ncols, 2 * (int64_t)c->sm_count);
    if (kp == 32) {
      using C = BppCta<32, 8>;
      k_bpp_cta<32, 8><<<grid, C::THREADS, C::SMEM, c->stream>>>(AtA, B, n, ncols, X, P, I, c->status_dev,
                                                                c->bpp_max_iter, warm);
    } else {
      using C = BppCta<64, 8>;
      k_bpp_cta<64, 8><<<grid, C::THREADS, C::SMEM, c->stream>>>(AtA, B, n, ncols, X, P, I, c->status_dev,
                                                                c->bpp_max_iter, warm);
    }
    return;
  }
  const unsigned blocks = (unsigned)((ncols + BPP_WARPS - 1) / BPP_WARPS);
  switch (kp) {
#define CASE(KP)                                                                                    \
  case KP:                                                                                          \
    k_bpp<KP><<<blocks, 32 * BPP_WARPS, bpp_smem_bytes(KP), c->stream>>>(AtA, B, n, ncols, X, P, I, \
                                                                         c->status_dev,             \
                                                                         c->bpp_max_iter, warm);    \
    break;
    CASE(8) CASE(16) CASE(32) CASE(64)
#undef CASE
  }
}

template <typename T>
void dalloc(T** p, size_t n) {
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  if (n == 0) return;
  CK(cudaMalloc((void**)p, n * sizeof(T)));
}

cudaEvent_t get_event(planc_gpu_ctx* c) {
  if (!c->ev_pool.empty()) {
    cudaEvent_t e = c->ev_pool.back();
    c->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  CK(cudaEventCreate(&e));
  return e;
}

void drain_timing(planc_gpu_ctx* c) {
  if (c->pending.empty()) return;
  CK(cudaStreamSynchronize(c->stream));
  for (auto& p : c->pending) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, p.a, p.b));
    c->kms[p.cls] += ms;
    c->klaunch[p.cls] += 1;
    c->ev_pool.push_back(p.a);
    c->ev_pool.push_back(p.b);
  }
  c->pending.clear();
}

// Launch wrapper: counts launches, checks the launch error, optionally
// brackets the launch with events of its kernel class.
template <typename Fn>
void launch(planc_gpu_ctx* c, int cls, Fn&& fn) {
  cudaEvent_t a = nullptr, b = nullptr;
  bool timed = c->timing && !c->capturing;
  if (timed) {
    a = get_event(c);
    b = get_event(c);
    CK(cudaEventRecord(a, c->stream));
  }
  fn();
  CK(cudaGetLastError());
  if (timed) {
    CK(cudaEventRecord(b, c->stream));
    c->pending.push_back({cls, a, b});
    if (c->pending.size() > (1u << 16)) drain_timing(c);
  }
  c->launch_count++;
}

// Launches `kern` as one thread-block cluster of `ncta` CTAs of NES_THREADS
// threads (cluster sizes above 8 need the kernel's non-portable attribute,
// set by enable_cluster16).
template <typename... KArgs, typename... Args>
void launch_cluster(void (*kern)(KArgs...), int ncta, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)ncta, 1, 1);
  cfg.blockDim = dim3(NES_THREADS, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)ncta;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, kern, args...));
}

// Allows clusters of 16 for `kern` and reports whether one fits on the device.
template <typename... KArgs>
bool enable_cluster16(void (*kern)(KArgs...)) {
  if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(NES_CTAS_MAX, 1, 1);
  cfg.blockDim = dim3(NES_THREADS, 1, 1);
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = NES_CTAS_MAX;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, (const void*)kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n >= 1;
}

template <int BE>
int ngc_cluster_size_of() {
  auto kern = k_normgram_cluster<BE>;
  for (int cl : {16, 8}) {
    if (cl == 16 &&
        cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ngc_smem_bytes(64)) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl, 1, 1);
    cfg.blockDim = dim3(NGC_THREADS, 1, 1);
    cfg.dynamicSmemBytes = ngc_smem_bytes(64);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int nc = 0;
    if (cudaOccupancyMaxActiveClusters(&nc, (const void*)kern, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (nc >= 1) return cl;
  }
  return 0;
}

// Cluster size of k_normgram_cluster on the current device: 16 where clusters
// of 16 fit, else 8 where 8 fit, else 0 (the three-launch form).
int ngc_cluster_size() {
  const int a = ngc_cluster_size_of<2>(), b = ngc_cluster_size_of<4>();
  return a < b ? a : b;
}

WGen make_wgen(planc_gpu_ctx* c, const std::vector<int>& modes) {
  WGen g;
  memset(&g, 0, sizeof(g));
  g.nf = (int)modes.size();
  int64_t stride = 1;
  for (int t = 0; t < g.nf; ++t) {
    g.f[t] = c->F[modes[t]];
    g.dim[t] = c->dims[modes[t]];
    g.stride[t] = stride;
    stride *= c->dims[modes[t]];
  }
  return g;
}

// ---------------------------------------------------------------- planning
struct ContractPlan {
  ContractGeom g;
  int nsplit;
  dim3 grid;
};

ContractPlan plan_contract(planc_gpu_ctx* c, bool left, int64_t M, int64_t ldx, int64_t A,
                           int64_t B, int64_t ldb) {
  ContractPlan p;
  memset(&p, 0, sizeof(p));
  p.g.M = M;
  p.g.ldx = ldx;
  p.g.A = A;
  p.g.B = B;
  p.g.ldb = ldb;
  const int bk = c->k > 32 ? ct_bk<64>() : ct_bk<32>();
  int64_t tilesA = (A + bk - 1) / bk;
  p.g.ktiles = left ? tilesA * B : tilesA;
  int64_t mtiles = (M + CT_BM - 1) / CT_BM;
  int64_t target = 2 * (int64_t)eff_sm(c);
  int64_t ns = (target + mtiles - 1) / mtiles;
  ns = std::max<int64_t>(1, std::min<int64_t>(ns, p.g.ktiles));
  ns = std::min<int64_t>(ns, 1024);
  p.g.tiles_per_split = (p.g.ktiles + ns - 1) / ns;
  ns = (p.g.ktiles + p.g.tiles_per_split - 1) / p.g.tiles_per_split;
  if (ns < 1) ns = 1;
  p.nsplit = (int)ns;
  p.g.split_stride = M * c->k;
  p.grid = dim3((unsigned)mtiles, (unsigned)ns, 1);
  return p;
}

size_t contract_scratch(const ContractPlan& p) {
  return p.nsplit > 1 ? (size_t)p.nsplit * p.g.split_stride : 0;
}

struct TtvRightPlan {
  int64_t bper;
  int nsplit;
  dim3 grid;
};

// Tiled right multi-TTV: a-tiles of 4096/KP rows; enough b-splits for about
// two CTAs per SM, capped so the partials stay a small fraction of T.
TtvRightPlan plan_ttv_right(planc_gpu_ctx* c, int64_t A, int64_t B) {
  TtvRightPlan p;
  const int KP = kpad(c->k);
  const int64_t AT = 16 * 256 / KP;
  const int64_t gx = (A + AT - 1) / AT;
  const int64_t target = 2 * (int64_t)eff_sm(c);
  int64_t ns = std::max<int64_t>(1, (target + gx - 1) / gx);
  ns = std::min<int64_t>(ns, std::max<int64_t>(1, B / 8));  // >= 8 b per split
  ns = std::min<int64_t>(ns, 512);
  p.bper = (B + ns - 1) / ns;
  ns = (B + p.bper - 1) / p.bper;
  p.nsplit = (int)ns;
  p.grid = dim3((unsigned)gx, (unsigned)ns, 1);
  return p;
}

void direct_geom(planc_gpu_ctx* c, int n, int64_t* A, int64_t* B) {
  *A = 1;
  *B = 1;
  for (int m = 0; m < n; ++m) *A *= c->dims[m];
  for (int m = n + 1; m < c->N; ++m) *B *= c->dims[m];
}

void ensure_buffers_impl(planc_gpu_ctx* c);

// Computes the largest scratch any MTTKRP path needs and (re)allocates; any
// reallocation invalidates the cached graph (it holds the old pointers).
void ensure_buffers(planc_gpu_ctx* c) {
  const void* before[7] = {c->scratch, c->P, c->P32, c->Q, c->tct.bimg, c->tct.bimg0, c->tct.wimg};
  ensure_buffers_impl(c);
  const void* after[7] = {c->scratch, c->P, c->P32, c->Q, c->tct.bimg, c->tct.bimg0, c->tct.wimg};
  for (int i = 0; i < 7; ++i)
    if (before[i] != after[i]) {
      c->buf_epoch++;
      break;
    }
}

// Error-history buffer of at least `n` entries (reallocation bumps the epoch).
void ensure_errs(planc_gpu_ctx* c, int n) {
  if (n < 1) n = 1;
  if (!c->errs_dev || n > c->errs_cap) {
    dalloc(&c->errs_dev, (size_t)n);
    c->errs_cap = n;
    c->buf_epoch++;
  }
}

// Whether the 3-way tensor-core tree's left contraction runs as the long-K
// kernel against a Khatri-Rao image (tc_long_prep + tc_long): when the
// factored form does not apply (I_0 % 64 != 0) and the context asks for it.
// The image (L rows of hi|lo BF16 values) is written once per call and read
// by every row group, where the producer-warp form regenerates each
// Khatri-Rao tile in every CTA that uses it.
bool left_via_long(const planc_gpu_ctx* c) {
  return c->left_long && c->N == 3 && !c->bal4 && c->precision != PLANC_GPU_PREC_FP64 &&
         c->tct.hi && !tc_left_factored(c->tct);
}
// The same choice for a direct-MTTKRP view (any number of modes).
bool direct_via_long(const planc_gpu_ctx* c, const TcTensor& t) {
  return c->left_long && c->precision != PLANC_GPU_PREC_FP64 && t.hi && !tc_left_factored(t);
}

void ensure_buffers_impl(planc_gpu_ctx* c) {
  const int k = c->k;
  size_t need = 0;
  if (c->N == 3 || c->N == 4) {
    ContractPlan pl = plan_contract(c, true, c->R, c->L, c->L, 1, 0);
    need = std::max(need, contract_scratch(pl));
    ContractPlan pr = plan_contract(c, false, c->L, c->L, c->R, 1, 0);
    need = std::max(need, contract_scratch(pr));
    TtvRightPlan tr = plan_ttv_right(c, c->dims[0], c->L / c->dims[0]);
    need = std::max(need, (size_t)tr.nsplit * c->dims[0] * k);
    if (c->N == 3 && c->precision != PLANC_GPU_PREC_FP64)
      need = std::max(need, (size_t)tc_right_ttv_nsplit(c->tct, k, eff_sm(c)) * c->dims[0] * k);
    if (c->N == 4) {
      TtvRightPlan t2 = plan_ttv_right(c, c->dims[1], c->dims[2]);
      need = std::max(need, (size_t)t2.nsplit * c->dims[1] * k);
    }
    need = std::max(need, tc_scratch_elems(c->tct, eff_sm(c), k));
    if (left_via_long(c)) {
      need = std::max(need, tc_long_scratch_elems(c->tct, true, k, eff_sm(c)));
      c->tct.wimg_K = std::max(c->tct.wimg_K, c->L);
    }
    if (c->bal4) {
      TtvRightPlan t3 = plan_ttv_right(c, c->dims[2], c->dims[3]);
      need = std::max(need, (size_t)t3.nsplit * c->dims[2] * k);
      need = std::max(need, tc_long_scratch_elems(c->tct, true, k, eff_sm(c)));
      need = std::max(need, tc_long_scratch_elems(c->tct, false, k, eff_sm(c)));
      c->tct.wimg_K = std::max(c->L, c->R);
    }
    CK(tc_ensure(c->tct, k));
  }
  for (int n = 0; n < c->N; ++n) {
    int64_t A, B;
    direct_geom(c, n, &A, &B);
    ContractPlan pl = n == 0 ? plan_contract(c, false, c->dims[0], c->dims[0], B, 1, 0)
                             : plan_contract(c, true, c->dims[n], A, A, B, A * c->dims[n]);
    need = std::max(need, contract_scratch(pl));
  }
  need = std::max<size_t>(need, 4096);
  if (need > c->scratch_elems) {
    dalloc(&c->scratch, need);
    c->scratch_elems = need;
  }
  if (c->bal4) {
    if (!c->P) dalloc(&c->P, (size_t)c->L * k);
    if (!c->Q) dalloc(&c->Q, (size_t)c->R * k);
  } else if ((c->N == 3 || c->N == 4)) {
    if (c->precision == PLANC_GPU_PREC_FP64) {
      if (!c->P) dalloc(&c->P, (size_t)c->L * k);
    } else {
      if (!c->P32) dalloc(&c->P32, (size_t)c->L * k);
    }
    if (c->N == 4 && !c->Q) dalloc(&c->Q, (size_t)c->dims[1] * c->dims[2] * k);
  }
}

// k_contract_f64 specialised on the Khatri-Rao factor count (1, 2, 3; any
// other count takes the generic generator)
template <int KP, bool LEFT>
void launch_contract_f64(dim3 grid, cudaStream_t st, const double* X, const ContractGeom& g,
                         const WGen& wg, int k, double* dst, bool runs = false) {
  constexpr size_t sm = ct_smem_bytes<KP, LEFT>();
  if constexpr (LEFT) {
    if (runs && wg.nf == 2) {
      k_contract_f64<KP, true, 2, true><<<grid, 256, sm, st>>>(X, g, wg, k, dst);
      return;
    }
    if (runs && wg.nf == 3) {
      k_contract_f64<KP, true, 3, true><<<grid, 256, sm, st>>>(X, g, wg, k, dst);
      return;
    }
  }
  switch (wg.nf) {
    case 1: k_contract_f64<KP, LEFT, 1><<<grid, 256, sm, st>>>(X, g, wg, k, dst); break;
    case 2: k_contract_f64<KP, LEFT, 2><<<grid, 256, sm, st>>>(X, g, wg, k, dst); break;
    case 3: k_contract_f64<KP, LEFT, 3><<<grid, 256, sm, st>>>(X, g, wg, k, dst); break;
    default: k_contract_f64<KP, LEFT, 0><<<grid, 256, sm, st>>>(X, g, wg, k, dst); break;
  }
}

template <int KP, bool LEFT>
void contract_f64_attrs_kp() {
  constexpr int sm = (int)ct_smem_bytes<KP, LEFT>();
  CK(cudaFuncSetAttribute(k_contract_f64<KP, LEFT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_contract_f64<KP, LEFT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_contract_f64<KP, LEFT, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  CK(cudaFuncSetAttribute(k_contract_f64<KP, LEFT, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  if constexpr (LEFT) {
    CK(cudaFuncSetAttribute(k_contract_f64<KP, true, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    CK(cudaFuncSetAttribute(k_contract_f64<KP, true, 3, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
  }
}

// Dynamic shared-memory limits of every k_contract_f64 instance (up to 92 KB)
// on device dev, set once per device before its first launch.
std::mutex g_contract_attr_mutex;
bool g_contract_attr_set[64] = {false};
void contract_f64_attrs(int dev) {
  std::lock_guard<std::mutex> lock(g_contract_attr_mutex);
  if (dev < 0 || dev >= 64 || g_contract_attr_set[dev]) return;
  contract_f64_attrs_kp<8, false>();
  contract_f64_attrs_kp<8, true>();
  contract_f64_attrs_kp<16, false>();
  contract_f64_attrs_kp<16, true>();
  contract_f64_attrs_kp<32, false>();
  contract_f64_attrs_kp<32, true>();
  contract_f64_attrs_kp<64, false>();
  contract_f64_attrs_kp<64, true>();
  g_contract_attr_set[dev] = true;
}

void run_contract(planc_gpu_ctx* c, const ContractPlan& p, bool left, const double* X,
                  const WGen& wg, double* out, bool runs = false) {
  const int k = c->k;
  if (contract_scratch(p) > c->scratch_elems)
    fail(PLANC_GPU_ERR_STATE, "internal: contraction scratch larger than planned");
  double* dst = p.nsplit > 1 ? c->scratch : out;
  launch(c, left ? KC_CONTRACT_LEFT : KC_CONTRACT, [&] {
    switch (kpad(k)) {
#define CASE(KP)                                                                      \
  case KP:                                                                            \
    if (left)                                                                         \
      launch_contract_f64<KP, true>(p.grid, c->stream, X, p.g, wg, k, dst, runs);     \
    else                                                                              \
      launch_contract_f64<KP, false>(p.grid, c->stream, X, p.g, wg, k, dst);          \
    break;
      CASE(8) CASE(16) CASE(32) CASE(64)
#undef CASE
    }
  });
  if (p.nsplit > 1) {
    int64_t n = p.g.M * k;
    launch(c, KC_REDUCE, [&] {
      reduce_splits(c->stream, c->scratch, p.nsplit, p.g.split_stride, n, out);
    });
  }
}

template <typename TT>
void run_ttv_right(planc_gpu_ctx* c, const TT* T, int64_t A, int64_t B, const WGen& wg,
                   double* out) {
  TtvRightPlan p = plan_ttv_right(c, A, B);
  if (p.nsplit > 1 && (size_t)p.nsplit * A * c->k > c->scratch_elems)
    fail(PLANC_GPU_ERR_STATE, "internal: multi-TTV scratch larger than planned");
  double* dst = p.nsplit > 1 ? c->scratch : out;
  int k = c->k;
  launch(c, KC_TTV, [&] {
    switch (kpad(k)) {
      case 8: k_ttv_right_tiled<TT, 8><<<p.grid, 256, 0, c->stream>>>(T, A, B, k, wg, p.bper, dst); break;
      case 16: k_ttv_right_tiled<TT, 16><<<p.grid, 256, 0, c->stream>>>(T, A, B, k, wg, p.bper, dst); break;
      case 32: k_ttv_right_tiled<TT, 32><<<p.grid, 256, 0, c->stream>>>(T, A, B, k, wg, p.bper, dst); break;
      default: k_ttv_right_tiled<TT, 64><<<p.grid, 256, 0, c->stream>>>(T, A, B, k, wg, p.bper, dst); break;
    }
  });
  if (p.nsplit > 1) {
    int64_t n = A * k;
    launch(c, KC_REDUCE, [&] {
      reduce_splits(c->stream, c->scratch, p.nsplit, n, n, out);
    });
  }
}

template <typename TT>
void run_ttv_left(planc_gpu_ctx* c, const TT* T, int64_t A, int64_t B, const double* Fa,
                  double* out) {
  int k = c->k;
  const int64_t g2 = (B + TTVL_NB - 1) / TTVL_NB;
  // the float4 kernel when its CTAs fill the SMs this context may use (a
  // batch member's share after the autotuner's parallelism fraction)
  if (std::is_same<TT, float>::value && k % 4 == 0 && g2 >= eff_sm(c) && g2 <= 65535) {
    launch(c, KC_TTV, [&] {
      k_ttv_left_f4<<<(unsigned)g2, 256, 0, c->stream>>>((const float*)T, A, B, k, Fa, out);
    });
    return;
  }
  launch(c, KC_TTV, [&] {
    k_ttv_left<TT><<<(unsigned)std::min<int64_t>(B, 65535), 256, 0, c->stream>>>(T, A, B, k, Fa, out);
  });
}

// ---------------------------------------------------------------- MTTKRP
// The tensor-core view whose left contraction is mode n's direct MTTKRP:
// the tree's copy for the last mode when its view splits before it, else the
// mode's own copy (ensure_direct makes them before any graph capture).
const TcTensor& direct_view(planc_gpu_ctx* c, int n) {
  if (n == c->N - 1 && !c->bal4 && c->s == c->N - 2) return c->tct;
  if (!c->tcd[n].hi) fail(PLANC_GPU_ERR_STATE, "internal: direct tensor-core copy missing");
  return c->tcd[n];
}

// Makes the direct-MTTKRP copies of a tensor-core context and sizes their
// images and split-K scratch (outside graph capture; any allocation bumps
// the buffer epoch so cached graphs are rebuilt).
void ensure_direct(planc_gpu_ctx* c) {
  if (c->precision == PLANC_GPU_PREC_FP64) return;
  bool grew = false;
  size_t need = 0, tail = 0;
  CK(tc_ensure(c->tct, c->k));
  for (int n = 0; n < c->N; ++n) {
    if (!(n == c->N - 1 && !c->bal4 && c->s == c->N - 2) && !c->tcd[n].hi) {
      cudaError_t e = tc_direct_copy(c->tcd[n], c->tct, c->dims, c->N, n, c->s, c->stream);
      if (e == cudaErrorInvalidValue)
        fail(PLANC_GPU_ERR_CUDA, "cuTensorMapEncodeTiled rejected a direct-MTTKRP view");
      CK(e);
      grew = true;
    }
    TcTensor& t = const_cast<TcTensor&>(direct_view(c, n));
    uint8_t* before[3] = {t.bimg, t.bimg0, t.wimg};
    if (direct_via_long(c, t)) {
      t.wimg_K = std::max(t.wimg_K, t.L);
      need = std::max(need, tc_long_scratch_elems(t, true, c->k, eff_sm(c)));
    }
    CK(tc_ensure(t, c->k));
    if (before[0] != t.bimg || before[1] != t.bimg0 || before[2] != t.wimg) grew = true;
    need = std::max(need, tc_scratch_elems(t, eff_sm(c), c->k));
    if (c->N - 1 >= 4) {  // tail image: the modes after the first listed one
      const int64_t rows = c->numel / (c->dims[n] * c->dims[n == 0 ? 1 : 0]);
      tail = std::max(tail, (size_t)rows * c->k);
    }
  }
  if (!c->ones_k || c->ones_cap < c->k) {
    dalloc(&c->ones_k, (size_t)kMaxRank);
    k_fill<<<1, 64, 0, c->stream>>>(c->ones_k, kMaxRank, 1.0);
    CK(cudaGetLastError());
    c->ones_cap = kMaxRank;
    grew = true;
  }
  if (tail > c->krp_tail_elems) {
    dalloc(&c->krp_tail, tail);
    c->krp_tail_elems = tail;
    grew = true;
  }
  if (need > c->scratch_elems) {
    dalloc(&c->scratch, need);
    c->scratch_elems = need;
    grew = true;
  }
  if (grew) c->buf_epoch++;
}

// Direct MTTKRP of mode n on the tensor cores: the left contraction of the
// (prod_{i != n} I_i) x I_n view against the Khatri-Rao rows of the other
// modes, split-K partials summed in a fixed order.
void mttkrp_direct_tc(planc_gpu_ctx* c, int n, double* out) {
  std::vector<int> modes;
  for (int m = 0; m < c->N; ++m)
    if (m != n) modes.push_back(m);
  WGen wg = make_wgen(c, modes);
  // the left contraction's producers generate W = F_a * (F_b [* F_c]): two
  // or three factors. One listed mode: F_a against a row of ones; four or
  // more: F_a against the image of the others' product (k_krp_rows), the
  // same product order F_a * (F_b * (...)).
  const int64_t Ia = c->dims[modes[0]];
  if (wg.nf == 1 || wg.nf >= 4) {
    WGen w2;
    memset(&w2, 0, sizeof(w2));
    w2.nf = 2;
    w2.f[0] = wg.f[0];
    w2.dim[0] = Ia;
    w2.stride[0] = 1;
    const int64_t rows = c->numel / (c->dims[n] * Ia);
    w2.dim[1] = rows;
    w2.stride[1] = Ia;
    if (wg.nf == 1) {
      if (!c->ones_k) fail(PLANC_GPU_ERR_STATE, "internal: ones row missing");
      w2.f[1] = c->ones_k;
    } else {
      if ((size_t)rows * c->k > c->krp_tail_elems)
        fail(PLANC_GPU_ERR_STATE, "internal: Khatri-Rao tail image larger than planned");
      std::vector<int> rest(modes.begin() + 1, modes.end());
      WGen wt = make_wgen(c, rest);
      launch(c, KC_PREP, [&] {
        const unsigned nb = (unsigned)std::min<int64_t>((rows * c->k + 255) / 256, 4096);
        k_krp_rows<<<nb, 256, 0, c->stream>>>(wt, rows, c->k, c->krp_tail);
      });
      w2.f[1] = c->krp_tail;
    }
    wg = w2;
  }
  const TcTensor& t = direct_view(c, n);
  if (t.left_nf != wg.nf) fail(PLANC_GPU_ERR_STATE, "internal: direct view generator mismatch");
  const int64_t nn = c->dims[n] * c->k;
  if (direct_via_long(c, t)) {
    // the Khatri-Rao image of the generator, then the long-K contraction
    if ((t.L + TC_BK - 1) / TC_BK > (t.wimg_K + TC_BK - 1) / TC_BK || !t.wimg)
      fail(PLANC_GPU_ERR_STATE, "internal: Khatri-Rao image smaller than planned");
    if (tc_long_scratch_elems(t, true, c->k, eff_sm(c)) > c->scratch_elems)
      fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
    launch(c, KC_PREP, [&] { tc_long_prep(t, true, wg, c->k, c->stream); });
    int nsplit = 1;
    launch(c, KC_CONTRACT_LEFT, [&] {
      nsplit = tc_long(t, true, c->k, out, c->scratch, c->status_dev, eff_sm(c), c->stream);
    });
    if (nsplit > 1)
      launch(c, KC_REDUCE, [&] { reduce_splits(c->stream, c->scratch, nsplit, nn, nn, out); });
    return;
  }
  if (tc_scratch_elems(t, eff_sm(c), c->k) > c->scratch_elems)
    fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
  int nsplit = 0;
  launch(c, KC_CONTRACT_LEFT, [&] {
    nsplit = tc_left(t, wg, c->k, c->scratch, c->status_dev, eff_sm(c), c->stream, c->left_chunks);
  });
  launch(c, KC_REDUCE, [&] { reduce_splits(c->stream, c->scratch, nsplit, nn, nn, out); });
}

// Direct MTTKRP of mode n (common/tensor.hpp:246-327): FP64 contraction, or
// on a tensor-core context the left contraction of mode n's view.
void mttkrp_direct(planc_gpu_ctx* c, int n, double* out) {
  if (c->precision != PLANC_GPU_PREC_FP64) {
    mttkrp_direct_tc(c, n, out);
    return;
  }
  if (!c->X64) fail(PLANC_GPU_ERR_STATE, "no FP64 tensor copy");
  std::vector<int> modes;
  for (int m = 0; m < c->N; ++m)
    if (m != n) modes.push_back(m);
  WGen wg = make_wgen(c, modes);
  int64_t A, B;
  direct_geom(c, n, &A, &B);
  if (n == 0) {
    ContractPlan p = plan_contract(c, false, c->dims[0], c->dims[0], B, 1, 0);
    run_contract(c, p, false, c->X64, wg, out);
  } else {
    // mode 1: the reduction index is already runs of I_0 (A = I_0), so each
    // tile takes one Khatri-Rao tail of the slower modes
    ContractPlan p = plan_contract(c, true, c->dims[n], A, A, B, A * c->dims[n]);
    run_contract(c, p, true, c->X64, wg, out, n == 1 && (wg.nf == 2 || wg.nf == 3));
  }
}

// Right contraction P = X_(L x R) * F_{N-1} (dimtrees.hpp:281-306).
void partial_right(planc_gpu_ctx* c) {
  if (c->precision == PLANC_GPU_PREC_FP64) {
    WGen wg = make_wgen(c, {c->N - 1});
    ContractPlan p = plan_contract(c, false, c->L, c->L, c->R, 1, 0);
    run_contract(c, p, false, c->X64, wg, c->P);
  } else {
    launch(c, KC_PREP, [&] { tc_right_prep(c->tct, c->F[c->N - 1], c->k, c->stream); });
    launch(c, KC_CONTRACT, [&] {
      tc_right(c->tct, c->k, c->P32, c->status_dev, eff_sm(c), c->stream, c->tc_cpa);
    });
  }
}

// Left contraction M_{N-1} = X^T * KRP(F_0..F_s) (dimtrees.hpp:250-271).
void long_contract(planc_gpu_ctx* c, bool left, const std::vector<int>& modes, double* out);

void partial_left(planc_gpu_ctx* c, double* out) {
  std::vector<int> modes;
  for (int m = 0; m <= c->s; ++m) modes.push_back(m);
  if (left_via_long(c)) {
    long_contract(c, true, modes, out);
    return;
  }
  if (c->precision == PLANC_GPU_PREC_FP64) {
    WGen wg = make_wgen(c, modes);
    // reduction tiles aligned to runs of I_0 (the same tiles and splits as the
    // flat view when I_0 is a multiple of the tile): one Khatri-Rao tail per tile
    const int64_t bk = kpad(c->k) == 64 ? ct_bk<64>() : ct_bk<32>();
    const bool runs = (wg.nf == 2 || wg.nf == 3) && c->dims[0] % bk == 0;
    ContractPlan p = runs ? plan_contract(c, true, c->R, c->L, c->dims[0], c->L / c->dims[0], c->dims[0])
                          : plan_contract(c, true, c->R, c->L, c->L, 1, 0);
    run_contract(c, p, true, c->X64, wg, out, runs);
  } else {
    WGen wg = make_wgen(c, modes);
    int nsplit = 0;
    if (wg.nf < 2 || wg.nf > 3) fail(PLANC_GPU_ERR_UNSUPPORTED, "left contraction needs 2 or 3 modes");
    if (tc_scratch_elems(c->tct, eff_sm(c), c->k) > c->scratch_elems)
      fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
    launch(c, KC_CONTRACT_LEFT, [&] {
      nsplit = tc_left(c->tct, wg, c->k, c->scratch, c->status_dev, eff_sm(c), c->stream,
                       c->left_chunks);
    });
    int64_t n = c->R * c->k;
    launch(c, KC_REDUCE, [&] {
      reduce_splits(c->stream, c->scratch, nsplit, n, n, out);
    });
  }
}

// Long-K tensor-core contraction of the balanced 4-way tree: the Khatri-Rao
// image of `modes`, then out = X W (right, L x k) or X^T W (left, R x k).
void long_contract(planc_gpu_ctx* c, bool left, const std::vector<int>& modes, double* out) {
  WGen wg = make_wgen(c, modes);
  launch(c, KC_PREP, [&] { tc_long_prep(c->tct, left, wg, c->k, c->stream); });
  if (tc_long_scratch_elems(c->tct, left, c->k, eff_sm(c)) > c->scratch_elems)
    fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
  int nsplit = 1;
  launch(c, left ? KC_CONTRACT_LEFT : KC_CONTRACT, [&] {
    nsplit = tc_long(c->tct, left, c->k, out, c->scratch, c->status_dev, eff_sm(c), c->stream);
  });
  if (nsplit > 1) {
    const int64_t n = (left ? c->R : c->L) * c->k;
    launch(c, KC_REDUCE, [&] {
      reduce_splits(c->stream, c->scratch, nsplit, n, n, out);
    });
  }
}

// MTTKRP of mode n on the balanced 4-way tree {0,1} | {2,3} (tensor-core
// paths). Same in-order reuse as DenseDimensionTree::in_order_reuse_MTTKRP
// (dimtree/ddt.hpp:134-243) with split mode 1 instead of N/2:
//   mode 0: P = X KRP(F_2, F_3) (L = I0 I1 rows), M_0 = multi-TTV of P with F_1
//   mode 1: M_1 = TTV of P with the updated F_0
//   mode 2: Q = X^T KRP(F_0, F_1) (R = I2 I3 rows), M_2 = multi-TTV of Q with F_3
//   mode 3: M_3 = TTV of Q with the updated F_2
// Both intermediates are (I0 I1 or I2 I3) x k, so an iteration streams X
// twice and nothing else of its size; the reference's split would write and
// re-read an (I0 I1 I2) x k intermediate.
void mttkrp_bal4(planc_gpu_ctx* c, int n, double* out) {
  const int64_t* d = c->dims;
  if (n == 0) {
    long_contract(c, false, {2, 3}, c->P);
    run_ttv_right<double>(c, c->P, d[0], d[1], make_wgen(c, {1}), out);
  } else if (n == 1) {
    run_ttv_left<double>(c, c->P, d[0], d[1], c->F[0], out);
  } else if (n == 2) {
    long_contract(c, true, {0, 1}, c->Q);
    run_ttv_right<double>(c, c->Q, d[2], d[3], make_wgen(c, {3}), out);
  } else {
    run_ttv_left<double>(c, c->Q, d[2], d[3], c->F[2], out);
  }
}

// Dimension-tree MTTKRP of mode n (DenseDimensionTree::in_order_reuse_MTTKRP,
// dimtree/ddt.hpp:134-243). Mode 0 recomputes P from the current F_{N-1};
// modes 1..s reuse it with the freshly updated F_0 (.. F_{n-1}).
void mttkrp_dimtree(planc_gpu_ctx* c, int n, double* out) {
  if (c->bal4) {
    mttkrp_bal4(c, n, out);
    return;
  }
  const int N = c->N;
  const bool f64 = c->precision == PLANC_GPU_PREC_FP64;
  if (n == 0) {
    if (!f64 && N == 3) {
      const int ns = tc_right_ttv_nsplit(c->tct, c->k, eff_sm(c));
      if (ns > 0 && (size_t)ns * c->dims[0] * c->k <= c->scratch_elems) {
        // P = X F_2 with M_0 = TTV(P, F_1) formed in the same pass
        launch(c, KC_PREP, [&] { tc_right_prep(c->tct, c->F[2], c->k, c->stream); });
        launch(c, KC_CONTRACT, [&] {
          tc_right_ttv(c->tct, c->k, c->P32, c->F[1], c->scratch, c->status_dev, eff_sm(c),
                       c->stream, c->tc_cpa);
        });
        const int64_t nn = c->dims[0] * c->k;
        launch(c, KC_REDUCE, [&] {
          reduce_splits(c->stream, c->scratch, ns, nn, nn, out);
        });
        return;
      }
    }
    partial_right(c);
    std::vector<int> modes;
    for (int m = 1; m <= c->s; ++m) modes.push_back(m);
    WGen wg = make_wgen(c, modes);
    if (f64)
      run_ttv_right<double>(c, c->P, c->dims[0], c->L / c->dims[0], wg, out);
    else
      run_ttv_right<float>(c, c->P32, c->dims[0], c->L / c->dims[0], wg, out);
    return;
  }
  if (n == c->s + 1) {
    partial_left(c, out);
    return;
  }
  if (N == 3) {  // n == 1
    if (f64)
      run_ttv_left<double>(c, c->P, c->dims[0], c->dims[1], c->F[0], out);
    else
      run_ttv_left<float>(c, c->P32, c->dims[0], c->dims[1], c->F[0], out);
    return;
  }
  // N == 4
  if (n == 1) {
    if (f64)
      run_ttv_left<double>(c, c->P, c->dims[0], c->dims[1] * c->dims[2], c->F[0], c->Q);
    else
      run_ttv_left<float>(c, c->P32, c->dims[0], c->dims[1] * c->dims[2], c->F[0], c->Q);
    WGen wg = make_wgen(c, {2});
    run_ttv_right<double>(c, c->Q, c->dims[1], c->dims[2], wg, out);
    return;
  }
  // n == 2
  run_ttv_left<double>(c, c->Q, c->dims[1], c->dims[2], c->F[1], out);
}

// Runs the tree modes that `mode` reuses (from the root of its branch, 0 or
// s + 1, up to mode - 1) so that a single call sees the state an in-order
// sweep would leave.
void dimtree_prereq(planc_gpu_ctx* c, int mode) {
  const int root = mode <= c->s ? 0 : c->s + 1;
  for (int m = root; m < mode; ++m) mttkrp_dimtree(c, m, c->M[m]);
}

void mttkrp_any(planc_gpu_ctx* c, int n, bool dimtree, double* out) {
  if (dimtree && (c->N == 3 || c->N == 4))
    mttkrp_dimtree(c, n, out);
  else
    mttkrp_direct(c, n, out);
}

// ---------------------------------------------------------------- updates
void run_update(planc_gpu_ctx* c, int algo, int n) {
  const int k = c->k;
  const int64_t I = c->dims[n];
  if (algo == PLANC_GPU_HALS || algo == PLANC_GPU_MU) {
    // one warp per factor row, 8 rows per CTA
    unsigned blocks = (unsigned)((I + 7) / 8);
    launch(c, KC_UPDATE, [&] {
      if (k <= 32) {
        if (algo == PLANC_GPU_HALS)
          k_hals_warp<32><<<blocks, 256, 0, c->stream>>>(c->F[n], c->M[n], c->Gloo, I, k);
        else
          k_mu_warp<32><<<blocks, 256, 0, c->stream>>>(c->F[n], c->M[n], c->Gloo, I, k, kEps6);
      } else {
        if (algo == PLANC_GPU_HALS)
          k_hals_warp<64><<<blocks, 256, 0, c->stream>>>(c->F[n], c->M[n], c->Gloo, I, k);
        else
          k_mu_warp<64><<<blocks, 256, 0, c->stream>>>(c->F[n], c->M[n], c->Gloo, I, k, kEps6);
      }
    });
  } else if (algo == PLANC_GPU_ANLSBPP) {
    // NTFANLSBPP::update (ntf/ntfanlsbpp.hpp:15-57): all I_n right-hand sides
    // in one launch; the 2000-column chunking does not change values.
    launch(c, KC_BPP, [&] {
      launch_bpp(c, c->Gloo, c->M[n], k, I, c->F[n], nullptr, nullptr, c->bpp_warm ? c->F[n] : nullptr);
    });
  } else if (algo == PLANC_GPU_AOADMM) {
    if (!c->admm_ready) fail(PLANC_GPU_ERR_STATE, "internal: AO-ADMM state not allocated");
    // NTFAOADMM::update (ntf/ntfaoadmm.hpp:23-77): Cholesky of G + alpha I,
    // at most admm_iter = 5 ADMM iterations, then the dual variable is
    // normalised. Up to 1024 rows (rank <= 32) or 512 rows (rank <= 64): one
    // cluster launch with the rows in registers.
    const int64_t warps = (int64_t)c->cl_ctas * (NES_THREADS / 32);
    const int64_t rpw = (I + warps - 1) / warps;
    if ((k <= 32 && rpw <= 8) || rpw <= 4) {
      launch(c, KC_UPDATE, [&] {
#define ADMM_CL(KP, R)                                                                       \
  launch_cluster(k_admm_cluster<KP, R>, c->cl_ctas, c->stream, c->F[n], c->aux[n],           \
                 (const double*)c->M[n], (const double*)c->Gloo, I, k, 0.01, c->status_dev)
        if (k <= 32 && rpw <= 1) ADMM_CL(32, 1);
        else if (k <= 32 && rpw <= 2) ADMM_CL(32, 2);
        else if (k <= 32 && rpw <= 4) ADMM_CL(32, 4);
        else if (k <= 32) ADMM_CL(32, 8);
        else if (rpw <= 1) ADMM_CL(64, 1);
        else if (rpw <= 2) ADMM_CL(64, 2);
        else ADMM_CL(64, 4);
#undef ADMM_CL
      });
      return;
    }
    // larger modes: one launch per ADMM iteration (each returns at once once
    // the stopping test has passed)
    launch(c, KC_UPDATE, [&] {
      k_admm_prep<<<1, 256, 0, c->stream>>>(c->Gloo, k, c->admm_L, c->admm_scal, c->admm_flag,
                                            c->admm_flag + 1, c->status_dev);
    });
    const unsigned nb =
        (unsigned)std::min<int64_t>((I + ADMM_WARPS - 1) / ADMM_WARPS, ADMM_MAX_BLOCKS);
    for (int it = 0; it < 5; ++it)
      launch(c, KC_UPDATE, [&] {
        if (k <= 32)
          k_admm_step<32><<<nb, 32 * ADMM_WARPS, 0, c->stream>>>(
              c->F[n], c->aux[n], c->M[n], c->admm_L, c->admm_scal, I, k, 0.01, c->admm_flag,
              c->admm_part, c->admm_flag + 1);
        else
          k_admm_step<64><<<nb, 32 * ADMM_WARPS, 0, c->stream>>>(
              c->F[n], c->aux[n], c->M[n], c->admm_L, c->admm_scal, I, k, 0.01, c->admm_flag,
              c->admm_part, c->admm_flag + 1);
      });
    const unsigned nc = (unsigned)((I + CN_ROWS - 1) / CN_ROWS);
    if ((size_t)nc * k > c->admm_part_elems)
      fail(PLANC_GPU_ERR_STATE, "internal: column-norm partial buffer too small");
    launch(c, KC_UPDATE, [&] {
      k_colsumsq_partial<<<nc, 256, 0, c->stream>>>(c->aux[n], I, k, c->admm_part);
    });
    launch(c, KC_UPDATE, [&] {
      k_colnorm_apply<<<nc, 256, 0, c->stream>>>(c->aux[n], I, k, c->admm_part, (int)nc);
    });
  } else if (algo == PLANC_GPU_NESTEROV) {
    if (!c->nes_ready) fail(PLANC_GPU_ERR_STATE, "internal: Nesterov state not allocated");
    // NTFNES::update (ntf/ntfnes.hpp:100-151): eigenvalue bounds of G, then
    // the accelerated proximal-gradient loop from the proximal point, in one
    // cluster launch.
    launch(c, KC_UPDATE, [&] {
      k_nes_prep<<<1, 256, 0, c->stream>>>(c->Gloo, k, c->nes, n, c->nes_lam, c->nes_lam + k);
    });
    // rows per warp of the cluster; up to 8 (rank <= 32) or 4 (rank <= 64)
    // rows stay in registers, beyond that the state lives in global scratch
    const int64_t warps = (int64_t)c->cl_ctas * (NES_THREADS / 32);
    const int64_t rpw = (I + warps - 1) / warps;
    launch(c, KC_UPDATE, [&] {
#define NES_REG(KP, R)                                                                       \
  launch_cluster(k_nes_inner_reg<KP, R>, c->cl_ctas, c->stream, c->F[n],                      \
                 (const double*)c->prox[n], c->prev[n], (const double*)c->M[n],               \
                 (const double*)c->Gloo, c->nes, I, k, c->nes_max_steps, c->status_dev)
      if (k <= 32 && rpw <= 1) NES_REG(32, 1);
      else if (k <= 32 && rpw <= 2) NES_REG(32, 2);
      else if (k <= 32 && rpw <= 4) NES_REG(32, 4);
      else if (k <= 32 && rpw <= 8) NES_REG(32, 8);
      else if (k > 32 && rpw <= 1) NES_REG(64, 1);
      else if (k > 32 && rpw <= 2) NES_REG(64, 2);
      else if (k > 32 && rpw <= 4) NES_REG(64, 4);
      else if (k <= 32)
        k_nes_inner<32><<<NES_CTAS, NES_THREADS, 0, c->stream>>>(
            c->F[n], c->prox[n], c->prev[n], c->M[n], c->Gloo, c->nes, c->nes_acc, c->nes_grad,
            c->nes_modM, I, k, c->nes_max_steps, c->status_dev);
      else
        k_nes_inner<64><<<NES_CTAS, NES_THREADS, 0, c->stream>>>(
            c->F[n], c->prox[n], c->prev[n], c->M[n], c->Gloo, c->nes, c->nes_acc, c->nes_grad,
            c->nes_modM, I, k, c->nes_max_steps, c->status_dev);
#undef NES_REG
    });
  } else {
    fail(PLANC_GPU_ERR_ARG, "unknown algorithm " + std::to_string(algo));
  }
}

unsigned elem_grid(int64_t n) { return (unsigned)std::min<int64_t>((n + 255) / 256, 1184); }

// NTFNES bookkeeping after mode n's update and normalisation: m_prox_t[n] is
// the normalised update, and after the last mode its lambda is the factor's
// (normalize_rows, ntf/ntfnes.hpp:148-149).
void nes_post(planc_gpu_ctx* c, int n) {
  if (!c->nes_ready) fail(PLANC_GPU_ERR_STATE, "internal: Nesterov state not allocated");
  const int64_t ne = c->dims[n] * c->k;
  launch(c, KC_UPDATE, [&] {
    k_nes_post<<<elem_grid(ne), 256, 0, c->stream>>>(c->F[n], c->prox[n], ne, c->lambda,
                                                     n == c->N - 1 ? c->nes_lam : nullptr, c->k);
  });
}

void normalize_gram(planc_gpu_ctx* c, int n, int next, double* lambda) {
  const int64_t I = c->dims[n];
  // one cluster launch per factor, a CTA per 64 rows (16 rows above rank 32,
  // where a row's outer product is four times the work) up to the largest
  // cluster: the size depends on I and k alone, so every context (a batch
  // member too) sums a factor's Gram in the same order, and small factors
  // take small clusters that run beside other contexts' kernels
  if (I <= NGC_MAX_ROWS && c->ngc_ctas > 0) {
    double* lam = lambda ? lambda : c->lam_tmp;
    const int64_t rpc = c->k > 32 ? 16 : NGC_TILE;
    const int cl = (int)std::min<int64_t>(c->ngc_ctas, std::max<int64_t>(1, (I + rpc - 1) / rpc));
    launch(c, KC_NORMGRAM, [&] {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)cl, 1, 1);
      cfg.blockDim = dim3(NGC_THREADS, 1, 1);
      cfg.dynamicSmemBytes = ngc_smem_bytes(c->k);
      cfg.stream = c->stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeClusterDimension;
      at[0].val.clusterDim.x = (unsigned)cl;
      at[0].val.clusterDim.y = 1;
      at[0].val.clusterDim.z = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      if (c->k <= 32)
        CK(cudaLaunchKernelEx(&cfg, k_normgram_cluster<2>, c->F[n], I, c->k, lam, c->Gall, c->N,
                              n, next, c->Gloo));
      else
        CK(cudaLaunchKernelEx(&cfg, k_normgram_cluster<4>, c->F[n], I, c->k, lam, c->Gall, c->N,
                              n, next, c->Gloo));
    });
    return;
  }
  const int rpb = gram_rows_per_block(I);
  const int nblk = (int)((I + rpb - 1) / rpb);
  if ((size_t)nblk * c->k * c->k > c->gram_part_elems)
    fail(PLANC_GPU_ERR_STATE, "internal: Gram partial buffer too small");
  launch(c, KC_NORMGRAM, [&] {
    k_gram_partial<<<nblk, 256, 0, c->stream>>>(c->F[n], I, c->k, rpb, c->gram_part);
  });
  double* lam = lambda ? lambda : c->lam_tmp;
  launch(c, KC_NORMGRAM, [&] {
    k_gram_finalize<<<1, 1024, 0, c->stream>>>(c->F[n], I, c->k, c->gram_part, nblk, lam,
                                               c->Gall, c->N, n, next, c->Gloo);
  });
  launch(c, KC_NORMGRAM, [&] {
    const int64_t ne = I * c->k;
    k_scale_cols<<<(unsigned)std::min<int64_t>((ne + 255) / 256, 2048), 256, 0, c->stream>>>(
        c->F[n], I, c->k, lam);
  });
}

void gram_loo(planc_gpu_ctx* c, int n) {
  launch(c, KC_NORMGRAM, [&] { k_gram_loo<<<1, 1024, 0, c->stream>>>(c->Gall, c->N, c->k, n, c->Gloo); });
}

// MTTKRP of the last mode from the current factors (the <X, model> term of
// the Gram-form error): through the tree from its second root (the state an
// in-order sweep leaves), or directly.
void last_mode_mttkrp(planc_gpu_ctx* c, bool dimtree) {
  const int last = c->N - 1;
  if (dimtree && (c->N == 3 || c->N == 4)) {
    dimtree_prereq(c, last);
    mttkrp_dimtree(c, last, c->M[last]);
  } else {
    mttkrp_direct(c, last, c->M[last]);
  }
}

void error_kernel(planc_gpu_ctx* c) {
  const int last = c->N - 1;
  launch(c, KC_ERROR, [&] {
    k_error<<<1, 1024, 0, c->stream>>>(c->M[last], c->F[last], c->dims[last], c->lambda, c->Gall,
                                      c->N, c->k, c->normX2, c->errs_dev, c->counter_dev);
  });
}

// NTFNES::accelerate (ntf/ntfnes.hpp:64-98) on the device, after the error
// of the iteration: extrapolate every mode from the previous iterate,
// normalise (the reference's reset(m_acc_t, true)), evaluate the error of the
// extrapolated model, then keep it (prox := it) or return to the proximal
// iterate (factors, Grams and lambda). The decision is made on the device.
void nes_accelerate(planc_gpu_ctx* c, bool dimtree) {
  if (!c->nes_ready) fail(PLANC_GPU_ERR_STATE, "internal: Nesterov state not allocated");
  const int N = c->N, k = c->k;
  double* lam_bak = c->nes_lam + 2 * k;
  launch(c, KC_UPDATE, [&] {
    k_nes_acc_begin<<<1, 256, 0, c->stream>>>(c->counter_dev, c->errs_dev, c->nes, c->lambda,
                                              lam_bak, c->Gall, c->nes_gbak, N * k * k, k);
  });
  for (int i = 0; i < N; ++i) {
    const bool last = i == N - 1;
    const int64_t ne = c->dims[i] * k;
    launch(c, KC_UPDATE, [&] {
      k_nes_extrap<<<elem_grid(ne), 256, 0, c->stream>>>(c->F[i], c->prev[i], ne, k,
                                                         last ? lam_bak : nullptr,
                                                         last ? c->nes_lam + k : nullptr, c->nes);
    });
    normalize_gram(c, i, (i + 1) % N, c->lambda);
  }
  last_mode_mttkrp(c, dimtree);
  launch(c, KC_ERROR, [&] {
    k_error<<<1, 1024, 0, c->stream>>>(c->M[N - 1], c->F[N - 1], c->dims[N - 1], c->lambda,
                                      c->Gall, N, k, c->normX2, &c->nes->acc_err,
                                      &c->nes->err_ctr);
  });
  launch(c, KC_UPDATE, [&] {
    k_nes_decide<<<1, 256, 0, c->stream>>>(c->nes, c->lambda, c->nes_lam, c->Gall, c->nes_gbak,
                                           N * k * k, c->Gall + (size_t)(N - 1) * k * k, k);
  });
  for (int i = 0; i < N; ++i) {
    const int64_t ne = c->dims[i] * k;
    launch(c, KC_UPDATE, [&] {
      k_nes_commit<<<elem_grid(ne), 256, 0, c->stream>>>(c->F[i], c->prox[i], ne, c->nes);
    });
  }
  gram_loo(c, 0);
}

// One AUNTF outer iteration (ntf/auntf.hpp:131-170); `accel` appends the
// Nesterov acceleration step (auntf.hpp:171).
void one_iteration(planc_gpu_ctx* c, int algo, bool dimtree, bool err, bool accel = false) {
  for (int n = 0; n < c->N; ++n) {
    mttkrp_any(c, n, dimtree, c->M[n]);
    run_update(c, algo, n);
    normalize_gram(c, n, (n + 1) % c->N, c->lambda);
    if (algo == PLANC_GPU_NESTEROV) nes_post(c, n);
  }
  if (err) error_kernel(c);
  if (accel) nes_accelerate(c, dimtree);
}

void require_ready(planc_gpu_ctx* c) {
  if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
  if (!c->have_tensor) fail(PLANC_GPU_ERR_STATE, "no tensor set");
  if (!c->have_factors) fail(PLANC_GPU_ERR_STATE, "no factors set");
}

void check_status(planc_gpu_ctx* c) {
  int st = 0;
  CK(cudaMemcpyAsync(&st, c->status_dev, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (st != 0) {
    CK(cudaMemsetAsync(c->status_dev, 0, sizeof(int), c->stream));
    const char* what = st == kStBppMaxIter ? "BPP failed (iteration cap 5k reached)"
                       : st == kStNonFinite ? "non-finite value in a BPP solve"
                       : st == kStSingular  ? "singular normal-equation matrix"
                       : st == kStTimeout   ? "bounded device wait timed out"
                       : st == kStMaxIter   ? "an iterative update reached its step cap"
                                            : "device status error";
    fail(st, what);
  }
}

void reset_graph(planc_gpu_ctx* c) {
  for (int v = 0; v < 2; ++v) {
    if (c->gexec[v]) {
      cudaGraphExecDestroy(c->gexec[v]);
      c->gexec[v] = nullptr;
    }
    c->g_algo[v] = c->g_dimtree[v] = c->g_err[v] = -1;
  }
}

void free_update_state(planc_gpu_ctx* c) {
  reset_graph(c);
  auto f = [](auto*& p) {
    if (p) cudaFree(p);
    p = nullptr;
  };
  for (int n = 0; n < kMaxModes; ++n) {
    f(c->aux[n]);
    f(c->prox[n]);
    f(c->prev[n]);
  }
  f(c->admm_L);
  f(c->admm_scal);
  f(c->admm_flag);
  f(c->admm_part);
  c->admm_part_elems = 0;
  f(c->nes_acc);
  f(c->nes_grad);
  f(c->nes_modM);
  f(c->nes_lam);
  f(c->nes_gbak);
  f(c->nes);
  c->admm_ready = c->nes_ready = false;
  if (c->nmf_gexec) cudaGraphExecDestroy(c->nmf_gexec);
  c->nmf_gexec = nullptr;
  c->nmf_galgo = -1;
  f(c->nmf_G);
  f(c->nmf_GW);
  f(c->nmf_GH);
  f(c->nmf_norms);
  f(c->nmf_part);
  c->nmf_part_elems = 0;
  f(c->nmf_ctr);
  f(c->nmf_obj);
  f(c->nmf_rel);
  c->nmf_cap = 0;
  c->nmf_ready = false;
}

// Allocates (zeroed) the solver-object state of `algo` if it is not there:
// the reference's constructors zero m_ncp_aux (ntfaoadmm.hpp:86) and
// m_prox_t / m_prev_t / m_acc_t / m_grad_t (ntfnes.hpp:179-182), set the
// NCPFactors lambdas to ones and acc_exp = 3, acc_fails = 0
// (ntfnes.hpp:186-189). Called outside stream capture.
void ensure_update_state(planc_gpu_ctx* c, int algo) {
  if ((algo == PLANC_GPU_AOADMM || algo == PLANC_GPU_NESTEROV) && !c->admm_ready &&
      !c->nes_ready) {
    // clusters of 16 where every register-resident kernel accepts them
    bool ok = true;
    ok = ok && enable_cluster16(k_admm_cluster<32, 1>) && enable_cluster16(k_admm_cluster<32, 2>);
    ok = ok && enable_cluster16(k_admm_cluster<32, 4>) && enable_cluster16(k_admm_cluster<32, 8>);
    ok = ok && enable_cluster16(k_admm_cluster<64, 1>) && enable_cluster16(k_admm_cluster<64, 2>);
    ok = ok && enable_cluster16(k_admm_cluster<64, 4>);
    ok = ok && enable_cluster16(k_nes_inner_reg<32, 1>) && enable_cluster16(k_nes_inner_reg<32, 2>);
    ok = ok && enable_cluster16(k_nes_inner_reg<32, 4>) && enable_cluster16(k_nes_inner_reg<32, 8>);
    ok = ok && enable_cluster16(k_nes_inner_reg<64, 1>) && enable_cluster16(k_nes_inner_reg<64, 2>);
    ok = ok && enable_cluster16(k_nes_inner_reg<64, 4>);
    c->cl_ctas = ok ? NES_CTAS_MAX : NES_CTAS;
  }
  const int k = c->k;
  int64_t maxI = 1;
  for (int n = 0; n < c->N; ++n) maxI = std::max(maxI, c->dims[n]);
  if (algo == PLANC_GPU_AOADMM && !c->admm_ready) {
    for (int n = 0; n < c->N; ++n) {
      dalloc(&c->aux[n], (size_t)c->dims[n] * k);
      CK(cudaMemsetAsync(c->aux[n], 0, (size_t)c->dims[n] * k * 8, c->stream));
    }
    dalloc(&c->admm_L, (size_t)k * k);
    dalloc(&c->admm_scal, 4);
    dalloc(&c->admm_flag, 2);
    CK(cudaMemsetAsync(c->admm_flag, 0, 2 * sizeof(int), c->stream));
    c->admm_part_elems =
        std::max<size_t>((size_t)ADMM_MAX_BLOCKS * 4, (size_t)((maxI + CN_ROWS - 1) / CN_ROWS) * k);
    dalloc(&c->admm_part, c->admm_part_elems);
    c->admm_ready = true;
    c->buf_epoch++;
  }
  if (algo == PLANC_GPU_NESTEROV && !c->nes_ready) {
    for (int n = 0; n < c->N; ++n) {
      dalloc(&c->prox[n], (size_t)c->dims[n] * k);
      dalloc(&c->prev[n], (size_t)c->dims[n] * k);
      CK(cudaMemsetAsync(c->prox[n], 0, (size_t)c->dims[n] * k * 8, c->stream));
      CK(cudaMemsetAsync(c->prev[n], 0, (size_t)c->dims[n] * k * 8, c->stream));
    }
    dalloc(&c->nes_acc, (size_t)maxI * k);
    dalloc(&c->nes_grad, (size_t)maxI * k);
    dalloc(&c->nes_modM, (size_t)maxI * k);
    dalloc(&c->nes_lam, (size_t)3 * k);
    std::vector<double> ones((size_t)3 * k, 1.0);
    CK(cudaMemcpyAsync(c->nes_lam, ones.data(), ones.size() * 8, cudaMemcpyHostToDevice, c->stream));
    dalloc(&c->nes_gbak, (size_t)c->N * k * k);
    dalloc(&c->nes, 1);
    NesDev init{};
    init.acc_exp = 3;
    CK(cudaMemcpyAsync(c->nes, &init, sizeof(NesDev), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->nes_ready = true;
    c->buf_epoch++;
  }
}

void free_all(planc_gpu_ctx* c) {
  free_update_state(c);
  auto f = [](auto*& p) {
    if (p) cudaFree(p);
    p = nullptr;
  };
  f(c->X64);
  c->x64_elems = 0;
  if (c->stage) cudaFree(c->stage);
  c->stage = nullptr;
  f(c->cp_part);
  if (c->cp_ctr) cudaFree(c->cp_ctr);
  c->cp_ctr = nullptr;
  f(c->norm_part);
  tc_free(c->tct);
  for (int n = 0; n < kMaxModes; ++n) tc_free(c->tcd[n]);
  f(c->ones_k);
  f(c->krp_tail);
  c->krp_tail_elems = 0;
  f(c->normX2);
  for (int n = 0; n < kMaxModes; ++n) {
    f(c->F[n]);
    f(c->M[n]);
    c->factor_cap[n] = 0;
  }
  f(c->Gall);
  f(c->gram_part);
  f(c->lam_tmp);
  c->gram_part_elems = 0;
  f(c->Gloo);
  f(c->lambda);
  f(c->P);
  f(c->P32);
  f(c->Q);
  f(c->scratch);
  c->scratch_elems = 0;
  f(c->errs_dev);
  c->errs_cap = 0;
  f(c->counter_dev);
  f(c->status_dev);
}

}  // namespace

// ===================================================================== ABI
extern "C" {

int planc_gpu_abi_version(void) { return PLANC_GPU_ABI_VERSION; }

const char* planc_gpu_last_error(void) { return g_last_error.c_str(); }

int planc_gpu_create(planc_gpu_ctx** out, int device, int precision, void* cuda_stream) {
  return guarded([&] {
    if (!out) fail(PLANC_GPU_ERR_ARG, "out is null");
    *out = nullptr;
    if (precision < PLANC_GPU_PREC_FP64 || precision > PLANC_GPU_PREC_BF16X2)
      fail(PLANC_GPU_ERR_ARG, "unknown precision " + std::to_string(precision));
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) fail(PLANC_GPU_ERR_ARG, "bad device index");
    CK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (precision != PLANC_GPU_PREC_FP64 && prop.major < 10)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "tensor-core precisions need an sm_100 device");
    {
      // k_bpp<64> needs more than the default 48 KB of dynamic shared memory
      static bool attrs_set[64] = {false};
      if (device < 64 && !attrs_set[device]) {
        CK(cudaFuncSetAttribute(k_bpp<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bpp_smem_bytes(64)));
        CK(cudaFuncSetAttribute(k_bpp<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)bpp_smem_bytes(32)));
        contract_f64_attrs(device);
        CK(cudaFuncSetAttribute(k_bpp_cta<64, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)BppCta<64, 8>::SMEM));
        CK(cudaFuncSetAttribute(k_bpp_cta<32, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)BppCta<32, 8>::SMEM));
        // the opt-in limit covers static and dynamic shared memory together
        CK(cudaFuncSetAttribute(k_nmf_hals_w_coop<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)nmfc_smem_limit(prop.sharedMemPerBlockOptin)));
        CK(cudaFuncSetAttribute(k_nmf_hals_w_coop<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)nmfc_smem_limit(prop.sharedMemPerBlockOptin)));
        attrs_set[device] = true;
      }
    }
    planc_gpu_ctx* c = new planc_gpu_ctx();
    c->device = device;
    c->precision = precision;
    c->sm_count = prop.multiProcessorCount;
    c->smem_optin = nmfc_smem_limit(prop.sharedMemPerBlockOptin);
    c->ngc_ctas = ngc_cluster_size();
    // PLANC_GPU_NES_MAX_STEPS lowers the Nesterov inner loop's step cap for
    // contexts created while it is set (1 .. NES_MAX_STEPS)
    if (const char* e = getenv("PLANC_GPU_NES_MAX_STEPS")) {
      const int v = atoi(e);
      if (v >= 1 && v <= NES_MAX_STEPS) c->nes_max_steps = v;
    }
    // PLANC_GPU_LEFT_CHUNKS=n: fewest chunks per split-K partial of the
    // tensor-core left contraction for contexts created while it is set
    if (const char* e = getenv("PLANC_GPU_LEFT_CHUNKS")) {
      const int v = atoi(e);
      if (v >= 0 && v <= (1 << 20)) c->left_chunks = v;
    }
    // PLANC_GPU_LEFT_FORM=image|producers picks how a 3-way tensor-core left
    // contraction without the factored form forms its Khatri-Rao rows, for
    // contexts created while it is set
    if (const char* e = getenv("PLANC_GPU_LEFT_FORM")) {
      if (!strcmp(e, "producers")) c->left_long = false;
      if (!strcmp(e, "image")) c->left_long = true;
    }
    // PLANC_GPU_LEFT_PARTS=n splits each run of the factored left
    // contraction into n work units (a divisor of I0 / 64) for contexts
    // created while it is set
    if (const char* e = getenv("PLANC_GPU_LEFT_PARTS")) {
      const int v = atoi(e);
      if (v >= 1 && v <= 1024) c->left_parts = v;
    }
    // PLANC_GPU_TC_LOADS=tma|cpasync picks how the tensor-core right and
    // factored left contractions fetch their tensor tiles, for contexts
    // created while it is set
    if (const char* e = getenv("PLANC_GPU_TC_LOADS")) {
      if (!strcmp(e, "tma")) c->tc_cpa = false;
      if (!strcmp(e, "cpasync")) c->tc_cpa = true;
    }
    // PLANC_GPU_BPP_KERNEL=warp|cta fixes the batched BPP kernel for contexts
    // created while it is set (default: chosen by the number of right-hand sides)
    if (const char* e = getenv("PLANC_GPU_BPP_KERNEL")) {
      if (!strcmp(e, "warp")) c->bpp_kernel = 1;
      if (!strcmp(e, "cta")) c->bpp_kernel = 2;
    }
    c->coop_launch = prop.cooperativeLaunch != 0;
    if (cuda_stream) {
      c->stream = (cudaStream_t)cuda_stream;
    } else {
      cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) {
        delete c;
        cuda_check(e, "cudaStreamCreateWithFlags");
      }
      c->own_stream = true;
    }
    try {
      CK(cudaMalloc(&c->normX2, sizeof(double)));
      CK(cudaMalloc(&c->counter_dev, sizeof(int)));
      CK(cudaMalloc(&c->status_dev, sizeof(int)));
      CK(cudaMemsetAsync(c->status_dev, 0, sizeof(int), c->stream));
    } catch (...) {
      free_all(c);
      if (c->own_stream) cudaStreamDestroy(c->stream);
      delete c;
      throw;
    }
    *out = c;
  });
}

int planc_gpu_destroy(planc_gpu_ctx* c) {
  if (!c) return PLANC_GPU_OK;
  return guarded([&] {
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& p : c->pending) {
      cudaEventDestroy(p.a);
      cudaEventDestroy(p.b);
    }
    for (auto e : c->ev_pool) cudaEventDestroy(e);
    free_all(c);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
  });
}

void* planc_gpu_stream(planc_gpu_ctx* c) { return c ? (void*)c->stream : nullptr; }

int planc_gpu_set_tensor(planc_gpu_ctx* c, const void* X, int dtype, const int64_t* dims,
                         int nmodes, int x_on_device) {
  return guarded([&] {
    if (!c || !X || !dims) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (nmodes < 2 || nmodes > kMaxModes)
      fail(PLANC_GPU_ERR_ARG, "nmodes must be in [2, " + std::to_string(kMaxModes) + "]");
    if (dtype != PLANC_GPU_F64 && dtype != PLANC_GPU_F32) fail(PLANC_GPU_ERR_ARG, "bad dtype");
    int64_t numel = 1;
    for (int i = 0; i < nmodes; ++i) {
      if (dims[i] < 1) fail(PLANC_GPU_ERR_ARG, "every mode size must be >= 1");
      numel *= dims[i];
    }
    set_device(c);
    reset_graph(c);
    // drop everything shaped by the previous tensor
    bool same = c->have_tensor && c->N == nmodes;
    for (int i = 0; same && i < nmodes; ++i) same = c->dims[i] == dims[i];
    if (!same) {
      c->have_factors = false;
      c->nmf_have = false;
      free_update_state(c);
      auto f = [](auto*& p) {
        if (p) cudaFree(p);
        p = nullptr;
      };
      f(c->P);
      f(c->P32);
      f(c->Q);
    }
    c->N = nmodes;
    for (int i = 0; i < nmodes; ++i) c->dims[i] = dims[i];
    c->numel = numel;
    c->s = nmodes / 2;  // ntf/auntf.hpp:122-123
    // a matrix (NMF): rows = mode 0 (L), columns = mode 1 (R)
    if (nmodes == 2) c->s = 0;
    // no tree above four modes: the tensor-core copy splits before the last
    // mode, whose direct MTTKRP it then serves as is
    if (nmodes > 4 && c->precision != PLANC_GPU_PREC_FP64) c->s = nmodes - 2;
    for (int n = 0; n < kMaxModes; ++n) tc_free(c->tcd[n]);
    // PLANC_GPU_DIMTREE_SPLIT=reference keeps the reference's split everywhere
    const char* split_env = getenv("PLANC_GPU_DIMTREE_SPLIT");
    const bool ref_split = split_env && strcmp(split_env, "reference") == 0;
    c->bal4 = !ref_split && nmodes == 4 && c->precision != PLANC_GPU_PREC_FP64 &&
              std::max(dims[0] * dims[1], dims[2] * dims[3]) <= kBal4MaxK;
    if (c->bal4) c->s = 1;
    c->L = 1;
    c->R = 1;
    for (int i = 0; i < nmodes; ++i) (i <= c->s ? c->L : c->R) *= dims[i];
    c->have_tensor = false;  // until the new tensor is in place
    const size_t esz = dtype == PLANC_GPU_F64 ? 8 : 4;
    // The tensor goes through in chunks of the natural order: from host memory
    // through one fixed staging buffer (no allocation per call), from device
    // memory in place. Each chunk adds its FP64 sum of squares (in a fixed
    // order, the same for both sources) and is converted into the resident
    // copy: FP64, or the tensor-core view (BF16 or a BF16 pair).
    const int64_t chunk = kStageBytes / (int64_t)esz;
    const bool f64 = c->precision == PLANC_GPU_PREC_FP64;
    if (!x_on_device && !c->stage) CK(cudaMalloc(&c->stage, kStageBytes));
    if (!c->norm_part) CK(cudaMalloc(&c->norm_part, kNormBlocks * sizeof(double)));
    if (f64) {
      if (!c->X64 || c->x64_elems != numel) {
        dalloc(&c->X64, (size_t)numel);
        c->x64_elems = numel;
      }
      tc_free(c->tct);
    } else {
      if (c->X64) {
        cudaFree(c->X64);
        c->X64 = nullptr;
        c->x64_elems = 0;
      }
      CK(tc_prepare(c->tct, c->L, c->R, c->dims[0], c->precision));
      c->tct.left_parts = c->left_parts > 0 ? c->left_parts : 1;
      c->tct.left_cpa = c->tc_cpa;
    }
    for (int64_t e0 = 0; e0 < numel; e0 += chunk) {
      const int64_t n = std::min<int64_t>(chunk, numel - e0);
      const char* src = (const char*)X + (size_t)e0 * esz;
      if (!x_on_device) {
        if (f64 && dtype == PLANC_GPU_F64) {  // straight into the resident copy
          CK(cudaMemcpyAsync(c->X64 + e0, src, n * esz, cudaMemcpyHostToDevice, c->stream));
          src = (const char*)(c->X64 + e0);
        } else {
          CK(cudaMemcpyAsync(c->stage, src, n * esz, cudaMemcpyHostToDevice, c->stream));
          src = (const char*)c->stage;
        }
      }
      const unsigned nb = (unsigned)std::min<int64_t>(kNormBlocks, (n + 255) / 256);
      if (dtype == PLANC_GPU_F64)
        k_sumsq_partial<double><<<nb, 256, 0, c->stream>>>((const double*)src, n, c->norm_part);
      else
        k_sumsq_partial<float><<<nb, 256, 0, c->stream>>>((const float*)src, n, c->norm_part);
      k_accum_norm<<<1, 32, 0, c->stream>>>(c->norm_part, (int)nb, c->normX2, e0 == 0);
      const unsigned cb = (unsigned)std::min<int64_t>(4096, (n + 255) / 256);
      if (f64) {
        if (dtype == PLANC_GPU_F64) {
          if ((const double*)src != c->X64 + e0)
            CK(cudaMemcpyAsync(c->X64 + e0, src, n * 8, cudaMemcpyDeviceToDevice, c->stream));
        } else {
          k_copy_to_f64<float><<<cb, 256, 0, c->stream>>>((const float*)src, n, c->X64 + e0);
        }
      } else if (dtype == PLANC_GPU_F64) {
        k_tc_convert_range<double><<<cb, 256, 0, c->stream>>>((const double*)src, e0, n, c->L,
                                                              c->tct.Lpad, c->tct.hi, c->tct.lo);
      } else {
        k_tc_convert_range<float><<<cb, 256, 0, c->stream>>>((const float*)src, e0, n, c->L,
                                                             c->tct.Lpad, c->tct.hi, c->tct.lo);
      }
      CK(cudaGetLastError());
    }
    if (!f64) {
      if (!tc_make_maps(c->tct))
        fail(PLANC_GPU_ERR_CUDA, "cuTensorMapEncodeTiled rejected the tensor map");
      c->tct.left_nf = tc_left_gen_nf(c->s + 1);
    }
    double nx = 0.0;
    CK(cudaMemcpyAsync(&nx, c->normX2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (!std::isfinite(nx)) {
      c->have_tensor = false;
      fail(PLANC_GPU_ERR_NONFINITE, "the tensor holds NaN or Inf values");
    }
    c->have_tensor = true;
  });
}

int planc_gpu_set_factors(planc_gpu_ctx* c, const double* const* F, const double* lambda, int k) {
  return guarded([&] {
    if (!c || !F) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (!c->have_tensor) fail(PLANC_GPU_ERR_STATE, "set the tensor before the factors");
    if (k < 1 || k > kMaxRank)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "rank must be in [1, " + std::to_string(kMaxRank) + "]");
    set_device(c);
    // Cached iteration graphs stay valid when no buffer moves: the new
    // factors are copied into the same device arrays. Any reallocation below
    // bumps the buffer epoch, which rebuilds the graphs before their next use.
    if (k != c->k) {
      reset_graph(c);
      free_update_state(c);
      auto f = [](auto*& p) {
        if (p) cudaFree(p);
        p = nullptr;
      };
      f(c->P);
      f(c->P32);
      f(c->Q);
      for (int n = 0; n < kMaxModes; ++n) c->factor_cap[n] = 0;
    }
    c->k = k;
    for (int n = 0; n < c->N; ++n) {
      if (!F[n]) fail(PLANC_GPU_ERR_ARG, "null factor");
      size_t need = (size_t)c->dims[n] * k;
      if (c->factor_cap[n] != (int64_t)need) {
        dalloc(&c->F[n], need);
        dalloc(&c->M[n], need);
        c->factor_cap[n] = (int64_t)need;
        c->buf_epoch++;
      }
      CK(cudaMemcpyAsync(c->F[n], F[n], need * 8, cudaMemcpyHostToDevice, c->stream));
    }
    if (!c->Gall || c->gall_elems != (size_t)c->N * k * k) {
      c->gall_elems = (size_t)c->N * k * k;
      dalloc(&c->Gall, c->gall_elems);
      c->buf_epoch++;
    }
    {
      int64_t maxI = 1;
      for (int n = 0; n < c->N; ++n) maxI = std::max(maxI, c->dims[n]);
      const size_t gp = (size_t)((maxI + GP_ROWS - 1) / GP_ROWS) * k * k;
      if (!c->gram_part || c->gram_part_elems < gp) {
        c->gram_part_elems = gp;
        dalloc(&c->gram_part, c->gram_part_elems);
        c->buf_epoch++;
      }
    }
    if (!c->Gloo || c->kvec != k) {
      dalloc(&c->Gloo, (size_t)k * k);
      dalloc(&c->lambda, (size_t)k);
      dalloc(&c->lam_tmp, (size_t)k);
      c->kvec = k;
      c->buf_epoch++;
    }
    // AUNTF::reset: update_factor_mode on every mode (normalise, Gram), then
    // set_lambda(new lambda)
    for (int n = 0; n < c->N; ++n) normalize_gram(c, n, n == c->N - 1 ? 0 : -1, c->lambda);
    std::vector<double> lam(k, 1.0);
    if (lambda) std::copy(lambda, lambda + k, lam.begin());
    CK(cudaMemcpyAsync(c->lambda, lam.data(), k * 8, cudaMemcpyHostToDevice, c->stream));
    ensure_buffers(c);
    CK(cudaStreamSynchronize(c->stream));
    c->have_factors = true;
    c->nmf_have = false;
  });
}

}  // extern "C"

namespace {

bool known_algo(int algo) {
  return algo == PLANC_GPU_MU || algo == PLANC_GPU_HALS || algo == PLANC_GPU_ANLSBPP ||
         algo == PLANC_GPU_AOADMM || algo == PLANC_GPU_NESTEROV;
}

// Captures (once) and returns the graph of one iteration; variant 1 appends
// the Nesterov acceleration.
cudaGraphExec_t iteration_graph(planc_gpu_ctx* c, int algo, bool dt, bool err, int variant) {
  if (c->gexec[variant] && c->g_algo[variant] == algo && c->g_dimtree[variant] == (int)dt &&
      c->g_err[variant] == (int)err)
    return c->gexec[variant];
  if (c->gexec[variant]) {
    cudaGraphExecDestroy(c->gexec[variant]);
    c->gexec[variant] = nullptr;
  }
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  c->capturing = true;
  try {
    one_iteration(c, algo, dt, err, variant == 1);
  } catch (...) {
    c->capturing = false;
    cudaStreamEndCapture(c->stream, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  c->capturing = false;
  CK(cudaStreamEndCapture(c->stream, &graph));
  cudaError_t e = cudaGraphInstantiate(&c->gexec[variant], graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(e, "cudaGraphInstantiate");
  c->g_algo[variant] = algo;
  c->g_dimtree[variant] = (int)dt;
  c->g_err[variant] = (int)err;
  return c->gexec[variant];
}

}  // namespace

extern "C" {

int planc_gpu_run(planc_gpu_ctx* c, int algo, int iters, int dimtree, int compute_error,
                  double* errs_out) {
  return guarded([&] {
    require_ready(c);
    if (iters < 0) fail(PLANC_GPU_ERR_ARG, "iters < 0");
    if (!known_algo(algo)) fail(PLANC_GPU_ERR_ARG, "unknown algorithm " + std::to_string(algo));
    bool dt = dimtree && (c->N == 3 || c->N == 4);
    if (iters == 0) return;
    set_device(c);
    ensure_buffers(c);
    if (!dt) ensure_direct(c);
    // NTFNES evaluates the error every iteration (accelerated(true),
    // ntf/ntfnes.hpp:193): its acceleration compares against it
    const bool nes = algo == PLANC_GPU_NESTEROV;
    const bool err = compute_error != 0 || nes;
    ensure_errs(c, err ? iters : 1);
    ensure_update_state(c, algo);
    if (c->g_epoch != c->buf_epoch) reset_graph(c);
    CK(cudaMemsetAsync(c->counter_dev, 0, sizeof(int), c->stream));
    gram_loo(c, 0);
    bool use_graph = !c->timing;
    // AUNTF::computeNTF restarts its iteration count at 0 on every call and
    // NTFNES accelerates from iteration acc_start + 1 = 6 on
    // (ntf/auntf.hpp:129, ntf/ntfnes.hpp:65)
    auto accel_at = [&](int it) { return nes && it > 5; };
    if (use_graph) {
      for (int it = 0; it < iters; ++it)
        CK(cudaGraphLaunch(iteration_graph(c, algo, dt, err, accel_at(it) ? 1 : 0), c->stream));
      c->g_epoch = c->buf_epoch;
    } else {
      for (int it = 0; it < iters; ++it) one_iteration(c, algo, dt, err, accel_at(it));
    }
    if (compute_error && errs_out)
      CK(cudaMemcpyAsync(errs_out, c->errs_dev, iters * sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
    check_status(c);
    drain_timing(c);
  });
}

int planc_gpu_get_factors(planc_gpu_ctx* c, double* const* F, double* lambda) {
  return guarded([&] {
    require_ready(c);
    set_device(c);
    if (F)
      for (int n = 0; n < c->N; ++n)
        if (F[n])
          CK(cudaMemcpyAsync(F[n], c->F[n], (size_t)c->dims[n] * c->k * 8, cudaMemcpyDeviceToHost,
                             c->stream));
    if (lambda)
      CK(cudaMemcpyAsync(lambda, c->lambda, c->k * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int planc_gpu_mttkrp(planc_gpu_ctx* c, int mode, int dimtree, double* out) {
  return guarded([&] {
    require_ready(c);
    if (mode < 0 || mode >= c->N || !out) fail(PLANC_GPU_ERR_ARG, "bad mode or null output");
    set_device(c);
    ensure_buffers(c);
    bool dt = dimtree && (c->N == 3 || c->N == 4);
    if (!dt) ensure_direct(c);
    if (dt) {
      // the tree state for `mode` comes from the current factors
      dimtree_prereq(c, mode);
      mttkrp_dimtree(c, mode, c->M[mode]);
    } else {
      mttkrp_direct(c, mode, c->M[mode]);
    }
    CK(cudaMemcpyAsync(out, c->M[mode], (size_t)c->dims[mode] * c->k * 8, cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    drain_timing(c);
  });
}

int planc_gpu_gram_loo(planc_gpu_ctx* c, int mode, double* out) {
  return guarded([&] {
    require_ready(c);
    if (mode < 0 || mode >= c->N || !out) fail(PLANC_GPU_ERR_ARG, "bad mode or null output");
    set_device(c);
    gram_loo(c, mode);
    CK(cudaMemcpyAsync(out, c->Gloo, (size_t)c->k * c->k * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int planc_gpu_objective_error(planc_gpu_ctx* c, double* err) {
  return guarded([&] {
    require_ready(c);
    if (!err) fail(PLANC_GPU_ERR_ARG, "null output");
    set_device(c);
    ensure_buffers(c);
    ensure_errs(c, 1);
    // <X, model> needs the MTTKRP of the last mode from the current factors:
    // directly on the FP64 tensor, through the tree on the tensor-core copy
    // (whose 4-way form is the balanced tree)
    const bool tree = c->precision != PLANC_GPU_PREC_FP64 && (c->N == 3 || c->N == 4);
    if (c->precision != PLANC_GPU_PREC_FP64 && !tree) ensure_direct(c);
    last_mode_mttkrp(c, tree);
    CK(cudaMemsetAsync(c->counter_dev, 0, sizeof(int), c->stream));
    error_kernel(c);
    CK(cudaMemcpyAsync(err, c->errs_dev, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    drain_timing(c);
  });
}

int planc_gpu_mode_begin(planc_gpu_ctx* c, int mode, int dimtree, double* gram_out,
                         double* mttkrp_out) {
  return guarded([&] {
    require_ready(c);
    if (mode < 0 || mode >= c->N) fail(PLANC_GPU_ERR_ARG, "bad mode");
    set_device(c);
    ensure_buffers(c);
    bool dt = dimtree && (c->N == 3 || c->N == 4);
    if (!dt) ensure_direct(c);
    gram_loo(c, mode);
    mttkrp_any(c, mode, dt, c->M[mode]);
    if (gram_out)
      CK(cudaMemcpyAsync(gram_out, c->Gloo, (size_t)c->k * c->k * 8, cudaMemcpyDeviceToHost,
                         c->stream));
    if (mttkrp_out)
      CK(cudaMemcpyAsync(mttkrp_out, c->M[mode], (size_t)c->dims[mode] * c->k * 8,
                         cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int planc_gpu_mode_end(planc_gpu_ctx* c, int mode, const double* factor) {
  return guarded([&] {
    require_ready(c);
    if (mode < 0 || mode >= c->N || !factor) fail(PLANC_GPU_ERR_ARG, "bad mode or null factor");
    set_device(c);
    reset_graph(c);
    CK(cudaMemcpyAsync(c->F[mode], factor, (size_t)c->dims[mode] * c->k * 8,
                       cudaMemcpyHostToDevice, c->stream));
    normalize_gram(c, mode, (mode + 1) % c->N, c->lambda);
    CK(cudaStreamSynchronize(c->stream));
  });
}

int planc_gpu_bpp_solve(planc_gpu_ctx* c, const double* AtA, const double* AtB, int n,
                        int64_t ncols, double* X, int32_t* passive, int32_t* iters) {
  return guarded([&] {
    if (!c || !AtA || !AtB || !X) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (n < 1 || n > kMaxRank) fail(PLANC_GPU_ERR_UNSUPPORTED, "n must be in [1, 64]");
    if (ncols < 0) fail(PLANC_GPU_ERR_ARG, "ncols < 0");
    if (ncols == 0) return;
    set_device(c);
    double *dA = nullptr, *dB = nullptr, *dX = nullptr;
    int *dP = nullptr, *dI = nullptr;
    auto cleanup = [&] {
      cudaFree(dA);
      cudaFree(dB);
      cudaFree(dX);
      cudaFree(dP);
      cudaFree(dI);
    };
    try {
      CK(cudaMalloc(&dA, (size_t)n * n * 8));
      CK(cudaMalloc(&dB, (size_t)n * ncols * 8));
      CK(cudaMalloc(&dX, (size_t)n * ncols * 8));
      CK(cudaMalloc(&dP, (size_t)n * ncols * 4));
      CK(cudaMalloc(&dI, (size_t)ncols * 4));
      CK(cudaMemcpyAsync(dA, AtA, (size_t)n * n * 8, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(dB, AtB, (size_t)n * ncols * 8, cudaMemcpyHostToDevice, c->stream));
      launch(c, KC_BPP, [&] { launch_bpp(c, dA, dB, n, ncols, dX, dP, dI, nullptr); });
      CK(cudaMemcpyAsync(X, dX, (size_t)n * ncols * 8, cudaMemcpyDeviceToHost, c->stream));
      if (passive)
        CK(cudaMemcpyAsync(passive, dP, (size_t)n * ncols * 4, cudaMemcpyDeviceToHost, c->stream));
      if (iters) CK(cudaMemcpyAsync(iters, dI, (size_t)ncols * 4, cudaMemcpyDeviceToHost, c->stream));
      check_status(c);
      drain_timing(c);
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

// ---- device building blocks of the distributed iteration
int planc_gpu_update_device(planc_gpu_ctx* c, int algo, double* H, const double* M,
                            const double* G, int64_t rows, int k) {
  return guarded([&] {
    if (!c || !H || !M || !G) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (rows < 0 || k < 1 || k > kMaxRank) fail(PLANC_GPU_ERR_ARG, "bad shape");
    if (algo != PLANC_GPU_HALS && algo != PLANC_GPU_MU && algo != PLANC_GPU_ANLSBPP)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "row-block updates are MU, HALS and ANLS/BPP");
    if (rows == 0) return;
    set_device(c);
    const unsigned blocks = (unsigned)((rows + 7) / 8);
    if (algo == PLANC_GPU_HALS || algo == PLANC_GPU_MU) {
      launch(c, KC_UPDATE, [&] {
        if (k <= 32) {
          if (algo == PLANC_GPU_HALS)
            k_hals_warp<32><<<blocks, 256, 0, c->stream>>>(H, M, G, rows, k);
          else
            k_mu_warp<32><<<blocks, 256, 0, c->stream>>>(H, M, G, rows, k, kEps6);
        } else {
          if (algo == PLANC_GPU_HALS)
            k_hals_warp<64><<<blocks, 256, 0, c->stream>>>(H, M, G, rows, k);
          else
            k_mu_warp<64><<<blocks, 256, 0, c->stream>>>(H, M, G, rows, k, kEps6);
        }
      });
      return;
    }
    launch(c, KC_BPP, [&] {
      launch_bpp(c, G, M, k, rows, H, nullptr, nullptr, c->bpp_warm ? H : nullptr);
    });
  });
}

int planc_gpu_gram_device(planc_gpu_ctx* c, const double* F, int64_t rows, int k, double* G) {
  return guarded([&] {
    if (!c || !F || !G) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (rows < 0 || k < 1 || k > kMaxRank) fail(PLANC_GPU_ERR_ARG, "bad shape");
    set_device(c);
    if (rows == 0) {
      CK(cudaMemsetAsync(G, 0, (size_t)k * k * 8, c->stream));
      return;
    }
    const int rpb = gram_rows_per_block(rows);
    const int nblk = (int)((rows + rpb - 1) / rpb);
    if ((size_t)nblk * k * k > c->gram_part_elems) {
      if (c->capturing) fail(PLANC_GPU_ERR_STATE, "Gram partials would grow during capture");
      dalloc(&c->gram_part, (size_t)nblk * k * k);
      c->gram_part_elems = (size_t)nblk * k * k;
      c->buf_epoch++;
    }
    launch(c, KC_NORMGRAM, [&] {
      k_gram_partial<<<nblk, 256, 0, c->stream>>>(F, rows, k, rpb, c->gram_part);
    });
    launch(c, KC_REDUCE, [&] {
      reduce_splits(c->stream, c->gram_part, nblk, (int64_t)k * k, (int64_t)k * k, G);
    });
  });
}

int planc_gpu_normalize_device(planc_gpu_ctx* c, double* F, int64_t rows, int k,
                               const double* G_in, double* lambda, double* G_out) {
  return guarded([&] {
    if (!c || !G_in || !lambda || !G_out || (rows > 0 && !F)) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (rows < 0 || k < 1 || k > kMaxRank) fail(PLANC_GPU_ERR_ARG, "bad shape");
    set_device(c);
    launch(c, KC_NORMGRAM, [&] { k_norm_from_gram<<<1, 1024, 0, c->stream>>>(G_in, k, lambda, G_out); });
    if (rows > 0) {
      const unsigned nb = (unsigned)std::min<int64_t>((rows * k + 255) / 256, 4096);
      launch(c, KC_NORMGRAM, [&] { k_scale_cols<<<nb, 256, 0, c->stream>>>(F, rows, k, lambda); });
    }
  });
}

int planc_gpu_coldot_device(planc_gpu_ctx* c, const double* A, const double* B, int64_t rows, int k,
                            double* out) {
  return guarded([&] {
    if (!c || !out || (rows > 0 && (!A || !B))) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (rows < 0 || k < 1 || k > kMaxRank) fail(PLANC_GPU_ERR_ARG, "bad shape");
    set_device(c);
    launch(c, KC_ERROR, [&] { k_coldot<<<1, 1024, 0, c->stream>>>(A, B, rows, k, out); });
  });
}

int planc_gpu_sync(planc_gpu_ctx* c) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    set_device(c);
    CK(cudaStreamSynchronize(c->stream));
    check_status(c);
    drain_timing(c);
  });
}

// ---- the differentiable CP loss
namespace {
CpFactors cp_factors(planc_gpu_ctx* c, const double* const* F) {
  CpFactors f;
  memset(&f, 0, sizeof(f));
  f.N = c->N;
  f.k = c->k;
  for (int n = 0; n < c->N; ++n) {
    if (!F[n]) fail(PLANC_GPU_ERR_ARG, "null factor");
    f.F[n] = F[n];
    f.I[n] = c->dims[n];
  }
  return f;
}
}  // namespace

int planc_gpu_cp_loss_device(planc_gpu_ctx* c, const double* const* F_dev, const double* M0_dev,
                             double* G_out, double* loss_out) {
  return guarded([&] {
    require_ready(c);
    if (!F_dev || !M0_dev || !G_out || !loss_out) fail(PLANC_GPU_ERR_ARG, "null argument");
    set_device(c);
    CpFactors f = cp_factors(c, F_dev);
    const int k = c->k;
    if (!c->cp_part) {
      if (c->capturing) fail(PLANC_GPU_ERR_STATE, "CP-loss buffers would be made during capture");
      CK(cudaMalloc(&c->cp_part, (size_t)kMaxModes * CPG_BLOCKS * kMaxRank * kMaxRank * 8));
      CK(cudaMalloc(&c->cp_ctr, kMaxModes * sizeof(unsigned)));
      CK(cudaMemsetAsync(c->cp_ctr, 0, kMaxModes * sizeof(unsigned), c->stream));
    }
    launch(c, KC_NORMGRAM, [&] {
      k_cp_grams<<<dim3(CPG_BLOCKS, c->N), 256, 0, c->stream>>>(f, c->cp_part, G_out, c->cp_ctr);
    });
    launch(c, KC_ERROR, [&] {
      k_cp_loss<<<1, 1024, 0, c->stream>>>(M0_dev, F_dev[0], c->dims[0], G_out, c->N, k, c->normX2,
                                            loss_out);
    });
  });
}

int planc_gpu_cp_grads_device(planc_gpu_ctx* c, const double* const* F_dev, const double* G,
                              const double* const* M_dev, const double* g_dev,
                              double* const* grad_dev) {
  return guarded([&] {
    require_ready(c);
    if (!F_dev || !G || !M_dev || !g_dev || !grad_dev) fail(PLANC_GPU_ERR_ARG, "null argument");
    set_device(c);
    CpFactors f = cp_factors(c, F_dev);
    CpGrad d;
    memset(&d, 0, sizeof(d));
    int64_t maxI = 1;
    for (int n = 0; n < c->N; ++n) {
      if (!M_dev[n] || !grad_dev[n]) fail(PLANC_GPU_ERR_ARG, "null MTTKRP or gradient");
      d.M[n] = M_dev[n];
      d.grad[n] = grad_dev[n];
      maxI = std::max(maxI, c->dims[n]);
    }
    const unsigned gx = (unsigned)std::min<int64_t>((maxI * c->k + 255) / 256, 1024);
    launch(c, KC_UPDATE, [&] {
      k_cp_grads<<<dim3(gx, c->N), 256, 0, c->stream>>>(f, G, d, g_dev);
    });
  });
}

int planc_gpu_cp_step_device(planc_gpu_ctx* c, const double* const* Y, const double* const* grad,
                             const double* const* Fprev, double eta, double mom, double* const* Fnew,
                             double* const* Ynew) {
  return guarded([&] {
    require_ready(c);
    if (!Y || !grad || !Fprev || !Fnew || !Ynew) fail(PLANC_GPU_ERR_ARG, "null argument");
    set_device(c);
    CpStep s;
    memset(&s, 0, sizeof(s));
    s.N = c->N;
    int64_t maxn = 1;
    for (int n = 0; n < c->N; ++n) {
      if (!Y[n] || !grad[n] || !Fprev[n] || !Fnew[n] || !Ynew[n]) fail(PLANC_GPU_ERR_ARG, "null factor");
      s.Y[n] = Y[n];
      s.grad[n] = grad[n];
      s.Fprev[n] = Fprev[n];
      s.Fnew[n] = Fnew[n];
      s.Ynew[n] = Ynew[n];
      s.n[n] = c->dims[n] * c->k;
      maxn = std::max(maxn, s.n[n]);
    }
    const unsigned gx = (unsigned)std::min<int64_t>((maxn + 255) / 256, 1024);
    launch(c, KC_UPDATE, [&] { k_cp_step<<<dim3(gx, c->N), 256, 0, c->stream>>>(s, eta, mom); });
  });
}

int planc_gpu_mttkrp_device(planc_gpu_ctx* c, int mode, const double* const* F_dev, double* M_dev,
                            int flags) {
  return guarded([&] {
    require_ready(c);
    if (mode < 0 || mode >= c->N || !F_dev || !M_dev) fail(PLANC_GPU_ERR_ARG, "bad mode or null pointer");
    for (int n = 0; n < c->N; ++n)
      if (!F_dev[n]) fail(PLANC_GPU_ERR_ARG, "null factor");
    set_device(c);
    ensure_buffers(c);
    const bool dt = (flags & 1) && (c->N == 3 || c->N == 4);
    const bool reuse = (flags & 2) != 0;
    if (!dt) ensure_direct(c);
    double* saved[kMaxModes];
    for (int n = 0; n < c->N; ++n) {
      saved[n] = c->F[n];
      c->F[n] = const_cast<double*>(F_dev[n]);
    }
    try {
      if (dt) {
        if (!reuse) dimtree_prereq(c, mode);
        mttkrp_dimtree(c, mode, M_dev);
      } else {
        mttkrp_direct(c, mode, M_dev);
      }
    } catch (...) {
      for (int n = 0; n < c->N; ++n) c->F[n] = saved[n];
      throw;
    }
    for (int n = 0; n < c->N; ++n) c->F[n] = saved[n];
  });
}

int planc_gpu_tensor_norm2(planc_gpu_ctx* c, double* out) {
  return guarded([&] {
    if (!c || !out) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (!c->have_tensor) fail(PLANC_GPU_ERR_STATE, "no tensor set");
    set_device(c);
    CK(cudaMemcpyAsync(out, c->normX2, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

int planc_gpu_set_bpp_max_iter(planc_gpu_ctx* c, int max_iter) {
  return guarded([&] {
    if (!c || max_iter < 0) fail(PLANC_GPU_ERR_ARG, "bad argument");
    c->bpp_max_iter = max_iter;
    reset_graph(c);
  });
}

int planc_gpu_set_bpp_warm_start(planc_gpu_ctx* c, int enable) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    if (c->bpp_warm != (enable != 0)) {
      c->bpp_warm = enable != 0;
      reset_graph(c);  // captured graphs hold the launch arguments
    }
  });
}

int planc_gpu_reset_update_state(planc_gpu_ctx* c) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    set_device(c);
    CK(cudaStreamSynchronize(c->stream));
    free_update_state(c);
  });
}

int planc_gpu_selftest_wait_timeout(int device, double seconds, int* status_out) {
  return guarded([&] {
    if (!status_out || !(seconds > 0) || seconds > 5) fail(PLANC_GPU_ERR_ARG, "bad argument");
    CK(cudaSetDevice(device));
    int clk_khz = 0;
    CK(cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, device));
    long long limit = (long long)(seconds * (double)clk_khz * 1e3);
    int* st = nullptr;
    CK(cudaMalloc(&st, sizeof(int)));
    cudaMemset(st, 0, sizeof(int));
    k_tc_wait_selftest<<<1, 32>>>(limit, st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&h, st, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(st);
    cuda_check(e, "wait self-test");
    *status_out = h;
  });
}

int planc_gpu_selftest_coop_timeout(int device, int* status_out) {
  return guarded([&] {
    if (!status_out) fail(PLANC_GPU_ERR_ARG, "null argument");
    CK(cudaSetDevice(device));
    const int nct = 4;
    double* part = nullptr;
    unsigned* flag = nullptr;
    int* st = nullptr;
    auto cleanup = [&] {
      cudaFree(part);
      cudaFree(flag);
      cudaFree(st);
    };
    try {
      CK(cudaMalloc(&part, nct * sizeof(double)));
      CK(cudaMalloc(&flag, sizeof(unsigned)));
      CK(cudaMalloc(&st, sizeof(int)));
      CK(cudaMemset(part, 0xff, nct * sizeof(double)));  // NMFC_EMPTY in every slot
      CK(cudaMemset(flag, 0, sizeof(unsigned)));
      CK(cudaMemset(st, 0, sizeof(int)));
      unsigned limit = 1u << 12;
      int skip = 1;
      void* args[] = {&part, &flag, &st, &limit, &skip};
      CK(cudaLaunchCooperativeKernel((const void*)k_nmfc_wait_selftest, dim3(nct), dim3(64), args,
                                     0, nullptr));
      CK(cudaDeviceSynchronize());
      int h = 0;
      CK(cudaMemcpy(&h, st, sizeof(int), cudaMemcpyDeviceToHost));
      *status_out = h;
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
  });
}

int planc_gpu_set_timing(planc_gpu_ctx* c, int enable) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    set_device(c);
    drain_timing(c);
    c->timing = enable != 0;
  });
}

int planc_gpu_get_kernel_times(planc_gpu_ctx* c, double* ms, int64_t* launches, int n) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    set_device(c);
    drain_timing(c);
    for (int i = 0; i < n && i < KC_COUNT; ++i) {
      if (ms) ms[i] = c->kms[i];
      if (launches) launches[i] = c->klaunch[i];
    }
    for (int i = 0; i < KC_COUNT; ++i) {
      c->kms[i] = 0;
      c->klaunch[i] = 0;
    }
  });
}

int64_t planc_gpu_launch_count(planc_gpu_ctx* c) { return c ? c->launch_count : -1; }

int planc_gpu_synth_cp_tensor(int device, void* X_dev, int dtype, const int64_t* dims, int nmodes,
                              const double* const* A, int k, double sigma, uint64_t seed, int clip,
                              void* cuda_stream) {
  return guarded([&] {
    if (!X_dev || !dims || !A) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (nmodes < 1 || nmodes > kMaxModes || k < 1) fail(PLANC_GPU_ERR_ARG, "bad shape");
    if (dtype != PLANC_GPU_F64 && dtype != PLANC_GPU_F32) fail(PLANC_GPU_ERR_ARG, "bad dtype");
    CK(cudaSetDevice(device));
    cudaStream_t st = (cudaStream_t)cuda_stream;
    SynthDesc d;
    memset(&d, 0, sizeof(d));
    d.N = nmodes;
    d.k = k;
    d.sigma = sigma;
    d.seed = seed;
    d.clip = clip;
    int64_t numel = 1;
    std::vector<double*> bufs;
    try {
      for (int m = 0; m < nmodes; ++m) {
        d.dims[m] = dims[m];
        numel *= dims[m];
        double* p = nullptr;
        CK(cudaMalloc(&p, (size_t)dims[m] * k * 8));
        bufs.push_back(p);
        CK(cudaMemcpyAsync(p, A[m], (size_t)dims[m] * k * 8, cudaMemcpyHostToDevice, st));
        d.A[m] = p;
      }
      if (dtype == PLANC_GPU_F32)
        k_synth_cp<float><<<8192, 256, 0, st>>>(d, numel, (float*)X_dev);
      else
        k_synth_cp<double><<<8192, 256, 0, st>>>(d, numel, (double*)X_dev);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(st));
    } catch (...) {
      for (auto p : bufs) cudaFree(p);
      throw;
    }
    for (auto p : bufs) cudaFree(p);
  });
}

}  // extern "C"

// ============================================================ batched factorisation
// Many independent tensors (uneven shapes and ranks) factorised together: one
// context per tensor, each bound to one of S worker streams; one outer
// iteration of every tensor is captured into ONE CUDA graph (fork from a
// master stream to the workers, join back) and that graph is launched once
// per iteration, so the tensors' kernels overlap on the GPU. The per-context
// parallelism (split-K / grid sizing) is chosen by an autotuner that times
// the whole batch graph for a few candidate settings per size class.
struct planc_gpu_batch {
  int device = 0;
  int precision = PLANC_GPU_PREC_FP64;
  cudaStream_t master = nullptr;
  std::vector<cudaStream_t> workers;
  std::vector<planc_gpu_ctx*> members;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  cudaGraphExec_t gexec = nullptr;
  int g_algo = -1, g_err = -1;
  int64_t g_epoch = -1;  // sum of the members' buffer epochs at capture
  // grouped iterations: argument tables of the grouped launches (device copy)
  bool group = true;     // PLANC_GPU_BATCH_GROUPED=0 turns grouped phases off
  uint8_t* grp_dev = nullptr;
  size_t grp_cap = 0;
  bool g_grouped = false;  // the cached graph runs grouped phases
};

namespace {

void batch_reset_graph(planc_gpu_batch* b);

int64_t batch_epoch(const planc_gpu_batch* b) {
  int64_t e = (int64_t)b->members.size();
  for (auto* m : b->members) e += m->buf_epoch;
  return e;
}

// every buffer the batch graph will reference, allocated before capture
void batch_ensure(planc_gpu_batch* b, int iters, bool err) {
  for (auto* m : b->members) {
    ensure_buffers(m);
    ensure_errs(m, err ? iters : 1);
  }
  if (b->g_epoch != batch_epoch(b)) batch_reset_graph(b);
}

void batch_reset_graph(planc_gpu_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->g_algo = b->g_err = -1;
}

// size class of a member for the autotuner: by element count
int batch_class(const planc_gpu_ctx* c) {
  return c->numel < (1 << 20) ? 0 : c->numel < (1 << 23) ? 1 : 2;
}

bool batch_groupable(const planc_gpu_batch* b, int algo);
void batch_capture_grouped(planc_gpu_batch* b, int algo, bool err);

void batch_capture(planc_gpu_batch* b, int algo, bool err) {
  if (batch_groupable(b, algo)) {
    batch_capture_grouped(b, algo, err);
    return;
  }
  batch_reset_graph(b);
  b->g_grouped = false;
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
  try {
    CK(cudaEventRecord(b->fork, b->master));
    for (auto w : b->workers) CK(cudaStreamWaitEvent(w, b->fork, 0));
    for (auto* m : b->members) {
      m->capturing = true;
      one_iteration(m, algo, true, err);
      m->capturing = false;
    }
    for (size_t i = 0; i < b->workers.size(); ++i) {
      CK(cudaEventRecord(b->joins[i], b->workers[i]));
      CK(cudaStreamWaitEvent(b->master, b->joins[i], 0));
    }
  } catch (...) {
    for (auto* m : b->members) m->capturing = false;
    cudaStreamEndCapture(b->master, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  CK(cudaStreamEndCapture(b->master, &graph));
  cudaError_t e = cudaGraphInstantiate(&b->gexec, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(e, "cudaGraphInstantiate (batch)");
  b->g_algo = algo;
  b->g_err = err ? 1 : 0;
  b->g_epoch = batch_epoch(b);
}

// ---------------------------------------------------------------- grouped phases
// A batch whose members are all 3-way tensor-core contexts running MU or HALS
// on the dimension tree (factors of at most NGC_MAX_ROWS rows) runs each
// outer iteration as phases: the tensor-core contractions of every member on
// the worker streams (one per member, as before), and every other step of
// the iteration -- the multi-TTVs, split-K sums, factor updates,
// normalisation + Gram and error -- as ONE launch for all members (blockIdx.z
// = member, batch_group.cuh). The members' arithmetic is that of their own
// iteration (mttkrp_dimtree + run_update + normalize_gram + error_kernel);
// a batched iteration is ~15 launches plus the contractions instead of
// ~15 launches per member.
bool batch_groupable(const planc_gpu_batch* b, int algo) {
  if (!b->group || (algo != PLANC_GPU_HALS && algo != PLANC_GPU_MU)) return false;
  for (auto* m : b->members) {
    if (m->N != 3 || m->precision == PLANC_GPU_PREC_FP64 || m->bal4 || m->ngc_ctas <= 0) return false;
    for (int n = 0; n < 3; ++n)
      if (m->dims[n] > NGC_MAX_ROWS) return false;
  }
  return true;
}

// Host copies of the argument tables, laid out as they are copied to the
// batch's device buffer after capture (the captured launches hold device
// addresses inside that buffer).
struct GrpTables {
  std::vector<uint8_t> host;
  uint8_t* dev = nullptr;
  size_t cap = 0;
  template <typename T>
  const T* put(const std::vector<T>& v) {
    size_t off = (host.size() + 255) & ~(size_t)255;
    const size_t bytes = v.size() * sizeof(T);
    if (off + bytes > cap) fail(PLANC_GPU_ERR_STATE, "internal: grouped argument tables too large");
    host.resize(off + bytes);
    memcpy(host.data() + off, v.data(), bytes);
    return reinterpret_cast<const T*>(dev + off);
  }
};

void grp_check(cudaError_t e) { cuda_check(e, "grouped launch"); }

template <typename T>
unsigned grp_max(const std::vector<T>& v, unsigned T::*f) {
  unsigned g = 1;
  for (const T& x : v) g = std::max(g, x.*f);
  return g;
}

void grp_reduce(GrpTables& tab, cudaStream_t st, const std::vector<GrpRed>& all) {
  std::vector<GrpRed> few, many;
  for (const GrpRed& r : all) (reduce_kind(r.nsplit) == 0 ? few : many).push_back(r);
  if (!few.empty())
    k_grp_reduce_few<<<dim3(grp_max(few, &GrpRed::gx), 1, (unsigned)few.size()), 256, 0, st>>>(tab.put(few));
  if (!many.empty())
    k_grp_reduce<<<dim3(grp_max(many, &GrpRed::gx), 1, (unsigned)many.size()), 256, 0, st>>>(tab.put(many));
  grp_check(cudaGetLastError());
}

GrpRed grp_red(const double* part, int nsplit, int64_t n, double* out) {
  return GrpRed{part, nsplit, n, n, out, reduce_blocks(nsplit, n)};
}

// run_update for every member (MU / HALS, one warp per row)
void grp_update(GrpTables& tab, cudaStream_t st, const std::vector<planc_gpu_ctx*>& ms, int algo, int n) {
  std::vector<GrpUpd> u32, u64;
  for (auto* m : ms) {
    const int64_t I = m->dims[n];
    GrpUpd u{m->F[n], m->M[n], m->Gloo, I, m->k, (unsigned)((I + 7) / 8)};
    (m->k <= 32 ? u32 : u64).push_back(u);
  }
  if (!u32.empty()) {
    const dim3 g(grp_max(u32, &GrpUpd::gx), 1, (unsigned)u32.size());
    if (algo == PLANC_GPU_HALS) k_grp_hals<32><<<g, 256, 0, st>>>(tab.put(u32));
    else k_grp_mu<32><<<g, 256, 0, st>>>(tab.put(u32), kEps6);
  }
  if (!u64.empty()) {
    const dim3 g(grp_max(u64, &GrpUpd::gx), 1, (unsigned)u64.size());
    if (algo == PLANC_GPU_HALS) k_grp_hals<64><<<g, 256, 0, st>>>(tab.put(u64));
    else k_grp_mu<64><<<g, 256, 0, st>>>(tab.put(u64), kEps6);
  }
  grp_check(cudaGetLastError());
}

// normalize_gram(n, next, lambda) for every member (its cluster path)
void grp_normgram(GrpTables& tab, cudaStream_t st, const std::vector<planc_gpu_ctx*>& ms, int n, int next) {
  std::vector<GrpNg> g2, g4;
  int cl2 = 1, cl4 = 1;
  for (auto* m : ms) {
    const int64_t I = m->dims[n];
    const int64_t rpc = m->k > 32 ? 16 : NGC_TILE;
    const int cl = (int)std::min<int64_t>(m->ngc_ctas, std::max<int64_t>(1, (I + rpc - 1) / rpc));
    GrpNg g{m->F[n], I, m->k, m->lambda, m->Gall, m->N, n, next, m->Gloo, cl};
    if (m->k <= 32) {
      g2.push_back(g);
      cl2 = std::max(cl2, cl);
    } else {
      g4.push_back(g);
      cl4 = std::max(cl4, cl);
    }
  }
  auto go = [&](auto kern, const std::vector<GrpNg>& v, int cl, int kp) {
    if (v.empty()) return;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cl, 1, (unsigned)v.size());
    cfg.blockDim = dim3(NGC_THREADS, 1, 1);
    cfg.dynamicSmemBytes = ngc_smem_bytes(kp);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    grp_check(cudaLaunchKernelEx(&cfg, kern, tab.put(v)));
  };
  go(k_grp_normgram<2>, g2, cl2, 32);
  go(k_grp_normgram<4>, g4, cl4, 64);
}

void batch_capture_grouped(planc_gpu_batch* b, int algo, bool err) {
  batch_reset_graph(b);
  const auto& ms = b->members;
  const size_t cap = 32 * ((size_t)ms.size() * 512 + 256);
  if (b->grp_cap < cap) {
    dalloc(&b->grp_dev, cap);
    b->grp_cap = cap;
  }
  GrpTables tab;
  tab.dev = b->grp_dev;
  tab.cap = b->grp_cap;
  cudaStream_t st = b->master;
  auto fork = [&] {
    CK(cudaEventRecord(b->fork, st));
    for (auto w : b->workers) CK(cudaStreamWaitEvent(w, b->fork, 0));
  };
  auto join = [&] {
    for (size_t i = 0; i < b->workers.size(); ++i) {
      CK(cudaEventRecord(b->joins[i], b->workers[i]));
      CK(cudaStreamWaitEvent(st, b->joins[i], 0));
    }
  };
  if (b->precision == PLANC_GPU_PREC_BF16X2) {
    CK((tcg_set_attrs<16, true>()));
    CK((tcg_set_attrs<32, true>()));
    CK((tcg_set_attrs<64, true>()));
  } else {
    CK((tcg_set_attrs<16, false>()));
    CK((tcg_set_attrs<32, false>()));
    CK((tcg_set_attrs<64, false>()));
  }
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  try {
    for (auto* m : ms) m->capturing = true;
    // every member's tensor maps: right hi, right lo, left hi, left lo
    std::vector<CUtensorMap> maps(4 * ms.size());
    for (size_t i = 0; i < ms.size(); ++i) {
      maps[4 * i] = ms[i]->tct.mR_hi;
      maps[4 * i + 1] = ms[i]->tct.mR_lo;
      maps[4 * i + 2] = ms[i]->tct.mL_hi;
      maps[4 * i + 3] = ms[i]->tct.mL_lo;
    }
    const CUtensorMap* dmaps = tab.put(maps);
    const bool x2 = b->precision == PLANC_GPU_PREC_BF16X2;
    const int sms = ms[0]->sm_count;
    int* gst = ms[0]->status_dev;  // status word of the grouped contractions
    auto kpi = [](int k) { return tc_kpad(k) == 16 ? 0 : tc_kpad(k) == 32 ? 1 : 2; };
    // ---- mode 0: P = X F_2 for every member (one grouped launch per rank
    // class; members whose right contraction also forms the mode-0 multi-TTV
    // keep their own launches); M_0 from P or from the fused TTV partials
    std::vector<GrpRed> red;
    std::vector<GrpTtvR> ttvr[4];
    std::vector<TcgRight> rmem(ms.size());
    std::vector<TcgBimg> bim[3];
    std::vector<int2> ritems[3];
    fork();
    for (size_t mi = 0; mi < ms.size(); ++mi) {
      planc_gpu_ctx* m = ms[mi];
      const int k = m->k;
      const int64_t I0 = m->dims[0];
      const int ns = tc_right_ttv_nsplit(m->tct, k, eff_sm(m));
      if (ns > 0 && (size_t)ns * I0 * k <= m->scratch_elems) {
        launch(m, KC_PREP, [&] { tc_right_prep(m->tct, m->F[2], k, m->stream); });
        launch(m, KC_CONTRACT, [&] {
          tc_right_ttv(m->tct, k, m->P32, m->F[1], m->scratch, m->status_dev, eff_sm(m), m->stream,
                       m->tc_cpa);
        });
        red.push_back(grp_red(m->scratch, ns, I0 * k, m->M[0]));
      } else {
        const int ci = kpi(k), kp = tc_kpad(k);
        const int nk = (int)((m->tct.R + TC_BK - 1) / TC_BK);
        bim[ci].push_back(TcgBimg{m->F[2], m->tct.R, k, nk, m->tct.bimg,
                                  (unsigned)std::min<int64_t>(((int64_t)nk * kp * TC_BK + 255) / 256, 1024)});
        rmem[mi] = TcgRight{m->tct.bimg, m->P32, m->tct.L, m->tct.R, k, 0};
        const int64_t ntiles = (m->tct.L + TC_BM - 1) / TC_BM;
        for (int64_t t = 0; t < ntiles; ++t) ritems[ci].push_back(make_int2((int)mi, (int)t));
        const int64_t A = I0, B = m->L / I0;
        TtvRightPlan p = plan_ttv_right(m, A, B);
        if (p.nsplit > 1 && (size_t)p.nsplit * A * k > m->scratch_elems)
          fail(PLANC_GPU_ERR_STATE, "internal: multi-TTV scratch larger than planned");
        const int ki = kpad(k) == 8 ? 0 : kpad(k) == 16 ? 1 : kpad(k) == 32 ? 2 : 3;
        ttvr[ki].push_back(GrpTtvR{m->P32, A, B, k, make_wgen(m, {1}), p.bper,
                                   p.nsplit > 1 ? m->scratch : m->M[0], p.grid.x, p.grid.y});
        if (p.nsplit > 1) red.push_back(grp_red(m->scratch, p.nsplit, A * k, m->M[0]));
      }
    }
    {
      const TcgRight* drm = tab.put(rmem);
      for (int ci = 0; ci < 3; ++ci) {
        if (ritems[ci].empty()) continue;
        const auto& bv = bim[ci];
        const dim3 gb(grp_max(bv, &TcgBimg::gx), 1, (unsigned)bv.size());
        const TcgBimg* db = tab.put(bv);
        const int2* di = tab.put(ritems[ci]);
        const int n = (int)ritems[ci].size();
        const int grid = std::min(n, sms);
#define TCG_RIGHT(KP)                                                                           \
  {                                                                                             \
    constexpr uint32_t SR16 = 2 * KP * 128;                                                     \
    const uint32_t stage = (x2 ? 2u : 1u) * TC_BM * TC_BK * 2 + SR16;                           \
    const int stg = tc_stages(stage);                                                           \
    const size_t smem = (size_t)stg * stage + 1024;                                             \
    k_tc_bimage_grp<KP><<<gb, 256, 0, st>>>(db);                                                \
    if (x2) k_tc_right_grp<KP, true><<<grid, TC_THREADS, smem, st>>>(dmaps, drm, di, n, stg, gst); \
    else k_tc_right_grp<KP, false><<<grid, TC_THREADS, smem, st>>>(dmaps, drm, di, n, stg, gst); \
  }
        if (ci == 0) TCG_RIGHT(16) else if (ci == 1) TCG_RIGHT(32) else TCG_RIGHT(64)
#undef TCG_RIGHT
        grp_check(cudaGetLastError());
      }
    }
    join();
    for (int ki = 0; ki < 4; ++ki) {
      const auto& v = ttvr[ki];
      if (v.empty()) continue;
      const dim3 g(grp_max(v, &GrpTtvR::gx), grp_max(v, &GrpTtvR::gy), (unsigned)v.size());
      const GrpTtvR* t = tab.put(v);
      if (ki == 0) k_grp_ttv_right<8><<<g, 256, 0, st>>>(t);
      else if (ki == 1) k_grp_ttv_right<16><<<g, 256, 0, st>>>(t);
      else if (ki == 2) k_grp_ttv_right<32><<<g, 256, 0, st>>>(t);
      else k_grp_ttv_right<64><<<g, 256, 0, st>>>(t);
      grp_check(cudaGetLastError());
    }
    grp_reduce(tab, st, red);
    grp_update(tab, st, ms, algo, 0);
    grp_normgram(tab, st, ms, 0, 1);
    // ---- mode 1: M_1 = TTV of P with the updated F_0 (run_ttv_left<float>)
    {
      std::vector<GrpTtvL> plain, f4;
      for (auto* m : ms) {
        const int k = m->k;
        const int64_t A = m->dims[0], B = m->dims[1];
        const int64_t g2 = (B + TTVL_NB - 1) / TTVL_NB;
        if (k % 4 == 0 && g2 >= eff_sm(m) && g2 <= 65535)
          f4.push_back(GrpTtvL{m->P32, A, B, k, m->F[0], m->M[1], (unsigned)g2});
        else
          plain.push_back(GrpTtvL{m->P32, A, B, k, m->F[0], m->M[1],
                                  (unsigned)std::min<int64_t>(B, 65535)});
      }
      if (!plain.empty())
        k_grp_ttv_left<<<dim3(grp_max(plain, &GrpTtvL::gx), 1, (unsigned)plain.size()), 256, 0, st>>>(
            tab.put(plain));
      if (!f4.empty())
        k_grp_ttv_left_f4<<<dim3(grp_max(f4, &GrpTtvL::gx), 1, (unsigned)f4.size()), 256, 0, st>>>(
            tab.put(f4));
      grp_check(cudaGetLastError());
    }
    grp_update(tab, st, ms, algo, 1);
    grp_normgram(tab, st, ms, 1, 2);
    // ---- mode 2: M_2 = X^T KRP(F_0, F_1) per member (split-K partials), then the sums
    // one grouped launch per (rank class, row tiles per CTA) for the generic
    // left contractions; the factored ones (I_0 % 64 == 0) keep their own
    red.clear();
    std::vector<TcgLeft> lmem(ms.size());
    std::vector<TcgUnit> lunits[3][2];
    fork();
    for (size_t mi = 0; mi < ms.size(); ++mi) {
      planc_gpu_ctx* m = ms[mi];
      WGen wg = make_wgen(m, {0, 1});
      if (tc_scratch_elems(m->tct, eff_sm(m), m->k) > m->scratch_elems)
        fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
      if (tc_left_factored(m->tct)) {
        int nsplit = 0;
        launch(m, KC_CONTRACT_LEFT, [&] {
          nsplit = tc_left(m->tct, wg, m->k, m->scratch, m->status_dev, eff_sm(m), m->stream,
                           m->left_chunks);
        });
        red.push_back(grp_red(m->scratch, nsplit, m->R * m->k, m->M[2]));
        continue;
      }
      if (left_via_long(m)) {
        // the member's own Khatri-Rao image and long-K contraction (as
        // long_contract), the split-K sum in the grouped reduction
        launch(m, KC_PREP, [&] { tc_long_prep(m->tct, true, wg, m->k, m->stream); });
        if (tc_long_scratch_elems(m->tct, true, m->k, eff_sm(m)) > m->scratch_elems)
          fail(PLANC_GPU_ERR_STATE, "internal: split-K scratch larger than planned");
        int nsplit = 1;
        launch(m, KC_CONTRACT_LEFT, [&] {
          nsplit = tc_long(m->tct, true, m->k, m->M[2], m->scratch, m->status_dev, eff_sm(m),
                           m->stream);
        });
        if (nsplit > 1) red.push_back(grp_red(m->scratch, nsplit, m->R * m->k, m->M[2]));
        continue;
      }
      int mg = 0, ns = 0;
      tc_left_plan(m->tct, m->k, eff_sm(m), &mg, &ns, m->left_chunks);
      const int MT = tc_left_mt(m->tct.R, m->k);
      lmem[mi] = TcgLeft{wg, m->scratch, m->tct.L, m->tct.R, m->k, ns};
      for (int jg = 0; jg < mg; ++jg)
        for (int y = 0; y < ns; ++y) lunits[kpi(m->k)][MT - 1].push_back(TcgUnit{(int)mi, jg, y, 0});
      red.push_back(grp_red(m->scratch, ns, m->R * m->k, m->M[2]));
    }
    {
      const TcgLeft* dlm = tab.put(lmem);
      for (int ci = 0; ci < 3; ++ci)
        for (int mt = 1; mt <= 2; ++mt) {
          const auto& uv = lunits[ci][mt - 1];
          if (uv.empty()) continue;
          const TcgUnit* du = tab.put(uv);
          const int n = (int)uv.size();
          const int grid = std::min(n, sms);
#define TCG_LEFT(KP, MTV)                                                                            \
  {                                                                                                  \
    const uint32_t stage = (x2 ? 2u : 1u) * MTV * TC_BM * TC_BK * 2 + 2 * KP * 128;                  \
    const int stg = tc_stages(stage);                                                                \
    const size_t smem = (size_t)stg * stage + 1024;                                                  \
    if (x2) k_tc_left_grp<KP, MTV, true><<<grid, TCL_THREADS, smem, st>>>(dmaps, dlm, du, n, stg, gst);  \
    else k_tc_left_grp<KP, MTV, false><<<grid, TCL_THREADS, smem, st>>>(dmaps, dlm, du, n, stg, gst);    \
  }
          if (ci == 0) { if (mt == 1) TCG_LEFT(16, 1) else TCG_LEFT(16, 2) }
          else if (ci == 1) { if (mt == 1) TCG_LEFT(32, 1) else TCG_LEFT(32, 2) }
          else { if (mt == 1) TCG_LEFT(64, 1) else TCG_LEFT(64, 2) }
#undef TCG_LEFT
          grp_check(cudaGetLastError());
        }
    }
    join();
    grp_reduce(tab, st, red);
    grp_update(tab, st, ms, algo, 2);
    grp_normgram(tab, st, ms, 2, 0);
    if (err) {
      std::vector<GrpErr> e;
      for (auto* m : ms)
        e.push_back(GrpErr{m->M[2], m->F[2], m->dims[2], m->lambda, m->Gall, m->N, m->k, m->normX2,
                           m->errs_dev, m->counter_dev});
      k_grp_error<<<dim3(1, 1, (unsigned)e.size()), 1024, 0, st>>>(tab.put(e));
      grp_check(cudaGetLastError());
    }
    for (auto* m : ms) m->capturing = false;
  } catch (...) {
    for (auto* m : ms) m->capturing = false;
    cudaStreamEndCapture(st, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  CK(cudaStreamEndCapture(st, &graph));
  cudaError_t e = cudaGraphInstantiate(&b->gexec, graph, 0);
  cudaGraphDestroy(graph);
  cuda_check(e, "cudaGraphInstantiate (grouped batch)");
  // the captured launches read their tables from grp_dev from the first replay
  // on (no earlier replay of this batch is still running: the master stream
  // is drained first)
  CK(cudaStreamSynchronize(st));
  CK(cudaMemcpy(b->grp_dev, tab.host.data(), tab.host.size(), cudaMemcpyHostToDevice));
  b->g_algo = algo;
  b->g_err = err ? 1 : 0;
  b->g_epoch = batch_epoch(b);
  b->g_grouped = true;
}

// per-run set-up of every member (error counters, first leave-one-out Gram),
// ordered before the graph launches on the master stream
void batch_prepare(planc_gpu_batch* b) {
  for (auto* m : b->members) {
    CK(cudaMemsetAsync(m->counter_dev, 0, sizeof(int), m->stream));
    gram_loo(m, 0);
  }
  for (size_t i = 0; i < b->workers.size(); ++i) {
    CK(cudaEventRecord(b->joins[i], b->workers[i]));
    CK(cudaStreamWaitEvent(b->master, b->joins[i], 0));
  }
}

void batch_finish(planc_gpu_batch* b) {
  CK(cudaStreamSynchronize(b->master));
  for (auto* m : b->members) check_status(m);
}

}  // namespace

extern "C" {

int planc_gpu_batch_create(planc_gpu_batch** out, int device, int precision, int nstreams) {
  return guarded([&] {
    if (!out) fail(PLANC_GPU_ERR_ARG, "out is null");
    *out = nullptr;
    if (nstreams < 1 || nstreams > 64) fail(PLANC_GPU_ERR_ARG, "nstreams must be in [1, 64]");
    if (precision < PLANC_GPU_PREC_FP64 || precision > PLANC_GPU_PREC_BF16X2)
      fail(PLANC_GPU_ERR_ARG, "unknown precision");
    CK(cudaSetDevice(device));
    planc_gpu_batch* b = new planc_gpu_batch();
    b->device = device;
    b->precision = precision;
    // PLANC_GPU_BATCH_GROUPED=0: per-member launches only (no grouped phases)
    if (const char* e = getenv("PLANC_GPU_BATCH_GROUPED")) b->group = strcmp(e, "0") != 0;
    try {
      // the grouped normalisation + Gram runs clusters of up to 16 CTAs with
      // up to 64 KB of dynamic shared memory (as k_normgram_cluster)
      for (auto kern : {k_grp_normgram<2>, k_grp_normgram<4>}) {
        if (cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess)
          cudaGetLastError();
        CK(cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ngc_smem_bytes(64)));
      }
      CK(cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking));
      CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
      for (int i = 0; i < nstreams; ++i) {
        cudaStream_t w;
        CK(cudaStreamCreateWithFlags(&w, cudaStreamNonBlocking));
        b->workers.push_back(w);
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->joins.push_back(e);
      }
    } catch (...) {
      for (auto w : b->workers) cudaStreamDestroy(w);
      for (auto e : b->joins) cudaEventDestroy(e);
      if (b->fork) cudaEventDestroy(b->fork);
      if (b->master) cudaStreamDestroy(b->master);
      delete b;
      throw;
    }
    *out = b;
  });
}

int planc_gpu_batch_add(planc_gpu_batch* b, const void* X, int dtype, const int64_t* dims,
                        int nmodes, int x_on_device, const double* const* F, int k, int* index) {
  return guarded([&] {
    if (!b) fail(PLANC_GPU_ERR_ARG, "null batch");
    if (nmodes != 3 && nmodes != 4)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "batched members run the dimension tree (N in {3,4})");
    batch_reset_graph(b);
    planc_gpu_ctx* m = nullptr;
    cudaStream_t w = b->workers[b->members.size() % b->workers.size()];
    int rc = planc_gpu_create(&m, b->device, b->precision, (void*)w);
    if (rc != PLANC_GPU_OK) throw Fail{rc};
    rc = planc_gpu_set_tensor(m, X, dtype, dims, nmodes, x_on_device);
    if (rc == PLANC_GPU_OK) rc = planc_gpu_set_factors(m, F, nullptr, k);
    if (rc != PLANC_GPU_OK) {
      std::string msg = g_last_error;
      planc_gpu_destroy(m);
      g_last_error = msg;
      throw Fail{rc};
    }
    b->members.push_back(m);
    if (index) *index = (int)b->members.size() - 1;
  });
}

int planc_gpu_batch_count(planc_gpu_batch* b) { return b ? (int)b->members.size() : -1; }

int planc_gpu_batch_set_factors(planc_gpu_batch* b, int index, const double* const* F, int k) {
  return guarded([&] {
    if (!b || index < 0 || index >= (int)b->members.size()) fail(PLANC_GPU_ERR_ARG, "bad index");
    int rc = planc_gpu_set_factors(b->members[index], F, nullptr, k);
    if (rc != PLANC_GPU_OK) throw Fail{rc};
    batch_reset_graph(b);
  });
}

int planc_gpu_batch_run(planc_gpu_batch* b, int algo, int iters, int compute_error, double* errs) {
  return guarded([&] {
    if (!b) fail(PLANC_GPU_ERR_ARG, "null batch");
    if (b->members.empty()) fail(PLANC_GPU_ERR_STATE, "empty batch");
    if (algo == PLANC_GPU_AOADMM || algo == PLANC_GPU_NESTEROV)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "batched runs take MU, HALS or ANLS/BPP");
    if (algo != PLANC_GPU_MU && algo != PLANC_GPU_HALS && algo != PLANC_GPU_ANLSBPP)
      fail(PLANC_GPU_ERR_ARG, "unknown algorithm");
    if (iters <= 0) return;
    CK(cudaSetDevice(b->device));
    const bool err = compute_error != 0;
    batch_ensure(b, iters, err);
    if (!b->gexec || b->g_algo != algo || b->g_err != (int)err) batch_capture(b, algo, err);
    batch_prepare(b);
    for (int it = 0; it < iters; ++it) CK(cudaGraphLaunch(b->gexec, b->master));
    batch_finish(b);
    if (err && errs) {
      for (size_t i = 0; i < b->members.size(); ++i)
        CK(cudaMemcpy(errs + i * iters, b->members[i]->errs_dev, iters * sizeof(double),
                      cudaMemcpyDeviceToHost));
    }
  });
}

int planc_gpu_batch_get_factors(planc_gpu_batch* b, int index, double* const* F, double* lambda) {
  return guarded([&] {
    if (!b || index < 0 || index >= (int)b->members.size()) fail(PLANC_GPU_ERR_ARG, "bad index");
    int rc = planc_gpu_get_factors(b->members[index], F, lambda);
    if (rc != PLANC_GPU_OK) throw Fail{rc};
  });
}

// Autotuner: for each member size class (by element count), tries the
// parallelism settings {1, 1/2, 1/4, 1/8, 1/16, 1/32} of the GPU per launch,
// timing `trials` graph launches of the whole batch for each, coordinate by
// coordinate, and keeps the fastest. Factors are restored afterwards.
int planc_gpu_batch_autotune(planc_gpu_batch* b, int algo, int trials, double* best_ms) {
  return guarded([&] {
    if (!b || b->members.empty()) fail(PLANC_GPU_ERR_STATE, "empty batch");
    if (trials < 1) trials = 1;
    CK(cudaSetDevice(b->device));
    // save factors so the tuning iterations leave no trace
    std::vector<std::vector<std::vector<double>>> saved(b->members.size());
    std::vector<std::vector<double>> saved_lam(b->members.size());
    for (size_t i = 0; i < b->members.size(); ++i) {
      planc_gpu_ctx* m = b->members[i];
      saved[i].resize(m->N);
      std::vector<double*> ptr(m->N);
      for (int n = 0; n < m->N; ++n) {
        saved[i][n].resize((size_t)m->dims[n] * m->k);
        ptr[n] = saved[i][n].data();
      }
      saved_lam[i].resize(m->k);
      int rc = planc_gpu_get_factors(m, ptr.data(), saved_lam[i].data());
      if (rc != PLANC_GPU_OK) throw Fail{rc};
    }
    const double cand[] = {1.0, 0.5, 0.25, 0.125, 0.0625, 0.03125};
    double scale[3] = {1.0, 1.0, 1.0};
    // fewest 64-element chunks per split-K partial of the left contraction
    const int lcand[] = {0, 8, 32, 128};
    int lch[3] = {0, 0, 0};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    auto time_cfg = [&]() -> float {
      for (auto* m : b->members) {
        m->par_scale = scale[batch_class(m)];
        m->left_chunks = lch[batch_class(m)];
      }
      batch_ensure(b, 1, false);
      batch_capture(b, algo, false);
      batch_prepare(b);
      CK(cudaGraphLaunch(b->gexec, b->master));  // warm-up
      CK(cudaEventRecord(e0, b->master));
      for (int t = 0; t < trials; ++t) CK(cudaGraphLaunch(b->gexec, b->master));
      CK(cudaEventRecord(e1, b->master));
      batch_finish(b);
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      return ms / trials;
    };
    float best = time_cfg();
    for (int cls = 0; cls < 3; ++cls) {
      bool present = false;
      for (auto* m : b->members) present |= batch_class(m) == cls;
      if (!present) continue;
      double keep = scale[cls];
      for (double cv : cand) {
        if (cv == keep) continue;
        scale[cls] = cv;
        float t = time_cfg();
        if (t < best) {
          best = t;
          keep = cv;
        }
      }
      scale[cls] = keep;
      // then the split-K length of the tensor-core left contraction
      if (b->precision != PLANC_GPU_PREC_FP64) {
        int lkeep = lch[cls];
        for (int lc : lcand) {
          if (lc == lkeep) continue;
          lch[cls] = lc;
          float t = time_cfg();
          if (t < best) {
            best = t;
            lkeep = lc;
          }
        }
        lch[cls] = lkeep;
      }
    }
    for (auto* m : b->members) {
      m->par_scale = scale[batch_class(m)];
      m->left_chunks = lch[batch_class(m)];
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    batch_reset_graph(b);
    for (size_t i = 0; i < b->members.size(); ++i) {
      planc_gpu_ctx* m = b->members[i];
      std::vector<const double*> ptr(m->N);
      for (int n = 0; n < m->N; ++n) ptr[n] = saved[i][n].data();
      int rc = planc_gpu_set_factors(m, ptr.data(), saved_lam[i].data(), m->k);
      if (rc != PLANC_GPU_OK) throw Fail{rc};
    }
    if (best_ms) *best_ms = best;
  });
}

int planc_gpu_batch_destroy(planc_gpu_batch* b) {
  if (!b) return PLANC_GPU_OK;
  return guarded([&] {
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->master);
    batch_reset_graph(b);
    for (auto* m : b->members) planc_gpu_destroy(m);
    for (auto w : b->workers) cudaStreamDestroy(w);
    for (auto e : b->joins) cudaEventDestroy(e);
    cudaEventDestroy(b->fork);
    cudaStreamDestroy(b->master);
    if (b->grp_dev) cudaFree(b->grp_dev);
    delete b;
  });
}

}  // extern "C"

// ============================================================ allocation-free MTTKRP
// A variant of the split-K FP64 contraction whose split-K partials live in a
// fixed, file-scope device array instead of memory obtained from cudaMalloc.
// It serves callers that cannot allocate device memory at the time they call
// this library: applications whose device memory is reserved up front by a
// pool allocator (a cudaMalloc would fail or bypass the pool's accounting),
// and latency-critical loops that must not pay the implicit device-wide
// synchronisation a cudaMalloc or cudaFree can cause. Every GPU that loads the
// library holds the array (kNoAllocScratchDoubles doubles = 8 MiB) until exit.
namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(1) << 20;
constexpr int kNoAllocMaxDevices = 64;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on the current device. The host-side
// name of the array is only a stand-in, so the address is resolved once per
// device with cudaGetSymbolAddress (with that device current) and cached.
double* noalloc_scratch(int dev) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_addr[dev];
}

}  // namespace

extern "C" int planc_gpu_mttkrp_last_mode_noalloc(const double* X_dev, const int64_t* dims,
                                                  int nmodes, const double* const* F_dev, int k,
                                                  double* out_dev, void* cuda_stream) {
  return guarded([&] {
    if (!X_dev || !dims || !F_dev || !out_dev) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (nmodes < 2 || nmodes > kMaxModes)
      fail(PLANC_GPU_ERR_ARG, "nmodes must be in [2, " + std::to_string(kMaxModes) + "]");
    if (k < 1 || k > kMaxRank) fail(PLANC_GPU_ERR_UNSUPPORTED, "rank must be in [1, 64]");
    for (int n = 0; n < nmodes; ++n) {
      if (dims[n] < 1) fail(PLANC_GPU_ERR_ARG, "every mode size must be >= 1");
      if (n < nmodes - 1 && !F_dev[n]) fail(PLANC_GPU_ERR_ARG, "null factor");
    }
    const int64_t R = dims[nmodes - 1];
    int64_t A = 1;
    for (int n = 0; n < nmodes - 1; ++n) A *= dims[n];
    if ((size_t)R * (size_t)k > kNoAllocScratchDoubles)
      fail(PLANC_GPU_ERR_UNSUPPORTED,
           "last mode size x rank = " + std::to_string(R * k) +
               " exceeds the allocation-free scratch of " +
               std::to_string(kNoAllocScratchDoubles) + " doubles");
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) fail(PLANC_GPU_ERR_UNSUPPORTED, "device index too large");
    double* scratch = noalloc_scratch(dev);
    contract_f64_attrs(dev);
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // Khatri-Rao operand over modes 0..N-2, lowest mode fastest
    WGen wg;
    memset(&wg, 0, sizeof(wg));
    wg.nf = nmodes - 1;
    int64_t stride = 1;
    for (int t = 0; t < wg.nf; ++t) {
      wg.f[t] = F_dev[t];
      wg.dim[t] = dims[t];
      wg.stride[t] = stride;
      stride *= dims[t];
    }
    // split-K plan of the left contraction out[j, r] = sum_a X[a + A*j] W(a, r),
    // capped so that every split's partial fits in the fixed scratch
    ContractGeom g;
    memset(&g, 0, sizeof(g));
    g.M = R;
    g.ldx = A;
    g.A = A;
    g.B = 1;
    g.ldb = 0;
    const int bk = k > 32 ? ct_bk<64>() : ct_bk<32>();
    g.ktiles = (A + bk - 1) / bk;
    const int64_t mtiles = (R + CT_BM - 1) / CT_BM;
    int64_t ns = (2 * (int64_t)sms + mtiles - 1) / mtiles;
    ns = std::max<int64_t>(1, std::min<int64_t>(ns, g.ktiles));
    ns = std::min<int64_t>(ns, (int64_t)(kNoAllocScratchDoubles / ((size_t)R * k)));
    g.tiles_per_split = (g.ktiles + ns - 1) / ns;
    ns = (g.ktiles + g.tiles_per_split - 1) / g.tiles_per_split;
    g.split_stride = R * k;
    const dim3 grid((unsigned)mtiles, (unsigned)ns, 1);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    // every split writes its whole R x k partial (zeros when it has no tiles),
    // so nothing left in the scratch by an earlier call is read
    switch (kpad(k)) {
      case 8: launch_contract_f64<8, true>(grid, st, X_dev, g, wg, k, scratch); break;
      case 16: launch_contract_f64<16, true>(grid, st, X_dev, g, wg, k, scratch); break;
      case 32: launch_contract_f64<32, true>(grid, st, X_dev, g, wg, k, scratch); break;
      default: launch_contract_f64<64, true>(grid, st, X_dev, g, wg, k, scratch); break;
    }
    CK(cudaGetLastError());
    const int64_t n = R * k;
    reduce_splits(st, scratch, (int)ns, n, n, out_dev);
    CK(cudaGetLastError());
  });
}


// ===================================================================== NMF
// Shared-memory NMF of a dense matrix A ~ W H^T (reference common/nmf.hpp,
// nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp) on a context holding A as its
// 2-way tensor (mode 0 = rows). A H and A^T W are the mode-0 and mode-1
// MTTKRPs: the FP64 contraction kernels, or the long-K tensor-core
// contraction against a hi|lo image of H or W. One CUDA graph per iteration.
namespace {

bool nmf_tc(const planc_gpu_ctx* c) { return c->precision != PLANC_GPU_PREC_FP64; }

void ensure_nmf(planc_gpu_ctx* c, int iters) {
  ensure_buffers(c);
  const int k = c->k;
  const int64_t m = c->dims[0], n = c->dims[1], maxI = std::max(m, n);
  if (nmf_tc(c)) {
    const void* before = c->tct.wimg;
    c->tct.wimg_K = std::max(c->L, c->R);
    CK(tc_ensure(c->tct, k));
    size_t need = std::max(tc_long_scratch_elems(c->tct, true, k, eff_sm(c)),
                           tc_long_scratch_elems(c->tct, false, k, eff_sm(c)));
    if (need > c->scratch_elems) {
      dalloc(&c->scratch, need);
      c->scratch_elems = need;
      c->buf_epoch++;
    }
    if (before != c->tct.wimg) c->buf_epoch++;
  }
  if (!c->nmf_ready) {
    dalloc(&c->nmf_G, (size_t)k * k);
    dalloc(&c->nmf_GW, (size_t)k * k);
    dalloc(&c->nmf_GH, (size_t)k * k);
    dalloc(&c->nmf_norms, (size_t)k);
    c->nmf_part_elems = std::max<size_t>(
        std::max<size_t>((size_t)((maxI + GP_ROWS - 1) / GP_ROWS) * k * k,
                         (size_t)((maxI + CN_ROWS - 1) / CN_ROWS) * k),
        (size_t)NMFW_MAX_BLOCKS * 4);
    dalloc(&c->nmf_part, c->nmf_part_elems);
    dalloc(&c->nmf_ctr, 8);
    CK(cudaMemset(c->nmf_ctr, 0, 8 * sizeof(int)));
    c->nmf_ready = true;
    c->buf_epoch++;
  }
  if (iters > c->nmf_cap) {
    dalloc(&c->nmf_obj, (size_t)iters);
    dalloc(&c->nmf_rel, (size_t)iters);
    c->nmf_cap = iters;
    c->buf_epoch++;
  }
}

// out = U^T U (+ l2 I + l1 ones + diag I)
void nmf_gram(planc_gpu_ctx* c, const double* U, int64_t I, double l2, double l1, double diag,
              double* out) {
  const int k = c->k;
  const int rpb = gram_rows_per_block(I);
  const int nblk = (int)((I + rpb - 1) / rpb);
  if ((size_t)nblk * k * k > c->nmf_part_elems) fail(PLANC_GPU_ERR_STATE, "internal: NMF partials");
  launch(c, KC_NORMGRAM, [&] {
    k_gram_partial<<<nblk, 256, 0, c->stream>>>(U, I, k, rpb, c->nmf_part);
  });
  launch(c, KC_NORMGRAM, [&] {
    k_nmf_gram<<<(unsigned)((k * k + 7) / 8), 256, 0, c->stream>>>(c->nmf_part, nblk, k, l2, l1,
                                                                  diag, out);
  });
}

// M[0] = A H
void nmf_AH(planc_gpu_ctx* c) {
  if (nmf_tc(c))
    long_contract(c, false, {1}, c->M[0]);
  else
    mttkrp_direct(c, 0, c->M[0]);
}

// M[1] = A^T W
void nmf_AtW(planc_gpu_ctx* c) {
  if (nmf_tc(c))
    long_contract(c, true, {0}, c->M[1]);
  else
    mttkrp_direct(c, 1, c->M[1]);
}

// NMF::normalize_by_W (common/nmf.hpp:150-160)
void nmf_normalize(planc_gpu_ctx* c) {
  const int64_t m = c->dims[0], n = c->dims[1];
  const unsigned nb = (unsigned)((m + NRM_ROWS - 1) / NRM_ROWS);
  const unsigned nr = (unsigned)((std::max(m, n) + NRM_ROWS - 1) / NRM_ROWS);
  if ((size_t)nb * c->k > c->nmf_part_elems) fail(PLANC_GPU_ERR_STATE, "internal: NMF partials");
  launch(c, KC_NORMGRAM, [&] {
    k_nmf_colnorms<<<nb, 256, 0, c->stream>>>(c->F[0], m, c->k, c->nmf_part, c->nmf_ctr + 1,
                                               c->nmf_norms);
  });
  launch(c, KC_NORMGRAM, [&] {
    k_nmf_rescale<<<nr, 256, 0, c->stream>>>(c->F[0], m, c->F[1], n, c->k, c->nmf_norms);
  });
}

// rows of U (I x k) from the Gram nmf_G and right-hand sides M: HALS
// (H only), MU or BPP
void nmf_row_update(planc_gpu_ctx* c, int algo, double* U, const double* M, int64_t I) {
  const int k = c->k;
  if (algo == PLANC_GPU_HALS || algo == PLANC_GPU_MU) {
    const unsigned blocks = (unsigned)((I + 7) / 8);
    launch(c, KC_UPDATE, [&] {
      if (algo == PLANC_GPU_HALS) {
        if (k <= 32)
          k_hals_warp<32><<<blocks, 256, 0, c->stream>>>(U, M, c->nmf_G, I, k);
        else
          k_hals_warp<64><<<blocks, 256, 0, c->stream>>>(U, M, c->nmf_G, I, k);
      } else {
        if (k <= 32)
          k_mu_warp<32><<<blocks, 256, 0, c->stream>>>(U, M, c->nmf_G, I, k, kEps17);
        else
          k_mu_warp<64><<<blocks, 256, 0, c->stream>>>(U, M, c->nmf_G, I, k, kEps17);
      }
    });
  } else {
    launch(c, KC_BPP, [&] {
      launch_bpp(c, c->nmf_G, M, k, I, U, nullptr, nullptr, c->bpp_warm ? U : nullptr);
    });
  }
}

// Plan of the cooperative W sweep: CTAs and rows per CTA (a thread per row up
// to NMFC_RPT rows a thread, all CTAs resident, W's rows in shared memory).
// False when W does not fit.
bool nmfc_plan(planc_gpu_ctx* c, int64_t m, int KP, int* grid, int* rows) {
  if (!c->coop_launch || m < 1) return false;
  int occ = 0;
  const int cap_rows = NMFC_THREADS * NMFC_RPT;
  // fewest CTAs first: a CTA of up to NMFC_THREADS rows takes as long as one
  // row, and fewer CTAs make the barriers cheaper
  int64_t g = (m + NMFC_THREADS - 1) / NMFC_THREADS;
  if (g > c->sm_count) g = c->sm_count;
  int64_t r = (m + g - 1) / g;
  if (r > cap_rows) return false;
  const size_t smem = nmfc_smem_bytes(KP, (int)r);
  if (smem > c->smem_optin) return false;
  if (KP == 32)
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_nmf_hals_w_coop<32>, NMFC_THREADS, smem));
  else
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_nmf_hals_w_coop<64>, NMFC_THREADS, smem));
  if ((int64_t)occ * c->sm_count < g) return false;
  if ((size_t)g * c->k > c->nmf_part_elems) return false;
  *grid = (int)g;
  *rows = (int)r;
  return true;
}

// HALSNMF's W sweep (nmf/hals.hpp:92-105): one cooperative launch when W fits
// in the CTAs' shared memory, else k + 1 launches, one per column plus the
// finishing normalisation of the last
void nmf_hals_w(planc_gpu_ctx* c) {
  const int k = c->k;
  const int64_t m = c->dims[0];
  const int KP = k <= 32 ? 32 : 64;
  int grid = 0, rows = 0;
  if (nmfc_plan(c, m, KP, &grid, &rows)) {
    // error flag clear, every column's partial-sum slots empty (all ones)
    unsigned* flag = reinterpret_cast<unsigned*>(c->nmf_ctr + 4);
    CK(cudaMemsetAsync(flag, 0, sizeof(unsigned), c->stream));
    CK(cudaMemsetAsync(c->nmf_part, 0xFF, (size_t)grid * k * sizeof(double), c->stream));
    launch(c, KC_UPDATE, [&] {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)grid, 1, 1);
      cfg.blockDim = dim3(NMFC_THREADS, 1, 1);
      cfg.dynamicSmemBytes = nmfc_smem_bytes(KP, rows);
      cfg.stream = c->stream;
      cudaLaunchAttribute at[1];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      cfg.attrs = at;
      cfg.numAttrs = 1;
      double* W = c->F[0];
      const double* AH = c->M[0];
      const double* G = c->nmf_G;
      if (KP == 32)
        CK(cudaLaunchKernelEx(&cfg, k_nmf_hals_w_coop<32>, W, AH, G, m, k, rows, c->nmf_norms,
                              c->nmf_part, flag, c->status_dev));
      else
        CK(cudaLaunchKernelEx(&cfg, k_nmf_hals_w_coop<64>, W, AH, G, m, k, rows, c->nmf_norms,
                              c->nmf_part, flag, c->status_dev));
    });
    return;
  }
  const unsigned nb = (unsigned)std::min<int64_t>((m + NMFW_WARPS - 1) / NMFW_WARPS, NMFW_MAX_BLOCKS);
  for (int x = 0; x <= k; ++x)
    launch(c, KC_UPDATE, [&] {
      if (k <= 32)
        k_nmf_hals_w<32><<<nb, 32 * NMFW_WARPS, 0, c->stream>>>(
            c->F[0], c->M[0], c->nmf_G, m, k, x, c->nmf_norms, c->nmf_part, c->nmf_ctr + 1);
      else
        k_nmf_hals_w<64><<<nb, 32 * NMFW_WARPS, 0, c->stream>>>(
            c->F[0], c->M[0], c->nmf_G, m, k, x, c->nmf_norms, c->nmf_part, c->nmf_ctr + 1);
    });
}

// out = G + l2 I + l1 ones + diag I from an unregularised Gram G that
// nmf_gram wrote (the same bits nmf_gram would give with the terms: the one
// partial is added to zero, then the terms in the same order)
void nmf_gram_reg(planc_gpu_ctx* c, const double* G, double l2, double l1, double diag,
                  double* out) {
  const int k = c->k;
  launch(c, KC_NORMGRAM, [&] {
    k_nmf_gram<<<(unsigned)((k * k + 7) / 8), 256, 0, c->stream>>>(G, 1, k, l2, l1, diag, out);
  });
}

// The objective from the Grams of the final W and H: `gw` / `gh` form them
// here, otherwise nmf_GW / nmf_GH already hold them.
void nmf_error(planc_gpu_ctx* c, bool gw, bool gh) {
  const int64_t m = c->dims[0], n = c->dims[1];
  if (gw) nmf_gram(c, c->F[0], m, 0, 0, 0, c->nmf_GW);
  if (gh) nmf_gram(c, c->F[1], n, 0, 0, 0, c->nmf_GH);
  NmfReg reg{c->nmf_reg[0], c->nmf_reg[1], c->nmf_reg[2], c->nmf_reg[3], c->nmf_reg[4]};
  const unsigned nb =
      (unsigned)std::min<int64_t>((std::max(m, n) + NMFE_WARPS - 1) / NMFE_WARPS, NMFW_MAX_BLOCKS);
  launch(c, KC_ERROR, [&] {
    k_nmf_error<<<nb, 32 * NMFE_WARPS, 0, c->stream>>>(
        c->F[0], m, c->F[1], n, c->k, c->M[1], c->nmf_GW, c->nmf_GH, c->normX2, reg,
        c->nmf_part, c->nmf_ctr + 1, c->nmf_obj, c->nmf_rel, c->nmf_ctr);
  });
}

// One iteration of HALSNMF / MUNMF / BPPNMF::computeNMF. HALS and MU find
// A^T W of the current W in M[1] (left there by the previous iteration's
// objective, or computed before the first). A factor's Gram is formed once
// per change of the factor: the unregularised W^T W / H^T H in nmf_GW /
// nmf_GH serve both the next update (regularised by nmf_gram_reg) and the
// objective; before the first iteration nmf_prereq_gram forms the one the
// first update needs.
void nmf_iteration(planc_gpu_ctx* c, int algo) {
  const int64_t m = c->dims[0], n = c->dims[1];
  const double* r = c->nmf_reg;
  const double sym = r[4];
  if (algo == PLANC_GPU_HALS || algo == PLANC_GPU_MU) {
    // H <- f(H, A^T W, W^T W + regH)   (nmf/hals.hpp:60-76, nmf/mu.hpp:60-68)
    nmf_gram_reg(c, c->nmf_GW, r[2], r[3], 0, c->nmf_G);
    nmf_row_update(c, algo, c->F[1], c->M[1], n);
    // W <- f(W, A H, H^T H + regW)     (nmf/hals.hpp:82-106, nmf/mu.hpp:72-80)
    nmf_AH(c);
    nmf_gram(c, c->F[1], n, 0, 0, 0, c->nmf_GH);
    nmf_gram_reg(c, c->nmf_GH, r[0], r[1], 0, c->nmf_G);
    if (algo == PLANC_GPU_HALS) {
      nmf_hals_w(c);
      nmf_normalize(c);  // rescales H too: both Grams are formed again
    } else {
      nmf_row_update(c, algo, c->F[0], c->M[0], m);
    }
    nmf_AtW(c);
    nmf_error(c, true, algo == PLANC_GPU_HALS);
  } else {
    // ANLS: W from (H^T H + regW, H^T A^T), then H from (W^T W + regH, W^T A),
    // each with the symmetric regularisation when set (nmf/bppnmf.hpp:24-80,
    // 208-214)
    nmf_AH(c);
    nmf_gram_reg(c, c->nmf_GH, r[0], r[1], sym, c->nmf_G);
    if (sym > 0)
      launch(c, KC_UPDATE, [&] {
        k_nmf_axpy<<<elem_grid(m * c->k), 256, 0, c->stream>>>(c->M[0], c->F[1], m * c->k, sym);
      });
    nmf_row_update(c, algo, c->F[0], c->M[0], m);
    nmf_AtW(c);
    nmf_gram(c, c->F[0], m, 0, 0, 0, c->nmf_GW);
    nmf_gram_reg(c, c->nmf_GW, r[2], r[3], sym, c->nmf_G);
    if (sym > 0)
      launch(c, KC_UPDATE, [&] {
        k_nmf_axpy<<<elem_grid(n * c->k), 256, 0, c->stream>>>(c->M[1], c->F[0], n * c->k, sym);
      });
    nmf_row_update(c, algo, c->F[1], c->M[1], n);
    if (sym > 0) nmf_AtW(c);  // the objective takes A^T W without the shift
    nmf_error(c, false, true);
  }
}

// Before a run's first iteration: the Gram the first update reads (W^T W
// for HALS / MU, H^T H for ANLS/BPP), unregularised.
void nmf_prereq_gram(planc_gpu_ctx* c, int algo) {
  if (algo == PLANC_GPU_ANLSBPP)
    nmf_gram(c, c->F[1], c->dims[1], 0, 0, 0, c->nmf_GH);
  else
    nmf_gram(c, c->F[0], c->dims[0], 0, 0, 0, c->nmf_GW);
}

void require_nmf(planc_gpu_ctx* c) {
  if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
  if (!c->have_tensor || c->N != 2) fail(PLANC_GPU_ERR_STATE, "NMF needs a matrix (2-way tensor)");
  if (!c->nmf_have) fail(PLANC_GPU_ERR_STATE, "no NMF factors set");
}

}  // namespace

extern "C" {

int planc_gpu_nmf_set_factors(planc_gpu_ctx* c, const double* W, const double* H, int k) {
  return guarded([&] {
    if (!c || !W || !H) fail(PLANC_GPU_ERR_ARG, "null argument");
    if (!c->have_tensor || c->N != 2) fail(PLANC_GPU_ERR_STATE, "set a matrix (2-way tensor) first");
    if (k < 1 || k > kMaxRank)
      fail(PLANC_GPU_ERR_UNSUPPORTED, "rank must be in [1, " + std::to_string(kMaxRank) + "]");
    set_device(c);
    reset_graph(c);
    if (k != c->k) {
      free_update_state(c);
      for (int i = 0; i < kMaxModes; ++i) c->factor_cap[i] = 0;
    }
    c->k = k;
    const double* src[2] = {W, H};
    for (int i = 0; i < 2; ++i) {
      const size_t need = (size_t)c->dims[i] * k;
      if (c->factor_cap[i] != (int64_t)need) {
        dalloc(&c->F[i], need);
        dalloc(&c->M[i], need);
        c->factor_cap[i] = (int64_t)need;
        c->buf_epoch++;
      }
      CK(cudaMemcpyAsync(c->F[i], src[i], need * 8, cudaMemcpyHostToDevice, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    c->have_factors = false;  // the NTF factors (normalised, with Grams) are not these
    c->nmf_have = true;
  });
}

int planc_gpu_nmf_set_regularization(planc_gpu_ctx* c, const double* regW, const double* regH,
                                     double symm_reg) {
  return guarded([&] {
    if (!c) fail(PLANC_GPU_ERR_ARG, "null context");
    double r[5] = {regW ? regW[0] : 0.0, regW ? regW[1] : 0.0, regH ? regH[0] : 0.0,
                   regH ? regH[1] : 0.0, symm_reg};
    for (double v : r)
      if (!(v >= 0) || !std::isfinite(v)) fail(PLANC_GPU_ERR_ARG, "regularisation must be >= 0");
    if (std::memcmp(r, c->nmf_reg, sizeof(r)) != 0) {
      std::memcpy(c->nmf_reg, r, sizeof(r));
      if (c->nmf_gexec) cudaGraphExecDestroy(c->nmf_gexec);  // the weights are launch arguments
      c->nmf_gexec = nullptr;
      c->nmf_galgo = -1;
    }
  });
}

int planc_gpu_nmf_run(planc_gpu_ctx* c, int algo, int iters, double* objective,
                      double* rel_error) {
  return guarded([&] {
    require_nmf(c);
    if (iters < 0) fail(PLANC_GPU_ERR_ARG, "iters < 0");
    if (algo != PLANC_GPU_MU && algo != PLANC_GPU_HALS && algo != PLANC_GPU_ANLSBPP)
      fail(PLANC_GPU_ERR_ARG, "NMF takes MU, HALS or ANLS/BPP");
    if (c->nmf_reg[4] > 0 && c->dims[0] != c->dims[1])
      fail(PLANC_GPU_ERR_ARG, "symmetric regularisation needs a square matrix");
    if (iters == 0) return;
    set_device(c);
    ensure_nmf(c, iters);
    if (c->nmf_gepoch != c->buf_epoch && c->nmf_gexec) {
      cudaGraphExecDestroy(c->nmf_gexec);
      c->nmf_gexec = nullptr;
      c->nmf_galgo = -1;
    }
    CK(cudaMemsetAsync(c->nmf_ctr, 0, sizeof(int), c->stream));
    if (algo == PLANC_GPU_HALS) nmf_normalize(c);  // HALSNMF's constructor, nmf/hals.hpp:44-48
    if (algo != PLANC_GPU_ANLSBPP) nmf_AtW(c);
    nmf_prereq_gram(c, algo);
    if (!c->timing) {
      if (!c->nmf_gexec || c->nmf_galgo != algo) {
        if (c->nmf_gexec) cudaGraphExecDestroy(c->nmf_gexec);
        c->nmf_gexec = nullptr;
        cudaGraph_t graph;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        try {
          nmf_iteration(c, algo);
        } catch (...) {
          c->capturing = false;
          cudaStreamEndCapture(c->stream, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        c->capturing = false;
        CK(cudaStreamEndCapture(c->stream, &graph));
        cudaError_t e = cudaGraphInstantiate(&c->nmf_gexec, graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "cudaGraphInstantiate (NMF)");
        c->nmf_galgo = algo;
        c->nmf_gepoch = c->buf_epoch;
      }
      for (int it = 0; it < iters; ++it) CK(cudaGraphLaunch(c->nmf_gexec, c->stream));
    } else {
      for (int it = 0; it < iters; ++it) nmf_iteration(c, algo);
    }
    // MUNMF / BPPNMF normalise by W after the loop (nmf/mu.hpp:90,
    // nmf/bppnmf.hpp:240)
    if (algo != PLANC_GPU_HALS) nmf_normalize(c);
    if (objective)
      CK(cudaMemcpyAsync(objective, c->nmf_obj, iters * sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
    if (rel_error)
      CK(cudaMemcpyAsync(rel_error, c->nmf_rel, iters * sizeof(double), cudaMemcpyDeviceToHost,
                         c->stream));
    check_status(c);
    drain_timing(c);
  });
}

int planc_gpu_nmf_get_factors(planc_gpu_ctx* c, double* W, double* H) {
  return guarded([&] {
    require_nmf(c);
    set_device(c);
    if (W)
      CK(cudaMemcpyAsync(W, c->F[0], (size_t)c->dims[0] * c->k * 8, cudaMemcpyDeviceToHost,
                         c->stream));
    if (H)
      CK(cudaMemcpyAsync(H, c->F[1], (size_t)c->dims[1] * c->k * 8, cudaMemcpyDeviceToHost,
                         c->stream));
    CK(cudaStreamSynchronize(c->stream));
  });
}

}  // extern "C"
