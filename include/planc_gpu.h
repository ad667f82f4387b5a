/* planc_gpu.h -- C ABI of the B200 (sm_100a) implementation of PLANC's
 * shared-memory NTF iteration (AUNTF with MU / HALS / ANLS-BPP updates and the
 * dimension-tree MTTKRP).
 *
 * Plain C types only: pointers, sizes and status codes. One context owns one
 * device-resident tensor, one set of CP factors and one CUDA stream. A
 * context is not thread-safe; distinct contexts are independent.
 *
 * Layouts (the reference's own memory layouts):
 *   tensor X : dense, column-major with mode 0 fastest
 *              (reference common/tensor.hpp:22-28, Tensor::m_data).
 *   factors  : row-major I_n x k, rank index fastest. This is the memory of
 *              the reference's ncp_mttkrp_t[n] (k x I_n column-major,
 *              ntf/auntf.hpp:95) and of the dimension-tree factors
 *              (dimtree/ddt.hpp:84-88); an Armadillo I_n x k factor
 *              (NCPFactors::factor) is its transpose in memory.
 *   k x k    : symmetric.
 *
 * Every function returns PLANC_GPU_OK (0) or a negative status; the message
 * of the last failure on the calling thread is planc_gpu_last_error(). The
 * reference reports the same failures with exit() (dimtree/dimtrees.hpp:48-64,
 * nnls/bppnnls.hpp:185-188) and assert (common/ncpfactors.hpp:113).
 */
#ifndef PLANC_GPU_H_
#define PLANC_GPU_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PLANC_GPU_ABI_VERSION 1

/* status codes */
#define PLANC_GPU_OK 0
#define PLANC_GPU_ERR_ARG (-1)         /* bad argument / shape */
#define PLANC_GPU_ERR_CUDA (-2)        /* CUDA runtime or driver error */
#define PLANC_GPU_ERR_STATE (-3)       /* call out of order (no tensor, no factors) */
#define PLANC_GPU_ERR_BPP_MAXITER (-4) /* BPP hit its 5k iteration cap ("BPP failed") */
#define PLANC_GPU_ERR_NONFINITE (-5)   /* NaN/Inf met in a solve */
#define PLANC_GPU_ERR_TIMEOUT (-6)     /* a bounded device wait ran out */
#define PLANC_GPU_ERR_UNSUPPORTED (-7) /* shape/rank outside what the kernels take */
#define PLANC_GPU_ERR_OOM (-8)         /* device allocation failed */
#define PLANC_GPU_ERR_SINGULAR (-9)    /* a normal-equation solve found no pivot */
#define PLANC_GPU_ERR_MAXITER (-10)    /* a Nesterov update reached its inner step cap */

/* MTTKRP precision. The Gram matrices, the factor updates, the BPP solves and
 * the error are FP64 in every mode. */
#define PLANC_GPU_PREC_FP64 0   /* FP64 tensor, FP64 contraction (plain path) */
#define PLANC_GPU_PREC_BF16 1   /* BF16 tensor, split-BF16 (hi+lo) factors, FP32 accumulate */
#define PLANC_GPU_PREC_BF16X2 2 /* tensor split into BF16 hi+lo, 3 products, FP32 accumulate */

/* update algorithms: values of the reference's algotype (common/utils.h:10) */
#define PLANC_GPU_MU 0
#define PLANC_GPU_HALS 1
#define PLANC_GPU_ANLSBPP 2
#define PLANC_GPU_AOADMM 4    /* NTFAOADMM, ntf/ntfaoadmm.hpp:23-77 */
#define PLANC_GPU_NESTEROV 5  /* NTFNES, ntf/ntfnes.hpp:11-166 */

/* element types of a tensor handed to planc_gpu_set_tensor */
#define PLANC_GPU_F64 0
#define PLANC_GPU_F32 1

typedef struct planc_gpu_ctx planc_gpu_ctx;

/* ABI version (PLANC_GPU_ABI_VERSION of the built library). */
int planc_gpu_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* planc_gpu_last_error(void);

/* Creates a context on `device`. `cuda_stream` is a cudaStream_t to run on
 * (NULL: the context creates and owns a non-blocking stream). */
int planc_gpu_create(planc_gpu_ctx** out, int device, int precision, void* cuda_stream);

/* Releases all device memory of the context. NULL is accepted. */
int planc_gpu_destroy(planc_gpu_ctx* ctx);

/* The CUDA stream the context launches on (as a cudaStream_t). */
void* planc_gpu_stream(planc_gpu_ctx* ctx);

/* Uploads the tensor (replaces Tensor(dims) / Tensor::read as the input of
 * AUNTF(const Tensor&, ...), ntf/auntf.hpp:83-105). X has prod(dims)
 * elements of `dtype`, column-major with mode 0 fastest; `x_on_device` != 0
 * means X is a device pointer on the context's device. ||X||^2 is computed in
 * FP64 from the values given (Tensor::norm, common/tensor.hpp:350-356). */
int planc_gpu_set_tensor(planc_gpu_ctx* ctx, const void* X, int dtype,
                         const int64_t* dims, int nmodes, int x_on_device);

/* Injects CP factors as AUNTF::reset(new_factors, false) does
 * (ntf/auntf.hpp:186-198): each mode is column-normalised
 * (NCPFactors::normalize(int), common/ncpfactors.hpp:346-351), then lambda is
 * set to `lambda` (k values; NULL means all ones). F[n] is row-major
 * I_n x k (host memory). Sets the rank k (1 <= k <= 64). */
int planc_gpu_set_factors(planc_gpu_ctx* ctx, const double* const* F,
                          const double* lambda, int k);

/* Runs `iters` outer iterations of AUNTF::computeNTF (ntf/auntf.hpp:128-177)
 * with update `algo` (PLANC_GPU_MU / HALS / ANLSBPP / AOADMM / NESTEROV).
 * `dimtree` != 0 uses the dimension tree (N in {3,4}; ddt.hpp:134-243), else
 * the direct MTTKRP (common/tensor.hpp:246-327). With `compute_error` != 0,
 * errs_out[it] receives the relative error after iteration it
 * (auntf.hpp:165-170), in the FP64 Gram form ||X||^2 - 2<X,M> + ||M||^2.
 * errs_out may be NULL. NESTEROV evaluates the error every iteration in any
 * case and, from iteration 6 of the call on, extrapolates the factors and
 * keeps the extrapolation when it lowers the error (NTFNES::accelerate,
 * ntf/ntfnes.hpp:64-98). AOADMM and NESTEROV keep per-mode state in the
 * context between calls, as the reference's solver objects do
 * (planc_gpu_reset_update_state clears it). */
int planc_gpu_run(planc_gpu_ctx* ctx, int algo, int iters, int dimtree,
                  int compute_error, double* errs_out);

/* Copies the current (normalised) factors and lambda to host memory
 * (AUNTF::ncp_factors(), ntf/auntf.hpp:118). F[n]: row-major I_n x k; either
 * argument may be NULL. */
int planc_gpu_get_factors(planc_gpu_ctx* ctx, double* const* F, double* lambda);

/* MTTKRP of mode n with the current factors, row-major I_n x k (host):
 * with `dimtree` != 0 through the dimension tree (the partial MTTKRP is
 * recomputed from the current factors), else the direct form
 * (ntf_utils.hpp:49-53 / tensor.hpp:246-327). */
int planc_gpu_mttkrp(planc_gpu_ctx* ctx, int mode, int dimtree, double* out);

/* Hadamard product of the Grams of all modes except n, k x k (host):
 * NCPFactors::gram_leave_out_one, common/ncpfactors.hpp:139-148. */
int planc_gpu_gram_loo(planc_gpu_ctx* ctx, int mode, double* out);

/* Relative error of the current factors and lambda
 * (AUNTF::computeObjectiveError, ntf/auntf.hpp:200-246), FP64 Gram form. */
int planc_gpu_objective_error(planc_gpu_ctx* ctx, double* err);

/* Per-mode extension point for host-side factor updates (the reference's
 * virtual MAT AUNTF::update(int mode), ntf/auntf.hpp:45): mode_begin computes
 * the leave-one-out Gram and the MTTKRP of `mode` from the current factors
 * (the steps of auntf.hpp:132-151) and copies them to the host (either
 * pointer may be NULL); mode_end takes the new, unnormalised factor (row-major
 * I_n x k, host) and applies AUNTF::update_factor_mode (auntf.hpp:66-79). */
int planc_gpu_mode_begin(planc_gpu_ctx* ctx, int mode, int dimtree,
                         double* gram_out, double* mttkrp_out);
int planc_gpu_mode_end(planc_gpu_ctx* ctx, int mode, const double* factor);

/* BPP NNLS on the device for host inputs: solves min ||A x - b|| s.t. x >= 0
 * for `ncols` right-hand sides from the normal equations, as
 * BPPNNLS<MAT,VEC>(AtA, AtB, true).solveNNLS() (nnls/bppnnls.hpp:67-191,
 * nnls/nnls.hpp:100-131). AtA: n x n; AtB and X: column-major n x ncols;
 * passive (may be NULL): n x ncols final passive-set mask; iters (may be
 * NULL): per-column BPP iteration counts. 1 <= n <= 64. */
int planc_gpu_bpp_solve(planc_gpu_ctx* ctx, const double* AtA, const double* AtB,
                        int n, int64_t ncols, double* X, int32_t* passive,
                        int32_t* iters);

/* ---- The differentiable CP loss 1/2 ||X - [[F_0..F_{N-1}]]||^2 on the
 * context's tensor, for caller-supplied DEVICE factors (row-major I_n x k
 * FP64; k and the mode sizes those of the context). Its gradient is the
 * reference's NTF gradient form (ntf/ntfnes.hpp:138-147, G_{-n} H^T - M^T in
 * the reference's k x I layout). Ordered on the context's stream. */

/* G_out (device, N x k x k) = F_n^T F_n of every factor, and *loss_out
 * (device) = 1/2 ||X||^2 - <M0, F_0> + 1/2 sum_ab prod_n G_n[a, b], with M0
 * the mode-0 MTTKRP of these factors (planc_gpu_mttkrp_device). */
int planc_gpu_cp_loss_device(planc_gpu_ctx* ctx, const double* const* F_dev, const double* M0_dev,
                             double* G_out, double* loss_out);

/* grad_dev[n] = g (F_n (prod_{m != n} G_m) - M_dev[n]) for every mode, with
 * G from planc_gpu_cp_loss_device, M_dev[n] the mode-n MTTKRPs and g the
 * device scalar at g_dev (the upstream gradient). */
int planc_gpu_cp_grads_device(planc_gpu_ctx* ctx, const double* const* F_dev, const double* G,
                              const double* const* M_dev, const double* g_dev,
                              double* const* grad_dev);

/* One projected accelerated gradient step on every factor:
 * Fnew[n] = max(Y[n] - eta grad[n], 0), Ynew[n] = Fnew[n] + mom (Fnew[n] - Fprev[n])
 * (element-wise; outputs may alias the inputs of the same factor). */
int planc_gpu_cp_step_device(planc_gpu_ctx* ctx, const double* const* Y, const double* const* grad,
                             const double* const* Fprev, double eta, double mom, double* const* Fnew,
                             double* const* Ynew);

/* ---- Device building blocks of the distributed NTF iteration (one slab of
 * the tensor per GPU; the caller runs the collectives between them). The
 * reference's distributed loop, distntf/distauntf.hpp, reduce-scatters the
 * partial MTTKRP (:305-315), updates its rows, all-reduces the column norms
 * and the k x k Grams (:92-115, ncpfactors.hpp distributed_normalize) and
 * all-gathers the factor (:164-234). All buffers are DEVICE memory, FP64,
 * row-major rows x k (k x k for Grams), on the context's device; the calls
 * are ordered on the context's stream and return without synchronising
 * (planc_gpu_sync waits and reports device-side failures). */

/* Updates `rows` rows of the factor block H in place from the matching rows
 * of the MTTKRP block M and the leave-one-out Gram G (k x k): NTFMU /
 * NTFHALS / NTFANLSBPP::update (ntf/ntfmu.hpp:11-16, ntfhals.hpp:13-29,
 * ntfanlsbpp.hpp:15-57) restricted to the block; the updates are row-separable. */
int planc_gpu_update_device(planc_gpu_ctx* ctx, int algo, double* H, const double* M,
                            const double* G, int64_t rows, int k);

/* G = F^T F of a rows x k block (un-normalised; deterministic order). */
int planc_gpu_gram_device(planc_gpu_ctx* ctx, const double* F, int64_t rows, int k, double* G);

/* From G_in = the factor's whole un-normalised Gram (summed over every block):
 * lambda_r = sqrt(G_in_rr), G_out = Gram of the normalised factor, and the
 * block F (rows x k) scaled column by column (NCPFactors::normalize(mode),
 * common/ncpfactors.hpp:346-351, columns of zero norm left as they are).
 * rows may be 0 (no block on this device). */
int planc_gpu_normalize_device(planc_gpu_ctx* ctx, double* F, int64_t rows, int k,
                               const double* G_in, double* lambda, double* G_out);

/* out_r = sum_i A[i, r] B[i, r] (k values): a block's share of <X, model>
 * in the Gram-form error (distntf/distauntf.hpp:685-727). */
int planc_gpu_coldot_device(planc_gpu_ctx* ctx, const double* A, const double* B, int64_t rows,
                            int k, double* out);

/* Waits for the context's stream and reports a device-side failure of the
 * work queued before it (BPP cap, non-finite values, ...), as the run calls do. */
int planc_gpu_sync(planc_gpu_ctx* ctx);

/* MTTKRP of `mode` for caller-supplied DEVICE factors F_dev[n] (row-major
 * I_n x k FP64, k = the rank set by planc_gpu_set_factors, on the context's
 * device), written to the device buffer M_dev (row-major I_mode x k FP64).
 * The context's own factors are not touched. flags: bit 0 = dimension tree
 * (N in {3,4}); bit 1 = reuse the partial MTTKRPs left by the previous calls
 * of the modes before `mode` in its branch of the tree, made in order with the
 * same factors (the in-order reuse of
 * DenseDimensionTree::in_order_reuse_MTTKRP, dimtree/ddt.hpp:134-243); without
 * it those modes' partial contractions are recomputed first. Runs on the context's stream and returns without
 * synchronising. This is the adjoint used by the differentiable CP loss. */
int planc_gpu_mttkrp_device(planc_gpu_ctx* ctx, int mode, const double* const* F_dev,
                            double* M_dev, int flags);

/* ||X||^2 of the context's tensor in FP64 (Tensor::norm,
 * common/tensor.hpp:350-356), written to host memory. */
int planc_gpu_tensor_norm2(planc_gpu_ctx* ctx, double* out);

/* ---- Batched factorisation of many independent tensors (uneven shapes and
 * ranks). Each member is a context bound to one of `nstreams` worker streams;
 * one outer iteration of every member is captured into a single CUDA graph,
 * launched once per iteration, so the members' kernels overlap. Members use
 * the dimension tree (N in {3,4}). The reference factorises tensors one at a
 * time with AUNTF::computeNTF (ntf/auntf.hpp:128-177); the batch runs the same
 * iteration for each member. */
typedef struct planc_gpu_batch planc_gpu_batch;
int planc_gpu_batch_create(planc_gpu_batch** out, int device, int precision, int nstreams);
/* Adds a member: tensor as planc_gpu_set_tensor, factors as
 * planc_gpu_set_factors (lambda = ones); *index receives its position. */
int planc_gpu_batch_add(planc_gpu_batch* b, const void* X, int dtype, const int64_t* dims,
                        int nmodes, int x_on_device, const double* const* F, int k, int* index);
int planc_gpu_batch_count(planc_gpu_batch* b);
int planc_gpu_batch_set_factors(planc_gpu_batch* b, int index, const double* const* F, int k);
/* `iters` iterations of every member; errs (may be NULL) receives
 * count x iters relative errors, member-major. */
int planc_gpu_batch_run(planc_gpu_batch* b, int algo, int iters, int compute_error, double* errs);
int planc_gpu_batch_get_factors(planc_gpu_batch* b, int index, double* const* F, double* lambda);
/* Times the batch graph under candidate settings per member size class and
 * keeps the fastest: the per-launch parallelism (fraction of the SMs a
 * member's launch is sized for) and, for the tensor-core precisions, the
 * split-K length of the left contraction (fewest 64-element chunks per
 * partial: 0, 8, 32 or 128). Members' factors are unchanged; a tensor-core
 * batch's later results may differ from the untuned ones by the rounding of
 * the reordered FP32 partial sums. best_ms (may be NULL) receives the tuned
 * time of one batched iteration. A batch whose members are all 3-way
 * tensor-core contexts running MU or HALS runs each phase of an iteration as
 * one launch for all members (PLANC_GPU_BATCH_GROUPED=0 turns that off). */
int planc_gpu_batch_autotune(planc_gpu_batch* b, int algo, int trials, double* best_ms);
int planc_gpu_batch_destroy(planc_gpu_batch* b);

/* MTTKRP of the last mode, allocation-free. No counterpart in the reference:
 * this entry point exists for callers that cannot allocate device memory when
 * they call the library -- applications whose GPU memory is reserved up front
 * by a pool allocator (a cudaMalloc would fail or escape the pool), and
 * latency-critical loops that must not pay the device-wide synchronisation a
 * cudaMalloc/cudaFree can imply. It makes no allocation of any kind: the
 * split-K partials go to a fixed 8 MiB device array (2^20 doubles) that every
 * GPU loading the library holds until exit.
 *   out[j, r] = sum_l X[l + L*j] * KRP(F_0..F_{N-2})[l, r],  j < I_{N-1}
 * with L = I_0 * ... * I_{N-2}, in FP64. X_dev:
 * device tensor, FP64, mode 0 fastest; F_dev[n] (n < N-1): device factors,
 * row-major I_n x k FP64; out_dev: device I_{N-1} x k FP64, row-major. The
 * caller passes all of them; I_{N-1} * k above 2^20 is rejected with
 * PLANC_GPU_ERR_UNSUPPORTED. Runs on `cuda_stream` on the current device and
 * returns without synchronising. All calls share the one array: calls that
 * overlap on the GPU (different streams or threads at once) race and must be
 * serialised by the caller. The first call on a device resolves the array's
 * device address (cudaGetSymbolAddress) and keeps it for the life of the
 * process; make that first call before any stream capture. A device reset
 * (cudaDeviceReset, or the primary context released and created again)
 * reloads the module and invalidates the kept address: do not call this entry
 * point on a device after resetting it. */
int planc_gpu_mttkrp_last_mode_noalloc(const double* X_dev, const int64_t* dims, int nmodes,
                                       const double* const* F_dev, int k, double* out_dev,
                                       void* cuda_stream);

/* ---- Shared-memory NMF of a dense matrix, A ~ W H^T (reference
 * common/nmf.hpp, nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp). A is the
 * context's tensor with two modes: planc_gpu_set_tensor(ctx, A, dtype,
 * {m, n}, 2, ...) with A column-major m x n (an Armadillo MAT). W is m x k
 * and H is n x k, both row-major here (the memory of the reference's W^T and
 * H^T). A H and A^T W are the tensor's mode-0 / mode-1 MTTKRPs (FP64, or the
 * tensor-core contraction at BF16 / split-BF16); Grams, updates and the
 * objective are FP64. */

/* Sets W and H as given, unnormalised: the NMF(A, W, H) constructor
 * (common/nmf.hpp:193-210). 1 <= k <= 64. */
int planc_gpu_nmf_set_factors(planc_gpu_ctx* ctx, const double* W, const double* H, int k);

/* Regularisation of the next runs (NMF::regW / regH / symm_reg,
 * common/nmf.hpp:467-480): regW = {L2, L1} and regH = {L2, L1} (NULL: none),
 * symm_reg > 0 (square A only) adds symm_reg I to the Grams and symm_reg *
 * the other factor to the right-hand sides of BPP (common/nmf.hpp:118-124)
 * and symm_reg ||W - H||^2 to the objective. All >= 0. */
int planc_gpu_nmf_set_regularization(planc_gpu_ctx* ctx, const double* regW, const double* regH,
                                     double symm_reg);

/* `iters` iterations of HALSNMF / MUNMF / BPPNMF::computeNMF
 * (nmf/hals.hpp:50-110, nmf/mu.hpp:55-92, nmf/bppnmf.hpp:190-240) with algo
 * PLANC_GPU_HALS / MU / ANLSBPP. HALS normalises by W first, as its
 * constructor does; MU and ANLS/BPP normalise by W after the last iteration.
 * objective[it] and rel_error[it] (either may be NULL) receive
 * NMF::computeObjectiveError's objective and sqrt(fit) / ||A|| after
 * iteration it (common/nmf.hpp:386-431). */
int planc_gpu_nmf_run(planc_gpu_ctx* ctx, int algo, int iters, double* objective,
                      double* rel_error);

/* Copies W (m x k) and H (n x k), row-major, to host memory
 * (getLeftLowRankFactor / getRightLowRankFactor, common/nmf.hpp:214-215);
 * either may be NULL. */
int planc_gpu_nmf_get_factors(planc_gpu_ctx* ctx, double* W, double* H);

/* Lowers the BPP iteration cap (0 restores the reference's 5k,
 * nnls/bppnnls.hpp:69). Used to exercise the "BPP failed" path
 * (PLANC_GPU_ERR_BPP_MAXITER) without a pathological input. */
int planc_gpu_set_bpp_max_iter(planc_gpu_ctx* ctx, int max_iter);

/* ANLS/BPP row solves of planc_gpu_run start from the passive set of the
 * factor being replaced (enable = 1, the default) or from the empty set as
 * NTFANLSBPP::update does (enable = 0, nnls/bppnnls.hpp:73-74). G is
 * positive definite, so the NNLS optimum is unique and BPP reaches it from
 * any start: the factors are the same, only the number of exchange steps
 * drops. planc_gpu_bpp_solve always starts from the empty set. */
int planc_gpu_set_bpp_warm_start(planc_gpu_ctx* ctx, int enable);

/* Returns the AO-ADMM dual variables and the Nesterov proximal / previous
 * iterates, lambdas and acceleration counters to their initial state (zeros,
 * ones, acc_exp = 3), i.e. the state of a newly constructed NTFAOADMM / NTFNES
 * object (ntf/ntfaoadmm.hpp:79-89, ntf/ntfnes.hpp:169-194). A new tensor shape
 * or rank does the same. */
int planc_gpu_reset_update_state(planc_gpu_ctx* ctx);

/* Self-test of the kernels' bounded waits: launches one thread that waits on
 * a barrier nothing ever signals, with a limit of `seconds` (0 < s <= 5).
 * The wait runs out, the kernel writes the timeout status and returns; the
 * status the device wrote is returned in *status_out (PLANC_GPU_ERR_TIMEOUT
 * when the bounded-wait path works) and the device stays usable. */
int planc_gpu_selftest_wait_timeout(int device, double seconds, int* status_out);

/* Self-test of the cooperative NMF W sweep's bounded waits (its per-column
 * wait for every CTA's partial sum, the routine the sweep itself runs): a
 * cooperative launch of four CTAs in which one CTA never stores its sum. The
 * other CTAs' waits run out after a few thousand polls, raise the sweep's
 * error flag and the timeout status, and every CTA returns. *status_out
 * receives the status the device wrote (PLANC_GPU_ERR_TIMEOUT when the
 * bounded-wait path works); the device stays usable. */
int planc_gpu_selftest_coop_timeout(int device, int* status_out);

/* Kernel timing, for roofline measurement: while enabled, CUDA events bracket
 * every launch of each kernel class on the context's stream. Class ids:
 *   0 partial MTTKRP, right contraction (P = X * F_last) and direct mode 0,
 *   1 multi-TTV, 2 factor update, 3 normalise + Gram, 4 error,
 *   5 split-K reduction, 6 BPP, 7 operand preparation (tensor-core B image),
 *   8 partial MTTKRP, left contraction (X^T * KRP) and direct modes > 0.
 * get_kernel_times fills ms[c] and launches[c] for c < n and resets them. */
int planc_gpu_set_timing(planc_gpu_ctx* ctx, int enable);
int planc_gpu_get_kernel_times(planc_gpu_ctx* ctx, double* ms, int64_t* launches, int n);

/* Number of kernel launches the library issued on this context so far. */
int64_t planc_gpu_launch_count(planc_gpu_ctx* ctx);

/* Synthetic input: writes into device memory `X_dev` (prod(dims) elements of
 * `dtype`, mode 0 fastest) the CP model [[A_0, ..., A_{N-1}]] of rank k from
 * host factors A[n] (row-major I_n x k), plus i.i.d. Gaussian noise of
 * standard deviation `sigma` (counter-based Philox stream of `seed`),
 * clipped at >= 0 when `clip` != 0. This is the reference's Gen_Tensor noise
 * model (dimtree/ddttensor.hpp:899-985) with a reproducible generator. */
int planc_gpu_synth_cp_tensor(int device, void* X_dev, int dtype, const int64_t* dims,
                              int nmodes, const double* const* A, int k, double sigma,
                              uint64_t seed, int clip, void* cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* PLANC_GPU_H_ */
