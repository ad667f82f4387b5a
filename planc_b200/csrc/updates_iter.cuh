// updates_iter.cuh -- the iterative factor updates of the planc NTF solver
// family on the device: AO-ADMM (reference ntf/ntfaoadmm.hpp:23-77) and the
// Nesterov-accelerated proximal gradient with its outer extrapolation
// (ntf/ntfnes.hpp:11-166).
//
// Both updates are row-separable: every row of the I_n x k factor solves its
// own small problem with the shared k x k matrix (G + alpha I, or G + lambda I),
// and the rows only meet in global stopping tests (Frobenius norms for ADMM,
// max / min for Nesterov). A warp owns a row (lane c holds columns c and
// c + 32), the k x k matrix sits in shared memory.
//  * AO-ADMM runs its fixed maximum of 5 iterations as 5 launches; the last
//    CTA of each launch sums the per-CTA partial norms in a fixed order and
//    writes the stop flag that makes the remaining launches return at once.
//  * The Nesterov inner loop has a data-dependent length, so it runs inside
//    one thread-block cluster: each step ends with a cluster barrier, before
//    which every CTA stores its partial max / min into the shared memory of
//    every CTA of the cluster (distributed shared memory); after it each CTA
//    combines the partials from its own shared memory. Max and min are exact,
//    so every CTA takes the same decision. No CTA spins on memory; the
//    barrier is the hardware one. A partial slot is double-buffered by step
//    parity: a CTA can be at most one barrier ahead of another, so it never
//    overwrites a slot another CTA has still to read, and no CTA stores into
//    another after the last barrier, so CTAs may leave in any order.
#pragma once
#include <cooperative_groups.h>

#include "common.cuh"

namespace pg {

namespace cg = cooperative_groups;

constexpr int kStMaxIter = -10;  // an iterative update reached its step cap

// Shape of the cluster launches: 16 warps per CTA; 8 CTAs (a portable
// cluster) for the global-memory Nesterov loop, and 16 CTAs where the device
// runs clusters of 16 (8 otherwise) for the register-resident kernels.
constexpr int NES_CTAS = 8;
constexpr int NES_CTAS_MAX = 16;
constexpr int NES_THREADS = 512;

// ---------------------------------------------------------------------------
// AO-ADMM
// ---------------------------------------------------------------------------
constexpr int ADMM_WARPS = 8;        // rows in flight per CTA
constexpr int ADMM_MAX_BLOCKS = 296; // 2 CTAs per SM; partial-norm buffer size

// alpha = trace(G) / k (0.01 if not positive) and L = chol(G + alpha I),
// lower (ntfaoadmm.hpp:29-35); resets the stop flag and the CTA counter.
// One CTA. A non-positive pivot (chol() failure in the reference) sets
// kStSingular.
__global__ void __launch_bounds__(256) k_admm_prep(const double* __restrict__ G, int k,
                                                   double* __restrict__ Lg,
                                                   double* __restrict__ scal, int* __restrict__ flag,
                                                   int* __restrict__ counter, int* __restrict__ status) {
  __shared__ double T[kMaxRank * (kMaxRank + 1)];
  __shared__ double s_alpha;
  __shared__ int s_bad;
  constexpr int LD = kMaxRank + 1;
  const int tid = threadIdx.x;
  if (tid == 0) {
    double tr = 0.0;
    for (int i = 0; i < k; ++i) tr += G[i * k + i];
    double a = tr / k;
    s_alpha = (a > 0) ? a : 0.01;
    s_bad = 0;
  }
  __syncthreads();
  for (int e = tid; e < k * k; e += blockDim.x) {
    const int i = e / k, j = e % k;
    T[i * LD + j] = G[e] + (i == j ? s_alpha : 0.0);
  }
  __syncthreads();
  // left-looking (dot-product) Cholesky, column j after columns < j
  for (int j = 0; j < k; ++j) {
    if (tid == 0) {
      double d = T[j * LD + j];
      for (int p = 0; p < j; ++p) d -= T[j * LD + p] * T[j * LD + p];
      if (!(d > 0.0)) s_bad = 1;
      T[j * LD + j] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    const double ljj = T[j * LD + j];
    for (int i = j + 1 + tid; i < k; i += blockDim.x) {
      double v = T[i * LD + j];
      for (int p = 0; p < j; ++p) v -= T[i * LD + p] * T[j * LD + p];
      T[i * LD + j] = v / ljj;
    }
    __syncthreads();
  }
  for (int e = tid; e < k * k; e += blockDim.x) {
    const int i = e / k, j = e % k;
    Lg[e] = j <= i ? T[i * LD + j] : 0.0;
  }
  if (tid == 0) {
    scal[0] = s_alpha;
    *flag = 0;
    *counter = 0;
    if (s_bad) atomicCAS(status, 0, kStSingular);
  }
}

// Selects register slot `p` of a lane's row slice with a compile-time index.
template <int PER>
__device__ __forceinline__ double slot_get(const double (&v)[PER], int p) {
  double r = v[0];
#pragma unroll
  for (int q = 1; q < PER; ++q)
    if (p == q) r = v[q];
  return r;
}

// One ADMM iteration over all rows (ntfaoadmm.hpp:40-72):
//   x   = (G + alpha I)^{-1} (m + alpha (h + u))  [two triangular solves]
//   h'  = max(x - u, 0),  u' = (u + h') - x
// plus the four squared norms of the stopping test. Returns at once when the
// previous launch set the stop flag; the last CTA to finish combines the
// per-CTA partials in CTA order and writes the flag for the next launch.
template <int KP>
__global__ void __launch_bounds__(32 * ADMM_WARPS) k_admm_step(
    double* __restrict__ H, double* __restrict__ U, const double* __restrict__ M,
    const double* __restrict__ Lg, const double* __restrict__ scal, int64_t I, int k, double tol,
    int* __restrict__ flag, double* __restrict__ part, int* __restrict__ counter) {
  if (*flag) return;  // written by the previous launch; uniform over the grid
  constexpr int PER = KP / 32;
  constexpr int LD = KP + 1;  // odd stride: row and column walks are conflict-free
  __shared__ double Ls[KP * LD];
  __shared__ double rinv[KP];
  __shared__ double wred[ADMM_WARPS][4];
  __shared__ int s_last;
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) Ls[(e / k) * LD + e % k] = Lg[e];
  if (threadIdx.x < k) rinv[threadIdx.x] = 1.0 / Lg[threadIdx.x * k + threadIdx.x];
  __syncthreads();
  const double alpha = scal[0];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double s_fac = 0.0, s_dual = 0.0, s_r = 0.0, s_s = 0.0;
  for (int64_t row = (int64_t)blockIdx.x * ADMM_WARPS + warp; row < I;
       row += (int64_t)gridDim.x * ADMM_WARPS) {
    double h[PER], u[PER], y[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      h[p] = c < k ? H[row * k + c] : 0.0;
      u[p] = c < k ? U[row * k + c] : 0.0;
      const double m = c < k ? M[row * k + c] : 0.0;
      y[p] = m + alpha * (h[p] + u[p]);
    }
    // forward substitution with L (column-oriented, the order of dtrsm; the
    // diagonal enters as its reciprocal)
    for (int j = 0; j < k; ++j) {
      const double yj = __shfl_sync(0xffffffffu, slot_get<PER>(y, j >> 5), j & 31) * rinv[j];
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c == j)
          y[p] = yj;
        else if (c > j && c < k)
          y[p] -= yj * Ls[c * LD + j];
      }
    }
    // back substitution with L^T
    for (int j = k - 1; j >= 0; --j) {
      const double xj = __shfl_sync(0xffffffffu, slot_get<PER>(y, j >> 5), j & 31) * rinv[j];
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c == j)
          y[p] = xj;
        else if (c < j)
          y[p] -= xj * Ls[j * LD + c];
      }
    }
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      if (c < k) {
        double hn = y[p] - u[p];
        hn = hn > 0.0 ? hn : 0.0;
        const double un = (u[p] + hn) - y[p];
        s_fac = fma(hn, hn, s_fac);
        s_dual = fma(un, un, s_dual);
        const double d = hn - y[p];
        s_r = fma(d, d, s_r);
        const double e = hn - h[p];
        s_s = fma(e, e, s_s);
        H[row * k + c] = hn;
        U[row * k + c] = un;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s_fac += __shfl_xor_sync(0xffffffffu, s_fac, o);
    s_dual += __shfl_xor_sync(0xffffffffu, s_dual, o);
    s_r += __shfl_xor_sync(0xffffffffu, s_r, o);
    s_s += __shfl_xor_sync(0xffffffffu, s_s, o);
  }
  if (lane == 0) {
    wred[warp][0] = s_fac;
    wred[warp][1] = s_dual;
    wred[warp][2] = s_r;
    wred[warp][3] = s_s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < ADMM_WARPS; ++w)
      for (int q = 0; q < 4; ++q) t[q] += wred[w][q];
    for (int q = 0; q < 4; ++q) part[blockIdx.x * 4 + q] = t[q];
    __threadfence();
    s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // the last CTA adds the CTAs' partials, in parallel and in a fixed order
  __shared__ double sh[32 * ADMM_WARPS];
  double t[4];
  for (int q = 0; q < 4; ++q) {
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) v += part[b * 4 + q];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
      if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
      __syncthreads();
    }
    t[q] = sh[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double facnorm = sqrt(t[0]), dualnorm = sqrt(t[1]);
    const double r = sqrt(t[2]), s = sqrt(t[3]);
    *flag = (r < tol * facnorm && s < tol * dualnorm) ? 1 : 0;
    *counter = 0;
  }
}

// The whole AO-ADMM update of one mode in one cluster of NES_CTAS CTAs, for
// modes of at most R * 128 rows (every row's h, u and m in registers):
// alpha and the Cholesky factor (each CTA computes the same one), at most 5
// ADMM iterations whose stopping norms are summed per warp, per CTA (warp
// order) and over the cluster (CTA order) -- the same sums in every CTA, so
// every CTA takes the same decision -- then the column normalisation of the
// dual variable with column sums formed the same way. Writes the new factor
// (unnormalised) and the dual variable.
template <int KP, int R>
__global__ void __launch_bounds__(NES_THREADS, 1)
    k_admm_cluster(double* __restrict__ H, double* __restrict__ U, const double* __restrict__ M,
                   const double* __restrict__ G, int64_t I, int k, double tol,
                   int* __restrict__ status) {
  constexpr int PER = KP / 32;
  constexpr int NW = NES_THREADS / 32;
  constexpr int LD = KP + 1;
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ double Ls[KP * LD];
  __shared__ double wred[NW][4];
  // per-CTA partials pushed into every CTA of the cluster (remote shared-
  // memory stores before the cluster barrier), read back locally after it
  __shared__ double slot[2][NES_CTAS_MAX][4];
  static_assert((NW + NES_CTAS_MAX) * KP <= KP * LD, "column partials must fit in Ls");
  __shared__ double rinv[KP];
  __shared__ double s_alpha;
  __shared__ int s_bad;
  const int tid = threadIdx.x;
  // alpha = trace(G) / k (0.01 if not positive), L = chol(G + alpha I)
  // (ntfaoadmm.hpp:29-35), left-looking
  if (tid == 0) {
    double tr = 0.0;
    for (int i = 0; i < k; ++i) tr += G[i * k + i];
    const double a = tr / k;
    s_alpha = (a > 0) ? a : 0.01;
    s_bad = 0;
  }
  __syncthreads();
  const double alpha = s_alpha;
  for (int e = tid; e < k * k; e += NES_THREADS) {
    const int i = e / k, j = e % k;
    Ls[i * LD + j] = G[e] + (i == j ? alpha : 0.0);
  }
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    if (tid == 0) {
      double d = Ls[j * LD + j];
      for (int p = 0; p < j; ++p) d -= Ls[j * LD + p] * Ls[j * LD + p];
      if (!(d > 0.0)) s_bad = 1;
      Ls[j * LD + j] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncthreads();
    const double ljj = Ls[j * LD + j];
    for (int i = j + 1 + tid; i < k; i += NES_THREADS) {
      double v = Ls[i * LD + j];
      for (int p = 0; p < j; ++p) v -= Ls[i * LD + p] * Ls[j * LD + p];
      Ls[i * LD + j] = v / ljj;
    }
    __syncthreads();
  }
  if (s_bad && blockIdx.x == 0 && tid == 0) atomicCAS(status, 0, kStSingular);
  // reciprocal diagonal: the substitutions multiply by it (as OpenBLAS's
  // triangular-solve kernels do) instead of dividing on the dependency chain
  if (tid < k) rinv[tid] = 1.0 / Ls[tid * LD + tid];
  __syncthreads();

  const int lane = tid & 31, warp = tid >> 5;
  const int64_t stride = (int64_t)gridDim.x * NW;
  const int64_t row0 = (int64_t)blockIdx.x * NW + warp;
  double h[R][PER], u[R][PER], m[R][PER];
  bool live[R][PER];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t row = row0 + r * stride;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      live[r][p] = row < I && c < k;
      h[r][p] = live[r][p] ? H[row * k + c] : 0.0;
      u[r][p] = live[r][p] ? U[row * k + c] : 0.0;
      m[r][p] = live[r][p] ? M[row * k + c] : 0.0;
    }
  }
  for (int it = 0; it < 5; ++it) {  // admm_iter, ntfaoadmm.hpp:87
    double y[R][PER];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < PER; ++p) y[r][p] = m[r][p] + alpha * (h[r][p] + u[r][p]);
    // forward substitution with L, then back substitution with L^T (the
    // column orders of dtrsm), all held rows interleaved
    for (int j = 0; j < k; ++j) {
      const double d = rinv[j];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double yj = __shfl_sync(0xffffffffu, slot_get<PER>(y[r], j >> 5), j & 31) * d;
#pragma unroll
        for (int p = 0; p < PER; ++p) {
          const int c = lane + 32 * p;
          if (c == j)
            y[r][p] = yj;
          else if (c > j && c < k)
            y[r][p] -= yj * Ls[c * LD + j];
        }
      }
    }
    for (int j = k - 1; j >= 0; --j) {
      const double d = rinv[j];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double xj = __shfl_sync(0xffffffffu, slot_get<PER>(y[r], j >> 5), j & 31) * d;
#pragma unroll
        for (int p = 0; p < PER; ++p) {
          const int c = lane + 32 * p;
          if (c == j)
            y[r][p] = xj;
          else if (c < j)
            y[r][p] -= xj * Ls[j * LD + c];
        }
      }
    }
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < PER; ++p)
        if (live[r][p]) {
          double hn = y[r][p] - u[r][p];
          hn = hn > 0.0 ? hn : 0.0;
          const double un = (u[r][p] + hn) - y[r][p];
          s4[0] = fma(hn, hn, s4[0]);
          s4[1] = fma(un, un, s4[1]);
          const double dr = hn - y[r][p];
          s4[2] = fma(dr, dr, s4[2]);
          const double ds = hn - h[r][p];
          s4[3] = fma(ds, ds, s4[3]);
          h[r][p] = hn;
          u[r][p] = un;
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int qd = 0; qd < 4; ++qd) s4[qd] += __shfl_xor_sync(0xffffffffu, s4[qd], o);
    if (lane == 0)
#pragma unroll
      for (int qd = 0; qd < 4; ++qd) wred[warp][qd] = s4[qd];
    __syncthreads();
    if (tid < (int)cluster.num_blocks()) {
      double t4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int w = 0; w < NW; ++w)
        for (int qd = 0; qd < 4; ++qd) t4[qd] += wred[w][qd];
      double* dst = cluster.map_shared_rank(&slot[it & 1][cluster.block_rank()][0], tid);
      for (int qd = 0; qd < 4; ++qd) dst[qd] = t4[qd];
    }
    cluster.sync();
    double tot[4] = {0.0, 0.0, 0.0, 0.0};
    for (unsigned b = 0; b < cluster.num_blocks(); ++b)
      for (int qd = 0; qd < 4; ++qd) tot[qd] += slot[it & 1][b][qd];
    const double facnorm = sqrt(tot[0]), dualnorm = sqrt(tot[1]);
    const double rn = sqrt(tot[2]), sn = sqrt(tot[3]);
    if (rn < tol * facnorm && sn < tol * dualnorm) break;  // ntfaoadmm.hpp:63-71
  }
  // dual variable column norms (m_ncp_aux.normalize(mode), ntfaoadmm.hpp:74).
  // Ls is dead in every CTA once all have passed the loop's last cluster
  // barrier, so its space holds the per-warp column sums and the per-CTA
  // partials the other CTAs push.
  double(*colw)[KP] = reinterpret_cast<double(*)[KP]>(Ls);
  double(*colpart)[KP] = reinterpret_cast<double(*)[KP]>(Ls + NW * KP);
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    double cs = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (live[r][p]) cs = fma(u[r][p], u[r][p], cs);
    colw[warp][lane + 32 * p] = cs;
  }
  __syncthreads();
  if (tid < k) {
    double t = 0.0;
    for (int w = 0; w < NW; ++w) t += colw[w][tid];
    for (unsigned b = 0; b < cluster.num_blocks(); ++b)
      *cluster.map_shared_rank(&colpart[cluster.block_rank()][tid], b) = t;
  }
  cluster.sync();
  double nrm[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    double t = 0.0;
    if (c < k)
      for (unsigned b = 0; b < cluster.num_blocks(); ++b) t += colpart[b][c];
    nrm[p] = sqrt(t);
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t row = row0 + r * stride;
#pragma unroll
    for (int p = 0; p < PER; ++p)
      if (live[r][p]) {
        const int c = lane + 32 * p;
        H[row * k + c] = h[r][p];
        U[row * k + c] = nrm[p] > 0 ? u[r][p] / nrm[p] : u[r][p];
      }
  }
}

// Column 2-norms of an I x k row-major matrix in two launches (per-CTA
// partial sums of squares, then every CTA sums the partials in CTA order and
// scales its own rows): NCPFactors::normalize(int) (ncpfactors.hpp:346-351)
// without keeping lambda.
constexpr int CN_ROWS = 64;
__global__ void __launch_bounds__(256) k_colsumsq_partial(const double* __restrict__ U, int64_t I,
                                                          int k, double* __restrict__ part) {
  __shared__ double red[256];
  const int tid = threadIdx.x;
  const int lanes = 256 / k;  // threads per column
  const int c = tid % k, l = tid / k;
  const int64_t row0 = (int64_t)blockIdx.x * CN_ROWS;
  double s = 0.0;
  if (l < lanes)
    for (int64_t i = row0 + l; i < I && i < row0 + CN_ROWS; i += lanes) s = fma(U[i * k + c], U[i * k + c], s);
  red[tid] = s;
  __syncthreads();
  if (tid < k) {
    double t = 0.0;
    for (int q = 0; q < lanes; ++q) t += red[q * k + tid];
    part[(int64_t)blockIdx.x * k + tid] = t;
  }
}

__global__ void __launch_bounds__(256) k_colnorm_apply(double* __restrict__ U, int64_t I, int k,
                                                       const double* __restrict__ part, int nblk) {
  __shared__ double nrm[kMaxRank];
  if (threadIdx.x < k) {
    double t = 0.0;
    for (int b = 0; b < nblk; ++b) t += part[(int64_t)b * k + threadIdx.x];
    nrm[threadIdx.x] = sqrt(t);
  }
  __syncthreads();
  const int64_t row0 = (int64_t)blockIdx.x * CN_ROWS;
  const int64_t rows = (I - row0) < CN_ROWS ? (I - row0) : CN_ROWS;
  for (int64_t e = threadIdx.x; e < rows * k; e += blockDim.x) {
    const double n = nrm[e % k];
    if (n > 0) U[row0 * k + e] = U[row0 * k + e] / n;
  }
}

// ---------------------------------------------------------------------------
// Normalisation + Gram of one factor in one cluster launch
// ---------------------------------------------------------------------------
// The outputs of k_gram_partial + k_gram_finalize + k_scale_cols
// (NCPFactors::normalize(int), ncpfactors.hpp:346-351; the Gram of the
// normalised factor, ncpfactors.hpp:144; the leave-one-out product for mode
// `next`, ncpfactors.hpp:139-148) from one cluster of CTAs that split U's rows
// evenly. Each CTA forms U^T U of its rows (64-row tiles in shared memory,
// rows in increasing order, a thread per 2 x 2 (k <= 32) or 4 x 4 block of
// outputs) in its own shared memory; after a cluster barrier CTA c adds slice
// c of the entries over the cluster's CTAs in rank order and stores the sums
// into every CTA's copy of the Gram (distributed shared memory); after a
// second barrier every CTA holds the same Gram, takes lambda_r =
// sqrt((U^T U)_rr), divides its own rows by lambda and writes its slice of
// G_n = (U^T U)_ab / (lambda_a lambda_b) and of the leave-one-out product;
// CTA 0 writes lambda. Meant for factors of up to NGC_MAX_ROWS rows, where three launches
// cost more than the work.
constexpr int NGC_THREADS = 256;
constexpr int NGC_TILE = 64;          // rows of a shared-memory tile
constexpr int64_t NGC_MAX_ROWS = 4096;
constexpr int NGC_MAX_CL = 16;        // largest cluster

inline size_t ngc_smem_bytes(int k) {
  const int kp = k <= 32 ? 32 : 64;
  return ((size_t)NGC_TILE * kp + (size_t)kp * kp) * sizeof(double);
}

// The rows are split over the first CLm CTAs of the cluster (CLm <= the
// cluster's size; a batch's grouped launch runs every member in a cluster of
// the largest member's size, and the CTAs past a member's own CLm add zeros).
template <int BE>  // edge of a thread's block of outputs: 2 (k <= 32) or 4
__device__ __forceinline__ void normgram_cluster_body(double* __restrict__ F, int64_t I, int k,
                                                      double* __restrict__ lambda,
                                                      double* __restrict__ Gall, int N, int n,
                                                      int next, double* __restrict__ Gloo, int CLm) {
  cg::cluster_group cluster = cg::this_cluster();
  const int CL = (int)cluster.num_blocks(), me = (int)cluster.block_rank();
  extern __shared__ double ngc_sm[];
  const int kp = k <= 32 ? 32 : 64;
  double* tile = ngc_sm;                   // NGC_TILE x k; later this CTA's copy of the Gram
  double* gpart = ngc_sm + NGC_TILE * kp;  // k x k: U^T U of this CTA's rows
  __shared__ double lam[kMaxRank];
  const int tid = threadIdx.x;
  const int kk2 = k * k;
  const int64_t per = (I + CLm - 1) / CLm;
  const int64_t r0 = (int64_t)me * per;
  const int64_t r1 = (r0 + per) < I ? (r0 + per) : I;
  const int kt = (k + BE - 1) / BE;
  const bool owner = tid < kt * kt;
  const int ta = tid / kt, tb = tid % kt;
  double acc[BE][BE];
#pragma unroll
  for (int u = 0; u < BE; ++u)
#pragma unroll
    for (int v = 0; v < BE; ++v) acc[u][v] = 0.0;
  for (int64_t c0 = r0; c0 < r1; c0 += NGC_TILE) {
    const int nrows = (int)((r1 - c0) < NGC_TILE ? (r1 - c0) : NGC_TILE);
    __syncthreads();
    // eight loads in flight per thread before the stores
    for (int e0 = tid; e0 < nrows * k; e0 += 8 * NGC_THREADS) {
      double tv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NGC_THREADS;
        tv[u] = e < nrows * k ? F[c0 * k + e] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * NGC_THREADS;
        if (e < nrows * k) tile[e] = tv[u];
      }
    }
    __syncthreads();
    if (owner)
      for (int i = 0; i < nrows; ++i) {
        const double* r = tile + i * k;
        double av[BE], bv[BE];
#pragma unroll
        for (int u = 0; u < BE; ++u) {
          const int a = ta + kt * u, b = tb + kt * u;
          av[u] = a < k ? r[a] : 0.0;
          bv[u] = b < k ? r[b] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < BE; ++u)
#pragma unroll
          for (int v = 0; v < BE; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
      }
  }
  if (owner)
#pragma unroll
    for (int u = 0; u < BE; ++u)
#pragma unroll
      for (int v = 0; v < BE; ++v) {
        const int a = ta + kt * u, b = tb + kt * v;
        if (a < k && b < k) gpart[a * k + b] = acc[u][v];
      }
  __syncthreads();  // the tile is free for the Gram copy
  cluster.sync();
  {
    const int sl = (kk2 + CL - 1) / CL;
    const int e0 = me * sl, e1 = (e0 + sl) < kk2 ? (e0 + sl) : kk2;
    for (int e = e0 + tid; e < e1; e += NGC_THREADS) {
      // all remote loads in flight before the in-order sum
      double v[NGC_MAX_CL];
#pragma unroll
      for (int b = 0; b < NGC_MAX_CL; ++b) v[b] = b < CL ? *cluster.map_shared_rank(gpart + e, b) : 0.0;
      double t = 0.0;
#pragma unroll
      for (int b = 0; b < NGC_MAX_CL; ++b)
        if (b < CL) t += v[b];
#pragma unroll
      for (int b = 0; b < NGC_MAX_CL; ++b)
        if (b < CL) *cluster.map_shared_rank(tile + e, b) = t;
    }
  }
  cluster.sync();
  const double* gs = tile;
  if (tid < k) lam[tid] = sqrt(gs[tid * k + tid]);
  __syncthreads();
  {
    // a thread keeps one column c of rows r0 + rr, r0 + rr + rstep, ...
    const int rstep = NGC_THREADS / k;
    const int c = tid % k;
    const int64_t rr = tid / k;
    const double nrm = lam[c];
    if (rr < rstep && nrm > 0)
      for (int64_t ra = r0 + rr; ra < r1; ra += 8 * (int64_t)rstep) {
        double fv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int64_t r = ra + (int64_t)u * rstep;
          fv[u] = r < r1 ? F[r * k + c] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int64_t r = ra + (int64_t)u * rstep;
          if (r < r1) F[r * k + c] = fv[u] / nrm;
        }
      }
  }
  if (me == 0 && tid < k && lambda) lambda[tid] = lam[tid];
  // G_n and the leave-one-out product: CTA me writes its slice of the entries
  const int sl = (kk2 + CL - 1) / CL;
  const int e0 = me * sl, e1 = (e0 + sl) < kk2 ? (e0 + sl) : kk2;
  double* Gn = Gall + (int64_t)n * kk2;
  for (int e = e0 + tid; e < e1; e += NGC_THREADS) {
    const int a = e / k, b = e % k;
    const double la = lam[a], lb = lam[b];
    const double gn = (la > 0 && lb > 0) ? gs[e] / (la * lb) : gs[e];
    Gn[e] = gn;
    if (next >= 0) {
      double g = 1.0;
      for (int i = 0; i < N; ++i)
        if (i != next) g = g * (i == n ? gn : Gall[(int64_t)i * kk2 + e]);
      Gloo[e] = g;
    }
  }
}
template <int BE>
__global__ void __launch_bounds__(NGC_THREADS, 1)
    k_normgram_cluster(double* __restrict__ F, int64_t I, int k, double* __restrict__ lambda,
                       double* __restrict__ Gall, int N, int n, int next,
                       double* __restrict__ Gloo) {
  normgram_cluster_body<BE>(F, I, k, lambda, Gall, N, n, next, Gloo,
                            (int)cg::this_cluster().num_blocks());
}

// ---------------------------------------------------------------------------
// Nesterov (NTFNES)
// ---------------------------------------------------------------------------
constexpr int NES_MAX_STEPS = 20000;

// Device state of the Nesterov solver object beyond its factor-sized arrays.
struct NesDev {
  double L, mu, lambda, q, inv;  // of the current mode's update
  double step;                   // acceleration step of this iteration
  double cur_err, acc_err;       // error after the sweep / of the extrapolation
  int acc_exp, acc_fails;        // ntfnes.hpp:186-189 (acc_exp starts at 3)
  int accepted;                  // last acceleration kept
  int err_ctr;                   // index slot for the error kernel
  int steps;                     // inner steps of the last update
};

// ntfnes.hpp:25-37
__device__ __forceinline__ double nes_lambda_of(double L, double mu) {
  const double q = L / mu;
  if (q > 1e6) return 10 * mu;
  if (q > 1e3) return mu;
  return mu / 10;
}

// ntfnes.hpp:39-50: root of x^2 + (alpha^2 - q) x - alpha^2 = 0
__device__ __forceinline__ double nes_alpha_of(double alpha, double q) {
  const double a = 1.0, b = alpha * alpha - q, c = -alpha * alpha;
  const double D = b * b - 4 * a * c;
  return (-b + sqrt(D)) / 2;
}

// Extreme eigenvalues of the symmetric G (arma::eig_sym, ntfnes.hpp:111-113)
// by cyclic Jacobi rotations, k/2 disjoint rotations per round in the
// round-robin order, until a sweep finds every off-diagonal entry below the
// rounding level of its two diagonal entries.
// Then lambda, q and 1/(L + lambda) of the update (ntfnes.hpp:114-117). For
// mode 0 it also copies the proximal lambda to the previous one
// (ntfnes.hpp:102-104). One CTA of 256 threads.
__global__ void __launch_bounds__(256) k_nes_prep(const double* __restrict__ G, int k,
                                                  NesDev* __restrict__ st, int mode,
                                                  const double* __restrict__ prox_lam,
                                                  double* __restrict__ prev_lam) {
  constexpr int LD = kMaxRank + 1;
  __shared__ double A[kMaxRank * LD];
  __shared__ double rc[kMaxRank / 2], rs[kMaxRank / 2];
  __shared__ int rp[kMaxRank / 2], rq[kMaxRank / 2];
  __shared__ int s_rot;
  const int tid = threadIdx.x;
  if (mode == 0 && tid < k) prev_lam[tid] = prox_lam[tid];
  for (int e = tid; e < k * k; e += blockDim.x) A[(e / k) * LD + e % k] = G[e];
  __syncthreads();
  const int n2 = (k + 1) & ~1;  // even player count of the round-robin
  const int np = n2 / 2;
  if (tid == 0) s_rot = 0;
  __syncthreads();
  for (int sweep = 0; sweep < 60; ++sweep) {
    for (int round = 0; round < n2 - 1; ++round) {
      if (tid < np) {
        // circle method: player 0 fixed, x_j = ((j + round) mod m) + 1 rotate;
        // pairs (0, x_0) and (x_j, x_{m-j}) for 0 < j < np
        const int m = n2 - 1;
        const int a = tid == 0 ? 0 : ((tid + round) % m) + 1;
        const int b = tid == 0 ? (round % m) + 1 : ((m - tid + round) % m) + 1;
        const int p = a < b ? a : b, q = a < b ? b : a;
        double c = 1.0, s = 0.0;
        if (q < k) {
          const double apq = A[p * LD + q];
          const double app = A[p * LD + p], aqq = A[q * LD + q];
          // a pair whose coupling is below the rounding level of its diagonal
          // is converged (the classical threshold of cyclic Jacobi)
          if (fabs(apq) > 1e-17 * sqrt(fabs(app * aqq)) && apq != 0.0) {
            const double theta = (aqq - app) / (2.0 * apq);
            double t;
            if (fabs(theta) > 1e150)
              t = 0.5 / theta;
            else
              t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(1.0 + theta * theta));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
            s_rot = 1;
          }
        }
        rp[tid] = p;
        rq[tid] = q;
        rc[tid] = c;
        rs[tid] = s;
      }
      __syncthreads();
      // A <- J^T A J in one pass: the rotations are disjoint, so every 2 x 2
      // block (pair pi's rows, pair pj's columns) changes only through its own
      // four entries; a thread rotates its block's rows, then its columns (the
      // same operations as a row pass followed by a column pass)
      for (int blk = tid; blk < np * np; blk += blockDim.x) {
        const int pi = blk / np, pj = blk % np;
        const int p1 = rp[pi], q1 = rq[pi], p2 = rp[pj], q2 = rq[pj];
        const double s1 = rs[pi], s2 = rs[pj];
        if (s1 == 0.0 && s2 == 0.0) continue;
        const double c1 = rc[pi], c2 = rc[pj];
        const bool q1ok = q1 < k, q2ok = q2 < k;
        const double a11 = A[p1 * LD + p2];
        const double a12 = q2ok ? A[p1 * LD + q2] : 0.0;
        const double a21 = q1ok ? A[q1 * LD + p2] : 0.0;
        const double a22 = (q1ok && q2ok) ? A[q1 * LD + q2] : 0.0;
        double r11 = a11, r12 = a12, r21 = a21, r22 = a22;
        if (s1 != 0.0) {
          r11 = c1 * a11 - s1 * a21;
          r21 = s1 * a11 + c1 * a21;
          r12 = c1 * a12 - s1 * a22;
          r22 = s1 * a12 + c1 * a22;
        }
        double o11 = r11, o12 = r12, o21 = r21, o22 = r22;
        if (s2 != 0.0) {
          o11 = c2 * r11 - s2 * r12;
          o12 = s2 * r11 + c2 * r12;
          o21 = c2 * r21 - s2 * r22;
          o22 = s2 * r21 + c2 * r22;
        }
        A[p1 * LD + p2] = o11;
        if (q2ok) A[p1 * LD + q2] = o12;
        if (q1ok) A[q1 * LD + p2] = o21;
        if (q1ok && q2ok) A[q1 * LD + q2] = o22;
      }
      __syncthreads();
    }
    const int rotated = s_rot;  // read by every thread before it is reset
    __syncthreads();
    if (!rotated) break;  // a sweep without a rotation: converged
    if (tid == 0) s_rot = 0;
    __syncthreads();
  }
  if (tid == 0) {
    double lo = A[0], hi = A[0];
    for (int i = 1; i < k; ++i) {
      const double d = A[i * LD + i];
      lo = d < lo ? d : lo;
      hi = d > hi ? d : hi;
    }
    const double lam = nes_lambda_of(hi, lo);
    st->L = hi;
    st->mu = lo;
    st->lambda = lam;
    st->q = (lo + lam) / (hi + lam);
    st->inv = 1 / (hi + lam);
  }
}

// NTFNES::update inner loop (ntfnes.hpp:100-151) for all rows of one mode,
// in one cluster of NES_CTAS CTAs:
//   prev = H0 = prox;  Ht = acc = H0;  modM = (-lambda) H0 - M
//   loop: grad = modM + (G + lambda I) acc
//         stop if max|grad .* acc| <= 1e-2 and min(grad) >= -1e-2
//         Ht' = max(acc - grad / (L + lambda), 0)
//         alpha, beta (ntfnes.hpp:143-145); acc = Ht' + beta (Ht' - Ht)
// Ht is the mode's factor buffer (the update's output, unnormalised); acc,
// grad and modM are I x k scratch arrays. A step cap (the reference loops
// without one) sets kStMaxIter.
template <int KP>
__global__ void __cluster_dims__(NES_CTAS, 1, 1) __launch_bounds__(NES_THREADS, 1)
    k_nes_inner(double* __restrict__ Ht, const double* __restrict__ prox, double* __restrict__ prev,
                const double* __restrict__ M, const double* __restrict__ G, NesDev* __restrict__ st,
                double* __restrict__ acc, double* __restrict__ grad, double* __restrict__ modM,
                int64_t I, int k, int max_steps, int* __restrict__ status) {
  constexpr int PER = KP / 32;
  constexpr int NW = NES_THREADS / 32;
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ double Gs[KP * KP];
  __shared__ double wmax[NW], wmin[NW];
  __shared__ double slot[2][NES_CTAS_MAX][2];  // pushed by every CTA, read locally
  const double lam = st->lambda, q = st->q, inv = st->inv;
  for (int e = threadIdx.x; e < k * k; e += NES_THREADS)
    Gs[e] = G[e] + ((e / k) == (e % k) ? lam : 0.0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * NW;
  const int64_t row0 = (int64_t)blockIdx.x * NW + warp;
  double vmax = 0.0, vmin = INFINITY;

  // grad = modM + Gs acc for one row (acc in registers), with the row's
  // contribution to the stopping test
  auto row_grad = [&](int64_t row, const double (&a)[PER], const double (&mm)[PER]) {
    double g[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) g[p] = 0.0;
    for (int j = 0; j < k; ++j) {
      const double aj = __shfl_sync(0xffffffffu, slot_get<PER>(a, j >> 5), j & 31);
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c < k) g[p] = fma(aj, Gs[j * k + c], g[p]);
      }
    }
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      if (c < k) {
        const double gr = mm[p] + g[p];
        grad[row * k + c] = gr;
        vmax = fmax(vmax, fabs(gr * a[p]));
        vmin = fmin(vmin, gr);
      }
    }
  };

  for (int64_t row = row0; row < I; row += stride) {
    double a[PER], mm[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      const double h0 = c < k ? prox[row * k + c] : 0.0;
      a[p] = h0;
      mm[p] = c < k ? (-1 * lam) * h0 - M[row * k + c] : 0.0;
      if (c < k) {
        prev[row * k + c] = h0;
        Ht[row * k + c] = h0;
        acc[row * k + c] = h0;
        modM[row * k + c] = mm[p];
      }
    }
    row_grad(row, a, mm);
  }

  double alpha = 1.0, beta = 1.0;
  int t = 0;
  for (;;) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      vmin = fmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
    }
    if (lane == 0) {
      wmax[warp] = vmax;
      wmin[warp] = vmin;
    }
    __syncthreads();
    if (warp == 0) {  // CTA max / min over the warps, pushed to every CTA
      double m = lane < NW ? wmax[lane] : 0.0, n = lane < NW ? wmin[lane] : INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        n = fmin(n, __shfl_xor_sync(0xffffffffu, n, o));
      }
      if (lane < (int)cluster.num_blocks()) {
        double* dst = cluster.map_shared_rank(&slot[t & 1][cluster.block_rank()][0], lane);
        dst[0] = m;
        dst[1] = n;
      }
    }
    cluster.sync();
    double gmax = 0.0, gmin = INFINITY;
    for (unsigned r = 0; r < cluster.num_blocks(); ++r) {
      gmax = fmax(gmax, slot[t & 1][r][0]);
      gmin = fmin(gmin, slot[t & 1][r][1]);
    }
    if (gmax <= 1e-2 && gmin >= -1e-2) break;  // stop_iter, ntfnes.hpp:52-62
    if (t >= max_steps) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(status, 0, kStMaxIter);
      break;
    }
    ++t;
    const double alpha_prev = alpha;
    alpha = nes_alpha_of(alpha_prev, q);
    beta = (alpha_prev * (1 - alpha_prev)) / (alpha + alpha_prev * alpha_prev);
    vmax = 0.0;
    vmin = INFINITY;
    for (int64_t row = row0; row < I; row += stride) {
      double a[PER], mm[PER];
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        a[p] = 0.0;
        mm[p] = 0.0;
        if (c < k) {
          const double hprev = Ht[row * k + c];
          const double v = acc[row * k + c] - (inv * grad[row * k + c]);
          const double hn = v > 0.0 ? v : 0.0;
          a[p] = hn + beta * (hn - hprev);
          mm[p] = modM[row * k + c];
          Ht[row * k + c] = hn;
          acc[row * k + c] = a[p];
        }
      }
      row_grad(row, a, mm);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->steps = t;
}

// The same loop with every row's state in registers: each warp holds up to
// R rows (row0 + r * 128); no global traffic inside the loop, and the R
// matrix-vector products of a step are interleaved. Used when the mode has at
// most R * 128 rows.
template <int KP, int R>
__global__ void __launch_bounds__(NES_THREADS, 1)
    k_nes_inner_reg(double* __restrict__ Ht_out, const double* __restrict__ prox,
                    double* __restrict__ prev, const double* __restrict__ M,
                    const double* __restrict__ G, NesDev* __restrict__ st, int64_t I, int k,
                    int max_steps, int* __restrict__ status) {
  constexpr int PER = KP / 32;
  constexpr int NW = NES_THREADS / 32;
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ double Gs[KP * KP];
  __shared__ double wmax[NW], wmin[NW];
  __shared__ double slot[2][NES_CTAS_MAX][2];  // pushed by every CTA, read locally
  const double lam = st->lambda, q = st->q, inv = st->inv;
  for (int e = threadIdx.x; e < k * k; e += NES_THREADS)
    Gs[e] = G[e] + ((e / k) == (e % k) ? lam : 0.0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t stride = (int64_t)gridDim.x * NW;
  const int64_t row0 = (int64_t)blockIdx.x * NW + warp;
  double ht[R][PER], acc[R][PER], gr[R][PER], mm[R][PER];
  bool live[R][PER];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t row = row0 + r * stride;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      live[r][p] = row < I && c < k;
      const double h0 = live[r][p] ? prox[row * k + c] : 0.0;
      ht[r][p] = h0;
      acc[r][p] = h0;
      mm[r][p] = live[r][p] ? (-1 * lam) * h0 - M[row * k + c] : 0.0;
      if (live[r][p]) prev[row * k + c] = h0;
    }
  }
  double vmax, vmin;
  // grad = modM + (G + lambda I) acc for every held row, and the stopping
  // test's max |grad .* acc| and min grad over them
  auto all_grads = [&]() {
    double g[R][PER];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < PER; ++p) g[r][p] = 0.0;
    for (int j = 0; j < k; ++j) {
      double gv[PER];
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        gv[p] = c < k ? Gs[j * k + c] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const double aj = __shfl_sync(0xffffffffu, slot_get<PER>(acc[r], j >> 5), j & 31);
#pragma unroll
        for (int p = 0; p < PER; ++p) g[r][p] = fma(aj, gv[p], g[r][p]);
      }
    }
    vmax = 0.0;
    vmin = INFINITY;
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        gr[r][p] = mm[r][p] + g[r][p];
        if (live[r][p]) {
          vmax = fmax(vmax, fabs(gr[r][p] * acc[r][p]));
          vmin = fmin(vmin, gr[r][p]);
        }
      }
  };
  all_grads();

  // Each step's cluster barrier is split: after a CTA has pushed its max /
  // min it arrives, forms the next step speculatively (the same arithmetic
  // the loop would do next), and only then waits; when the test says stop,
  // the step's iterate saved before the speculation is the result. The
  // barrier's latency overlaps a step's math; the values are unchanged.
  double alpha = 1.0, beta = 1.0;
  int t = 0;
  double hsave[R][PER];
  cluster.sync();  // every CTA of the cluster running before remote stores
  for (;;) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
      vmin = fmin(vmin, __shfl_xor_sync(0xffffffffu, vmin, o));
    }
    if (lane == 0) {
      wmax[warp] = vmax;
      wmin[warp] = vmin;
    }
    __syncthreads();
    if (warp == 0) {  // CTA max / min over the warps, pushed to every CTA
      double m = lane < NW ? wmax[lane] : 0.0, n = lane < NW ? wmin[lane] : INFINITY;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        n = fmin(n, __shfl_xor_sync(0xffffffffu, n, o));
      }
      if (lane < (int)cluster.num_blocks()) {
        double* dst = cluster.map_shared_rank(&slot[t & 1][cluster.block_rank()][0], lane);
        dst[0] = m;
        dst[1] = n;
      }
    }
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    // speculative step t + 1
    const double alpha_n = nes_alpha_of(alpha, q);
    const double beta_n = (alpha * (1 - alpha)) / (alpha_n + alpha * alpha);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        hsave[r][p] = ht[r][p];
        if (live[r][p]) {
          const double hprev = ht[r][p];
          const double v = acc[r][p] - (inv * gr[r][p]);
          const double hn = v > 0.0 ? v : 0.0;
          acc[r][p] = hn + beta_n * (hn - hprev);
          ht[r][p] = hn;
        }
      }
    all_grads();
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    double gmax = 0.0, gmin = INFINITY;
    for (unsigned r = 0; r < cluster.num_blocks(); ++r) {
      gmax = fmax(gmax, slot[t & 1][r][0]);
      gmin = fmin(gmin, slot[t & 1][r][1]);
    }
    const bool stop = gmax <= 1e-2 && gmin >= -1e-2;  // stop_iter, ntfnes.hpp:52-62
    if (stop || t >= max_steps) {
      if (!stop && blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(status, 0, kStMaxIter);
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int p = 0; p < PER; ++p) ht[r][p] = hsave[r][p];
      break;
    }
    ++t;
    alpha = alpha_n;
    beta = beta_n;
  }
  (void)beta;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int64_t row = row0 + r * stride;
#pragma unroll
    for (int p = 0; p < PER; ++p)
      if (live[r][p]) Ht_out[row * k + lane + 32 * p] = ht[r][p];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) st->steps = t;
}

// After the mode's normalisation: prox = the normalised factor, and for the
// last mode the proximal lambda = the factor's lambda (normalize_rows of
// m_prox_t, ntfnes.hpp:148-149).
__global__ void __launch_bounds__(256) k_nes_post(const double* __restrict__ F,
                                                  double* __restrict__ prox, int64_t n,
                                                  const double* __restrict__ lambda,
                                                  double* __restrict__ prox_lam, int k) {
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < n; e += (int64_t)gridDim.x * 256)
    prox[e] = F[e];
  if (prox_lam && blockIdx.x == 0 && threadIdx.x < k) prox_lam[threadIdx.x] = lambda[threadIdx.x];
}

// Start of NTFNES::accelerate (ntfnes.hpp:64-75) for the iteration whose
// error was just written: acc_step = (iter + 1)^(1 / acc_exp); keeps the
// current error, lambda and Grams (the state a failed extrapolation returns
// to) and resets the error slot index of the extrapolation's error.
__global__ void __launch_bounds__(256) k_nes_acc_begin(const int* __restrict__ counter,
                                                       const double* __restrict__ errs,
                                                       NesDev* __restrict__ st,
                                                       const double* __restrict__ lambda,
                                                       double* __restrict__ lam_bak,
                                                       const double* __restrict__ Gall,
                                                       double* __restrict__ gall_bak, int nG, int k) {
  if (threadIdx.x == 0) {
    const int iter = *counter - 1;
    st->cur_err = errs[iter];
    st->step = pow((double)(iter + 1), 1.0 / st->acc_exp);
    st->err_ctr = 0;
  }
  if (threadIdx.x < k) lam_bak[threadIdx.x] = lambda[threadIdx.x];
  for (int e = threadIdx.x; e < nG; e += 256) gall_bak[e] = Gall[e];
}

// Extrapolated factor of one mode (ntfnes.hpp:76-88), written over the
// factor: a = cur + step (cur - prv), cur = diag(sc) F, prv = diag(sp) prev,
// with sc / sp the current / previous lambda for the last mode (the only
// unnormalised one) and the identity otherwise.
__global__ void __launch_bounds__(256) k_nes_extrap(double* __restrict__ F,
                                                    const double* __restrict__ prev, int64_t n, int k,
                                                    const double* __restrict__ sc,
                                                    const double* __restrict__ sp,
                                                    const NesDev* __restrict__ st) {
  const double step = st->step;
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < n; e += (int64_t)gridDim.x * 256) {
    const int r = (int)(e % k);
    const double cur = sc ? sc[r] * F[e] : F[e];
    const double prv = sp ? sp[r] * prev[e] : prev[e];
    double a = cur - prv;
    a *= step;
    a += cur;
    F[e] = a;
  }
}

// Acceptance test of the extrapolation (ntfnes.hpp:89-98). Rejected: the
// Grams and lambda of the proximal iterate come back (its factors by
// k_nes_commit), the failure count rises and every fail_limit + 1 failures
// the step exponent grows. Accepted: the proximal lambda becomes the norms
// of the (normalised) extrapolated last factor, sqrt(diag G_{N-1}).
__global__ void __launch_bounds__(256) k_nes_decide(NesDev* __restrict__ st,
                                                    double* __restrict__ lambda,
                                                    double* __restrict__ prox_lam,
                                                    double* __restrict__ Gall,
                                                    const double* __restrict__ gall_bak, int nG,
                                                    const double* __restrict__ Glast, int k) {
  __shared__ int s_acc;
  if (threadIdx.x == 0) s_acc = st->acc_err < st->cur_err;
  __syncthreads();
  const int accepted = s_acc;
  if (accepted) {
    if (threadIdx.x < k) prox_lam[threadIdx.x] = sqrt(Glast[threadIdx.x * k + threadIdx.x]);
  } else {
    if (threadIdx.x < k) lambda[threadIdx.x] = prox_lam[threadIdx.x];
    for (int e = threadIdx.x; e < nG; e += 256) Gall[e] = gall_bak[e];
  }
  if (threadIdx.x == 0) {
    st->accepted = accepted;
    if (!accepted) {
      st->acc_fails++;
      if (st->acc_fails > 5) {  // fail_limit, ntfnes.hpp:190
        st->acc_fails = 0;
        st->acc_exp++;
      }
    }
  }
}

// Factor side of the decision for one mode: accepted -> prox = F (the
// extrapolated, normalised factor); rejected -> F = prox.
__global__ void __launch_bounds__(256) k_nes_commit(double* __restrict__ F, double* __restrict__ prox,
                                                    int64_t n, const NesDev* __restrict__ st) {
  const int accepted = st->accepted;
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < n; e += (int64_t)gridDim.x * 256) {
    if (accepted)
      prox[e] = F[e];
    else
      F[e] = prox[e];
  }
}

}  // namespace pg
