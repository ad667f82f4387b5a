// nmf.cuh -- the small kernels of the shared-memory NMF A ~ W H^T (reference
// common/nmf.hpp, nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp). The products
// A H and A^T W are the two MTTKRPs of the 2-way tensor A (the contraction
// kernels of the NTF path); H's HALS sweep is the NTF HALS kernel, MU and BPP
// are the NTF kernels with NMF's constants. What is NMF's own is here:
// regularised Grams, HALS's column-normalised W sweep, normalize_by_W and the
// objective with its regularisation terms.
//
// W (m x k) and H (n x k) are row-major, rank fastest.
#pragma once
#include "common.cuh"

namespace pg {

// Sum of v[i * stride] for i < n by a whole CTA in a fixed order: thread t
// adds entries t, t + blockDim.x, ... and a fixed tree over the threads adds
// the rest (sh: blockDim.x doubles, blockDim.x a power of two). Every thread
// returns the total.
// Sum of one value per thread over the CTA by a fixed tree (sh: blockDim.x
// doubles, blockDim.x a power of two). Every thread returns the total.
__device__ __forceinline__ double cta_tree_fixed(double s, double* sh) {
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double t = sh[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ double cta_sum_fixed(const double* __restrict__ v, int n, int stride,
                                                double* sh) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[(int64_t)i * stride];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x >> 1; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  const double t = sh[0];
  __syncthreads();
  return t;
}

// Gram U^T U from k_gram_partial's row-block partials plus NMF::applyReg
// (common/nmf.hpp:76-92: l2 I, then l1 ones) and an extra diagonal shift (the
// symmetric regularisation of BPPNMF, common/nmf.hpp:118-124). A warp per
// entry: lane l adds partials l, l + 32, ... in order, then a fixed shuffle
// tree adds the lanes. 8 entries per CTA.
__global__ void __launch_bounds__(256) k_nmf_gram(const double* __restrict__ part, int nblk, int k,
                                                  double l2, double l1, double diag,
                                                  double* __restrict__ out) {
  const int kk2 = k * k;
  const int lane = threadIdx.x & 31;
  const int e = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (e >= kk2) return;
  double s = 0.0;
  for (int b = lane; b < nblk; b += 32) s += part[(int64_t)b * kk2 + e];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) {
    const bool d = (e / k) == (e % k);
    if (l2 > 0 && d) s = s + l2;
    if (l1 > 0) s = s + l1;
    if (diag > 0 && d) s = s + diag;
    out[e] = s;
  }
}

// out += a * U, elementwise (the symmetric regularisation's right-hand side
// given^T input + symm_reg given^T, nmf/bppnmf.hpp:36-40).
__global__ void __launch_bounds__(256) k_nmf_axpy(double* __restrict__ out, const double* __restrict__ U,
                                                  int64_t n, double a) {
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < n; e += (int64_t)gridDim.x * 256)
    out[e] = out[e] + a * U[e];
}

constexpr int NMFW_WARPS = 8;
constexpr int NMFW_MAX_BLOCKS = 296;

// Column x of HALSNMF's W sweep (nmf/hals.hpp:92-105), all rows (a warp per
// row): first the previous column is finished, W(:, x-1) /= ||Wx-1|| (the
// norm the last launch left in norms[x-1]); then
//   Wx = W(:,x) HtH(x,x) + (AH(:,x) - W HtH(:,x)),  entries < 1e-17 -> 1e-17
// is stored unnormalised and its squared norm summed (per CTA in warp order,
// over CTAs in CTA order by the last CTA to finish, which writes norms[x]).
// The sweep is launches x = 0 .. k; the last only finishes column k-1.
constexpr int NMFW_ROWS = 4;  // rows of a warp whose loads are in flight together

template <int KP>
__global__ void __launch_bounds__(32 * NMFW_WARPS) k_nmf_hals_w(
    double* __restrict__ W, const double* __restrict__ AH, const double* __restrict__ G, int64_t m,
    int k, int x, double* __restrict__ norms, double* __restrict__ part, int* __restrict__ counter) {
  constexpr int PER = KP / 32;
  __shared__ double wred[NMFW_WARPS];
  __shared__ double sh[32 * NMFW_WARPS];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double nprev = x > 0 ? norms[x - 1] : 0.0;
  double gx[PER];  // G(:, x) for this lane's columns
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    gx[p] = (x < k && c < k) ? G[c * k + x] : 0.0;
  }
  const double gxx = x < k ? G[x * k + x] : 0.0;
  double ss = 0.0;
  const int64_t wstride = (int64_t)gridDim.x * NMFW_WARPS;
  for (int64_t row0 = (int64_t)blockIdx.x * NMFW_WARPS + warp; row0 < m;
       row0 += wstride * NMFW_ROWS) {
    double w[NMFW_ROWS][PER], ah[NMFW_ROWS];
#pragma unroll
    for (int u = 0; u < NMFW_ROWS; ++u) {
      const int64_t row = row0 + wstride * u;
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        w[u][p] = (row < m && c < k) ? W[row * k + c] : 0.0;
      }
      ah[u] = (row < m && x < k) ? AH[row * k + x] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < NMFW_ROWS; ++u) {
      const int64_t row = row0 + wstride * u;
      if (row >= m) continue;  // warp-uniform
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c == x - 1 && nprev != 0) {
          w[u][p] = w[u][p] / nprev;
          W[row * k + c] = w[u][p];
        }
      }
      if (x < k) {
        // s = sum_j W(row, j) G(j, x), reduced across the warp in a fixed order
        double s = 0.0;
#pragma unroll
        for (int p = 0; p < PER; ++p) s = fma(w[u][p], gx[p], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
#pragma unroll
        for (int p = 0; p < PER; ++p) {
          const int c = lane + 32 * p;
          if (c == x) {
            double v = (w[u][p] * gxx) + (ah[u] - s);
            v = (v < kEps17) ? kEps17 : v;
            W[row * k + x] = v;
            ss = fma(v, v, ss);
          }
        }
      }
    }
  }
  if (x >= k) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
  if (lane == 0) wred[warp] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w2 = 0; w2 < NMFW_WARPS; ++w2) t += wred[w2];
    part[blockIdx.x] = t;
    __threadfence();
    s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const double t = cta_sum_fixed(part, gridDim.x, 1, sh);
  if (threadIdx.x == 0) {
    norms[x] = sqrt(t);
    *counter = 0;
  }
}

// NMF::normalize_by_W (common/nmf.hpp:150-160), first launch: per-CTA column
// sums of W^2 over NRM_ROWS rows; the last CTA to finish adds the CTAs'
// partials in CTA order (a warp per column: lane l adds partials l, l + 32,
// ..., then a fixed shuffle tree) and writes norms[c] = ||W(:, c)||.
constexpr int NRM_ROWS = 64;
__global__ void __launch_bounds__(256) k_nmf_colnorms(const double* __restrict__ W, int64_t m,
                                                      int k, double* __restrict__ part,
                                                      int* __restrict__ ticket,
                                                      double* __restrict__ norms) {
  __shared__ double red[256];
  __shared__ int s_last;
  const int tid = threadIdx.x;
  const int lanes = 256 / k;  // threads per column
  const int c = tid % k, l = tid / k;
  const int64_t row0 = (int64_t)blockIdx.x * NRM_ROWS;
  double s = 0.0;
  if (l < lanes)
    for (int64_t i = row0 + l; i < m && i < row0 + NRM_ROWS; i += lanes)
      s = fma(W[i * k + c], W[i * k + c], s);
  red[tid] = s;
  __syncthreads();
  if (tid < k) {
    double t = 0.0;
    for (int q = 0; q < lanes; ++q) t += red[q * k + tid];
    part[(int64_t)blockIdx.x * k + tid] = t;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  const int lane = tid & 31;
  for (int cc = tid >> 5; cc < k; cc += 8) {
    double t = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) t += __ldcg(part + (int64_t)b * k + cc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) norms[cc] = sqrt(t);
  }
  if (tid == 0) *ticket = 0;
}

// Second launch: W(:, c) /= norm_c and H(:, c) *= norm_c (norm_c > 0) over
// NRM_ROWS rows of each.
__global__ void __launch_bounds__(256) k_nmf_rescale(double* __restrict__ W, int64_t m,
                                                     double* __restrict__ H, int64_t n, int k,
                                                     const double* __restrict__ norms) {
  __shared__ double nrm[kMaxRank];
  if (threadIdx.x < k) nrm[threadIdx.x] = norms[threadIdx.x];
  __syncthreads();
  const int64_t row0 = (int64_t)blockIdx.x * NRM_ROWS;
  for (int64_t e = threadIdx.x; e < (int64_t)NRM_ROWS * k; e += 256) {
    const int64_t row = row0 + e / k;
    const int c = (int)(e % k);
    const double v = nrm[c];
    if (v > 0) {
      if (row < m) W[row * k + c] = W[row * k + c] / v;
      if (row < n) H[row * k + c] = H[row * k + c] * v;
    }
  }
}

// ---------------------------------------------------------------------------
// HALSNMF's W sweep in one cooperative launch (nmf/hals.hpp:92-105)
// ---------------------------------------------------------------------------
// Each CTA keeps its block of W's rows in shared memory for the whole sweep
// (a thread per row, up to NMFC_RPT rows a thread). For column x every thread
// forms, for its rows,
//   Wx = W(:,x) HtH(x,x) + (AH(:,x) - W HtH(:,x)),  entries < 1e-17 -> 1e-17
// the CTA adds its squares in a fixed order and stores the sum in
// part[x][cta]; every CTA then waits until all CTAs' sums of column x are
// there, adds them in the same fixed order and divides column x by ||Wx||, so
// all CTAs see the same normalised column before column x + 1 reads it.
//
// part[x][*] is filled with the bit pattern NMFC_EMPTY (all ones, a NaN no
// arithmetic here produces; a sum with those bits is stored as another NaN)
// before the launch; a slot holds a CTA's sum once it reads otherwise. While
// warp 0 waits, every thread forms W HtH(:, x+1) of its rows without the
// term of column x, which it adds once ||Wx|| is known. The waits are
// bounded: after NMFC_SPINS polls a CTA sets an error flag (flag[0]) and
// kStTimeout and returns, and waiting CTAs leave when they see the flag, so
// the launch always ends. The launch is cooperative (all CTAs resident).
constexpr int NMFC_THREADS = 256;
constexpr int NMFC_RPT = 4;
constexpr unsigned NMFC_SPINS = 1u << 21;
constexpr long long NMFC_EMPTY = -1LL;

// Dynamic shared memory k_nmf_hals_w_coop may take on a device whose opt-in
// limit per CTA is `optin` (1 KB stays for its static variables).
inline size_t nmfc_smem_limit(size_t optin) { return optin > 1024 ? optin - 1024 : 0; }

// Shared memory of k_nmf_hals_w_coop for `rows` rows a CTA.
inline size_t nmfc_smem_bytes(int KP, int rows) {
  return ((size_t)rows * (KP + 1) + (size_t)KP * KP + NMFC_THREADS) * sizeof(double);
}

// Warp 0's bounded wait for the nslots per-CTA sums of one column: polls the
// slots until none holds NMFC_EMPTY, or another CTA raised the error flag, or
// `limit` polls went by (then it raises the flag and kStTimeout itself).
// Returns 1 with q = the fixed-order sum (lane l: slots l, l + 32, ...; then a
// fixed shuffle tree), or 0 when the sweep must stop.
__device__ __forceinline__ int nmfc_wait_slots(const double* slot, int nslots, unsigned* flag,
                                               int* status, unsigned limit, double& q) {
  const int lane = threadIdx.x & 31;
  int ok = 1;
  for (unsigned spins = 0;; ++spins) {
    bool have = true;
    q = 0.0;
    for (int b = lane; b < nslots; b += 32) {
      const double v = __ldcv(slot + b);
      have = have && (__double_as_longlong(v) != NMFC_EMPTY);
      q += v;
    }
    if (__all_sync(0xffffffffu, have)) break;
    if (*(volatile unsigned*)flag) {
      ok = 0;
      break;
    }
    if (spins > limit) {
      if (lane == 0) {
        atomicExch(flag, 1u);
        atomicCAS(status, 0, kStTimeout);
      }
      ok = 0;
      break;
    }
    __nanosleep(20);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  return ok;
}

// Self-test of that wait: every CTA but `skip` stores its slot, then warp 0
// of every CTA waits with a limit of `limit` polls. The skipped slot never
// fills, so the waits run out, the flag and kStTimeout are raised and every
// CTA returns (no fault, no hang). Launched cooperatively, as the sweep is.
__global__ void k_nmfc_wait_selftest(double* part, unsigned* flag, int* status, unsigned limit,
                                     int skip) {
  if (threadIdx.x == 0 && (int)blockIdx.x != skip) __stcg(part + blockIdx.x, 1.0);
  if (threadIdx.x < 32) {
    double q = 0.0;
    nmfc_wait_slots(part, (int)gridDim.x, flag, status, limit, q);
  }
}

template <int KP>
__global__ void __launch_bounds__(NMFC_THREADS) k_nmf_hals_w_coop(
    double* __restrict__ W, const double* __restrict__ AH, const double* __restrict__ G, int64_t m,
    int k, int rows_per_cta, double* __restrict__ norms, double* __restrict__ part,
    unsigned* __restrict__ flag, int* __restrict__ status) {
  constexpr int LD = KP + 1;  // odd row stride: a warp's rows fall in distinct banks
  extern __shared__ double nmfc_sm[];
  double* Ws = nmfc_sm;                          // rows_per_cta x LD
  double* Gs = Ws + (size_t)rows_per_cta * LD;   // Gs[x * KP + j] = G(j, x)
  double* red = Gs + KP * KP;                    // NMFC_THREADS
  __shared__ double s_norm;
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * rows_per_cta;
  const int nrows = (int)((m - row0) < rows_per_cta ? (m - row0) : rows_per_cta);
  for (int e = tid; e < nrows * k; e += NMFC_THREADS)
    Ws[(e / k) * LD + (e % k)] = W[row0 * k + e];
  for (int e = tid; e < k * k; e += NMFC_THREADS) Gs[(e % k) * KP + (e / k)] = G[e];
  double ah[NMFC_RPT], s[NMFC_RPT];
#pragma unroll
  for (int u = 0; u < NMFC_RPT; ++u) {
    const int r = tid + u * NMFC_THREADS;
    ah[u] = r < nrows ? AH[(row0 + r) * k] : 0.0;
    s[u] = 0.0;
  }
  __syncthreads();
  // W HtH(:, 0)
  for (int j = 0; j < k; ++j) {
    const double g = Gs[j];
#pragma unroll
    for (int u = 0; u < NMFC_RPT; ++u) {
      const int r = tid + u * NMFC_THREADS;
      if (r < nrows) s[u] = fma(Ws[r * LD + j], g, s[u]);
    }
  }
  for (int x = 0; x < k; ++x) {
    const double gxx = Gs[x * KP + x];
    double ss = 0.0;
#pragma unroll
    for (int u = 0; u < NMFC_RPT; ++u) {
      const int r = tid + u * NMFC_THREADS;
      if (r < nrows) {
        double v = (Ws[r * LD + x] * gxx) + (ah[u] - s[u]);
        v = (v < kEps17) ? kEps17 : v;
        Ws[r * LD + x] = v;
        ss = fma(v, v, ss);
        // next column's right-hand side, in flight across the wait
        if (x + 1 < k) ah[u] = AH[(row0 + r) * k + x + 1];
      }
    }
    // the CTA's sum: a fixed shuffle tree per warp, then thread 0 adds the
    // warps in order (one barrier)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((tid & 31) == 0) red[tid >> 5] = ss;
    __syncthreads();
    double* slot = part + (int64_t)x * gridDim.x;
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < NMFC_THREADS / 32; ++w) t += red[w];
      if (__double_as_longlong(t) == NMFC_EMPTY) t = __longlong_as_double(0x7ff8000000000000LL);
      __stcg(slot + blockIdx.x, t);
    }
    // W HtH(:, x+1) without column x's term
    const double* gn = Gs + (x + 1 < k ? x + 1 : 0) * KP;
#pragma unroll
    for (int u = 0; u < NMFC_RPT; ++u) s[u] = 0.0;
    if (x + 1 < k)
      for (int j = 0; j < k; ++j) {
        if (j == x) continue;
        const double g = gn[j];
#pragma unroll
        for (int u = 0; u < NMFC_RPT; ++u) {
          const int r = tid + u * NMFC_THREADS;
          if (r < nrows) s[u] = fma(Ws[r * LD + j], g, s[u]);
        }
      }
    // ||Wx||: warp 0 waits for every CTA's slot, adds them (lane l: CTAs l,
    // l + 32, ...; then a fixed shuffle tree), the same sum in every CTA
    if (tid < 32) {
      double q = 0.0;
      const int ok = nmfc_wait_slots(slot, (int)gridDim.x, flag, status, NMFC_SPINS, q);
      if (tid == 0) {
        s_ok = ok;
        s_norm = sqrt(q);
        if (blockIdx.x == 0 && ok) norms[x] = s_norm;
      }
    }
    __syncthreads();
    if (!s_ok) return;
    const double nrm = s_norm;
    const double gx1 = x + 1 < k ? gn[x] : 0.0;
#pragma unroll
    for (int u = 0; u < NMFC_RPT; ++u) {
      const int r = tid + u * NMFC_THREADS;
      if (r < nrows) {
        double w = Ws[r * LD + x];
        if (nrm != 0) {
          w = w / nrm;
          Ws[r * LD + x] = w;
        }
        s[u] = fma(w, gx1, s[u]);
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < nrows * k; e += NMFC_THREADS) W[row0 * k + e] = Ws[(e / k) * LD + (e % k)];
}

// Regularisation weights of the objective.
struct NmfReg {
  double w2, w1, h2, h1, sym;  // regW L2, L1; regH L2, L1; symm_reg
};

// NMF::computeObjectiveError (common/nmf.hpp:386-425) from AtW = A^T W of the
// current W and the (unregularised) Grams of W and H:
//   fit = ||A||^2 - 2 tr(H^T AtW) + tr(WtW HtH)
//   objective = fit + regW(0) ||W||^2 + regH(0) ||H||^2
//             + regW(1) ||W 1||^2 + regH(1) ||H 1||^2 + symm_reg ||W - H||^2
// and the relative error sqrt(fit) / ||A|| (||A|| when fit <= 0,
// common/nmf.hpp:428-431). Each CTA sums its share of the row terms (a warp
// per row, fixed order) into part[cta][4]; the last CTA to finish adds the
// CTAs in order, writes obj[*ctr], rel[*ctr] and increments *ctr.
constexpr int NMFE_WARPS = 8;
__global__ void __launch_bounds__(32 * NMFE_WARPS) k_nmf_error(
    const double* __restrict__ W, int64_t m, const double* __restrict__ H, int64_t n, int k,
    const double* __restrict__ AtW, const double* __restrict__ GW, const double* __restrict__ GH,
    const double* __restrict__ normA2, NmfReg reg, double* __restrict__ part,
    int* __restrict__ ticket, double* __restrict__ obj, double* __restrict__ rel,
    int* __restrict__ ctr) {
  __shared__ double wred[NMFE_WARPS][4];
  __shared__ double sh[32 * NMFE_WARPS];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // q0: tr(H^T AtW), q1: ||W 1||^2, q2: ||H 1||^2, q3: ||W - H||^2
  double q[4] = {0.0, 0.0, 0.0, 0.0};
  const int64_t rows = m > n ? m : n;
  for (int64_t r = (int64_t)blockIdx.x * NMFE_WARPS + warp; r < rows;
       r += (int64_t)gridDim.x * NMFE_WARPS) {
    double hw = 0.0, ws = 0.0, hs = 0.0, dd = 0.0;
    for (int c = lane; c < k; c += 32) {
      const double w = r < m ? W[r * k + c] : 0.0;
      const double h = r < n ? H[r * k + c] : 0.0;
      if (r < n) hw = fma(h, AtW[r * k + c], hw);
      ws += w;
      hs += h;
      if (reg.sym > 0 && r < m && r < n) dd = fma(w - h, w - h, dd);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      hw += __shfl_xor_sync(0xffffffffu, hw, o);
      ws += __shfl_xor_sync(0xffffffffu, ws, o);
      hs += __shfl_xor_sync(0xffffffffu, hs, o);
      dd += __shfl_xor_sync(0xffffffffu, dd, o);
    }
    q[0] += hw;
    q[1] = fma(ws, ws, q[1]);
    q[2] = fma(hs, hs, q[2]);
    q[3] += dd;
  }
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < 4; ++i) wred[warp][i] = q[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int w = 0; w < NMFE_WARPS; ++w)
      for (int i = 0; i < 4; ++i) t[i] += wred[w][i];
    for (int i = 0; i < 4; ++i) part[blockIdx.x * 4 + i] = t[i];
    __threadfence();
    s_last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  double t[4];
  for (int i = 0; i < 4; ++i) t[i] = cta_sum_fixed(part + i, gridDim.x, 4, sh);
  // tr(WtW HtH) and the Gram traces: thread j takes entries j, j + blockDim.x,
  // ... of the k x k products, a fixed tree adds the threads
  double pw = 0.0, pfw = 0.0, pfh = 0.0;
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    const int a = e / k, b = e % k;
    pw = fma(GW[e], GH[b * k + a], pw);
    if (a == b) {
      pfw += GW[e];
      pfh += GH[e];
    }
  }
  const double ww = cta_tree_fixed(pw, sh);
  const double fro_w = cta_tree_fixed(pfw, sh);
  const double fro_h = cta_tree_fixed(pfh, sh);
  if (threadIdx.x != 0) return;
  const double a2 = *normA2;
  const double fit = a2 - (2 * t[0]) + ww;
  const double o = fit + reg.w2 * fro_w + reg.h2 * fro_h + reg.w1 * t[1] + reg.h1 * t[2] +
                   (reg.sym > 0 ? reg.sym * t[3] : 0.0);
  const double na = sqrt(a2);
  const int c = *ctr;
  obj[c] = o;
  rel[c] = (fit > 0 ? sqrt(fit) : na) / na;
  *ctr = c + 1;
  *ticket = 0;
}

}  // namespace pg
