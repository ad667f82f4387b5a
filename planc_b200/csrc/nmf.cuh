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

// Gram U^T U from k_gram_partial's row-block partials, summed in block order,
// plus NMF::applyReg (common/nmf.hpp:76-92: l2 I, then l1 ones) and an extra
// diagonal shift (the symmetric regularisation of BPPNMF, common/nmf.hpp:
// 118-124). One CTA.
__global__ void __launch_bounds__(1024) k_nmf_gram(const double* __restrict__ part, int nblk, int k,
                                                   double l2, double l1, double diag,
                                                   double* __restrict__ out) {
  const int kk2 = k * k;
  for (int e = threadIdx.x; e < kk2; e += 1024) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * kk2 + e];
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
template <int KP>
__global__ void __launch_bounds__(32 * NMFW_WARPS) k_nmf_hals_w(
    double* __restrict__ W, const double* __restrict__ AH, const double* __restrict__ G, int64_t m,
    int k, int x, double* __restrict__ norms, double* __restrict__ part, int* __restrict__ counter) {
  constexpr int PER = KP / 32;
  __shared__ double wred[NMFW_WARPS];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double nprev = x > 0 ? norms[x - 1] : 0.0;
  double ss = 0.0;
  for (int64_t row = (int64_t)blockIdx.x * NMFW_WARPS + warp; row < m;
       row += (int64_t)gridDim.x * NMFW_WARPS) {
    double w[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      w[p] = c < k ? W[row * k + c] : 0.0;
      if (c == x - 1 && nprev != 0) {
        w[p] = w[p] / nprev;
        W[row * k + c] = w[p];
      }
    }
    if (x < k) {
      // s = sum_j W(row, j) G(j, x), reduced across the warp in a fixed order
      double s = 0.0;
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c < k) s = fma(w[p], G[c * k + x], s);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
#pragma unroll
      for (int p = 0; p < PER; ++p) {
        const int c = lane + 32 * p;
        if (c == x) {
          double v = (w[p] * G[x * k + x]) + (AH[row * k + x] - s);
          v = (v < kEps17) ? kEps17 : v;
          W[row * k + x] = v;
          ss = fma(v, v, ss);
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
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    double t = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) t += part[b];
    norms[x] = sqrt(t);
    *counter = 0;
  }
}

// NMF::normalize_by_W (common/nmf.hpp:150-160) from k_colsumsq_partial's
// per-CTA column sums of W^2: every CTA adds the partials in CTA order, then
// W(:, c) /= norm_c and H(:, c) *= norm_c (norm_c > 0) over its rows.
constexpr int NRM_ROWS = 64;
__global__ void __launch_bounds__(256) k_nmf_rescale(double* __restrict__ W, int64_t m,
                                                     double* __restrict__ H, int64_t n, int k,
                                                     const double* __restrict__ part, int nblk) {
  __shared__ double nrm[kMaxRank];
  if (threadIdx.x < k) {
    double t = 0.0;
    for (int b = 0; b < nblk; ++b) t += part[(int64_t)b * k + threadIdx.x];
    nrm[threadIdx.x] = sqrt(t);
  }
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
// common/nmf.hpp:428-431). Writes obj[*ctr], rel[*ctr] and increments *ctr.
// One CTA of 1024 threads; every sum is in a fixed order.
__global__ void __launch_bounds__(1024) k_nmf_error(const double* __restrict__ W, int64_t m,
                                                    const double* __restrict__ H, int64_t n, int k,
                                                    const double* __restrict__ AtW,
                                                    const double* __restrict__ GW,
                                                    const double* __restrict__ GH,
                                                    const double* __restrict__ normA2, NmfReg reg,
                                                    double* __restrict__ obj, double* __restrict__ rel,
                                                    int* __restrict__ ctr) {
  __shared__ double red[5][1024];
  const int tid = threadIdx.x;
  double tr = 0.0, l1w = 0.0, l1h = 0.0, sym = 0.0, ww = 0.0;
  for (int64_t e = tid; e < n * k; e += 1024) tr = fma(H[e], AtW[e], tr);
  // row sums: thread per row
  for (int64_t r = tid; r < m; r += 1024) {
    double s = 0.0;
    for (int c = 0; c < k; ++c) s += W[r * k + c];
    l1w = fma(s, s, l1w);
  }
  for (int64_t r = tid; r < n; r += 1024) {
    double s = 0.0;
    for (int c = 0; c < k; ++c) s += H[r * k + c];
    l1h = fma(s, s, l1h);
  }
  if (reg.sym > 0)
    for (int64_t e = tid; e < m * k; e += 1024) {
      const double d = W[e] - H[e];
      sym = fma(d, d, sym);
    }
  for (int e = tid; e < k * k; e += 1024) ww = fma(GW[e], GH[(e % k) * k + e / k], ww);
  red[0][tid] = tr;
  red[1][tid] = l1w;
  red[2][tid] = l1h;
  red[3][tid] = sym;
  red[4][tid] = ww;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (tid < s)
#pragma unroll
      for (int q = 0; q < 5; ++q) red[q][tid] += red[q][tid + s];
    __syncthreads();
  }
  if (tid == 0) {
    double fro_w = 0.0, fro_h = 0.0;
    for (int i = 0; i < k; ++i) {
      fro_w += GW[i * k + i];
      fro_h += GH[i * k + i];
    }
    const double a2 = *normA2;
    const double fit = a2 - (2 * red[0][0]) + red[4][0];
    const double o = fit + reg.w2 * fro_w + reg.h2 * fro_h + reg.w1 * red[1][0] +
                     reg.h1 * red[2][0] + (reg.sym > 0 ? reg.sym * red[3][0] : 0.0);
    const double na = sqrt(a2);
    const int c = *ctr;
    obj[c] = o;
    rel[c] = (fit > 0 ? sqrt(fit) : na) / na;
    *ctr = c + 1;
  }
}

}  // namespace pg
