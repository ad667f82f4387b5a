// bpp.cuh -- batched block-principal-pivoting NNLS (Kim & Park), one warp per
// right-hand side, all right-hand sides of a mode in one launch.
//
// Restates nnls/bppnnls.hpp:67-191 per column. In the reference every column
// carries its own P / Ninf counters and passive set, and a column that became
// optimal is never touched again (its X/Y only see the idempotent 1e-12
// zeroing), so each column's trajectory depends only on its own data; the
// reference's grouping of columns with equal passive sets
// (bppnnls.hpp:204-287) shares factorisations without changing values.
// Passive sets are bitmasks (k <= 64). Solves are FP64 Cholesky of the
// passive principal submatrix of AtA (arma::solve(..., likely_sympd)), with
// Gaussian elimination with partial pivoting when the Cholesky meets a
// non-positive pivot.
#pragma once
#include "common.cuh"

namespace pg {

constexpr int BPP_WARPS = 2;  // right-hand sides per CTA (they share the AtA copy)

__device__ __forceinline__ uint64_t warp_mask64(bool pred_lo, bool pred_hi) {
  uint64_t lo = __ballot_sync(0xffffffffu, pred_lo);
  uint64_t hi = __ballot_sync(0xffffffffu, pred_hi);
  return lo | (hi << 32);
}

// Cholesky solve of A z = rhs for the m x m matrix in A (column-major,
// leading dimension ld, overwritten by L), rhs in/out in z; dinv receives
// 1/L(j,j), so the column scaling and both triangular solves multiply instead
// of dividing (one division and one square root per column on the critical
// path). Warp-cooperative; at step j lane l owns rows j+1+l, j+33+l.
// Returns false (A, z clobbered) when a pivot is not positive and finite.
__device__ bool warp_chol_solve(double* A, int ld, int m, double* z, double* dinv) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < m; ++j) {
    double ajj = A[j + ld * j];
    if (!(ajj > 0.0) || !isfinite(ajj)) return false;  // uniform across the warp
    const double ljj = sqrt(ajj);
    const double inv = 1.0 / ljj;
    __syncwarp();
    for (int i = j + 1 + lane; i < m; i += 32) A[i + ld * j] = A[i + ld * j] * inv;
    if (lane == 0) {
      A[j + ld * j] = ljj;
      dinv[j] = inv;
    }
    __syncwarp();
    for (int i = j + 1 + lane; i < m; i += 32) {
      double lij = A[i + ld * j];
      for (int c = j + 1; c <= i; ++c) A[i + ld * c] = fma(-lij, A[c + ld * j], A[i + ld * c]);
    }
    __syncwarp();
  }
  for (int j = 0; j < m; ++j) {  // L y = z
    double yj = z[j] * dinv[j];
    __syncwarp();
    if (lane == 0) z[j] = yj;
    for (int i = j + 1 + lane; i < m; i += 32) z[i] = fma(-A[i + ld * j], yj, z[i]);
    __syncwarp();
  }
  for (int j = m - 1; j >= 0; --j) {  // L^T x = y
    double xj = z[j] * dinv[j];
    __syncwarp();
    if (lane == 0) z[j] = xj;
    for (int i = lane; i < j; i += 32) z[i] = fma(-A[j + ld * i], xj, z[i]);
    __syncwarp();
  }
  return true;
}

// Gaussian elimination with partial pivoting (the general-solver fallback of
// a failed Cholesky). Returns 0 or kStSingular.
__device__ int warp_lu_solve(double* A, int ld, int m, double* z) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < m; ++j) {
    double best = -1.0;
    int piv = j;
    for (int i = j + lane; i < m; i += 32) {
      double v = fabs(A[i + ld * j]);
      if (v > best) { best = v; piv = i; }
    }
    for (int off = 16; off > 0; off >>= 1) {
      double ob = __shfl_down_sync(0xffffffffu, best, off);
      int op = __shfl_down_sync(0xffffffffu, piv, off);
      if (ob > best || (ob == best && op < piv)) { best = ob; piv = op; }
    }
    best = __shfl_sync(0xffffffffu, best, 0);
    piv = __shfl_sync(0xffffffffu, piv, 0);
    if (!(best > 0.0) || !isfinite(best)) return kStSingular;
    if (piv != j) {
      for (int c = lane; c < m; c += 32) {
        double t = A[j + ld * c];
        A[j + ld * c] = A[piv + ld * c];
        A[piv + ld * c] = t;
      }
      if (lane == 0) {
        double t = z[j];
        z[j] = z[piv];
        z[piv] = t;
      }
    }
    __syncwarp();
    double d = A[j + ld * j];
    for (int i = j + 1 + lane; i < m; i += 32) {
      double f = A[i + ld * j] / d;
      for (int c = j + 1; c < m; ++c) A[i + ld * c] = fma(-f, A[j + ld * c], A[i + ld * c]);
      z[i] = fma(-f, z[j], z[i]);
    }
    __syncwarp();
  }
  for (int j = m - 1; j >= 0; --j) {
    double xj = z[j] / A[j + ld * j];
    __syncwarp();
    if (lane == 0) z[j] = xj;
    for (int i = lane; i < j; i += 32) z[i] = fma(-A[i + ld * j], xj, z[i]);
    __syncwarp();
  }
  return 0;
}

// One warp per right-hand side c, BPP_WARPS right-hand sides per CTA: AtA
// (n x n) is staged once in shared memory for all warps of the CTA; rhs
// b_c = B[c*n .. c*n+n-1] (row-major ncols x n == column-major n x ncols),
// X_c written the same way. passive/iters (optional) receive the final
// passive set and the iteration count. *status receives the most negative
// failure code (0 if none). Dynamic shared memory: bpp_smem_bytes(KP).
__host__ __device__ constexpr size_t bpp_smem_bytes(int KP) {
  return (size_t)KP * KP * 8 * (1 + BPP_WARPS) + (size_t)BPP_WARPS * (5 * KP * 8 + KP * 4);
}

template <int KP>
__global__ void __launch_bounds__(32 * BPP_WARPS) k_bpp(const double* __restrict__ AtA_g,
                                                        const double* __restrict__ Bm, int n,
                                                        int64_t ncols, double* __restrict__ Xout,
                                                        int* __restrict__ passive_out,
                                                        int* __restrict__ iters_out,
                                                        int* __restrict__ status, int max_iter_override) {
  extern __shared__ __align__(16) unsigned char bpp_smem[];
  double* AtA = reinterpret_cast<double*>(bpp_smem);  // n x n, leading dimension n
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) AtA[e] = AtA_g[e];
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* A = AtA + KP * KP + (size_t)w * (KP * KP + 5 * KP);
  double* x = A + KP * KP;
  double* y = x + KP;
  double* b = y + KP;
  double* z = b + KP;
  double* dinv = z + KP;
  int* idx = reinterpret_cast<int*>(AtA + KP * KP + (size_t)BPP_WARPS * (KP * KP + 5 * KP)) + w * KP;
  const int64_t c = (int64_t)blockIdx.x * BPP_WARPS + w;
  if (c >= ncols) return;  // whole warp leaves together (no CTA barrier follows)
  const bool has_lo = lane < n, has_hi = lane + 32 < n;
  for (int i = lane; i < n; i += 32) {
    b[i] = Bm[c * n + i];
    x[i] = 0.0;
    y[i] = -b[i];  // Y = AtA*0 - AtB, bppnnls.hpp:73
  }
  __syncwarp();
  uint64_t passive = 0;  // PassiveSet = (X > 0) = {}, bppnnls.hpp:74
  const int pbar = 3;
  int P = pbar, Ninf = n + 1;  // bppnnls.hpp:76-81
  // bppnnls.hpp:69 (MAX_ITERATIONS = 5n); a positive override lowers the cap
  const unsigned max_it = max_iter_override > 0 ? (unsigned)max_iter_override : 5u * (unsigned)n;
  auto classify = [&](uint64_t& nonopt, uint64_t& infea) {
    bool lo_no = has_lo && (y[lane] < 0) && !((passive >> lane) & 1);
    bool hi_no = has_hi && (y[lane + 32] < 0) && !((passive >> (lane + 32)) & 1);
    bool lo_in = has_lo && (x[lane] < 0) && ((passive >> lane) & 1);
    bool hi_in = has_hi && (x[lane + 32] < 0) && ((passive >> (lane + 32)) & 1);
    nonopt = warp_mask64(lo_no, hi_no);
    infea = warp_mask64(lo_in, hi_in);
  };
  uint64_t nonopt, infea;
  classify(nonopt, infea);
  int notgood = __popcll(nonopt) + __popcll(infea);
  unsigned iter = 0;
  int st = 0;
  while (notgood > 0) {
    ++iter;
    if (iter > max_it) { st = kStBppMaxIter; break; }
    if (notgood < Ninf) {  // Cols1, bppnnls.hpp:109, 115-129
      P = pbar;
      Ninf = notgood;
      passive = (passive | nonopt) & ~infea;
    } else if (P >= 1) {  // Cols2, bppnnls.hpp:110, 133-146
      P -= 1;
      passive = (passive | nonopt) & ~infea;
    } else {  // backup rule: flip the largest offending index, bppnnls.hpp:149-160
      int rowidx = 63 - __clzll(nonopt | infea);
      passive ^= (1ull << rowidx);
    }
    // gather the passive submatrix, bppnnls.hpp:163-166 / 204-259
    const int m = __popcll(passive);
    // idx[q] = position of the q-th passive index (warp-parallel compaction)
    if ((passive >> lane) & 1) idx[__popcll(passive & ((1ull << lane) - 1ull))] = lane;
    if ((passive >> (lane + 32)) & 1)
      idx[__popcll(passive & ((1ull << (lane + 32)) - 1ull))] = lane + 32;
    __syncwarp();
    auto gather = [&]() {
      for (int e = lane; e < m * m; e += 32) {
        int ii = e % m, jj = e / m;
        A[ii + KP * jj] = AtA[idx[ii] + n * idx[jj]];
      }
      for (int i = lane; i < m; i += 32) z[i] = b[idx[i]];
      __syncwarp();
    };
    gather();
    if (m > 0 && !warp_chol_solve(A, KP, m, z, dinv)) {
      gather();
      int rc = warp_lu_solve(A, KP, m, z);
      if (rc != 0) { st = rc; break; }
    }
    for (int i = lane; i < n; i += 32) x[i] = 0.0;
    __syncwarp();
    for (int i = lane; i < m; i += 32) x[idx[i]] = z[i];
    __syncwarp();
    // Y = AtA*X - AtB (bppnnls.hpp:167-168), then the 1e-12 zeroing (170-172)
    for (int i = lane; i < n; i += 32) {
      double acc = 0.0;
      for (int j = 0; j < n; ++j) acc = fma(AtA[i + n * j], x[j], acc);
      double yi = acc - b[i];
      y[i] = (fabs(yi) < kEps12) ? 0.0 : yi;
      double xi = x[i];
      if (!isfinite(xi) || !isfinite(yi)) st = kStNonFinite;
      x[i] = (fabs(xi) < kEps12) ? 0.0 : xi;
    }
    __syncwarp();
    st = __reduce_min_sync(0xffffffffu, st);
    if (st != 0) break;
    classify(nonopt, infea);
    notgood = __popcll(nonopt) + __popcll(infea);
  }
  for (int i = lane; i < n; i += 32) {
    Xout[c * n + i] = x[i];
    if (passive_out) passive_out[c * n + i] = (int)((passive >> i) & 1);
  }
  if (lane == 0) {
    if (iters_out) iters_out[c] = (int)iter;
    if (st != 0) atomicMin(status, st);
  }
}

}  // namespace pg
