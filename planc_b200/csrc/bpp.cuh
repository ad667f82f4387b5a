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

// Blocked left-looking (Crout) Cholesky of the passive principal submatrix
// A(i,j) = AtA[idx[i] + n*idx[j]], i,j < m, into Ls (column-major, leading
// dimension KP+1: odd, so that walking a row and walking a column are both
// free of shared-memory bank conflicts). Lane l owns rows l and l+32 of the
// factor; inv[q] receives 1/L(row,row) for its rows. Columns go in panels of
// NB: first every owned row at or below the panel takes the contribution of
// all finished columns to the NB panel columns (NB independent accumulators
// per row, one load of L(row,c) shared by NB fused multiply-adds), then the
// panel is factored column by column in registers, the panel rows' entries
// travelling by shuffle. Only the strict lower triangle is stored.
// Returns false when a pivot is not positive and finite (uniform across the
// warp), where the reference's Cholesky solve fails too.
template <int KP>
__device__ __forceinline__ bool warp_chol_crout(const double* __restrict__ AtA, int n, const int* idx,
                                                int m, double* Ls, double (&inv)[KP > 32 ? 2 : 1]) {
  constexpr int LD = KP + 1, R = KP > 32 ? 2 : 1, NB = 8;
  const int lane = threadIdx.x & 31;
  int gi[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int row = lane + 32 * q;
    gi[q] = row < m ? idx[row] : 0;
    inv[q] = 0.0;
  }
  for (int j0 = 0; j0 < m; j0 += NB) {
    const int pw = min(NB, m - j0);
    double acc[R][NB];
#pragma unroll
    for (int q = 0; q < R; ++q)
#pragma unroll
      for (int t = 0; t < NB; ++t) acc[q][t] = 0.0;
    // contribution of the finished columns c < j0
    for (int c = 0; c < j0; ++c) {
      double lj[NB];
#pragma unroll
      for (int t = 0; t < NB; ++t) lj[t] = t < pw ? Ls[j0 + t + LD * c] : 0.0;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int row = lane + 32 * q;
        if (32 * q + 31 >= j0) {  // warp-uniform: some owned row of this slot is in play
          const double li = (row >= j0 && row < m) ? Ls[row + LD * c] : 0.0;
#pragma unroll
          for (int t = 0; t < NB; ++t) acc[q][t] = fma(li, lj[t], acc[q][t]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      if (t < pw) {
        const double* colA = AtA + (size_t)n * idx[j0 + t];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int row = lane + 32 * q;
          acc[q][t] = (row >= j0 && row < m) ? colA[gi[q]] - acc[q][t] : 0.0;
        }
      }
    }
    // factor the panel
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      if (t < pw) {
        const int jj = j0 + t;
        const double sjj = __shfl_sync(0xffffffffu, jj < 32 ? acc[0][t] : acc[R - 1][t], jj & 31);
        if (!(sjj > 0.0) || !isfinite(sjj)) return false;
        const double ij = rsqrt(sjj);
        double lcol[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int row = lane + 32 * q;
          lcol[q] = acc[q][t] * ij;
          if (row > jj && row < m) Ls[row + LD * jj] = lcol[q];
          if (row == jj) inv[q] = ij;
        }
#pragma unroll
        for (int t2 = t + 1; t2 < NB; ++t2) {
          if (t2 < pw) {
            const int r2 = j0 + t2;
            const double l2 = __shfl_sync(0xffffffffu, r2 < 32 ? lcol[0] : lcol[R - 1], r2 & 31);
#pragma unroll
            for (int q = 0; q < R; ++q) acc[q][t2] = fma(-lcol[q], l2, acc[q][t2]);
          }
        }
      }
    }
    __syncwarp();
  }
  return true;
}

// Forward and back substitution with the factor of warp_chol_crout: z (the
// owned rows' right-hand side) becomes the solution in place. Each step is
// one shuffle of the finished entry plus one fused multiply-add per owned
// row; the factor entries are independent loads that the compiler hoists.
template <int KP>
__device__ __forceinline__ void warp_chol_subst(const double* Ls, int m, const double (&inv)[KP > 32 ? 2 : 1],
                                double (&z)[KP > 32 ? 2 : 1]) {
  constexpr int LD = KP + 1, R = KP > 32 ? 2 : 1;
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < m; ++j) {  // L y = z
    const double t = j < 32 ? z[0] * inv[0] : z[R - 1] * inv[R - 1];
    const double yj = __shfl_sync(0xffffffffu, t, j & 31);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = lane + 32 * q;
      if (row == j) z[q] = yj;
      else if (row > j && row < m) z[q] = fma(-Ls[row + LD * j], yj, z[q]);
    }
  }
  for (int j = m - 1; j >= 0; --j) {  // L^T x = y
    const double t = j < 32 ? z[0] * inv[0] : z[R - 1] * inv[R - 1];
    const double xj = __shfl_sync(0xffffffffu, t, j & 31);
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = lane + 32 * q;
      if (row == j) z[q] = xj;
      else if (row < j) z[q] = fma(-Ls[j + LD * row], xj, z[q]);
    }
  }
}

// Gaussian elimination with partial pivoting (the general-solver fallback of
// a failed Cholesky). Returns 0 or kStSingular.
__device__ __forceinline__ int warp_lu_solve(double* A, int ld, int m, double* z) {
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
// Per warp: the factor (KP x (KP+1)), x, y, b and the compacted solution zs
// (KP each), and the passive index list idx (KP ints).
__host__ __device__ constexpr size_t bpp_smem_bytes(int KP) {
  return (size_t)KP * KP * 8 + (size_t)BPP_WARPS * ((size_t)KP * (KP + 1) * 8 + 4 * KP * 8 + KP * 4);
}

template <int KP>
__global__ void __launch_bounds__(32 * BPP_WARPS, 1) k_bpp(const double* __restrict__ AtA_g,
                                                        const double* __restrict__ Bm, int n,
                                                        int64_t ncols, double* __restrict__ Xout,
                                                        int* __restrict__ passive_out,
                                                        int* __restrict__ iters_out,
                                                        int* __restrict__ status, int max_iter_override,
                                                        const double* __restrict__ Pinit) {
  constexpr int LD = KP + 1, R = KP > 32 ? 2 : 1;
  extern __shared__ __align__(16) unsigned char bpp_smem[];
  double* AtA = reinterpret_cast<double*>(bpp_smem);  // n x n, leading dimension n
  {
    const int nn = n * n;
    for (int e0 = threadIdx.x; e0 < nn; e0 += 8 * blockDim.x) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * blockDim.x;
        v[u] = e < nn ? __ldg(AtA_g + e) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int e = e0 + u * blockDim.x;
        if (e < nn) AtA[e] = v[u];
      }
    }
  }
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* Ls = AtA + KP * KP + (size_t)w * (KP * LD + 4 * KP);
  double* x = Ls + KP * LD;
  double* y = x + KP;
  double* b = y + KP;
  double* zs = b + KP;
  int* idx = reinterpret_cast<int*>(AtA + KP * KP + (size_t)BPP_WARPS * (KP * LD + 4 * KP)) + w * KP;
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
  // X(P) = solve(AtA(P,P), AtB(P)), X(~P) = 0, Y = AtA X - AtB and the 1e-12
  // zeroing for the current passive set; returns 0 or a failure status
  auto solve_passive = [&]() -> int {
    int bad = 0;
    // solve the passive system AtA(P,P) x_P = AtB(P), bppnnls.hpp:163-166 / 204-259
    const int m = __popcll(passive);
    // idx[q] = position of the q-th passive index (warp-parallel compaction)
    if ((passive >> lane) & 1) idx[__popcll(passive & ((1ull << lane) - 1ull))] = lane;
    if ((passive >> (lane + 32)) & 1)
      idx[__popcll(passive & ((1ull << (lane + 32)) - 1ull))] = lane + 32;
    __syncwarp();
    double z[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = lane + 32 * q;
      z[q] = row < m ? b[idx[row]] : 0.0;
    }
    double inv[R];
    if (m > 0) {
      if (warp_chol_crout<KP>(AtA, n, idx, m, Ls, inv)) {
        warp_chol_subst<KP>(Ls, m, inv, z);
      } else {  // not positive definite: the general solver, as arma::solve falls back
        for (int e = lane; e < m * m; e += 32) {
          const int ii = e % m, jj = e / m;
          Ls[ii + LD * jj] = AtA[idx[ii] + n * idx[jj]];
        }
        for (int i = lane; i < m; i += 32) zs[i] = b[idx[i]];
        __syncwarp();
        const int rc = warp_lu_solve(Ls, LD, m, zs);
        if (rc != 0) return rc;
        __syncwarp();
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int row = lane + 32 * q;
          z[q] = row < m ? zs[row] : 0.0;
        }
      }
    }
    // scatter: X(P) = x_P, X(~P) = 0
    for (int i = lane; i < n; i += 32) x[i] = 0.0;
    __syncwarp();
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int row = lane + 32 * q;
      if (row < m) {
        x[idx[row]] = z[q];
        zs[row] = z[q];
      }
    }
    __syncwarp();
    // Y = AtA*X - AtB over the passive columns (bppnnls.hpp:167-168), then the
    // 1e-12 zeroing of X and Y (bppnnls.hpp:170-172)
    for (int i = lane; i < n; i += 32) {
      double a0 = 0.0, a1 = 0.0;
      int q = 0;
      for (; q + 2 <= m; q += 2) {
        a0 = fma(AtA[i + n * idx[q]], zs[q], a0);
        a1 = fma(AtA[i + n * idx[q + 1]], zs[q + 1], a1);
      }
      if (q < m) a0 = fma(AtA[i + n * idx[q]], zs[q], a0);
      const double yi = (a0 + a1) - b[i];
      y[i] = (fabs(yi) < kEps12) ? 0.0 : yi;
      const double xi = x[i];
      if (!isfinite(xi) || !isfinite(yi)) bad = kStNonFinite;
      x[i] = (fabs(xi) < kEps12) ? 0.0 : xi;
    }
    __syncwarp();
    __syncwarp();
    return __reduce_min_sync(0xffffffffu, bad);
  };
  unsigned iter = 0;
  int st = 0;
  if (Pinit) {
    // warm start from the previous solution's passive set: with AtA positive
    // definite BPP reaches the unique NNLS optimum from any starting set (Kim
    // & Park), so the result is the reference's; only the number of exchange
    // steps changes. When AtA is singular (a component whose factor column
    // collapsed to zero leaves a zero row and column) the optimum is not
    // unique and the warm set's system may be singular: a failed warm solve
    // restarts from the reference's start, X = 0 (bppnnls.hpp:73-74).
    const bool lo = has_lo && Pinit[c * n + lane] > 0.0;
    const bool hi = has_hi && Pinit[c * n + lane + 32] > 0.0;
    passive = warp_mask64(lo, hi);
    __syncwarp();  // every lane has read its Pinit before any store below
    if (passive) {
      ++iter;
      st = solve_passive();
      if (st != 0) {
        st = 0;
        iter = 0;
        passive = 0;
        for (int i = lane; i < n; i += 32) {
          x[i] = 0.0;
          y[i] = -b[i];
        }
        __syncwarp();
      }
    }
  }
  uint64_t nonopt = 0, infea = 0;
  int notgood = 0;
  if (st == 0) {
    classify(nonopt, infea);
    notgood = __popcll(nonopt) + __popcll(infea);
  }
  while (st == 0 && notgood > 0) {
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
    st = solve_passive();
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

// ------------------------------------------------------------ CTA per row
// The same BPP trajectory with one CTA per right-hand side (k_bpp gives each
// one warp): for the few-hundred-row modes of a 4-way tensor a warp per row
// leaves most SMs and schedulers idle and every step waits on one warp's
// dependency chain, so the passive solve is spread over the whole CTA.
//
// Passive solve: right-looking Cholesky of the passive principal submatrix
// bordered by the right-hand side, [S; z^T] (rows 0..m-1 the compacted
// passive indices, row KP the right-hand side). Eliminating column j
// subtracts S(i, j) S(c, j) / S(j, j) from every later entry (i, c); the
// bordered row then holds y = L^{-1} z, and one warp finishes with the back
// substitution L^T x = y. The lower triangle is held in registers: the
// thread of segment t owns SEGW consecutive entries (row i, columns c0 ..
// c0+SEGW-1) for the whole factorisation. After its update of column j the
// owner of column j+1 publishes it to cbuf(:, j+1), and the owner of the
// diagonal entry also publishes s = 1 / sqrt(pivot) and s^2 (or marks the
// pivot as failed), so each column costs one barrier of the threads that own
// segments; cbuf keeps every column, which is the factor the back
// substitution reads (L(i, j) = cbuf(i, j) * s_j). Column entries sit at
// i + i / 8, so the eight entries a segment reads lie in distinct banks for
// the segments of one warp. Segments are numbered row by row (row i has
// i / SEGW + 1 of them), so the segments of an m-row system are the first
// ones for every m, followed by the ceil(m / SEGW) segments of the bordered
// row.
template <int KP, int SEGW>
struct BppCta {
  static constexpr int NBLK = KP / SEGW;                       // segments of a full row
  static constexpr int NSEG = SEGW * NBLK * (NBLK + 1) / 2 + NBLK;
  static constexpr int THREADS = (NSEG + 31) / 32 * 32;
  // column stride of cbuf: entries 0..KP at i + i / 8; odd, so that walking a
  // row across columns is conflict-free too
  static constexpr int LDC = KP + KP / 8 + 1;
  // threads per row of the Y = AtA X - AtB product (a power of two <= 32)
  static constexpr int TPR = THREADS / KP >= 8 ? 8 : THREADS / KP >= 4 ? 4 : THREADS / KP >= 2 ? 2 : 1;
  static constexpr size_t SMEM = ((size_t)KP * KP + (size_t)KP * LDC + 6 * (size_t)KP) * 8 + (size_t)KP * 4 + 16;
};

// segments of the rows 0..m-1 (row i has i / segw + 1)
__host__ __device__ constexpr int bppc_row_segments(int m, int segw) {
  return segw * (m / segw) * (m / segw + 1) / 2 + (m % segw) * (m / segw + 1);
}

template <int KP, int SEGW>
__global__ void __launch_bounds__(BppCta<KP, SEGW>::THREADS, 2)
    k_bpp_cta(const double* __restrict__ AtA_g, const double* __restrict__ Bm, int n, int64_t ncols,
              double* __restrict__ Xout, int* __restrict__ passive_out, int* __restrict__ iters_out,
              int* __restrict__ status, int max_iter_override, const double* __restrict__ Pinit) {
  using C = BppCta<KP, SEGW>;
  constexpr int LDC = C::LDC, TPR = C::TPR, NT = C::THREADS;
  extern __shared__ __align__(16) unsigned char bppc_smem[];
  double* AtA = reinterpret_cast<double*>(bppc_smem);  // n x n, leading dimension n
  double* cbuf = AtA + KP * KP;                         // column j: cbuf[j * LDC + i + i / 8], i <= KP
  double* sv = cbuf + KP * LDC;                         // 1 / sqrt(pivot j)
  double* qv = sv + KP;                                 // 1 / pivot j
  double* x = qv + KP;
  double* y = x + KP;
  double* b = y + KP;
  double* z = b + KP;  // compacted solution
  int* idx = reinterpret_cast<int*>(z + KP);
  __shared__ int lu_rc;
  __shared__ int bad_at;  // first pivot that is not positive and finite (KP + 1: none)
  const int tid = threadIdx.x, lane = tid & 31;
  for (int e = tid; e < n * n; e += NT) AtA[e] = __ldg(AtA_g + e);
  // this thread's segment of the full triangle: row block q holds rows
  // q*SEGW .. q*SEGW+SEGW-1 with q+1 segments each
  int seg_row = -1, seg_c0 = 0;
  {
    int base = 0;
    for (int q = 0; q < C::NBLK; ++q) {
      const int cnt = SEGW * (q + 1);
      if (tid >= base && tid < base + cnt) {
        seg_row = q * SEGW + (tid - base) / (q + 1);
        seg_c0 = SEGW * ((tid - base) % (q + 1));
      }
      base += cnt;
    }
  }
  const bool has_lo = lane < n, has_hi = lane + 32 < n;
  const int pbar = 3;
  const unsigned max_it = max_iter_override > 0 ? (unsigned)max_iter_override : 5u * (unsigned)n;

  for (int64_t c = blockIdx.x; c < ncols; c += gridDim.x) {
    __syncthreads();  // AtA staged / the previous row's buffers are free
    for (int i = tid; i < n; i += NT) {
      b[i] = Bm[c * n + i];
      x[i] = 0.0;
      y[i] = -b[i];  // Y = AtA*0 - AtB, bppnnls.hpp:73
    }
    uint64_t passive = 0;  // bppnnls.hpp:74
    int P = pbar, Ninf = n + 1;  // bppnnls.hpp:76-81

    // X(P) = solve(AtA(P,P), AtB(P)), X(~P) = 0, Y = AtA X - AtB and the
    // 1e-12 zeroing (bppnnls.hpp:163-172); uniform across the CTA
    auto solve_passive = [&]() -> int {
      const int m = __popcll(passive);
      __syncthreads();  // x, y, b of the previous step read by every warp
      if (tid < 32) {
        if ((passive >> lane) & 1) idx[__popcll(passive & ((1ull << lane) - 1ull))] = lane;
        if ((passive >> (lane + 32)) & 1)
          idx[__popcll(passive & ((1ull << (lane + 32)) - 1ull))] = lane + 32;
        if (lane == 0) bad_at = KP + 1;
      }
      __syncthreads();
      const int nrow = bppc_row_segments(m, SEGW);
      const int nact = nrow + (m + SEGW - 1) / SEGW;
      int row = -1, c0 = 0;
      if (tid < nrow) {
        row = seg_row;
        c0 = seg_c0;
      } else if (tid < nact) {
        row = KP;  // the bordered right-hand-side row
        c0 = SEGW * (tid - nrow);
      }
      const int cb0 = c0 + (c0 >> 3);  // position of column c0 in a cbuf column
      const int rpos = row + (row >> 3);
      auto publish_pivot = [&](int j, double d) {
        if (!(d > 0.0) || !isfinite(d)) {
          bad_at = j;
        } else {
          const double sj = rsqrt(d);
          sv[j] = sj;
          qv[j] = sj * sj;
        }
      };
      double v[SEGW];
      {
        const int gi = (row >= 0 && row < KP) ? idx[row] : 0;
#pragma unroll
        for (int u = 0; u < SEGW; ++u) {
          const int cc = c0 + u;
          double e = 0.0;
          if (row == KP) {
            if (cc < m) e = b[idx[cc]];
          } else if (row >= 0 && cc <= row) {
            e = AtA[gi + n * idx[cc]];
          }
          v[u] = e;
        }
      }
      if (row >= 0 && c0 == 0) {
        cbuf[rpos] = v[0];
        if (row == 0) publish_pivot(0, v[0]);
      }
      __syncthreads();
      // the warps that own segments step through the columns; bad_at only
      // ever changes to j + 1 during step j, so every thread takes the same
      // exit
      const int nthr = (nact + 31) & ~31;
      if (tid < nthr) {
        for (int j = 0; j < m; ++j) {
          if (bad_at <= j) break;
          const double* col = cbuf + j * LDC;
          if (row >= 0 && (row == KP || row > j) && c0 + SEGW - 1 > j) {
            const double w = col[rpos] * qv[j];
            // entries left of column j + 1, right of the row's last column,
            // or past m are never read again: updating them unconditionally
            // keeps the inner loop free of predicates
#pragma unroll
            for (int u = 0; u < SEGW; ++u) v[u] = fma(-w, col[cb0 + u], v[u]);
            const int jn = j + 1;
            if (jn < m && jn >= c0 && jn < c0 + SEGW && (row == KP || row >= jn)) {
#pragma unroll
              for (int u = 0; u < SEGW; ++u)
                if (c0 + u == jn) {
                  cbuf[jn * LDC + rpos] = v[u];
                  if (row == jn) publish_pivot(jn, v[u]);
                }
            }
          }
          asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory");
        }
      }
      __syncthreads();
      const bool chol_ok = bad_at > KP;
      if (chol_ok) {
        if (tid < 32 && m > 0) {  // L^T x = y, y_j = cbuf(KP, j) * s_j
          double r[2], sl[2];
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int cc = lane + 32 * q;
            sl[q] = cc < m ? sv[cc] : 0.0;
            r[q] = cc < m ? cbuf[cc * LDC + KP + KP / 8] * sl[q] : 0.0;
          }
          for (int j = m - 1; j >= 0; --j) {
            const double t = (j < 32 ? r[0] : r[1]) * sv[j];
            const double xj = __shfl_sync(0xffffffffu, t, j & 31);
            const int jpos = j + (j >> 3);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
              const int cc = lane + 32 * q;
              if (cc < j) r[q] = fma(-(cbuf[cc * LDC + jpos] * sl[q]), xj, r[q]);
              else if (cc == j) r[q] = xj;
            }
          }
#pragma unroll
          for (int q = 0; q < 2; ++q) {
            const int cc = lane + 32 * q;
            if (cc < m) z[cc] = r[q];
          }
        }
      } else {
        // not positive definite: the general solver, as arma::solve falls back
        __syncthreads();  // every thread has read the failing pivot before cbuf is reused
        double* Ls = cbuf;
        for (int e = tid; e < m * m; e += NT) {
          const int ii = e % m, jj = e / m;
          Ls[ii + LDC * jj] = AtA[idx[ii] + n * idx[jj]];
        }
        for (int i = tid; i < m; i += NT) z[i] = b[idx[i]];
        __syncthreads();
        if (tid < 32) {
          const int rc = warp_lu_solve(Ls, LDC, m, z);
          if (lane == 0) lu_rc = rc;
        }
        __syncthreads();
        if (lu_rc != 0) return lu_rc;
      }
      __syncthreads();  // z complete
      // Y = AtA*X - AtB over the passive columns (bppnnls.hpp:167-168), then
      // the 1e-12 zeroing of X and Y (bppnnls.hpp:170-172)
      int bad = 0;
      for (int base = 0; base < n; base += NT / TPR) {
        const int i = base + tid / TPR, part = tid % TPR;
        double acc = 0.0;
        if (i < n)
          for (int q = part; q < m; q += TPR) acc = fma(AtA[i + n * idx[q]], z[q], acc);
#pragma unroll
        for (int off = TPR / 2; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        if (i < n && part == 0) {
          const double yi = acc - b[i];
          y[i] = (fabs(yi) < kEps12) ? 0.0 : yi;
          const double xi =
              ((passive >> i) & 1) ? z[__popcll(passive & ((1ull << i) - 1ull))] : 0.0;
          if (!isfinite(xi) || !isfinite(yi)) bad = 1;
          x[i] = (fabs(xi) < kEps12) ? 0.0 : xi;
        }
      }
      return __syncthreads_or(bad) ? kStNonFinite : 0;
    };
    auto classify = [&](uint64_t& nonopt, uint64_t& infea) {
      bool lo_no = has_lo && (y[lane] < 0) && !((passive >> lane) & 1);
      bool hi_no = has_hi && (y[lane + 32] < 0) && !((passive >> (lane + 32)) & 1);
      bool lo_in = has_lo && (x[lane] < 0) && ((passive >> lane) & 1);
      bool hi_in = has_hi && (x[lane + 32] < 0) && ((passive >> (lane + 32)) & 1);
      nonopt = warp_mask64(lo_no, hi_no);
      infea = warp_mask64(lo_in, hi_in);
    };

    unsigned iter = 0;
    int st = 0;
    if (Pinit) {
      // warm start from the previous solution's passive set (see k_bpp): a
      // failed warm solve restarts from the reference's X = 0
      const bool lo = has_lo && Pinit[c * n + lane] > 0.0;
      const bool hi = has_hi && Pinit[c * n + lane + 32] > 0.0;
      passive = warp_mask64(lo, hi);
      if (passive) {
        ++iter;
        st = solve_passive();
        if (st != 0) {
          st = 0;
          iter = 0;
          passive = 0;
          __syncthreads();
          for (int i = tid; i < n; i += NT) {
            x[i] = 0.0;
            y[i] = -b[i];
          }
        }
      }
    }
    __syncthreads();  // b, x, y visible to every warp
    uint64_t nonopt = 0, infea = 0;
    int notgood = 0;
    if (st == 0) {
      classify(nonopt, infea);
      notgood = __popcll(nonopt) + __popcll(infea);
    }
    while (st == 0 && notgood > 0) {
      ++iter;
      if (iter > max_it) { st = kStBppMaxIter; break; }
      if (notgood < Ninf) {  // Cols1, bppnnls.hpp:109, 115-129
        P = pbar;
        Ninf = notgood;
        passive = (passive | nonopt) & ~infea;
      } else if (P >= 1) {  // Cols2, bppnnls.hpp:110, 133-146
        P -= 1;
        passive = (passive | nonopt) & ~infea;
      } else {  // backup rule, bppnnls.hpp:149-160
        int rowidx = 63 - __clzll(nonopt | infea);
        passive ^= (1ull << rowidx);
      }
      st = solve_passive();
      if (st != 0) break;
      classify(nonopt, infea);
      notgood = __popcll(nonopt) + __popcll(infea);
    }
    for (int i = tid; i < n; i += NT) {
      Xout[c * n + i] = x[i];
      if (passive_out) passive_out[c * n + i] = (int)((passive >> i) & 1);
    }
    if (tid == 0) {
      if (iters_out) iters_out[c] = (int)iter;
      if (st != 0) atomicMin(status, st);
    }
  }
}

}  // namespace pg
