// kernels_f64.cuh -- FP64 kernels of the NTF iteration: tensor contractions
// (partial / direct MTTKRP), multi-TTV, split-K reduction, MU / HALS row
// sweeps, normalisation + Gram, Gram-form error, tensor norm, synthetic data.
#pragma once
#include "common.cuh"

namespace pg {

// ---------------------------------------------------------------------------
// Tensor contraction with a generated Khatri-Rao operand (FP64, DMMA).
//
//   RIGHT  (partial MTTKRP right contraction, dimtree/dimtrees.hpp:106-138,
//           and the direct mode-0 MTTKRP, common/tensor.hpp:279-281):
//             out[m, r] = sum_j X[m + ldx * j] * W(j, r),       j < K
//   LEFT   (partial MTTKRP left contraction, dimtrees.hpp:72-105, and the
//           direct mode-n MTTKRP as a batch over trailing slices,
//           tensor.hpp:298-325):
//             out[m, r] = sum_b sum_a X[a + ldx*m + ldb*b] * W(a + A*b, r)
//
// out is row-major (m, r) with row stride k; with a split-K grid
// (gridDim.y > 1) each y-slice writes its partial to out + y*split_stride and
// k_reduce_splits sums them in a fixed order (deterministic).
//
// CTA tile: 128 rows x KP ranks x BK reduction steps, 256 threads (8 warps).
// The products run on the FP64 tensor cores: warp-level
// mma.sync.m8n8k4.f64 (the only FP64 MMA of sm_100a), each warp owning a
// (128 / WARPS_M) x (KP / WARPS_N) block of the output as 8 x 8 accumulator
// tiles (a warp whose rows all lie past M skips its products). The next
// reduction tile is loaded into registers while the current one is
// multiplied out of shared memory, then stored into the other of two
// shared-memory stages: one CTA barrier per tile. Dynamic shared memory:
// ct_smem_bytes<KP, LEFT>(). Shared-memory layouts are chosen so
// that every fragment load is two 128-byte wavefronts (no bank conflicts):
//   RIGHT: Xs[kk][m], row stride 128 + 4 doubles (X is m-contiguous);
//   LEFT : Xs[m][kk], row stride BK + 4 doubles (X is kk-contiguous);
//   both : Ws[kk][r], row stride KP + 4.
// Fragment layouts of m8n8k4 (f64): A element (row g, col t), B element
// (row t, col g), C elements (row g, cols 2t, 2t+1), g = lane / 4, t = lane % 4.
// ---------------------------------------------------------------------------
constexpr int CT_BM = 128;
template <int KP>
constexpr int ct_bk() { return KP == 64 ? 16 : 32; }
// Row strides (in doubles) of the shared-memory tiles. A fragment load of
// lane (g, t) = (lane / 4, lane % 4) reads word t * S + g (+ a constant);
// a half warp (g < 4 or g >= 4) is one 128-byte wavefront when t * S mod 16
// takes the values 0, 4, 8, 12, i.e. when S = 4 or 12 (mod 16) doubles.
template <int KP>
constexpr int ct_ws() { return KP + 4; }
constexpr int CT_SXR = CT_BM + 4;  // RIGHT: Xs[kk][m]
// doubles of one shared-memory stage (X tile + W tile)
template <int KP, bool LEFT>
constexpr int ct_stage_elems() {
  return (LEFT ? CT_BM * (ct_bk<KP>() + 4) : ct_bk<KP>() * CT_SXR) + ct_bk<KP>() * ct_ws<KP>();
}
template <int KP, bool LEFT>
constexpr size_t ct_smem_bytes() { return 2 * sizeof(double) * (size_t)ct_stage_elems<KP, LEFT>(); }

struct ContractGeom {
  int64_t M;        // output rows
  int64_t ldx;      // RIGHT: column stride of X; LEFT: row (m) stride
  int64_t A;        // RIGHT: K (reduction length); LEFT: contiguous extent a
  int64_t B;        // LEFT: number of batches b (1 for a plain 2-D view)
  int64_t ldb;      // LEFT: batch stride of X
  int64_t ktiles;   // total reduction tiles
  int64_t tiles_per_split;
  int64_t split_stride;
};

__device__ __forceinline__ void dmma_m8n8k4(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// W(row, r) of a Khatri-Rao generator with NF = 1, 2 or 3 factors, digits
// in registers (NF = 0: any number of factors, wgen_eval). The product order
// is wgen_eval's, F_0 * (F_1 * F_2). `row` must be below the product of the
// dims (the caller checks its range).
template <int NF>
__device__ __forceinline__ double wgen_at(const WGen& wg, int64_t row, int r, int k) {
  if constexpr (NF == 1) {
    return wg.f[0][row * k + r];
  } else if constexpr (NF == 2) {
    const int64_t i1 = row / wg.dim[0], i0 = row - i1 * wg.dim[0];
    return wg.f[0][i0 * k + r] * wg.f[1][i1 * k + r];
  } else if constexpr (NF == 3) {
    const int64_t q = row / wg.dim[0], i0 = row - q * wg.dim[0];
    const int64_t i2 = q / wg.dim[1], i1 = q - i2 * wg.dim[1];
    return wg.f[0][i0 * k + r] * (wg.f[1][i1 * k + r] * wg.f[2][i2 * k + r]);
  } else {
    return wgen_eval(wg, row, r, k);
  }
}
// Division by a divisor fixed for the whole kernel (Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, and for n < 2^31
// n / d = (umulhi(n, m) + n) >> l (the sum stays below 2^32).
struct FastDiv {
  uint32_t d, m;
  int l;
};
__device__ __forceinline__ FastDiv make_fastdiv(uint32_t d) {
  int l = 0;
  while (l < 31 && (1u << l) < d) ++l;
  const uint64_t num = ((uint64_t)1 << 32) * (((uint64_t)1 << l) - d);
  return FastDiv{d, (uint32_t)(num / d + 1), l};
}
__device__ __forceinline__ uint32_t fast_div(uint32_t n, const FastDiv& f) {
  return (__umulhi(n, f.m) + n) >> f.l;
}

// W(row, r) as wgen_at with 32-bit digit arithmetic (the product of the dims
// < 2^31) and the digit divisions by dims 0 and 1 precomputed
template <int NF>
__device__ __forceinline__ double wgen_at32(const WGen& wg, const FastDiv& f0, const FastDiv& f1,
                                            uint32_t row, int r, int k) {
  if constexpr (NF == 2) {
    const uint32_t i1 = fast_div(row, f0), i0 = row - i1 * f0.d;
    return wg.f[0][(int64_t)i0 * k + r] * wg.f[1][(int64_t)i1 * k + r];
  } else if constexpr (NF == 3) {
    const uint32_t q = fast_div(row, f0), i0 = row - q * f0.d;
    const uint32_t i2 = fast_div(q, f1), i1 = q - i2 * f1.d;
    return wg.f[0][(int64_t)i0 * k + r] *
           (wg.f[1][(int64_t)i1 * k + r] * wg.f[2][(int64_t)i2 * k + r]);
  } else {
    return wgen_at<NF>(wg, (int64_t)row, r, k);
  }
}

// RUNS (LEFT, NF = 2 or 3): the reduction index is laid out as runs of
// g.A = dim[0] values of the fastest generator mode (g.B = the runs, g.ldb =
// g.A), so every reduction tile lies in one run b and its Khatri-Rao rows are
// W(a + A b, r) = F_0[a, r] * tail(b, r), tail = F_1[b, r] (NF = 2) or
// F_1[i1, r] * F_2[i2, r] with b = i1 + dim[1] i2 (NF = 3): a thread takes
// tail once per tile, then one F_0 load and one multiply per entry (the same
// products as wgen_at, so the same W).
template <int KP, bool LEFT, int NF, bool RUNS = false>
__global__ void __launch_bounds__(256, 2) k_contract_f64(const double* __restrict__ X,
                                                         ContractGeom g, WGen wg, int k,
                                                         double* __restrict__ out) {
  static_assert(!RUNS || (LEFT && (NF == 2 || NF == 3)), "runs of the fastest mode");
  constexpr int BK = ct_bk<KP>();
  constexpr int XPT = BK * CT_BM / 256;  // X elements per thread per tile
  constexpr int WPT = (BK * KP + 255) / 256;
  constexpr int WARPS_M = KP >= 32 ? 4 : 8;
  constexpr int WARPS_N = 8 / WARPS_M;
  constexpr int MT = CT_BM / WARPS_M / 8;  // 8-row MMA tiles per warp
  constexpr int NT = KP / WARPS_N / 8;     // 8-rank MMA tiles per warp
  constexpr int SX = LEFT ? BK + 4 : CT_SXR;
  constexpr int SW = ct_ws<KP>();
  constexpr int XS_ELEMS = LEFT ? CT_BM * SX : BK * SX;
  constexpr int STAGE = ct_stage_elems<KP, LEFT>();
  extern __shared__ __align__(16) double ct_smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int fg = lane >> 2, ft = lane & 3;
  const int wm0 = (warp % WARPS_M) * (MT * 8);
  const int wn0 = (warp / WARPS_M) * (NT * 8);
  const int64_t m0 = (int64_t)blockIdx.x * CT_BM;
  const int64_t t_begin = (int64_t)blockIdx.y * g.tiles_per_split;
  int64_t t_end = t_begin + g.tiles_per_split;
  if (t_end > g.ktiles) t_end = g.ktiles;
  const int64_t tilesA = (g.A + BK - 1) / BK;
  // Khatri-Rao row indices fit 32-bit digit arithmetic
  const bool small_rows = (LEFT ? g.A * g.B : g.A) < ((int64_t)1 << 31);
  FastDiv fd0{1, 1, 0}, fd1{1, 1, 0};
  if (NF >= 2 && small_rows && !RUNS) {
    fd0 = make_fastdiv((uint32_t)wg.dim[0]);
    if (NF >= 3) fd1 = make_fastdiv((uint32_t)wg.dim[1]);
  }
  const bool warp_live = m0 + wm0 < g.M;  // warp-uniform

  double acc[MT][NT][2];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  double xr[XPT];
  double wr[WPT];

  auto load_tile = [&](int64_t t) {
    if constexpr (!LEFT) {
      const int64_t j0 = t * BK;
      const int64_t gm = m0 + (tid & 127);
      const bool mrow = gm < g.M;
      // rows kk = (tid >> 7) + 2 i of the tile through one running pointer
      const int64_t jt = j0 + (tid >> 7);
      const double* xp = X + gm + g.ldx * jt;
      const int64_t xstep = 2 * g.ldx;
      if (mrow && j0 + BK <= g.A) {
#pragma unroll
        for (int i = 0; i < XPT; ++i) {
          xr[i] = *xp;
          xp += xstep;
        }
      } else {
#pragma unroll
        for (int i = 0; i < XPT; ++i) {
          xr[i] = (mrow && jt + 2 * i < g.A) ? *xp : 0.0;
          xp += xstep;
        }
      }
      if constexpr (NF == 1) {
        // 256 is a multiple of KP: entry i of this thread is (kk, r) =
        // (tid / KP + (256 / KP) i, tid % KP)
        const int r = tid % KP;
        const int64_t jw = j0 + tid / KP;
        const double* wp = wg.f[0] + jw * k + r;
        const int64_t wstep = (int64_t)(256 / KP) * k;
#pragma unroll
        for (int i = 0; i < WPT; ++i) {
          wr[i] = (r < k && jw + (256 / KP) * i < g.A) ? *wp : 0.0;
          wp += wstep;
        }
      } else {
#pragma unroll
        for (int i = 0; i < WPT; ++i) {
          int e = tid + 256 * i;
          double v = 0.0;
          if (e < BK * KP) {
            int kk = e / KP, r = e % KP;
            int64_t gj = j0 + kk;
            if (r < k && gj < g.A)
              v = small_rows ? wgen_at32<NF>(wg, fd0, fd1, (uint32_t)gj, r, k)
                             : wgen_at<NF>(wg, gj, r, k);
          }
          wr[i] = v;
        }
      }
    } else {
      const int64_t b = t / tilesA;
      const int64_t a0 = (t % tilesA) * BK;
      const int aa = tid % BK;
      const int64_t ga = a0 + aa;
      // rows mm = tid / BK + (256 / BK) i of the tile through one running pointer
      constexpr int MSTEP = 256 / BK;
      const int64_t gm0 = m0 + tid / BK;
      const double* xp = X + ga + g.ldx * gm0 + g.ldb * b;
      const int64_t xstep = MSTEP * g.ldx;
      if (ga < g.A && m0 + CT_BM <= g.M) {
#pragma unroll
        for (int i = 0; i < XPT; ++i) {
          xr[i] = *xp;
          xp += xstep;
        }
      } else {
#pragma unroll
        for (int i = 0; i < XPT; ++i) {
          xr[i] = (gm0 + MSTEP * i < g.M && ga < g.A) ? *xp : 0.0;
          xp += xstep;
        }
      }
      const int64_t wrow0 = a0 + g.A * b;
      if constexpr (RUNS) {
        // 256 is a multiple of KP: entry i of this thread is row
        // a = a0 + tid / KP + (256 / KP) i, rank r = tid % KP
        const int r = tid % KP;
        const int64_t a = a0 + tid / KP;
        double tail = 0.0;
        if (r < k) {
          if (NF == 2) {
            tail = wg.f[1][b * k + r];
          } else {
            const int64_t i2 = b / wg.dim[1], i1 = b - i2 * wg.dim[1];
            tail = wg.f[1][i1 * k + r] * wg.f[2][i2 * k + r];
          }
        }
        const double* fp = wg.f[0] + a * k + r;
        const int64_t fstep = (int64_t)(256 / KP) * k;
#pragma unroll
        for (int i = 0; i < WPT; ++i) {
          wr[i] = (r < k && a + (256 / KP) * i < g.A) ? *fp * tail : 0.0;
          fp += fstep;
        }
        return;
      }
      if constexpr (NF == 2 || NF == 3) {
        if (small_rows) {
          // 256 is a multiple of KP: entry i of this thread is row
          // kk = tid / KP + (256 / KP) i, rank r = tid % KP; its Khatri-Rao
          // digits advance by 256 / KP per entry (one division per tile)
          constexpr uint32_t RSTEP = 256 / KP;
          const int r = tid % KP;
          const int kk0 = tid / KP;
          const uint32_t d0 = fd0.d, d1 = fd1.d;
          uint32_t row = (uint32_t)(wrow0 + kk0);
          uint32_t i1 = fast_div(row, fd0), i0 = row - i1 * d0, i2 = 0;
          if (NF == 3) {
            const uint32_t q = i1;
            i2 = fast_div(q, fd1);
            i1 = q - i2 * d1;
          }
#pragma unroll
          for (int i = 0; i < WPT; ++i) {
            double v = 0.0;
            if (r < k && a0 + kk0 + (int64_t)RSTEP * i < g.A) {
              if (NF == 2)
                v = wg.f[0][(int64_t)i0 * k + r] * wg.f[1][(int64_t)i1 * k + r];
              else
                v = wg.f[0][(int64_t)i0 * k + r] *
                    (wg.f[1][(int64_t)i1 * k + r] * wg.f[2][(int64_t)i2 * k + r]);
            }
            wr[i] = v;
            i0 += RSTEP;
            while (i0 >= d0) {
              i0 -= d0;
              if (NF == 3 && ++i1 == d1) {
                i1 = 0;
                ++i2;
              } else if (NF == 2) {
                ++i1;
              }
            }
          }
          return;
        }
      }
#pragma unroll
      for (int i = 0; i < WPT; ++i) {
        int e = tid + 256 * i;
        double v = 0.0;
        if (e < BK * KP) {
          int kk = e / KP, r = e % KP;
          int64_t gaa = a0 + kk;
          if (r < k && gaa < g.A)
            v = small_rows ? wgen_at32<NF>(wg, fd0, fd1, (uint32_t)(wrow0 + kk), r, k)
                           : wgen_at<NF>(wg, wrow0 + kk, r, k);
        }
        wr[i] = v;
      }
    }
  };
  auto store_tile = [&](int stage) {
    double* Xs = ct_smem + stage * STAGE;
    double* Ws = Xs + XS_ELEMS;
    if constexpr (!LEFT) {
      const int mm = tid & 127;
#pragma unroll
      for (int i = 0; i < XPT; ++i) Xs[((tid >> 7) + 2 * i) * SX + mm] = xr[i];
    } else {
      const int aa = tid % BK;
#pragma unroll
      for (int i = 0; i < XPT; ++i) Xs[(tid / BK + (256 / BK) * i) * SX + aa] = xr[i];
    }
#pragma unroll
    for (int i = 0; i < WPT; ++i) {
      int e = tid + 256 * i;
      if (e < BK * KP) Ws[(e / KP) * SW + (e % KP)] = wr[i];
    }
  };

  if (t_begin < t_end) {
    load_tile(t_begin);
    store_tile(0);
  }
  for (int64_t t = t_begin; t < t_end; ++t) {
    const int stage = (int)((t - t_begin) & 1);
    // stage `stage` is complete and every warp is done with the other one
    __syncthreads();
    if (t + 1 < t_end) load_tile(t + 1);
    if (warp_live) {
      const double* Xs = ct_smem + stage * STAGE;
      const double* Ws = Xs + XS_ELEMS;
#pragma unroll
      for (int s4 = 0; s4 < BK / 4; ++s4) {
        const int kk = s4 * 4 + ft;
        double af[MT], bf[NT];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          const int m = wm0 + i * 8 + fg;
          af[i] = LEFT ? Xs[m * SX + kk] : Xs[kk * SX + m];
        }
#pragma unroll
        for (int j = 0; j < NT; ++j) bf[j] = Ws[kk * SW + wn0 + j * 8 + fg];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[i][j], af[i], bf[j]);
      }
    }
    if (t + 1 < t_end) store_tile(stage ^ 1);
  }
  double* o = out + (int64_t)blockIdx.y * g.split_stride;
#pragma unroll
  for (int i = 0; i < MT; ++i) {
    const int64_t gm = m0 + wm0 + i * 8 + fg;
    if (gm >= g.M) continue;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int r = wn0 + j * 8 + 2 * ft;
      if (r < k) o[gm * k + r] = acc[i][j][0];
      if (r + 1 < k) o[gm * k + r + 1] = acc[i][j][1];
    }
  }
}

// out[i] = sum_{s < nsplit} part[s * stride + i] in a fixed order: eight
// lanes per output each sum the splits s = lane8, lane8 + 8, ... and a fixed
// shuffle tree adds the eight (deterministic run to run; eight times the
// loads in flight of a thread-per-output loop).
__device__ __forceinline__ void reduce_splits_body(const double* __restrict__ part, int nsplit,
                                                   int64_t stride, int64_t n,
                                                   double* __restrict__ out, int64_t bx, int64_t gx) {
  const int sub = threadIdx.x & 7;
  const int64_t step = (gx * blockDim.x) >> 3;
  // every lane of a warp runs the same number of iterations (shuffles below)
  const int64_t base = ((bx * blockDim.x + threadIdx.x) >> 5) << 2;
  for (int64_t i0 = base; i0 < n; i0 += step) {
    const int64_t i = i0 + ((threadIdx.x >> 3) & 3);
    double s = 0.0;
    if (i < n) {
      int p = sub;
      for (; p + 24 < nsplit; p += 32) {
        const double v0 = part[p * stride + i], v1 = part[(p + 8) * stride + i];
        const double v2 = part[(p + 16) * stride + i], v3 = part[(p + 24) * stride + i];
        s += v0;
        s += v1;
        s += v2;
        s += v3;
      }
      for (; p < nsplit; p += 8) s += part[p * stride + i];
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    if (sub == 0 && i < n) out[i] = s;
  }
}
__global__ void k_reduce_splits(const double* __restrict__ part, int nsplit, int64_t stride,
                                int64_t n, double* __restrict__ out) {
  reduce_splits_body(part, nsplit, stride, n, out, blockIdx.x, gridDim.x);
}

// Grid of k_reduce_splits for n outputs (256-thread blocks, 8 lanes each).
inline unsigned reduce_grid(int64_t n) {
  const int64_t b = (8 * n + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 8192 ? 8192 : b));
}

// k_reduce_splits for nsplit <= 8: a thread per output, coalesced across the
// warp, adding the partials with the same pairwise tree the eight lanes of
// k_reduce_splits form ((p0 + p1) + (p2 + p3)) + ((p4 + p5) + (p6 + p7)),
// absent partials reading as 0, so both kernels give the same bits.
__device__ __forceinline__ void reduce_splits_few_body(const double* __restrict__ part, int nsplit,
                                                       int64_t stride, int64_t n,
                                                       double* __restrict__ out, int64_t bx,
                                                       int64_t gx) {
  for (int64_t i = bx * 256 + threadIdx.x; i < n; i += gx * 256) {
    double v[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = p < nsplit ? part[p * stride + i] : 0.0;
    out[i] = ((v[0] + v[1]) + (v[2] + v[3])) + ((v[4] + v[5]) + (v[6] + v[7]));
  }
}
__global__ void __launch_bounds__(256) k_reduce_splits_few(const double* __restrict__ part,
                                                           int nsplit, int64_t stride, int64_t n,
                                                           double* __restrict__ out) {
  reduce_splits_few_body(part, nsplit, stride, n, out, blockIdx.x, gridDim.x);
}

// Grid of the split-K sum for n outputs of nsplit partials (the launch
// reduce_splits makes): 0 selects k_reduce_splits_few, 1 k_reduce_splits.
inline int reduce_kind(int nsplit) { return nsplit <= 8 ? 0 : 1; }
inline unsigned reduce_blocks(int nsplit, int64_t n) {
  if (nsplit <= 8) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 1 ? 1 : (b > 4096 ? 4096 : b));
  }
  return reduce_grid(n);
}

// out[i] = sum over the nsplit partials part[p * stride + i], i < n.
inline void reduce_splits(cudaStream_t st, const double* part, int nsplit, int64_t stride,
                          int64_t n, double* out) {
  if (nsplit <= 8) {
    const int64_t b = (n + 255) / 256;
    k_reduce_splits_few<<<(unsigned)(b < 1 ? 1 : (b > 4096 ? 4096 : b)), 256, 0, st>>>(
        part, nsplit, stride, n, out);
  } else {
    k_reduce_splits<<<reduce_grid(n), 256, 0, st>>>(part, nsplit, stride, n, out);
  }
}

// ---------------------------------------------------------------------------
// Multi-TTV on a row-major (A*B) x k intermediate T (rank index fastest),
// dimtree/dimtrees.hpp:315-410:
//   left : out[b, r] = sum_a T[(a + A*b)*k + r] * F[a*k + r]
//   right: out[a, r] = sum_b T[(a + A*b)*k + r] * W(b, r)
// ---------------------------------------------------------------------------
// (kernel bodies take the CTA's index and the grid size as arguments, so that
// the grouped launches of a batch run every member through the same code)
template <typename TT>
__device__ __forceinline__ void ttv_left_body(const TT* __restrict__ T, int64_t A, int64_t B, int k,
                                              const double* __restrict__ F, double* __restrict__ out,
                                              int64_t bx, int64_t gx) {
  __shared__ double red[256];
  const int lanes = 256 / k;
  const int tid = threadIdx.x;
  const int r = tid % k, lane = tid / k;
  for (int64_t b = bx; b < B; b += gx) {
    double s = 0.0;
    if (lane < lanes) {
      const TT* Tb = T + (A * b) * k + r;
      const double* Fr = F + r;
      double s1 = 0.0, s2 = 0.0, s3 = 0.0;
      const int64_t step = (int64_t)lanes * k;
      int64_t a = lane;
      for (; a + 3 * lanes < A; a += 4 * lanes) {
        const int64_t o = a * k;
        s = fma((double)Tb[o], Fr[o], s);
        s1 = fma((double)Tb[o + step], Fr[o + step], s1);
        s2 = fma((double)Tb[o + 2 * step], Fr[o + 2 * step], s2);
        s3 = fma((double)Tb[o + 3 * step], Fr[o + 3 * step], s3);
      }
      for (; a < A; a += lanes) s = fma((double)Tb[a * k], Fr[a * k], s);
      s = (s + s1) + (s2 + s3);
    }
    red[tid] = s;
    __syncthreads();
    if (tid < k) {
      double t = 0.0;
      for (int l = 0; l < lanes; ++l) t += red[l * k + tid];
      out[b * k + tid] = t;
    }
    __syncthreads();
  }
}
template <typename TT>
__global__ void __launch_bounds__(256) k_ttv_left(const TT* __restrict__ T, int64_t A, int64_t B,
                                                  int k, const double* __restrict__ F,
                                                  double* __restrict__ out) {
  ttv_left_body<TT>(T, A, B, k, F, out, blockIdx.x, gridDim.x);
}

// k_ttv_left for an FP32 T with k a multiple of 4: a CTA takes TTVL_NB
// consecutive b at once, so each F row it loads serves TTVL_NB rows of T. A
// thread owns 4 ranks (one float4 of T and two double2 of F per row a) and
// the rows a = l, l + RL, ... of its row lane l, four rows' loads in flight;
// the CTA adds its RL row lanes in order through shared memory. Four CTAs
// an SM (64 registers a thread): the loop is bound by loads in flight.
constexpr int TTVL_NB = 2;
__device__ __forceinline__ void ttv_left_f4_body(const float* __restrict__ T, int64_t A, int64_t B,
                                                 int k, const double* __restrict__ F,
                                                 double* __restrict__ out, int64_t bx) {
  __shared__ double red[256 * TTVL_NB * 4];
  const int q = k >> 2;                  // float4 per row
  const int tpr = q <= 8 ? 8 : 16;       // threads per row
  const int RL = 256 / tpr;              // row lanes
  const int tid = threadIdx.x;
  const int r4 = tid % tpr, rl = tid / tpr;
  const bool active = r4 < q;
  const int64_t b0 = bx * TTVL_NB;
  const int nb = (int)((B - b0) < TTVL_NB ? (B - b0) : TTVL_NB);
  double acc[TTVL_NB][4];
#pragma unroll
  for (int j = 0; j < TTVL_NB; ++j)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[j][c] = 0.0;
  if (active) {
    // rows a, a + RL, a + 2 RL: every load of the three rows is issued
    // before the first product (then one row at a time for the rest; three
    // rows' values fill the 64 registers of four CTAs an SM)
    constexpr int U = 3;
    int64_t a = rl;
    for (; a + (U - 1) * RL < A; a += U * RL) {
      double2 f01[U], f23[U];
      float4 t[U][TTVL_NB];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t au = a + u * RL;
        f01[u] = *reinterpret_cast<const double2*>(F + au * k + 4 * r4);
        f23[u] = *reinterpret_cast<const double2*>(F + au * k + 4 * r4 + 2);
#pragma unroll
        for (int j = 0; j < TTVL_NB; ++j)
          t[u][j] = j < nb ? *reinterpret_cast<const float4*>(T + (au + A * (b0 + j)) * k + 4 * r4)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
#pragma unroll
        for (int j = 0; j < TTVL_NB; ++j) {
          acc[j][0] = fma((double)t[u][j].x, f01[u].x, acc[j][0]);
          acc[j][1] = fma((double)t[u][j].y, f01[u].y, acc[j][1]);
          acc[j][2] = fma((double)t[u][j].z, f23[u].x, acc[j][2]);
          acc[j][3] = fma((double)t[u][j].w, f23[u].y, acc[j][3]);
        }
    }
    for (; a < A; a += RL) {
      const double2 f01 = *reinterpret_cast<const double2*>(F + a * k + 4 * r4);
      const double2 f23 = *reinterpret_cast<const double2*>(F + a * k + 4 * r4 + 2);
      float4 t[TTVL_NB];
#pragma unroll
      for (int j = 0; j < TTVL_NB; ++j)
        t[j] = j < nb ? *reinterpret_cast<const float4*>(T + (a + A * (b0 + j)) * k + 4 * r4)
                      : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int j = 0; j < TTVL_NB; ++j) {
        acc[j][0] = fma((double)t[j].x, f01.x, acc[j][0]);
        acc[j][1] = fma((double)t[j].y, f01.y, acc[j][1]);
        acc[j][2] = fma((double)t[j].z, f23.x, acc[j][2]);
        acc[j][3] = fma((double)t[j].w, f23.y, acc[j][3]);
      }
    }
  }
  // red[l][j * k + r]
  if (active)
#pragma unroll
    for (int j = 0; j < TTVL_NB; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) red[rl * (TTVL_NB * k) + j * k + 4 * r4 + c] = acc[j][c];
  __syncthreads();
  for (int e = tid; e < nb * k; e += 256) {
    double t = 0.0;
    for (int l = 0; l < RL; ++l) t += red[l * (TTVL_NB * k) + e];
    out[b0 * k + e] = t;
  }
}
__global__ void __launch_bounds__(256, 4) k_ttv_left_f4(const float* __restrict__ T, int64_t A,
                                                        int64_t B, int k,
                                                        const double* __restrict__ F,
                                                        double* __restrict__ out) {
  ttv_left_f4_body(T, A, B, k, F, out, blockIdx.x);
}

template <typename TT>
__global__ void __launch_bounds__(256) k_ttv_right(const TT* __restrict__ T, int64_t A, int64_t B,
                                                   int k, WGen wg, int64_t b_per_split,
                                                   int64_t split_stride,
                                                   double* __restrict__ out) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= A * k) return;
  const int64_t a = e / k;
  const int r = (int)(e % k);
  int64_t b0 = (int64_t)blockIdx.y * b_per_split;
  int64_t b1 = b0 + b_per_split;
  if (b1 > B) b1 = B;
  if (b0 >= b1) {
    out[(int64_t)blockIdx.y * split_stride + e] = 0.0;
    return;
  }
  double s = 0.0;
  const TT* Tp = T + (a + A * b0) * k + r;
  const int64_t tstride = A * k;
  if (wg.nf == 1) {
    const double* W = wg.f[0] + r;
    double s1 = 0.0;
    int64_t b = b0;
    for (; b + 1 < b1; b += 2) {
      s = fma((double)Tp[0], W[b * k], s);
      s1 = fma((double)Tp[tstride], W[(b + 1) * k], s1);
      Tp += 2 * tstride;
    }
    if (b < b1) s = fma((double)Tp[0], W[b * k], s);
    s += s1;
  } else {
    WIdx wi;
    widx_init(wg, b0, wi);
    for (int64_t b = b0; b < b1; ++b) {
      s = fma((double)Tp[0], wgen_row(wg, wi, r, k), s);
      Tp += tstride;
      widx_advance(wg, wi, 1);
    }
  }
  out[(int64_t)blockIdx.y * split_stride + e] = s;
}

// Tiled right multi-TTV: a CTA owns AT = 4096/KP consecutive a values (all
// ranks) and a range of b; per b it reads the AT*k contiguous entries of
// T[(a0..a0+AT-1) + A*b, :] (coalesced), each thread owning rank r = tid % KP
// and 16 rows. W(b, r) comes from the row digits of b, advanced per step.
// Writes one partial (A x k) per b-range; k_reduce_splits sums them.
template <typename TT, int KP>
__device__ __forceinline__ void ttv_right_tiled_body(const TT* __restrict__ T, int64_t A, int64_t B,
                                                     int k, const WGen& wg, int64_t b_per_split,
                                                     double* __restrict__ out, int64_t bx,
                                                     int64_t by) {
  constexpr int J = 16;
  constexpr int AT = J * 256 / KP;
  constexpr int BC = 32;  // b values per shared-memory W chunk
  __shared__ double Ws[BC][KP];
  const int tid = threadIdx.x;
  const int r = tid % KP;
  const int arow = tid / KP;  // 0 .. 256/KP - 1
  const int64_t a0 = bx * AT;
  const int64_t b0 = by * b_per_split;
  int64_t b1 = b0 + b_per_split;
  if (b1 > B) b1 = B;
  double acc[J];
#pragma unroll
  for (int j = 0; j < J; ++j) acc[j] = 0.0;
  const bool rok = r < k;
  for (int64_t bc = b0; bc < b1; bc += BC) {
    const int nb = (int)((b1 - bc) < BC ? (b1 - bc) : BC);
    __syncthreads();
    // W(b, r) for this chunk: thread tid < nb*KP computes one entry
    for (int e = tid; e < nb * KP; e += 256) {
      const int bb = e / KP, rr = e % KP;
      Ws[bb][rr] = rr < k ? wgen_eval(wg, bc + bb, rr, k) : 0.0;
    }
    __syncthreads();
    if (rok) {
      const TT* Tb = T + (A * bc) * k + r;
      const int64_t tstride = A * k;
      int bb = 0;
      for (; bb + 1 < nb; bb += 2) {
        const double w0 = Ws[bb][r], w1 = Ws[bb + 1][r];
        const TT* T0 = Tb + bb * tstride;
        const TT* T1 = T0 + tstride;
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const int64_t a = a0 + arow + (int64_t)(256 / KP) * j;
          if (a < A) {
            const double x0 = (double)T0[a * k], x1 = (double)T1[a * k];
            acc[j] = fma(x1, w1, fma(x0, w0, acc[j]));
          }
        }
      }
      if (bb < nb) {
        const double w0 = Ws[bb][r];
        const TT* T0 = Tb + bb * tstride;
#pragma unroll
        for (int j = 0; j < J; ++j) {
          const int64_t a = a0 + arow + (int64_t)(256 / KP) * j;
          if (a < A) acc[j] = fma((double)T0[a * k], w0, acc[j]);
        }
      }
    }
  }
  if (!rok) return;
  double* o = out + by * A * k;
#pragma unroll
  for (int j = 0; j < J; ++j) {
    const int64_t a = a0 + arow + (int64_t)(256 / KP) * j;
    if (a < A) o[a * k + r] = acc[j];
  }
}
template <typename TT, int KP>
__global__ void __launch_bounds__(256) k_ttv_right_tiled(const TT* __restrict__ T, int64_t A,
                                                         int64_t B, int k, WGen wg,
                                                         int64_t b_per_split,
                                                         double* __restrict__ out) {
  ttv_right_tiled_body<TT, KP>(T, A, B, k, wg, b_per_split, out, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Factor updates, one thread per factor row (each row's recurrence reads only
// that row of H and M, and G).
// ---------------------------------------------------------------------------
// HALS, ntf/ntfhals.hpp:13-29 + common/utils.hpp:59-64:
//   for i < k: u = h_i + (m_i - sum_j h_j G[j,i]);  h_i = (u < 1e-17) ? 1e-17 : u
// Column i of H is replaced in place before column i+1 is computed; the
// reference's ||u||^2 > 0 guard always holds once every entry is >= 1e-17.
template <int KP>
__global__ void __launch_bounds__(128) k_hals_rows(double* __restrict__ H, const double* __restrict__ M,
                                                   const double* __restrict__ G, int64_t I, int k) {
  __shared__ double Gs[KP * KP];
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) Gs[e] = G[e];
  __syncthreads();
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= I) return;
  double h[KP], m[KP];
#pragma unroll
  for (int j = 0; j < KP; ++j) {
    h[j] = j < k ? H[row * k + j] : 0.0;
    m[j] = j < k ? M[row * k + j] : 0.0;
  }
#pragma unroll
  for (int i = 0; i < KP; ++i) {
    if (i < k) {
      double p0 = 0.0, p1 = 0.0, p2 = 0.0, p3 = 0.0;
#pragma unroll
      for (int j = 0; j < KP; j += 4) {
        if (j < k) p0 = fma(h[j], Gs[j * k + i], p0);
        if (j + 1 < k) p1 = fma(h[j + 1], Gs[(j + 1) * k + i], p1);
        if (j + 2 < k) p2 = fma(h[j + 2], Gs[(j + 2) * k + i], p2);
        if (j + 3 < k) p3 = fma(h[j + 3], Gs[(j + 3) * k + i], p3);
      }
      double hg = (p0 + p1) + (p2 + p3);
      double u = h[i] + (m[i] - hg);
      h[i] = (u < kEps17) ? kEps17 : u;
    }
  }
#pragma unroll
  for (int j = 0; j < KP; ++j)
    if (j < k) H[row * k + j] = h[j];
}

// MU, ntf/ntfmu.hpp:11-16: H = (H % M^T) / (H*G + 1e-6), H*G from the old H.
template <int KP>
__global__ void __launch_bounds__(128) k_mu_rows(double* __restrict__ H, const double* __restrict__ M,
                                                 const double* __restrict__ G, int64_t I, int k) {
  __shared__ double Gs[KP * KP];
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) Gs[e] = G[e];
  __syncthreads();
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= I) return;
  double h[KP], t[KP];
#pragma unroll
  for (int j = 0; j < KP; ++j) h[j] = j < k ? H[row * k + j] : 0.0;
#pragma unroll
  for (int c = 0; c < KP; ++c) {
    double p0 = 0.0, p1 = 0.0;
#pragma unroll
    for (int j = 0; j < KP; j += 2) {
      if (j < k && c < k) p0 = fma(h[j], Gs[j * k + c], p0);
      if (j + 1 < k && c < k) p1 = fma(h[j + 1], Gs[(j + 1) * k + c], p1);
    }
    t[c] = (p0 + p1) + kEps6;
  }
#pragma unroll
  for (int c = 0; c < KP; ++c)
    if (c < k) H[row * k + c] = (h[c] * M[row * k + c]) / t[c];
}

// Warp-per-row forms of the same updates (lane c owns columns c and c + 32).
// HALS keeps g = H(row,:) * G up to date incrementally: after column i moves
// by delta, g += delta * G(i,:), so g(i) always equals the reference's
// H(row,:) * G(:,i) with columns < i already replaced (ntf/ntfhals.hpp:17-18).
// k x k matrix G into shared memory, four loads in flight per thread, then a
// CTA barrier
__device__ __forceinline__ void stage_gram(const double* __restrict__ G, int k, double* Gs) {
  const int kk = k * k;
  for (int e0 = threadIdx.x; e0 < kk; e0 += 4 * blockDim.x) {
    double g[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      g[u] = e < kk ? G[e] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = e0 + u * blockDim.x;
      if (e < kk) Gs[e] = g[u];
    }
  }
  __syncthreads();
}

template <int KP>
__device__ __forceinline__ void hals_warp_body(double* __restrict__ H, const double* __restrict__ M,
                                               const double* __restrict__ G, int64_t I, int k,
                                               int64_t bx) {
  constexpr int PER = KP / 32;
  __shared__ double Gs[KP * KP];
  stage_gram(G, k, Gs);
  const int lane = threadIdx.x & 31;
  const int64_t row = bx * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= I) return;
  double h[PER], m[PER], g[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    h[p] = c < k ? H[row * k + c] : 0.0;
    m[p] = c < k ? M[row * k + c] : 0.0;
    g[p] = 0.0;
  }
  for (int j = 0; j < k; ++j) {
    const double hj = (PER == 1 || j < 32) ? __shfl_sync(0xffffffffu, h[0], j & 31)
                                           : __shfl_sync(0xffffffffu, h[PER - 1], j & 31);
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      if (c < k) g[p] = fma(hj, Gs[j * k + c], g[p]);
    }
  }
  for (int i = 0; i < k; ++i) {
    const int owner = i & 31, pi = i >> 5;
    double delta = 0.0;
    if (lane == owner) {
#pragma unroll
      for (int p = 0; p < PER; ++p)
        if (p == pi) {
          double u = h[p] + (m[p] - g[p]);
          u = (u < kEps17) ? kEps17 : u;
          delta = u - h[p];
          h[p] = u;
        }
    }
    delta = __shfl_sync(0xffffffffu, delta, owner);
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      if (c < k) g[p] = fma(delta, Gs[i * k + c], g[p]);
    }
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    if (c < k) H[row * k + c] = h[p];
  }
}
template <int KP>
__global__ void __launch_bounds__(256) k_hals_warp(double* __restrict__ H, const double* __restrict__ M,
                                                   const double* __restrict__ G, int64_t I, int k) {
  hals_warp_body<KP>(H, M, G, I, k, blockIdx.x);
}

// MU: H = (H .* M) ./ (H G + eps); eps is 1e-6 for NTF (ntf/ntfmu.hpp:14) and
// 1e-17 for NMF (nmf/mu.hpp:68, 80).
template <int KP>
__device__ __forceinline__ void mu_warp_body(double* __restrict__ H, const double* __restrict__ M,
                                             const double* __restrict__ G, int64_t I, int k,
                                             double eps, int64_t bx) {
  constexpr int PER = KP / 32;
  __shared__ double Gs[KP * KP];
  stage_gram(G, k, Gs);
  const int lane = threadIdx.x & 31;
  const int64_t row = bx * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (row >= I) return;
  double h[PER], t[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    h[p] = c < k ? H[row * k + c] : 0.0;
    t[p] = 0.0;
  }
  for (int j = 0; j < k; ++j) {
    const double hj = (PER == 1 || j < 32) ? __shfl_sync(0xffffffffu, h[0], j & 31)
                                           : __shfl_sync(0xffffffffu, h[PER - 1], j & 31);
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int c = lane + 32 * p;
      if (c < k) t[p] = fma(hj, Gs[j * k + c], t[p]);
    }
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int c = lane + 32 * p;
    if (c < k) H[row * k + c] = (h[p] * M[row * k + c]) / (t[p] + eps);
  }
}
template <int KP>
__global__ void __launch_bounds__(256) k_mu_warp(double* __restrict__ H, const double* __restrict__ M,
                                                 const double* __restrict__ G, int64_t I, int k,
                                                 double eps) {
  mu_warp_body<KP>(H, M, G, I, k, eps, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Normalisation + Gram over many CTAs: each CTA adds U^T U of a block of rows
// of the new (unnormalised) factor U; k_gram_finalize sums the blocks in a
// fixed order, takes lambda_r = sqrt((U^T U)_rr) = ||U(:,r)||, writes the Gram
// of the normalised factor G_n = (U^T U)_ab / (lambda_a lambda_b), normalises
// U in place (ncpfactors.hpp:346-351) and forms the next leave-one-out product.
// ---------------------------------------------------------------------------
constexpr int GP_ROWS = 16;      // fewest rows per block (partial buffers are sized for it)
constexpr int GP_ROWS_MAX = 64;  // most rows per block (shared-memory tile)

// Rows per block: about 32 blocks per factor (more blocks than that only
// lengthen k_gram_finalize's fixed-order sum), between GP_ROWS and GP_ROWS_MAX.
inline int gram_rows_per_block(int64_t I) {
  int64_t r = (I + 31) / 32;
  r = (r + GP_ROWS - 1) / GP_ROWS * GP_ROWS;
  return (int)(r < GP_ROWS ? GP_ROWS : (r > GP_ROWS_MAX ? GP_ROWS_MAX : r));
}

// 256 threads; thread (ta, tb) owns the 4 x 4 outputs a = ta + kt*u,
// b = tb + kt*v (kt = ceil(k/4)), so a warp's loads of the b-values are
// consecutive in shared memory.
__global__ void __launch_bounds__(256) k_gram_partial(const double* __restrict__ U, int64_t I, int k,
                                                      int rows_per_block, double* __restrict__ part) {
  __shared__ double tile[GP_ROWS_MAX * kMaxRank];
  const int64_t row0 = (int64_t)blockIdx.x * rows_per_block;
  const int nrows = (int)((I - row0) < rows_per_block ? (I - row0) : rows_per_block);
  for (int e = threadIdx.x; e < nrows * k; e += 256) tile[e] = U[row0 * k + e];
  __syncthreads();
  const int kt = (k + 3) / 4;
  const int t = threadIdx.x;
  if (t >= kt * kt) return;
  const int ta = t / kt, tb = t % kt;
  double acc[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
  for (int i = 0; i < nrows; ++i) {
    const double* r = tile + i * k;
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int a = ta + kt * u, b = tb + kt * u;
      av[u] = a < k ? r[a] : 0.0;
      bv[u] = b < k ? r[b] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
  }
  double* dst = part + (int64_t)blockIdx.x * k * k;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int a = ta + kt * u, b = tb + kt * v;
      if (a < k && b < k) dst[a * k + b] = acc[u][v];
    }
}

// One CTA: sums the row-block partials in a fixed order (eight independent
// running sums per element), lambda_r = sqrt((U^T U)_rr), G_n = (U^T U)_ab /
// (lambda_a lambda_b) and the next leave-one-out product; k_scale_cols then
// normalises U.
__global__ void __launch_bounds__(1024) k_gram_finalize(double* __restrict__ F, int64_t I, int k,
                                                        const double* __restrict__ part, int nblk,
                                                        double* __restrict__ lambda,
                                                        double* __restrict__ Gall, int N, int n,
                                                        int next, double* __restrict__ Gloo) {
  __shared__ double lam[kMaxRank];
  __shared__ double gs[kMaxRank * kMaxRank];
  const int tid = threadIdx.x;
  const int kk2 = k * k;
  for (int e = tid; e < kk2; e += 1024) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int b = 0;
    for (; b + 8 <= nblk; b += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) s[u] += part[(int64_t)(b + u) * kk2 + e];
    }
    for (; b < nblk; ++b) s[0] += part[(int64_t)b * kk2 + e];
    gs[e] = ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
  }
  __syncthreads();
  if (tid < k) {
    const double nrm = sqrt(gs[tid * k + tid]);
    lam[tid] = nrm;
    if (lambda) lambda[tid] = nrm;
  }
  __syncthreads();
  double* Gn = Gall + (int64_t)n * kk2;
  for (int e = tid; e < kk2; e += 1024) {
    const int a = e / k, b = e % k;
    const double la = lam[a], lb = lam[b];
    Gn[e] = (la > 0 && lb > 0) ? gs[e] / (la * lb) : gs[e];
  }
  if (next < 0) return;
  __syncthreads();
  for (int e = tid; e < kk2; e += 1024) {
    double g = 1.0;
    for (int i = 0; i < N; ++i)
      if (i != next) g = g * Gall[(int64_t)i * kk2 + e];
    Gloo[e] = g;
  }
}

// F(:, r) /= lambda_r where lambda_r > 0 (ncpfactors.hpp:346-351), many CTAs.
__global__ void __launch_bounds__(256) k_scale_cols(double* __restrict__ F, int64_t I, int k,
                                                    const double* __restrict__ lambda) {
  const int64_t n = I * k;
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < n; e += (int64_t)gridDim.x * 256) {
    const double nrm = lambda[e % k];
    if (nrm > 0) F[e] = F[e] / nrm;
  }
}

// From an un-normalised Gram G_in = U^T U (summed over every row block of the
// factor, possibly on other devices): lambda_r = sqrt((U^T U)_rr) and the Gram
// of the normalised factor, G_out_ab = G_in_ab / (lambda_a lambda_b) (entries
// of a zero column kept), the same arithmetic as k_gram_finalize. One CTA.
__global__ void __launch_bounds__(1024) k_norm_from_gram(const double* __restrict__ Gin, int k,
                                                         double* __restrict__ lambda,
                                                         double* __restrict__ Gout) {
  __shared__ double lam[kMaxRank];
  const int tid = threadIdx.x;
  if (tid < k) {
    const double nrm = sqrt(Gin[tid * k + tid]);
    lam[tid] = nrm;
    lambda[tid] = nrm;
  }
  __syncthreads();
  for (int e = tid; e < k * k; e += 1024) {
    const double la = lam[e / k], lb = lam[e % k];
    Gout[e] = (la > 0 && lb > 0) ? Gin[e] / (la * lb) : Gin[e];
  }
}

// out_r = sum_i A[i, r] B[i, r] over row-major I x k blocks, in a fixed order
// (two running sums per lane, then a tree over the lanes). One CTA.
__global__ void __launch_bounds__(1024) k_coldot(const double* __restrict__ A,
                                                 const double* __restrict__ B, int64_t I, int k,
                                                 double* __restrict__ out) {
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  const int r = tid % k, lane = tid / k, lanes = 1024 / k;
  double v = 0.0;
  if (lane < lanes) {
    double s0 = 0.0, s1 = 0.0;
    int64_t i = lane;
    for (; i + lanes < I; i += 2 * lanes) {
      s0 = fma(A[i * k + r], B[i * k + r], s0);
      s1 = fma(A[(i + lanes) * k + r], B[(i + lanes) * k + r], s1);
    }
    if (i < I) s0 = fma(A[i * k + r], B[i * k + r], s0);
    v = s0 + s1;
  }
  red[tid] = v;
  __syncthreads();
  if (tid < k) {
    double s = 0.0;
    for (int l = 0; l < lanes; ++l) s += red[l * k + tid];
    out[tid] = s;
  }
}

// ---------------------------------------------------------------------------
// Normalise mode n (NCPFactors::normalize(int), common/ncpfactors.hpp:346-351:
// lambda_r = ||F(:,r)||, F(:,r) /= lambda_r when > 0), then G_n = F^T F of the
// normalised factor (ncpfactors.hpp:144) and, if next >= 0, the leave-one-out
// Hadamard product for mode `next` (ncpfactors.hpp:139-148, modes in
// increasing order starting from ones). One CTA of 1024 threads.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_normalize_gram(double* __restrict__ F, int64_t I, int k,
                                                         double* __restrict__ lambda,
                                                         double* __restrict__ Gall, int N, int n,
                                                         int next, double* __restrict__ Gloo) {
  constexpr int ROWS = 64;
  __shared__ double red[1024];
  __shared__ double lam[kMaxRank];
  __shared__ double tile[ROWS * kMaxRank];
  const int tid = threadIdx.x;
  const int lanes = 1024 / k;
  const int r = tid % k, lane = tid / k;
  double ss = 0.0;
  if (lane < lanes)
    for (int64_t i = lane; i < I; i += lanes) {
      double v = F[i * k + r];
      ss = fma(v, v, ss);
    }
  red[tid] = ss;
  __syncthreads();
  if (tid < k) {
    double t = 0.0;
    for (int l = 0; l < lanes; ++l) t += red[l * k + tid];
    double nrm = sqrt(t);
    lam[tid] = nrm;
    if (lambda) lambda[tid] = nrm;
  }
  __syncthreads();
  // normalise row blocks in place and accumulate F^T F from shared memory;
  // thread tid owns Gram entries e = tid + 1024*q (q < 4 since k <= 64)
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const int kk2 = k * k;
  for (int64_t row0 = 0; row0 < I; row0 += ROWS) {
    const int nrows = (int)((I - row0) < ROWS ? (I - row0) : ROWS);
    for (int e = tid; e < nrows * k; e += 1024) {
      int64_t g = row0 * k + e;
      double nrm = lam[e % k];
      double v = F[g];
      if (nrm > 0) {
        v = v / nrm;
        F[g] = v;
      }
      tile[e] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + 1024 * q;
      if (e < kk2) {
        int a = e / k, b = e % k;
        double s = acc[q];
        for (int i = 0; i < nrows; ++i) s = fma(tile[i * k + a], tile[i * k + b], s);
        acc[q] = s;
      }
    }
    __syncthreads();
  }
  double* Gn = Gall + (int64_t)n * kk2;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int e = tid + 1024 * q;
    if (e < kk2) Gn[e] = acc[q];
  }
  if (next < 0) return;
  __syncthreads();
  for (int e = tid; e < kk2; e += 1024) {
    double g = 1.0;
    for (int i = 0; i < N; ++i)
      if (i != next) g = g * Gall[(int64_t)i * kk2 + e];
    Gloo[e] = g;
  }
}

// Leave-one-out Hadamard product from cached Grams.
__global__ void k_gram_loo(const double* __restrict__ Gall, int N, int k, int n,
                           double* __restrict__ Gloo) {
  for (int e = threadIdx.x; e < k * k; e += blockDim.x) {
    double g = 1.0;
    for (int i = 0; i < N; ++i)
      if (i != n) g = g * Gall[(int64_t)i * k * k + e];
    Gloo[e] = g;
  }
}

// ---------------------------------------------------------------------------
// Relative error in FP64 Gram form (the form of distntf/distauntf.hpp:685-727;
// value of AUNTF::computeObjectiveError, ntf/auntf.hpp:200-246):
//   ||X - [[lambda; F]]||^2 = ||X||^2 - 2 sum_r lambda_r <M_last(:,r), F_last(:,r)>
//                             + lambda^T (*_i G_i) lambda
// M_last is the MTTKRP of the last mode, computed from the final F_0..F_{N-2}.
// Writes errs[*counter] and increments *counter (so one captured graph can be
// replayed across iterations). One CTA of 256 threads.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void error_body(const double* __restrict__ Mlast,
                                           const double* __restrict__ Flast, int64_t I,
                                           const double* __restrict__ lambda,
                                           const double* __restrict__ Gall, int N, int k,
                                           const double* __restrict__ normX2,
                                           double* __restrict__ errs, int* __restrict__ counter) {
  __shared__ double red[1024];
  __shared__ double red2[1024];
  const int tid = threadIdx.x;
  const int r = tid % k, lane = tid / k, lanes = 1024 / k;
  double inner = 0.0;
  if (lane < lanes) {
    double s0 = 0.0, s1 = 0.0;
    int64_t i = lane;
    for (; i + lanes < I; i += 2 * lanes) {
      s0 = fma(Mlast[i * k + r], Flast[i * k + r], s0);
      s1 = fma(Mlast[(i + lanes) * k + r], Flast[(i + lanes) * k + r], s1);
    }
    if (i < I) s0 = fma(Mlast[i * k + r], Flast[i * k + r], s0);
    inner = (s0 + s1) * lambda[r];
  }
  double mn = 0.0;
  for (int e = tid; e < k * k; e += 1024) {
    double g = 1.0;
    for (int i = 0; i < N; ++i) g = g * Gall[(int64_t)i * k * k + e];
    mn = fma(lambda[e / k] * lambda[e % k], g, mn);
  }
  red[tid] = inner;
  red2[tid] = mn;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if (tid < s) {
      red[tid] += red[tid + s];
      red2[tid] += red2[tid + s];
    }
    __syncthreads();
  }
  if (tid == 0) {
    double nx = *normX2;
    double e2 = nx - 2.0 * red[0] + red2[0];
    double err = sqrt(fabs(e2) / nx);
    int c = *counter;
    errs[c] = err;
    *counter = c + 1;
  }
}
__global__ void __launch_bounds__(1024) k_error(const double* __restrict__ Mlast,
                                                const double* __restrict__ Flast, int64_t I,
                                                const double* __restrict__ lambda,
                                                const double* __restrict__ Gall, int N, int k,
                                                const double* __restrict__ normX2,
                                                double* __restrict__ errs, int* __restrict__ counter) {
  error_body(Mlast, Flast, I, lambda, Gall, N, k, normX2, errs, counter);
}

// Sum of squares in FP64 (Tensor::norm, common/tensor.hpp:350-356), per-block
// partials; k_reduce_splits with nsplit = blocks finishes it.
template <typename T>
__global__ void __launch_bounds__(256) k_sumsq_partial(const T* __restrict__ X, int64_t n,
                                                       double* __restrict__ part) {
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
    double v = (double)X[i];
    s = fma(v, v, s);
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if (threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// ---------------------------------------------------------------------------
// Differentiable CP loss, 1/2 ||X - [[F_0..F_{N-1}]]||^2, in three fused
// launches around the MTTKRPs (the gradient form of ntf/ntfnes.hpp:138-147).
// ---------------------------------------------------------------------------
constexpr int CPG_BLOCKS = 8;  // row blocks per factor of the Gram kernel

struct CpFactors {
  const double* F[kMaxModes];
  int64_t I[kMaxModes];
  int N, k;
};

// Grams G_n = F_n^T F_n of every factor: block (b, n) sums its share of the
// rows of F_n into part[n][b]; the last block of factor n to finish (counter
// ctr[n], left at 0 again) adds the CPG_BLOCKS partials in order into G_n.
__global__ void __launch_bounds__(256) k_cp_grams(CpFactors f, double* __restrict__ part,
                                                  double* __restrict__ G, unsigned* __restrict__ ctr) {
  __shared__ bool last;
  const int n = blockIdx.y, b = blockIdx.x, k = f.k, kk2 = k * k;
  const int64_t I = f.I[n];
  const int64_t per = (I + CPG_BLOCKS - 1) / CPG_BLOCKS;
  const int64_t r0 = b * per, r1 = (r0 + per) < I ? (r0 + per) : I;
  const double* F = f.F[n];
  double* dst = part + ((int64_t)n * CPG_BLOCKS + b) * kk2;
  for (int e = threadIdx.x; e < kk2; e += 256) {
    const int a = e / k, c = e % k;
    double s0 = 0.0, s1 = 0.0;
    int64_t i = r0;
    for (; i + 1 < r1; i += 2) {
      s0 = fma(F[i * k + a], F[i * k + c], s0);
      s1 = fma(F[(i + 1) * k + a], F[(i + 1) * k + c], s1);
    }
    if (i < r1) s0 = fma(F[i * k + a], F[i * k + c], s0);
    dst[e] = s0 + s1;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ctr + n, 1u) == CPG_BLOCKS - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* src = part + (int64_t)n * CPG_BLOCKS * kk2;
  for (int e = threadIdx.x; e < kk2; e += 256) {
    double t = 0.0;
    for (int q = 0; q < CPG_BLOCKS; ++q) t += __ldcg(src + (int64_t)q * kk2 + e);
    G[(int64_t)n * kk2 + e] = t;
  }
  if (threadIdx.x == 0) ctr[n] = 0;
}

// loss = 1/2 ||X||^2 - <M_0, F_0> + 1/2 sum_ab prod_n G_n[a, b]  (one CTA)
__global__ void __launch_bounds__(1024) k_cp_loss(const double* __restrict__ M0,
                                                  const double* __restrict__ F0, int64_t I0,
                                                  const double* __restrict__ G, int N, int k,
                                                  const double* __restrict__ normX2,
                                                  double* __restrict__ loss) {
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  double v = 0.0;
  for (int64_t e = tid; e < I0 * k; e += 1024) v = fma(M0[e], F0[e], v);
  double mm = 0.0;
  for (int e = tid; e < k * k; e += 1024) {
    double g = 1.0;
    for (int n = 0; n < N; ++n) g *= G[(int64_t)n * k * k + e];
    mm += g;
  }
  red[tid] = 0.5 * mm - v;
  __syncthreads();
  for (int st = 512; st > 0; st >>= 1) {
    if (tid < st) red[tid] += red[tid + st];
    __syncthreads();
  }
  if (tid == 0) *loss = 0.5 * (*normX2) + red[0];
}

// grad_n = g * (F_n H_n - M_n), H_n = prod_{m != n} G_m (Hadamard), for every
// mode: block (b, n) forms H_n in shared memory and does its rows.
struct CpGrad {
  const double* M[kMaxModes];
  double* grad[kMaxModes];
};
__global__ void __launch_bounds__(256) k_cp_grads(CpFactors f, const double* __restrict__ G,
                                                  CpGrad d, const double* __restrict__ gscale) {
  __shared__ double H[kMaxRank * kMaxRank];
  const int n = blockIdx.y, k = f.k, kk2 = k * k;
  for (int e = threadIdx.x; e < kk2; e += 256) {
    double h = 1.0;
    for (int m = 0; m < f.N; ++m)
      if (m != n) h *= G[(int64_t)m * kk2 + e];
    H[e] = h;
  }
  __syncthreads();
  const double g = *gscale;
  const int64_t I = f.I[n];
  const double* F = f.F[n];
  const double* Mn = d.M[n];
  double* out = d.grad[n];
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < I * k;
       e += (int64_t)gridDim.x * 256) {
    const int64_t i = e / k;
    const int r = (int)(e % k);
    double s = 0.0;
    for (int c = 0; c < k; ++c) s = fma(F[i * k + c], H[c * k + r], s);
    out[e] = g * (s - Mn[e]);
  }
}

// One projected accelerated gradient step on every factor:
//   F_new = max(Y - eta * grad, 0),  Y_new = F_new + mom * (F_new - F_prev)
struct CpStep {
  const double* Y[kMaxModes];
  const double* grad[kMaxModes];
  const double* Fprev[kMaxModes];
  double* Fnew[kMaxModes];
  double* Ynew[kMaxModes];
  int64_t n[kMaxModes];  // elements of each factor
  int N;
};
__global__ void __launch_bounds__(256) k_cp_step(CpStep s, double eta, double mom) {
  const int m = blockIdx.y;
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < s.n[m];
       e += (int64_t)gridDim.x * 256) {
    double v = s.Y[m][e] - eta * s.grad[m][e];
    v = v > 0.0 ? v : 0.0;
    const double fp = s.Fprev[m][e];
    s.Fnew[m][e] = v;
    s.Ynew[m][e] = v + mom * (v - fp);
  }
}

// Rows of a Khatri-Rao product, out[g, r] = W(g, r) of `wg` (the product
// order of wgen_eval), g < rows: the tail image of a long direct MTTKRP.
__global__ void __launch_bounds__(256) k_krp_rows(WGen wg, int64_t rows, int k,
                                                  double* __restrict__ out) {
  for (int64_t e = (int64_t)blockIdx.x * 256 + threadIdx.x; e < rows * k;
       e += (int64_t)gridDim.x * 256)
    out[e] = wgen_eval(wg, e / k, (int)(e % k), k);
}

// out[e] = v for e < n
__global__ void k_fill(double* __restrict__ out, int64_t n, double v) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x)
    out[e] = v;
}

// acc = (first ? 0 : acc) + the nb partials summed in a fixed order (one
// warp: lane l adds partials l, l + 32, ..., then a fixed shuffle tree).
__global__ void k_accum_norm(const double* __restrict__ part, int nb, double* __restrict__ acc,
                             int first) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += part[b];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) *acc = first ? s : *acc + s;
}

template <typename T>
__global__ void k_copy_to_f64(const T* __restrict__ in, int64_t n, double* __restrict__ out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// ---------------------------------------------------------------------------
// Synthetic CP tensor: X = [[A_0..A_{N-1}]] + sigma * N(0,1), optionally
// clipped at 0. Normals come from Philox-4x32-10 (Salmon et al., SC'11) keyed
// by `seed` and counted by the element index, through the Box-Muller
// transform, so the tensor is a pure function of (factors, sigma, seed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void philox4x32_10(uint32_t ctr[4], uint32_t key[2]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int round = 0; round < 10; ++round) {
    uint32_t hi0 = __umulhi(M0, ctr[0]), lo0 = M0 * ctr[0];
    uint32_t hi1 = __umulhi(M1, ctr[2]), lo1 = M1 * ctr[2];
    uint32_t n0 = hi1 ^ ctr[1] ^ key[0];
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ ctr[3] ^ key[1];
    uint32_t n3 = lo0;
    ctr[0] = n0; ctr[1] = n1; ctr[2] = n2; ctr[3] = n3;
    key[0] += W0;
    key[1] += W1;
  }
}

struct SynthDesc {
  const double* A[kMaxModes];
  int64_t dims[kMaxModes];
  int N, k;
  double sigma;
  uint64_t seed;
  int clip;
};

template <typename T>
__global__ void __launch_bounds__(256) k_synth_cp(SynthDesc d, int64_t numel, T* __restrict__ X) {
  for (int64_t idx = (int64_t)blockIdx.x * 256 + threadIdx.x; idx < numel;
       idx += (int64_t)gridDim.x * 256) {
    int64_t rem = idx;
    int64_t sub[kMaxModes];
    for (int m = 0; m < d.N; ++m) {
      sub[m] = rem % d.dims[m];
      rem /= d.dims[m];
    }
    double v = 0.0;
    for (int r = 0; r < d.k; ++r) {
      double p = 1.0;
      for (int m = d.N - 1; m >= 0; --m) p = d.A[m][sub[m] * d.k + r] * p;
      v += p;
    }
    if (d.sigma > 0) {
      uint32_t ctr[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0x5eedu, 0u};
      uint32_t key[2] = {(uint32_t)d.seed, (uint32_t)(d.seed >> 32)};
      philox4x32_10(ctr, key);
      double u1 = ((double)ctr[0] + 1.0) * (1.0 / 4294967296.0);  // (0, 1]
      double u2 = (double)ctr[1] * (1.0 / 4294967296.0);          // [0, 1)
      double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
      v += d.sigma * z;
    }
    if (d.clip && v < 0) v = 0;
    X[idx] = (T)v;
  }
}

}  // namespace pg
