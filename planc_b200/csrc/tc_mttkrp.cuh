// tc_mttkrp.cuh -- tensor-core partial MTTKRP for the BF16 precisions:
// tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in TMEM), operands
// staged in shared memory by TMA (cp.async.bulk.tensor) and bulk copies,
// warp-specialised persistent kernels with mbarrier pipelines.
//
// The tensor is held as a 2-D matrix X[l + Lpad*j] (l < L = prod_{i<=s} I_i,
// j < R = prod_{i>s} I_i, Lpad = L rounded up to 8 so every TMA row starts on
// a 16-byte boundary) in BF16 (PREC_BF16) or as a BF16 hi/lo pair
// (PREC_BF16X2: x = hi + lo, each rounded to nearest).
//
//   right contraction (dimtree/dimtrees.hpp:106-138, P = X * F_{N-1}):
//     A = X tile 128(l) x 64(j), MN-major (l contiguous), TMA box {64,64} x2
//     B = F_{N-1} slab, pre-split into hi|lo BF16 rows and pre-swizzled in
//         global memory, one bulk copy per stage (K-major, 128B swizzle)
//     D = TMEM 128 lanes x (2*kp) columns: [X*F_hi | X*F_lo]; two
//         accumulators double-buffered so the epilogue of tile t overlaps the
//         MMAs of tile t+1. Epilogue: P32[l*k + r] = D[l, r] + D[l, kp + r].
//   left contraction (dimtrees.hpp:72-105, M_{N-1} = X^T * KRP(F_0..F_s)):
//     A = X^T tile 128(j) x 64(l), K-major, TMA box {64,128}
//     B = Khatri-Rao rows for 64 values of l, generated in shared memory by
//         four producer warps (FP64 product, split hi|lo), K-major 128B swizzle
//     split-K over the CTAs; each CTA writes an FP64 partial R x k that a
//     fixed-order reduction sums (deterministic).
//
// All mbarrier waits are bounded (about 2 s of clock64); a wait that runs out
// sets *status = kStTimeout and a shared abort flag that every other wait
// honours, then the CTA drains its in-flight copies (bounded), frees its TMEM
// and returns.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>

#include <cstdlib>
#include <type_traits>

#include "common.cuh"

namespace pg {

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9 GHz

// Bounded wait on phase `parity`. Returns false (and raises the abort flag)
// when the wait runs out or another warp already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                          int* status, long long limit = kWaitCycles) {
  if (mbar_try(bar, parity)) return true;
  long long t0 = clock64();
  while (true) {
    if (mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (clock64() - t0 > limit) {
      *abort_flag = 1;
      atomicMin(status, kStTimeout);
      return false;
    }
    __nanosleep(64);
  }
}

// After an abort, give every copy already issued time to land (bulk copies
// complete in microseconds) before the CTA's shared memory is released.
__device__ __forceinline__ void tc_drain_after_abort() {
  long long t0 = clock64();
  while (clock64() - t0 < 20000000LL) __nanosleep(1000);
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "l"((uint64_t)src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// SMEM matrix descriptor (tcgen05): start, leading / stride byte offsets (all
// >> 4), version 1, base offset 0, 128-byte swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;  // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::f16: BF16 A and B, FP32 D, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16(int n, bool a_mn_major, bool b_mn_major) {
  return (1u << 4)                          // D format F32
         | (1u << 7)                        // A format BF16
         | (1u << 10)                       // B format BF16
         | ((a_mn_major ? 1u : 0u) << 15)   // A major
         | ((b_mn_major ? 1u : 0u) << 16)   // B major
         | ((uint32_t)(n >> 3) << 17)       // N >> 3
         | ((uint32_t)(128 >> 4) << 24);    // M >> 4
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Two 32-column loads (lane quarter of the calling warp) and one wait.
__device__ __forceinline__ void tmem_ld32x2(uint32_t ta, uint32_t tb, float* va, float* vb) {
  uint32_t a[32], b[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%64];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,"
      "%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%65];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3]), "=r"(a[4]), "=r"(a[5]), "=r"(a[6]),
        "=r"(a[7]), "=r"(a[8]), "=r"(a[9]), "=r"(a[10]), "=r"(a[11]), "=r"(a[12]), "=r"(a[13]),
        "=r"(a[14]), "=r"(a[15]), "=r"(a[16]), "=r"(a[17]), "=r"(a[18]), "=r"(a[19]), "=r"(a[20]),
        "=r"(a[21]), "=r"(a[22]), "=r"(a[23]), "=r"(a[24]), "=r"(a[25]), "=r"(a[26]), "=r"(a[27]),
        "=r"(a[28]), "=r"(a[29]), "=r"(a[30]), "=r"(a[31]),
        "=r"(b[0]), "=r"(b[1]), "=r"(b[2]), "=r"(b[3]), "=r"(b[4]), "=r"(b[5]), "=r"(b[6]),
        "=r"(b[7]), "=r"(b[8]), "=r"(b[9]), "=r"(b[10]), "=r"(b[11]), "=r"(b[12]), "=r"(b[13]),
        "=r"(b[14]), "=r"(b[15]), "=r"(b[16]), "=r"(b[17]), "=r"(b[18]), "=r"(b[19]), "=r"(b[20]),
        "=r"(b[21]), "=r"(b[22]), "=r"(b[23]), "=r"(b[24]), "=r"(b[25]), "=r"(b[26]), "=r"(b[27]),
        "=r"(b[28]), "=r"(b[29]), "=r"(b[30]), "=r"(b[31])
      : "r"(ta), "r"(tb)
      : "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    va[i] = __uint_as_float(a[i]);
    vb[i] = __uint_as_float(b[i]);
  }
}

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

// Byte offset of element (row, kk) (kk < 64 BF16 values along K) inside a
// K-major 128B-swizzled tile whose rows are 128 bytes and whose 8-row groups
// are 1024 bytes apart.
__host__ __device__ __forceinline__ uint32_t sw128_kmajor_off(int row, int kk) {
  uint32_t chunk = (uint32_t)(kk >> 3);        // 16-byte chunk within the row
  uint32_t phys = chunk ^ (uint32_t)(row & 7);  // 128B swizzle
  return (uint32_t)(row >> 3) * 1024u + (uint32_t)(row & 7) * 128u + phys * 16u +
         (uint32_t)(kk & 7) * 2u;
}

__device__ __forceinline__ void split_bf16(double w, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __double2bfloat16(w);
  lo = __double2bfloat16(w - (double)__bfloat162float(hi));
}

constexpr int TC_BM = 128;   // rows per MMA tile
constexpr int TC_BK = 64;    // K per pipeline stage (one 128-byte swizzle row of BF16)
constexpr int TC_THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue / KRP producers
// Stages of a TMA / cp.async ring of stage_bytes each in ~200 KB of shared
// memory (2 .. 8).
__host__ __device__ constexpr int tc_stages(uint32_t stage_bytes) {
  return (int)(200u * 1024u / stage_bytes) < 2 ? 2
         : (int)(200u * 1024u / stage_bytes) > 8 ? 8 : (int)(200u * 1024u / stage_bytes);
}
// cp.async groups (stages) each producer thread keeps in flight for a ring of
// stage_bytes stages: up to 5, leaving at least 3 stages for the MMAs'
// turnaround (with one or two to spare the producers wait on the MMAs); the
// cp.async instances are used when this is at least 2.
__host__ __device__ constexpr int tc_cpa_depth(uint32_t stage_bytes) {
  return tc_stages(stage_bytes) - 3 < 5 ? tc_stages(stage_bytes) - 3 : 5;
}

// Shared memory the right contraction's four epilogue warps stage their rows
// of P in (32 rows of KP floats each), after the stage ring; the 16-column
// instance stores directly.
template <int KP>
__host__ __device__ constexpr uint32_t tc_right_pstage() {
  return KP >= 32 ? 4u * 32u * (uint32_t)KP * 4u : 0u;
}

// 16-byte cp.async (L1 bypassed) that reads `bytes` (0..16) from src and
// zero-fills the rest of the destination; src must be 16-byte aligned.
__device__ __forceinline__ void cp_async16_zfill(uint32_t dst, const void* src, uint32_t bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ------------------------------------------------------------ right kernel
// P32[l*k + r] = sum_j X[l, j] * F[j, r], l < L, r < k.
// With TTV (3-way tree, I0 a multiple of 128, gridDim a multiple of
// tpb = I0 / 128) the epilogue also forms the mode-0 multi-TTV of the tiles
// it drains: tile t covers rows l = i0 + I0 * i1 with i1 = t / tpb and
// i0 = (t % tpb) * 128 + row, and t % tpb = blockIdx % tpb for every tile of
// a CTA, so each epilogue thread keeps one i0's sums
//   sum_{i1 of its tiles} P[i0 + I0 i1, r] * F1[i1, r]   (FP64)
// and writes them to part[blockIdx / tpb][i0][r]; k_reduce_splits adds the
// gridDim / tpb partials into M_0 (the sum k_ttv_right_tiled forms from P).
//
// With CPA the A tiles are not fetched by TMA: four more warps (6-9) copy
// them with 16-byte cp.async into the same 128B-swizzled MN-major layout,
// tc_cpa_depth(STAGE) stages of copies in flight per thread (on B200 this
// streams the 256-byte row pieces of a tile ~15 % faster than two {64, 64}
// TMA boxes). Each producer thread waits for its oldest group, makes it
// visible to the tensor cores' async proxy and arrives on the stage's full
// barrier (count 1 + 128: warp 0's B-image expect_tx and the 128 producers).
// Rows l >= L and columns j >= R are zero-filled through the copy's source
// size. Needs stages = tc_stages(STAGE) and a row stride Lpad that is a
// multiple of 8.
template <int KP, bool X2, bool TTV = false, bool CPA = false>
__global__ void __launch_bounds__(CPA ? TC_THREADS + 128 : TC_THREADS, 1)
    k_tc_right(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
               const uint8_t* __restrict__ bimg, int64_t L, int64_t R, int k, int stages,
               float* __restrict__ P, int* __restrict__ status, const double* __restrict__ F1 = nullptr,
               int tpb = 1, int64_t I0 = 0, double* __restrict__ part = nullptr,
               const __nv_bfloat16* __restrict__ xhi = nullptr,
               const __nv_bfloat16* __restrict__ xlo = nullptr, int64_t Lpad = 0) {
  constexpr int NCOL = 2 * KP;                       // hi | lo columns
  constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2;    // one BF16 A tile
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;           // NCOL rows x 128 B
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr int NBUF = 4;  // accumulators in flight
  constexpr uint32_t TMEM_COLS = NBUF * NCOL < 32 ? 32 : NBUF * NCOL;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, true, false);
  // P staging of one epilogue warp, after the stage ring (0: direct stores)
  constexpr uint32_t PST_BYTES = tc_right_pstage<KP>() / 4;
  constexpr int DEPTH = tc_cpa_depth(STAGE);

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 2 * NBUF];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ntiles = (L + TC_BM - 1) / TC_BM;
  const int nk = (int)((R + TC_BK - 1) / TC_BK);
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[8 + s]); };
  auto accf = [&](int b) { return smem_u32(&bars[16 + b]); };
  auto acce = [&](int b) { return smem_u32(&bars[16 + NBUF + b]); };

  if (threadIdx.x == 0) {
    abort_sh = 0;
    for (int s = 0; s < stages; ++s) {
      mbar_init(full(s), CPA ? 1 + 128 : 1);
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(accf(b), 1);
      mbar_init(acce(b), 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  volatile int* abort_flag = &abort_sh;

  if (warp == 0) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const int l0 = (int)(t * TC_BM);
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
          const uint32_t st = smem0 + s * STAGE;
          if (CPA) {
            mbar_expect_tx(full(s), B_STAGE);
          } else {
            mbar_expect_tx(full(s), STAGE);
            tma_load_2d(st, &tm_hi, l0, kb * TC_BK, full(s));
            tma_load_2d(st + A_BYTES / 2, &tm_hi, l0 + 64, kb * TC_BK, full(s));
            if (X2) {
              tma_load_2d(st + A_BYTES, &tm_lo, l0, kb * TC_BK, full(s));
              tma_load_2d(st + A_BYTES + A_BYTES / 2, &tm_lo, l0 + 64, kb * TC_BK, full(s));
            }
          }
          bulk_load(st + A_STAGE, bimg + (size_t)kb * B_STAGE, B_STAGE, full(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      int buf = 0;
      uint32_t aph = 0;  // bit b: phase of accumulator b
      bool ok = true;
      for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        if (!mbar_wait(acce(buf), ((aph >> buf) & 1) ^ 1, abort_flag, status)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * NCOL;
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(full(s), ph, abort_flag, status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem0 + s * STAGE;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk) {
            // MN-major A: K advances 16 rows = two 1024 B k-groups
            const uint64_t bdesc = smem_desc(st + A_STAGE + kk * 32, 16, 1024);
            const uint64_t adesc = smem_desc(st + kk * 2048, A_BYTES / 2, 1024);
            umma_bf16(d, adesc, bdesc, IDESC, (kb | kk) != 0);
            if (X2) {
              const uint64_t adesc2 = smem_desc(st + A_BYTES + kk * 2048, A_BYTES / 2, 1024);
              umma_bf16(d, adesc2, bdesc, IDESC, 1);
            }
          }
          umma_commit(empty(s));  // frees the stage once these MMAs finish
          if (++s == stages) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(accf(buf));
        aph ^= 1u << buf;
        buf = (buf + 1) % NBUF;
      }
    }
  } else if (warp < 6) {
    // epilogue warps 2..5: TMEM lane quarter = warp % 4
    const int q = warp & 3;
    int buf = 0;
    uint32_t aph = 0;
    double tacc[TTV ? KP : 1];
#pragma unroll
    for (int r = 0; r < (TTV ? KP : 1); ++r) tacc[r] = 0.0;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
      if (!mbar_wait(accf(buf), (aph >> buf) & 1, abort_flag, status)) break;
      tc_fence_after();
      const int64_t row = t * TC_BM + q * 32 + lane;
      const uint32_t tacc_addr = tmem + ((uint32_t)(q * 32) << 16) + buf * NCOL;
      // with k == KP (KP >= 32) the warp's 32 rows of P are one contiguous
      // block: they are staged in shared memory (row lane's 16-byte chunk c
      // at c ^ (lane % 8), no bank conflicts) and written back with coalesced
      // stores; otherwise each thread stores its row. The accumulator is
      // drained 16 columns at a time.
      const bool staged = PST_BYTES > 0 && k == KP;
      uint8_t* sp = smem + (size_t)stages * STAGE + (size_t)(warp - 2) * PST_BYTES;
      const double* f = TTV ? F1 + (t / tpb) * k : nullptr;
#pragma unroll
      for (int h = 0; h < KP / 16; ++h) {
        float a[16], b[16];
        tmem_ld16(tacc_addr + h * 16, a);
        tmem_ld16(tacc_addr + KP + h * 16, b);
        if (staged) {
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const float4 o = make_float4(a[4 * c] + b[4 * c], a[4 * c + 1] + b[4 * c + 1],
                                         a[4 * c + 2] + b[4 * c + 2], a[4 * c + 3] + b[4 * c + 3]);
            *reinterpret_cast<float4*>(sp + lane * (KP * 4) + (((h * 4 + c) ^ (lane & 7)) << 4)) = o;
          }
        } else if (row < L) {
          float* dst = P + row * k + h * 16;
          if (k == KP) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
              *reinterpret_cast<float4*>(dst + 4 * c) =
                  make_float4(a[4 * c] + b[4 * c], a[4 * c + 1] + b[4 * c + 1],
                              a[4 * c + 2] + b[4 * c + 2], a[4 * c + 3] + b[4 * c + 3]);
          } else {
#pragma unroll
            for (int r = 0; r < 16; ++r)
              if (h * 16 + r < k) dst[r] = a[r] + b[r];
          }
        }
        if constexpr (TTV) {
          if (row < L) {
#pragma unroll
            for (int r = 0; r < 16; ++r)
              if (h * 16 + r < k)
                tacc[h * 16 + r] = fma((double)(a[r] + b[r]), f[h * 16 + r], tacc[h * 16 + r]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(buf));
      aph ^= 1u << buf;
      buf = (buf + 1) % NBUF;
      if (staged) {
        const int64_t row0 = t * TC_BM + q * 32;
#pragma unroll
        for (int it = 0; it < KP / 4; ++it) {
          const int u = it * 32 + lane;  // 16-byte unit of the block
          const int j = u / (KP / 4), c = u % (KP / 4);
          const float4 o = *reinterpret_cast<const float4*>(sp + j * (KP * 4) + ((c ^ (j & 7)) << 4));
          if (row0 + j < L) *reinterpret_cast<float4*>(P + (row0 + j) * KP + 4 * c) = o;
        }
        __syncwarp();
      }
    }
    if constexpr (TTV) {
      const int64_t i0 = (int64_t)(blockIdx.x % tpb) * TC_BM + q * 32 + lane;
      double* dst = part + (int64_t)(blockIdx.x / tpb) * I0 * k + i0 * k;
#pragma unroll
      for (int r = 0; r < KP; ++r)
        if (r < k) dst[r] = tacc[r];
    }
  } else if (CPA) {
    // A-tile producers, warps 6..9: per stage 1024 (2048 with X2) copies of
    // 16 bytes; copy q = pt + 128 i takes the 16-byte piece c16 = q % 16 of
    // row j = q / 16 of the K block (l = l0 + 8 c16), which lands in box
    // c16 / 8, chunk (c16 % 8) ^ (j % 8) of the swizzled row j
    // (c16 and j % 8 are fixed per thread: its copies step 8 rows = 1 KB)
    const int pt = threadIdx.x - TC_THREADS;
    const int c16 = pt & 15, jt = pt >> 4;
    const uint32_t dofs = (uint32_t)(c16 >> 3) * (A_BYTES / 2) + (uint32_t)jt * 128u +
                          ((uint32_t)((c16 & 7) ^ jt) << 4);
    int s = 0;
    uint32_t ph = 0;
    int inflight = 0;  // copy groups committed, not yet announced
    int ps = 0;        // stage of the oldest of them (groups go in stage order)
    bool ok = true;
    for (int64_t t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
      const int64_t l = t * TC_BM + 8 * c16;
      const int64_t left = L - l;
      const uint32_t lbytes = left <= 0 ? 0u : left >= 8 ? 16u : (uint32_t)left * 2u;
      for (int kb = 0; kb < nk; ++kb) {
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
        const uint32_t dst = smem0 + s * STAGE + dofs;
        const int64_t j0 = (int64_t)kb * TC_BK + jt;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int64_t jj = j0 + 8 * i;
          const uint32_t bytes = jj < R ? lbytes : 0u;
          const size_t off = bytes ? (size_t)jj * (size_t)Lpad + (size_t)l : 0;
          cp_async16_zfill(dst + 1024u * i, xhi + off, bytes);
          if (X2) cp_async16_zfill(dst + 1024u * i + A_BYTES, xlo + off, bytes);
        }
        cp_async_commit();
        if (++inflight > DEPTH) {
          cp_async_wait<DEPTH>();
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(full(ps));
          if (++ps == stages) ps = 0;
          --inflight;
        }
        if (++s == stages) { s = 0; ph ^= 1; }
      }
    }
    cp_async_wait<0>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (ok)
      for (; inflight > 0; --inflight) {
        mbar_arrive(full(ps));
        if (++ps == stages) ps = 0;
      }
  }
  __syncthreads();
  if (abort_sh) tc_drain_after_abort();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// Pre-swizzled B image for the right contraction: for stage kb, NCOL rows of
// 128 bytes (K-major, 128B swizzle); row r < KP holds hi(F[j, r]) and row
// KP + r holds lo(F[j, r]) for j = kb*64 .. kb*64+63 (zero beyond R or k).
template <int KP>
__device__ __forceinline__ void tc_bimage_body(const double* __restrict__ F, int64_t R, int k, int nk,
                                               uint8_t* __restrict__ img, int64_t bx, int64_t gx) {
  constexpr int NCOL = 2 * KP;
  const int64_t total = (int64_t)nk * KP * TC_BK;
  for (int64_t e = bx * blockDim.x + threadIdx.x; e < total; e += gx * blockDim.x) {
    const int kk = (int)(e % TC_BK);
    const int r = (int)((e / TC_BK) % KP);
    const int kb = (int)(e / ((int64_t)TC_BK * KP));
    const int64_t j = (int64_t)kb * TC_BK + kk;
    __nv_bfloat16 hi = __float2bfloat16(0.f), lo = __float2bfloat16(0.f);
    if (j < R && r < k) split_bf16(F[j * k + r], hi, lo);
    uint8_t* st = img + (size_t)kb * NCOL * 128;
    *reinterpret_cast<__nv_bfloat16*>(st + sw128_kmajor_off(r, kk)) = hi;
    *reinterpret_cast<__nv_bfloat16*>(st + sw128_kmajor_off(KP + r, kk)) = lo;
  }
}
template <int KP>
__global__ void k_tc_bimage(const double* __restrict__ F, int64_t R, int k, int nk,
                            uint8_t* __restrict__ img) {
  tc_bimage_body<KP>(F, R, k, nk, img, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------ left kernel
// part[split][j*k + r] = sum_{l in split} X[l, j] * W(l, r), W = KRP(F_0..F_s).
// Grid: (mgroups, nsplit); a CTA owns MT consecutive 128-row tiles of j.
// Split y takes the 64-wide chunks of l numbered y, y + nsplit, y + 2*nsplit..
// so the CTAs running together read neighbouring 128-byte pieces of the same
// rows of X (DRAM page locality). The tensor-core accumulator is restarted
// every TCL_GROUP chunks (double-buffered in TMEM) and drained by four
// dedicated warps into register running sums, which keeps every FP32
// accumulation chain short.
constexpr int TCL_GROUP = 8;        // chunks per accumulator group
constexpr int TCL_THREADS = 320;    // warp 0 TMA, 1 MMA, 2-5 KRP producers, 6-9 drain

template <int KP, int MT, bool X2>
__global__ void __launch_bounds__(TCL_THREADS, 1)
    k_tc_left(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
              WGen wg, int64_t L, int64_t R, int k, int stages, double* __restrict__ part,
              int* __restrict__ status) {
  constexpr int NCOL = 2 * KP;
  constexpr uint32_t A_TILE = TC_BM * TC_BK * 2;  // 16 KB
  constexpr uint32_t A_BYTES = MT * A_TILE;
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr uint32_t ACC_COLS = MT * NCOL;  // one accumulator buffer
  constexpr uint32_t TMEM_NEED = 2 * ACC_COLS;
  constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128
                                 : TMEM_NEED <= 256 ? 256 : 512;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, false, false);
  // running sums of the drain warps: FP64 when they fit in registers
  using Acc = typename std::conditional<(MT * KP <= 64), double, float>::type;

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 4];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nchunks = (L + TC_BK - 1) / TC_BK;
  const int64_t ns = gridDim.y;
  const int64_t y = blockIdx.y;
  const int64_t my_chunks = y < nchunks ? (nchunks - y + ns - 1) / ns : 0;
  const int64_t ngroups = (my_chunks + TCL_GROUP - 1) / TCL_GROUP;
  const int j0 = blockIdx.x * MT * TC_BM;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[8 + s]); };
  auto accf = [&](int b) { return smem_u32(&bars[16 + b]); };
  auto acce = [&](int b) { return smem_u32(&bars[18 + b]); };

  if (threadIdx.x == 0) {
    abort_sh = 0;
    for (int s = 0; s < stages; ++s) {
      mbar_init(full(s), 1 + 4);  // TMA expect_tx arrival + 4 producer warps
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(accf(b), 1);
      mbar_init(acce(b), 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  volatile int* abort_flag = &abort_sh;

  if (warp == 0) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      for (int64_t i = 0; i < my_chunks; ++i) {
        const int64_t c = y + i * ns;
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) break;
        const uint32_t st = smem0 + s * STAGE;
        mbar_expect_tx(full(s), A_STAGE);
        for (int mt = 0; mt < MT; ++mt) {
          tma_load_2d(st + mt * A_TILE, &tm_hi, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
          if (X2) tma_load_2d(st + A_BYTES + mt * A_TILE, &tm_lo, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
        }
        if (++s == stages) { s = 0; ph ^= 1; }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t aph[2] = {0, 0};
      bool ok = true;
      int64_t i = 0;
      for (int64_t g = 0; g < ngroups && ok; ++g) {
        const int buf = (int)(g & 1);
        if (!mbar_wait(acce(buf), aph[buf] ^ 1, abort_flag, status)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * ACC_COLS;
        const int64_t iend = (i + TCL_GROUP < my_chunks) ? i + TCL_GROUP : my_chunks;
        for (int64_t i0 = i; i < iend; ++i) {
          if (!mbar_wait(full(s), ph, abort_flag, status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem0 + s * STAGE;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk) {
            const uint64_t bdesc = smem_desc(st + A_STAGE + kk * 32, 16, 1024);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
              const uint64_t adesc = smem_desc(st + mt * A_TILE + kk * 32, 16, 1024);
              umma_bf16(d + mt * NCOL, adesc, bdesc, IDESC, (i != i0 || kk != 0) ? 1u : 0u);
              if (X2) {
                const uint64_t adesc2 = smem_desc(st + A_BYTES + mt * A_TILE + kk * 32, 16, 1024);
                umma_bf16(d + mt * NCOL, adesc2, bdesc, IDESC, 1);
              }
            }
          }
          umma_commit(empty(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(accf(buf));
        aph[buf] ^= 1;
      }
    }
  } else if (warp < 6) {
    // producer warps 2..5 build the Khatri-Rao B tile of every chunk:
    // thread pt owns rank r = pt % KP and octets of l (8 consecutive values,
    // one 16-byte swizzled store per octet for hi and for lo); a warp's lanes
    // read 32 consecutive ranks of a factor row (coalesced).
    constexpr int OCT_LANES = 128 / KP;        // threads per rank
    constexpr int OCT_PER = 8 / OCT_LANES;     // octets per thread per chunk
    const int pt = threadIdx.x - 64;           // 0..127
    const int r = pt % KP;
    const int oct0 = pt / KP;
    const bool rok = r < k;
    const int nf = wg.nf;                      // 2 (N = 3) or 3 (N = 4)
    const double* F0 = wg.f[0];
    const double* F1 = wg.f[1];
    const double* F2 = nf > 2 ? wg.f[2] : wg.f[1];
    const int64_t D0 = wg.dim[0], D1 = wg.dim[1];
    // digits of l0 = c * 64 for the first chunk of this split
    int64_t b0, b1, b2;
    {
      const int64_t l0 = y * TC_BK;
      b0 = l0 % D0;
      b1 = (l0 / D0) % D1;
      b2 = nf > 2 ? l0 / (D0 * D1) : 0;
    }
    const int64_t step = TC_BK * ns;  // l advance between this split's chunks
    int s = 0;
    uint32_t ph = 0;
    for (int64_t i = 0; i < my_chunks; ++i) {
      const int64_t c = y + i * ns;
      if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) break;
      uint8_t* bt = smem + s * STAGE + A_STAGE;
#pragma unroll
      for (int t = 0; t < OCT_PER; ++t) {
        const int j = oct0 + OCT_LANES * t;  // octet 0..7
        int64_t d0 = b0 + 8 * j, d1 = b1, d2 = b2;
        while (d0 >= D0) { d0 -= D0; ++d1; }
        if (nf > 2) while (d1 >= D1) { d1 -= D1; ++d2; }
        const int64_t lbase = c * TC_BK + 8 * j;
        // product of the slower modes' factor entries, constant along a run of l
        auto tail_of = [&](int64_t e1, int64_t e2) -> float {
          double tl = F1[e1 * k + r];
          if (nf > 2) tl = tl * F2[e2 * k + r];
          return (float)tl;
        };
        float tail = (rok && lbase < L) ? tail_of(d1, d2) : 0.f;
        uint32_t hw[4], lw[4];
#pragma unroll
        for (int e = 0; e < 8; e += 2) {
          float w[2];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            w[u] = 0.f;
            if (rok && lbase + e + u < L) w[u] = (float)F0[d0 * k + r] * tail;
            if (++d0 == D0) {
              d0 = 0;
              if (++d1 == D1 && nf > 2) { d1 = 0; ++d2; }
              if (rok && lbase + e + u + 1 < L) tail = tail_of(d1, d2);
            }
          }
          // FP32 product split into BF16 hi + lo (w - hi is exact in FP32)
          __nv_bfloat162 h2 = __floats2bfloat162_rn(w[0], w[1]);
          float2 hf = __bfloat1622float2(h2);
          __nv_bfloat162 l2 = __floats2bfloat162_rn(w[0] - hf.x, w[1] - hf.y);
          hw[e >> 1] = *reinterpret_cast<uint32_t*>(&h2);
          lw[e >> 1] = *reinterpret_cast<uint32_t*>(&l2);
        }
        *reinterpret_cast<uint4*>(bt + sw128_kmajor_off(r, 8 * j)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(bt + sw128_kmajor_off(KP + r, 8 * j)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
      }
      // advance the chunk base digits by `step`
      b0 += step;
      if (b0 >= D0) {
        int64_t q = b0 / D0;
        b0 -= q * D0;
        b1 += q;
        if (nf > 2 && b1 >= D1) {
          int64_t q2 = b1 / D1;
          b1 -= q2 * D1;
          b2 += q2;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(full(s));
      if (++s == stages) { s = 0; ph ^= 1; }
    }
  } else {
    // drain warps 6..9: TMEM lane quarter = warp % 4
    const int q = warp & 3;
    Acc sum[MT][KP];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int r = 0; r < KP; ++r) sum[mt][r] = 0;
    uint32_t aph[2] = {0, 0};
    bool ok = true;
    for (int64_t g = 0; g < ngroups; ++g) {
      const int buf = (int)(g & 1);
      if (!mbar_wait(accf(buf), aph[buf], abort_flag, status)) { ok = false; break; }
      tc_fence_after();
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
        for (int cc = 0; cc < NCOL; cc += 32) {
          float v[32];
          tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * ACC_COLS + mt * NCOL + cc, v);
#pragma unroll
          for (int i = 0; i < 32; ++i) sum[mt][(cc + i) % KP] += (Acc)v[i];  // hi then lo column
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(buf));
      aph[buf] ^= 1;
    }
    if (ok) {
      double* dst = part + y * R * k;
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int64_t j = (int64_t)j0 + mt * TC_BM + q * 32 + lane;
        if (j < R) {
#pragma unroll
          for (int r = 0; r < KP; ++r)
            if (r < k) dst[j * k + r] = (double)sum[mt][r];
        }
      }
    }
  }
  __syncthreads();
  if (abort_sh) tc_drain_after_abort();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// ------------------------------------------------------------ left kernel, factored form
// When I_0 is a multiple of 64, every 64-wide chunk of l lies inside one run
// of I_0 consecutive values of l that share the slower modes' digits, so the
// Khatri-Rao row factors as W(l, r) = F_0[i_0, r] * tail(g, r) with
// g = l / I_0 and tail = F_1[i_1, r] (* F_2[i_2, r]) (the reference's
// product F_0 * (F_1 * F_2) up to rounding). Then
//     M[j, r] = sum_g tail(g, r) * sum_{i_0} X[i_0 + I_0 g, j] * F_0[i_0, r]
// The inner sums are tensor-core MMAs against a static operand, F_0 split into
// BF16 hi|lo rows and pre-swizzled in global memory (one bulk copy per stage,
// as in the right contraction); the accumulator of each run g is drained and
// scaled by tail(g, .) in FP64 by four drain warps. No producer warps, and the
// tensor-core accumulation chain is one run (I_0/64 chunks) long.
// Work units are parts of runs: with hp parts per run, unit u covers chunks
// (u % hp) * G/hp .. of run u / hp (the accumulator is restarted and scaled
// per unit, which the sum allows since tail(g, r) is common to the run).
// Split y takes units y, y + nsplit, ..., so concurrent CTAs read adjacent
// pieces of the same rows of X.
constexpr int TCF_THREADS = 192;  // warp 0 TMA, 1 MMA, 2-5 drain

// Shared-memory stage of k_tc_left_fac: KBS 64-wide K blocks of MT 128-row
// A tiles (a second set for the lo part with X2) and KBS B slabs.
__host__ __device__ constexpr uint32_t tcf_stage_bytes(int kp, int mt, bool x2, int kbs) {
  return (x2 ? 2u : 1u) * kbs * mt * (uint32_t)(TC_BM * TC_BK * 2) + kbs * 2u * kp * 128u;
}

// With CPA (MT = 1) the A tiles come from four cp.async producer warps
// (6-9) instead of TMA: 16-byte copies written to the swizzled positions,
// zero-filled past R. A copy group fills a pair of stages (two consecutive
// K blocks), so each warp-wide copy reads two 256-byte row pieces of X (on
// B200 cp.async streams this pattern at ~6.9 TB/s, 128-byte pieces at ~4.9
// and TMA boxes of any shape at ~6.0); tcf_cpa_depth(stages) pairs are in
// flight per thread (up to 2, leaving at least two pairs for the MMAs'
// turnaround: at 1024^3 rank 32, an 8-stage ring, the kernel takes 0.340 ms
// with 2, 0.363 with 1 and 0.54 with 3). Warp 0 then loads only the B slab of a stage, and the full
// barrier counts its expect_tx and the 128 producers. Needs an even number
// of stages and units of an even number of chunks.
__host__ __device__ constexpr int tcf_cpa_depth(int stages) { return stages / 2 - 2 < 2 ? stages / 2 - 2 : 2; }
// Whether the cp.async instance exists for (KP, X2): rank <= 32 (the drain
// warps' sums within the 10-warp register budget) and an even ring of at
// least 6 stages.
__host__ __device__ constexpr bool tcf_cpa_ok(int kp, bool x2) {
  return kp <= 32 && tc_stages(tcf_stage_bytes(kp, 1, x2, 1)) % 2 == 0 &&
         tcf_cpa_depth(tc_stages(tcf_stage_bytes(kp, 1, x2, 1))) >= 2;
}
template <int KP, int MT, bool X2, bool CPA = false>
__global__ void __launch_bounds__(CPA ? TCF_THREADS + 128 : TCF_THREADS, 1)
    k_tc_left_fac(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
                  const uint8_t* __restrict__ img0, const double* __restrict__ F1,
                  const double* __restrict__ F2, int64_t D1, int64_t I0, int64_t L, int64_t R, int k,
                  int stages, double* __restrict__ part, int* __restrict__ status, int hp = 1,
                  const __nv_bfloat16* __restrict__ xhi = nullptr,
                  const __nv_bfloat16* __restrict__ xlo = nullptr, int64_t Lpad = 0) {
  static_assert(!CPA || MT == 1, "the cp.async instance takes one 128-row tile");
  constexpr int KBS = 1;                           // K blocks per stage
  constexpr int NCOL = 2 * KP;
  constexpr uint32_t A_TILE = TC_BM * TC_BK * 2;  // 16 KB
  constexpr uint32_t A_BYTES = KBS * MT * A_TILE;  // tile (kb, mt) at (kb * MT + mt) * A_TILE
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;         // one slab of the F_0 image
  constexpr uint32_t STAGE = A_STAGE + KBS * B_STAGE;
  static_assert(STAGE == tcf_stage_bytes(KP, MT, X2, KBS), "stage layout");
  constexpr uint32_t ACC_COLS = MT * NCOL;
  constexpr int NBUF = 4 * ACC_COLS <= 512 ? 4 : 2;  // accumulators in flight
  constexpr uint32_t TMEM_NEED = NBUF * ACC_COLS;
  constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128
                                 : TMEM_NEED <= 256 ? 256 : 512;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, false, false);
  using Acc = typename std::conditional<(MT * KP <= 64), double, float>::type;

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 2 * NBUF];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  __shared__ double tail_w[4][KP];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t G = I0 / TC_BK;          // chunks per run
  const int64_t GH = G / hp;             // chunks per unit (a part of a run)
  const int64_t nunits = L / I0 * hp;
  const int64_t ns = gridDim.y;
  const int64_t y = blockIdx.y;
  const int64_t my_units = y < nunits ? (nunits - y + ns - 1) / ns : 0;
  const int j0 = blockIdx.x * MT * TC_BM;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[8 + s]); };
  auto accf = [&](int b) { return smem_u32(&bars[16 + b]); };
  auto acce = [&](int b) { return smem_u32(&bars[16 + NBUF + b]); };

  if (threadIdx.x == 0) {
    abort_sh = 0;
    for (int s = 0; s < stages; ++s) {
      mbar_init(full(s), CPA ? 1 + 128 : 1);
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(accf(b), 1);
      mbar_init(acce(b), 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  volatile int* abort_flag = &abort_sh;

  if (warp == 0) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int64_t i = 0; i < my_units && ok; ++i) {
        const int64_t u = y + i * ns;
        for (int64_t q = (u % hp) * GH, qe = q + GH; q < qe; q += KBS) {
          const int64_t c = (u / hp) * G + q;
          if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
          const uint32_t st = smem0 + s * STAGE;
          if (CPA) {
            mbar_expect_tx(full(s), KBS * B_STAGE);
          } else {
            mbar_expect_tx(full(s), STAGE);
            for (int mt = 0; mt < MT; ++mt) {
              tma_load_2d(st + mt * A_TILE, &tm_hi, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
              if (X2) tma_load_2d(st + A_BYTES + mt * A_TILE, &tm_lo, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
            }
          }
          bulk_load(st + A_STAGE, img0 + (size_t)q * B_STAGE, KBS * B_STAGE, full(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t aph = 0;  // bit b: phase of accumulator b
      bool ok = true;
      for (int64_t i = 0; i < my_units && ok; ++i) {
        const int buf = (int)(i % NBUF);
        if (!mbar_wait(acce(buf), ((aph >> buf) & 1) ^ 1, abort_flag, status)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * ACC_COLS;
        for (int64_t q = 0; q < GH; q += KBS) {
          if (!mbar_wait(full(s), ph, abort_flag, status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem0 + s * STAGE;
#pragma unroll
          for (int kb = 0; kb < KBS; ++kb)
#pragma unroll
            for (int kk = 0; kk < TC_BK / 16; ++kk) {
              const uint64_t bdesc = smem_desc(st + A_STAGE + kb * B_STAGE + kk * 32, 16, 1024);
#pragma unroll
              for (int mt = 0; mt < MT; ++mt) {
                const uint32_t at = st + (kb * MT + mt) * A_TILE + kk * 32;
                umma_bf16(d + mt * NCOL, smem_desc(at, 16, 1024), bdesc, IDESC,
                          (q != 0 || kb != 0 || kk != 0) ? 1u : 0u);
                if (X2) umma_bf16(d + mt * NCOL, smem_desc(at + A_BYTES, 16, 1024), bdesc, IDESC, 1);
              }
            }
          umma_commit(empty(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(accf(buf));
        aph ^= 1u << buf;
      }
    }
  } else if (warp < 6) {
    // drain warps 2..5: TMEM lane quarter = warp % 4. Each warp stages the
    // run's tail(g, .) in its own shared-memory slice (no cross-warp wait).
    const int q4 = warp & 3;
    double* tail = tail_w[warp - 2];
    Acc sum[MT][KP];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int r = 0; r < KP; ++r) sum[mt][r] = 0;
    uint32_t aph = 0;
    bool ok = true;
    for (int64_t i = 0; i < my_units; ++i) {
      const int buf = (int)(i % NBUF);
      const int64_t g = (y + i * ns) / hp;
      const int64_t i1 = F2 ? g % D1 : g;
      const int64_t i2 = F2 ? g / D1 : 0;
      __syncwarp();
      for (int r = lane; r < KP; r += 32) {
        double t = 0.0;
        if (r < k) {
          t = F1[i1 * k + r];
          if (F2) t = t * F2[i2 * k + r];
        }
        tail[r] = t;
      }
      __syncwarp();
      if (!mbar_wait(accf(buf), (aph >> buf) & 1, abort_flag, status)) { ok = false; break; }
      tc_fence_after();
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const uint32_t base = tmem + ((uint32_t)(q4 * 32) << 16) + buf * ACC_COLS + mt * NCOL;
        if (KP == 16) {
          float v[32];
          tmem_ld32(base, v);  // columns 0..15 hi, 16..31 lo
#pragma unroll
          for (int r = 0; r < 16; ++r)
            sum[mt][r] += (Acc)(tail[r] * ((double)v[r] + (double)v[16 + r]));
        } else {
#pragma unroll
          for (int cc = 0; cc < KP; cc += 16) {
            float vh[16], vl[16];
            tmem_ld16(base + cc, vh);
            tmem_ld16(base + KP + cc, vl);
#pragma unroll
            for (int e = 0; e < 16; ++e)
              sum[mt][cc + e] += (Acc)(tail[cc + e] * ((double)vh[e] + (double)vl[e]));
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(buf));
      aph ^= 1u << buf;
    }
    if (ok) {
      double* dst = part + y * R * k;
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int64_t j = (int64_t)j0 + mt * TC_BM + q4 * 32 + lane;
        if (j < R) {
#pragma unroll
          for (int r = 0; r < KP; ++r)
            if (r < k) dst[j * k + r] = (double)sum[mt][r];
        }
      }
    }
  } else if (CPA) {
    // A-tile producers, warps 6..9: per pair of stages 2048 (x2 with X2)
    // copies of 16 bytes; copy u = pt + 128 i takes the 16-byte piece
    // p = u % 16 (l = 64 c + 8 p, chunk c of the pair's first stage) of tile
    // row u / 16 (j = j0 + u / 16), which lands in stage p / 8 of the pair,
    // chunk (p % 8) ^ (row % 8) of the swizzled row. p and row % 8 are fixed
    // per thread: its copies step 8 rows = 1 KB.
    constexpr int DEPTH = tcf_cpa_depth(tc_stages(STAGE));
    static_assert(!CPA || (tc_stages(STAGE) % 2 == 0 && DEPTH >= 2), "stage pairs");
    const int pt = threadIdx.x - TCF_THREADS;
    const int p = pt & 15, jt = pt >> 4;
    const uint32_t dofs = (uint32_t)(p >> 3) * STAGE + (uint32_t)jt * 128u + ((uint32_t)((p & 7) ^ jt) << 4);
    int s = 0;  // first stage of the pair (even)
    uint32_t ph = 0;
    int inflight = 0;  // copy groups (pairs) committed, not yet announced
    int ps = 0;        // first stage of the oldest of them
    bool ok = true;
    for (int64_t i = 0; i < my_units && ok; ++i) {
      const int64_t u = y + i * ns;
      for (int64_t q = (u % hp) * GH, qe = q + GH; q < qe; q += 2) {
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status) ||
            !mbar_wait(empty(s + 1), ph ^ 1, abort_flag, status)) { ok = false; break; }
        const uint32_t dst = smem0 + s * STAGE + dofs;
        const int64_t l = ((u / hp) * G + q) * TC_BK + 8 * p;
        const int64_t left = L - l;
        const uint32_t lbytes = left <= 0 ? 0u : left >= 8 ? 16u : (uint32_t)left * 2u;
#pragma unroll
        for (int i8 = 0; i8 < 16; ++i8) {
          const int64_t j = (int64_t)j0 + jt + 8 * i8;
          const uint32_t bytes = j < R ? lbytes : 0u;
          const size_t off = bytes ? (size_t)j * (size_t)Lpad + (size_t)l : 0;
          cp_async16_zfill(dst + 1024u * i8, xhi + off, bytes);
          if (X2) cp_async16_zfill(dst + 1024u * i8 + A_BYTES, xlo + off, bytes);
        }
        cp_async_commit();
        if (++inflight > DEPTH) {
          cp_async_wait<DEPTH>();
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          mbar_arrive(full(ps));
          mbar_arrive(full(ps + 1));
          if ((ps += 2) == stages) ps = 0;
          --inflight;
        }
        if ((s += 2) == stages) { s = 0; ph ^= 1; }
      }
    }
    cp_async_wait<0>();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (ok)
      for (; inflight > 0; --inflight) {
        mbar_arrive(full(ps));
        mbar_arrive(full(ps + 1));
        if ((ps += 2) == stages) ps = 0;
      }
  }
  __syncthreads();
  if (abort_sh) tc_drain_after_abort();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// (s0, s1) += (a0 + b0, a1 + b1) with two packed FP32x2 adds (each lane
// rounded to nearest, as two scalar adds would be).
__device__ __forceinline__ void add2_acc(float& s0, float& s1, float a0, float a1, float b0, float b1) {
  asm("{\n\t.reg .b64 s, a, b;\n\t"
      "mov.b64 s, {%0, %1};\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t"
      "add.rn.f32x2 a, a, b;\n\tadd.rn.f32x2 s, s, a;\n\t"
      "mov.b64 {%0, %1}, s;\n\t}"
      : "+f"(s0), "+f"(s1)
      : "f"(a0), "f"(a1), "f"(b0), "f"(b1));
}

// ------------------------------------------------------------ long-K kernel
// part[y][row*k + r] = sum over the K blocks of split y of A(row, K) W(K, r)
// with W a pre-swizzled hi|lo image (k_tc_wimage):
//   KMAJ  (left contraction)  rows = j < R, K = l < L: A = X^T, K-major tiles
//          (one 64 x 128 box, the same tiles as the factored left kernel);
//   !KMAJ (right contraction) rows = l < L, K = j < R: A = X, MN-major tiles
//          (two 64 x 64 boxes, the same tiles as k_tc_right).
// K blocks go in groups of `group` (tc_long_group); a group is one
// tensor-core accumulation chain in a double-buffered TMEM accumulator,
// drained by four warps into register running sums, so K of any length keeps
// every FP32 chain short.
// Grid (mgroups, nsplit): a CTA owns MT consecutive 128-row tiles; split y
// takes groups y, y + nsplit, ...
constexpr int TCG_GROUP = 2;  // default K blocks per accumulation chain

template <int KP, int MT, bool X2, bool KMAJ>
__global__ void __launch_bounds__(TCF_THREADS, 1)
    k_tc_long(const __grid_constant__ CUtensorMap tm_hi, const __grid_constant__ CUtensorMap tm_lo,
              const uint8_t* __restrict__ wimg, int64_t rows, int64_t K, int k, int stages,
              int group, double* __restrict__ part, int* __restrict__ status) {
  constexpr int NCOL = 2 * KP;
  constexpr uint32_t A_TILE = TC_BM * TC_BK * 2;  // 16 KB
  constexpr uint32_t A_BYTES = MT * A_TILE;
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr uint32_t ACC_COLS = MT * NCOL;
  constexpr int NBUF = 4;  // accumulators in flight (4 * ACC_COLS <= 512 columns)
  constexpr uint32_t TMEM_NEED = NBUF * ACC_COLS;
  constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128
                                 : TMEM_NEED <= 256 ? 256 : 512;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, !KMAJ, false);
  using Acc = float;  // register adds round to nearest: no drift from the many drains

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 2 * NBUF];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t nk = (K + TC_BK - 1) / TC_BK;
  const int64_t ngroups = (nk + group - 1) / group;
  const int64_t ns = gridDim.y;
  const int64_t y = blockIdx.y;
  const int64_t my_groups = y < ngroups ? (ngroups - y + ns - 1) / ns : 0;
  const int row0 = blockIdx.x * MT * TC_BM;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[8 + s]); };
  auto accf = [&](int b) { return smem_u32(&bars[16 + b]); };
  auto acce = [&](int b) { return smem_u32(&bars[16 + NBUF + b]); };

  if (threadIdx.x == 0) {
    abort_sh = 0;
    for (int s = 0; s < stages; ++s) {
      mbar_init(full(s), 1);
      mbar_init(empty(s), 1);
    }
    for (int b = 0; b < NBUF; ++b) {
      mbar_init(accf(b), 1);
      mbar_init(acce(b), 4);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) tmem_alloc(smem_u32(&tmem_base_sh), TMEM_COLS);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  volatile int* abort_flag = &abort_sh;

  if (warp == 0) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int64_t i = 0; i < my_groups && ok; ++i) {
        const int64_t g = y + i * ns;
        const int64_t kb1 = min((g + 1) * group, nk);
        for (int64_t kb = g * group; kb < kb1; ++kb) {
          if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
          const uint32_t st = smem0 + s * STAGE;
          const int kx = (int)(kb * TC_BK);
          mbar_expect_tx(full(s), STAGE);
#pragma unroll
          for (int mt = 0; mt < MT; ++mt) {
            const int r0 = row0 + mt * TC_BM;
            if (KMAJ) {
              tma_load_2d(st + mt * A_TILE, &tm_hi, kx, r0, full(s));
              if (X2) tma_load_2d(st + A_BYTES + mt * A_TILE, &tm_lo, kx, r0, full(s));
            } else {
              tma_load_2d(st + mt * A_TILE, &tm_hi, r0, kx, full(s));
              tma_load_2d(st + mt * A_TILE + A_TILE / 2, &tm_hi, r0 + 64, kx, full(s));
              if (X2) {
                tma_load_2d(st + A_BYTES + mt * A_TILE, &tm_lo, r0, kx, full(s));
                tma_load_2d(st + A_BYTES + mt * A_TILE + A_TILE / 2, &tm_lo, r0 + 64, kx, full(s));
              }
            }
          }
          bulk_load(st + A_STAGE, wimg + (size_t)kb * B_STAGE, B_STAGE, full(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t aph = 0;  // bit b: phase of accumulator b
      bool ok = true;
      for (int64_t i = 0; i < my_groups && ok; ++i) {
        const int buf = (int)(i % NBUF);
        const int64_t g = y + i * ns;
        const int64_t kb0 = g * group, kb1 = min((g + 1) * group, nk);
        if (!mbar_wait(acce(buf), ((aph >> buf) & 1) ^ 1, abort_flag, status)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * ACC_COLS;
        for (int64_t kb = kb0; kb < kb1; ++kb) {
          if (!mbar_wait(full(s), ph, abort_flag, status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem0 + s * STAGE;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk) {
            const uint64_t bdesc = smem_desc(st + A_STAGE + kk * 32, 16, 1024);
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
              // K-major A: +32 B per K = 16; MN-major A: K advances 16 rows =
              // two 1024 B groups, the two 64-row halves 8 KB apart
              const uint32_t a0 = st + mt * A_TILE + (KMAJ ? kk * 32 : kk * 2048);
              const uint64_t adesc = KMAJ ? smem_desc(a0, 16, 1024) : smem_desc(a0, A_TILE / 2, 1024);
              umma_bf16(d + mt * NCOL, adesc, bdesc, IDESC, (kb != kb0 || kk != 0) ? 1u : 0u);
              if (X2) {
                const uint64_t adesc2 = KMAJ ? smem_desc(a0 + A_BYTES, 16, 1024)
                                             : smem_desc(a0 + A_BYTES, A_TILE / 2, 1024);
                umma_bf16(d + mt * NCOL, adesc2, bdesc, IDESC, 1);
              }
            }
          }
          umma_commit(empty(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(accf(buf));
        aph ^= 1u << buf;
      }
    }
  } else {
    // drain warps 2..5: TMEM lane quarter = warp % 4
    const int q4 = warp & 3;
    Acc sum[MT][KP];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int r = 0; r < KP; ++r) sum[mt][r] = 0;
    uint32_t aph = 0;
    bool ok = true;
    for (int64_t i = 0; i < my_groups; ++i) {
      const int buf = (int)(i % NBUF);
      if (!mbar_wait(accf(buf), (aph >> buf) & 1, abort_flag, status)) { ok = false; break; }
      tc_fence_after();
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const uint32_t base = tmem + ((uint32_t)(q4 * 32) << 16) + buf * ACC_COLS + mt * NCOL;
        if (KP == 16) {
          float v[32];
          tmem_ld32(base, v);  // columns 0..15 hi, 16..31 lo
#pragma unroll
          for (int r = 0; r < 16; ++r) sum[mt][r] += v[r] + v[16 + r];
        } else {
#pragma unroll
          for (int cc = 0; cc < KP; cc += 32) {  // hi and lo 32-column slices, one wait
            float vh[32], vl[32];
            tmem_ld32x2(base + cc, base + KP + cc, vh, vl);
#pragma unroll
            for (int e = 0; e < 32; e += 2)
              add2_acc(sum[mt][cc + e], sum[mt][cc + e + 1], vh[e], vh[e + 1], vl[e], vl[e + 1]);
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(buf));
      aph ^= 1u << buf;
    }
    if (ok) {
      double* dst = part + y * rows * k;
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int64_t row = (int64_t)row0 + mt * TC_BM + q4 * 32 + lane;
        if (row < rows) {
#pragma unroll
          for (int r = 0; r < KP; ++r)
            if (r < k) dst[row * k + r] = (double)sum[mt][r];
        }
      }
    }
  }
  __syncthreads();
  if (abort_sh) tc_drain_after_abort();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, TMEM_COLS);
  }
}

// Pre-swizzled hi|lo image of a Khatri-Rao product W(kk, r) = prod_t
// F_t[digit_t(kk), r] (the B operand of k_tc_long), laid out as k_tc_bimage.
// One thread per (k block, r, 16-byte chunk): eight consecutive kk, written
// as one 16-byte store each for hi and lo. Two-mode products with K < 2^31
// (the balanced 4-way tree) take their digits with 32-bit arithmetic.
template <int KP>
__global__ void k_tc_wimage(const WGen wg, int64_t K, int k, int64_t nk, uint8_t* __restrict__ img) {
  constexpr int NCOL = 2 * KP;
  const int64_t total = nk * KP * (TC_BK / 8);
  const bool two32 = wg.nf == 2 && K < ((int64_t)1 << 31);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(e % (TC_BK / 8));
    const int r = (int)((e / (TC_BK / 8)) % KP);
    const int64_t kb = e / ((int64_t)(TC_BK / 8) * KP);
    alignas(16) __nv_bfloat16 hi[8], lo[8];
    // the eight rows' factor values are all loaded before any is converted
    // (one memory latency per thread, not eight)
    double w[8];
    if (wg.nf == 1) {
      const double* f0 = wg.f[0];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t j = kb * TC_BK + ch * 8 + u;
        w[u] = (j < K && r < k) ? f0[j * k + r] : 0.0;
      }
    } else if (two32) {
      const int d0 = (int)wg.dim[0];
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t j = kb * TC_BK + ch * 8 + u;
        const bool in = j < K && r < k;
        const int jj = in ? (int)j : 0;
        const int i1 = jj / d0, i0 = jj - i1 * d0;
        a[u] = in ? wg.f[0][(int64_t)i0 * k + r] : 0.0;
        b[u] = in ? wg.f[1][(int64_t)i1 * k + r] : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) w[u] = a[u] * b[u];
    } else {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int64_t j = kb * TC_BK + ch * 8 + u;
        w[u] = (j < K && r < k) ? wgen_eval(wg, j, r, k) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) split_bf16(w[u], hi[u], lo[u]);
    uint8_t* st = img + (size_t)kb * NCOL * 128;
    *reinterpret_cast<uint4*>(st + sw128_kmajor_off(r, ch * 8)) = *reinterpret_cast<const uint4*>(hi);
    *reinterpret_cast<uint4*>(st + sw128_kmajor_off(KP + r, ch * 8)) = *reinterpret_cast<const uint4*>(lo);
  }
}

// 32-bit mix of a 64-bit counter (the finaliser of the splitmix64 generator,
// Steele, Lea & Flood 2014), the random source of the stochastic rounding.
__device__ __forceinline__ uint32_t sr_hash(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return (uint32_t)((z ^ (z >> 31)) >> 32);
}

// BF16 of a finite float by stochastic rounding: up with probability equal
// to the discarded fraction of an ulp, so E[result] = x. Round-to-nearest is
// biased on data whose density falls across each binade (nonnegative CP
// tensors: about -3e-6 relative in every MTTKRP entry); the stochastic
// errors have mean zero and average out in the long MTTKRP sums. `r` supplies
// the 16 random bits.
__device__ __forceinline__ __nv_bfloat16 bf16_stochastic(float x, uint32_t r) {
  const uint32_t u = __float_as_uint(x);
  if ((u & 0x7f800000u) == 0x7f800000u) return __float2bfloat16(x);  // Inf / NaN
  const uint32_t v = u + (r & 0xffffu);
  if ((v & 0x7f800000u) == 0x7f800000u) return __float2bfloat16(x);  // would overflow
  return __ushort_as_bfloat16((unsigned short)(v >> 16));
}

// Copy of the tensor-core operand with mode n moved last, for the direct
// (non-tree) MTTKRP of mode n as one left contraction. Element (i_0..i_{N-1})
// sits at l + Lpad * j in the source view (l over modes <= s, j over the
// others, lowest mode fastest in each) and goes to l' + Lpad' * i_n, l' over
// the modes other than n in increasing order, lowest fastest (the row order
// of the reference's krp_leave_out_one, common/ncpfactors.hpp:171-233). A
// permutation of the stored BF16 values: the copies hold exactly the numbers
// the tree's copy holds. Rows l' >= L' (padding) are zero.
struct TcPermDesc {
  int64_t dims[kMaxModes];
  int N, n, s;
  int64_t Lpad;         // source row stride
  int64_t Lp, Lppad;    // target rows (numel / I_n) and row stride
};

__global__ void k_tc_permute(const __nv_bfloat16* __restrict__ hi, const __nv_bfloat16* __restrict__ lo,
                             TcPermDesc d, __nv_bfloat16* __restrict__ ohi,
                             __nv_bfloat16* __restrict__ olo) {
  const int64_t total = d.Lppad * d.dims[d.n];
  const __nv_bfloat16 zero = __ushort_as_bfloat16((unsigned short)0);
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t lp = e % d.Lppad, in = e / d.Lppad;
    __nv_bfloat16 vh = zero, vl = zero;
    if (lp < d.Lp) {
      int64_t rem = lp, l = 0, j = 0, sl = 1, sj = 1;
      for (int m = 0; m < d.N; ++m) {
        int64_t im;
        if (m == d.n) {
          im = in;
        } else {
          im = rem % d.dims[m];
          rem /= d.dims[m];
        }
        if (m <= d.s) {
          l += im * sl;
          sl *= d.dims[m];
        } else {
          j += im * sj;
          sj *= d.dims[m];
        }
      }
      const int64_t src = l + d.Lpad * j;
      vh = hi[src];
      if (lo) vl = lo[src];
    }
    ohi[e] = vh;
    if (olo) olo[e] = vl;
  }
}

// The tensor-core copy of the tensor, converted over a range of its elements
// in their natural order (mode 0 fastest): bf16x2 (lo != nullptr) stores the
// BF16 pair hi = RN(x), lo = RN(x - hi); single BF16 rounds RN_f32(x)
// stochastically, seeded by the destination index (deterministic, unbiased:
// round-to-nearest of a nonnegative tensor is biased low). Source element
// e0 + i is src[i]; it lands at l + Lpad * j (l = index % L, j = index / L),
// and the element that ends a column (l = L - 1) also zeroes that column's
// padding rows. The result does not depend on how the tensor is cut into
// ranges.
template <typename T>
__global__ void k_tc_convert_range(const T* __restrict__ src, int64_t e0, int64_t n, int64_t L,
                                   int64_t Lpad, __nv_bfloat16* __restrict__ hi,
                                   __nv_bfloat16* __restrict__ lo) {
  const __nv_bfloat16 zero = __ushort_as_bfloat16((unsigned short)0);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = e0 + i;
    const int64_t l = g % L, j = g / L;
    const int64_t e = l + Lpad * j;
    const double x = (double)src[i];
    if (lo) {
      __nv_bfloat16 h = __double2bfloat16(x);
      hi[e] = h;
      lo[e] = __double2bfloat16(x - (double)__bfloat162float(h));
    } else {
      hi[e] = bf16_stochastic((float)x, sr_hash((uint64_t)e));
    }
    if (l == L - 1)
      for (int64_t pl = L; pl < Lpad; ++pl) {
        hi[pl + Lpad * j] = zero;
        if (lo) lo[pl + Lpad * j] = zero;
      }
  }
}

// Self-test of the bounded-wait path: one thread waits on an mbarrier that no
// one ever arrives on, with a limit of `limit` cycles; the wait runs out, sets
// *status = kStTimeout and the kernel returns normally.
__global__ void k_tc_wait_selftest(long long limit, int* status) {
  __shared__ uint64_t bar;
  __shared__ int abort_sh;
  if (threadIdx.x == 0) {
    abort_sh = 0;
    mbar_init(smem_u32(&bar), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = mbar_wait(smem_u32(&bar), 0, &abort_sh, status, limit);
    if (ok) atomicExch(status, 1);  // cannot happen: nothing arrives
  }
  __syncthreads();
}

// ------------------------------------------------------------ host side
struct TcTensor {
  __nv_bfloat16* hi = nullptr;
  __nv_bfloat16* lo = nullptr;
  int64_t L = 0, R = 0, Lpad = 0;
  int prec = 0;
  CUtensorMap mR_hi, mR_lo, mL_hi, mL_lo;
  uint8_t* bimg = nullptr;   // B image of F_{N-1} (right contraction)
  size_t bimg_bytes = 0;
  uint8_t* bimg0 = nullptr;  // B image of F_0 (factored left contraction)
  size_t bimg0_bytes = 0;
  int kpad = 0;
  int64_t I0 = 0;            // mode-0 size (factored left contraction when I0 % 64 == 0)
  int left_nf = 0;           // factors of the left contraction's Khatri-Rao generator
  int left_parts = 1;        // parts each run of I0 splits into (factored left contraction)
  bool left_cpa = false;     // factored left contraction through cp.async producers when it applies
  uint8_t* wimg = nullptr;   // Khatri-Rao image of the long-K kernel (k_tc_long)
  size_t wimg_bytes = 0;
  int64_t wimg_K = 0;        // longest K it must hold (0: long-K kernel unused)
};

inline int tc_kpad(int k) { return k <= 16 ? 16 : k <= 32 ? 32 : 64; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn tc_encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  }
  return fn;
}

// 2-D BF16 map over (L rows fastest, R columns), row stride Lpad elements.
inline bool tc_make_map(CUtensorMap* m, void* base, int64_t L, int64_t R, int64_t Lpad,
                        uint32_t box0, uint32_t box1) {
  EncodeTiledFn fn = tc_encode_fn();
  if (!fn) return false;
  cuuint64_t gdim[2] = {(cuuint64_t)L, (cuuint64_t)R};
  cuuint64_t gstride[1] = {(cuuint64_t)(Lpad * 2)};
  cuuint32_t box[2] = {box0, box1};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, gdim, gstride, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

inline void tc_free(TcTensor& t) {
  if (t.hi) cudaFree(t.hi);
  if (t.lo) cudaFree(t.lo);
  if (t.bimg) cudaFree(t.bimg);
  if (t.bimg0) cudaFree(t.bimg0);
  if (t.wimg) cudaFree(t.wimg);
  t.hi = t.lo = nullptr;
  t.bimg = t.bimg0 = t.wimg = nullptr;
  t.bimg_bytes = t.bimg0_bytes = t.wimg_bytes = 0;
}

// Factors a view's left-contraction generator takes: the listed modes when
// two or three, else two (F_first against a row of ones, or against the
// image of the other modes' product).
inline int tc_left_gen_nf(int listed) { return (listed == 2 || listed == 3) ? listed : 2; }

// The factored left contraction takes W = F_first x tail with a tail of one
// or two factors.
inline bool tc_left_factored(const TcTensor& t) {
  return t.I0 > 0 && t.I0 % TC_BK == 0 && t.left_nf >= 2 && t.left_nf <= 3;
}
// Parts per run of the factored left contraction's work units: left_parts
// when it divides the run's I0 / 64 chunks, else 1.
inline int tc_left_hp(const TcTensor& t) {
  const int64_t G = t.I0 / TC_BK;
  return (t.left_parts > 1 && G > 0 && G % t.left_parts == 0) ? t.left_parts : 1;
}

// Storage of the BF16 view (L rows, R columns, row stride L rounded up to 8)
// for conversion in ranges (k_tc_convert_range); buffers of the same view and
// precision are kept (with their images).
inline cudaError_t tc_prepare(TcTensor& t, int64_t L, int64_t R, int64_t I0, int prec) {
  const int64_t Lpad = (L + 7) / 8 * 8;
  if (t.hi && t.L == L && t.R == R && t.prec == prec) {
    t.I0 = I0;
    return cudaSuccess;
  }
  tc_free(t);
  t.I0 = I0;
  t.L = L;
  t.R = R;
  t.Lpad = Lpad;
  t.prec = prec;
  const size_t n = (size_t)Lpad * R;
  cudaError_t e = cudaMalloc(&t.hi, n * 2);
  if (e == cudaSuccess && prec == 2) e = cudaMalloc(&t.lo, n * 2);
  return e;
}

// Tensor maps of a prepared view (host-side encodes). False when the driver
// rejects a map.
inline bool tc_make_maps(TcTensor& t) {
  bool ok = tc_make_map(&t.mR_hi, t.hi, t.L, t.R, t.Lpad, 64, 64) &&
            tc_make_map(&t.mL_hi, t.hi, t.L, t.R, t.Lpad, 64, 128);
  if (ok && t.lo)
    ok = tc_make_map(&t.mR_lo, t.lo, t.L, t.R, t.Lpad, 64, 64) &&
         tc_make_map(&t.mL_lo, t.lo, t.L, t.R, t.Lpad, 64, 128);
  else if (ok) {
    t.mR_lo = t.mR_hi;
    t.mL_lo = t.mL_hi;
  }
  return ok;
}


// Direct-MTTKRP copy of mode n (k_tc_permute) from the tree's copy `src`
// whose view splits at s. dst's view: L' = numel / I_n rows, R' = I_n, with
// I0 the size of the fastest remaining mode (the factored left contraction
// applies when it is a multiple of 64). Returns cudaSuccess or an error;
// failed map creation is reported as cudaErrorInvalidValue.
inline cudaError_t tc_direct_copy(TcTensor& dst, const TcTensor& src, const int64_t* dims, int N,
                                  int n, int s, cudaStream_t st) {
  tc_free(dst);
  TcPermDesc d;
  memset(&d, 0, sizeof(d));
  int64_t numel = 1;
  for (int m = 0; m < N; ++m) {
    d.dims[m] = dims[m];
    numel *= dims[m];
  }
  d.N = N;
  d.n = n;
  d.s = s;
  d.Lpad = src.Lpad;
  d.Lp = numel / dims[n];
  d.Lppad = (d.Lp + 7) / 8 * 8;
  dst.L = d.Lp;
  dst.R = dims[n];
  dst.Lpad = d.Lppad;
  dst.prec = src.prec;
  dst.I0 = dims[n == 0 ? 1 : 0];
  dst.left_nf = tc_left_gen_nf(N - 1);
  dst.left_parts = src.left_parts;
  dst.left_cpa = src.left_cpa;
  const size_t cnt = (size_t)d.Lppad * dims[n];
  cudaError_t e = cudaMalloc(&dst.hi, cnt * 2);
  if (e != cudaSuccess) return e;
  if (src.lo) {
    e = cudaMalloc(&dst.lo, cnt * 2);
    if (e != cudaSuccess) return e;
  }
  k_tc_permute<<<4096, 256, 0, st>>>(src.hi, src.lo, d, dst.hi, dst.lo);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  bool ok = tc_make_map(&dst.mR_hi, dst.hi, dst.L, dst.R, dst.Lpad, 64, 64) &&
            tc_make_map(&dst.mL_hi, dst.hi, dst.L, dst.R, dst.Lpad, 64, 128);
  if (ok && dst.lo)
    ok = tc_make_map(&dst.mR_lo, dst.lo, dst.L, dst.R, dst.Lpad, 64, 64) &&
         tc_make_map(&dst.mL_lo, dst.lo, dst.L, dst.R, dst.Lpad, 64, 128);
  else if (ok) {
    dst.mR_lo = dst.mR_hi;
    dst.mL_lo = dst.mL_hi;
  }
  return ok ? cudaSuccess : cudaErrorInvalidValue;
}


// j-tiles per CTA of the left contraction: 2 when R > 128, except at the
// 64-wide rank (keeps the drain warps' running sums in registers)
inline int tc_left_mt(int64_t R, int k) { return (R > 128 && k <= 32) ? 2 : 1; }

// Whether the factored left contraction runs its cp.async instance (one
// 128-row tile a CTA): asked for (left_cpa), rank <= 32 (the drain warps'
// sums within the 10-warp register budget), units of an even number of
// chunks and an even ring of at least 6 stages.
inline bool tc_left_cpa(const TcTensor& t, int k) {
  if (!t.left_cpa || !tc_left_factored(t) || !tcf_cpa_ok(tc_kpad(k), t.prec == 2)) return false;
  return (t.I0 / TC_BK / tc_left_hp(t)) % 2 == 0;
}
// j-tiles per CTA of the contraction tc_left launches for t
inline int tc_left_tiles(const TcTensor& t, int k) { return tc_left_cpa(t, k) ? 1 : tc_left_mt(t.R, k); }

// min_units > 0 caps the split count so that every split takes at least
// that many chunks (runs): fewer, longer splits for small tensors whose
// parallelism comes from elsewhere (a grouped batch)
inline void tc_left_plan(const TcTensor& t, int k, int sm_count, int* mgroups, int* nsplit,
                         int min_units = 0) {
  const int MT = tc_left_tiles(t, k);
  *mgroups = (int)((t.R + MT * TC_BM - 1) / (MT * TC_BM));
  int ns = sm_count / *mgroups;
  if (ns < 1) ns = 1;
  const int64_t units = tc_left_factored(t) ? t.L / t.I0 * tc_left_hp(t) : (t.L + TC_BK - 1) / TC_BK;
  if (ns > units) ns = (int)units;
  if (min_units > 0) {
    const int64_t cap = (units + min_units - 1) / min_units;
    if (ns > cap) ns = (int)(cap < 1 ? 1 : cap);
  }
  *nsplit = ns;
}

inline size_t tc_scratch_elems(const TcTensor& t, int sm_count, int k) {
  if (!t.hi) return 0;
  int mg, ns;
  tc_left_plan(t, k, sm_count, &mg, &ns);
  return (size_t)ns * t.R * k;
}

template <int KP, bool X2>
inline cudaError_t tc_set_attrs() {
  constexpr uint32_t SR = (X2 ? 2 : 1) * TC_BM * TC_BK * 2 + 2 * KP * 128;
  constexpr uint32_t SL1 = (X2 ? 2 : 1) * 1 * TC_BM * TC_BK * 2 + 2 * KP * 128;
  constexpr uint32_t SL2 = (X2 ? 2 : 1) * 2 * TC_BM * TC_BK * 2 + 2 * KP * 128;
  const int smr = (int)(tc_stages(SR) * SR + tc_right_pstage<KP>() + 1024);
  cudaError_t e = cudaFuncSetAttribute(k_tc_right<KP, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smr);
  if (e == cudaSuccess && tc_cpa_depth(SR) >= 2)
    e = cudaFuncSetAttribute(k_tc_right<KP, X2, false, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smr);
  if constexpr (KP <= 32) {  // the multi-TTV instances (rank <= 32)
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_tc_right<KP, X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smr);
    if (e == cudaSuccess && tc_cpa_depth(SR) >= 2)
      e = cudaFuncSetAttribute(k_tc_right<KP, X2, true, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, smr);
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left<KP, 1, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL1) * SL1 + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left<KP, 2, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL2) * SL2 + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left_fac<KP, 1, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL1) * SL1 + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left_fac<KP, 2, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL2) * SL2 + 1024));
  if constexpr (tcf_cpa_ok(KP, X2)) {
    constexpr uint32_t SC = tcf_stage_bytes(KP, 1, X2, 1);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_tc_left_fac<KP, 1, X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(tc_stages(SC) * SC + 1024));
  }
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_long<KP, 1, X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL1) * SL1 + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_long<KP, 1, X2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL1) * SL1 + 1024));
  if constexpr (KP <= 32) {  // two tiles per CTA (tc_long_mt)
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_tc_long<KP, 2, X2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(tc_stages(SL2) * SL2 + 1024));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_tc_long<KP, 2, X2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(tc_stages(SL2) * SL2 + 1024));
  }
  return e;
}

// Allocates the B image for rank k and sets the kernels' shared-memory
// limits (host calls made outside any graph capture).
inline cudaError_t tc_ensure(TcTensor& t, int k) {
  if (!t.hi) return cudaSuccess;
  const int kp = tc_kpad(k);
  const bool x2 = t.prec == 2;
  cudaError_t e = kp == 16 ? (x2 ? tc_set_attrs<16, true>() : tc_set_attrs<16, false>())
                  : kp == 32 ? (x2 ? tc_set_attrs<32, true>() : tc_set_attrs<32, false>())
                             : (x2 ? tc_set_attrs<64, true>() : tc_set_attrs<64, false>());
  if (e != cudaSuccess) return e;
  const int nk = (int)((t.R + TC_BK - 1) / TC_BK);
  size_t need = (size_t)nk * 2 * kp * 128;
  size_t need0 = tc_left_factored(t) ? (size_t)(t.I0 / TC_BK) * 2 * kp * 128 : 0;
  size_t needw = (size_t)((t.wimg_K + TC_BK - 1) / TC_BK) * 2 * kp * 128;
  if (t.bimg && t.bimg_bytes >= need && t.kpad == kp && t.bimg0_bytes >= need0 &&
      t.wimg_bytes >= needw)
    return cudaSuccess;
  if (t.bimg) cudaFree(t.bimg);
  if (t.bimg0) cudaFree(t.bimg0);
  if (t.wimg) cudaFree(t.wimg);
  t.bimg = t.bimg0 = t.wimg = nullptr;
  t.kpad = kp;
  t.bimg_bytes = need;
  t.bimg0_bytes = need0;
  t.wimg_bytes = needw;
  e = cudaMalloc(&t.bimg, need);
  if (e == cudaSuccess && need0) e = cudaMalloc(&t.bimg0, need0);
  if (e == cudaSuccess && needw) e = cudaMalloc(&t.wimg, needw);
  return e;
}

// Builds the pre-swizzled hi|lo B image of F_{N-1} for the right contraction.
inline void tc_right_prep(const TcTensor& t, const double* F, int k, cudaStream_t st) {
  const int nk = (int)((t.R + TC_BK - 1) / TC_BK);
  const int kp = tc_kpad(k);
  const unsigned blocks = (unsigned)std::min<int64_t>(((int64_t)nk * kp * TC_BK + 255) / 256, 1024);
  if (kp == 16)
    k_tc_bimage<16><<<blocks, 256, 0, st>>>(F, t.R, k, nk, t.bimg);
  else if (kp == 32)
    k_tc_bimage<32><<<blocks, 256, 0, st>>>(F, t.R, k, nk, t.bimg);
  else
    k_tc_bimage<64><<<blocks, 256, 0, st>>>(F, t.R, k, nk, t.bimg);
}

// cpa: A tiles through cp.async producer warps (when the stage ring holds at
// least 3 stages) instead of TMA; the same shared-memory image, hence the
// same results.
template <int KP, bool X2>
inline void tc_right_launch(const TcTensor& t, int k, float* P, int* status, int sm_count,
                            cudaStream_t st, bool cpa) {
  constexpr uint32_t STAGE = (X2 ? 2 : 1) * TC_BM * TC_BK * 2 + 2 * KP * 128;
  const int stages = tc_stages(STAGE);
  const size_t smem = (size_t)stages * STAGE + tc_right_pstage<KP>() + 1024;
  const int64_t ntiles = (t.L + TC_BM - 1) / TC_BM;
  const int grid = (int)std::min<int64_t>(ntiles, sm_count);
  if (cpa && tc_cpa_depth(STAGE) >= 2)
    k_tc_right<KP, X2, false, true><<<grid, TC_THREADS + 128, smem, st>>>(
        t.mR_hi, t.mR_lo, t.bimg, t.L, t.R, k, stages, P, status, nullptr, 1, 0, nullptr, t.hi,
        t.lo, t.Lpad);
  else
    k_tc_right<KP, X2><<<grid, TC_THREADS, smem, st>>>(t.mR_hi, t.mR_lo, t.bimg, t.L, t.R, k,
                                                       stages, P, status);
}

// Whether the mode-0 multi-TTV can ride on the right contraction: 3-way
// tree with I0 a multiple of 128 (tiles never straddle an i1), rank <= 32,
// and at least one CTA per i0 block.
inline int tc_right_ttv_tpb(const TcTensor& t, int k, int sm_count) {
  if (k > 32 || t.I0 <= 0 || t.I0 % TC_BM != 0) return 0;
  const int64_t tpb = t.I0 / TC_BM;
  if (tpb > sm_count || t.L % t.I0 != 0) return 0;
  return (int)tpb;
}
// Partials it writes (nsplit x I0 x k), and nsplit.
inline int tc_right_ttv_nsplit(const TcTensor& t, int k, int sm_count) {
  const int tpb = tc_right_ttv_tpb(t, k, sm_count);
  if (!tpb) return 0;
  const int64_t ntiles = (t.L + TC_BM - 1) / TC_BM;
  const int64_t grid = std::min<int64_t>(ntiles, sm_count) / tpb * tpb;
  return (int)(grid / tpb);
}

template <int KP, bool X2>
inline void tc_right_ttv_launch(const TcTensor& t, int k, float* P, const double* F1, double* part,
                                int* status, int sm_count, cudaStream_t st, bool cpa) {
  constexpr uint32_t STAGE = (X2 ? 2 : 1) * TC_BM * TC_BK * 2 + 2 * KP * 128;
  const int stages = tc_stages(STAGE);
  const size_t smem = (size_t)stages * STAGE + tc_right_pstage<KP>() + 1024;
  const int tpb = tc_right_ttv_tpb(t, k, sm_count);
  const int grid = tc_right_ttv_nsplit(t, k, sm_count) * tpb;
  if (cpa && tc_cpa_depth(STAGE) >= 2)
    k_tc_right<KP, X2, true, true><<<grid, TC_THREADS + 128, smem, st>>>(
        t.mR_hi, t.mR_lo, t.bimg, t.L, t.R, k, stages, P, status, F1, tpb, t.I0, part, t.hi, t.lo,
        t.Lpad);
  else
    k_tc_right<KP, X2, true><<<grid, TC_THREADS, smem, st>>>(t.mR_hi, t.mR_lo, t.bimg, t.L, t.R, k,
                                                             stages, P, status, F1, tpb, t.I0, part);
}

// P32 = X * F_{N-1} and the mode-0 multi-TTV partials against F1
// (tc_right_ttv_tpb(...) != 0; call tc_right_prep first). Returns nsplit.
inline int tc_right_ttv(const TcTensor& t, int k, float* P, const double* F1, double* part,
                        int* status, int sm_count, cudaStream_t st, bool cpa = true) {
  const bool x2 = t.prec == 2;
  if (tc_kpad(k) == 16)
    x2 ? tc_right_ttv_launch<16, true>(t, k, P, F1, part, status, sm_count, st, cpa)
       : tc_right_ttv_launch<16, false>(t, k, P, F1, part, status, sm_count, st, cpa);
  else
    x2 ? tc_right_ttv_launch<32, true>(t, k, P, F1, part, status, sm_count, st, cpa)
       : tc_right_ttv_launch<32, false>(t, k, P, F1, part, status, sm_count, st, cpa);
  return tc_right_ttv_nsplit(t, k, sm_count);
}

// P32 = X * F_{N-1} on the tensor cores (call tc_right_prep first).
inline void tc_right(const TcTensor& t, int k, float* P, int* status, int sm_count,
                     cudaStream_t st, bool cpa = true) {
  const bool x2 = t.prec == 2;
  switch (tc_kpad(k)) {
    case 16: x2 ? tc_right_launch<16, true>(t, k, P, status, sm_count, st, cpa)
                : tc_right_launch<16, false>(t, k, P, status, sm_count, st, cpa); break;
    case 32: x2 ? tc_right_launch<32, true>(t, k, P, status, sm_count, st, cpa)
                : tc_right_launch<32, false>(t, k, P, status, sm_count, st, cpa); break;
    default: x2 ? tc_right_launch<64, true>(t, k, P, status, sm_count, st, cpa)
                : tc_right_launch<64, false>(t, k, P, status, sm_count, st, cpa); break;
  }
}

template <int KP, int MT, bool X2>
inline void tc_left_launch(const TcTensor& t, const WGen& wg, int k, double* part, int* status,
                           int sm_count, cudaStream_t st, int* nsplit_out, int min_units) {
  int mg, ns;
  tc_left_plan(t, k, sm_count, &mg, &ns, min_units);
  constexpr uint32_t STAGE = (X2 ? 2 : 1) * MT * TC_BM * TC_BK * 2 + 2 * KP * 128;
  const int stages = tc_stages(STAGE);
  const size_t smem = (size_t)stages * STAGE + 1024;
  if (tc_left_factored(t)) {
    // F_0 image (hi|lo rows, swizzled), then the factored kernel over runs of I_0
    const int nslab = (int)(t.I0 / TC_BK);
    k_tc_bimage<KP><<<(unsigned)std::min<int64_t>(((int64_t)nslab * KP * TC_BK + 255) / 256, 1024),
                      256, 0, st>>>(wg.f[0], t.I0, k, nslab, t.bimg0);
    const double* F2 = wg.nf > 2 ? wg.f[2] : nullptr;
    bool done = false;
    if constexpr (MT == 1 && tcf_cpa_ok(KP, X2)) {
      if (tc_left_cpa(t, k)) {
        constexpr uint32_t SC = tcf_stage_bytes(KP, 1, X2, 1);
        k_tc_left_fac<KP, 1, X2, true><<<dim3(mg, ns), TCF_THREADS + 128, (size_t)tc_stages(SC) * SC + 1024,
                                         st>>>(t.mL_hi, t.mL_lo, t.bimg0, wg.f[1], F2, wg.dim[1], t.I0, t.L,
                                               t.R, k, tc_stages(SC), part, status, tc_left_hp(t), t.hi,
                                               t.lo, t.Lpad);
        done = true;
      }
    }
    if (!done)
      k_tc_left_fac<KP, MT, X2><<<dim3(mg, ns), TCF_THREADS, smem, st>>>(
          t.mL_hi, t.mL_lo, t.bimg0, wg.f[1], F2, wg.dim[1], t.I0, t.L, t.R, k, stages, part, status,
          tc_left_hp(t));
  } else {
    k_tc_left<KP, MT, X2><<<dim3(mg, ns), TCL_THREADS, smem, st>>>(t.mL_hi, t.mL_lo, wg, t.L, t.R, k,
                                                                   stages, part, status);
  }
  *nsplit_out = ns;
}

// Returns the number of split-K partials written to `part`.
inline int tc_left(const TcTensor& t, const WGen& wg, int k, double* part, int* status,
                   int sm_count, cudaStream_t st, int min_units = 0) {
  const bool x2 = t.prec == 2;
  const int MT = tc_left_tiles(t, k);
  int ns = 1;
#define TCL(KP)                                                                                  \
  if (MT == 2) {                                                                                 \
    x2 ? tc_left_launch<KP, 2, true>(t, wg, k, part, status, sm_count, st, &ns, min_units)                  \
       : tc_left_launch<KP, 2, false>(t, wg, k, part, status, sm_count, st, &ns, min_units);                \
  } else {                                                                                       \
    x2 ? tc_left_launch<KP, 1, true>(t, wg, k, part, status, sm_count, st, &ns, min_units)                  \
       : tc_left_launch<KP, 1, false>(t, wg, k, part, status, sm_count, st, &ns, min_units);                \
  }
  switch (tc_kpad(k)) {
    case 16: TCL(16) break;
    case 32: TCL(32) break;
    default: TCL(64) break;
  }
#undef TCL
  return ns;
}

// ---- long-K kernel (k_tc_long): plan, image, launch
// 128-row tiles per CTA: 2 when there are more than one (halves the image's
// share of the shared-memory traffic), except at the 64-wide rank, whose two
// tiles' running sums would not fit the drain warps' registers.
inline int tc_long_mt(int64_t rows, int k) { return (rows > TC_BM && tc_kpad(k) <= 32) ? 2 : 1; }

// K blocks per tensor-core accumulation chain of k_tc_long (environment
// PLANC_GPU_TC_GROUP overrides the default).
inline int tc_long_group() {
  static int g = [] {
    const char* e = getenv("PLANC_GPU_TC_GROUP");
    int v = e ? atoi(e) : TCG_GROUP;
    return v < 1 ? 1 : (v > 1024 ? 1024 : v);
  }();
  return g;
}

inline void tc_long_plan(int64_t rows, int64_t K, int k, int sm_count, int* mgroups, int* nsplit) {
  const int MT = tc_long_mt(rows, k);
  *mgroups = (int)((rows + MT * TC_BM - 1) / (MT * TC_BM));
  int ns = sm_count / *mgroups;
  if (ns < 1) ns = 1;
  const int64_t ngroups = ((K + TC_BK - 1) / TC_BK + tc_long_group() - 1) / tc_long_group();
  if (ns > ngroups) ns = (int)ngroups;
  *nsplit = ns;
}

// Split-K partials the long-K kernel writes for `left` (0 when it writes the
// output directly).
inline size_t tc_long_scratch_elems(const TcTensor& t, bool left, int k, int sm_count) {
  const int64_t rows = left ? t.R : t.L, K = left ? t.L : t.R;
  int mg, ns;
  tc_long_plan(rows, K, k, sm_count, &mg, &ns);
  return ns > 1 ? (size_t)ns * rows * k : 0;
}

// Image of W = KRP over the K index of the left (K = l, rows j) or right
// (K = j, rows l) contraction.
inline void tc_long_prep(const TcTensor& t, bool left, const WGen& wg, int k, cudaStream_t st) {
  const int64_t K = left ? t.L : t.R;
  const int64_t nk = (K + TC_BK - 1) / TC_BK;
  const int kp = tc_kpad(k);
  const unsigned blocks = (unsigned)std::min<int64_t>((nk * kp * (TC_BK / 8) + 255) / 256, 2048);
  if (kp == 16)
    k_tc_wimage<16><<<blocks, 256, 0, st>>>(wg, K, k, nk, t.wimg);
  else if (kp == 32)
    k_tc_wimage<32><<<blocks, 256, 0, st>>>(wg, K, k, nk, t.wimg);
  else
    k_tc_wimage<64><<<blocks, 256, 0, st>>>(wg, K, k, nk, t.wimg);
}

template <int KP, int MT, bool X2, bool KMAJ>
inline void tc_long_launch(const TcTensor& t, int k, int mg, int ns, double* part, int* status,
                           cudaStream_t st) {
  constexpr uint32_t STAGE = (X2 ? 2 : 1) * MT * TC_BM * TC_BK * 2 + 2 * KP * 128;
  const int stages = tc_stages(STAGE);
  const size_t smem = (size_t)stages * STAGE + 1024;
  k_tc_long<KP, MT, X2, KMAJ><<<dim3(mg, ns), TCF_THREADS, smem, st>>>(
      KMAJ ? t.mL_hi : t.mR_hi, KMAJ ? t.mL_lo : t.mR_lo, t.wimg, KMAJ ? t.R : t.L,
      KMAJ ? t.L : t.R, k, stages, tc_long_group(), part, status);
}

// Left (out = X^T W, R x k) or right (out = X W, L x k) contraction against
// the image built by tc_long_prep. Writes `out` directly and returns 1, or
// writes that many split-K partials to `part` (R or L x k each).
inline int tc_long(const TcTensor& t, bool left, int k, double* out, double* part, int* status,
                   int sm_count, cudaStream_t st) {
  const int64_t rows = left ? t.R : t.L, K = left ? t.L : t.R;
  int mg, ns;
  tc_long_plan(rows, K, k, sm_count, &mg, &ns);
  double* dst = ns > 1 ? part : out;
  const bool x2 = t.prec == 2;
  const int MT = tc_long_mt(rows, k);
#define TCG(KP, M)                                                                           \
  if (left)                                                                                  \
    x2 ? tc_long_launch<KP, M, true, true>(t, k, mg, ns, dst, status, st)                    \
       : tc_long_launch<KP, M, false, true>(t, k, mg, ns, dst, status, st);                  \
  else                                                                                       \
    x2 ? tc_long_launch<KP, M, true, false>(t, k, mg, ns, dst, status, st)                   \
       : tc_long_launch<KP, M, false, false>(t, k, mg, ns, dst, status, st);
  switch (tc_kpad(k)) {
    case 16: if (MT == 2) { TCG(16, 2) } else { TCG(16, 1) } break;
    case 32: if (MT == 2) { TCG(32, 2) } else { TCG(32, 1) } break;
    default: TCG(64, 1) break;
  }
#undef TCG
  return ns;
}

}  // namespace pg
