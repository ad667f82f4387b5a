// tc_group.cuh -- grouped tensor-core partial MTTKRPs for a batch of small
// tensors: ONE persistent launch works through the tiles of every member.
//
// A member's own contraction kernel (k_tc_right / k_tc_left) on a tensor of a
// few MB pays its set-up (mbarrier and TMEM allocation, pipeline fill and
// drain, the Khatri-Rao producers' first tiles) for 1-3 units of work per
// CTA. The grouped kernels below keep one pipeline running across members:
// a CTA takes work items it, it + gridDim.x, ... of a list that covers every
// member, the TMA producer, the MMA issuer and the drain warps walk the same
// list, and the stage / accumulator phases carry over from item to item.
// Each member's tensor maps live in a device table (four per member: right
// hi, right lo, left hi, left lo), written by the host before the first
// launch and never modified on the device.
//
// Work items are exactly the CTAs of the member's own launch (a 128-row tile
// of the right contraction; a (row group, split) pair of the left one, with
// the member's own split count), and each item runs the code of that CTA, so
// a grouped run computes the same bits as the members' own launches.
#pragma once
#include "tc_mttkrp.cuh"

namespace pg {

// Orders the tensor-map reads of the TMA unit after the descriptor's
// contents (written to global memory before the launch).
__device__ __forceinline__ void tmap_acquire(const CUtensorMap* m) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((uint64_t)m) : "memory");
}

// right contraction of one member: P[l*k + r] = sum_j X[l, j] F[j, r]
struct TcgRight {
  const uint8_t* bimg;  // the member's B image of F_{N-1} (k_tc_bimage layout)
  float* P;
  int64_t L, R;
  int k;
  int pad;
};

template <int KP, bool X2>
__global__ void __launch_bounds__(TC_THREADS, 1)
    k_tc_right_grp(const CUtensorMap* __restrict__ maps, const TcgRight* __restrict__ mem,
                   const int2* __restrict__ items, int nitems, int stages, int* __restrict__ status) {
  constexpr int NCOL = 2 * KP;
  constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2;
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr int NBUF = 4;
  constexpr uint32_t TMEM_COLS = NBUF * NCOL < 32 ? 32 : NBUF * NCOL;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, true, false);

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 2 * NBUF];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
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
      for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        const int2 w = items[it];
        const TcgRight& m = mem[w.x];
        const CUtensorMap* mh = maps + 4 * w.x;
        tmap_acquire(mh);
        if (X2) tmap_acquire(mh + 1);
        const int l0 = w.y * TC_BM;
        const int nk = (int)((m.R + TC_BK - 1) / TC_BK);
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
          const uint32_t st = smem0 + s * STAGE;
          mbar_expect_tx(full(s), STAGE);
          tma_load_2d(st, mh, l0, kb * TC_BK, full(s));
          tma_load_2d(st + A_BYTES / 2, mh, l0 + 64, kb * TC_BK, full(s));
          if (X2) {
            tma_load_2d(st + A_BYTES, mh + 1, l0, kb * TC_BK, full(s));
            tma_load_2d(st + A_BYTES + A_BYTES / 2, mh + 1, l0 + 64, kb * TC_BK, full(s));
          }
          bulk_load(st + A_STAGE, m.bimg + (size_t)kb * B_STAGE, B_STAGE, full(s));
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
      for (int it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
        const int2 w = items[it];
        const int nk = (int)((mem[w.x].R + TC_BK - 1) / TC_BK);
        if (!mbar_wait(acce(buf), ((aph >> buf) & 1) ^ 1, abort_flag, status)) break;
        tc_fence_after();
        const uint32_t d = tmem + buf * NCOL;
        for (int kb = 0; kb < nk; ++kb) {
          if (!mbar_wait(full(s), ph, abort_flag, status)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem0 + s * STAGE;
#pragma unroll
          for (int kk = 0; kk < TC_BK / 16; ++kk) {
            const uint64_t bdesc = smem_desc(st + A_STAGE + kk * 32, 16, 1024);
            const uint64_t adesc = smem_desc(st + kk * 2048, A_BYTES / 2, 1024);
            umma_bf16(d, adesc, bdesc, IDESC, (kb | kk) != 0);
            if (X2) {
              const uint64_t adesc2 = smem_desc(st + A_BYTES + kk * 2048, A_BYTES / 2, 1024);
              umma_bf16(d, adesc2, bdesc, IDESC, 1);
            }
          }
          umma_commit(empty(s));
          if (++s == stages) { s = 0; ph ^= 1; }
        }
        if (!ok) break;
        umma_commit(accf(buf));
        aph ^= 1u << buf;
        buf = (buf + 1) % NBUF;
      }
    }
  } else {
    // epilogue warps 2..5: TMEM lane quarter = warp % 4
    const int q = warp & 3;
    int buf = 0;
    uint32_t aph = 0;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
      const int2 w = items[it];
      const TcgRight& m = mem[w.x];
      if (!mbar_wait(accf(buf), (aph >> buf) & 1, abort_flag, status)) break;
      tc_fence_after();
      const int64_t row = (int64_t)w.y * TC_BM + q * 32 + lane;
      float v[NCOL];
#pragma unroll
      for (int c = 0; c < NCOL; c += 32)
        tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * NCOL + c, v + c);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(buf));
      aph ^= 1u << buf;
      buf = (buf + 1) % NBUF;
      if (row < m.L) {
        const int k = m.k;
        float* dst = m.P + row * k;
        if (k == KP && (KP % 4) == 0) {
#pragma unroll
          for (int r = 0; r < KP; r += 4) {
            float4 o = make_float4(v[r] + v[KP + r], v[r + 1] + v[KP + r + 1],
                                   v[r + 2] + v[KP + r + 2], v[r + 3] + v[KP + r + 3]);
            *reinterpret_cast<float4*>(dst + r) = o;
          }
        } else {
#pragma unroll
          for (int r = 0; r < KP; ++r)
            if (r < k) dst[r] = v[r] + v[KP + r];
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

// left contraction of one member (generic Khatri-Rao producers):
// part[y][j*k + r] = sum_{l in split y} X[l, j] W(l, r)
struct TcgLeft {
  WGen wg;       // Khatri-Rao generator of modes 0..s (2 or 3 factors)
  double* part;  // the member's split-K partials
  int64_t L, R;
  int k;
  int nsplit;    // the member's own split count
};
struct TcgUnit {
  int member, jg, y, pad;  // row group and split of one CTA of the member's launch
};

template <int KP, int MT, bool X2>
__global__ void __launch_bounds__(TCL_THREADS, 1)
    k_tc_left_grp(const CUtensorMap* __restrict__ maps, const TcgLeft* __restrict__ mem,
                  const TcgUnit* __restrict__ units, int nunits, int stages, int* __restrict__ status) {
  constexpr int NCOL = 2 * KP;
  constexpr uint32_t A_TILE = TC_BM * TC_BK * 2;
  constexpr uint32_t A_BYTES = MT * A_TILE;
  constexpr uint32_t A_STAGE = X2 ? 2 * A_BYTES : A_BYTES;
  constexpr uint32_t B_STAGE = NCOL * 128;
  constexpr uint32_t STAGE = A_STAGE + B_STAGE;
  constexpr uint32_t ACC_COLS = MT * NCOL;
  constexpr uint32_t TMEM_NEED = 2 * ACC_COLS;
  constexpr uint32_t TMEM_COLS = TMEM_NEED <= 32 ? 32 : TMEM_NEED <= 64 ? 64 : TMEM_NEED <= 128 ? 128
                                 : TMEM_NEED <= 256 ? 256 : 512;
  constexpr uint32_t IDESC = idesc_bf16(NCOL, false, false);
  using Acc = typename std::conditional<(MT * KP <= 64), double, float>::type;

  extern __shared__ uint8_t smem_raw[];
  __shared__ uint64_t bars[2 * 8 + 4];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int abort_sh;
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const uint32_t smem0 = smem_u32(smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto full = [&](int s) { return smem_u32(&bars[s]); };
  auto empty = [&](int s) { return smem_u32(&bars[8 + s]); };
  auto accf = [&](int b) { return smem_u32(&bars[16 + b]); };
  auto acce = [&](int b) { return smem_u32(&bars[18 + b]); };
  // chunks of a unit: split y of the member takes chunks y, y + nsplit, ...
  auto unit_chunks = [&](const TcgLeft& m, int y) -> int64_t {
    const int64_t nchunks = (m.L + TC_BK - 1) / TC_BK;
    return y < nchunks ? (nchunks - y + m.nsplit - 1) / m.nsplit : 0;
  };

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
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const TcgUnit U = units[u];
        const TcgLeft& m = mem[U.member];
        const CUtensorMap* mh = maps + 4 * U.member + 2;
        tmap_acquire(mh);
        if (X2) tmap_acquire(mh + 1);
        const int64_t my_chunks = unit_chunks(m, U.y);
        const int j0 = U.jg * MT * TC_BM;
        for (int64_t i = 0; i < my_chunks; ++i) {
          const int64_t c = U.y + i * m.nsplit;
          if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
          const uint32_t st = smem0 + s * STAGE;
          mbar_expect_tx(full(s), A_STAGE);
          for (int mt = 0; mt < MT; ++mt) {
            tma_load_2d(st + mt * A_TILE, mh, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
            if (X2) tma_load_2d(st + A_BYTES + mt * A_TILE, mh + 1, (int)(c * TC_BK), j0 + mt * TC_BM, full(s));
          }
          if (++s == stages) { s = 0; ph ^= 1; }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      uint32_t aph[2] = {0, 0};
      int64_t gcount = 0;  // accumulator groups issued so far (all units)
      bool ok = true;
      for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
        const TcgUnit U = units[u];
        const int64_t my_chunks = unit_chunks(mem[U.member], U.y);
        const int64_t ngroups = (my_chunks + TCL_GROUP - 1) / TCL_GROUP;
        int64_t i = 0;
        for (int64_t g = 0; g < ngroups && ok; ++g, ++gcount) {
          const int buf = (int)(gcount & 1);
          if (!mbar_wait(acce(buf), aph[buf] ^ 1, abort_flag, status)) { ok = false; break; }
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
    }
  } else if (warp < 6) {
    // producer warps 2..5: the Khatri-Rao B tile of every chunk (as k_tc_left)
    constexpr int OCT_LANES = 128 / KP;
    constexpr int OCT_PER = 8 / OCT_LANES;
    const int pt = threadIdx.x - 64;
    const int r = pt % KP;
    const int oct0 = pt / KP;
    int s = 0;
    uint32_t ph = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
      const TcgUnit U = units[u];
      const TcgLeft& m = mem[U.member];
      const int k = m.k;
      const bool rok = r < k;
      const int nf = m.wg.nf;
      const double* F0 = m.wg.f[0];
      const double* F1 = m.wg.f[1];
      const double* F2 = nf > 2 ? m.wg.f[2] : m.wg.f[1];
      const int64_t D0 = m.wg.dim[0], D1 = m.wg.dim[1];
      const int64_t L = m.L;
      const int64_t ns = m.nsplit;
      const int64_t my_chunks = unit_chunks(m, U.y);
      int64_t b0, b1, b2;
      {
        const int64_t l0 = (int64_t)U.y * TC_BK;
        b0 = l0 % D0;
        b1 = (l0 / D0) % D1;
        b2 = nf > 2 ? l0 / (D0 * D1) : 0;
      }
      const int64_t step = TC_BK * ns;
      for (int64_t i = 0; i < my_chunks; ++i) {
        const int64_t c = U.y + i * ns;
        if (!mbar_wait(empty(s), ph ^ 1, abort_flag, status)) { ok = false; break; }
        uint8_t* bt = smem + s * STAGE + A_STAGE;
#pragma unroll
        for (int t = 0; t < OCT_PER; ++t) {
          const int j = oct0 + OCT_LANES * t;
          int64_t d0 = b0 + 8 * j, d1 = b1, d2 = b2;
          while (d0 >= D0) { d0 -= D0; ++d1; }
          if (nf > 2) while (d1 >= D1) { d1 -= D1; ++d2; }
          const int64_t lbase = c * TC_BK + 8 * j;
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
            for (int uu = 0; uu < 2; ++uu) {
              w[uu] = 0.f;
              if (rok && lbase + e + uu < L) w[uu] = (float)F0[d0 * k + r] * tail;
              if (++d0 == D0) {
                d0 = 0;
                if (++d1 == D1 && nf > 2) { d1 = 0; ++d2; }
                if (rok && lbase + e + uu + 1 < L) tail = tail_of(d1, d2);
              }
            }
            __nv_bfloat162 h2 = __floats2bfloat162_rn(w[0], w[1]);
            float2 hf = __bfloat1622float2(h2);
            __nv_bfloat162 l2 = __floats2bfloat162_rn(w[0] - hf.x, w[1] - hf.y);
            hw[e >> 1] = *reinterpret_cast<uint32_t*>(&h2);
            lw[e >> 1] = *reinterpret_cast<uint32_t*>(&l2);
          }
          *reinterpret_cast<uint4*>(bt + sw128_kmajor_off(r, 8 * j)) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
          *reinterpret_cast<uint4*>(bt + sw128_kmajor_off(KP + r, 8 * j)) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
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
    }
  } else {
    // drain warps 6..9: TMEM lane quarter = warp % 4
    const int q = warp & 3;
    uint32_t aph[2] = {0, 0};
    int64_t gcount = 0;
    bool ok = true;
    for (int u = blockIdx.x; u < nunits && ok; u += gridDim.x) {
      const TcgUnit U = units[u];
      const TcgLeft& m = mem[U.member];
      const int64_t my_chunks = unit_chunks(m, U.y);
      const int64_t ngroups = (my_chunks + TCL_GROUP - 1) / TCL_GROUP;
      Acc sum[MT][KP];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int r = 0; r < KP; ++r) sum[mt][r] = 0;
      for (int64_t g = 0; g < ngroups; ++g, ++gcount) {
        const int buf = (int)(gcount & 1);
        if (!mbar_wait(accf(buf), aph[buf], abort_flag, status)) { ok = false; break; }
        tc_fence_after();
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
#pragma unroll
          for (int cc = 0; cc < NCOL; cc += 32) {
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + buf * ACC_COLS + mt * NCOL + cc, v);
#pragma unroll
            for (int i = 0; i < 32; ++i) sum[mt][(cc + i) % KP] += (Acc)v[i];
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(acce(buf));
        aph[buf] ^= 1;
      }
      if (!ok) break;
      const int k = m.k;
      double* dst = m.part + (int64_t)U.y * m.R * k;
      const int j0 = U.jg * MT * TC_BM;
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int64_t j = (int64_t)j0 + mt * TC_BM + q * 32 + lane;
        if (j < m.R) {
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

// B images of the right contractions of many members (k_tc_bimage)
struct TcgBimg {
  const double* F;
  int64_t R;
  int k, nk;
  uint8_t* img;
  unsigned gx;  // the member's own grid
};

template <int KP>
__global__ void k_tc_bimage_grp(const TcgBimg* __restrict__ a) {
  const TcgBimg& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx) return;
  tc_bimage_body<KP>(g.F, g.R, g.k, g.nk, g.img, blockIdx.x, g.gx);
}

// dynamic shared-memory limits of the grouped contractions (host, outside capture)
template <int KP, bool X2>
inline cudaError_t tcg_set_attrs() {
  constexpr uint32_t SR = (X2 ? 2 : 1) * TC_BM * TC_BK * 2 + 2 * KP * 128;
  constexpr uint32_t SL1 = (X2 ? 2 : 1) * 1 * TC_BM * TC_BK * 2 + 2 * KP * 128;
  constexpr uint32_t SL2 = (X2 ? 2 : 1) * 2 * TC_BM * TC_BK * 2 + 2 * KP * 128;
  cudaError_t e = cudaFuncSetAttribute(k_tc_right_grp<KP, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(tc_stages(SR) * SR + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left_grp<KP, 1, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL1) * SL1 + 1024));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_tc_left_grp<KP, 2, X2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(tc_stages(SL2) * SL2 + 1024));
  return e;
}

}  // namespace pg
