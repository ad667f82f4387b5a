// common.cuh -- shared definitions of the planc_gpu CUDA library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pg {

// Maximum number of tensor modes and maximum rank handled by the kernels.
constexpr int kMaxModes = 8;
constexpr int kMaxRank = 64;

// common/utils.h:46-49 of the reference.
constexpr double kEps17 = 0.00000000000000001;  // EPSILON_1EMINUS16 (1e-17)
constexpr double kEps6 = 0.000001;               // EPSILON
constexpr double kEps12 = 1e-12;                 // EPSILON_1EMINUS12

// Kernel classes for the optional event timing (planc_gpu_set_timing).
enum KClass { KC_CONTRACT = 0, KC_TTV = 1, KC_UPDATE = 2, KC_NORMGRAM = 3,
              KC_ERROR = 4, KC_REDUCE = 5, KC_BPP = 6, KC_PREP = 7, KC_CONTRACT_LEFT = 8,
              KC_COUNT = 9 };

// Device status codes written by kernels (match planc_gpu.h).
constexpr int kStBppMaxIter = -4;
constexpr int kStNonFinite = -5;
constexpr int kStTimeout = -6;
constexpr int kStSingular = -9;

// Product of factor rows over a list of modes:
//   W(kk, r) = prod_t F_t[(kk / stride_t) % dim_t, r]
// i.e. one row of the reverse Khatri-Rao product with the lowest listed mode
// fastest (common/ncpfactors.hpp:171-233, dimtree/ddttensor.hpp:993-1060).
// Factors are row-major I x k. The product is evaluated from the last listed
// factor down, F_0 * (F_1 * (F_2 ...)), the order of both reference KRPs.
struct WGen {
  const double* f[kMaxModes];
  int64_t dim[kMaxModes];
  int64_t stride[kMaxModes];
  int nf;
};

__device__ __forceinline__ double wgen_eval(const WGen& g, int64_t kk, int r, int k) {
  if (g.nf == 1) return g.f[0][kk * k + r];  // single factor, stride 1
  double w = 1.0;
  for (int t = g.nf - 1; t >= 0; --t) {
    int64_t i = (kk / g.stride[t]) % g.dim[t];
    w = g.f[t][i * k + r] * w;
  }
  return w;
}

// Mixed-radix digits of a Khatri-Rao row index over a WGen's modes, advanced
// incrementally (no division in the steady state).
struct WIdx {
  int64_t i[kMaxModes];
};

__device__ __forceinline__ void widx_init(const WGen& g, int64_t kk, WIdx& w) {
  for (int t = 0; t < g.nf; ++t) w.i[t] = (kk / g.stride[t]) % g.dim[t];
}

__device__ __forceinline__ void widx_advance(const WGen& g, WIdx& w, int64_t step) {
  int64_t carry = step;
  for (int t = 0; t < g.nf && carry; ++t) {
    int64_t v = w.i[t] + carry;
    if (t + 1 < g.nf) {
      if (v < g.dim[t]) {
        carry = 0;
      } else if (v < 2 * g.dim[t]) {
        carry = 1;
        v -= g.dim[t];
      } else {
        carry = v / g.dim[t];
        v -= carry * g.dim[t];
      }
    } else {
      carry = 0;  // the last digit may run past its range (row beyond the end)
    }
    w.i[t] = v;
  }
}

// W(row, r) for the row whose digits are w (same product order as wgen_eval).
__device__ __forceinline__ double wgen_row(const WGen& g, const WIdx& w, int r, int k) {
  double v = 1.0;
  for (int t = g.nf - 1; t >= 0; --t) v = g.f[t][w.i[t] * k + r] * v;
  return v;
}

}  // namespace pg
