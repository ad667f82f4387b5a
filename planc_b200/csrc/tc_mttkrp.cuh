// tc_mttkrp.cuh -- tensor-core (tcgen05 / TMEM / TMA) partial MTTKRP for the
// BF16 precisions. (placeholder: filled in by the sm_100a kernels)
#pragma once
#include "common.cuh"

namespace pg {

struct TcTensor {
  void* hi = nullptr;
  void* lo = nullptr;
  int64_t L = 0, R = 0, Lpad = 0;
  int prec = 0;
};

inline size_t tc_scratch_elems(const TcTensor&, int, int) { return 0; }
inline void tc_free(TcTensor& t) {
  if (t.hi) cudaFree(t.hi);
  if (t.lo) cudaFree(t.lo);
  t.hi = t.lo = nullptr;
}
inline void tc_set_tensor(TcTensor&, const void*, bool, int64_t, int64_t, int, cudaStream_t) {}
inline void tc_right(const TcTensor&, const double*, int, float*, cudaStream_t) {}
inline int tc_left(const TcTensor&, const WGen&, int, double*, int, cudaStream_t) { return 1; }

}  // namespace pg
