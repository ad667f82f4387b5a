// mu.hpp -- planc::MUNMF (reference nmf/mu.hpp:10-97): multiplicative-update
// NMF, H = H .* (A^T W) ./ (H W^T W + eps), W likewise, normalize_by_W after
// the last iteration; the iterations run on the device.
#pragma once
#include "nmf.hpp"

namespace planc {

template <class T>
class MUNMF : public NMF<T> {
 public:
  MUNMF(const T& A, int lowrank) : NMF<T>(A, lowrank) { this->m_updalgo = MU; }
  MUNMF(const T& A, const MAT& llf, const MAT& rlf) : NMF<T>(A, llf, rlf) { this->m_updalgo = MU; }
  void computeNMF() { this->run_on_device(PLANC_GPU_MU); }
};

}  // namespace planc
