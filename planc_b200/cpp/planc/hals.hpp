// hals.hpp -- planc::HALSNMF (reference nmf/hals.hpp:10-114): HALS NMF. The
// constructors normalise by W as the reference's do; computeNMF runs the
// iterations on the device (H sweep, then the column-normalised W sweep and
// normalize_by_W, then the objective) and prints the objective lines.
#pragma once
#include "nmf.hpp"

namespace planc {

template <class T>
class HALSNMF : public NMF<T> {
 public:
  HALSNMF(const T& A, int lowrank) : NMF<T>(A, lowrank) {
    this->m_updalgo = HALS;
    this->normalize_by_W();
  }
  HALSNMF(const T& A, const MAT& llf, const MAT& rlf) : NMF<T>(A, llf, rlf) {
    this->m_updalgo = HALS;
    this->normalize_by_W();
  }
  void computeNMF() { this->run_on_device(PLANC_GPU_HALS); }
};

}  // namespace planc
