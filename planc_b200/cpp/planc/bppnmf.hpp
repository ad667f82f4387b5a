// bppnmf.hpp -- planc::BPPNMF (reference nmf/bppnmf.hpp:18-259): ANLS NMF
// with block principal pivoting, W then H per iteration, each row an NNLS
// problem (all rows of a factor in one batched BPP launch on the device),
// with the symmetric regularisation when symm_reg > 0 and normalize_by_W
// after the last iteration.
#pragma once
#include "nmf.hpp"

namespace planc {

template <class T>
class BPPNMF : public NMF<T> {
 public:
  BPPNMF(const T& A, int lowrank) : NMF<T>(A, lowrank) { this->m_updalgo = ANLSBPP; }
  BPPNMF(const T& A, const MAT& llf, const MAT& rlf) : NMF<T>(A, llf, rlf) {
    this->m_updalgo = ANLSBPP;
  }
  void computeNMF() { this->run_on_device(PLANC_GPU_ANLSBPP); }
  double getObjectiveError() { return this->objective_err; }
};

}  // namespace planc
