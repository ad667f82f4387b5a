// ntfaoadmm.hpp -- planc::NTFAOADMM (reference ntf/ntfaoadmm.hpp:13-96).
// The update runs on the device (k_admm_prep / k_admm_step: Cholesky of
// G + alpha I, at most 5 ADMM iterations with the reference's stopping test,
// tolerance 0.01); the dual variables m_ncp_aux live in the device context
// for the lifetime of the solver object, zero at construction.
#pragma once
#include "auntf.hpp"

namespace planc {

class NTFAOADMM : public AUNTF {
 protected:
  // The update exists on the device only; computeNTF never calls this.
  MAT update(const int mode) override {
    ERR << "NTFAOADMM::update(" << mode << ") runs on the device inside computeNTF" << std::endl;
    exit(EXIT_FAILURE);
  }
  int device_algo() const override { return PLANC_GPU_AOADMM; }

 public:
  NTFAOADMM(const Tensor& i_tensor, const int i_k, algotype i_algo)
      : AUNTF(i_tensor, i_k, i_algo) {}
};

}  // namespace planc
