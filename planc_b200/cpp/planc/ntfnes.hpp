// ntfnes.hpp -- planc::NTFNES (reference ntf/ntfnes.hpp:11-197), the
// Nesterov-accelerated NTF. The update (eigenvalue bounds of G, the
// accelerated proximal-gradient loop) and the outer extrapolation with its
// accept / reject test both run on the device inside computeNTF; the
// proximal, previous and extrapolated iterates and the acceleration counters
// (acc_start 5, acc_exp 3, fail_limit 5) live in the device context for the
// lifetime of the solver object. As in the reference the constructor switches
// acceleration, and with it the error evaluation, on.
#pragma once
#include "auntf.hpp"

namespace planc {

class NTFNES : public AUNTF {
 protected:
  // The update exists on the device only; computeNTF never calls this.
  MAT update(const int mode) override {
    ERR << "NTFNES::update(" << mode << ") runs on the device inside computeNTF" << std::endl;
    exit(EXIT_FAILURE);
  }
  int device_algo() const override { return PLANC_GPU_NESTEROV; }

 public:
  NTFNES(const Tensor& i_tensor, const int i_k, algotype i_algo) : AUNTF(i_tensor, i_k, i_algo) {
    this->accelerated(true);  // ntfnes.hpp:193
  }
};

}  // namespace planc
