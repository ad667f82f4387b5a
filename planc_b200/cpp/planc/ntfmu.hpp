// ntfmu.hpp -- planc::NTFMU (reference ntf/ntfmu.hpp:11-16). The device runs
// the update (k_mu_rows); update() is the host form of the same rule.
#pragma once
#include "auntf.hpp"

namespace planc {

class NTFMU : public AUNTF {
 protected:
  MAT update(const int mode) override {
    MAT H(this->m_ncp_factors.factor(mode));
    const MAT& Mt = this->ncp_mttkrp_t[mode];
    const MAT& G = this->gram_without_one;
    MAT out(H.n_rows, H.n_cols);
    for (UWORD r = 0; r < H.n_rows; ++r)
      for (UWORD c = 0; c < H.n_cols; ++c) {
        double t = 0;
        for (UWORD j = 0; j < H.n_cols; ++j) t += H(r, j) * G(j, c);
        out(r, c) = (H(r, c) * Mt(c, r)) / (t + EPSILON);
      }
    return out.t();
  }
  int device_algo() const override { return PLANC_GPU_MU; }

 public:
  NTFMU(const Tensor& i_tensor, const int i_k, algotype i_algo) : AUNTF(i_tensor, i_k, i_algo) {}
};

}  // namespace planc
