// ntfhals.hpp -- planc::NTFHALS (reference ntf/ntfhals.hpp:13-29). The device
// runs the update (k_hals_rows); update() is the same sweep on the host, used
// when a subclass chooses the host path.
#pragma once
#include "auntf.hpp"

namespace planc {

class NTFHALS : public AUNTF {
 protected:
  MAT update(const int mode) override {
    MAT H(this->m_ncp_factors.factor(mode));
    const MAT& Mt = this->ncp_mttkrp_t[mode];  // k x I
    const MAT& G = this->gram_without_one;
    for (UWORD i = 0; i < H.n_cols; i++) {
      std::vector<double> u(H.n_rows);
      for (UWORD r = 0; r < H.n_rows; ++r) {
        double hg = 0;
        for (UWORD j = 0; j < H.n_cols; ++j) hg += H(r, j) * G(j, i);
        double v = H(r, i) + (Mt(i, r) - hg);
        u[r] = v < EPSILON_1EMINUS16 ? EPSILON_1EMINUS16 : v;
      }
      double nrm2 = 0;
      for (double x : u) nrm2 += x * x;
      if (nrm2 > 0)
        for (UWORD r = 0; r < H.n_rows; ++r) H(r, i) = u[r];
    }
    return H.t();
  }
  int device_algo() const override { return PLANC_GPU_HALS; }

 public:
  NTFHALS(const Tensor& i_tensor, const int i_k, algotype i_algo) : AUNTF(i_tensor, i_k, i_algo) {}
};

}  // namespace planc
