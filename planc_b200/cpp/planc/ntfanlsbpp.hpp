// ntfanlsbpp.hpp -- planc::NTFANLSBPP (reference ntf/ntfanlsbpp.hpp:15-57).
// The device solves every row's NNLS in one batched BPP launch (k_bpp);
// update() is the host-path form, which hands the same normal equations to
// planc_gpu_bpp_solve (BPPNNLS<MAT,VEC>(G, M, true), nnls/bppnnls.hpp).
#pragma once
#include "auntf.hpp"

namespace planc {

class NTFANLSBPP : public AUNTF {
 protected:
  MAT update(const int mode) override {
    const MAT& Mt = this->ncp_mttkrp_t[mode];  // k x I (column-major RHS)
    MAT X(Mt.n_rows, Mt.n_cols);
    int rc = planc_gpu_bpp_solve(this->gpu_context(), this->gram_without_one.memptr(), Mt.memptr(),
                                 (int)Mt.n_rows, (int64_t)Mt.n_cols, X.memptr(), nullptr, nullptr);
    if (rc != PLANC_GPU_OK) {
      ERR << "BPP failed: " << planc_gpu_last_error() << std::endl;
      exit(EXIT_FAILURE);
    }
    return X;  // k x I
  }
  int device_algo() const override { return PLANC_GPU_ANLSBPP; }

 public:
  NTFANLSBPP(const Tensor& i_tensor, const int i_k, algotype i_algo)
      : AUNTF(i_tensor, i_k, i_algo) {}
};

}  // namespace planc
