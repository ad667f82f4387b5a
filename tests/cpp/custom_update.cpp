// A user-defined AUNTF subclass with its own host-side update(), the
// reference's extension point (ntf/auntf.hpp:45): it runs between the
// device's Gram/MTTKRP and normalisation steps. The update is the HALS rule
// written against the protected members the reference exposes
// (m_ncp_factors, ncp_mttkrp_t, gram_without_one).
//   custom_update <I0> <I1> <I2> <k> <iters> <init prefix> <out prefix>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "planc/auntf.hpp"

class MyHALS : public planc::AUNTF {
 protected:
  MAT update(const int mode) override {
    MAT H(this->m_ncp_factors.factor(mode));
    const MAT& Mt = this->ncp_mttkrp_t[mode];
    const MAT& G = this->gram_without_one;
    for (UWORD i = 0; i < H.n_cols; i++) {
      std::vector<double> u(H.n_rows);
      for (UWORD r = 0; r < H.n_rows; ++r) {
        double hg = 0;
        for (UWORD j = 0; j < H.n_cols; ++j) hg += H(r, j) * G(j, i);
        double v = H(r, i) + (Mt(i, r) - hg);
        u[r] = v < EPSILON_1EMINUS16 ? EPSILON_1EMINUS16 : v;
      }
      for (UWORD r = 0; r < H.n_rows; ++r) H(r, i) = u[r];
    }
    return H.t();
  }

 public:
  MyHALS(const planc::Tensor& t, int k) : planc::AUNTF(t, k, HALS) {}
};

int main(int argc, char** argv) {
  if (argc < 8) return 2;
  UVEC dims({(uint64_t)std::stoull(argv[1]), (uint64_t)std::stoull(argv[2]),
             (uint64_t)std::stoull(argv[3])});
  const int k = std::stoi(argv[4]), iters = std::stoi(argv[5]);
  planc::Tensor X(dims);  // mt19937(103) data, as the reference
  MyHALS solver(X, k);
  solver.throw_on_error(true);
  solver.num_it(iters);
  solver.compute_error(true);
  solver.dim_tree(true);
  planc::NCPFactors init(dims, k, false);
  for (int n = 0; n < 3; ++n) {
    std::ifstream f(std::string(argv[6]) + "_" + std::to_string(n) + ".txt");
    MAT F(dims(n), k);
    for (UWORD i = 0; i < F.n_rows; ++i)
      for (UWORD r = 0; r < F.n_cols; ++r) f >> F(i, r);
    init.set(n, F);
  }
  solver.reset(init);
  solver.computeNTF();
  planc::NCPFactors& F = solver.ncp_factors();
  for (int n = 0; n < 3; ++n) {
    std::ofstream f(std::string(argv[7]) + "_" + std::to_string(n) + ".txt");
    f.precision(17);
    const MAT& M = F.factor(n);
    for (UWORD i = 0; i < M.n_rows; ++i) {
      for (UWORD r = 0; r < M.n_cols; ++r) f << (r ? " " : "") << M(i, r);
      f << "\n";
    }
  }
  std::cout << "final_error " << solver.current_error() << std::endl;
  return 0;
}
