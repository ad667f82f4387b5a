// nmf.hpp -- planc::NMF, the shared-memory NMF base of the planc C++ API
// (reference common/nmf.hpp:22-522): A (m x n, dense MAT) ~ W H^T with W
// (m x k) and H (n x k). Same public interface: the NMF(A, k) and
// NMF(A, W, H) constructors, computeNMF(), getLeftLowRankFactor(),
// getRightLowRankFactor(), num_iterations, tolerance, regW / regH (FVEC of
// {L2, L1}), symm_reg, updalgo, computeObjectiveError and printObjective.
//
// The subclasses HALSNMF, MUNMF and BPPNMF run their iterations on the B200
// through the C ABI (planc_gpu_nmf_*): the matrix and both factors go to the
// device once per computeNMF, the iterations run as CUDA graphs, and W, H and
// the objective come back at the end. The device evaluates the objective of
// every iteration; printObjective prints the reference's lines for each.
//
// Random initialisation (NMF(A, k)): the reference seeds Armadillo's generator
// with 89 for W and 73 for H (common/nmf.hpp:176-181); without Armadillo the
// factors come from std::mt19937 with the same seeds and
// uniform_real_distribution<>(0, 1) in column-major order. Pass W and H to
// reproduce a given start. Only dense matrices: the reference's sparse
// (SP_MAT) instantiation has no counterpart here. Environment:
// PLANC_GPU_DEVICE, PLANC_GPU_PRECISION (fp64 | bf16 | bf16x2) as for AUNTF.
#pragma once
#include <cassert>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "mat.hpp"
#include "planc_gpu.h"
#include "utils.hpp"

namespace planc {

template <class T>
class NMF {
 protected:
  const T& A;    /// input matrix of size m x n
  MAT W, H;      /// low-rank factors, m x k and n x k
  MAT Winit, Hinit;
  UINT m, n, k;  /// rows, columns and rank
  double objective_err = 1e12, fit_err_sq = 0;
  double normA = 0, normW = 0, normH = 0, l1normW = 0, l1normH = 0;
  double symmdiff = 0;
  double m_symm_reg = 0;
  unsigned int m_num_iterations = 20;
  double m_tolerance = 0;
  algotype m_updalgo = HALS;
  FVEC m_regW, m_regH;
  std::vector<double> m_objective, m_relerr;  // per iteration of the last run

  // NMF::normalize_by_W, common/nmf.hpp:150-160
  void normalize_by_W() {
    for (UINT i = 0; i < k; i++) {
      double ss = 0;
      for (UINT r = 0; r < m; ++r) ss += W(r, i) * W(r, i);
      const double nrm = std::sqrt(ss);
      if (nrm > 0) {
        for (UINT r = 0; r < m; ++r) W(r, i) = W(r, i) / nrm;
        for (UINT r = 0; r < n; ++r) H(r, i) = H(r, i) * nrm;
      }
    }
  }

  // Runs `algo` for num_iterations() on the device from the current W and H
  // and brings W, H and the per-iteration objective back.
  void run_on_device(int algo) {
    planc_gpu_ctx* ctx = nullptr;
    const char* d = std::getenv("PLANC_GPU_DEVICE");
    const char* p = std::getenv("PLANC_GPU_PRECISION");
    int prec = PLANC_GPU_PREC_FP64;
    if (p && !std::strcmp(p, "bf16")) prec = PLANC_GPU_PREC_BF16;
    if (p && !std::strcmp(p, "bf16x2")) prec = PLANC_GPU_PREC_BF16X2;
    check(planc_gpu_create(&ctx, d ? std::atoi(d) : 0, prec, nullptr), ctx);
    const int64_t dims[2] = {(int64_t)m, (int64_t)n};
    check(planc_gpu_set_tensor(ctx, A.memptr(), PLANC_GPU_F64, dims, 2, 0), ctx);
    std::vector<double> w = rowmajor(W), h = rowmajor(H);
    check(planc_gpu_nmf_set_factors(ctx, w.data(), h.data(), (int)k), ctx);
    const double rw[2] = {regW_at(m_regW, 0), regW_at(m_regW, 1)};
    const double rh[2] = {regW_at(m_regH, 0), regW_at(m_regH, 1)};
    check(planc_gpu_nmf_set_regularization(ctx, rw, rh, m_symm_reg > 0 ? m_symm_reg : 0.0), ctx);
    m_objective.assign(m_num_iterations, 0.0);
    m_relerr.assign(m_num_iterations, 0.0);
    if (m_num_iterations > 0)
      check(planc_gpu_nmf_run(ctx, algo, (int)m_num_iterations, m_objective.data(),
                              m_relerr.data()),
            ctx);
    check(planc_gpu_nmf_get_factors(ctx, w.data(), h.data()), ctx);
    planc_gpu_destroy(ctx);
    from_rowmajor(w, &W);
    from_rowmajor(h, &H);
    for (unsigned it = 0; it < m_num_iterations; ++it) {
      objective_err = m_objective[it];
      const double e = m_relerr[it] * normA;
      fit_err_sq = e * e;
      printObjective((int)it);
    }
  }

 private:
  static double regW_at(const FVEC& r, UWORD i) { return r.n_elem > i ? (double)r(i) : 0.0; }
  static std::vector<double> rowmajor(const MAT& F) {
    std::vector<double> v(F.n_elem);
    for (UWORD i = 0; i < F.n_rows; ++i)
      for (UWORD r = 0; r < F.n_cols; ++r) v[i * F.n_cols + r] = F(i, r);
    return v;
  }
  static void from_rowmajor(const std::vector<double>& v, MAT* F) {
    for (UWORD i = 0; i < F->n_rows; ++i)
      for (UWORD r = 0; r < F->n_cols; ++r) (*F)(i, r) = v[i * F->n_cols + r];
  }
  static void check(int rc, planc_gpu_ctx* ctx) {
    if (rc == PLANC_GPU_OK) return;
    ERR << "planc_gpu error " << rc << ": " << planc_gpu_last_error() << std::endl;
    planc_gpu_destroy(ctx);
    exit(EXIT_FAILURE);
  }
  void otherInitializations() {
    double s = 0;
    for (UWORD e = 0; e < A.n_elem; ++e) s += A(e) * A(e);
    normA = std::sqrt(s);  // arma::norm(A, "fro")
    m_regW.zeros(2);
    m_regH.zeros(2);
  }
  static void randu(MAT* F, unsigned seed) {
    std::mt19937 gen(seed);
    std::uniform_real_distribution<> dis(0, 1);
    for (UWORD e = 0; e < F->n_elem; ++e) (*F)(e) = dis(gen);
  }

 public:
  // common/nmf.hpp:170-185
  NMF(const T& input, const unsigned int rank) : A(input) {
    m = (UINT)A.n_rows;
    n = (UINT)A.n_cols;
    k = rank;
    W.set_size(m, k);
    H.set_size(n, k);
    randu(&W, 89);
    randu(&H, 73);
    otherInitializations();
    normalize_by_W();
  }
  // common/nmf.hpp:193-210
  NMF(const T& input, const MAT& leftlowrankfactor, const MAT& rightlowrankfactor) : A(input) {
    assert(leftlowrankfactor.n_cols == rightlowrankfactor.n_cols);
    W = leftlowrankfactor;
    H = rightlowrankfactor;
    Winit = W;
    Hinit = H;
    m = (UINT)A.n_rows;
    n = (UINT)A.n_cols;
    k = (UINT)W.n_cols;
    otherInitializations();
  }
  virtual ~NMF() {}

  virtual void computeNMF() = 0;

  MAT getLeftLowRankFactor() { return W; }
  MAT getRightLowRankFactor() { return H; }

  // common/nmf.hpp:386-425, on the host from the current factors
  void computeObjectiveError() {
    std::vector<double> WtW((size_t)k * k, 0), HtH((size_t)k * k, 0), AtW((size_t)n * k, 0);
    for (UINT a = 0; a < k; ++a)
      for (UINT b = 0; b < k; ++b) {
        double s = 0, t = 0;
        for (UINT r = 0; r < m; ++r) s += W(r, a) * W(r, b);
        for (UINT r = 0; r < n; ++r) t += H(r, a) * H(r, b);
        WtW[a * k + b] = s;
        HtH[a * k + b] = t;
      }
    for (UINT j = 0; j < n; ++j)
      for (UINT r = 0; r < k; ++r) {
        double s = 0;
        for (UINT i = 0; i < m; ++i) s += A(i, j) * W(i, r);
        AtW[j * k + r] = s;
      }
    double tr = 0, trww = 0, frow = 0, froh = 0, l1w = 0, l1h = 0, sym = 0;
    for (UINT j = 0; j < n; ++j)
      for (UINT r = 0; r < k; ++r) tr += H(j, r) * AtW[j * k + r];
    for (UINT a = 0; a < k; ++a) {
      frow += WtW[a * k + a];
      froh += HtH[a * k + a];
      for (UINT b = 0; b < k; ++b) trww += WtW[a * k + b] * HtH[b * k + a];
    }
    for (UINT r = 0; r < m; ++r) {
      double s = 0;
      for (UINT c = 0; c < k; ++c) s += W(r, c);
      l1w += s * s;
    }
    for (UINT r = 0; r < n; ++r) {
      double s = 0;
      for (UINT c = 0; c < k; ++c) s += H(r, c);
      l1h += s * s;
    }
    normW = std::sqrt(frow);
    normH = std::sqrt(froh);
    l1normW = std::sqrt(l1w);
    l1normH = std::sqrt(l1h);
    fit_err_sq = normA * normA - 2 * tr + trww;
    if (m_symm_reg > 0) {
      for (UWORD e = 0; e < W.n_elem; ++e) sym += (W(e) - H(e)) * (W(e) - H(e));
      symmdiff = std::sqrt(sym);
    }
    objective_err = fit_err_sq + regW_at(m_regW, 0) * frow + regW_at(m_regH, 0) * froh +
                    regW_at(m_regW, 1) * l1w + regW_at(m_regH, 1) * l1h +
                    (m_symm_reg > 0 ? m_symm_reg * sym : 0.0);
  }

  // common/nmf.hpp:428-446
  void printObjective(const int itr) {
    double err = (fit_err_sq > 0) ? std::sqrt(fit_err_sq) : normA;
    INFO << "Completed it = " << itr << "::algo::" << m_updalgo << "::k::" << k << std::endl;
    INFO << "objective::" << objective_err << "::squared error::" << fit_err_sq << std::endl
         << "error::" << err << "::relative error::" << err / normA << std::endl;
  }

  void num_iterations(const int it) { m_num_iterations = it; }
  void tolerance(const double tol) { m_tolerance = tol; }
  double tolerance() { return m_tolerance; }
  void regW(const FVEC& iregW) { m_regW = iregW; }
  void regH(const FVEC& iregH) { m_regH = iregH; }
  FVEC regW() { return m_regW; }
  FVEC regH() { return m_regH; }
  void symm_reg(const double& i_symm_reg) { m_symm_reg = i_symm_reg; }
  double symm_reg() { return m_symm_reg; }
  void updalgo(algotype dat) { m_updalgo = dat; }
  const unsigned int num_iterations() const { return m_num_iterations; }
  /// objective and relative error of every iteration of the last computeNMF
  const std::vector<double>& objective_history() const { return m_objective; }
  const std::vector<double>& relative_error_history() const { return m_relerr; }
};

}  // namespace planc
