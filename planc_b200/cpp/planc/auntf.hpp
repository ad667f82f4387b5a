// auntf.hpp -- planc::AUNTF, the alternating-update NTF solver of the planc C++
// API (reference ntf/auntf.hpp:40-251), running on the B200 through the C ABI
// of libplanc_gpu.so (include/planc_gpu.h).
//
// Same public interface and call order as the reference: construct with a
// Tensor, rank and algotype; num_it / compute_error / dim_tree / reset /
// accelerated; computeNTF(); ncp_factors(), current_error(), current_it(),
// computeObjectiveError(). The protected extension point is the same too:
// subclasses implement `MAT update(int mode)` and see m_ncp_factors,
// ncp_mttkrp_t[mode] (k x I_mode) and gram_without_one (k x k).
//
// The built-in subclasses (NTFMU, NTFHALS, NTFANLSBPP, NTFAOADMM, NTFNES)
// also report device_algo(), which lets computeNTF run the whole iteration on
// the GPU (one CUDA graph per iteration; NTFNES's acceleration included); any
// other subclass runs its update() on the host between the device's Gram /
// MTTKRP and normalisation steps. With accelerated(true) on a built-in update
// other than NTFNES, the device runs one iteration at a time and the host
// calls accelerate() after each, as the reference's loop does.
//
// Differences from the reference, all documented behaviour of this build:
//  * the relative error is computed in the FP64 Gram form
//    ||X||^2 - 2<X,M> + ||M||^2 on the device (same value as the reference's
//    explicit reconstruction, ntf/auntf.hpp:200-246, to ~1e-12);
//  * dim_tree(true) may be called before or after reset();
//  * errors: by default a failing GPU call prints its message and exits,
//    like the reference's exit() paths; throw_on_error(true) throws
//    planc::GpuError instead. The environment variables PLANC_GPU_DEVICE
//    (default 0) and PLANC_GPU_PRECISION (fp64 | bf16 | bf16x2, default fp64)
//    select the device and the MTTKRP precision.
#pragma once
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "ncpfactors.hpp"
#include "planc_gpu.h"
#include "tensor.hpp"

namespace planc {

class GpuError : public std::runtime_error {
 public:
  GpuError(int code, const std::string& m) : std::runtime_error(m), code(code) {}
  int code;
};

class AUNTF {
 protected:
  NCPFactors m_ncp_factors;
  MAT* ncp_mttkrp_t;
  MAT gram_without_one;
  virtual MAT update(const int mode) = 0;
  // PLANC_GPU_MU / _HALS / _ANLSBPP / _AOADMM / _NESTEROV when update() is
  // one of the device updates; -1 runs update() on the host.
  virtual int device_algo() const { return -1; }

 private:
  const Tensor& m_input_tensor;
  int m_num_it = 20;
  int m_current_it = 0;
  bool m_compute_error = false;
  const int m_low_rank_k;
  const algotype m_updalgo;
  bool m_enable_dim_tree = false;
  bool m_accelerated = false;
  bool m_throw = false;
  double m_rel_error = 0.0;
  double m_normA;
  std::vector<bool> m_stale_mttkrp;
  planc_gpu_ctx* m_ctx = nullptr;
  bool m_tensor_on_device = false;
  bool m_factors_on_device = false;

  void check(int rc) const {
    if (rc == PLANC_GPU_OK) return;
    std::string msg = std::string("planc_gpu error ") + std::to_string(rc) + ": " +
                      planc_gpu_last_error();
    if (m_throw) throw GpuError(rc, msg);
    ERR << msg << std::endl;
    exit(EXIT_FAILURE);
  }

  static int env_precision() {
    const char* p = std::getenv("PLANC_GPU_PRECISION");
    if (!p) return PLANC_GPU_PREC_FP64;
    if (!std::strcmp(p, "bf16")) return PLANC_GPU_PREC_BF16;
    if (!std::strcmp(p, "bf16x2")) return PLANC_GPU_PREC_BF16X2;
    return PLANC_GPU_PREC_FP64;
  }

  void ensure_context() {
    if (m_ctx) return;
    const char* d = std::getenv("PLANC_GPU_DEVICE");
    check(planc_gpu_create(&m_ctx, d ? std::atoi(d) : 0, env_precision(), nullptr));
  }

  void upload_tensor() {
    ensure_context();
    if (m_tensor_on_device) return;
    const int N = m_input_tensor.modes();
    std::vector<int64_t> dims(N);
    for (int i = 0; i < N; ++i) dims[i] = (int64_t)m_input_tensor.dimensions()(i);
    check(planc_gpu_set_tensor(m_ctx, m_input_tensor.m_data.data(), PLANC_GPU_F64, dims.data(), N,
                               0));
    m_tensor_on_device = true;
  }

  // host NCPFactors (I x k column-major) -> device (row-major I x k), as
  // AUNTF::reset does (every mode normalised, lambda from the host).
  void upload_factors() {
    upload_tensor();
    const int N = m_input_tensor.modes();
    std::vector<std::vector<double>> rm(N);
    std::vector<const double*> ptr(N);
    for (int n = 0; n < N; ++n) {
      MAT& F = m_ncp_factors.factor(n);
      rm[n].resize(F.n_elem);
      for (UWORD i = 0; i < F.n_rows; ++i)
        for (UWORD r = 0; r < F.n_cols; ++r) rm[n][i * F.n_cols + r] = F(i, r);
      ptr[n] = rm[n].data();
    }
    VEC lam = m_ncp_factors.lambda();
    check(planc_gpu_set_factors(m_ctx, ptr.data(), lam.memptr(), m_low_rank_k));
    m_factors_on_device = true;
  }

  void download_factors() {
    const int N = m_input_tensor.modes();
    std::vector<std::vector<double>> rm(N);
    std::vector<double*> ptr(N);
    for (int n = 0; n < N; ++n) {
      rm[n].resize((size_t)m_input_tensor.dimensions()(n) * m_low_rank_k);
      ptr[n] = rm[n].data();
    }
    VEC lam(m_low_rank_k, 1);
    check(planc_gpu_get_factors(m_ctx, ptr.data(), lam.memptr()));
    for (int n = 0; n < N; ++n) {
      MAT F(m_input_tensor.dimensions()(n), m_low_rank_k);
      for (UWORD i = 0; i < F.n_rows; ++i)
        for (UWORD r = 0; r < F.n_cols; ++r) F(i, r) = rm[n][i * F.n_cols + r];
      m_ncp_factors.set(n, F);
    }
    m_ncp_factors.set_lambda(lam);
  }

  void print_iteration(int it, bool err, double e) {
    INFO << "iter::" << it << std::endl;
    if (err) INFO << "relative_error at it::" << it << "::" << e << std::endl;
  }

  virtual void accelerate() {}

 public:
  // ntf/auntf.hpp:83-105
  AUNTF(const Tensor& i_tensor, const int i_k, algotype i_algo)
      : m_ncp_factors(i_tensor.dimensions(), i_k, false),
        m_input_tensor(i_tensor),
        m_low_rank_k(i_k),
        m_updalgo(i_algo) {
    m_ncp_factors.normalize();
    gram_without_one.zeros(i_k, i_k);
    ncp_mttkrp_t = new MAT[i_tensor.modes()];
    for (int i = 0; i < i_tensor.modes(); i++) {
      ncp_mttkrp_t[i].zeros(i_k, i_tensor.dimensions()(i));
      m_stale_mttkrp.push_back(true);
    }
    m_normA = i_tensor.norm();
  }
  virtual ~AUNTF() {
    delete[] ncp_mttkrp_t;
    planc_gpu_destroy(m_ctx);
  }
  AUNTF(const AUNTF&) = delete;
  AUNTF& operator=(const AUNTF&) = delete;

  NCPFactors& ncp_factors() { return m_ncp_factors; }
  void dim_tree(bool i_dim_tree) { m_enable_dim_tree = i_dim_tree; }
  double current_error() const { return m_rel_error; }
  void num_it(const int i_n) { m_num_it = i_n; }
  int current_it() const { return m_current_it; }
  void compute_error(bool e) { m_compute_error = e; }
  void accelerated(const bool& a) {
    m_accelerated = a;
    m_compute_error = true;
  }
  bool is_stale_mttkrp(const int& m) const { return m_stale_mttkrp[m]; }
  void throw_on_error(bool t) { m_throw = t; }
  algotype algorithm() const { return m_updalgo; }
  // The device context (for callers that want the C ABI directly).
  planc_gpu_ctx* gpu_context() {
    upload_factors_if_needed();
    return m_ctx;
  }

  void upload_factors_if_needed() {
    if (!m_factors_on_device) upload_factors();
  }

  // ntf/auntf.hpp:186-198
  void reset(const NCPFactors& new_factors, bool trans = false) {
    const int N = m_input_tensor.modes();
    for (int i = 0; i < N; i++) {
      m_ncp_factors.set(i, trans ? new_factors.factor(i).t() : new_factors.factor(i));
      m_ncp_factors.normalize(i);
    }
    m_ncp_factors.set_lambda(new_factors.lambda());
    upload_factors();
  }

  // ntf/auntf.hpp:128-177
  void computeNTF() {
    upload_factors_if_needed();
    const int algo = device_algo();
    const bool want_err = m_compute_error || m_accelerated;
    if (algo >= 0 && (!m_accelerated || algo == PLANC_GPU_NESTEROV)) {
      std::vector<double> errs(m_num_it > 0 ? m_num_it : 1, 0.0);
      check(planc_gpu_run(m_ctx, algo, m_num_it, m_enable_dim_tree ? 1 : 0, want_err ? 1 : 0,
                          errs.data()));
      for (m_current_it = 0; m_current_it < m_num_it; m_current_it++)
        print_iteration(m_current_it, want_err, errs[m_current_it]);
      if (want_err && m_num_it > 0) m_rel_error = errs[m_num_it - 1];
      for (auto&& s : m_stale_mttkrp) s = false;
      download_factors();
      return;
    }
    if (algo >= 0) {  // built-in device update, host acceleration hook
      for (m_current_it = 0; m_current_it < m_num_it; m_current_it++) {
        check(planc_gpu_run(m_ctx, algo, 1, m_enable_dim_tree ? 1 : 0, 1, &m_rel_error));
        print_iteration(m_current_it, true, m_rel_error);
        for (auto&& s : m_stale_mttkrp) s = false;
        download_factors();
        accelerate();
      }
      return;
    }
    const int N = m_input_tensor.modes();
    for (m_current_it = 0; m_current_it < m_num_it; m_current_it++) {
      INFO << "iter::" << m_current_it << std::endl;
      for (int j = 0; j < N; j++) {
        download_factors();
        check(planc_gpu_mode_begin(m_ctx, j, m_enable_dim_tree ? 1 : 0, gram_without_one.memptr(),
                                   ncp_mttkrp_t[j].memptr()));
        MAT factor = update(j);  // k x I_j, i.e. row-major I_j x k in memory
        check(planc_gpu_mode_end(m_ctx, j, factor.memptr()));
        m_stale_mttkrp[j] = false;
      }
      download_factors();
      if (want_err) {
        check(planc_gpu_objective_error(m_ctx, &m_rel_error));
        INFO << "relative_error at it::" << m_current_it << "::" << m_rel_error << std::endl;
      }
      if (m_accelerated) accelerate();
    }
  }

  // ntf/auntf.hpp:200-246
  double computeObjectiveError() {
    upload_factors_if_needed();
    double e = 0;
    check(planc_gpu_objective_error(m_ctx, &e));
    return e;
  }
  double computeObjectiveError(const NCPFactors& new_factors_t) {
    reset(new_factors_t, true);
    return computeObjectiveError();
  }
};

}  // namespace planc
