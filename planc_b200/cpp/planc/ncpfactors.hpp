// ncpfactors.hpp -- planc::NCPFactors, the CP factor set of the planc C++ API
// (reference common/ncpfactors.hpp:22-446): N factors F_i (I_i x k, MAT,
// column-major) and lambda (k). Host-side; the GPU solver keeps its own
// device copies and syncs back into this object.
//
// Random initialisation: the reference seeds Armadillo's generator with 103
// (ncpfactors.hpp:46-56); Armadillo is not a dependency here, so the
// factors are drawn from std::mt19937(seed) + uniform_real_distribution<>(0,1)
// in column-major order, mode by mode. Injected factors (AUNTF::reset) are
// the way to reproduce a given start.
#pragma once
#include <cassert>
#include <cmath>
#include <random>
#include <vector>

#include "tensor.hpp"

namespace planc {

class NCPFactors {
 public:
  NCPFactors(const UVEC& i_dimensions, const int& i_k, bool trans)
      : m_modes((unsigned)i_dimensions.n_elem), m_k((unsigned)i_k), m_dimensions(i_dimensions) {
    m_factors.resize(m_modes);
    std::mt19937 gen(103);
    std::uniform_real_distribution<> dis(0, 1);
    for (unsigned i = 0; i < m_modes; i++) {
      UWORD rsize = m_dimensions(i) > 0 ? m_dimensions(i) : 1;
      if (trans)
        m_factors[i].set_size(m_k, rsize);
      else
        m_factors[i].set_size(rsize, m_k);
      for (UWORD e = 0; e < m_factors[i].n_elem; ++e) m_factors[i](e) = dis(gen);
    }
    m_lambda.ones(m_k, 1);
  }

  int rank() const { return (int)m_k; }
  UVEC dimensions() const { return m_dimensions; }
  MAT& factor(const int i_n) const { return const_cast<MAT&>(m_factors[i_n]); }
  int modes() const { return (int)m_modes; }
  VEC lambda() const { return m_lambda; }

  // ncpfactors.hpp:112-115
  void set(const int i_n, const MAT& i_factor) {
    assert(i_factor.size() == m_factors[i_n].size());
    m_factors[i_n] = i_factor;
  }
  void set_lambda(const VEC& l) { m_lambda = l; }

  // F^T F, k x k
  static MAT gram_of(const MAT& F) {
    MAT G(F.n_cols, F.n_cols);
    for (UWORD a = 0; a < F.n_cols; ++a)
      for (UWORD b = 0; b < F.n_cols; ++b) {
        double s = 0;
        for (UWORD i = 0; i < F.n_rows; ++i) s += F(i, a) * F(i, b);
        G(a, b) = s;
      }
    return G;
  }
  // ncpfactors.hpp:123-129
  void gram(MAT* o_UtU) {
    for (unsigned i = 0; i < m_modes; i++) {
      MAT g = gram_of(m_factors[i]);
      for (UWORD e = 0; e < g.n_elem; ++e) (*o_UtU)(e) *= g(e);
    }
  }
  // ncpfactors.hpp:139-148
  void gram_leave_out_one(const unsigned i_n, MAT* o_UtU) {
    o_UtU->ones(m_k, m_k);
    for (unsigned i = 0; i < m_modes; i++) {
      if (i == i_n) continue;
      MAT g = gram_of(m_factors[i]);
      for (UWORD e = 0; e < g.n_elem; ++e) (*o_UtU)(e) *= g(e);
    }
  }
  // ncpfactors.hpp:171-233: reverse Khatri-Rao product leaving out i_n,
  // (prod_{j != i_n} I_j) x k, lowest remaining mode fastest.
  void krp_leave_out_one(const unsigned i_n, MAT* o_krp) {
    UWORD rows = 1;
    for (unsigned i = 0; i < m_modes; i++)
      if (i != i_n) rows *= m_dimensions(i);
    o_krp->zeros(rows, m_k);
    std::vector<unsigned> order;
    for (int i = (int)m_modes - 1; i >= 0; i--)
      if ((unsigned)i != i_n) order.push_back((unsigned)i);
    std::vector<double> ab, nab;
    for (unsigned n = 0; n < m_k; n++) {
      const MAT& f0 = m_factors[order[0]];
      ab.assign(f0.n_rows, 0.0);
      for (UWORD i = 0; i < f0.n_rows; ++i) ab[i] = f0(i, n);
      for (size_t t = 1; t < order.size(); ++t) {
        const MAT& f = m_factors[order[t]];
        nab.resize(f.n_rows * ab.size());
        for (size_t b = 0; b < ab.size(); ++b)
          for (UWORD a = 0; a < f.n_rows; ++a) nab[a + f.n_rows * b] = f(a, n) * ab[b];
        ab.swap(nab);
      }
      for (UWORD r = 0; r < rows; ++r) (*o_krp)(r, n) = ab[r];
    }
  }
  MAT krp_leave_out_one(const unsigned i_n) {
    MAT k;
    krp_leave_out_one(i_n, &k);
    return k;
  }
  // ncpfactors.hpp:329-339 (initialisation only; resets lambda)
  void normalize() {
    m_lambda.ones();
    for (unsigned i = 0; i < m_modes; i++)
      for (unsigned j = 0; j < m_k; j++) {
        double nrm = col_norm(m_factors[i], j);
        if (nrm > 0)
          for (UWORD r = 0; r < m_factors[i].n_rows; ++r) m_factors[i](r, j) /= nrm;
        m_lambda(j) *= nrm;
      }
  }
  // ncpfactors.hpp:346-351 (replaces lambda)
  void normalize(int mode) {
    for (unsigned j = 0; j < m_k; j++) {
      m_lambda(j) = col_norm(m_factors[mode], j);
      if (m_lambda(j) > 0)
        for (UWORD r = 0; r < m_factors[mode].n_rows; ++r) m_factors[mode](r, j) /= m_lambda(j);
    }
  }
  // ncpfactors.hpp:358-363
  void normalize_rows(unsigned mode) {
    for (unsigned i = 0; i < m_k; i++) {
      MAT& F = m_factors[mode];
      double s = 0;
      for (UWORD c = 0; c < F.n_cols; ++c) s += F(i, c) * F(i, c);
      m_lambda(i) = std::sqrt(s);
      if (m_lambda(i) > 0)
        for (UWORD c = 0; c < F.n_cols; ++c) F(i, c) /= m_lambda(i);
    }
  }
  // ncpfactors.hpp:371-380 (std::mt19937 stands in for Armadillo's generator)
  void randu(const int i_seed) {
    std::mt19937 gen((unsigned)i_seed);
    std::uniform_real_distribution<> dis(0, 1);
    for (unsigned i = 0; i < m_modes; i++) {
      if (m_dimensions(i) > 0) {
        for (UWORD e = 0; e < m_factors[i].n_elem; ++e) m_factors[i](e) = dis(gen);
      } else {
        m_factors[i].zeros();
      }
    }
  }
  void zeros() {
    for (auto& f : m_factors) f.zeros();
  }
  void trans(NCPFactors& factor_t) {
    for (unsigned i = 0; i < m_modes; i++) factor_t.set(i, m_factors[i].t());
  }
  void printinfo() {
    INFO << "modes::" << m_modes << "::k::" << m_k << std::endl;
  }
  void print() {
    printinfo();
    for (unsigned i = 0; i < m_modes; i++) print(i);
  }
  void print(const unsigned i_n) {
    std::cout << i_n << "th factor" << std::endl << "=============" << std::endl;
    const MAT& F = m_factors[i_n];
    for (UWORD r = 0; r < F.n_rows; ++r) {
      for (UWORD c = 0; c < F.n_cols; ++c) std::cout << " " << F(r, c);
      std::cout << std::endl;
    }
  }

 private:
  static double col_norm(const MAT& F, UWORD j) {
    double s = 0;
    for (UWORD r = 0; r < F.n_rows; ++r) s += F(r, j) * F(r, j);
    return std::sqrt(s);
  }
  unsigned m_modes, m_k;
  UVEC m_dimensions;
  std::vector<MAT> m_factors;
  VEC m_lambda;
};

}  // namespace planc
