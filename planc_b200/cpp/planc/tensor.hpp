// tensor.hpp -- planc::Tensor, the dense N-way tensor of the planc C++ API
// (reference common/tensor.hpp:36-521). Storage and semantics are the
// reference's: std::vector<double> m_data, column-major with mode 0 fastest;
// Tensor(dims) fills with std::mt19937(103) + uniform_real_distribution<>(0,1)
// in linear order; norm() and err() return SQUARED norms; write/read use a
// text ".info" sidecar (modes, then one dimension per line) and raw FP64.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "utils.hpp"

namespace planc {

class Tensor {
 public:
  std::vector<double> m_data;

  Tensor() : m_modes(0), m_numel(0), rand_seed(103) {}
  // tensor.hpp:86-93
  explicit Tensor(const UVEC& i_dimensions)
      : m_modes((int)i_dimensions.n_elem), m_dimensions(i_dimensions), rand_seed(103) {
    m_numel = prod(i_dimensions);
    m_data.resize(m_numel);
    randu();
  }
  Tensor(const UVEC& i_dimensions, const UVEC& i_start_idx) : Tensor(i_dimensions) {
    m_global_idx = i_start_idx;
  }
  // tensor.hpp:108-115: copies numel doubles
  Tensor(const UVEC& i_dimensions, const double* i_data)
      : m_modes((int)i_dimensions.n_elem), m_dimensions(i_dimensions), rand_seed(103) {
    m_numel = prod(i_dimensions);
    m_data.assign(i_data, i_data + m_numel);
  }

  int modes() const { return m_modes; }
  UVEC dimensions() const { return m_dimensions; }
  UVEC global_idx() const { return m_global_idx; }
  int dimension(int i) const { return (int)m_dimensions(i); }
  UWORD numel() const { return m_numel; }
  void set_idx(const UVEC& i) { m_global_idx = i; }
  void clear() {
    m_numel = 0;
    m_data.clear();
  }
  void zeros() { std::fill(m_data.begin(), m_data.end(), 0.0); }

  // tensor.hpp:219-235 (single generator, linear order)
  void randu(const int i_seed = -1) {
    std::uniform_real_distribution<> dis(0, 1);
    std::mt19937 gen(i_seed == -1 ? rand_seed : (unsigned)i_seed);
    for (UWORD i = 0; i < m_numel; i++) m_data[i] = dis(gen);
  }
  // squared Frobenius norm, tensor.hpp:350-356
  double norm() const {
    double s = 0;
    for (UWORD i = 0; i < m_numel; i++) s += m_data[i] * m_data[i];
    return s;
  }
  // squared distance, tensor.hpp:361-369
  double err(const Tensor& b) const {
    double s = 0;
    for (UWORD i = 0; i < m_numel; i++) {
      double d = m_data[i] - b.m_data[i];
      s += d * d;
    }
    return s;
  }
  template <typename T>
  void scale(T v) {
    for (auto& x : m_data) x = x * v;
  }
  template <typename T>
  void shift(T v) {
    for (auto& x : m_data) x = x + v;
  }
  template <typename T>
  void bound(T lo, T hi) {
    for (auto& x : m_data) {
      if (x < lo) x = lo;
      if (x > hi) x = hi;
    }
  }
  template <typename T>
  void lower_bound(T lo) {
    for (auto& x : m_data)
      if (x < lo) x = lo;
  }

  // tensor.hpp:430-457
  void write(std::string filename, std::ios_base::openmode = std::ios_base::out) {
    std::string info = filename.substr(0, filename.find_last_of(".")) + ".info";
    std::ofstream ofs(info);
    ofs << m_modes << std::endl;
    for (int i = 0; i < m_modes; i++) ofs << m_dimensions(i) << std::endl;
    ofs << std::endl;
    ofs.close();
    FILE* fp = fopen(filename.c_str(), "wb");
    if (!fp) {
      WARN << "cannot open " << filename << std::endl;
      return;
    }
    size_t n = fwrite(m_data.data(), sizeof(double), m_numel, fp);
    if (n != m_numel) WARN << "something wrong ::write::" << n << "::numel::" << m_numel << std::endl;
    fclose(fp);
  }
  // tensor.hpp:464-503
  void read(std::string filename, std::ios_base::openmode = std::ios_base::in) {
    m_data.clear();
    m_numel = 0;
    std::string info = filename.substr(0, filename.find_last_of(".")) + ".info";
    std::ifstream ifs(info);
    ifs >> m_modes;
    m_dimensions.zeros(m_modes);
    for (int i = 0; i < m_modes; i++) ifs >> m_dimensions(i);
    ifs.close();
    m_numel = prod(m_dimensions);
    m_data.resize(m_numel);
    FILE* fp = fopen(filename.c_str(), "rb");
    size_t n = fp ? fread(m_data.data(), sizeof(double), m_numel, fp) : 0;
    if (n != m_numel) WARN << "something wrong ::write::" << n << "::numel::" << m_numel << std::endl;
    if (fp) fclose(fp);
  }
  UWORD sub2ind(const UVEC& sub) const {
    UWORD idx = 0, stride = 1;
    for (int i = 0; i < m_modes; i++) {
      idx += sub(i) * stride;
      stride *= m_dimensions(i);
    }
    return idx;
  }
  double at(const UVEC& sub) const { return m_data[sub2ind(sub)]; }

 private:
  int m_modes;
  UVEC m_dimensions;
  UWORD m_numel;
  UVEC m_global_idx;
  unsigned int rand_seed;
};

}  // namespace planc
