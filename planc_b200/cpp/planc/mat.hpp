// mat.hpp -- the dense types of the planc C++ API (MAT, VEC, UVEC).
//
// The reference types MAT/VEC/UVEC are Armadillo's arma::mat / arma::vec /
// arma::uvec (common/utils.h:57-69): column-major dense storage. When
// PLANC_USE_ARMADILLO is defined they are exactly those; otherwise this header
// supplies a small column-major replacement with the subset of the Armadillo
// interface that the NTF API uses (n_rows, n_cols, n_elem, memptr, element
// access, zeros/ones, t, col, row, size).
#pragma once

#ifdef PLANC_USE_ARMADILLO
#include <armadillo>
#define MAT arma::mat
#define VEC arma::vec
#define FVEC arma::fvec
#define UVEC arma::uvec
#define UWORD arma::uword
#else
#include <cstdint>
#include <initializer_list>
#include <stdexcept>
#include <vector>

namespace planc {

typedef uint64_t uword;

template <typename T>
class DenseMat {
 public:
  uword n_rows = 0, n_cols = 0, n_elem = 0;

  DenseMat() {}
  DenseMat(uword r, uword c) { set_size(r, c); }
  // column vector from a list (UVEC dims = {64, 64, 64})
  DenseMat(std::initializer_list<T> v) : data_(v) {
    n_rows = v.size();
    n_cols = 1;
    n_elem = n_rows;
  }
  explicit DenseMat(const std::vector<T>& v) : data_(v) {
    n_rows = v.size();
    n_cols = 1;
    n_elem = n_rows;
  }

  void set_size(uword r, uword c) {
    n_rows = r;
    n_cols = c;
    n_elem = r * c;
    data_.assign(n_elem, T(0));
  }
  void set_size(uword r) { set_size(r, 1); }
  DenseMat& zeros() {
    std::fill(data_.begin(), data_.end(), T(0));
    return *this;
  }
  DenseMat& zeros(uword r, uword c) {
    set_size(r, c);
    return *this;
  }
  DenseMat& zeros(uword r) { return zeros(r, 1); }
  DenseMat& ones() {
    std::fill(data_.begin(), data_.end(), T(1));
    return *this;
  }
  DenseMat& ones(uword r, uword c) {
    set_size(r, c);
    return ones();
  }
  DenseMat& fill(T v) {
    std::fill(data_.begin(), data_.end(), v);
    return *this;
  }

  T* memptr() { return data_.data(); }
  const T* memptr() const { return data_.data(); }
  uword size() const { return n_elem; }
  bool empty() const { return n_elem == 0; }

  T& operator()(uword i) { return data_[i]; }
  const T& operator()(uword i) const { return data_[i]; }
  T& operator[](uword i) { return data_[i]; }
  const T& operator[](uword i) const { return data_[i]; }
  T& operator()(uword i, uword j) { return data_[i + n_rows * j]; }
  const T& operator()(uword i, uword j) const { return data_[i + n_rows * j]; }
  T& at(uword i, uword j) { return (*this)(i, j); }

  DenseMat t() const {
    DenseMat o(n_cols, n_rows);
    for (uword j = 0; j < n_cols; ++j)
      for (uword i = 0; i < n_rows; ++i) o(j, i) = (*this)(i, j);
    return o;
  }
  DenseMat col(uword j) const {
    DenseMat o(n_rows, 1);
    for (uword i = 0; i < n_rows; ++i) o(i) = (*this)(i, j);
    return o;
  }
  DenseMat row(uword i) const {
    DenseMat o(1, n_cols);
    for (uword j = 0; j < n_cols; ++j) o(j) = (*this)(i, j);
    return o;
  }
  void set_col(uword j, const DenseMat& v) {
    for (uword i = 0; i < n_rows; ++i) (*this)(i, j) = v(i);
  }

 private:
  std::vector<T> data_;
};

template <typename T>
T prod(const DenseMat<T>& v) {
  T p = 1;
  for (uword i = 0; i < v.n_elem; ++i) p *= v(i);
  return p;
}

}  // namespace planc

#define MAT planc::DenseMat<double>
#define VEC planc::DenseMat<double>
#define FVEC planc::DenseMat<float>
#define UVEC planc::DenseMat<uint64_t>
#define UWORD planc::uword
#endif
