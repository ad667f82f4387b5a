// npyio.hpp -- planc::NumPyArray, the .npy tensor reader of the planc C++ API
// (reference common/npyio.hpp:13-107): load(file) parses the NumPy header and
// reads the data into a new planc::Tensor with the header's shape
// (m_input_tensor), printInfo() reports what was read.
//
// Same contract as the reference for the files it reads: little-endian FP64
// data is taken as stored, as the tensor's m_data (mode 0 fastest), whatever
// the header's fortran_order says (the reference reads the raw words the same
// way; a C-order array therefore arrives with its modes reversed in memory,
// and this reader says so on stderr). Beyond the reference: the header length
// is taken from the header (format versions 1.0, 2.0 and 3.0, so headers
// longer than 255 bytes read correctly), and little-endian FP32 data ('<f4')
// is widened to FP64 instead of being read as 8-byte words. Failures print
// the reason and exit, as the reference's exit(-1) paths do.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "tensor.hpp"

namespace planc {

class NumPyArray {
 private:
  int64_t m_word_size = 0;
  bool m_fortran_order = false;
  int64_t m_modes = 0;
  UVEC m_dims;
  char m_kind = 'f';

  static void fail(const std::string& what) {
    ERR << what << std::endl;
    exit(-1);
  }

  // common/npyio.hpp:19-76: magic, version, header length, then the header
  // dictionary {'descr': '<f8', 'fortran_order': True, 'shape': (d0, d1, ...), }
  void parse_npy_header(FILE* fp) {
    unsigned char pre[8];
    if (fread(pre, 1, 8, fp) != 8 || std::memcmp(pre, "\x93NUMPY", 6) != 0)
      fail("Something wrong. Could not read header ");
    const int major = pre[6];
    uint32_t hlen = 0;
    if (major == 1) {
      unsigned char l[2];
      if (fread(l, 1, 2, fp) != 2) fail("Something wrong. Could not read header ");
      hlen = (uint32_t)l[0] | ((uint32_t)l[1] << 8);
    } else {
      unsigned char l[4];
      if (fread(l, 1, 4, fp) != 4) fail("Something wrong. Could not read header ");
      hlen = (uint32_t)l[0] | ((uint32_t)l[1] << 8) | ((uint32_t)l[2] << 16) |
             ((uint32_t)l[3] << 24);
    }
    std::string header(hlen, '\0');
    if (fread(&header[0], 1, hlen, fp) != hlen) fail("Something wrong. Could not read header ");

    size_t loc = header.find("fortran_order");
    if (loc == std::string::npos) fail("could not find fortran_order");
    m_fortran_order = header.compare(header.find(':', loc) + 1, 5, " True") == 0 ||
                      header.compare(header.find(':', loc) + 1, 4, "True") == 0;

    size_t l1 = header.find('('), l2 = header.find(')');
    if (l1 == std::string::npos || l2 == std::string::npos) fail("could not find ()");
    std::vector<uint64_t> dims;
    std::string shape = header.substr(l1 + 1, l2 - l1 - 1);
    size_t p = 0;
    while (p < shape.size()) {
      size_t q = shape.find(',', p);
      std::string tok = shape.substr(p, q == std::string::npos ? std::string::npos : q - p);
      if (tok.find_first_of("0123456789") != std::string::npos)
        dims.push_back(std::strtoull(tok.c_str(), nullptr, 10));
      if (q == std::string::npos) break;
      p = q + 1;
    }
    if (dims.empty()) dims.push_back(1);  // a 0-d array holds one value
    m_modes = (int64_t)dims.size();
    m_dims = UVEC(dims);

    loc = header.find("descr");
    if (loc == std::string::npos) fail("could not find descr");
    size_t quote = header.find('\'', header.find(':', loc));
    const char order = header[quote + 1];
    if (!(order == '<' || order == '|' || order == '='))
      fail("only little-endian .npy data is supported");
    m_kind = header[quote + 2];
    m_word_size = std::atoi(header.c_str() + quote + 3);
    if (m_kind != 'f' || (m_word_size != 8 && m_word_size != 4))
      fail("only float64 and float32 .npy data is supported");
  }

 public:
  Tensor* m_input_tensor = nullptr;

  NumPyArray() {}
  ~NumPyArray() { delete m_input_tensor; }
  NumPyArray(const NumPyArray&) = delete;
  NumPyArray& operator=(const NumPyArray&) = delete;

  // common/npyio.hpp:86-100
  void load(std::string fname) {
    FILE* fp = fopen(fname.c_str(), "rb");
    if (fp == NULL) fail("Could not load the file " + fname);
    parse_npy_header(fp);
    if (!m_fortran_order && m_modes > 1)
      WARN << "NumPyArray: " << fname << " is in C order; its data is read as stored "
           << "(mode 0 fastest), as the reference does" << std::endl;
    delete m_input_tensor;
    std::vector<double> data(prod(m_dims));
    size_t nread = 0;
    if (m_word_size == 8) {
      nread = fread(data.data(), sizeof(double), data.size(), fp);
    } else {
      std::vector<float> f(data.size());
      nread = fread(f.data(), sizeof(float), f.size(), fp);
      for (size_t i = 0; i < nread; ++i) data[i] = f[i];
    }
    fclose(fp);
    if (nread != data.size())
      WARN << "something wrong ::read::" << nread << "::numel::" << data.size()
           << "::word_size::" << m_word_size << std::endl;
    m_input_tensor = new Tensor(m_dims, data.data());
  }

  // common/npyio.hpp:101-105
  void printInfo() {
    INFO << "modes::" << m_modes << "::dims::";
    for (uword i = 0; i < m_dims.n_elem; ++i) INFO << " " << m_dims(i);
    INFO << "::fortran_order::" << m_fortran_order << "::word_size::" << m_word_size
         << std::endl;
  }
  UVEC dimensions() const { return m_dims; }
  bool fortran_order() const { return m_fortran_order; }
  int64_t word_size() const { return m_word_size; }
};

}  // namespace planc
