// nmf.cpp -- command-line driver of the B200 shared-memory NMF, the
// counterpart of the reference's dense nmf driver (nmf/nmf.cpp:14-322,
// options of common/parsecommandline.hpp:156-300):
//
//   dense_nmf -a <0 MU|1 HALS|2 ANLSBPP> -d "m n" -k <rank> -t <iters>
//             [-i <file>|rand_uniform|rand_normal|rand_lowrank] [-o <prefix>]
//             [-r "regW_l2 regW_l1 regH_l2 regH_l1"] [--symm <alpha>]
//             [--normalization l2|max] [--seed <n>] [--init <prefix>]
//             [--precision fp64|bf16|bf16x2]
//
// -i reads a .npy matrix (NumPyArray) or raw FP64 with a .info sidecar
// (Tensor::read); otherwise A is generated. The generators and the initial
// W, H follow the reference's recipe (uniform, normal clipped at 0, or
// W_true H_true; symmetric variants for --symm) with std::mt19937 in place of
// Armadillo's generator, so the numbers differ from the reference's draws.
// --init reads W and H from <prefix>_W.txt and <prefix>_H.txt (rows of k
// values) instead. -o writes <prefix>_W and <prefix>_H as text, one row per
// line (the raw_ascii output of nmf/nmf.cpp:222-228). --symm alpha enables
// the symmetric regularisation (alpha = 0: max(A)^2), -1 (default) disables it.
#include <getopt.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "planc/bppnmf.hpp"
#include "planc/hals.hpp"
#include "planc/mu.hpp"
#include "planc/npyio.hpp"
#include "planc/tensor.hpp"

namespace {

struct Opts {
  int algo = ANLSBPP;
  std::vector<uint64_t> dims;
  int k = 20, iters = 20;
  std::string input = "rand_uniform", output, init, precision, normalization;
  std::vector<double> reg;
  double symm = -1;
  unsigned seed = 193957;  // common/parsecommandline.hpp:145
};

void usage() {
  std::cout << "usage: dense_nmf -a <0 MU|1 HALS|2 ANLSBPP> -d \"m n\" -k <rank> -t <iters>\n"
               "                 [-i <file>|rand_uniform|rand_normal|rand_lowrank] [-o <prefix>]\n"
               "                 [-r \"regW_l2 regW_l1 regH_l2 regH_l1\"] [--symm <alpha>]\n"
               "                 [--normalization l2|max] [--seed <n>] [--init <prefix>]\n"
               "                 [--precision fp64|bf16|bf16x2]\n";
}

bool parse(int argc, char** argv, Opts& o) {
  enum { SYMM = 1000, NORM, SEED, INIT, PRECISION };
  static struct option opts[] = {{"algo", required_argument, 0, 'a'},
                                 {"dimensions", required_argument, 0, 'd'},
                                 {"input", required_argument, 0, 'i'},
                                 {"lowrank", required_argument, 0, 'k'},
                                 {"output", required_argument, 0, 'o'},
                                 {"regularizer", required_argument, 0, 'r'},
                                 {"iter", required_argument, 0, 't'},
                                 {"symm", required_argument, 0, SYMM},
                                 {"normalization", required_argument, 0, NORM},
                                 {"seed", required_argument, 0, SEED},
                                 {"init", required_argument, 0, INIT},
                                 {"precision", required_argument, 0, PRECISION},
                                 {"help", no_argument, 0, 'h'},
                                 {0, 0, 0, 0}};
  int c, idx;
  while ((c = getopt_long(argc, argv, "a:d:e:i:k:o:r:t:h", opts, &idx)) != -1) {
    switch (c) {
      case 'a': o.algo = std::atoi(optarg); break;
      case 'd': {
        std::stringstream ss(optarg);
        uint64_t v;
        while (ss >> v) o.dims.push_back(v);
        break;
      }
      case 'e': break;  // the shared-memory NMF always computes the error
      case 'i': o.input = optarg; break;
      case 'k': o.k = std::atoi(optarg); break;
      case 'o': o.output = optarg; break;
      case 'r': {
        std::stringstream ss(optarg);
        double v;
        while (ss >> v) o.reg.push_back(v);
        break;
      }
      case 't': o.iters = std::atoi(optarg); break;
      case SYMM: o.symm = std::atof(optarg); break;
      case NORM: o.normalization = optarg; break;
      case SEED: o.seed = (unsigned)std::atoi(optarg); break;
      case INIT: o.init = optarg; break;
      case PRECISION: o.precision = optarg; break;
      default: usage(); return false;
    }
  }
  return true;
}

MAT read_rows(const std::string& f, UWORD rows, UWORD k) {
  std::ifstream in(f);
  if (!in) {
    ERR << "cannot read " << f << std::endl;
    exit(EXIT_FAILURE);
  }
  MAT M(rows, k);
  for (UWORD i = 0; i < rows; ++i)
    for (UWORD r = 0; r < k; ++r) in >> M(i, r);
  return M;
}

void write_rows(const std::string& f, const MAT& M) {
  std::ofstream out(f);
  out.precision(17);
  for (UWORD i = 0; i < M.n_rows; ++i) {
    for (UWORD r = 0; r < M.n_cols; ++r) out << (r ? " " : "") << M(i, r);
    out << "\n";
  }
}

MAT load_matrix(const Opts& o, UWORD* m, UWORD* n) {
  const std::string& f = o.input;
  const bool npy = f.size() > 4 && f.compare(f.size() - 4, 4, ".npy") == 0;
  if (f.compare(0, 5, "rand_") != 0) {
    planc::Tensor t;
    if (npy) {
      planc::NumPyArray a;
      a.load(f);
      t = *a.m_input_tensor;
    } else {
      t.read(f);
    }
    if (t.modes() != 2) {
      ERR << f << " does not hold a matrix" << std::endl;
      exit(EXIT_FAILURE);
    }
    *m = (UWORD)t.dimension(0);
    *n = (UWORD)t.dimension(1);
    MAT A(*m, *n);
    std::copy(t.m_data.begin(), t.m_data.end(), A.memptr());
    return A;
  }
  // nmf/nmf.cpp:69-160 (dense): uniform, normal clipped at 0, or low rank
  *m = o.dims[0];
  *n = o.dims[1];
  const bool symm = o.symm != -1;
  std::mt19937 gen(o.seed);
  std::uniform_real_distribution<> uni(0, 1);
  std::normal_distribution<> nor(0, 1);
  MAT A(*m, *n);
  if (f == "rand_normal") {
    for (UWORD e = 0; e < A.n_elem; ++e) A(e) = nor(gen);
  } else if (f == "rand_lowrank") {
    MAT Wt(*m, o.k), Ht(o.k, *n);
    for (UWORD e = 0; e < Wt.n_elem; ++e) Wt(e) = uni(gen);
    for (UWORD e = 0; e < Ht.n_elem; ++e) Ht(e) = uni(gen);
    for (UWORD j = 0; j < *n; ++j)
      for (UWORD i = 0; i < *m; ++i) {
        double s = 0;
        for (int r = 0; r < o.k; ++r) s += Wt(i, r) * (symm ? Wt(j, r) : Ht(r, j));
        A(i, j) = s;
      }
    return A;
  } else {
    for (UWORD e = 0; e < A.n_elem; ++e) A(e) = uni(gen);
  }
  if (symm) {
    MAT B = A;
    for (UWORD j = 0; j < *n; ++j)
      for (UWORD i = 0; i < *m; ++i) A(i, j) = 0.5 * (B(i, j) + B(j, i));
  }
  if (f == "rand_normal")
    for (UWORD e = 0; e < A.n_elem; ++e) A(e) = A(e) < 0 ? 0.0 : A(e);
  return A;
}

template <class NMFTYPE>
int callNMF(const Opts& o) {
  UWORD m = 0, n = 0;
  MAT A = load_matrix(o, &m, &n);
  // nmf/nmf.cpp:162-172: input normalisation
  if (o.normalization == "l2") {
    for (UWORD j = 0; j < n; ++j) {
      double s = 0;
      for (UWORD i = 0; i < m; ++i) s += A(i, j) * A(i, j);
      s = std::sqrt(s);
      if (s > 0)
        for (UWORD i = 0; i < m; ++i) A(i, j) /= s;
    }
  } else if (o.normalization == "max") {
    double mx = *std::max_element(A.memptr(), A.memptr() + A.n_elem);
    for (UWORD e = 0; e < A.n_elem; ++e) A(e) = (1 / mx) * A(e);
  }
  const bool symm = o.symm != -1;
  if (symm && m != n) {
    ERR << "symmetric regularisation needs a square matrix" << std::endl;
    return 1;
  }
  MAT W(m, o.k), H(n, o.k);
  double symm_reg = o.symm;
  if (!o.init.empty()) {
    W = read_rows(o.init + "_W.txt", m, o.k);
    H = read_rows(o.init + "_H.txt", n, o.k);
  } else {
    // nmf/nmf.cpp:186-199
    std::mt19937 gen(o.seed);
    std::uniform_real_distribution<> uni(0, 1);
    for (UWORD e = 0; e < W.n_elem; ++e) W(e) = uni(gen);
    for (UWORD e = 0; e < H.n_elem; ++e) H(e) = uni(gen);
    if (symm) {
      double mean = 0;
      for (UWORD e = 0; e < A.n_elem; ++e) mean += A(e);
      mean /= (double)A.n_elem;
      for (UWORD e = 0; e < H.n_elem; ++e) H(e) = 2 * std::sqrt(mean / o.k) * H(e);
      W = H;
    }
  }
  if (symm && symm_reg == 0.0) {
    double mx = *std::max_element(A.memptr(), A.memptr() + A.n_elem);
    symm_reg = mx * mx;
  }
  NMFTYPE nmfAlgorithm(A, W, H);
  nmfAlgorithm.num_iterations(o.iters);
  nmfAlgorithm.symm_reg(symm ? symm_reg : -1);
  nmfAlgorithm.updalgo(static_cast<algotype>(o.algo));
  if (o.reg.size() == 4) {
    FVEC rw, rh;
    rw.zeros(2);
    rh.zeros(2);
    rw(0) = (float)o.reg[0];
    rw(1) = (float)o.reg[1];
    rh(0) = (float)o.reg[2];
    rh(1) = (float)o.reg[3];
    nmfAlgorithm.regW(rw);
    nmfAlgorithm.regH(rh);
  }
  nmfAlgorithm.computeNMF();
  if (!o.output.empty()) {
    write_rows(o.output + "_W", nmfAlgorithm.getLeftLowRankFactor());
    write_rows(o.output + "_H", nmfAlgorithm.getRightLowRankFactor());
  }
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  Opts o;
  if (!parse(argc, argv, o)) return 0;
  if (o.input.compare(0, 5, "rand_") == 0 && o.dims.size() != 2) {
    usage();
    return 1;
  }
  if (!o.precision.empty()) setenv("PLANC_GPU_PRECISION", o.precision.c_str(), 1);
  switch (o.algo) {
    case MU: return callNMF<planc::MUNMF<MAT>>(o);
    case HALS: return callNMF<planc::HALSNMF<MAT>>(o);
    case ANLSBPP: return callNMF<planc::BPPNMF<MAT>>(o);
    default:
      ERR << "Wrong algorithm choice. Quitting.." << o.algo << std::endl;
      return 1;
  }
}
