// ntf.cpp -- command-line driver of the B200 NTF solver, the counterpart of the
// reference's dense_ntf (ntf/ntf.cpp:19-71, options of
// common/parsecommandline.hpp:156-260):
//
//   dense_ntf -a <algo> -d "I0 I1 ..." -k <rank> -t <iters> -e <0|1>
//             [-i <file>] [--dimtree <0|1>] [--precision fp64|bf16|bf16x2]
//             [--seed <n>] [--init <file prefix>] [-o <output prefix>]
//
// -a takes the reference's algotype integers (0 MU, 1 HALS, 2 ANLSBPP,
// 4 AOADMM, 5 NESTEROV). -i reads raw FP64 with a .info sidecar
// (Tensor::read) or, for a name ending in .npy, a NumPy array
// (NumPyArray::load, common/npyio.hpp); with .npy the shape comes from the
// file and -d may be left out.
// Without -i (or with an -i starting with "rand_") the tensor is
// Tensor(dims): std::mt19937(103) uniform values, as in the reference.
// --init reads initial factors written by -o (<prefix>_<n>.txt, I_n rows of k
// values) and injects them with AUNTF::reset. -o writes the final factors and
// lambda as text (the role of distntf's raw_ascii output).
#include <getopt.h>

#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "planc/auntf.hpp"
#include "planc/npyio.hpp"
#include "planc/ntfanlsbpp.hpp"
#include "planc/ntfaoadmm.hpp"
#include "planc/ntfhals.hpp"
#include "planc/ntfmu.hpp"
#include "planc/ntfnes.hpp"
#include "planc/tensor.hpp"

namespace {

struct Opts {
  int algo = ANLSBPP;  // parsecommandline.hpp:137
  std::vector<uint64_t> dims;
  int k = 20;          // :135
  int iters = 20;      // :136
  int err = 0;         // :138
  int dimtree = 1;     // :140
  std::string input, init, output, precision;
};

void usage() {
  std::cout << "usage: dense_ntf -a <0 MU|1 HALS|2 ANLSBPP|4 AOADMM|5 NESTEROV> -d \"I0 I1 ...\"\n"
               "                 -k <rank> -t <iters>\n"
               "                 -e <0|1> [-i <file>] [--dimtree <0|1>]\n"
               "                 [--precision fp64|bf16|bf16x2] [--init <prefix>] [-o <prefix>]\n";
}

bool parse(int argc, char** argv, Opts& o) {
  enum { DIMTREE = 1000, PRECISION, INIT, SEED };
  static struct option opts[] = {{"algo", required_argument, 0, 'a'},
                                 {"dimensions", required_argument, 0, 'd'},
                                 {"error", required_argument, 0, 'e'},
                                 {"input", required_argument, 0, 'i'},
                                 {"lowrank", required_argument, 0, 'k'},
                                 {"output", required_argument, 0, 'o'},
                                 {"iter", required_argument, 0, 't'},
                                 {"dimtree", required_argument, 0, DIMTREE},
                                 {"precision", required_argument, 0, PRECISION},
                                 {"init", required_argument, 0, INIT},
                                 {"help", no_argument, 0, 'h'},
                                 {0, 0, 0, 0}};
  int c, idx;
  while ((c = getopt_long(argc, argv, "a:d:e:i:k:o:t:h", opts, &idx)) != -1) {
    switch (c) {
      case 'a': o.algo = std::atoi(optarg); break;
      case 'd': {
        std::stringstream ss(optarg);
        uint64_t v;
        while (ss >> v) o.dims.push_back(v);
        break;
      }
      case 'e': o.err = std::atoi(optarg); break;
      case 'i': o.input = optarg; break;
      case 'k': o.k = std::atoi(optarg); break;
      case 'o': o.output = optarg; break;
      case 't': o.iters = std::atoi(optarg); break;
      case DIMTREE: o.dimtree = std::atoi(optarg); break;
      case PRECISION: o.precision = optarg; break;
      case INIT: o.init = optarg; break;
      case 'h': usage(); return false;
      default: usage(); return false;
    }
  }
  return true;
}

template <class NTFTYPE>
int callNTF(const Opts& o) {
  const std::string rand_prefix("rand_");
  const bool npy = o.input.size() > 4 && o.input.compare(o.input.size() - 4, 4, ".npy") == 0;
  planc::Tensor my_tensor;
  if (npy) {
    planc::NumPyArray npyreader;
    npyreader.load(o.input);
    npyreader.printInfo();
    my_tensor = *npyreader.m_input_tensor;
  } else {
    my_tensor = planc::Tensor(UVEC(o.dims));
    if (!o.input.empty() && o.input.compare(0, rand_prefix.size(), rand_prefix) != 0)
      my_tensor.read(o.input);
  }
  NTFTYPE ntfsolver(my_tensor, o.k, static_cast<algotype>(o.algo));
  ntfsolver.num_it(o.iters);
  ntfsolver.compute_error(o.err != 0);
  if (o.dimtree) ntfsolver.dim_tree(true);
  if (!o.init.empty()) {
    planc::NCPFactors init(my_tensor.dimensions(), o.k, false);
    for (int n = 0; n < my_tensor.modes(); ++n) {
      std::ifstream f(o.init + "_" + std::to_string(n) + ".txt");
      MAT F(my_tensor.dimensions()(n), o.k);
      for (UWORD i = 0; i < F.n_rows; ++i)
        for (UWORD r = 0; r < F.n_cols; ++r) f >> F(i, r);
      init.set(n, F);
    }
    ntfsolver.reset(init);
  }
  ntfsolver.computeNTF();
  if (!o.output.empty()) {
    planc::NCPFactors& F = ntfsolver.ncp_factors();
    for (int n = 0; n < F.modes(); ++n) {
      std::ofstream f(o.output + "_" + std::to_string(n) + ".txt");
      f.precision(17);
      const MAT& M = F.factor(n);
      for (UWORD i = 0; i < M.n_rows; ++i) {
        for (UWORD r = 0; r < M.n_cols; ++r) f << (r ? " " : "") << M(i, r);
        f << "\n";
      }
    }
    std::ofstream f(o.output + "_lambda.txt");
    f.precision(17);
    VEC l = F.lambda();
    for (UWORD r = 0; r < l.n_elem; ++r) f << l(r) << "\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char* argv[]) {
  Opts o;
  if (!parse(argc, argv, o)) return 0;
  const bool npy = o.input.size() > 4 && o.input.compare(o.input.size() - 4, 4, ".npy") == 0;
  if (o.dims.size() < 2 && !npy) {
    usage();
    return 1;
  }
  if (!o.precision.empty()) setenv("PLANC_GPU_PRECISION", o.precision.c_str(), 1);
  switch (o.algo) {
    case MU: return callNTF<planc::NTFMU>(o);
    case HALS: return callNTF<planc::NTFHALS>(o);
    case ANLSBPP: return callNTF<planc::NTFANLSBPP>(o);
    case AOADMM: return callNTF<planc::NTFAOADMM>(o);
    case NESTEROV: return callNTF<planc::NTFNES>(o);
    default:
      ERR << "Wrong algorithm choice. Quitting.." << o.algo << std::endl;
      return 1;
  }
}
