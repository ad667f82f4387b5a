// ref_planc_driver.cpp -- a C ABI over the REFERENCE's own shared-memory NTF
// code, compiled unmodified from the reference tree by oracle/Makefile into
// oracle/_ref/libref_planc.so:
//   ntf/auntf.hpp, ntf/ntf{mu,hals,anlsbpp,aoadmm,nes}.hpp (AUNTF and its
//   updates), nnls/{nnls,bppnnls,SortBooleanMatrix}.hpp (BPP),
//   common/{tensor,ncpfactors,utils,ntf_utils}.hpp, dimtree/ddt.hpp (the
//   dimension tree) with dimtree/{dimtrees,ddttensor}.hpp.
// Armadillo is not installed here; the headers compile against the subset
// re-implemented in oracle/ref_shim/armadillo, with BLAS/LAPACK from the
// OpenBLAS shipped in the image.
//
// TEST INFRASTRUCTURE ONLY (a checker and the timed CPU baseline, never part
// of the product).
//
// Layouts: tensors column-major, mode 0 fastest (common/tensor.hpp:22-28);
// factors passed in and out row-major I_n x k (the memory of the reference's
// k x I_n transposes, ntf/auntf.hpp:95).
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>

#include <omp.h>

#include "ntf/ntfanlsbpp.hpp"
#include "ntf/ntfaoadmm.hpp"
#include "ntf/ntfhals.hpp"
#include "ntf/ntfmu.hpp"
#include "ntf/ntfnes.hpp"

namespace {

// The reference logs with INFO (std::cout) every iteration; the driver keeps
// its callers' stdout clean while reference code runs.
struct Quiet {
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Quiet() { std::cout.rdbuf(old); }
};

arma::uvec dims_of(const long* dims, int N) {
  arma::uvec d(N);
  for (int i = 0; i < N; ++i) d(i) = (arma::uword)dims[i];
  return d;
}

// row-major I x k buffer -> Armadillo I x k matrix (column-major)
arma::mat from_rowmajor(const double* F, arma::uword I, arma::uword k) {
  arma::mat m(I, k);
  for (arma::uword i = 0; i < I; ++i)
    for (arma::uword r = 0; r < k; ++r) m(i, r) = F[i * k + r];
  return m;
}
void to_rowmajor(const arma::mat& m, double* F) {
  for (arma::uword i = 0; i < m.n_rows; ++i)
    for (arma::uword r = 0; r < m.n_cols; ++r) F[i * m.n_cols + r] = m(i, r);
}

// The updates are protected members; a derived class reaches them with the
// inputs an AUNTF iteration would hold (factor, MTTKRP k x I, leave-one-out
// Gram) and returns what update() returns (k x I).
template <class Base>
struct UpdateProbe : Base {
  UpdateProbe(const planc::Tensor& t, int k, algotype a) : Base(t, k, a) {}
  arma::mat call(int mode, const arma::mat& H, const arma::mat& Mt, const arma::mat& G) {
    this->m_ncp_factors.set(mode, H);
    this->ncp_mttkrp_t[mode] = Mt;
    this->gram_without_one = G;
    return this->update(mode);
  }
};

struct NtfHandle {
  planc::Tensor* tensor;  // owned when created from a buffer
  planc::AUNTF* solver;
  int N, k;
};

planc::AUNTF* make_solver(const planc::Tensor& t, int k, int algo) {
  switch (algo) {
    case MU: return new planc::NTFMU(t, k, MU);
    case HALS: return new planc::NTFHALS(t, k, HALS);
    case ANLSBPP: return new planc::NTFANLSBPP(t, k, ANLSBPP);
    case AOADMM: return new planc::NTFAOADMM(t, k, AOADMM);
    case NESTEROV: return new planc::NTFNES(t, k, NESTEROV);
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

// ---- planc::Tensor
// Tensor(dims): the reference's constructor, filled by randu() with
// std::mt19937(103) (common/tensor.hpp:86-93, 219-235). That fill runs in an
// OpenMP loop over one shared generator, so its values depend on the thread
// count; with serial != 0 the constructor runs with one OpenMP thread (the
// reference's sequence as OMP_NUM_THREADS=1 gives it).
void* ref_tensor_new(const long* dims, int N, int serial) {
  const int nt = omp_get_max_threads();
  if (serial) omp_set_num_threads(1);
  planc::Tensor* t = new planc::Tensor(dims_of(dims, N));
  if (serial) omp_set_num_threads(nt);
  return t;
}
// Tensor(dims, data): copies numel doubles (common/tensor.hpp:113-121).
void* ref_tensor_from(const long* dims, int N, double* data) {
  return new planc::Tensor(dims_of(dims, N), data);
}
double* ref_tensor_data(void* t) { return &((planc::Tensor*)t)->m_data[0]; }
double ref_tensor_norm(void* t) { return ((planc::Tensor*)t)->norm(); }
void ref_tensor_free(void* t) { delete (planc::Tensor*)t; }

// Tensor::mttkrp (the direct MTTKRP, common/tensor.hpp:246-327) of mode n
// with the Khatri-Rao product NCPFactors::krp_leave_out_one builds from the
// given row-major factors. out: row-major I_n x k.
void ref_tensor_mttkrp(void* t, const double* const* F, int k, int n, double* out) {
  planc::Tensor* T = (planc::Tensor*)t;
  planc::NCPFactors f(T->dimensions(), k, false);
  for (int i = 0; i < T->modes(); ++i) f.set(i, from_rowmajor(F[i], T->dimension(i), k));
  arma::mat krp = f.krp_leave_out_one(n);
  arma::mat mt(k, T->dimension(n));  // ncp_mttkrp_t layout: k x I_n
  T->mttkrp(n, krp, &mt);
  // k x I_n column-major is row-major I_n x k
  std::memcpy(out, mt.memptr(), sizeof(double) * k * T->dimension(n));
}

// ---- NCPFactors (common/ncpfactors.hpp)
// gram_leave_out_one(n) of the given factors (:139-148). G: k x k.
void ref_gram_leave_out_one(const long* dims, int N, int k, const double* const* F, int n,
                            double* G) {
  planc::NCPFactors f(dims_of(dims, N), k, false);
  for (int i = 0; i < N; ++i) f.set(i, from_rowmajor(F[i], dims[i], k));
  arma::mat g(k, k);
  f.gram_leave_out_one(n, &g);
  std::memcpy(G, g.memptr(), sizeof(double) * k * k);
}
// normalize(mode) of factor H (row-major I x k, in place) and the lambda it
// sets (:346-351).
void ref_normalize_mode(double* H, long I, int k, double* lambda) {
  arma::uvec d(1);
  d(0) = (arma::uword)I;
  planc::NCPFactors f(d, k, false);
  f.set(0, from_rowmajor(H, I, k));
  f.normalize(0);
  to_rowmajor(f.factor(0), H);
  arma::vec l = f.lambda();
  std::memcpy(lambda, l.memptr(), sizeof(double) * k);
}

// ---- the updates of one mode, in isolation
// algo: the reference's algotype (MU 0, HALS 1, ANLSBPP 2, AOADMM 4,
// NESTEROV 5). H: current factor, row-major I x k; M: MTTKRP, row-major I x k
// (= ncp_mttkrp_t[mode], k x I); G: gram_without_one, k x k. out: the factor
// update() returns, as row-major I x k. Returns 0, or -1 for an unknown algo.
// AO-ADMM and Nesterov start from a fresh solver's auxiliary state.
int ref_update(int algo, const double* H, const double* M, const double* G, long I, int k,
               double* out) {
  Quiet q;
  arma::uvec d(3);
  d(0) = (arma::uword)I;
  d(1) = 1;
  d(2) = 1;
  planc::Tensor t(d);
  arma::mat Hm = from_rowmajor(H, I, k);
  arma::mat Mt(k, I);
  std::memcpy(Mt.memptr(), M, sizeof(double) * k * I);
  arma::mat Gm(k, k);
  std::memcpy(Gm.memptr(), G, sizeof(double) * k * k);
  arma::mat r;
  switch (algo) {
    case MU: { UpdateProbe<planc::NTFMU> p(t, k, MU); r = p.call(0, Hm, Mt, Gm); break; }
    case HALS: { UpdateProbe<planc::NTFHALS> p(t, k, HALS); r = p.call(0, Hm, Mt, Gm); break; }
    case ANLSBPP: { UpdateProbe<planc::NTFANLSBPP> p(t, k, ANLSBPP); r = p.call(0, Hm, Mt, Gm); break; }
    case AOADMM: { UpdateProbe<planc::NTFAOADMM> p(t, k, AOADMM); r = p.call(0, Hm, Mt, Gm); break; }
    default: return -1;
  }
  // update() returns k x I for MU/HALS/ANLSBPP/AOADMM
  std::memcpy(out, r.memptr(), sizeof(double) * k * I);
  return 0;
}

// ---- BPPNNLS (nnls/bppnnls.hpp:67-191) on normal equations
// AtA: n x n, AtB: n x ncols (column-major); X: n x ncols (column-major).
// Returns the BPP iteration count. (A run that hits the reference's cap exits
// the process with "BPP failed", as the reference does.)
int ref_bpp_solve(const double* AtA, const double* AtB, int n, long ncols, double* X) {
  arma::mat A(n, n), B(n, ncols);
  std::memcpy(A.memptr(), AtA, sizeof(double) * n * n);
  std::memcpy(B.memptr(), AtB, sizeof(double) * n * ncols);
  BPPNNLS<arma::mat, arma::vec> p(A, B, true);
  const int it = p.solveNNLS();
  arma::mat S = p.getSolutionMatrix();
  std::memcpy(X, S.memptr(), sizeof(double) * n * ncols);
  return it;
}

// ---- AUNTF (ntf/auntf.hpp) driven as a library user drives it:
// construct, dim_tree(...) before reset(), reset(initial factors),
// compute_error(...), num_it(T), computeNTF().
// tensor: from ref_tensor_new / ref_tensor_from (must outlive the handle).
// F: initial factors, row-major I_n x k; they are set unnormalised through
// NCPFactors::set and handed to reset() (which normalises each mode).
// serial_setup != 0 runs the constructor with one OpenMP thread: AUNTF's
// constructor builds its reconstruction buffer with Tensor(dims), whose fill
// loop shares one random generator among the OpenMP threads.
void* ref_ntf_create(void* tensor, int k, int algo, int dimtree, const double* const* F,
                     int compute_error, int serial_setup) {
  Quiet q;
  planc::Tensor* T = (planc::Tensor*)tensor;
  const int nt = omp_get_max_threads();
  if (serial_setup) omp_set_num_threads(1);
  planc::AUNTF* s = make_solver(*T, k, algo);
  if (serial_setup) omp_set_num_threads(nt);
  if (!s) return nullptr;
  if (dimtree) s->dim_tree(true);
  planc::NCPFactors init(T->dimensions(), k, false);
  for (int i = 0; i < T->modes(); ++i) init.set(i, from_rowmajor(F[i], T->dimension(i), k));
  s->reset(init, false);
  s->compute_error(compute_error != 0);
  if (algo == NESTEROV) s->accelerated(true);
  NtfHandle* h = new NtfHandle{T, s, T->modes(), k};
  return h;
}

// T outer iterations in one computeNTF() call; returns current_error() (the
// relative error of the last iteration when errors are computed, else 0).
double ref_ntf_run(void* hv, int iters) {
  Quiet q;
  NtfHandle* h = (NtfHandle*)hv;
  h->solver->num_it(iters);
  h->solver->computeNTF();
  return h->solver->current_error();
}

// The current factors (row-major I_n x k) and lambda (k).
void ref_ntf_factors(void* hv, double** F, double* lambda) {
  NtfHandle* h = (NtfHandle*)hv;
  planc::NCPFactors& f = h->solver->ncp_factors();
  for (int i = 0; i < h->N; ++i) to_rowmajor(f.factor(i), F[i]);
  arma::vec l = f.lambda();
  std::memcpy(lambda, l.memptr(), sizeof(double) * h->k);
}

// computeObjectiveError() of the current factors (explicit reconstruction,
// ntf/auntf.hpp:200-246).
double ref_ntf_objective_error(void* hv) {
  Quiet q;
  return ((NtfHandle*)hv)->solver->computeObjectiveError();
}

void ref_ntf_destroy(void* hv) {
  NtfHandle* h = (NtfHandle*)hv;
  delete h->solver;
  delete h;
}

// ---- DenseDimensionTree (dimtree/ddt.hpp) on its own
struct RefDimTree {
  planc::Tensor* T;
  planc::NCPFactors* F;
  DenseDimensionTree* kdt;
};

// X: column-major tensor (copied into a planc::Tensor); F: row-major factors.
// The tree splits at N/2 as AUNTF::dim_tree does (ntf/auntf.hpp:122-123) and
// runs with the 16 threads its constructor fixes (ddt.hpp:53).
void* ref_dimtree_create(double* X, const long* dims, int N, int k, const double* const* F) {
  RefDimTree* h = new RefDimTree();
  h->T = new planc::Tensor(dims_of(dims, N), X);
  h->F = new planc::NCPFactors(dims_of(dims, N), k, false);
  for (int i = 0; i < N; ++i) h->F->set(i, from_rowmajor(F[i], dims[i], k));
  h->kdt = new DenseDimensionTree(*h->T, *h->F, N / 2);
  return h;
}
// set_factor(F_n^T) as AUNTF::update_factor_mode passes it (row-major I x k)
void ref_dimtree_set_factor(void* hv, long mode, const double* F) {
  ((RefDimTree*)hv)->kdt->set_factor(F, mode);
}
// in_order_reuse_MTTKRP(n) with colmajor = false: row-major I_n x k.
void ref_dimtree_mttkrp(void* hv, long n, double* out) {
  Quiet q;
  double t1 = 0, t2 = 0;
  ((RefDimTree*)hv)->kdt->in_order_reuse_MTTKRP(n, out, false, t1, t2);
}
void ref_dimtree_destroy(void* hv) {
  RefDimTree* h = (RefDimTree*)hv;
  delete h->kdt;
  delete h->F;
  delete h->T;
  delete h;
}

}  // extern "C"
