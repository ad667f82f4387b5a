// ntf_oracle.cpp -- CPU oracle for PLANC's shared-memory NTF iteration.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker the CUDA path is compared
// against; nothing in the product (libplanc_gpu.so, the C++ API, the Python
// binding) links, loads or calls it. Only tests/, __graft_entry__.smoke() and
// the cpu_baseline / --impl reference legs of bench.py use it.
//
// It restates, in plain C++ over OpenBLAS (the same BLAS family the reference
// links through Armadillo), the algorithm of the reference files below. Every
// function names the reference lines it follows. Armadillo is not available
// here, so Armadillo expressions are written out as loops with the same
// semantics; `arma::solve(..., likely_sympd)` is restated as a Cholesky solve
// (LAPACK dposv) with an LU (dgesv) fallback when the Cholesky fails.
//
// Layout conventions (all buffers owned by the caller):
//   X        : dense tensor, column-major with mode 0 fastest
//              (common/tensor.hpp:22-28).
//   factors  : row-major I_n x k ("r fastest"); this is the memory layout of
//              the reference's ncp_mttkrp_t[n] (k x I_n column-major,
//              ntf/auntf.hpp:95) and of the dimension-tree factors
//              (dimtree/ddt.hpp:84-88).
//   k x k    : symmetric, layout irrelevant.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

extern "C" {
// OpenBLAS / LAPACK prototypes (LP64).
enum { CblasRowMajor = 101, CblasColMajor = 102 };
enum { CblasNoTrans = 111, CblasTrans = 112 };
void cblas_dgemm(int order, int ta, int tb, int m, int n, int k, double alpha,
                 const double* a, int lda, const double* b, int ldb,
                 double beta, double* c, int ldc);
void dposv_(const char* uplo, const int* n, const int* nrhs, double* a,
            const int* lda, double* b, const int* ldb, int* info);
void dgesv_(const int* n, const int* nrhs, double* a, const int* lda,
            int* ipiv, double* b, const int* ldb, int* info);
void dpotrf_(const char* uplo, const int* n, double* a, const int* lda, int* info);
void dsyev_(const char* jobz, const char* uplo, const int* n, double* a,
            const int* lda, double* w, double* work, const int* lwork, int* info);
}

namespace {

// common/utils.h:46-49
constexpr double kEps17 = 0.00000000000000001;  // EPSILON_1EMINUS16 (= 1e-17)
constexpr double kEps6 = 0.000001;               // EPSILON
constexpr double kEps12 = 1e-12;                 // EPSILON_1EMINUS12
// ntf/ntfanlsbpp.hpp:11
constexpr int64_t kChunk = 2000;                 // ONE_THREAD_MATRIX_SIZE

enum Algo { MU = 0, HALS = 1, ANLSBPP = 2, AOADMM = 4, NESTEROV = 5 };  // common/utils.h:10

int64_t prod(const int64_t* d, int a, int b) {
  int64_t p = 1;
  for (int i = a; i < b; ++i) p *= d[i];
  return p;
}

// Gram F^T F of a row-major I x k factor. common/ncpfactors.hpp:144
void gram(const double* F, int64_t I, int k, double* G) {
  cblas_dgemm(CblasColMajor, CblasNoTrans, CblasTrans, k, k, (int)I, 1.0, F, k,
              F, k, 0.0, G, k);
}

// Leave-one-out Hadamard product of Grams. common/ncpfactors.hpp:139-148
void gram_loo(const double* const* F, const int64_t* dims, int N, int k, int n,
              double* G) {
  std::vector<double> cur((size_t)k * k);
  for (int i = 0; i < k * k; ++i) G[i] = 1.0;
  for (int m = 0; m < N; ++m) {
    if (m == n) continue;
    gram(F[m], dims[m], k, cur.data());
    for (int i = 0; i < k * k; ++i) G[i] *= cur[i];
  }
}

// Reverse Khatri-Rao product of all factors except n, stored column-major
// (prod_{m!=n} I_m) x k. Row index is the column-major linear index over the
// remaining modes with the lowest mode fastest.
// common/ncpfactors.hpp:171-233 (per-column outer products, matorder
// reversed).
void krp_leave_out_one(const double* const* F, const int64_t* dims, int N,
                       int k, int n, double* KRP) {
  int64_t rows = 1;
  for (int m = 0; m < N; ++m)
    if (m != n) rows *= dims[m];
  std::vector<int> order;
  for (int m = N - 1; m >= 0; --m)
    if (m != n) order.push_back(m);
  std::vector<double> ab, nab;
  for (int r = 0; r < k; ++r) {
    int m0 = order[0];
    ab.resize(dims[m0]);
    for (int64_t i = 0; i < dims[m0]; ++i) ab[i] = F[m0][i * k + r];
    for (size_t t = 1; t < order.size(); ++t) {
      int m = order[t];
      int64_t Im = dims[m];
      nab.resize((size_t)Im * ab.size());
      // ab = currentvec * oldabvec.t(), vectorised column-major
      for (size_t b = 0; b < ab.size(); ++b)
        for (int64_t a = 0; a < Im; ++a)
          nab[a + Im * b] = F[m][a * k + r] * ab[b];
      ab.swap(nab);
    }
    std::memcpy(KRP + (size_t)r * rows, ab.data(), sizeof(double) * rows);
  }
}

// Direct MTTKRP with a materialised KRP. common/tensor.hpp:246-327.
// out is row-major I_n x k.
void mttkrp_direct(const double* X, const int64_t* dims, int N,
                   const double* const* F, int k, int n, double* out) {
  int64_t In = dims[n];
  int64_t krows = prod(dims, 0, N) / In;
  std::vector<double> KRP((size_t)krows * k);
  krp_leave_out_one(F, dims, N, k, n, KRP.data());
  if (n == 0) {
    // tensor.hpp:279-281: out(I0 x k, row-major) = X_(0) * KRP
    cblas_dgemm(CblasRowMajor, CblasTrans, CblasTrans, (int)In, k, (int)krows,
                1.0, X, (int)In, KRP.data(), (int)krows, 0.0, out, k);
  } else {
    int64_t ncols = prod(dims, 0, n);
    int64_t nmats = prod(dims, n + 1, N);
    // tensor.hpp:298-325: one dgemm per trailing slice, beta = 1 after the
    // first.
    for (int64_t i = 0; i < nmats; ++i) {
      cblas_dgemm(CblasRowMajor, CblasNoTrans, CblasTrans, (int)In, k,
                  (int)ncols, 1.0, X + i * ncols * In, (int)ncols,
                  KRP.data() + i * ncols, (int)(ncols * nmats),
                  i == 0 ? 0.0 : 1.0, out, k);
    }
  }
}

// Dimension-tree state, restating DenseDimensionTree (dimtree/ddt.hpp) for
// N in {3, 4} with split s = N/2 (ntf/auntf.hpp:122-123). P holds the
// right-contracted partial MTTKRP (prod_{i<=s} I_i) x k, column-major with
// the left modes' linear index fastest (dimtrees.hpp:281-306, ColMajor).
// Q holds P contracted with the updated F_0 (N = 4 only,
// ddt.hpp:218-226).
struct DimTree {
  int N, k, s;
  const int64_t* dims;
  int64_t L, R;
  std::vector<double> P, Q;
};

// ddt.hpp:134-243 restated. Writes the mode-n MTTKRP row-major I_n x k.
void dimtree_mttkrp(DimTree& t, const double* X, const double* const* F, int n,
                    double* out) {
  const int N = t.N, k = t.k, s = t.s;
  const int64_t* d = t.dims;
  if (n == 0) {
    // partial_MTTKRP_with_KRP_output_T(s, right, ...): P = X_(L x R) * KRP_right
    int64_t R = t.R, L = t.L;
    // For N in {3, 4} and s = N/2 the right group is the single last mode.
    const double* B = F[N - 1];  // row-major R x k
    // C(L x k, col-major) = X(L x R col-major) * B^T  where B is k x R col-major
    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasTrans, (int)L, k, (int)R, 1.0,
                X, (int)L, B, k, 0.0, t.P.data(), (int)L);
    // multi_TTV right over modes 1..s: M0[i0,r] = sum_{rest} P[i0,rest,r] *
    // prod_{1<=m<=s} F_m[i_m, r]   (dimtrees.hpp:464-479)
    int64_t I0 = d[0];
    int64_t rest = t.L / I0;
    std::fill(out, out + I0 * k, 0.0);
    std::vector<double> w((size_t)rest);
    for (int r = 0; r < k; ++r) {
      for (int64_t q = 0; q < rest; ++q) {
        int64_t idx = q;
        double v = 1.0;
        for (int m = 1; m <= s; ++m) {
          int64_t im = idx % d[m];
          idx /= d[m];
          v *= F[m][im * k + r];
        }
        w[q] = v;
      }
      const double* Pr = t.P.data() + (size_t)r * t.L;
      for (int64_t i0 = 0; i0 < I0; ++i0) {
        double acc = 0.0;
        for (int64_t q = 0; q < rest; ++q) acc += Pr[i0 + I0 * q] * w[q];
        out[i0 * k + r] = acc;
      }
    }
    return;
  }
  if (n == s + 1) {
    // partial_MTTKRP_with_KRP_output_FM(left, ...): M = X^T * KRP_left
    // (dimtrees.hpp:250-271, KRP from ddttensor.hpp:872-897)
    int64_t L = t.L, R = t.R;
    std::vector<double> colmaj((size_t)L * k);
    std::vector<const double*> sub(F, F + s + 1);
    krp_leave_out_one(sub.data(), d, s + 2, k, s + 1, colmaj.data());
    // out(R x k row-major) = X^T (R x L) * KRP (L x k)
    // as col-major: out^T (k x R) = KRP^T (k x L) * X (L x R)
    cblas_dgemm(CblasColMajor, CblasTrans, CblasNoTrans, k, (int)R, (int)L, 1.0,
                colmaj.data(), (int)L, X, (int)L, 0.0, out, k);
    return;
  }
  // 1 <= n <= s: multi-TTV on P (and Q for N = 4).
  if (N == 3) {
    // n == 1, s == 1: M1[i1,r] = sum_{i0} P[i0,i1,r] F0[i0,r]
    // (ddt.hpp:207-212, multi_TTV left)
    int64_t I0 = d[0], I1 = d[1];
    for (int r = 0; r < k; ++r) {
      const double* Pr = t.P.data() + (size_t)r * t.L;
      for (int64_t i1 = 0; i1 < I1; ++i1) {
        double acc = 0.0;
        for (int64_t i0 = 0; i0 < I0; ++i0)
          acc += Pr[i0 + I0 * i1] * F[0][i0 * k + r];
        out[i1 * k + r] = acc;
      }
    }
    return;
  }
  // N == 4, s == 2
  int64_t I0 = d[0], I1 = d[1], I2 = d[2];
  if (n == 1) {
    // Q[i1,i2,r] = sum_{i0} P[i0,i1,i2,r] F0[i0,r]   (ddt.hpp:218-226)
    t.Q.assign((size_t)I1 * I2 * k, 0.0);
    for (int r = 0; r < k; ++r) {
      const double* Pr = t.P.data() + (size_t)r * t.L;
      double* Qr = t.Q.data() + (size_t)r * I1 * I2;
      for (int64_t q = 0; q < I1 * I2; ++q) {
        double acc = 0.0;
        for (int64_t i0 = 0; i0 < I0; ++i0)
          acc += Pr[i0 + I0 * q] * F[0][i0 * k + r];
        Qr[q] = acc;
      }
    }
    // M1[i1,r] = sum_{i2} Q[i1,i2,r] F2[i2,r]   (ddt.hpp:231-232)
    for (int r = 0; r < k; ++r) {
      const double* Qr = t.Q.data() + (size_t)r * I1 * I2;
      for (int64_t i1 = 0; i1 < I1; ++i1) {
        double acc = 0.0;
        for (int64_t i2 = 0; i2 < I2; ++i2)
          acc += Qr[i1 + I1 * i2] * F[2][i2 * k + r];
        out[i1 * k + r] = acc;
      }
    }
    return;
  }
  // n == 2: M2[i2,r] = sum_{i1} Q[i1,i2,r] F1[i1,r]   (ddt.hpp:207-212)
  for (int r = 0; r < k; ++r) {
    const double* Qr = t.Q.data() + (size_t)r * I1 * I2;
    for (int64_t i2 = 0; i2 < I2; ++i2) {
      double acc = 0.0;
      for (int64_t i1 = 0; i1 < I1; ++i1)
        acc += Qr[i1 + I1 * i2] * F[1][i1 * k + r];
      out[i2 * k + r] = acc;
    }
  }
}

// Column normalisation of mode n; replaces lambda. ncpfactors.hpp:346-351
void normalize_mode(double* F, int64_t I, int k, double* lambda) {
  for (int r = 0; r < k; ++r) {
    double ss = 0.0;
    for (int64_t i = 0; i < I; ++i) ss += F[i * k + r] * F[i * k + r];
    double nrm = std::sqrt(ss);
    lambda[r] = nrm;
    if (nrm > 0)
      for (int64_t i = 0; i < I; ++i) F[i * k + r] /= nrm;
  }
}

// HALS update, ntf/ntfhals.hpp:13-29 with fixNumericalError
// (common/utils.hpp:59-64): u = H(:,i) + (M(i,:)^T - H*G(:,i)); u[u<1e-17] =
// 1e-17; if ||u||^2 > 0: H(:,i) = u. H is updated in place (Gauss-Seidel).
void hals_update(double* H, int64_t I, int k, const double* M,
                 const double* G) {
  std::vector<double> u((size_t)I);
  for (int i = 0; i < k; ++i) {
    for (int64_t row = 0; row < I; ++row) {
      double hg = 0.0;
      for (int j = 0; j < k; ++j) hg += H[row * k + j] * G[j + (size_t)k * i];
      double v = H[row * k + i] + (M[row * k + i] - hg);
      u[row] = (v < kEps17) ? kEps17 : v;
    }
    double nrm2 = 0.0;
    for (int64_t row = 0; row < I; ++row) nrm2 += u[row] * u[row];
    if (nrm2 > 0)
      for (int64_t row = 0; row < I; ++row) H[row * k + i] = u[row];
  }
}

// MU update, ntf/ntfmu.hpp:11-16: H = (H % M^T) / (H*G + 1e-6).
void mu_update(double* H, int64_t I, int k, const double* M, const double* G) {
  std::vector<double> t((size_t)k);
  for (int64_t row = 0; row < I; ++row) {
    for (int c = 0; c < k; ++c) {
      double acc = 0.0;
      for (int j = 0; j < k; ++j) acc += H[row * k + j] * G[j + (size_t)k * c];
      t[c] = acc + kEps6;
    }
    for (int c = 0; c < k; ++c)
      H[row * k + c] = (H[row * k + c] * M[row * k + c]) / t[c];
  }
}

// Solve A(P,P) x = b(P) for one column (arma::solve likely_sympd restated:
// Cholesky, then LU on failure). Returns 0 on success.
int solve_subset(const double* AtA, int n, const std::vector<int>& pset,
                 const double* b, double* x) {
  int m = (int)pset.size();
  if (m == 0) return 0;
  std::vector<double> A((size_t)m * m), A2, rhs(m), rhs2;
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < m; ++r) A[r + (size_t)m * c] = AtA[pset[r] + (size_t)n * pset[c]];
  for (int r = 0; r < m; ++r) rhs[r] = b[pset[r]];
  A2 = A;
  rhs2 = rhs;
  int one = 1, info = 0;
  char uplo = 'L';
  dposv_(&uplo, &m, &one, A.data(), &m, rhs.data(), &m, &info);
  if (info != 0) {
    std::vector<int> ipiv(m);
    dgesv_(&m, &one, A2.data(), &m, ipiv.data(), rhs2.data(), &m, &info);
    if (info != 0) return -1;
    rhs = rhs2;
  }
  for (int r = 0; r < m; ++r) x[pset[r]] = rhs[r];
  return 0;
}

// Block principal pivoting NNLS for multiple RHS, nnls/bppnnls.hpp:67-191.
// AtA: n x n, AtB: n x ncols column-major; X (out): n x ncols column-major.
// The reference groups columns with identical passive sets
// (bppnnls.hpp:204-287) only to share one factorisation; every column's
// values are the same as a per-column solve, which is what is done here.
// Returns the iteration count, or -1 if the iteration cap (5n) was hit
// (the reference prints "BPP failed" and exits, bppnnls.hpp:185-188).
int bpp_solve(const double* AtA, const double* AtB, int n, int64_t ncols,
              double* X, int* passive_out) {
  const unsigned MAX_IT = 5u * (unsigned)n;
  const int pbar = 3;
  std::vector<double> Y((size_t)n * ncols);
  std::vector<unsigned char> PS((size_t)n * ncols, 0), NonOpt((size_t)n * ncols),
      Infea((size_t)n * ncols);
  std::vector<int> P(ncols, pbar), Ninf(ncols, n + 1), NotGood(ncols);
  std::vector<unsigned char> NotOpt(ncols);
  std::fill(X, X + (size_t)n * ncols, 0.0);
  for (size_t i = 0; i < (size_t)n * ncols; ++i) Y[i] = -AtB[i];  // AtA*0 - AtB
  auto classify = [&](int64_t c) {
    int ng = 0;
    for (int r = 0; r < n; ++r) {
      size_t e = r + (size_t)n * c;
      NonOpt[e] = (Y[e] < 0) && !PS[e];
      Infea[e] = (X[e] < 0) && PS[e];
      ng += NonOpt[e] + Infea[e];
    }
    NotGood[c] = ng;
    NotOpt[c] = ng > 0;
  };
  int64_t numNonOpt = 0;
  for (int64_t c = 0; c < ncols; ++c) {
    classify(c);
    numNonOpt += NotOpt[c];
  }
  unsigned iter = 0;
  std::vector<int> pset;
  std::vector<double> xs(n);
  while (numNonOpt > 0) {
    ++iter;
    if (MAX_IT > 0 && iter > MAX_IT) return -1;
    for (int64_t c = 0; c < ncols; ++c) {
      if (!NotOpt[c]) continue;
      bool c1 = NotGood[c] < Ninf[c];
      bool c2 = !c1 && (NotGood[c] >= Ninf[c]) && (P[c] >= 1);
      if (c1) {  // bppnnls.hpp:115-129
        P[c] = pbar;
        Ninf[c] = NotGood[c];
      } else if (c2) {  // bppnnls.hpp:133-146
        P[c] -= 1;
      }
      if (c1 || c2) {
        for (int r = 0; r < n; ++r) {
          size_t e = r + (size_t)n * c;
          if (NonOpt[e]) PS[e] = 1;
          if (Infea[e]) PS[e] = 0;
        }
      } else {  // backup rule, bppnnls.hpp:149-160: flip the largest index
        int rowidx = -1;
        for (int r = 0; r < n; ++r) {
          size_t e = r + (size_t)n * c;
          if (NonOpt[e] + Infea[e]) rowidx = r;
        }
        size_t e = rowidx + (size_t)n * c;
        PS[e] = PS[e] ? 0 : 1;
      }
    }
    // solve on passive sets, bppnnls.hpp:163-168 / 204-259
    for (int64_t c = 0; c < ncols; ++c) {
      if (!NotOpt[c]) continue;
      pset.clear();
      for (int r = 0; r < n; ++r)
        if (PS[r + (size_t)n * c]) pset.push_back(r);
      std::fill(xs.begin(), xs.end(), 0.0);
      if (solve_subset(AtA, n, pset, AtB + (size_t)n * c, xs.data()) != 0)
        return -2;
      for (int r = 0; r < n; ++r) X[r + (size_t)n * c] = xs[r];
      for (int r = 0; r < n; ++r) {
        double acc = 0.0;
        for (int j = 0; j < n; ++j) acc += AtA[r + (size_t)n * j] * xs[j];
        Y[r + (size_t)n * c] = acc - AtB[r + (size_t)n * c];
      }
    }
    // bppnnls.hpp:170-172: zero |.| < 1e-12 in all of X and Y
    for (size_t i = 0; i < (size_t)n * ncols; ++i) {
      if (std::fabs(X[i]) < kEps12) X[i] = 0.0;
      if (std::fabs(Y[i]) < kEps12) Y[i] = 0.0;
    }
    numNonOpt = 0;
    for (int64_t c = 0; c < ncols; ++c) {
      classify(c);
      numNonOpt += NotOpt[c];
    }
  }
  if (passive_out)
    for (size_t i = 0; i < (size_t)n * ncols; ++i) passive_out[i] = PS[i];
  return (int)iter;
}

// ANLS/BPP update, ntf/ntfanlsbpp.hpp:15-57: chunks of 2000 RHS, X0 = 0.
// M is row-major I x k == column-major k x I (ncp_mttkrp_t); H (out) row-major.
int bpp_update(double* H, int64_t I, int k, const double* M, const double* G,
               int* passive_out) {
  int maxit = 0;
  for (int64_t start = 0; start < I; start += kChunk) {
    int64_t cnt = std::min(kChunk, I - start);
    int it = bpp_solve(G, M + start * k, k, cnt, H + start * k,
                       passive_out ? passive_out + start * k : nullptr);
    if (it < 0) return it;
    maxit = std::max(maxit, it);
  }
  return maxit;
}

// Relative error by explicit reconstruction, ntf/auntf.hpp:200-246:
// lowrank = (F0 diag(lambda)) * KRP_{-0}^T, err = sqrt(||X - lowrank||^2 /
// ||X||^2) with the squared norms of common/tensor.hpp:350-369.
double explicit_error(const double* X, const int64_t* dims, int N,
                      const double* const* F, const double* lambda, int k,
                      double normA) {
  int64_t I0 = dims[0];
  int64_t rest = prod(dims, 1, N);
  std::vector<double> KRP((size_t)rest * k);
  krp_leave_out_one(F, dims, N, k, 0, KRP.data());
  std::vector<double> U((size_t)I0 * k);  // column-major I0 x k
  for (int64_t i = 0; i < I0; ++i)
    for (int r = 0; r < k; ++r) U[i + I0 * r] = F[0][i * k + r] * lambda[r];
  double err = 0.0;
  const int64_t blk = 4096;
  std::vector<double> low((size_t)I0 * blk);
  for (int64_t c0 = 0; c0 < rest; c0 += blk) {
    int64_t nc = std::min(blk, rest - c0);
    cblas_dgemm(CblasColMajor, CblasNoTrans, CblasTrans, (int)I0, (int)nc, k,
                1.0, U.data(), (int)I0, KRP.data() + c0, (int)rest, 0.0,
                low.data(), (int)I0);
    const double* Xb = X + c0 * I0;
    for (int64_t i = 0; i < I0 * nc; ++i) {
      double dlt = Xb[i] - low[i];
      err += dlt * dlt;
    }
  }
  return std::sqrt(err / normA);
}


// ---------------------------------------------------------------------------
// AO-ADMM update, ntf/ntfaoadmm.hpp:23-77 (NTFAOADMM::update). H (in) is the
// current normalised factor, (out) the new unnormalised one; U is the ADMM
// auxiliary (dual) variable m_ncp_aux of this mode, I x k, kept between calls
// and column-normalised after the loop (ntfaoadmm.hpp:74). All row-major
// I x k, which is the memory of the reference's k x I transposed matrices.
// Returns the number of ADMM iterations run, or -2 if chol() fails.
int admm_update(double* H, double* U, int64_t I, int k, const double* M,
                const double* G, int admm_iter, double tol) {
  // alpha = trace(G) / k, 0.01 if not positive (ntfaoadmm.hpp:30-32)
  double tr = 0.0;
  for (int i = 0; i < k; ++i) tr += G[i * k + i];
  double alpha = tr / k;
  alpha = (alpha > 0) ? alpha : 0.01;
  // L = chol(G + alpha I, "lower") (ntfaoadmm.hpp:33-35), LAPACK dpotrf
  std::vector<double> A((size_t)k * k);
  for (int e = 0; e < k * k; ++e) A[e] = G[e];
  for (int i = 0; i < k; ++i) A[i * k + i] += alpha;
  int n = k, info = 0;
  dpotrf_("L", &n, A.data(), &n, &info);  // column-major lower = row-major upper
  if (info != 0) return -2;
  std::vector<double> L((size_t)k * k, 0.0);  // row-major lower: L[i*k+j], i >= j
  for (int i = 0; i < k; ++i)
    for (int j = 0; j <= i; ++j) L[i * k + j] = A[i + (size_t)j * k];
  std::vector<double> prev((size_t)I * k), b(k);
  bool stop = false;
  int it = 0;
  for (int i = 0; i < admm_iter && !stop; i++, it++) {
    std::copy(H, H + (size_t)I * k, prev.begin());
    double fac = 0.0, dual = 0.0, rr = 0.0, ss = 0.0;
    for (int64_t row = 0; row < I; ++row) {
      double* h = H + row * k;
      double* u = U + row * k;
      const double* m = M + row * k;
      // rhs = M^T + alpha (H^T + U^T) (ntfaoadmm.hpp:44-47)
      for (int c = 0; c < k; ++c) b[c] = m[c] + alpha * (h[c] + u[c]);
      // solve(trimatl(L), .) then solve(trimatu(L^T), .): the column
      // substitutions of BLAS dtrsm (Left, Lower / Upper, NoTrans)
      for (int j = 0; j < k; ++j) {
        b[j] = b[j] / L[j * k + j];
        for (int c = j + 1; c < k; ++c) b[c] -= b[j] * L[c * k + j];
      }
      for (int j = k - 1; j >= 0; --j) {
        b[j] = b[j] / L[j * k + j];
        for (int c = 0; c < j; ++c) b[c] -= b[j] * L[j * k + c];
      }
      for (int c = 0; c < k; ++c) {
        // H = max(aux_t^T - U, 0); U = U + H - aux_t^T (ntfaoadmm.hpp:52-61)
        double hn = b[c] - u[c];
        hn = hn > 0.0 ? hn : 0.0;
        double un = (u[c] + hn) - b[c];
        fac += hn * hn;
        dual += un * un;
        double d = hn - b[c];
        rr += d * d;
        double e = hn - prev[row * k + c];
        ss += e * e;
        h[c] = hn;
        u[c] = un;
      }
    }
    // stopping test (ntfaoadmm.hpp:63-71)
    double facnorm = std::sqrt(fac), dualnorm = std::sqrt(dual);
    double r = std::sqrt(rr), sres = std::sqrt(ss);
    if (r < (tol * facnorm) && sres < (tol * dualnorm)) stop = true;
  }
  std::vector<double> lam(k);
  normalize_mode(U, I, k, lam.data());  // m_ncp_aux.normalize(mode)
  return it;
}

// ---------------------------------------------------------------------------
// Nesterov-accelerated NTF, ntf/ntfnes.hpp:11-166 (NTFNES). Every NCPFactors
// of the class is "trans" (k x I_n), i.e. row-major I_n x k here; their
// lambdas are k-vectors. State of one solver object:
struct NesState {
  int N = 0, k = 0;
  std::vector<std::vector<double>> prox, prev, acc;  // m_prox_t, m_prev_t, m_acc_t
  std::vector<double> prox_lam, prev_lam, acc_lam;
  // ntfnes.hpp:184-191
  double delta1 = 1e-2, delta2 = 1e-2;
  int acc_start = 5, acc_exp = 3, acc_fails = 0, fail_limit = 5;
  int max_inner = 20000;  // the reference loops without a bound (ntfnes.hpp:121)
};

void nes_init(NesState& st, const int64_t* dims, int N, int k) {
  st.N = N;
  st.k = k;
  st.prox.assign(N, {});
  st.prev.assign(N, {});
  st.acc.assign(N, {});
  for (int n = 0; n < N; ++n) {
    st.prox[n].assign((size_t)dims[n] * k, 0.0);  // zeros() (ntfnes.hpp:179-182)
    st.prev[n].assign((size_t)dims[n] * k, 0.0);
    st.acc[n].assign((size_t)dims[n] * k, 0.0);
  }
  st.prox_lam.assign(k, 1.0);  // NCPFactors ctor: lambda = ones
  st.prev_lam.assign(k, 1.0);
  st.acc_lam.assign(k, 1.0);
}

// NCPFactors::normalize_rows of a trans factor (ncpfactors.hpp:358-363):
// rank component r is column r of the row-major I x k array.
void normalize_rows_t(double* F, int64_t I, int k, double* lambda) {
  normalize_mode(F, I, k, lambda);
}

// ntfnes.hpp:25-37
double nes_get_lambda(double L, double mu) {
  double q = L / mu;
  double lambda = 0.0;
  if (q > 1e6)
    lambda = 10 * mu;
  else if (q > 1e3)
    lambda = mu;
  else
    lambda = mu / 10;
  return lambda;
}

// ntfnes.hpp:39-50
double nes_get_alpha(double alpha, double q) {
  double a, b, c, D, x;
  a = 1.0;
  b = alpha * alpha - q;
  c = -alpha * alpha;
  D = b * b - 4 * a * c;
  x = (-b + std::sqrt(D)) / 2;
  return x;
}

// Extreme eigenvalues of a symmetric k x k matrix: arma::eig_sym (LAPACK
// dsyev, eigenvalues only, ascending).
void sym_eig_minmax(const double* G, int k, double* lmin, double* lmax) {
  std::vector<double> A(G, G + (size_t)k * k), w(k);
  int n = k, lwork = -1, info = 0;
  double wq = 0.0;
  dsyev_("N", "L", &n, A.data(), &n, w.data(), &wq, &lwork, &info);
  lwork = (int)wq;
  std::vector<double> work(lwork > 1 ? lwork : 1);
  dsyev_("N", "L", &n, A.data(), &n, w.data(), work.data(), &lwork, &info);
  *lmin = w[0];
  *lmax = w[k - 1];
}

// NTFNES::update (ntfnes.hpp:100-151). Writes the unnormalised Ht to H.
// Returns the number of inner gradient steps, or -1 at the step cap.
int nes_update(NesState& st, int mode, double* H, int64_t I, const double* M,
               const double* G) {
  const int k = st.k;
  const size_t n = (size_t)I * k;
  if (mode == 0) st.prev_lam = st.prox_lam;
  st.prev[mode] = st.prox[mode];
  std::vector<double> Ht(st.prox[mode]), Htprev(Ht);
  std::vector<double>& acc = st.acc[mode];
  acc = Ht;
  double L, mu;
  sym_eig_minmax(G, k, &mu, &L);
  double lambda = nes_get_lambda(L, mu);
  std::vector<double> modG(G, G + (size_t)k * k);
  for (int i = 0; i < k; ++i) modG[i * k + i] += lambda;
  double q = (mu + lambda) / (L + lambda);
  std::vector<double> modM(n), grad(n);
  for (size_t e = 0; e < n; ++e) modM[e] = (-1 * lambda) * acc[e] - M[e];
  double alpha = 1, alpha_prev = 1, beta = 1;
  const double inv = 1 / (L + lambda);
  int steps = 0;
  while (true) {
    // grad = modM + modG * acc
    for (int64_t row = 0; row < I; ++row)
      for (int c = 0; c < k; ++c) {
        double s = 0.0;
        for (int j = 0; j < k; ++j) s += modG[c * k + j] * acc[row * k + j];
        grad[row * k + c] = modM[row * k + c] + s;
      }
    // stop_iter (ntfnes.hpp:52-62)
    double absmax = 0.0, amin = grad.empty() ? 0.0 : grad[0];
    for (size_t e = 0; e < n; ++e) {
      absmax = std::max(absmax, std::fabs(grad[e] * acc[e]));
      amin = std::min(amin, grad[e]);
    }
    if (absmax <= st.delta1 && amin >= -st.delta2) break;
    if (steps >= st.max_inner) return -1;
    ++steps;
    Htprev = Ht;
    for (size_t e = 0; e < n; ++e) {
      double v = acc[e] - (inv * grad[e]);
      Ht[e] = v > 0.0 ? v : 0.0;
    }
    alpha_prev = alpha;
    alpha = nes_get_alpha(alpha_prev, q);
    beta = (alpha_prev * (1 - alpha_prev)) / (alpha + alpha_prev * alpha_prev);
    for (size_t e = 0; e < n; ++e) acc[e] = Ht[e] + beta * (Ht[e] - Htprev[e]);
  }
  st.prox[mode] = Ht;
  normalize_rows_t(st.prox[mode].data(), I, k, st.prox_lam.data());
  std::copy(Ht.begin(), Ht.end(), H);
  return steps;
}


// NTFNES::accelerate (ntfnes.hpp:64-98), after the error of iteration `iter`
// (cur_err). The extrapolated factors are installed and evaluated through
// computeObjectiveError(m_acc_t) = reset(acc, true) + the explicit error
// (auntf.hpp:186-198, 200-249); on failure reset(m_prox_t, true) restores the
// proximal iterate.
void nes_accelerate(NesState& st, int iter, double cur_err, const double* X,
                    const int64_t* dims, int N, int k, double* const* F,
                    double* lambda, double normA) {
  if (iter <= st.acc_start) return;
  double acc_step = std::pow(iter + 1, (1.0 / st.acc_exp));
  for (int mode = 0; mode < N; mode++) {
    const bool last = mode == N - 1;  // only the last mode is unnormalised
    const size_t n = (size_t)dims[mode] * k;
    std::vector<double>& acc = st.acc[mode];
    for (size_t e = 0; e < n; ++e) {
      const int r = (int)(e % k);
      double cur = last ? lambda[r] * F[mode][e] : F[mode][e];
      double prv = last ? st.prev_lam[r] * st.prev[mode][e] : st.prev[mode][e];
      double a = cur - prv;
      a *= acc_step;
      a += cur;
      acc[e] = a;
    }
    normalize_rows_t(acc.data(), dims[mode], k, st.acc_lam.data());
  }
  for (int i = 0; i < N; ++i) {
    std::copy(st.acc[i].begin(), st.acc[i].end(), F[i]);
    normalize_mode(F[i], dims[i], k, lambda);
  }
  std::copy(st.acc_lam.begin(), st.acc_lam.end(), lambda);
  double acc_err = explicit_error(X, dims, N, F, lambda, k, normA);
  if (acc_err < cur_err) {
    for (int mode = 0; mode < N; mode++) {
      st.prox[mode] = st.acc[mode];
      normalize_rows_t(st.prox[mode].data(), dims[mode], k, st.prox_lam.data());
    }
  } else {
    for (int i = 0; i < N; ++i) {
      std::copy(st.prox[i].begin(), st.prox[i].end(), F[i]);
      normalize_mode(F[i], dims[i], k, lambda);
    }
    std::copy(st.prox_lam.begin(), st.prox_lam.end(), lambda);
    st.acc_fails++;
    if (st.acc_fails > st.fail_limit) {
      st.acc_fails = 0;
      st.acc_exp++;
    }
  }
}


// ===========================================================================
// Shared-memory NMF of a dense matrix, A ~ W H^T (common/nmf.hpp,
// nmf/hals.hpp, nmf/mu.hpp, nmf/bppnmf.hpp). A is column-major m x n
// (Armadillo MAT); W (m x k) and H (n x k) are row-major here, the memory of
// the reference's W^T and H^T.
// ===========================================================================
struct NmfReg {
  double w2 = 0, w1 = 0, h2 = 0, h1 = 0, sym = 0;  // regW(0..1), regH(0..1), symm_reg
};

// out (row-major m x k) = A H (nmf/hals.hpp:86 "AH = A * H")
void nmf_AH(const double* A, int64_t m, int64_t n, int k, const double* H, double* out) {
  cblas_dgemm(CblasColMajor, CblasNoTrans, CblasTrans, k, (int)m, (int)n, 1.0, H, k, A, (int)m,
              0.0, out, k);
}
// out (row-major n x k) = A^T W (nmf/mu.hpp:60 "AtW = At * W")
void nmf_AtW(const double* A, int64_t m, int64_t n, int k, const double* W, double* out) {
  cblas_dgemm(CblasColMajor, CblasNoTrans, CblasNoTrans, k, (int)n, (int)m, 1.0, W, k, A, (int)m,
              0.0, out, k);
}

// NMF::applyReg (common/nmf.hpp:76-92): L2 adds l2 I, L1 adds l1 ones.
void nmf_apply_reg(double* G, int k, double l2, double l1) {
  if (l2 > 0)
    for (int i = 0; i < k; ++i) G[i * k + i] += l2;
  if (l1 > 0)
    for (int e = 0; e < k * k; ++e) G[e] += l1;
}

// NMF::normalize_by_W (common/nmf.hpp:150-160)
void nmf_normalize_by_W(double* W, int64_t m, double* H, int64_t n, int k) {
  for (int i = 0; i < k; ++i) {
    double ss = 0.0;
    for (int64_t r = 0; r < m; ++r) ss += W[r * k + i] * W[r * k + i];
    const double nrm = std::sqrt(ss);
    if (nrm > 0) {
      for (int64_t r = 0; r < m; ++r) W[r * k + i] = W[r * k + i] / nrm;
      for (int64_t r = 0; r < n; ++r) H[r * k + i] = H[r * k + i] * nrm;
    }
  }
}

// HALSNMF W sweep (nmf/hals.hpp:92-105): column by column,
// Wx = W(:,x) HtH(x,x) + (AH(:,x) - W HtH(:,x)), entries < 1e-17 set to
// 1e-17, then W(:,x) = Wx / ||Wx|| when ||Wx|| != 0.
void nmf_hals_w(double* W, int64_t m, int k, const double* AH, const double* G) {
  std::vector<double> wx((size_t)m);
  for (int x = 0; x < k; ++x) {
    for (int64_t r = 0; r < m; ++r) {
      double s = 0.0;
      for (int j = 0; j < k; ++j) s += W[r * k + j] * G[j * k + x];
      double v = (W[r * k + x] * G[x * k + x]) + (AH[r * k + x] - s);
      wx[r] = (v < kEps17) ? kEps17 : v;
    }
    double ss = 0.0;
    for (int64_t r = 0; r < m; ++r) ss += wx[r] * wx[r];
    const double nrm = std::sqrt(ss);
    if (nrm != 0)
      for (int64_t r = 0; r < m; ++r) W[r * k + x] = wx[r] / nrm;
  }
}

// MUNMF update of one factor (nmf/mu.hpp:68, 80): U = (U % M) / (U G + 1e-17)
void nmf_mu(double* U, int64_t I, int k, const double* M, const double* G) {
  std::vector<double> t((size_t)k);
  for (int64_t r = 0; r < I; ++r) {
    for (int c = 0; c < k; ++c) {
      double acc = 0.0;
      for (int j = 0; j < k; ++j) acc += U[r * k + j] * G[j * k + c];
      t[c] = acc + kEps17;
    }
    for (int c = 0; c < k; ++c) U[r * k + c] = (U[r * k + c] * M[r * k + c]) / t[c];
  }
}

// NMF::computeObjectiveError (common/nmf.hpp:386-425) from AtW = A^T W of the
// current W. Writes the objective and the relative error sqrt(fit)/||A||.
void nmf_error(const double* W, int64_t m, const double* H, int64_t n, int k, const double* AtW,
               double normA, const NmfReg& reg, double* objective, double* relerr) {
  std::vector<double> WtW((size_t)k * k), HtH((size_t)k * k);
  gram(W, m, k, WtW.data());
  gram(H, n, k, HtH.data());
  const double sqnormA = normA * normA;
  double tr_htatw = 0.0;
  for (int64_t e = 0; e < n * k; ++e) tr_htatw += H[e] * AtW[e];
  double tr_ww_hh = 0.0;
  for (int a = 0; a < k; ++a)
    for (int b = 0; b < k; ++b) tr_ww_hh += WtW[a * k + b] * HtH[b * k + a];
  double fro_w = 0.0, fro_h = 0.0;
  for (int i = 0; i < k; ++i) {
    fro_w += WtW[i * k + i];
    fro_h += HtH[i * k + i];
  }
  auto l1sq = [k](const double* U, int64_t I) {
    double s = 0.0;
    for (int64_t r = 0; r < I; ++r) {
      double rs = 0.0;
      for (int c = 0; c < k; ++c) rs += U[r * k + c];
      s += rs * rs;
    }
    return s;  // ||sum(U, 1)||_2^2
  };
  const double fit = sqnormA - (2 * tr_htatw) + tr_ww_hh;
  double sym_obj = 0.0;
  if (reg.sym > 0) {
    double d = 0.0;
    for (int64_t e = 0; e < m * k; ++e) d += (W[e] - H[e]) * (W[e] - H[e]);
    sym_obj = reg.sym * d;
  }
  *objective = fit + reg.w2 * fro_w + reg.h2 * fro_h + reg.w1 * l1sq(W, m) +
               reg.h1 * l1sq(H, n) + sym_obj;
  const double err = fit > 0 ? std::sqrt(fit) : normA;
  *relerr = err / normA;
}

// BPPNMF::updateOtherGivenOneMultipleRHS (nmf/bppnmf.hpp:24-80): solves the
// rows of `out` (I x k) from G = given^T given + reg (+ symm_reg I) and the
// right-hand sides M (+ symm_reg given). Returns -1 on a BPP failure.
int nmf_bpp(double* out, int64_t I, int k, const double* M, const double* given,
            int64_t gI, double l2, double l1, double sym) {
  std::vector<double> G((size_t)k * k), R(M, M + (size_t)I * k);
  gram(given, gI, k, G.data());
  nmf_apply_reg(G.data(), k, l2, l1);
  if (sym > 0) {
    for (int i = 0; i < k; ++i) G[i * k + i] += sym;
    for (int64_t e = 0; e < I * k; ++e) R[e] += sym * given[e];
  }
  return bpp_solve(G.data(), R.data(), k, I, out, nullptr) < 0 ? -1 : 0;
}

}  // namespace

extern "C" {

int orc_version() { return 1; }

// Tensor(dims) uniform fill: one std::mt19937(seed) and
// std::uniform_real_distribution<>(0, 1) drawn in linear (mode-0-fastest)
// order, common/tensor.hpp:86-93 and 219-235 (the single-threaded order; the
// reference's OpenMP loop shares one generator across threads).
void orc_tensor_randu(int64_t numel, unsigned seed, double* out) {
  std::uniform_real_distribution<> dis(0, 1);
  std::mt19937 gen(seed);
  for (int64_t i = 0; i < numel; ++i) out[i] = dis(gen);
}

// Synthetic CP tensor on the host: X = [[A_0..A_{N-1}]] + sigma * N(0,1),
// clipped at 0 when `clip`; the same pure function of (factors, sigma, seed)
// as the library's device generator (planc_gpu_synth_cp_tensor): normals from
// Philox-4x32-10 (Salmon et al., SC'11) keyed by the seed and counted by the
// element index, through the Box-Muller transform. The noise model is the
// reference's (dimtree/ddttensor.hpp:951-952, sigma = rho ||M|| / sqrt(numel)).
// A[m]: row-major I_m x k. X: column-major, mode 0 fastest. With round_f32
// every value is rounded to FP32 (and stored widened), as the device
// generator's FP32 output is. OpenMP-parallel.
static inline void philox4x32_10(uint32_t c[4], uint32_t key[2]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int round = 0; round < 10; ++round) {
    const uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ key[0];
    const uint32_t n1 = (uint32_t)p1;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ key[1];
    const uint32_t n3 = (uint32_t)p0;
    c[0] = n0, c[1] = n1, c[2] = n2, c[3] = n3;
    key[0] += W0;
    key[1] += W1;
  }
}

void orc_synth_cp(const int64_t* dims, int N, const double* const* A, int k, double sigma,
                  uint64_t seed, int clip, int round_f32, double* X) {
  int64_t numel = 1;
  for (int m = 0; m < N; ++m) numel *= dims[m];
  const double pi = 3.14159265358979323846;
#pragma omp parallel for schedule(static)
  for (int64_t idx = 0; idx < numel; ++idx) {
    int64_t rem = idx, sub[16];
    for (int m = 0; m < N; ++m) {
      sub[m] = rem % dims[m];
      rem /= dims[m];
    }
    double v = 0.0;
    for (int r = 0; r < k; ++r) {
      double p = 1.0;
      for (int m = N - 1; m >= 1; --m) p = A[m][sub[m] * k + r] * p;
      v = std::fma(A[0][sub[0] * k + r], p, v);
    }
    if (sigma > 0) {
      uint32_t c[4] = {(uint32_t)idx, (uint32_t)(idx >> 32), 0x5eedu, 0u};
      uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
      philox4x32_10(c, key);
      const double u1 = ((double)c[0] + 1.0) * (1.0 / 4294967296.0);  // (0, 1]
      const double u2 = (double)c[1] * (1.0 / 4294967296.0);          // [0, 1)
      const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(pi * (2.0 * u2));
      v = std::fma(sigma, z, v);
    }
    if (clip && v < 0) v = 0;
    X[idx] = round_f32 ? (double)(float)v : v;
  }
}

void orc_gram_loo(const double* const* F, const int64_t* dims, int N, int k,
                  int n, double* G) {
  gram_loo(F, dims, N, k, n, G);
}

void orc_krp_leave_out_one(const double* const* F, const int64_t* dims, int N,
                           int k, int n, double* KRP_colmajor) {
  krp_leave_out_one(F, dims, N, k, n, KRP_colmajor);
}

void orc_mttkrp_direct(const double* X, const int64_t* dims, int N,
                       const double* const* F, int k, int n, double* out) {
  mttkrp_direct(X, dims, N, F, k, n, out);
}

// All-mode dimension-tree MTTKRP with fixed factors (no updates between
// modes), for comparison with the direct form.
int orc_mttkrp_dimtree_all(const double* X, const int64_t* dims, int N,
                           const double* const* F, int k, double* const* out) {
  if (N != 3 && N != 4) return -1;
  DimTree t;
  t.N = N;
  t.k = k;
  t.s = N / 2;
  t.dims = dims;
  t.L = prod(dims, 0, t.s + 1);
  t.R = prod(dims, t.s + 1, N);
  t.P.assign((size_t)t.L * k, 0.0);
  for (int n = 0; n < N; ++n) dimtree_mttkrp(t, X, F, n, out[n]);
  return 0;
}

void orc_normalize(double* F, int64_t I, int k, double* lambda) {
  normalize_mode(F, I, k, lambda);
}

void orc_hals_update(double* H, int64_t I, int k, const double* M,
                     const double* G) {
  hals_update(H, I, k, M, G);
}

void orc_mu_update(double* H, int64_t I, int k, const double* M,
                   const double* G) {
  mu_update(H, I, k, M, G);
}

int orc_bpp_update(double* H, int64_t I, int k, const double* M,
                   const double* G, int* passive_out) {
  return bpp_update(H, I, k, M, G, passive_out);
}

int orc_bpp_solve(const double* AtA, const double* AtB, int n, int64_t ncols,
                  double* X, int* passive_out) {
  return bpp_solve(AtA, AtB, n, ncols, X, passive_out);
}

double orc_explicit_error(const double* X, const int64_t* dims, int N,
                          const double* const* F, const double* lambda, int k) {
  int64_t numel = prod(dims, 0, N);
  double normA = 0.0;
  for (int64_t i = 0; i < numel; ++i) normA += X[i] * X[i];
  return explicit_error(X, dims, N, F, lambda, k, normA);
}

// The AUNTF loop, ntf/auntf.hpp:128-177, starting from injected factors as
// AUNTF::reset(init, false) leaves them (auntf.hpp:186-198): every mode
// column-normalised by update_factor_mode (auntf.hpp:66-79), lambda := the
// injected lambda.
//   F (in/out): N row-major I_n x k factors (initial values in, final out)
//   lambda (in/out): k
//   errs: iters entries (relative error per iteration, if compute_error)
// Returns 0, or a negative code on BPP failure (-1 iteration cap).
int orc_ntf_run(const double* X, const int64_t* dims, int N, int k,
                double* const* F, double* lambda, int algo, int iters,
                int dimtree, int compute_error, double* errs) {
  std::vector<double> tmp(k);
  for (int n = 0; n < N; ++n) normalize_mode(F[n], dims[n], k, tmp.data());
  int64_t numel = prod(dims, 0, N);
  double normA = 0.0;  // Tensor::norm (squared), tensor.hpp:350-356
  for (int64_t i = 0; i < numel; ++i) normA += X[i] * X[i];
  bool use_dt = dimtree && (N == 3 || N == 4);
  DimTree t;
  if (use_dt) {
    t.N = N;
    t.k = k;
    t.s = N / 2;
    t.dims = dims;
    t.L = prod(dims, 0, t.s + 1);
    t.R = prod(dims, t.s + 1, N);
    t.P.assign((size_t)t.L * k, 0.0);
  }
  std::vector<double> G((size_t)k * k);
  int64_t maxI = 0;
  for (int n = 0; n < N; ++n) maxI = std::max(maxI, dims[n]);
  std::vector<double> M((size_t)maxI * k);
  const double* const* Fc = F;
  // solver-object state of NTFAOADMM (m_ncp_aux, zeros, ntfaoadmm.hpp:86) and
  // NTFNES (ntfnes.hpp:173-191)
  std::vector<std::vector<double>> aux;
  if (algo == AOADMM)
    for (int n = 0; n < N; ++n) aux.emplace_back((size_t)dims[n] * k, 0.0);
  NesState nes;
  if (algo == NESTEROV) nes_init(nes, dims, N, k);
  for (int it = 0; it < iters; ++it) {
    for (int n = 0; n < N; ++n) {
      gram_loo(Fc, dims, N, k, n, G.data());
      if (use_dt)
        dimtree_mttkrp(t, X, Fc, n, M.data());
      else
        mttkrp_direct(X, dims, N, Fc, k, n, M.data());
      if (algo == HALS) {
        hals_update(F[n], dims[n], k, M.data(), G.data());
      } else if (algo == MU) {
        mu_update(F[n], dims[n], k, M.data(), G.data());
      } else if (algo == ANLSBPP) {
        int rc = bpp_update(F[n], dims[n], k, M.data(), G.data(), nullptr);
        if (rc < 0) return rc;
      } else if (algo == AOADMM) {
        int rc = admm_update(F[n], aux[n].data(), dims[n], k, M.data(), G.data(), 5, 0.01);
        if (rc < 0) return rc;
      } else if (algo == NESTEROV) {
        int rc = nes_update(nes, n, F[n], dims[n], M.data(), G.data());
        if (rc < 0) return -4;
      } else {
        return -3;
      }
      normalize_mode(F[n], dims[n], k, lambda);
    }
    // NTFNES switches the error on (accelerated(true), ntfnes.hpp:193) and
    // its acceleration reads it
    if (compute_error || algo == NESTEROV) {
      double e = explicit_error(X, dims, N, Fc, lambda, k, normA);
      if (compute_error) errs[it] = e;
      if (algo == NESTEROV) nes_accelerate(nes, it, e, X, dims, N, k, F, lambda, normA);
    }
  }
  return 0;
}

// One AO-ADMM mode update (NTFAOADMM::update, ntf/ntfaoadmm.hpp:23-77) with
// the ADMM iteration count and tolerance as parameters (the reference fixes
// 5 and 0.01, ntfaoadmm.hpp:87-88). H, U in/out. Returns iterations run.
int orc_admm_update(double* H, double* U, int64_t I, int k, const double* M,
                    const double* G, int admm_iter, double tol) {
  return admm_update(H, U, I, k, M, G, admm_iter, tol);
}

// One Nesterov mode update from a given proximal point H0 (NTFNES::update,
// ntf/ntfnes.hpp:100-151) with the stopping thresholds as parameters (the
// reference uses delta1 = delta2 = 1e-2, ntfnes.hpp:184-185). Writes the
// unnormalised update to H; returns the inner step count (-1 at the cap).
int orc_nes_update(const double* H0, double* H, int64_t I, int k, const double* M,
                   const double* G, double delta1, double delta2, int max_inner) {
  NesState st;
  int64_t dims[1] = {I};
  nes_init(st, dims, 1, k);
  std::copy(H0, H0 + (size_t)I * k, st.prox[0].begin());
  st.delta1 = delta1;
  st.delta2 = delta2;
  st.max_inner = max_inner;
  return nes_update(st, 0, H, I, M, G);
}

// Extreme eigenvalues of a symmetric k x k matrix (arma::eig_sym, LAPACK dsyev).
void orc_sym_eig_minmax(const double* G, int k, double* lmin, double* lmax) {
  sym_eig_minmax(G, k, lmin, lmax);
}


// The NMF loop of HALSNMF / MUNMF / BPPNMF::computeNMF (nmf/hals.hpp:50-110,
// nmf/mu.hpp:55-92, nmf/bppnmf.hpp:190-240) from injected W0, H0 (the
// NMF(A, W, H) constructor, common/nmf.hpp:193-210; HALSNMF normalises by W
// first, nmf/hals.hpp:44-48). A column-major m x n; W, H row-major (in/out).
// reg = {regW L2, regW L1, regH L2, regH L1, symm_reg} (may be NULL). The
// objective and relative error of every iteration go to obj / relerr.
int orc_nmf_run(const double* A, int64_t m, int64_t n, int k, double* W, double* H, int algo,
                int iters, const double* reg5, double* obj, double* relerr) {
  NmfReg reg;
  if (reg5) {
    reg.w2 = reg5[0];
    reg.w1 = reg5[1];
    reg.h2 = reg5[2];
    reg.h1 = reg5[3];
    reg.sym = reg5[4];
  }
  if (reg.sym > 0 && m != n) return -2;
  double normA = 0.0;
  for (int64_t e = 0; e < m * n; ++e) normA += A[e] * A[e];
  normA = std::sqrt(normA);  // arma::norm(A, "fro")
  std::vector<double> AH((size_t)m * k), AtW((size_t)n * k), G((size_t)k * k);
  if (algo == HALS) nmf_normalize_by_W(W, m, H, n, k);
  for (int it = 0; it < iters; ++it) {
    if (algo == HALS || algo == MU) {
      nmf_AtW(A, m, n, k, W, AtW.data());
      gram(W, m, k, G.data());
      nmf_apply_reg(G.data(), k, reg.h2, reg.h1);
      if (algo == HALS)
        hals_update(H, n, k, AtW.data(), G.data());
      else
        nmf_mu(H, n, k, AtW.data(), G.data());
      nmf_AH(A, m, n, k, H, AH.data());
      gram(H, n, k, G.data());
      nmf_apply_reg(G.data(), k, reg.w2, reg.w1);
      if (algo == HALS) {
        nmf_hals_w(W, m, k, AH.data(), G.data());
        nmf_normalize_by_W(W, m, H, n, k);
      } else {
        nmf_mu(W, m, k, AH.data(), G.data());
      }
    } else if (algo == ANLSBPP) {
      nmf_AH(A, m, n, k, H, AH.data());
      if (nmf_bpp(W, m, k, AH.data(), H, n, reg.w2, reg.w1, reg.sym) < 0) return -1;
      nmf_AtW(A, m, n, k, W, AtW.data());
      if (nmf_bpp(H, n, k, AtW.data(), W, m, reg.h2, reg.h1, reg.sym) < 0) return -1;
    } else {
      return -3;
    }
    nmf_AtW(A, m, n, k, W, AtW.data());
    nmf_error(W, m, H, n, k, AtW.data(), normA, reg, &obj[it], &relerr[it]);
  }
  if (algo == MU || algo == ANLSBPP) nmf_normalize_by_W(W, m, H, n, k);
  return 0;
}

}  // extern "C"
