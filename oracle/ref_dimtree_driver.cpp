// ref_dimtree_driver.cpp -- drives the REFERENCE's own dimension-tree MTTKRP
// kernels (dimtree/dimtrees.hpp, dimtree/ddttensor.hpp, compiled unmodified
// from the reference tree by oracle/Makefile into oracle/_ref/).
//
// TEST INFRASTRUCTURE ONLY (a checker, never part of the product).
//
// DenseDimensionTree (dimtree/ddt.hpp) itself cannot be compiled here because
// it includes the Armadillo-typed NCPFactors/Tensor headers and Armadillo is
// not installed. This file therefore repeats its bookkeeping in plain C++:
// the constructor (ddt.hpp:24-91), set_factor (ddt.hpp:93-98) and the call
// sequence of in_order_reuse_MTTKRP (ddt.hpp:134-243), calling the reference's
// C kernels (partial_MTTKRP_with_KRP_output_{FM,T}, multi_TTV_with_KRP_output_
// {FM,T}, LR_* reorderings) for all arithmetic.
#include <cstdlib>
#include <cstring>

#include "dimtree/dimtrees.hpp"

namespace {

struct RefDimTree {
  ktensor Y;        // m_local_Y
  tensor T;         // m_local_T
  tensor proj;      // projection_Tensor
  tensor buf;       // buffer_Tensor
  ktensor projK;    // projection_Ktensor
  long int s;
  long int nthreads;
};

}  // namespace

extern "C" {

// X: column-major mode-0-fastest tensor (not copied; must outlive the handle).
// F: N row-major I_n x k factors (copied).
void* ref_dimtree_create(double* X, const long int* dims, long int N,
                         long int k, double* const* F, long int nthreads) {
  RefDimTree* h = new RefDimTree();
  h->s = N / 2;  // ntf/auntf.hpp:122-123
  h->nthreads = nthreads > 0 ? nthreads : 16;  // ddt.hpp:53 hardcodes 16
  h->T.data = X;
  h->T.nmodes = N;
  h->T.dims = (long int*)malloc(sizeof(long int) * N);
  h->T.dims_product = 1;
  h->Y.nmodes = N;
  h->Y.rank = k;
  h->Y.dims = (long int*)malloc(sizeof(long int) * N);
  h->Y.factors = (double**)malloc(sizeof(double*) * N);
  h->Y.lambdas = (double*)malloc(sizeof(double) * k);
  for (long int r = 0; r < k; ++r) h->Y.lambdas[r] = 1.0;
  h->Y.dims_product = 1;
  for (long int i = 0; i < N; ++i) {
    h->T.dims[i] = dims[i];
    h->Y.dims[i] = dims[i];
    h->T.dims_product *= dims[i];
    h->Y.dims_product *= dims[i];
    h->Y.factors[i] = (double*)malloc(sizeof(double) * k * dims[i]);
    memcpy(h->Y.factors[i], F[i], sizeof(double) * k * dims[i]);
  }
  long int ldp = 1, rdp = 1;  // set_left_right_product, ddt.hpp:118-128
  for (long int i = 0; i < N; ++i) {
    if (i <= h->s)
      ldp *= dims[i];
    else
      rdp *= dims[i];
  }
  long int big = ldp > rdp ? ldp : rdp;
  h->proj.data = (double*)malloc(sizeof(double) * big * k);
  h->buf.data = (double*)malloc(sizeof(double) * big * k);
  h->proj.nmodes = N;
  h->buf.nmodes = N;
  h->proj.dims = (long int*)malloc(sizeof(long int) * N);
  h->buf.dims = (long int*)malloc(sizeof(long int) * N);
  for (long int i = 0; i < N; ++i) {
    h->proj.dims[i] = dims[i];
    h->buf.dims[i] = dims[i];
  }
  h->proj.dims_product = h->T.dims_product;
  h->buf.dims_product = h->T.dims_product;
  ktensor_copy_constructor(&h->Y, &h->projK);
  return h;
}

void ref_dimtree_set_factor(void* hv, long int mode, const double* F) {
  RefDimTree* h = (RefDimTree*)hv;
  memcpy(h->Y.factors[mode], F, sizeof(double) * h->Y.dims[mode] * h->Y.rank);
}

// Same branch structure as in_order_reuse_MTTKRP (ddt.hpp:134-243); output
// row-major I_n x k (colmajor = false).
void ref_dimtree_mttkrp(void* hv, long int n, double* out) {
  RefDimTree* h = (RefDimTree*)hv;
  ktensor* Y = &h->Y;
  long int s = h->s;
  direction D;
  if (n == 0) {
    D = ::direction::right;
    LR_Ktensor_Reordering_existingY(Y, &h->projK, s + 1, opposite_direction(D));
    if (h->projK.nmodes == 1) {
      partial_MTTKRP_with_KRP_output_FM(D, Y, &h->T, h->nthreads);
    } else {
      partial_MTTKRP_with_KRP_output_T(s, D, Y, &h->T, &h->proj, h->nthreads);
      multi_TTV_with_KRP_output_FM(D, &h->proj, &h->projK, h->nthreads);
    }
  } else if (n == s + 1) {
    D = ::direction::left;
    LR_Ktensor_Reordering_existingY(Y, &h->projK, s, opposite_direction(D));
    if (h->projK.nmodes == 1) {
      partial_MTTKRP_with_KRP_output_FM(D, Y, &h->T, h->nthreads);
    } else {
      partial_MTTKRP_with_KRP_output_T(s, D, Y, &h->T, &h->proj, h->nthreads);
      multi_TTV_with_KRP_output_FM(opposite_direction(D), &h->proj, &h->projK,
                                   h->nthreads);
    }
  } else {
    D = ::direction::left;
    if (h->projK.nmodes == 2) {
      multi_TTV_with_KRP_output_FM(D, &h->proj, &h->projK, h->nthreads);
    } else {
      multi_TTV_with_KRP_output_T(0, D, &h->proj, &h->projK, &h->buf,
                                  h->nthreads);
      LR_tensor_Reduction(&h->buf, &h->proj, h->buf.nmodes, D);
      tensor_data_swap(&h->proj, &h->buf);
      remove_mode_Ktensor(&h->projK, 0);
      multi_TTV_with_KRP_output_FM(::direction::right, &h->proj, &h->projK,
                                   h->nthreads);
    }
  }
  memcpy(out, Y->factors[n], sizeof(double) * Y->rank * Y->dims[n]);
}

void ref_dimtree_destroy(void* hv) {
  RefDimTree* h = (RefDimTree*)hv;
  for (long int i = 0; i < h->Y.nmodes; ++i) free(h->Y.factors[i]);
  free(h->Y.factors);
  free(h->Y.dims);
  free(h->Y.lambdas);
  free(h->T.dims);
  free(h->proj.data);
  free(h->buf.data);
  free(h->proj.dims);
  free(h->buf.dims);
  free(h->projK.factors);
  free(h->projK.dims);
  free(h->projK.lambdas);
  delete h;
}

}  // extern "C"
