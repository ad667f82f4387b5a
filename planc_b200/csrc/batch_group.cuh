// batch_group.cuh -- grouped launches of a batch of independent factorisations.
//
// One launch runs one phase of the NTF iteration (an update sweep, the
// normalisation + Gram, a multi-TTV, a split-K sum, the error) for every
// member of a batch: blockIdx.z selects the member, whose arguments sit in a
// device table built when the batch's graph is captured. Each member runs
// through the same kernel body, CTA layout and summation order as its own
// launch would (the bodies are shared with the per-context kernels), so a
// grouped run gives the same bits as running the members one by one; the CTAs
// past a member's own grid return at once.
#pragma once
#include "kernels_f64.cuh"
#include "updates_iter.cuh"

namespace pg {

// HALS / MU sweep of one factor (k_hals_warp / k_mu_warp)
struct GrpUpd {
  double* H;
  const double* M;
  const double* G;
  int64_t I;
  int k;
  unsigned gx;  // the member's own grid
};

template <int KP>
__global__ void __launch_bounds__(256) k_grp_hals(const GrpUpd* __restrict__ a) {
  const GrpUpd& u = a[blockIdx.z];
  if (blockIdx.x >= u.gx) return;
  hals_warp_body<KP>(u.H, u.M, u.G, u.I, u.k, blockIdx.x);
}

template <int KP>
__global__ void __launch_bounds__(256) k_grp_mu(const GrpUpd* __restrict__ a, double eps) {
  const GrpUpd& u = a[blockIdx.z];
  if (blockIdx.x >= u.gx) return;
  mu_warp_body<KP>(u.H, u.M, u.G, u.I, u.k, eps, blockIdx.x);
}

// normalisation + Gram + next leave-one-out product (k_normgram_cluster); the
// launch's cluster spans x and has the largest member's size
struct GrpNg {
  double* F;
  int64_t I;
  int k;
  double* lambda;
  double* Gall;
  int N, n, next;
  double* Gloo;
  int CLm;  // the member's own cluster size
};

template <int BE>
__global__ void __launch_bounds__(NGC_THREADS, 1) k_grp_normgram(const GrpNg* __restrict__ a) {
  const GrpNg& g = a[blockIdx.z];
  normgram_cluster_body<BE>(g.F, g.I, g.k, g.lambda, g.Gall, g.N, g.n, g.next, g.Gloo, g.CLm);
}

// left multi-TTV of the FP32 intermediate (k_ttv_left<float> / k_ttv_left_f4)
struct GrpTtvL {
  const float* T;
  int64_t A, B;
  int k;
  const double* F;
  double* out;
  unsigned gx;
};

__global__ void __launch_bounds__(256) k_grp_ttv_left(const GrpTtvL* __restrict__ a) {
  const GrpTtvL& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx) return;
  ttv_left_body<float>(g.T, g.A, g.B, g.k, g.F, g.out, blockIdx.x, g.gx);
}

__global__ void __launch_bounds__(256, 4) k_grp_ttv_left_f4(const GrpTtvL* __restrict__ a) {
  const GrpTtvL& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx) return;
  ttv_left_f4_body(g.T, g.A, g.B, g.k, g.F, g.out, blockIdx.x);
}

// right multi-TTV of the FP32 intermediate (k_ttv_right_tiled<float, KP>)
struct GrpTtvR {
  const float* T;
  int64_t A, B;
  int k;
  WGen wg;
  int64_t bper;
  double* out;
  unsigned gx, gy;
};

template <int KP>
__global__ void __launch_bounds__(256) k_grp_ttv_right(const GrpTtvR* __restrict__ a) {
  const GrpTtvR& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx || blockIdx.y >= g.gy) return;
  ttv_right_tiled_body<float, KP>(g.T, g.A, g.B, g.k, g.wg, g.bper, g.out, blockIdx.x, blockIdx.y);
}

// fixed-order split-K sum (k_reduce_splits_few / k_reduce_splits)
struct GrpRed {
  const double* part;
  int nsplit;
  int64_t stride, n;
  double* out;
  unsigned gx;
};

__global__ void __launch_bounds__(256) k_grp_reduce_few(const GrpRed* __restrict__ a) {
  const GrpRed& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx) return;
  reduce_splits_few_body(g.part, g.nsplit, g.stride, g.n, g.out, blockIdx.x, g.gx);
}

__global__ void k_grp_reduce(const GrpRed* __restrict__ a) {
  const GrpRed& g = a[blockIdx.z];
  if (blockIdx.x >= g.gx) return;
  reduce_splits_body(g.part, g.nsplit, g.stride, g.n, g.out, blockIdx.x, g.gx);
}

// Gram-form relative error (k_error)
struct GrpErr {
  const double* Mlast;
  const double* Flast;
  int64_t I;
  const double* lambda;
  const double* Gall;
  int N, k;
  const double* normX2;
  double* errs;
  int* counter;
};

__global__ void __launch_bounds__(1024) k_grp_error(const GrpErr* __restrict__ a) {
  const GrpErr& g = a[blockIdx.z];
  error_body(g.Mlast, g.Flast, g.I, g.lambda, g.Gall, g.N, g.k, g.normX2, g.errs, g.counter);
}

}  // namespace pg
