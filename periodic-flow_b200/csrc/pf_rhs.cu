// SpaceSolver.compute_rhs(a) as separate arrays (space_solver.py:273-310).
//
// The time step never materialises these arrays: the stage update consumes
// every part of the right-hand side per mode, in registers.  This kernel is
// the plugin-contract form for callers that read rhs_linear, rhs_nonlinear,
// noise, forcing and p_hat between steps.  It runs the same per-mode code as
// the update (pf_mode.cuh, pf_update.cuh), so the arrays are the terms the
// next step's first stage would use with noise factor a.
#include "pf_kernels.h"
#include "pf_update.cuh"

namespace pf {

template <typename R, int D, int NC>
__global__ void __launch_bounds__(256) k_rhs_parts(UpdateArgs<R> A, RhsOut<R> out) {
  using C = cx<R>;
  const Geo& g = A.g;
  const StageScalars<R> sc = stage_scalars<R>(A);
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<R, D> mk_ = mode_k<R, D>(g, m);
    C un[D];
#pragma unroll
    for (int a = 0; a < D; ++a) un[a] = A.uhat[a * g.nspec + m];
    // compute_rhs_linear: L u_hat (math.py:52-68)
    const R L = A.lop ? A.lop[m] : (R)(-A.nu) * mk_.k2;
#pragma unroll
    for (int a = 0; a < D; ++a) out.rhs_linear[a * g.nspec + m] = cscale(un[a], L);
    // compute_rhs_nonlinear: projected, optionally Nyquist-masked (:297-300)
    C nv[D];
#pragma unroll
    for (int a = 0; a < D; ++a) nv[a] = A.nl ? A.nl[a * g.nspec + m] : czero<C>();
    if (A.nl) {
      leray<R, D>(nv, mk_.k, mk_.k2);
      if (A.nyq_mask && is_nyquist<D>(g, mk_.ix)) {
#pragma unroll
        for (int a = 0; a < D; ++a) nv[a] = czero<C>();
      }
    }
#pragma unroll
    for (int a = 0; a < D; ++a) out.rhs_nonlinear[a * g.nspec + m] = nv[a];
    // add_noise (:240-252): the last projection of compute_rhs, so p_hat
    // keeps the pressure of the unscaled noise as in the reference
    C xi[D];
    C p = czero<C>();
    if (A.noise_src != kNoiseNone) {
      C w1[NC], w2[NC];
      load_noise<R, D, NC>(A, m, mk_, w1, w2);
      const R corr = A.corr ? A.corr[m] : R(0);
      noise_raw<R, D, NC>(xi, w1, w2, (R)A.coef.a, A.noise_type, mk_.k, corr);
      p = leray<R, D>(xi, mk_.k, mk_.k2);
#pragma unroll
      for (int a = 0; a < D; ++a) xi[a] = cscale(xi[a], (R)A.noise_mag);
    } else {
#pragma unroll
      for (int a = 0; a < D; ++a) xi[a] = czero<C>();
    }
#pragma unroll
    for (int a = 0; a < D; ++a) out.noise[a * g.nspec + m] = xi[a];
    out.p_hat[m] = p;
    // add_forcing: band forcing eps / (2 E_band) u on 0 < |k|^2 <= kf^2
    const bool band = A.forcing && mk_.k2 > R(0) && (double)mk_.k2 <= A.f_kf2;
#pragma unroll
    for (int a = 0; a < D; ++a)
      out.forcing[a * g.nspec + m] = band ? cscale(un[a], sc.fcoef) : czero<C>();
  }
}

template <typename R>
cudaError_t launch_rhs_parts(const UpdateArgs<R>& A, int ncomp, const RhsOut<R>& out,
                             cudaStream_t st) {
  long long b = (A.g.nspec + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  if (b < 1) b = 1;
  const unsigned grid = (unsigned)b;
  if (A.g.dim == 3) {
    if (ncomp == 9) k_rhs_parts<R, 3, 9><<<grid, 256, 0, st>>>(A, out);
    else k_rhs_parts<R, 3, 3><<<grid, 256, 0, st>>>(A, out);
  } else {
    if (ncomp == 4) k_rhs_parts<R, 2, 4><<<grid, 256, 0, st>>>(A, out);
    else k_rhs_parts<R, 2, 2><<<grid, 256, 0, st>>>(A, out);
  }
  return launched();
}

template cudaError_t launch_rhs_parts<float>(const UpdateArgs<float>&, int, const RhsOut<float>&,
                                             cudaStream_t);
template cudaError_t launch_rhs_parts<double>(const UpdateArgs<double>&, int,
                                              const RhsOut<double>&, cudaStream_t);

}  // namespace pf
