// Argument blocks and launchers of the pointwise kernels.
#pragma once
#include "pf_internal.h"
#include "pf_mode.cuh"

namespace pf {

// device scalar slots of a solver
enum ScalarSlot {
  kScalDt = 0,      // current dt
  kScalBandE = 1,   // forcing band energy (2 slots: reduction writes [1], [2])
  kScalTime = 3,    // simulation time accumulated on the device
  kScalCount = 8
};

template <typename R> struct UpdateArgs {
  cx<R>* uhat;
  cx<R>* u0;
  const cx<R>* nl;     // unprojected nonlinear term or nullptr
  const R* lop;        // user L(k) or nullptr (-nu k^2)
  const R* corr;       // correlation function C(k) or nullptr (zero)
  const cx<R>* winj;   // injected w1, w2: (2 * ncomp, nspec) or nullptr
  const double* dscal; // device scalars
  double* diag;        // E, Z accumulators or nullptr
  Geo g;
  StageCoef coef;
  double nu, noise_mag, noise_norm, f_eps, f_kf2;
  uint64_t seed, step;
  int noise_src, noise_type, save_u0, nyq_mask, forcing;
  // batched boxes (member mb of a launch): state at uhat/u0 + mb * mstride,
  // scalars at dscal + mb * kScalCount, E/Z sums at diag + 2 mb, Philox key
  // seed + mb
  long long mstride;
  // first stage of a step whose state buffers swap roles (or nullptr): the
  // new state goes here and uhat, left as it is, is the step's u0 (no copy)
  cx<R>* uout;
};

template <typename R> struct StokesArgs {
  cx<R>* uhat;
  const R* lop;
  const R* corr;
  const cx<R>* winj;
  Geo g;
  Scheme scheme;
  double dt, nu, noise_mag, noise_norm;
  uint64_t seed, step0;
  int nsteps, noise_src, noise_type;
  int first_stage;  // 1: skip a stage the next one never reads (implicit PC, linear)
};

// SpaceSolver.compute_rhs(a) outside the time step (space_solver.py:273-310):
// the stage's parts written to separate arrays instead of being folded into
// the update.  `A` supplies the state, L, C, noise source and forcing set-up
// (A.coef.a is the stage's noise factor); nl is the unprojected nonlinear
// term or nullptr.
template <typename R> struct RhsOut {
  cx<R>* rhs_linear;     // (d, nspec)
  cx<R>* rhs_nonlinear;  // (d, nspec)
  cx<R>* noise;          // (d, nspec)
  cx<R>* forcing;        // (d, nspec)
  cx<R>* p_hat;          // (nspec)
};

// What the ensemble batch needs to know about a member solver.
struct SolverView {
  Geo g;
  int prec, ncomp, integrator, noise_type, noise_src;
  bool linear_only;  // no nonlinear term, forcing or adaptive dt
  void* uhat;
  const void* lop;
  const void* corr;
  double* dscal;
  double nu, noise_mag, noise_norm, dt;
  uint64_t seed;
  long long step;
};

template <typename R> cudaError_t launch_update(const UpdateArgs<R>& A, int ncomp, cudaStream_t st);
template <typename R>
cudaError_t launch_rhs_parts(const UpdateArgs<R>& A, int ncomp, const RhsOut<R>& out,
                             cudaStream_t st);
template <typename R> cudaError_t launch_stokes(const StokesArgs<R>& A, int ncomp, cudaStream_t st);
template <typename R>
cudaError_t launch_mask_copy(cx<R>* dst, const cx<R>* src, const Geo& g, int ncomp, cudaStream_t st);
template <typename R>
cudaError_t launch_curl_masked(cx<R>* dst, const cx<R>* u, const Geo& g, cudaStream_t st);
template <typename R>
cudaError_t launch_cross(R* u, const R* w, const Geo& g, unsigned long long* maxbits, cudaStream_t st);
// The per-step scalar kernels cover nmem members (dscal, maxbits, u strided
// by kScalCount, 1 and d nspec per member).
// (reads each member's CFL maximum and resets the word to zero)
cudaError_t launch_set_dt(double* dscal, unsigned long long* maxbits, double cfl, cudaStream_t st,
                          int nmem = 1);
// 3/2 rule: N-grid spectrum (or its curl) onto the M = 3N/2 grid, and back
template <typename R>
cudaError_t launch_pad(cx<R>* dst, const cx<R>* src, const Geo& gN, const Geo& gM, int ncomp,
                       int curl, cudaStream_t st);
template <typename R>
cudaError_t launch_truncate(cx<R>* dst, const cx<R>* src, const Geo& gN, const Geo& gM,
                            int ncomp, cudaStream_t st);
cudaError_t launch_advance_time(double* dscal, int n, cudaStream_t st, int nmem = 1);
template <typename R>
cudaError_t launch_band_energy(const cx<R>* u, const Geo& g, double kf2, double* dscal,
                               cudaStream_t st, int nmem = 1);
template <typename R>
cudaError_t launch_energy(const cx<R>* u, const Geo& g, double* out2, cudaStream_t st);
template <typename R>
cudaError_t launch_spectrum(const cx<R>* u, const Geo& g, double* out, int nbins, double kunit,
                            cudaStream_t st);

}  // namespace pf

struct pf_solver;
namespace pf {
SolverView solver_view(const ::pf_solver* h);
void solver_add_steps(::pf_solver* h, long long n);
Scheme scheme_for(int integrator);
}  // namespace pf
