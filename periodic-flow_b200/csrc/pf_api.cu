// C-ABI solver: owns the device state of one periodic box and runs the
// reference's time loop (simulation.py:205-217) on one CUDA stream.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "../../include/periodicflow_b200.h"
#include "pf_fused.h"
#include "pf_kernels.h"

using namespace pf;

struct pf_solver {
  pf_config cfg;
  Geo g;
  int d = 0, ncomp = 0, prec = 0;
  // members: nmem boxes of this configuration advanced together, laid out one
  // after another in uhat, u0, nl (d nspec complex each), dscal (kScalCount)
  // and maxbits; the fused passes cover them in one launch per pass
  int nmem = 1;
  int nact = 1;  // members [0, nact) take part in pf_step (pf_set_active_members)
  size_t rsz = 4;  // sizeof(real)
  cudaStream_t st = nullptr;
  void* uhat = nullptr;   // d * nspec complex
  void* u0 = nullptr;     // d * nspec complex
  void* nl = nullptr;     // d * nspec complex
  void* spec_tmp = nullptr;  // 3 * nspec complex
  void* phys_u = nullptr; // d * nphys real
  void* phys_w = nullptr; // (3D: 3, 2D: 1) * nphys real
  // 3/2 rule: padded grid M = 3N/2 and its work arrays
  Geo gM;
  bool padded = false;
  void* specM = nullptr;    // 3 * nspec(M) complex
  void* physM_u = nullptr;  // d * nphys(M) real
  void* physM_w = nullptr;  // (3D: 3, 2D: 1) * nphys(M) real
  void* lop = nullptr;    // nspec real (user L)
  void* corr = nullptr;   // nspec real (user C)
  void* winj = nullptr;   // 2 * ncomp * nspec complex
  void* rhs = nullptr;    // pf_compute_rhs arrays: (4 d + 1) * nspec complex, on first use
  double* stage64 = nullptr;  // FP64 staging for transfers
  size_t stage64_elems = 0;
  double* dscal = nullptr;
  unsigned long long* maxbits = nullptr;
  double* hist_dev = nullptr;  // 2 * kHist doubles
  int hist_fill = 0;
  bool record_hist = false;
  bool noise_ready = false;
  std::vector<double> hist;
  long long step = 0;
  double t = 0.0;
  FusedPlan* fused = nullptr;
  // per-pass CUDA-event timing (pf_kernel_timer)
  int tpass = -1;
  std::vector<cudaEvent_t> tev;
  size_t tused = 0;
  // captured "advance graph_steps" (pf_graph_capture / pf_graph_replay)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int graph_steps = 0;
  long long graph_launches = 0;
  bool capturing = false;
  // private one-step graph of pf_step (noise-free, no history, no timer):
  // recorded on its own stream, replayed once per step on st; one per state
  // buffer holding the current state (the roles swap every step)
  cudaGraph_t agraph[2] = {nullptr, nullptr};
  cudaGraphExec_t agexec[2] = {nullptr, nullptr};
  cudaStream_t astream = nullptr;
  long long a_launches = 0;
  bool auto_graph = true;
  // One box on the fused schedule: the first stage of a step writes the new
  // state into the u0 buffer and keeps the old one where it is as the step's
  // u0 (no copy of the state); uhat and u0 then swap roles.  sbuf0 is the
  // buffer that held the state at creation (parity 0).
  bool swap_state = false;
  void* sbuf0 = nullptr;
  bool no_swap_next = false;  // the next recorded or run step keeps its buffers
  int graph_parity = 0;       // state buffer the captured graph starts from
  std::string err;
};

// Kernel arguments recorded in the private step graph change: record again.
static void drop_auto_graph(pf_solver* h) {
  for (int p = 0; p < 2; ++p) {
    if (h->agexec[p]) { cudaGraphExecDestroy(h->agexec[p]); h->agexec[p] = nullptr; }
    if (h->agraph[p]) { cudaGraphDestroy(h->agraph[p]); h->agraph[p] = nullptr; }
  }
}

// which state buffer holds the current state (0: the one it started in)
static int state_parity(const pf_solver* h) { return h->uhat == h->sbuf0 ? 0 : 1; }

// record an event on the solver stream when `pass` is the timed pass; events
// come in (begin, end) pairs around each launch of that pass.  Inside a
// pf_graph_capture the records become event nodes of the graph (external
// records), so a replay of the captured steps times every launch in it.
static void tmark(pf_solver* h, int pass) {
  if (h->tpass != pass) return;
  if (h->tused == h->tev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    h->tev.push_back(e);
  }
  if (h->capturing) cudaEventRecordWithFlags(h->tev[h->tused++], h->st, cudaEventRecordExternal);
  else cudaEventRecord(h->tev[h->tused++], h->st);
}

static const int kHist = 4096;
static std::string g_static_err;

static int fail(pf_solver* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_static_err = msg;
  return code;
}

int pf::set_static_error(int code, const std::string& msg) { return fail(nullptr, code, msg); }

// Read-only view of a solver for the ensemble batch (pf_batch.cu).
pf::SolverView pf::solver_view(const pf_solver* h) {
  SolverView v;
  v.g = h->g;
  v.prec = h->prec;
  v.ncomp = h->ncomp;
  v.integrator = h->cfg.integrator;
  v.noise_type = h->cfg.noise_type;
  v.noise_src = h->cfg.noise_mag == 0.0 ? 0 : (h->cfg.noise_source == PF_NOISE_SRC_INJECTED ? 2 : 1);
  v.linear_only = !h->cfg.is_nonlinear && h->cfg.forcing_eps <= 0.0 && h->cfg.cfl <= 0.0;
  v.uhat = h->uhat;
  v.lop = h->lop;
  v.corr = h->corr;
  v.dscal = h->dscal;
  v.nu = h->cfg.viscosity;
  v.noise_mag = h->cfg.noise_mag;
  v.noise_norm = 1.0 / std::sqrt((double)h->g.nphys) / std::sqrt(2.0 - 2.0 / h->d);
  v.dt = h->cfg.dt;
  v.seed = h->cfg.seed;
  v.step = h->step;
  return v;
}

void pf::solver_add_steps(pf_solver* h, long long n) { h->step += n; }

#define PF_CUDA(h, call)                                                              \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return fail(h, PF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------- conversions
template <typename R>
__global__ void k_from64(R* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (R)src[i];
}
template <typename R>
__global__ void k_to64(double* __restrict__ dst, const R* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
template <typename R>
__global__ void k_scale_mask0(cx<R>* u, Geo g, int ncomp) {
  // zero the k = 0 mode of every component
  if (blockIdx.x == 0 && threadIdx.x < ncomp) u[threadIdx.x * g.nspec] = czero<cx<R>>();
}
template <typename R, int D>
__global__ void k_project(cx<R>* u, Geo g) {
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeIdx ix = mode_index(g, m);
    const KInt<D> ki = kint_of<D>(g, ix);
    R k[D];
    double k2 = 0.0;
    for (int a = 0; a < D; ++a) {
      const double ka = g.kscale[a] * ki.k[a];
      k[a] = (R)ka;
      k2 += ka * ka;
    }
    cx<R> v[D];
    for (int a = 0; a < D; ++a) v[a] = u[a * g.nspec + m];
    leray<R, D>(v, k, (R)k2);
    for (int a = 0; a < D; ++a) u[a * g.nspec + m] = v[a];
  }
}

static unsigned blocks_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// ------------------------------------------------------------ transforms
template <typename R>
static cudaError_t backward_g(pf_solver* h, const Geo& g, cx<R>* X, R* P, int nc) {
  cudaError_t e;
  if (g.dim == 3) {
    const long long plane = (long long)g.s[1] * g.nh;
    tmark(h, PF_PASS_FFT_STRIDED);
    e = fft_strided<R>(X, g.n[0], +1, plane, nc, g.nspec, plane, 1.0, h->st);
    tmark(h, PF_PASS_FFT_STRIDED);
    if (e != cudaSuccess) return e;
    tmark(h, PF_PASS_FFT_STRIDED);
    e = fft_strided<R>(X, g.n[1], +1, g.nh, (long long)nc * g.n[0], plane, g.nh, 1.0, h->st);
    tmark(h, PF_PASS_FFT_STRIDED);
    if (e != cudaSuccess) return e;
    tmark(h, PF_PASS_FFT_LAST);
    e = fft_c2r_last<R>(X, P, g.n[2], (long long)nc * g.n[0] * g.n[1], g.nh, g.n[2], h->st);
    tmark(h, PF_PASS_FFT_LAST);
    return e;
  }
  tmark(h, PF_PASS_FFT_STRIDED);
  e = fft_strided<R>(X, g.n[0], +1, g.nh, nc, g.nspec, g.nh, 1.0, h->st);
  tmark(h, PF_PASS_FFT_STRIDED);
  if (e != cudaSuccess) return e;
  tmark(h, PF_PASS_FFT_LAST);
  e = fft_c2r_last<R>(X, P, g.n[1], (long long)nc * g.n[0], g.nh, g.n[1], h->st);
  tmark(h, PF_PASS_FFT_LAST);
  return e;
}

template <typename R>
static cudaError_t backward_inplace(pf_solver* h, cx<R>* X, R* P, int nc) {
  return backward_g<R>(h, h->g, X, P, nc);
}

template <typename R>
static cudaError_t forward_g(pf_solver* h, const Geo& g, const R* P, cx<R>* X, int nc) {
  const double scale = 1.0 / (double)g.nphys;
  cudaError_t e;
  if (g.dim == 3) {
    const long long plane = (long long)g.s[1] * g.nh;
    tmark(h, PF_PASS_FFT_LAST);
    e = fft_r2c_last<R>(P, X, g.n[2], (long long)nc * g.n[0] * g.n[1], g.n[2], g.nh, scale, h->st);
    tmark(h, PF_PASS_FFT_LAST);
    if (e != cudaSuccess) return e;
    tmark(h, PF_PASS_FFT_STRIDED);
    e = fft_strided<R>(X, g.n[1], -1, g.nh, (long long)nc * g.n[0], plane, g.nh, 1.0, h->st);
    tmark(h, PF_PASS_FFT_STRIDED);
    if (e != cudaSuccess) return e;
    tmark(h, PF_PASS_FFT_STRIDED);
    e = fft_strided<R>(X, g.n[0], -1, plane, nc, g.nspec, plane, 1.0, h->st);
    tmark(h, PF_PASS_FFT_STRIDED);
    return e;
  }
  tmark(h, PF_PASS_FFT_LAST);
  e = fft_r2c_last<R>(P, X, g.n[1], (long long)nc * g.n[0], g.n[1], g.nh, scale, h->st);
  tmark(h, PF_PASS_FFT_LAST);
  if (e != cudaSuccess) return e;
  tmark(h, PF_PASS_FFT_STRIDED);
  e = fft_strided<R>(X, g.n[0], -1, g.nh, nc, g.nspec, g.nh, 1.0, h->st);
  tmark(h, PF_PASS_FFT_STRIDED);
  return e;
}

template <typename R>
static cudaError_t forward_into(pf_solver* h, const R* P, cx<R>* X, int nc) {
  return forward_g<R>(h, h->g, P, X, nc);
}

// 3/2 rule (basis.py:80-81): u and omega = i k x u padded onto the M = 3N/2
// grid, u x omega there, forward transform normalised by 1 / prod M, then
// truncated back to the N grid, unprojected, into h->nl
template <typename R>
static cudaError_t nonlinear_padded(pf_solver* h, bool want_max) {
  const Geo& g = h->g;
  const Geo& gM = h->gM;
  cx<R>* tmp = (cx<R>*)h->specM;
  const int wc = g.dim == 3 ? 3 : 1;
  cudaError_t e = launch_pad<R>(tmp, (const cx<R>*)h->uhat, g, gM, h->d, 1, h->st);
  if (e != cudaSuccess) return e;
  e = backward_g<R>(h, gM, tmp, (R*)h->physM_w, wc);
  if (e != cudaSuccess) return e;
  e = launch_pad<R>(tmp, (const cx<R>*)h->uhat, g, gM, h->d, 0, h->st);
  if (e != cudaSuccess) return e;
  e = backward_g<R>(h, gM, tmp, (R*)h->physM_u, h->d);
  if (e != cudaSuccess) return e;
  if (want_max) {
    e = cudaMemsetAsync(h->maxbits, 0, sizeof(unsigned long long), h->st);
    if (e != cudaSuccess) return e;
  }
  // iterate over the M grid, measure |u_i| / dx_i with the N-grid spacing
  Geo gx = g;
  gx.nphys = gM.nphys;
  e = launch_cross<R>((R*)h->physM_u, (const R*)h->physM_w, gx, want_max ? h->maxbits : nullptr,
                      h->st);
  if (e != cudaSuccess) return e;
  e = forward_g<R>(h, gM, (const R*)h->physM_u, tmp, h->d);
  if (e != cudaSuccess) return e;
  return launch_truncate<R>((cx<R>*)h->nl, tmp, g, gM, h->d, h->st);
}

// nonlinear term u x w (unprojected) of the current state into h->nl
template <typename R>
static cudaError_t nonlinear_generic(pf_solver* h, bool want_max) {
  const Geo& g = h->g;
  cx<R>* tmp = (cx<R>*)h->spec_tmp;
  cudaError_t e;
  const int wc = g.dim == 3 ? 3 : 1;
  e = launch_curl_masked<R>(tmp, (const cx<R>*)h->uhat, g, h->st);
  if (e != cudaSuccess) return e;
  e = backward_inplace<R>(h, tmp, (R*)h->phys_w, wc);
  if (e != cudaSuccess) return e;
  e = launch_mask_copy<R>(tmp, (const cx<R>*)h->uhat, g, h->d, h->st);
  if (e != cudaSuccess) return e;
  e = backward_inplace<R>(h, tmp, (R*)h->phys_u, h->d);
  if (e != cudaSuccess) return e;
  if (want_max) {
    e = cudaMemsetAsync(h->maxbits, 0, sizeof(unsigned long long), h->st);
    if (e != cudaSuccess) return e;
  }
  e = launch_cross<R>((R*)h->phys_u, (const R*)h->phys_w, g, want_max ? h->maxbits : nullptr,
                      h->st);
  if (e != cudaSuccess) return e;
  return forward_into<R>(h, (const R*)h->phys_u, (cx<R>*)h->nl, h->d);
}

// ------------------------------------------------------------------ schemes
static Scheme make_scheme(int integ) {
  Scheme s;
  memset(&s, 0, sizeof(s));
  auto set = [&](int i, double cu0, double cun, double cd, double cL, double cx, double a,
                 int Lu0, int impl) {
    s.st[i].cu0 = cu0; s.st[i].cun = cun; s.st[i].cd = cd; s.st[i].cL = cL;
    s.st[i].cx = cx; s.st[i].a = a; s.st[i].L_on_u0 = Lu0; s.st[i].implicit = impl;
  };
  const double rh = std::sqrt(0.5);
  switch (integ) {
    case PF_EXPLICIT_PC:  // time_integrator.py:45-56
      s.nstages = 2;
      set(0, 1, 0, 0.5, 0.5, rh, 0.0, 0, 0);
      set(1, 1, 0, 1.0, 1.0, rh, 1.0, 0, 0);
      break;
    case PF_IMPLICIT_PC:  // time_integrator.py:102-119
      s.nstages = 2;
      set(0, 1, 0, 0.5, 0.0, rh, 0.0, 0, 1);
      set(1, 1, 0, 1.0, 0.5, rh, 1.0, 1, 1);
      break;
    case PF_RK2:  // time_integrator.py:170-180 (noise_factor supplied as zeros)
      s.nstages = 2;
      set(0, 0.0, 1.0, 1.0, 1.0, 0, 0.0, 0, 0);
      set(1, 0.5, 0.5, 0.5, 0.5, 0, 0.0, 0, 0);
      break;
    case PF_RK3: {  // time_integrator.py:222-241
      s.nstages = 3;
      const double r2 = std::sqrt(2.0), r3 = std::sqrt(3.0);
      set(0, 0.0, 1.0, 1.0, 1.0, 1.0, (2 * r2 + r3) / 5, 0, 0);
      set(1, 0.75, 0.25, 0.25, 0.25, 0.25, (-4 * r2 + 3 * r3) / 5, 0, 0);
      set(2, 1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0, (r2 - 2 * r3) / 10, 0, 0);
      break;
    }
    default:  // PF_RK4, time_integrator.py:287-293
      s.nstages = 4;
      set(0, 1, 0, 0.25, 0.25, 0, 0.0, 0, 0);
      set(1, 1, 0, 1.0 / 3.0, 1.0 / 3.0, 0, 0.0, 0, 0);
      set(2, 1, 0, 0.5, 0.5, 0, 0.0, 0, 0);
      set(3, 1, 0, 1.0, 1.0, 0, 0.0, 0, 0);
      break;
  }
  return s;
}

static double noise_norm(const pf_solver* h) {
  return 1.0 / std::sqrt((double)h->g.nphys) / std::sqrt(2.0 - 2.0 / h->d);
}

static int noise_src(const pf_solver* h) {
  if (h->cfg.noise_mag == 0.0) return kNoiseNone;
  return h->cfg.noise_source == PF_NOISE_SRC_INJECTED ? kNoiseInjected : kNoisePhilox;
}

// --------------------------------------------------------------- one step
template <typename R>
static int step_generic(pf_solver* h) {
  const Geo& g = h->g;
  const Scheme sc = make_scheme(h->cfg.integrator);
  const bool cfl = h->cfg.cfl > 0.0;
  const bool forcing = h->cfg.forcing_eps > 0.0;
  const bool use_fused = h->fused != nullptr && h->cfg.fused && h->cfg.is_nonlinear;
  // the first stage writes the new state into the u0 buffer (roles swap)
  const bool swap = use_fused && h->swap_state && !h->no_swap_next;
  h->no_swap_next = false;
  void* const old_state = h->uhat;
  void* const new_state = swap ? h->u0 : h->uhat;
  for (int s = 0; s < sc.nstages; ++s) {
    void* const cur = s == 0 ? old_state : new_state;  // the stage's input state
    if (h->cfg.is_nonlinear) {
      if (use_fused) {
        // (the CFL words start at zero: zeroed at creation, and k_set_dt resets
        // them after reading)
        for (int p = 1; p <= 4; ++p) {
          tmark(h, PF_PASS_FUSED_P1 + p - 1);
          cudaError_t fe = fused_pass(h->fused, p, cur, h->nl,
                                      (s == 0 && cfl && p == 3) ? h->maxbits : nullptr, h->st);
          tmark(h, PF_PASS_FUSED_P1 + p - 1);
          PF_CUDA(h, fe);
        }
      } else {
        PF_CUDA(h, h->padded ? nonlinear_padded<R>(h, s == 0 && cfl)
                             : nonlinear_generic<R>(h, s == 0 && cfl));
      }
      if (s == 0 && cfl)
        PF_CUDA(h, launch_set_dt(h->dscal, h->maxbits, h->cfg.cfl, h->st, h->nact));
    } else if (s == 0 && cfl) {
      return fail(h, PF_ERR_UNSUPPORTED, "CFL-adaptive dt needs the nonlinear term");
    }
    if (forcing)
      PF_CUDA(h, launch_band_energy<R>((const cx<R>*)cur, g,
                                       h->cfg.forcing_kf * h->cfg.forcing_kf, h->dscal, h->st,
                                       h->nact));
    UpdateArgs<R> A;
    memset(&A, 0, sizeof(A));
    A.uhat = (cx<R>*)cur;
    A.u0 = (cx<R>*)(swap ? old_state : h->u0);
    A.uout = (swap && s == 0) ? (cx<R>*)new_state : nullptr;
    A.nl = h->cfg.is_nonlinear ? (const cx<R>*)h->nl : nullptr;
    A.lop = (const R*)h->lop;
    A.corr = (const R*)h->corr;
    A.winj = (const cx<R>*)h->winj;
    A.dscal = h->dscal;
    A.diag = (h->record_hist && s == sc.nstages - 1) ? h->hist_dev + 2 * h->hist_fill : nullptr;
    A.g = g;
    A.coef = sc.st[s];
    A.nu = h->cfg.viscosity;
    A.noise_mag = h->cfg.noise_mag;
    A.noise_norm = noise_norm(h);
    A.f_eps = h->cfg.forcing_eps;
    A.f_kf2 = h->cfg.forcing_kf * h->cfg.forcing_kf;
    A.seed = h->cfg.seed;
    A.step = (uint64_t)(h->step + 1);
    A.noise_src = noise_src(h);
    A.noise_type = h->cfg.noise_type;
    A.save_u0 = s == 0;
    A.nyq_mask = h->cfg.mask_nyquist;
    A.forcing = forcing;
    A.mstride = (long long)h->d * g.nspec;
    cudaError_t ue;
    if (use_fused) {
      tmark(h, PF_PASS_FUSED_P5);
      ue = fused_update(h->fused, A, h->ncomp, h->nl, h->st);
      tmark(h, PF_PASS_FUSED_P5);
    } else {
      tmark(h, PF_PASS_UPDATE);
      ue = launch_update<R>(A, h->ncomp, h->st);
      tmark(h, PF_PASS_UPDATE);
    }
    PF_CUDA(h, ue);
  }
  if (!cfl) PF_CUDA(h, launch_advance_time(h->dscal, 1, h->st, h->nact));
  if (swap) std::swap(h->uhat, h->u0);
  return PF_OK;
}

template <typename R>
static int step_stokes(pf_solver* h, int nsteps) {
  StokesArgs<R> A;
  memset(&A, 0, sizeof(A));
  A.uhat = (cx<R>*)h->uhat;
  A.lop = (const R*)h->lop;
  A.corr = (const R*)h->corr;
  A.winj = (const cx<R>*)h->winj;
  A.g = h->g;
  A.scheme = make_scheme(h->cfg.integrator);
  A.dt = h->cfg.dt;
  A.nu = h->cfg.viscosity;
  A.noise_mag = h->cfg.noise_mag;
  A.noise_norm = noise_norm(h);
  A.seed = h->cfg.seed;
  A.step0 = (uint64_t)(h->step + 1);
  A.nsteps = nsteps;
  A.noise_src = noise_src(h);
  A.noise_type = h->cfg.noise_type;
  // the implicit predictor's output is never read by the corrector here
  A.first_stage = h->cfg.integrator == PF_IMPLICIT_PC ? 1 : 0;
  tmark(h, PF_PASS_STOKES);
  cudaError_t se = launch_stokes<R>(A, h->ncomp, h->st);
  tmark(h, PF_PASS_STOKES);
  PF_CUDA(h, se);
  PF_CUDA(h, launch_advance_time(h->dscal, nsteps, h->st));
  return PF_OK;
}

// Error word of bounded waits inside the fused passes (synchronous read).
static int check_dev_errors(pf_solver* h) {
  if (!h->fused) return PF_OK;
  const int v = fused_device_error(h->fused);
  if (v != 0)
    return fail(h, PF_ERR_CUDA,
                "a bounded device wait gave up (code " + std::to_string(v) +
                    "): a bulk copy did not complete in time; results of the step are invalid");
  return PF_OK;
}

static int flush_hist(pf_solver* h) {
  if (h->hist_fill == 0) return PF_OK;
  std::vector<double> tmp(2 * h->hist_fill);
  PF_CUDA(h, cudaMemcpyAsync(tmp.data(), h->hist_dev, sizeof(double) * tmp.size(),
                             cudaMemcpyDeviceToHost, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  h->hist.insert(h->hist.end(), tmp.begin(), tmp.end());
  h->hist_fill = 0;
  PF_CUDA(h, cudaMemsetAsync(h->hist_dev, 0, sizeof(double) * 2 * kHist, h->st));
  return PF_OK;
}

// Record one step (step_generic) as a graph on the private stream.
template <typename R>
static int record_auto_graph(pf_solver* h) {
  if (!h->astream) PF_CUDA(h, cudaStreamCreateWithFlags(&h->astream, cudaStreamNonBlocking));
  const int par = state_parity(h);
  void* const uhat = h->uhat;
  void* const u0 = h->u0;
  cudaStream_t user = h->st;
  h->st = h->astream;
  h->no_swap_next = false;
  const long long l0 = launch_total();
  h->capturing = true;
  cudaError_t e = cudaStreamBeginCapture(h->astream, cudaStreamCaptureModeThreadLocal);
  int rc = PF_OK;
  if (e == cudaSuccess) {
    rc = step_generic<R>(h);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(h->astream, &g);
    if (e == cudaSuccess) e = e2;
    h->agraph[par] = g;
  }
  h->capturing = false;
  h->st = user;
  h->uhat = uhat;  // recorded, not run: the buffers keep their roles
  h->u0 = u0;
  h->a_launches = launch_total() - l0;
  add_launches(-h->a_launches);  // recorded, not launched
  if (rc == PF_OK && e == cudaSuccess) e = cudaGraphInstantiate(&h->agexec[par], h->agraph[par], 0);
  if (rc != PF_OK || e != cudaSuccess) {
    drop_auto_graph(h);
    cudaGetLastError();
    h->auto_graph = false;  // step without it from now on
    return rc != PF_OK ? rc : fail(h, PF_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(e));
  }
  return PF_OK;
}

template <typename R>
static int step_impl(pf_solver* h, int nsteps) {
  const bool stokes_fast = !h->cfg.is_nonlinear && h->cfg.forcing_eps <= 0.0 &&
                           h->cfg.cfl <= 0.0;
  const bool injected = noise_src(h) == kNoiseInjected;
  if (injected && (nsteps > 1 || !h->noise_ready))
    return fail(h, PF_ERR_INVALID,
                "injected noise: call pf_inject_noise before every single pf_step(h, 1)");
  int done = 0;
  // noise-free runs without history or timer: one recorded step graph per
  // step (the step's launches cost one graph launch; dt, time and the CFL
  // reduction live in device scalars, so the graph is step-independent),
  // unless the caller's stream is being captured itself
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(h->st, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusActive;
  }
  const bool graphable = !stokes_fast && h->auto_graph && !injected && noise_src(h) == kNoiseNone &&
                         !h->record_hist && h->tpass < 0 && nsteps >= 1 &&
                         cap == cudaStreamCaptureStatusNone;
  if (graphable) {
    for (; done < nsteps; ++done) {
      const int par = state_parity(h);
      if (!h->agexec[par]) {
        int rc = record_auto_graph<R>(h);
        if (rc) return rc;
        if (!h->agexec[par]) break;  // recording failed: plain steps from here
      }
      PF_CUDA(h, cudaGraphLaunch(h->agexec[par], h->st));
      add_launches(h->a_launches);
      h->step += 1;
      if (h->swap_state) std::swap(h->uhat, h->u0);
    }
    if (done == nsteps) return PF_OK;
  }
  while (done < nsteps) {
    int chunk = nsteps - done;
    if (h->record_hist) chunk = 1;
    if (stokes_fast) {
      int rc = step_stokes<R>(h, chunk);
      if (rc) return rc;
      if (h->record_hist)
        PF_CUDA(h, launch_energy<R>((const cx<R>*)h->uhat, h->g, h->hist_dev + 2 * h->hist_fill,
                                    h->st));
    } else {
      chunk = 1;
      int rc = step_generic<R>(h);
      if (rc) return rc;
    }
    h->step += chunk;
    done += chunk;
    if (h->record_hist) {
      h->hist_fill += 1;
      if (h->hist_fill == kHist) {
        int rc = flush_hist(h);
        if (rc) return rc;
      }
    }
  }
  h->noise_ready = false;
  return PF_OK;
}

// ================================================================ C ABI
extern "C" {

int pf_config_default(pf_config* c) {
  if (!c) return fail(nullptr, PF_ERR_INVALID, "pf_config_default: null config");
  memset(c, 0, sizeof(*c));
  c->dim = 3;
  c->n[0] = c->n[1] = c->n[2] = 64;
  for (int i = 0; i < 3; ++i) { c->domain[i][0] = 0.0; c->domain[i][1] = 2.0 * M_PI; }
  c->is_nonlinear = 1;
  c->integrator = PF_RK2;
  c->viscosity = 1e-3;
  c->noise_type = PF_NOISE_THERMAL;
  c->noise_mag = 0.0;
  c->dealias = PF_DEALIAS_TRUNCATE;
  c->mask_nyquist = 0;
  c->precision = PF_FP32;
  c->dt = 1e-3;
  c->seed = 0;
  c->noise_source = PF_NOISE_SRC_PHILOX;
  c->forcing_kf = 2.5;
  c->fused = 1;
  return PF_OK;
}

const char* pf_last_error(const pf_solver* h) {
  return h ? h->err.c_str() : g_static_err.c_str();
}

static int validate(const pf_config* c) {
  if (c->dim != 2 && c->dim != 3)
    return fail(nullptr, PF_ERR_INVALID, "NS solver only supports 2D and 3D problems.");
  for (int a = 0; a < c->dim; ++a) {
    if (!fft_length_supported(c->n[a]))
      return fail(nullptr, PF_ERR_UNSUPPORTED,
                  "grid size " + std::to_string(c->n[a]) +
                      " not built: sides 2^b from 4 to 1024 and 3 * 2^b from 12 to 768 are supported");
    if (!(c->domain[a][1] > c->domain[a][0]))
      return fail(nullptr, PF_ERR_INVALID, "Invalid domain.");
  }
  if (c->integrator < PF_EXPLICIT_PC || c->integrator > PF_RK4)
    return fail(nullptr, PF_ERR_INVALID, "Time integrator not found.");
  if (c->noise_type != PF_NOISE_THERMAL && c->noise_type != PF_NOISE_CORRELATED)
    return fail(nullptr, PF_ERR_INVALID,
                "Invalid noise type. Options are 'thermal' or 'correlated'.");
  if (c->dealias != PF_DEALIAS_TRUNCATE && c->dealias != PF_DEALIAS_PAD)
    return fail(nullptr, PF_ERR_INVALID, "FourierSpace: Invalid dealiasing rule.");
  if (c->dealias == PF_DEALIAS_PAD && c->is_nonlinear) {
    for (int a = 0; a < c->dim; ++a)
      if (c->n[a] % 2 != 0 || !fft_length_supported(3 * c->n[a] / 2))
        return fail(nullptr, PF_ERR_UNSUPPORTED,
                    "3/2 padding needs a padded size 3n/2 with a built FFT (n = 8..512)");
  }
  if (c->precision != PF_FP32 && c->precision != PF_FP64)
    return fail(nullptr, PF_ERR_INVALID, "precision must be PF_FP32 or PF_FP64");
  if (!(c->dt > 0.0)) return fail(nullptr, PF_ERR_INVALID, "dt must be positive");
  return PF_OK;
}

}  // extern "C"

int pf::config_validate(const pf_config* c) { return validate(c); }

// Box geometry of a configuration (wavenumber scales 2 pi / L, 2/3-rule kmax).
Geo pf::config_geo(const pf_config* cfg) {
  Geo g;
  memset(&g, 0, sizeof(g));
  const int d = cfg->dim;
  g.dim = d;
  g.n[2] = 1;
  for (int a = 0; a < d; ++a) {
    g.n[a] = cfg->n[a];
    g.kscale[a] = 2.0 * M_PI / (cfg->domain[a][1] - cfg->domain[a][0]);
    g.kmax[a] = (cfg->n[a] - 1) / 3;
    g.s[a] = cfg->n[a];
  }
  g.nh = cfg->n[d - 1] / 2 + 1;
  g.s[d - 1] = g.nh;
  g.nspec = 1;
  g.nphys = 1;
  for (int a = 0; a < d; ++a) { g.nspec *= g.s[a]; g.nphys *= g.n[a]; }
  return g;
}

extern "C" {

static int create_impl(const pf_config* cfg, int nmem, pf_solver** out) {
  if (!cfg || !out) return fail(nullptr, PF_ERR_INVALID, "pf_create: null argument");
  *out = nullptr;
  int rc = validate(cfg);
  if (rc) return rc;
  if (nmem < 1) return fail(nullptr, PF_ERR_INVALID, "pf_create_members: members must be >= 1");
  if (nmem > 1 && (!cfg->is_nonlinear || !cfg->fused))
    return fail(nullptr, PF_ERR_UNSUPPORTED,
                "pf_create_members: members advance through the fused nonlinear passes "
                "(linear ensembles: pf_batch_create)");
  if (nmem > 1 && cfg->noise_mag != 0.0 && cfg->noise_source == PF_NOISE_SRC_INJECTED)
    return fail(nullptr, PF_ERR_UNSUPPORTED, "pf_create_members: injected noise is per solver");
  cudaError_t ce = ensure_tables();
  if (ce != cudaSuccess)
    return fail(nullptr, PF_ERR_CUDA, std::string("twiddle tables: ") + cudaGetErrorString(ce));
  pf_solver* h = new pf_solver();
  h->cfg = *cfg;
  h->nmem = nmem;
  h->nact = nmem;
  h->d = cfg->dim;
  h->prec = cfg->precision;
  h->rsz = h->prec == PF_FP64 ? 8 : 4;
  h->ncomp = cfg->noise_type == PF_NOISE_THERMAL ? h->d * h->d : h->d;
  h->g = pf::config_geo(cfg);
  Geo& g = h->g;
  const size_t cb = 2 * h->rsz;  // complex bytes
  auto alloc = [&](void** p, size_t bytes) -> bool {
    if (cudaMalloc(p, bytes) != cudaSuccess) return false;
    return cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  const int wc = h->d == 3 ? 3 : 1;
  h->stage64_elems = std::max((size_t)(2 * h->d * g.nspec), (size_t)(h->d * g.nphys));
  h->stage64_elems = std::max(h->stage64_elems, (size_t)(4 * h->ncomp * g.nspec));
  const size_t M = (size_t)nmem;
  bool ok = alloc(&h->uhat, cb * h->d * g.nspec * M) && alloc(&h->u0, cb * h->d * g.nspec * M) &&
            alloc(&h->spec_tmp, cb * 3 * g.nspec) &&
            alloc((void**)&h->stage64, sizeof(double) * h->stage64_elems) &&
            alloc((void**)&h->dscal, sizeof(double) * kScalCount * M) &&
            alloc((void**)&h->maxbits, sizeof(unsigned long long) * M) &&
            alloc((void**)&h->hist_dev, sizeof(double) * 2 * kHist);
  if (ok && cfg->is_nonlinear && cfg->dealias == PF_DEALIAS_PAD) {
    h->padded = true;
    Geo& gM = h->gM;
    gM = g;
    gM.nspec = 1;
    gM.nphys = 1;
    for (int a = 0; a < h->d; ++a) {
      gM.n[a] = 3 * g.n[a] / 2;
      gM.s[a] = gM.n[a];
    }
    gM.nh = gM.n[h->d - 1] / 2 + 1;
    gM.s[h->d - 1] = gM.nh;
    for (int a = 0; a < h->d; ++a) { gM.nspec *= gM.s[a]; gM.nphys *= gM.n[a]; }
    ok = alloc(&h->nl, cb * h->d * g.nspec) && alloc(&h->specM, cb * 3 * gM.nspec) &&
         alloc(&h->physM_u, h->rsz * h->d * gM.nphys) &&
         alloc(&h->physM_w, h->rsz * wc * gM.nphys);
  } else if (ok && cfg->is_nonlinear) {
    ok = alloc(&h->nl, cb * h->d * g.nspec * M) && alloc(&h->phys_u, h->rsz * h->d * g.nphys) &&
         alloc(&h->phys_w, h->rsz * wc * g.nphys);
  }
  if (ok && cfg->noise_mag != 0.0 && cfg->noise_source == PF_NOISE_SRC_INJECTED)
    ok = alloc(&h->winj, cb * 2 * h->ncomp * g.nspec);
  if (!ok) {
    std::string m = std::string("device allocation failed: ") + cudaGetErrorString(cudaGetLastError());
    pf_destroy(h);
    return fail(nullptr, PF_ERR_NOMEM, m);
  }
  double dt0 = cfg->dt;
  for (int m = 0; m < nmem; ++m)
    cudaMemcpy(h->dscal + (size_t)m * kScalCount + kScalDt, &dt0, sizeof(double),
               cudaMemcpyHostToDevice);
  if (cfg->is_nonlinear && cfg->fused) {
    h->fused = fused_create(g, h->prec, cfg->dealias, nmem);  // nullptr when no fused path fits
  }
  h->sbuf0 = h->uhat;
  h->swap_state = h->fused != nullptr && nmem == 1;
  if (const char* v = getenv("PF_STATE_SWAP")) h->swap_state = h->swap_state && atoi(v) != 0;
  if (nmem > 1 && !h->fused) {
    pf_destroy(h);
    return fail(nullptr, PF_ERR_UNSUPPORTED,
                "pf_create_members: no fused schedule for this geometry, precision and rule");
  }
  if (const char* v = getenv("PF_STEP_GRAPH")) h->auto_graph = atoi(v) != 0;  // 0: plain launches
  *out = h;
  return PF_OK;
}

int pf_create(const pf_config* cfg, pf_solver** out) { return create_impl(cfg, 1, out); }

int pf_create_members(const pf_config* cfg, int members, pf_solver** out) {
  return create_impl(cfg, members, out);
}

int pf_members(const pf_solver* h, int* members) {
  if (!h || !members) return fail(nullptr, PF_ERR_INVALID, "pf_members: null argument");
  *members = h->nmem;
  return PF_OK;
}

int pf_set_active_members(pf_solver* h, int active) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (active < 1 || active > h->nmem)
    return fail(h, PF_ERR_INVALID, "pf_set_active_members: active must be in [1, members]");
  if (h->capturing) return fail(h, PF_ERR_INVALID, "pf_set_active_members: inside a capture");
  if (active == h->nact) return PF_OK;
  h->nact = active;
  if (h->fused) fused_set_members(h->fused, active);
  drop_auto_graph(h);  // the recorded launches cover the old count
  return PF_OK;
}

int pf_copy_member(pf_solver* h, int dst, int src) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (dst < 0 || dst >= h->nmem || src < 0 || src >= h->nmem)
    return fail(h, PF_ERR_INVALID, "pf_copy_member: bad member");
  if (dst == src) return PF_OK;
  const size_t sb = 2 * h->rsz * (size_t)h->d * h->g.nspec;  // bytes of one member's state
  PF_CUDA(h, cudaMemcpyAsync((char*)h->uhat + dst * sb, (const char*)h->uhat + src * sb, sb,
                             cudaMemcpyDeviceToDevice, h->st));
  PF_CUDA(h, cudaMemcpyAsync(h->dscal + (size_t)dst * kScalCount, h->dscal + (size_t)src * kScalCount,
                             sizeof(double) * kScalCount, cudaMemcpyDeviceToDevice, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}

int pf_set_time_member(pf_solver* h, int m, double t, double dt) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (m < 0 || m >= h->nmem) return fail(h, PF_ERR_INVALID, "pf_set_time_member: bad member");
  if (!(dt > 0.0)) return fail(h, PF_ERR_INVALID, "pf_set_time_member: dt must be positive");
  double* d = h->dscal + (size_t)m * kScalCount;
  PF_CUDA(h, cudaMemcpyAsync(d + kScalTime, &t, sizeof(double), cudaMemcpyHostToDevice, h->st));
  PF_CUDA(h, cudaMemcpyAsync(d + kScalDt, &dt, sizeof(double), cudaMemcpyHostToDevice, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}

int pf_destroy(pf_solver* h) {
  if (!h) return PF_OK;
  void* ptrs[] = {h->uhat, h->u0, h->nl, h->spec_tmp, h->phys_u, h->phys_w,
                  h->specM, h->physM_u, h->physM_w, h->lop,
                  h->corr, h->winj, h->rhs, h->stage64, h->dscal, h->maxbits, h->hist_dev};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (h->fused) fused_destroy(h->fused);
  for (cudaEvent_t e : h->tev) cudaEventDestroy(e);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  drop_auto_graph(h);
  if (h->astream) cudaStreamDestroy(h->astream);
  delete h;
  return PF_OK;
}

int pf_set_stream(pf_solver* h, void* stream) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  h->st = (cudaStream_t)stream;
  return PF_OK;
}

int pf_sizes(const pf_solver* h, long long* nspec, long long* nphys, int* ncomp) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (nspec) *nspec = h->g.nspec;
  if (nphys) *nphys = h->g.nphys;
  if (ncomp) *ncomp = h->ncomp;
  return PF_OK;
}

// copy n doubles from (host|device) src into the FP64 staging buffer
static int stage_in(pf_solver* h, const double* src, size_t n, int where) {
  PF_CUDA(h, cudaMemcpyAsync(h->stage64, src, sizeof(double) * n,
                             where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->st));
  return PF_OK;
}
static int stage_out(pf_solver* h, double* dst, size_t n, int where) {
  PF_CUDA(h, cudaMemcpyAsync(dst, h->stage64, sizeof(double) * n,
                             where ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}
static cudaError_t convert_in(pf_solver* h, void* dst, size_t n) {
  if (h->prec == PF_FP64)
    return cudaMemcpyAsync(dst, h->stage64, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st);
  k_from64<float><<<blocks_for(n), 256, 0, h->st>>>((float*)dst, h->stage64, (long long)n);
  return launched();
}
static cudaError_t convert_out(pf_solver* h, const void* src, size_t n) {
  if (h->prec == PF_FP64)
    return cudaMemcpyAsync(h->stage64, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st);
  k_to64<float><<<blocks_for(n), 256, 0, h->st>>>(h->stage64, (const float*)src, (long long)n);
  return launched();
}

// state of member m (d nspec complex values) from / to complex128 data
static int set_member(pf_solver* h, int m, const double* u_hat, int where) {
  const size_t n = 2 * (size_t)h->d * h->g.nspec;  // doubles
  int rc = stage_in(h, u_hat, n, where);
  if (rc) return rc;
  PF_CUDA(h, convert_in(h, (char*)h->uhat + (size_t)m * n * h->rsz, n));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}
static int get_member(pf_solver* h, int m, double* u_hat, int where) {
  const size_t n = 2 * (size_t)h->d * h->g.nspec;
  PF_CUDA(h, convert_out(h, (const char*)h->uhat + (size_t)m * n * h->rsz, n));
  return stage_out(h, u_hat, n, where);
}

int pf_set_fourier(pf_solver* h, const double* u_hat, int where) {
  if (!h || !u_hat) return fail(h, PF_ERR_INVALID, "pf_set_fourier: null argument");
  const size_t n = 2 * (size_t)h->d * h->g.nspec;
  for (int m = 0; m < h->nmem; ++m) {
    int rc = set_member(h, m, u_hat + (size_t)m * n, where);
    if (rc) return rc;
  }
  return PF_OK;
}

int pf_get_fourier(pf_solver* h, double* u_hat, int where) {
  if (!h || !u_hat) return fail(h, PF_ERR_INVALID, "pf_get_fourier: null argument");
  const size_t n = 2 * (size_t)h->d * h->g.nspec;
  for (int m = 0; m < h->nmem; ++m) {
    int rc = get_member(h, m, u_hat + (size_t)m * n, where);
    if (rc) return rc;
  }
  return check_dev_errors(h);
}

int pf_set_fourier_member(pf_solver* h, int m, const double* u_hat, int where) {
  if (!h || !u_hat) return fail(h, PF_ERR_INVALID, "pf_set_fourier_member: null argument");
  if (m < 0 || m >= h->nmem) return fail(h, PF_ERR_INVALID, "pf_set_fourier_member: bad member");
  return set_member(h, m, u_hat, where);
}

int pf_get_fourier_member(pf_solver* h, int m, double* u_hat, int where) {
  if (!h || !u_hat) return fail(h, PF_ERR_INVALID, "pf_get_fourier_member: null argument");
  if (m < 0 || m >= h->nmem) return fail(h, PF_ERR_INVALID, "pf_get_fourier_member: bad member");
  int rc = get_member(h, m, u_hat, where);
  return rc ? rc : check_dev_errors(h);
}

int pf_set_physical(pf_solver* h, const double* u, int where) {
  if (!h || !u) return fail(h, PF_ERR_INVALID, "pf_set_physical: null argument");
  if (h->nmem > 1) return fail(h, PF_ERR_UNSUPPORTED, "pf_set_physical: one member at a time (pf_get_fourier_member)");
  const size_t n = (size_t)h->d * h->g.nphys;
  void* phys = h->phys_u;
  void* own = nullptr;
  if (!phys) {
    PF_CUDA(h, cudaMalloc(&own, h->rsz * n));
    phys = own;
  }
  int rc = stage_in(h, u, n, where);
  if (!rc) {
    cudaError_t e = convert_in(h, phys, n);
    if (e == cudaSuccess)
      e = h->prec == PF_FP64 ? forward_into<double>(h, (const double*)phys, (double2*)h->uhat, h->d)
                             : forward_into<float>(h, (const float*)phys, (float2*)h->uhat, h->d);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) rc = fail(h, PF_ERR_CUDA, std::string("pf_set_physical: ") + cudaGetErrorString(e));
  }
  if (own) cudaFree(own);
  return rc;
}

int pf_get_physical(pf_solver* h, double* u, int where) {
  if (!h || !u) return fail(h, PF_ERR_INVALID, "pf_get_physical: null argument");
  if (h->nmem > 1) return fail(h, PF_ERR_UNSUPPORTED, "pf_get_physical: one member at a time (pf_get_fourier_member)");
  const size_t n = (size_t)h->d * h->g.nphys;
  void* phys = h->phys_u;
  void* own = nullptr;
  if (!phys) {
    PF_CUDA(h, cudaMalloc(&own, h->rsz * n));
    phys = own;
  }
  const size_t cb = 2 * h->rsz;
  cudaError_t e = cudaMemcpyAsync(h->spec_tmp, h->uhat, cb * h->d * h->g.nspec,
                                  cudaMemcpyDeviceToDevice, h->st);
  if (e == cudaSuccess)
    e = h->prec == PF_FP64
            ? backward_inplace<double>(h, (double2*)h->spec_tmp, (double*)phys, h->d)
            : backward_inplace<float>(h, (float2*)h->spec_tmp, (float*)phys, h->d);
  if (e == cudaSuccess) e = convert_out(h, phys, n);
  int rc = PF_OK;
  if (e != cudaSuccess) rc = fail(h, PF_ERR_CUDA, std::string("pf_get_physical: ") + cudaGetErrorString(e));
  if (!rc) rc = stage_out(h, u, n, where);
  if (own) cudaFree(own);
  return rc;
}

int pf_mask_zero_mode(pf_solver* h) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  const size_t ms = (size_t)h->d * h->g.nspec;  // complex values per member
  for (int m = 0; m < h->nmem; ++m) {
    if (h->prec == PF_FP64)
      k_scale_mask0<double><<<1, 32, 0, h->st>>>((double2*)h->uhat + m * ms, h->g, h->d);
    else k_scale_mask0<float><<<1, 32, 0, h->st>>>((float2*)h->uhat + m * ms, h->g, h->d);
    PF_CUDA(h, launched());
  }
  return PF_OK;
}

int pf_project(pf_solver* h) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  const unsigned b = blocks_for(h->g.nspec);
  const size_t ms = (size_t)h->d * h->g.nspec;
  for (int m = 0; m < h->nmem; ++m) {
    if (h->prec == PF_FP64) {
      double2* u = (double2*)h->uhat + m * ms;
      if (h->d == 3) k_project<double, 3><<<b, 256, 0, h->st>>>(u, h->g);
      else k_project<double, 2><<<b, 256, 0, h->st>>>(u, h->g);
    } else {
      float2* u = (float2*)h->uhat + m * ms;
      if (h->d == 3) k_project<float, 3><<<b, 256, 0, h->st>>>(u, h->g);
      else k_project<float, 2><<<b, 256, 0, h->st>>>(u, h->g);
    }
    PF_CUDA(h, launched());
  }
  return PF_OK;
}

static int set_scalar_field(pf_solver* h, void** slot, const double* src, int where) {
  const size_t n = (size_t)h->g.nspec;
  if (!src) {
    if (*slot) cudaFree(*slot);
    *slot = nullptr;
    return PF_OK;
  }
  if (!*slot) PF_CUDA(h, cudaMalloc(slot, h->rsz * n));
  int rc = stage_in(h, src, n, where);
  if (rc) return rc;
  PF_CUDA(h, convert_in(h, *slot, n));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}

int pf_set_linear_operator(pf_solver* h, const double* L, int where) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  drop_auto_graph(h);  // the operator array may be newly allocated
  return set_scalar_field(h, &h->lop, L, where);
}

int pf_set_correlation(pf_solver* h, const double* C, int where) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  drop_auto_graph(h);
  return set_scalar_field(h, &h->corr, C, where);
}

int pf_inject_noise(pf_solver* h, const double* w1, const double* w2, int where) {
  if (!h || !w1 || !w2) return fail(h, PF_ERR_INVALID, "pf_inject_noise: null argument");
  if (!h->winj)
    return fail(h, PF_ERR_INVALID,
                "pf_inject_noise: solver was not created with PF_NOISE_SRC_INJECTED and noise_mag != 0");
  const size_t n = 2 * (size_t)h->ncomp * h->g.nspec;  // doubles per field
  int rc = stage_in(h, w1, n, where);
  if (rc) return rc;
  PF_CUDA(h, convert_in(h, h->winj, n));
  rc = stage_in(h, w2, n, where);
  if (rc) return rc;
  PF_CUDA(h, convert_in(h, (char*)h->winj + h->rsz * n, n));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  h->noise_ready = true;
  return PF_OK;
}

int pf_step(pf_solver* h, int nsteps) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (nsteps < 0) return fail(h, PF_ERR_INVALID, "nsteps must be >= 0");
  if (nsteps == 0) return PF_OK;
  return h->prec == PF_FP64 ? step_impl<double>(h, nsteps) : step_impl<float>(h, nsteps);
}

int pf_get_time_member(pf_solver* h, int m, double* t, double* dt) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (m < 0 || m >= h->nmem) return fail(h, PF_ERR_INVALID, "pf_get_time_member: bad member");
  double sc[kScalCount];
  PF_CUDA(h, cudaMemcpyAsync(sc, h->dscal + (size_t)m * kScalCount, sizeof(sc),
                             cudaMemcpyDeviceToHost, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  if (t) *t = sc[kScalTime];
  if (dt) *dt = sc[kScalDt];
  return check_dev_errors(h);
}

int pf_get_time(pf_solver* h, double* t, long long* step, double* dt) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  double sc[kScalCount];
  PF_CUDA(h, cudaMemcpyAsync(sc, h->dscal, sizeof(sc), cudaMemcpyDeviceToHost, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  if (t) *t = sc[kScalTime];
  if (step) *step = h->step;
  if (dt) *dt = sc[kScalDt];
  return check_dev_errors(h);
}

int pf_set_time(pf_solver* h, double t, long long step) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  for (int m = 0; m < h->nmem; ++m)
    PF_CUDA(h, cudaMemcpyAsync(h->dscal + (size_t)m * kScalCount + kScalTime, &t, sizeof(double),
                               cudaMemcpyHostToDevice, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  h->step = step;
  return PF_OK;
}

int pf_energy(pf_solver* h, double* energy, double* enstrophy) {
  return pf_energy_member(h, 0, energy, enstrophy);
}

int pf_energy_member(pf_solver* h, int m, double* energy, double* enstrophy) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (m < 0 || m >= h->nmem) return fail(h, PF_ERR_INVALID, "pf_energy_member: bad member");
  double* tmp = h->dscal + 4;  // slots 4, 5 of member 0 (scratch)
  const size_t ms = (size_t)m * h->d * h->g.nspec;
  PF_CUDA(h, cudaMemsetAsync(tmp, 0, 2 * sizeof(double), h->st));
  cudaError_t e = h->prec == PF_FP64
                      ? launch_energy<double>((const double2*)h->uhat + ms, h->g, tmp, h->st)
                      : launch_energy<float>((const float2*)h->uhat + ms, h->g, tmp, h->st);
  PF_CUDA(h, e);
  double r[2];
  PF_CUDA(h, cudaMemcpyAsync(r, tmp, sizeof(r), cudaMemcpyDeviceToHost, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  if (energy) *energy = r[0];
  if (enstrophy) *enstrophy = r[1];
  return check_dev_errors(h);
}

int pf_record_history(pf_solver* h, int enable) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (enable && h->nmem > 1)
    return fail(h, PF_ERR_UNSUPPORTED, "pf_record_history: per-member energies: pf_energy_member");
  h->record_hist = enable != 0;
  return PF_OK;
}

int pf_history(pf_solver* h, double* out, int max_steps, int* count) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  int rc = flush_hist(h);
  if (rc) return rc;
  const int n = (int)(h->hist.size() / 2);
  const int m = n < max_steps ? n : max_steps;
  if (out && m > 0) memcpy(out, h->hist.data(), sizeof(double) * 2 * m);
  if (count) *count = m;
  h->hist.erase(h->hist.begin(), h->hist.begin() + 2 * m);
  return PF_OK;
}

int pf_spectrum(pf_solver* h, double* out, int nbins) {
  if (!h || !out || nbins <= 0) return fail(h, PF_ERR_INVALID, "pf_spectrum: bad argument");
  if (h->nmem > 1) return fail(h, PF_ERR_UNSUPPORTED, "pf_spectrum: one member per solver");
  double* tmp = nullptr;
  PF_CUDA(h, cudaMalloc(&tmp, sizeof(double) * nbins));
  cudaError_t e = cudaMemsetAsync(tmp, 0, sizeof(double) * nbins, h->st);
  if (e == cudaSuccess)
    e = h->prec == PF_FP64
            ? launch_spectrum<double>((const double2*)h->uhat, h->g, tmp, nbins, h->g.kscale[0], h->st)
            : launch_spectrum<float>((const float2*)h->uhat, h->g, tmp, nbins, h->g.kscale[0], h->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, tmp, sizeof(double) * nbins, cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  if (e != cudaSuccess) return fail(h, PF_ERR_CUDA, std::string("pf_spectrum: ") + cudaGetErrorString(e));
  return PF_OK;
}

}  // extern "C"

// compute_rhs(a) (space_solver.py:302-310) into h->rhs: the nonlinear term by
// the per-operator path (the fused passes hand it to the update without an
// axis-0 spectral copy), then every part per mode.
template <typename R>
static int compute_rhs_impl(pf_solver* h, double a) {
  const Geo& g = h->g;
  const size_t cb = 2 * h->rsz;
  if (!h->rhs) PF_CUDA(h, cudaMalloc(&h->rhs, cb * ((size_t)4 * h->d + 1) * g.nspec));
  if (h->cfg.is_nonlinear)
    PF_CUDA(h, h->padded ? nonlinear_padded<R>(h, false) : nonlinear_generic<R>(h, false));
  const bool forcing = h->cfg.forcing_eps > 0.0;
  if (forcing)
    PF_CUDA(h, launch_band_energy<R>((const cx<R>*)h->uhat, g,
                                     h->cfg.forcing_kf * h->cfg.forcing_kf, h->dscal, h->st));
  UpdateArgs<R> A;
  memset(&A, 0, sizeof(A));
  A.uhat = (cx<R>*)h->uhat;
  A.u0 = (cx<R>*)h->u0;
  A.nl = h->cfg.is_nonlinear ? (const cx<R>*)h->nl : nullptr;
  A.lop = (const R*)h->lop;
  A.corr = (const R*)h->corr;
  A.winj = (const cx<R>*)h->winj;
  A.dscal = h->dscal;
  A.g = g;
  A.coef.a = a;
  A.nu = h->cfg.viscosity;
  A.noise_mag = h->cfg.noise_mag;
  A.noise_norm = noise_norm(h);
  A.f_eps = h->cfg.forcing_eps;
  A.f_kf2 = h->cfg.forcing_kf * h->cfg.forcing_kf;
  A.seed = h->cfg.seed;
  A.step = (uint64_t)(h->step + 1);  // the draws of the next step
  A.noise_src = noise_src(h);
  A.noise_type = h->cfg.noise_type;
  A.nyq_mask = h->cfg.mask_nyquist;
  A.forcing = forcing;
  const long long f = (long long)h->d * g.nspec;
  cx<R>* base = (cx<R>*)h->rhs;
  RhsOut<R> o;
  o.rhs_linear = base;
  o.rhs_nonlinear = base + f;
  o.noise = base + 2 * f;
  o.forcing = base + 3 * f;
  o.p_hat = base + 4 * f;
  PF_CUDA(h, launch_rhs_parts<R>(A, h->ncomp, o, h->st));
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  return PF_OK;
}

extern "C" {

int pf_compute_rhs(pf_solver* h, double a) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (h->nmem > 1) return fail(h, PF_ERR_UNSUPPORTED, "pf_compute_rhs: one member per solver");
  if (h->capturing) return fail(h, PF_ERR_INVALID, "pf_compute_rhs: not inside a graph capture");
  return h->prec == PF_FP64 ? compute_rhs_impl<double>(h, a) : compute_rhs_impl<float>(h, a);
}

int pf_get_rhs(pf_solver* h, int which, double* out, int where) {
  if (!h || !out) return fail(h, PF_ERR_INVALID, "pf_get_rhs: null argument");
  if (which < PF_RHS_LINEAR || which > PF_RHS_P_HAT)
    return fail(h, PF_ERR_INVALID, "pf_get_rhs: unknown array");
  if (!h->rhs) return fail(h, PF_ERR_INVALID, "pf_get_rhs: call pf_compute_rhs first");
  const size_t f = (size_t)h->d * h->g.nspec;
  const size_t n = 2 * (which == PF_RHS_P_HAT ? (size_t)h->g.nspec : f);  // doubles
  PF_CUDA(h, convert_out(h, (const char*)h->rhs + 2 * h->rsz * f * which, n));
  return stage_out(h, out, n, where);
}

int pf_kernel_timer(pf_solver* h, int pass) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  h->tpass = pass;
  h->tused = 0;
  return PF_OK;
}

int pf_kernel_timer_read(pf_solver* h, double* total_ms, long long* launches) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  PF_CUDA(h, cudaStreamSynchronize(h->st));
  double tot = 0.0;
  long long n = 0;
  for (size_t i = 0; i + 1 < h->tused; i += 2) {
    float ms = 0.f;
    PF_CUDA(h, cudaEventElapsedTime(&ms, h->tev[i], h->tev[i + 1]));
    tot += ms;
    ++n;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = n;
  h->tused = 0;
  return PF_OK;
}

int pf_launch_count(long long* count) {
  if (!count) return fail(nullptr, PF_ERR_INVALID, "null pointer");
  *count = launch_total();
  return PF_OK;
}

}  // extern "C"

// Stage coefficients of an integrator (shared with the ensemble batch).
pf::Scheme pf::scheme_for(int integrator) { return make_scheme(integrator); }

template <typename R>
static int capture_steps(pf_solver* h, int nsteps) {
  const bool linear = !h->cfg.is_nonlinear && h->cfg.forcing_eps <= 0.0 && h->cfg.cfl <= 0.0;
  if (linear) return step_stokes<R>(h, nsteps);
  for (int i = 0; i < nsteps; ++i) {
    // an odd count ends with a step that keeps its buffers, so the graph ends
    // on the buffer it starts from and can be replayed again
    h->no_swap_next = (nsteps & 1) && i == nsteps - 1;
    int rc = step_generic<R>(h);
    if (rc) return rc;
  }
  return PF_OK;
}

extern "C" int pf_graph_capture(pf_solver* h, int nsteps) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (nsteps <= 0) return fail(h, PF_ERR_INVALID, "pf_graph_capture: nsteps must be > 0");
  if (!h->st)
    return fail(h, PF_ERR_INVALID, "pf_graph_capture: set a non-default stream first (pf_set_stream)");
  if (noise_src(h) != kNoiseNone)
    return fail(h, PF_ERR_UNSUPPORTED,
                "pf_graph_capture: noisy solvers cannot be captured (the noise step counter is a "
                "launch argument); use pf_step");
  if (h->record_hist)
    return fail(h, PF_ERR_UNSUPPORTED, "pf_graph_capture: history recording is not captured");
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
  const long long l0 = launch_total();
  void* const uhat = h->uhat;
  void* const u0 = h->u0;
  h->graph_parity = state_parity(h);
  h->capturing = true;
  cudaError_t e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal);
  int rc = PF_OK;
  if (e == cudaSuccess) {
    rc = h->prec == PF_FP64 ? capture_steps<double>(h, nsteps) : capture_steps<float>(h, nsteps);
    e = cudaStreamEndCapture(h->st, &h->graph);
  }
  h->capturing = false;
  h->no_swap_next = false;
  h->uhat = uhat;  // recorded, not run
  h->u0 = u0;
  h->graph_launches = launch_total() - l0;
  add_launches(-h->graph_launches);  // recorded, not launched
  if (rc) return rc;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&h->gexec, h->graph, 0);
  if (e != cudaSuccess)
    return fail(h, PF_ERR_CUDA, std::string("pf_graph_capture: ") + cudaGetErrorString(e));
  h->graph_steps = nsteps;
  return PF_OK;
}

extern "C" int pf_graph_replay(pf_solver* h) {
  if (!h || !h->gexec) return fail(h, PF_ERR_INVALID, "pf_graph_replay: nothing captured");
  if (state_parity(h) != h->graph_parity) {
    // steps since the capture left the state in the other buffer: move it back
    PF_CUDA(h, cudaMemcpyAsync(h->u0, h->uhat, 2 * h->rsz * h->d * h->g.nspec * h->nmem,
                               cudaMemcpyDeviceToDevice, h->st));
    std::swap(h->uhat, h->u0);
  }
  PF_CUDA(h, cudaGraphLaunch(h->gexec, h->st));
  add_launches(h->graph_launches);
  h->step += h->graph_steps;
  return PF_OK;
}

extern "C" int pf_autotune(pf_solver* h, int* picks) {
  if (!h) return fail(nullptr, PF_ERR_INVALID, "null handle");
  if (h->capturing) return fail(h, PF_ERR_INVALID, "pf_autotune: not inside a graph capture");
  if (!h->fused) {  // nothing to choose: the per-operator path has one schedule
    if (picks) fused_variants(nullptr, picks);
    return PF_OK;
  }
  PF_CUDA(h, fused_autotune(h->fused, h->uhat, h->nl, h->st, picks));
  drop_auto_graph(h);  // record the new launch variants
  return PF_OK;
}

extern "C" int pf_fused_variants(pf_solver* h, int* out) {
  if (!h || !out) return fail(h, PF_ERR_INVALID, "pf_fused_variants: null argument");
  fused_variants(h->fused, out);
  return PF_OK;
}

extern "C" int pf_footprint(const pf_config* c, unsigned long long* bytes) {
  return pf_footprint_members(c, 1, bytes);
}

// Device bytes of create_impl(c, nmem): per-member buffers (state, u0, nl,
// scalars, fused pass buffers) times nmem, shared scratch once.
extern "C" int pf_footprint_members(const pf_config* c, int nmem, unsigned long long* bytes) {
  if (!c || !bytes) return fail(nullptr, PF_ERR_INVALID, "pf_footprint: null argument");
  if (nmem < 1) return fail(nullptr, PF_ERR_INVALID, "pf_footprint_members: members must be >= 1");
  int rc = validate(c);
  if (rc) return rc;
  const unsigned long long M = (unsigned long long)nmem;
  const int d = c->dim;
  long long nspec = 1, nphys = 1;
  for (int a = 0; a < d; ++a) {
    nspec *= (a == d - 1) ? (c->n[a] / 2 + 1) : c->n[a];
    nphys *= c->n[a];
  }
  const unsigned long long rsz = c->precision == PF_FP64 ? 8 : 4, cb = 2 * rsz;
  const int ncomp = c->noise_type == PF_NOISE_THERMAL ? d * d : d;
  unsigned long long st64 = std::max((unsigned long long)(2 * d * nspec), (unsigned long long)(d * nphys));
  st64 = std::max(st64, (unsigned long long)(4 * ncomp * nspec));
  unsigned long long b = M * (cb * d * nspec * 2 + 8 * kScalCount + 8) + cb * 3 * nspec +
                         8 * st64 + 16 * kHist;
  if (c->is_nonlinear && c->dealias == PF_DEALIAS_PAD) {
    unsigned long long msp = 1, mph = 1;
    for (int a = 0; a < d; ++a) {
      const int m = 3 * c->n[a] / 2;
      msp *= (a == d - 1) ? (m / 2 + 1) : m;
      mph *= m;
    }
    b += cb * d * nspec + cb * 3 * msp + rsz * d * mph + rsz * (d == 3 ? 3 : 1) * mph;
    bool fz = d == 3 && c->fused && c->n[2] <= 256;
    for (int a = 0; fz && a < 3; ++a)
      fz = c->n[a] >= 16 && c->n[a] <= 256 && (c->n[a] & (c->n[a] - 1)) == 0;
    if (fz) {  // fused 3/2 schedule: pass buffers on the padded x0 (and x1) grid
      const unsigned long long t0 = 3ull * c->n[0] / 2, t1 = 3ull * c->n[1] / 2;
      const unsigned long long nh = c->n[2] / 2 + 1;
      b += M * cb * (5ull * t0 * c->n[1] * nh + 6ull * t0 * t1 * nh + 3ull * t0 * t1 * nh);
    }
  } else if (c->is_nonlinear) {
    b += M * cb * d * nspec + rsz * d * nphys + rsz * (d == 3 ? 3 : 1) * nphys;
    bool pow2 = d == 3 && c->fused;
    const int nmax = c->precision == PF_FP32 ? 512 : 256;
    for (int a = 0; pow2 && a < 3; ++a) {
      const int n = c->n[a], m = n / 3;
      const bool p2 = n >= 16 && n <= nmax && (n & (n - 1)) == 0 && (a < 2 || n <= 256);
      const bool t2 = c->precision == PF_FP32 && n % 3 == 0 && n >= 48 && n <= 384 &&
                      (m & (m - 1)) == 0;
      pow2 = p2 || t2;
    }
    if (pow2) {
      const unsigned long long k1 = (c->n[1] - 1) / 3, k2 = (c->n[2] - 1) / 3;
      b += M * cb * (5ull * c->n[0] * (2 * k1 + 1) * (k2 + 1) + 6ull * c->n[0] * c->n[1] * (k2 + 1));
    }
    bool f2 = d == 2 && c->fused;
    for (int a = 0; f2 && a < 2; ++a)
      f2 = c->n[a] >= 16 && c->n[a] <= 1024 && (c->n[a] & (c->n[a] - 1)) == 0;
    if (f2) b += M * cb * 3ull * c->n[0] * ((c->n[1] - 1) / 3 + 1);  // 2D fused pass-1 scratch
  }
  if (c->noise_mag != 0.0 && c->noise_source == PF_NOISE_SRC_INJECTED) b += cb * 2 * ncomp * nspec;
  *bytes = b;
  return PF_OK;
}
