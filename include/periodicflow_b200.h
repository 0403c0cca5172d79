/*
 * periodicflow_b200.h -- C ABI of the B200 backend of periodicflow's
 * right-hand-side and time-stepping path.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (PF_OK == 0).  Complex arrays are interleaved (re, im) doubles in the
 * reference's layout: spectral fields (comp, n0, n1, n2/2+1) in 3D and
 * (comp, n0, n1/2+1) in 2D; physical fields (comp, n0, n1[, n2]).  A handle
 * is not thread-safe; all of its work is ordered on one CUDA stream.
 *
 * Reference interfaces replaced (paths inside the periodic-flow project):
 *   Solver.__init__            src/periodicflow/simulation.py:56-114
 *   SpaceSolver.__init__       src/periodicflow/space_solver.py:107-150
 *   FourierSpace.__init__      src/periodicflow/basis.py:34-92
 *   Solver.initialize          src/periodicflow/simulation.py:161-180
 *   initialize_velocity        src/periodicflow/space_solver.py:180-213
 *   forward / backward         src/periodicflow/space_solver.py:215-225
 *   set_linear_operator        src/periodicflow/simulation.py:182-184
 *   update_linear_operator     src/periodicflow/time_integrator.py:31-33
 *   set_correlation_function   src/periodicflow/simulation.py:186-187
 *   random_fields              src/periodicflow/space_solver.py:227-238
 *   Solver.solve loop body     src/periodicflow/simulation.py:205-217
 *   compute_rhs                src/periodicflow/space_solver.py:302-310
 *   TimeIntegrator.stepping    src/periodicflow/time_integrator.py:36-318
 *   math.cross/curl/apply_linear_operator/leray_projection
 *                              src/periodicflow/math.py:4-100
 *   _symmetrize/_noise_divergence
 *                              src/periodicflow/space_solver.py:15-64
 */
#ifndef PERIODICFLOW_B200_H
#define PERIODICFLOW_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PF_OK 0
#define PF_ERR_INVALID 1     /* bad argument (the reference raises ValueError) */
#define PF_ERR_CUDA 2        /* CUDA runtime error */
#define PF_ERR_UNSUPPORTED 3 /* valid in the reference, not built here */
#define PF_ERR_NOMEM 4

/* integrators: registry names of time_integrator.py:36,93,161,213,278 */
#define PF_EXPLICIT_PC 0
#define PF_IMPLICIT_PC 1
#define PF_RK2 2
#define PF_RK3 3
#define PF_RK4 4

#define PF_NOISE_THERMAL 0    /* space_solver.py:254-259 */
#define PF_NOISE_CORRELATED 1 /* space_solver.py:261-265 */

#define PF_NOISE_SRC_PHILOX 1   /* counter-based, Hermitian-symmetric draws */
#define PF_NOISE_SRC_INJECTED 2 /* caller supplies w1, w2 every step */

#define PF_DEALIAS_TRUNCATE 0 /* '2/3' / 'truncate' (basis.py:82-83) */
#define PF_DEALIAS_PAD 1      /* '3/2' / 'pad' (basis.py:80-81) */

#define PF_FP32 0
#define PF_FP64 1

typedef struct pf_config {
  int dim;                /* 2 or 3 */
  int n[3];               /* grid points per axis: 2^b 4..1024 or 3 * 2^b 12..768 */
  double domain[3][2];    /* (start, end) per axis */
  int is_nonlinear;       /* simulation.py:61 */
  int integrator;         /* PF_EXPLICIT_PC .. PF_RK4 */
  double viscosity;       /* L = -viscosity |k|^2 (space_solver.py:147) */
  int noise_type;         /* PF_NOISE_THERMAL / PF_NOISE_CORRELATED */
  double noise_mag;       /* 0 disables the noise term */
  int dealias;            /* PF_DEALIAS_TRUNCATE or PF_DEALIAS_PAD */
  int mask_nyquist;       /* zero Nyquist modes of the nonlinear term */
  int precision;          /* PF_FP32 / PF_FP64 */
  double dt;
  unsigned long long seed;/* Philox key */
  int noise_source;       /* PF_NOISE_SRC_PHILOX / PF_NOISE_SRC_INJECTED */
  double forcing_eps;     /* >0: linear band forcing at injection rate eps */
  double forcing_kf;      /* forced band 0 < |k| <= kf */
  double cfl;             /* >0: dt = cfl / max(sum_i |u_i| / dx_i) each step */
  int fused;              /* 1: fused pencil passes where built; 0: per-operator */
} pf_config;

typedef struct pf_solver pf_solver;

/* Fill cfg with the reference's defaults (simulation.py:56-79; dealias 2/3). */
int pf_config_default(pf_config* cfg);

/* Create a solver on the current CUDA device; state is zero. */
int pf_create(const pf_config* cfg, pf_solver** out);
/* Device bytes pf_create allocates for cfg (admission control; no device use). */
int pf_footprint(const pf_config* cfg, unsigned long long* bytes);
int pf_destroy(pf_solver* h);
/* Order the handle's work on this cudaStream_t (NULL = legacy default). */
int pf_set_stream(pf_solver* h, void* stream);
/* Message of the last failing call on h (static text when h is NULL). */
const char* pf_last_error(const pf_solver* h);

/* Extents: spectral modes per component, physical points per component,
 * noise components (d*d thermal, d correlated). */
int pf_sizes(const pf_solver* h, long long* nspec, long long* nphys, int* ncomp);

/* State transfer.  `where` = 0: host pointer, 1: device pointer.
 * Fourier data are complex128 (2 doubles per value), physical data float64. */
int pf_set_fourier(pf_solver* h, const double* u_hat, int where);
int pf_get_fourier(pf_solver* h, double* u_hat, int where);
/* physical -> spectral with the normalised forward transform (V.forward) */
int pf_set_physical(pf_solver* h, const double* u, int where);
/* spectral -> physical with the backward transform (V.backward) */
int pf_get_physical(pf_solver* h, double* u, int where);
/* initialize(): zero the k = 0 mode (space_solver.py:208-209) */
int pf_mask_zero_mode(pf_solver* h);
/* initialize(project=True): Leray projection of the state (simulation.py:170-176) */
int pf_project(pf_solver* h);

/* L(k) and C(k) as float64 arrays of the scalar spectral shape; NULL restores
 * the defaults (-viscosity |k|^2 and zero). */
int pf_set_linear_operator(pf_solver* h, const double* L, int where);
int pf_set_correlation(pf_solver* h, const double* C, int where);

/* Noise of the next step for PF_NOISE_SRC_INJECTED: w1, w2 as stored by the
 * reference after random_fields() (normal factor applied), complex128 of shape
 * (ncomp, spectral). */
int pf_inject_noise(pf_solver* h, const double* w1, const double* w2, int where);

/* Advance nsteps full time steps (all stages) on the device. */
int pf_step(pf_solver* h, int nsteps);
/* Capture "advance nsteps" as a CUDA graph on the handle's (non-default)
 * stream; pf_graph_replay launches it with one call.  Noise-free solvers only
 * (the noise step counter is a launch argument), without history recording. */
int pf_graph_capture(pf_solver* h, int nsteps);
int pf_graph_replay(pf_solver* h);

/* Autotuner (no reference counterpart; the reference has one CPU schedule):
 * times every launch variant of the fused passes 1-4 (radix width, columns
 * per CTA, register cap, staging depth, values per lane) inside the chain of
 * passes 1-4 on this solver's buffers and keeps the fastest; later solvers of the same geometry (precision, dealias rule,
 * sides) in this process start from the picks.  Leaves the state unchanged;
 * synchronous; not inside a graph capture.  picks (12 ints, may be NULL):
 * variants of passes 0..5 for 256-point axes, then for 384-point axes.
 * A no-op for solvers without the fused schedule. */
int pf_autotune(pf_solver* h, int* picks);
/* Current launch variants (same 12-int layout as pf_autotune). */
int pf_fused_variants(pf_solver* h, int* out);

/* Time, step counter and current dt (synchronises the stream). */
int pf_get_time(pf_solver* h, double* t, long long* step, double* dt);
/* Set time / step counter (restart). */
int pf_set_time(pf_solver* h, double t, long long step);
/* Kinetic energy and enstrophy of the current state (FP64 reductions). */
int pf_energy(pf_solver* h, double* energy, double* enstrophy);
/* Per-step E, Z recorded by pf_step since the last call (2 doubles per
 * step, at most max_steps); returns the count in *count. */
int pf_history(pf_solver* h, double* out, int max_steps, int* count);
/* Record E, Z of every step inside pf_step (0/1). */
int pf_record_history(pf_solver* h, int enable);
/* Shell spectrum E(k), nbins bins of width 2 pi / L0. */
int pf_spectrum(pf_solver* h, double* out, int nbins);

/* SpaceSolver.compute_rhs(a) (space_solver.py:302-310) on the current state,
 * into arrays of the solver read back with pf_get_rhs (the time step itself
 * fuses these terms into the stage update and never stores them):
 *   PF_RHS_LINEAR     L u_hat                          (space_solver.py:273-277)
 *   PF_RHS_NONLINEAR  P[F(u x omega)], Nyquist-masked if configured; zero for
 *                     linear solvers                   (space_solver.py:279-300)
 *   PF_RHS_NOISE      noise_mag P[xi(w1 + a w2)] with the noise fields of the
 *                     next step (Philox draws keyed by it, or the last
 *                     injected w1, w2)                 (space_solver.py:240-265)
 *   PF_RHS_FORCING    the band forcing (zero without)  (space_solver.py:267-271)
 *   PF_RHS_P_HAT      (k/k^2).xi before the noise_mag scale: the output of the
 *                     last Leray projection of compute_rhs, as the reference
 *                     leaves p_hat; zero when noise_mag is 0 (no draws)
 * Arrays are (dim, spectral) complex128, p_hat (spectral).  Synchronous. */
#define PF_RHS_LINEAR 0
#define PF_RHS_NONLINEAR 1
#define PF_RHS_NOISE 2
#define PF_RHS_FORCING 3
#define PF_RHS_P_HAT 4
int pf_compute_rhs(pf_solver* h, double a);
int pf_get_rhs(pf_solver* h, int which, double* out, int where);

/* ---- measurement ------------------------------------------------------- */
/* kernel passes that can be timed */
#define PF_PASS_UPDATE 0        /* fused stage update (Leray, L, noise, forcing) */
#define PF_PASS_FFT_STRIDED 1   /* complex FFT along a strided axis */
#define PF_PASS_FFT_LAST 2      /* C2R / R2C along the contiguous axis */
#define PF_PASS_STOKES 4        /* whole steps of the linear problem */
#define PF_PASS_FUSED_P1 11     /* fused nonlinear passes P1..P5 */
#define PF_PASS_FUSED_P2 12
#define PF_PASS_FUSED_P3 13
#define PF_PASS_FUSED_P4 14
#define PF_PASS_FUSED_P5 15
/* Time every launch of `pass` with CUDA events on the handle's stream
 * (-1 disables); accumulators restart.  Steps captured with pf_graph_capture
 * while the timer is on carry its events as graph nodes: read the timer after
 * one replay (a further replay records the same events again). */
int pf_kernel_timer(pf_solver* h, int pass);
/* Sum of the timed launch durations (ms) and their count since the last read. */
int pf_kernel_timer_read(pf_solver* h, double* total_ms, long long* launches);
/* Total kernels launched by this library in this process. */
int pf_launch_count(long long* count);

/* ---- ensembles of linear boxes -------------------------------------------
 * No single reference counterpart: the reference runs one realisation per
 * mpirun (simulation.py:189-225).  A batch advances many independent linear
 * solvers (is_nonlinear = 0, no forcing, fixed dt, Philox or no noise) of
 * mixed sizes and dimensions with one kernel launch per call, each mode's
 * state in registers for all stages and steps.  Members keep owning their
 * state; they must share precision, integrator and noise type, and must be
 * idle (no work queued on their own streams) while batch work runs. */
typedef struct pf_batch pf_batch;
int pf_batch_create(pf_solver* const* members, int count, pf_batch** out);
int pf_batch_destroy(pf_batch* b);
int pf_batch_set_stream(pf_batch* b, void* stream);
const char* pf_batch_last_error(const pf_batch* b);
/* Advance every member nsteps (synchronous). */
int pf_batch_step(pf_batch* b, int nsteps);
/* Capture "advance nsteps" into a CUDA graph on the batch stream (must be a
 * non-default stream); pf_batch_replay launches it (asynchronous). */
int pf_batch_capture(pf_batch* b, int nsteps);
int pf_batch_replay(pf_batch* b);
int pf_batch_sync(pf_batch* b);

/* ---- realisations of one configuration in one launch ---------------------
 * No single reference counterpart: the reference runs one realisation per
 * mpirun (simulation.py:189-225).  pf_create_members makes one handle for
 * `members` boxes of cfg -- nonlinear, with a fused schedule (3D 2/3 rule
 * FP32/FP64 and 3/2 rule, 2D 2/3 rule), no injected noise -- whose states sit
 * one after another on the device; every fused pass of a stage is one launch
 * over all members, and each member keeps its own dt (CFL), time and forcing
 * band energy.  Member m draws Philox noise with seed cfg->seed + m, so it
 * equals a single solver created with that seed.  pf_step, pf_graph_capture /
 * pf_graph_replay, pf_autotune, pf_set_linear_operator / pf_set_correlation
 * (shared by all members), pf_project and pf_mask_zero_mode act on every
 * member; pf_set_fourier / pf_get_fourier move all members' states as one
 * (members, dim, spectral) array; pf_get_time and pf_energy report member 0.
 * Physical-space transfers, pf_spectrum, pf_compute_rhs and history
 * recording take one-member handles (PF_ERR_UNSUPPORTED otherwise). */
int pf_create_members(const pf_config* cfg, int members, pf_solver** out);
int pf_footprint_members(const pf_config* cfg, int members, unsigned long long* bytes);
int pf_members(const pf_solver* h, int* members);
int pf_set_fourier_member(pf_solver* h, int member, const double* u_hat, int where);
int pf_get_fourier_member(pf_solver* h, int member, double* u_hat, int where);
int pf_get_time_member(pf_solver* h, int member, double* t, double* dt);
int pf_energy_member(pf_solver* h, int member, double* energy, double* enstrophy);
/* Continuous batching of members (no reference counterpart): pf_step advances
 * only members [0, active) -- the others keep their state and time -- so
 * requests join at slot `active` and leave by moving the last active member
 * into their slot.  Changing the count re-records the internal step graph;
 * graphs captured with pf_graph_capture keep the count they were captured
 * with.  pf_copy_member copies state, time and dt (device to device);
 * pf_set_time_member sets one member's time and dt. */
int pf_set_active_members(pf_solver* h, int active);
int pf_copy_member(pf_solver* h, int dst, int src);
int pf_set_time_member(pf_solver* h, int member, double t, double dt);

/* ---- slab decomposition of one box ---------------------------------------
 * Replaces the reference's decomposition='slab' (basis.py:64, the shenfun
 * TensorProductSpace with slab=True built over simulation.py:81-83's
 * COMM_WORLD): the box is split into S slabs; slab r holds the spectral rows
 * k1 in [r n1/S, (r+1) n1/S) of every (k0, k2) -- its u_hat is the local
 * array [3][n0][n1/S][n2/2+1] complex128 -- and, between the transposes of
 * the nonlinear term, the physical planes x0 in [r n0/S, (r+1) n0/S).  The
 * transposes are stores of the passes before them into the destination
 * slab's buffers.  Built for the 3D nonlinear problem with the 2/3 rule
 * (FP32, FP64; the fused-schedule sides), every integrator, CFL dt, band
 * forcing, Nyquist mask and thermal Philox noise (draws equal to a single
 * box's); S <= 8 dividing n0 and n1, (n0/S) n1 a multiple of 64.
 *
 * pf_slab_create_group holds all S slabs in this process on the current
 * device.  pf_slab_create holds slab `slab` only (one process per GPU):
 * every process exports its exchange buffers (pf_slab_export, CUDA IPC
 * handles), process 0 makes an NCCL id (pf_slab_nccl_id, 128 bytes), both
 * are shared (e.g. by an MPI allgather / bcast), and pf_slab_connect maps the
 * peers' buffers and joins the NCCL communicator that carries the exchange
 * barriers and the CFL / forcing reductions.  pf_slab_step is collective. */
typedef struct pf_slab pf_slab;
int pf_slab_layout(int n0, int n1, int slabs, int slab, int* out6);  /* n0/S, n1/S, x0 first, k1 first, kept compact k1 first, count */
int pf_slab_create_group(const pf_config* cfg, int slabs, pf_slab** out);
int pf_slab_create(const pf_config* cfg, int slabs, int slab, pf_slab** out);
int pf_slab_export(const pf_slab* h, void* out, size_t cap, size_t* used);
int pf_slab_nccl_id(void* out, size_t cap);
int pf_slab_connect(pf_slab* h, const void* exports, const void* nccl_id);  /* exports: S blocks in slab order */
int pf_slab_destroy(pf_slab* h);
const char* pf_slab_last_error(const pf_slab* h);
int pf_slab_set_stream(pf_slab* h, void* stream);
int pf_slab_sizes(const pf_slab* h, int* first, int* count, long long* nspec);  /* slabs held, modes per slab */
int pf_slab_set_fourier(pf_slab* h, int slab, const double* u_hat, int where);
int pf_slab_get_fourier(pf_slab* h, int slab, double* u_hat, int where);
int pf_slab_step(pf_slab* h, int nsteps);
int pf_slab_sync(pf_slab* h);
int pf_slab_get_time(pf_slab* h, double* t, long long* step, double* dt);
int pf_slab_energy(pf_slab* h, int slab, double* energy, double* enstrophy);  /* the slab's part */

/* ---- backward transform without device allocation ----------------------
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc (a fixed memory budget handed over by an embedding application,
 * a context where the allocator must not be entered, up-front accounting of
 * every allocation).  Same result as pf_get_physical (the reference's
 * V.backward, space_solver.py:221-225) for a spectral field the caller already
 * holds on the device: u_hat (dim, spectral) complex and u (dim, n...) real,
 * both device arrays of the given precision.  The transform's work copy lives
 * in one fixed 32 MiB device array of the library (held by every GPU that
 * loads it until exit): requests needing more than dim * nspec complex values
 * of 32 MiB are rejected with PF_ERR_INVALID.  The first call on a device sets
 * up that array's address and the FFT tables -- make it before any stream
 * capture.  Calls share the array, so calls that overlap on the GPU race;
 * serialise them on one stream.  Allocates nothing. */
int pf_backward_noalloc(int precision, int dim, const int* n, const void* u_hat, void* u,
                        void* stream);

/* ---- operators on device arrays (math.py / space_solver.py kernels) ------
 * Arrays are device pointers of element type double (PF_FP64) or float
 * (PF_FP32); complex arrays interleaved.  shape = spatial extents of one
 * component (dim entries).  Semantics are those of the reference functions. */
int pf_op_cross(int precision, int dim, const long long* shape, void* c, const void* a,
                const void* b, void* stream);
int pf_op_curl(int precision, int dim, const long long* shape, void* c, const void* k,
               const void* a, void* stream);
int pf_op_apply_linear_operator(int precision, int dim, const long long* shape, void* Lu,
                                const void* L, const void* u, void* stream);
int pf_op_leray_projection(int precision, int dim, const long long* shape, void* u,
                           const void* k, const void* k_over_k2, void* p_hat, void* stream);
int pf_op_symmetrize(int precision, int dim, const long long* shape, void* w_sym,
                     const void* w, void* stream);
int pf_op_noise_divergence(int precision, int dim, const long long* shape, void* noise,
                           const void* w_sym, const void* k, void* stream);
/* One stage of an integrator on device arrays (TimeIntegrator.stepping):
 * unew updated in place; for PF_IMPLICIT_PC the last stage overwrites
 * rhs_linear with L u0 as the reference does.  L may be NULL for integrators
 * that do not use it. */
int pf_op_stepping(int precision, int integrator, int stage, double dt, long long n,
                   void* unew, const void* u0, const void* rhs_nonlinear, void* rhs_linear,
                   const void* forcing, const void* noise, const void* L,
                   long long n_per_comp, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PERIODICFLOW_B200_H */
