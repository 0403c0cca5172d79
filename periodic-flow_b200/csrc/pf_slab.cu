// Slab decomposition of one 3D box over S slabs -- the reference's
// decomposition='slab' (basis.py:64: shenfun's TensorProductSpace with
// slab=True, which keeps physical arrays split along axis 0 and spectral
// arrays along axis 1, and moves between them by alltoall transposes).
//
// Slab r holds the spectral rows k1 in [r n1/S, (r+1) n1/S) of every (k0, k2):
// its state is u_hat[3][n0][n1/S][nh].  One evaluation of the nonlinear term
// runs the fused 2/3-rule schedule with the two transposes folded into the
// stores of the passes before them:
//
//   P1  (slab r) inverse FFT along axis 0 of r's kept columns; plane x0 is
//       stored straight into slab x0 / (n0/S)'s pass-1 buffer
//   --  exchange barrier
//   P2, P3, P4 (slab s) on s's n0/S planes x0 (the whole-box kernels); P4's
//       row k1 is stored straight into slab k1 / (n1/S)'s nonlinear buffer
//   --  exchange barrier; CFL maximum and forcing band energy reduced over
//       the slabs
//   P5  (slab r) forward FFT along axis 0 and the stage update of r's columns
//
// Two barriers per stage order every cross-slab store after the reads of the
// previous use of its destination (a slab's P1 of stage s+1 follows the
// barrier after every slab's P4 of stage s, hence after their P2 reads; a
// slab's P4 follows the barrier after every slab's P1, hence after their P5).
//
// Two ways to hold the slabs:
//  * a group: all S slabs in one process on one device; the destinations
//    are the other slabs' buffers and the barriers are stream order;
//  * one slab per process and GPU: the destinations are the peers' buffers
//    mapped by CUDA IPC (plain stores over NVLink, no multicast), and the
//    barriers and reductions are NCCL all-reduces on the solver's stream
//    (libnccl.so.2 loaded at connect time).
#include <dlfcn.h>
#include <nccl.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/periodicflow_b200.h"
#include "pf_fused_impl.cuh"

namespace pf {
namespace {

// ------------------------------------------------------------ slab layout
struct SlabLayout {
  int n0s, n1s;  // planes x0 / rows k1 per slab
  int x0, i1;    // first plane / row of slab r
  int c0, nc;    // its kept compact k1 rows (2/3 rule)
};

// compact index of kept row i (|kfreq(i)| <= kmax) of an axis of n points
int compact_of(int i, int n, int kmax) { return i <= kmax ? i : i - (n - (2 * kmax + 1)); }

SlabLayout slab_layout(int n0, int n1, int S, int r) {
  SlabLayout L;
  L.n0s = n0 / S;
  L.n1s = n1 / S;
  L.x0 = r * L.n0s;
  L.i1 = r * L.n1s;
  const int kmax = (n1 - 1) / 3;
  // kept rows of [i1, i1 + n1s) form one compact range (the compact map is
  // increasing on the kept rows)
  int lo = -1, hi = -1;
  for (int i = L.i1; i < L.i1 + L.n1s; ++i) {
    if (std::abs(kfreq(i, n1)) > kmax) continue;
    const int c = compact_of(i, n1, kmax);
    if (lo < 0) lo = c;
    hi = c + 1;
  }
  L.c0 = lo < 0 ? 0 : lo;
  L.nc = lo < 0 ? 0 : hi - lo;
  return L;
}

// ------------------------------------------------------------ kernels
// E_band (forcing) of one slab: 1/2 sum over its modes with 0 < |k|^2 <= kf2
// of w |u|^2 into dscal[kScalBandE] (zeroed by the caller).  Visits the
// slab's rows k1 against the index box |k0| <= K0, k2 <= K2.
template <typename R>
__global__ void k_slab_band_energy(const cx<R>* __restrict__ u, Geo g, int n1s, int i1lo,
                                   double kf2, int cnt0, int K0, int cnt2, double* dscal) {
  double acc = 0.0;
  const long long total = (long long)cnt0 * n1s * cnt2;
  for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < total;
       b += (long long)gridDim.x * blockDim.x) {
    const int i2 = (int)(b % cnt2);
    const long long r = b / cnt2;
    const int i1l = (int)(r % n1s);
    const int s0 = (int)(r / n1s);
    const int i0 = cnt0 == g.n[0] ? s0 : ((s0 - K0) % g.n[0] + g.n[0]) % g.n[0];
    const int i1 = i1l + i1lo;
    const double k0 = g.kscale[0] * kfreq(i0, g.n[0]), k1 = g.kscale[1] * kfreq(i1, g.n[1]),
                 k2 = g.kscale[2] * i2;
    const double kk = k0 * k0 + k1 * k1 + k2 * k2;
    if (kk > 0.0 && kk <= kf2) {
      const long long m = ((long long)i0 * n1s + i1l) * g.nh + i2;
      double e = 0.0;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const cx<R> z = u[a * g.nspec + m];
        e += (double)z.x * z.x + (double)z.y * z.y;
      }
      ModeIdx ix;
      ix.i0 = i0; ix.i1 = i1; ix.i2 = i2;
      acc += 0.5 * half_weight(g, ix) * e;
    }
  }
  block_add2(acc, 0.0, dscal + kScalBandE);
}

// E and Z of one slab's modes into out2[0], out2[1] (zeroed by the caller).
template <typename R>
__global__ void k_slab_energy(const cx<R>* __restrict__ u, Geo g, int n1s, int i1lo,
                              double* out2) {
  double accE = 0.0, accZ = 0.0;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const int i2 = (int)(m % g.nh);
    const long long r = m / g.nh;
    const int i1 = (int)(r % n1s) + i1lo;
    const int i0 = (int)(r / n1s);
    const double k0 = g.kscale[0] * kfreq(i0, g.n[0]), k1 = g.kscale[1] * kfreq(i1, g.n[1]),
                 k2 = g.kscale[2] * i2;
    double e = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const cx<R> z = u[a * g.nspec + m];
      e += (double)z.x * z.x + (double)z.y * z.y;
    }
    ModeIdx ix;
    ix.i0 = i0; ix.i1 = i1; ix.i2 = i2;
    const double w = half_weight(g, ix);
    accE += 0.5 * w * e;
    accZ += 0.5 * w * e * (k0 * k0 + k1 * k1 + k2 * k2);
  }
  block_add2(accE, accZ, out2);
}

// The reductions of a group (one thread): CFL maximum over the slabs'
// words, band energy summed over the slabs' rows; the result to every slab.
struct GroupScalars {
  unsigned long long* maxbits[kMaxSlabs];
  double* dscal[kMaxSlabs];
};
__global__ void k_group_reduce(GroupScalars gs, int S, int do_max, int do_band) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (do_max) {
    unsigned long long m = 0;
    for (int s = 0; s < S; ++s) m = *gs.maxbits[s] > m ? *gs.maxbits[s] : m;
    for (int s = 0; s < S; ++s) *gs.maxbits[s] = m;
  }
  if (do_band) {
    double e = 0.0;
    for (int s = 0; s < S; ++s) e += gs.dscal[s][kScalBandE];
    for (int s = 0; s < S; ++s) gs.dscal[s][kScalBandE] = e;
  }
}

// ------------------------------------------------------------ launchers
// P1 of one slab: the one-field-per-CTA-row form with the default tile.
template <typename R, int N> cudaError_t slab_p1_n(const FGeo& f, const cx<R>* uh, cudaStream_t st) {
  using TS = TuneS<N, R>;
  constexpr int E = TS::E, T = TS::T, G = N / E;
  if (f.sl_nc == 0) return cudaSuccess;  // no kept row k1 in this slab
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const size_t sm = strided_smem<R, N, E, T, false>();
  auto kern = k_p1<R, N, E, T, 0, false, true, false, true>;
  cudaError_t e = set_smem(kern, sm);
  if (e != cudaSuccess) return e;
  const long long ncols = (long long)f.sl_nc * f.c2;
  kern<<<dim3((unsigned)((ncols + T - 1) / T), 5), dim3(T, G), sm, st>>>(uh, nullptr, f, tw);
  return launched();
}

template <typename R, int N> cudaError_t slab_p4_n(const FGeo& f, cx<R>* nl, cudaStream_t st) {
  using TS = TuneS<N, R>;
  constexpr int E = TS::E, T = TS::T, G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const size_t sm = strided_smem<R, N, E, T, false>();
  auto kern = k_p4<R, N, E, T, 0, false, false, true>;
  cudaError_t e = set_smem(kern, sm);
  if (e != cudaSuccess) return e;
  const long long ncols = (long long)3 * f.t0 * f.nh;
  kern<<<(unsigned)((ncols + T - 1) / T), dim3(T, G), sm, st>>>(nl, f, tw);
  return launched();
}

template <typename R, int N, bool NOISE, int NC>
cudaError_t slab_p5_go(const FGeo& f, const UpdateArgs<R>& U, const cx<R>* nl, cudaStream_t st) {
  using TN = TuneU<N, R>;
  constexpr int CH = sizeof(R) == 8 ? 2 : 4;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const size_t sm = sizeof(cx<R>) * 3 * N * TN::T;
  auto kern = k_p5<R, N, NC, NOISE, CH, false, false, true>;
  cudaError_t e = set_smem(kern, sm);
  if (e != cudaSuccess) return e;
  const long long ncols = (long long)f.sl_n1 * f.nh;
  kern<<<dim3((unsigned)((ncols + TN::T - 1) / TN::T), 1), dim3(TN::T, TN::G), sm, st>>>(U, nl, f,
                                                                                         tw);
  return launched();
}
template <typename R, int N>
cudaError_t slab_p5_n(const FGeo& f, const UpdateArgs<R>& U, const cx<R>* nl, cudaStream_t st) {
  if (U.noise_src == kNoiseNone) return slab_p5_go<R, N, false, 3>(f, U, nl, st);
  return slab_p5_go<R, N, true, 9>(f, U, nl, st);  // thermal noise, Philox draws
}

template <typename R> cudaError_t slab_p1(const FGeo& f, const void* uh, cudaStream_t st) {
#define PF_CALL(NN) slab_p1_n<R, NN>(f, (const cx<R>*)uh, st)
  if constexpr (sizeof(R) == 4) {
    PF_SWITCH_T(f.n0, PF_CALL)
  } else {
    PF_SWITCH_S(f.n0, PF_CALL)
  }
#undef PF_CALL
}
template <typename R> cudaError_t slab_p4(const FGeo& f, void* nl, cudaStream_t st) {
#define PF_CALL(NN) slab_p4_n<R, NN>(f, (cx<R>*)nl, st)
  if constexpr (sizeof(R) == 4) {
    PF_SWITCH_T(f.n1, PF_CALL)
  } else {
    PF_SWITCH_S(f.n1, PF_CALL)
  }
#undef PF_CALL
}
template <typename R>
cudaError_t slab_p5(const FGeo& f, const UpdateArgs<R>& U, const void* nl, cudaStream_t st) {
#define PF_CALL(NN) slab_p5_n<R, NN>(f, U, (const cx<R>*)nl, st)
  if constexpr (sizeof(R) == 4) {
    PF_SWITCH_T(f.n0, PF_CALL)
  } else {
    PF_SWITCH_S(f.n0, PF_CALL)
  }
#undef PF_CALL
}

// ------------------------------------------------------------ NCCL
// The few entry points the slab exchange uses, from libnccl.so.2 (the copy
// already loaded by the process, e.g. torch's, when there is one).
struct Nccl {
  bool ok = false;
  std::string why;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
};

const Nccl& nccl() {
  static Nccl n;
  static std::once_flag once;
  std::call_once(once, [] {
    void* lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) lib = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!lib) {
      const char* e = dlerror();
      n.why = std::string("libnccl.so.2 not found: ") + (e ? e : "");
      return;
    }
    n.GetUniqueId = (decltype(n.GetUniqueId))dlsym(lib, "ncclGetUniqueId");
    n.CommInitRank = (decltype(n.CommInitRank))dlsym(lib, "ncclCommInitRank");
    n.AllReduce = (decltype(n.AllReduce))dlsym(lib, "ncclAllReduce");
    n.CommDestroy = (decltype(n.CommDestroy))dlsym(lib, "ncclCommDestroy");
    n.GetErrorString = (decltype(n.GetErrorString))dlsym(lib, "ncclGetErrorString");
    n.ok = n.GetUniqueId && n.CommInitRank && n.AllReduce && n.CommDestroy && n.GetErrorString;
    if (!n.ok) n.why = "libnccl.so.2 lacks an entry point";
  });
  return n;
}

}  // namespace
}  // namespace pf

using namespace pf;

// One slab's buffers.  A (pass-1 buffer, in the pencil plan) and nlx (P4's
// destination, P5's input) are written by every slab.
struct SlabBuf {
  void* uhat = nullptr;      // [3][n0][n1s][nh]
  void* u0 = nullptr;
  void* nl = nullptr;        // P3 output / P4 input [3][n0s][n1][nh]
  void* nlx = nullptr;       // [3][n0][n1s][nh]
  double* dscal = nullptr;   // kScalCount doubles
  unsigned long long* maxbits = nullptr;
  double* e2 = nullptr;      // energy sums
  FusedPlan* pp = nullptr;   // pencil plan: A, B, passes 2-4
  FGeo fc{};                 // P1 / P5 geometry (dst: every slab's A)
  FGeo fp{};                 // P4 geometry (the pencil plan's, dst: every slab's nlx)
  SlabLayout L{};
};

struct pf_slab {
  pf_config cfg{};
  Geo g{};                   // the whole box (nspec: one slab's modes)
  int prec = 0, S = 1, first = 0, nloc = 1;  // slabs [first, first + nloc) live here
  std::vector<SlabBuf> sl;
  cudaStream_t st = nullptr;
  long long step = 0;
  bool peer = false;         // one slab per process: IPC peers + NCCL
  bool connected = false;
  ncclComm_t comm = nullptr;
  int* bar = nullptr;        // barrier word of the NCCL all-reduce
  std::vector<void*> opened; // IPC mappings of the peers' buffers
  cudaGraphExec_t gexec = nullptr;  // one recorded step of a noise-free group
  cudaStream_t gst = nullptr;       // its capture stream
  std::string err;
};

namespace pf {
namespace {

std::string g_slab_err;

int sfail(pf_slab* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  else g_slab_err = msg;
  return code;
}

#define PF_SCUDA(h, call)                                                              \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return sfail(h, PF_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define PF_SNCCL(h, call)                                                              \
  do {                                                                                 \
    ncclResult_t r_ = (call);                                                          \
    if (r_ != ncclSuccess)                                                             \
      return sfail(h, PF_ERR_CUDA, std::string(#call) + ": " + nccl().GetErrorString(r_)); \
  } while (0)

}  // namespace
}  // namespace pf

namespace pf {
namespace {

// The checks of pf_slab_create on top of pf_create's: what the slab
// schedule covers.
int slab_check(const pf_config* c, int S) {
  int rc = config_validate(c);
  if (rc) return rc;
  if (S < 1 || S > kMaxSlabs)
    return sfail(nullptr, PF_ERR_INVALID, "slabs must be 1.." + std::to_string(kMaxSlabs));
  if (c->dim != 3 || !c->is_nonlinear || c->dealias != PF_DEALIAS_TRUNCATE)
    return sfail(nullptr, PF_ERR_UNSUPPORTED,
                 "slab decomposition is built for the 3D nonlinear problem with the 2/3 rule");
  if (c->noise_mag != 0.0 &&
      (c->noise_type != PF_NOISE_THERMAL || c->noise_source != PF_NOISE_SRC_PHILOX))
    return sfail(nullptr, PF_ERR_UNSUPPORTED,
                 "slab decomposition draws thermal noise on the device (Philox) only");
  if (c->n[0] % S != 0 || c->n[1] % S != 0)
    return sfail(nullptr, PF_ERR_INVALID, "slabs must divide n0 and n1");
  if ((long long)(c->n[0] / S) * c->n[1] % 64 != 0)
    return sfail(nullptr, PF_ERR_UNSUPPORTED,
                 "(n0 / slabs) n1 must be a multiple of 64 (line groups of pass 3)");
  return PF_OK;
}

void free_slab(SlabBuf& b) {
  for (void* p : {b.uhat, b.u0, b.nl, b.nlx, (void*)b.dscal, (void*)b.maxbits, (void*)b.e2})
    if (p) cudaFree(p);
  if (b.pp) fused_destroy(b.pp);
  b = SlabBuf();
}

int alloc_slab(pf_slab* h, int r, SlabBuf& b) {
  const Geo& g = h->g;
  const size_t cb = h->prec == PF_FP64 ? 16 : 8;
  b.L = slab_layout(g.n[0], g.n[1], h->S, r);
  const long long ns = g.nspec;  // one slab's modes n0 n1s nh
  const long long npen = (long long)b.L.n0s * g.n[1] * g.nh;
  auto alloc = [&](void** p, size_t bytes) {
    return cudaMalloc(p, bytes) == cudaSuccess && cudaMemset(*p, 0, bytes) == cudaSuccess;
  };
  bool ok = alloc(&b.uhat, cb * 3 * ns) && alloc(&b.u0, cb * 3 * ns) &&
            alloc(&b.nl, cb * 3 * npen) && alloc(&b.nlx, cb * 3 * ns) &&
            alloc((void**)&b.dscal, sizeof(double) * kScalCount) &&
            alloc((void**)&b.maxbits, sizeof(unsigned long long)) &&
            alloc((void**)&b.e2, sizeof(double) * 2);
  if (ok && h->S > 1) {
    Geo gb = g;
    gb.nspec = (long long)g.n[0] * g.n[1] * g.nh;
    b.pp = fused_create_pencil(gb, h->prec, h->S);
    ok = b.pp != nullptr;
  } else if (ok) {
    Geo gb = g;
    b.pp = fused_create(gb, h->prec, 0, 1);
    ok = b.pp != nullptr;
  }
  if (!ok) {
    cudaGetLastError();
    return sfail(h, PF_ERR_NOMEM, "slab buffers or plan could not be created");
  }
  const double dt0 = h->cfg.dt;
  PF_SCUDA(h, cudaMemcpy(b.dscal + kScalDt, &dt0, sizeof(double), cudaMemcpyHostToDevice));
  // P1 / P5 geometry: the box's wavenumbers, the slab's state layout
  FGeo& fc = b.fc;
  fc = b.pp->f;
  fc.n0 = fc.t0 = g.n[0];
  fc.nspec = ns;
  fc.nlrow = b.L.n1s * g.nh;
  fc.nlcomp = ns;
  fc.nmem = 1;
  fc.ilv = 0;  // slab P1 numbers its fields by blockIdx.y
  // P4: the pencil plan's geometry
  b.fp = b.pp->f;
  for (FGeo* f : {&fc, &b.fp}) {
    f->sl_S = h->S;
    f->sl_n0 = b.L.n0s;
    f->sl_n1 = b.L.n1s;
    f->sl_x0 = b.L.x0;
    f->sl_i1 = b.L.i1;
    f->sl_c0 = b.L.c0;
    f->sl_nc = b.L.nc;
    f->sl_N0 = g.n[0];
  }
  return PF_OK;
}

// Destination tables: P1 stores into every slab's A, P4 into every slab's nlx.
void set_dst(SlabBuf& b, const std::vector<void*>& A, const std::vector<void*>& nlx) {
  for (int s = 0; s < kMaxSlabs; ++s) {
    b.fc.sl_dst[s] = s < (int)A.size() ? A[s] : nullptr;
    b.fp.sl_dst[s] = s < (int)nlx.size() ? nlx[s] : nullptr;
  }
}

int make_handle(const pf_config* cfg, int S, int first, int nloc, bool peer, pf_slab** out) {
  if (!cfg || !out) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_create: null argument");
  *out = nullptr;
  int rc = slab_check(cfg, S);
  if (rc) return rc;
  cudaError_t ce = ensure_tables();
  if (ce != cudaSuccess)
    return sfail(nullptr, PF_ERR_CUDA, std::string("twiddle tables: ") + cudaGetErrorString(ce));
  pf_slab* h = new pf_slab();
  h->cfg = *cfg;
  h->prec = cfg->precision;
  h->S = S;
  h->first = first;
  h->nloc = nloc;
  h->peer = peer;
  h->g = config_geo(cfg);
  h->g.nspec = (long long)cfg->n[0] * (cfg->n[1] / S) * h->g.nh;
  h->sl.resize(nloc);
  for (int i = 0; i < nloc; ++i) {
    rc = alloc_slab(h, first + i, h->sl[i]);
    if (rc) {
      std::string m = h->err;
      pf_slab_destroy(h);
      return sfail(nullptr, rc, m);
    }
  }
  if (!peer) {
    std::vector<void*> A, nlx;
    for (auto& b : h->sl) {
      A.push_back(b.pp->A);
      nlx.push_back(b.nlx);
    }
    for (auto& b : h->sl) set_dst(b, A, nlx);
    h->connected = true;
  }
  *out = h;
  return PF_OK;
}

// The exchange barrier between a pass that stores into other slabs and the
// pass that reads them.
int barrier(pf_slab* h) {
  if (!h->peer) return PF_OK;  // one stream orders the group's launches
  PF_SNCCL(h, nccl().AllReduce(h->bar, h->bar, 1, ncclInt32, ncclSum, h->comm, h->st));
  return PF_OK;
}

// CFL maximum and band energy over the slabs.
int reduce_scalars(pf_slab* h, bool do_max, bool do_band) {
  if (!do_max && !do_band) return PF_OK;
  if (h->peer) {
    SlabBuf& b = h->sl[0];
    if (do_max)
      PF_SNCCL(h, nccl().AllReduce(b.maxbits, b.maxbits, 1, ncclUint64, ncclMax, h->comm, h->st));
    if (do_band)
      PF_SNCCL(h, nccl().AllReduce(b.dscal + kScalBandE, b.dscal + kScalBandE, 1, ncclFloat64,
                                   ncclSum, h->comm, h->st));
    return PF_OK;
  }
  GroupScalars gs;
  memset(&gs, 0, sizeof(gs));
  for (int i = 0; i < h->nloc; ++i) {
    gs.maxbits[i] = h->sl[i].maxbits;
    gs.dscal[i] = h->sl[i].dscal;
  }
  k_group_reduce<<<1, 32, 0, h->st>>>(gs, h->nloc, do_max ? 1 : 0, do_band ? 1 : 0);
  PF_SCUDA(h, launched());
  return PF_OK;
}

template <typename R> int band_energy(pf_slab* h, SlabBuf& b) {
  const Geo& g = h->g;
  const double kf2 = h->cfg.forcing_kf * h->cfg.forcing_kf, kf = h->cfg.forcing_kf;
  const int K0 = (int)std::floor(kf / g.kscale[0] + 1e-9);
  const int K2 = (int)std::floor(kf / g.kscale[2] + 1e-9);
  const int cnt0 = 2 * K0 + 1 >= g.n[0] ? g.n[0] : 2 * K0 + 1;
  const int cnt2 = K2 + 1 >= g.nh ? g.nh : K2 + 1;
  PF_SCUDA(h, cudaMemsetAsync(b.dscal + kScalBandE, 0, 2 * sizeof(double), h->st));
  const long long total = (long long)cnt0 * b.L.n1s * cnt2;
  const unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 1024);
  k_slab_band_energy<R><<<blocks, 256, 0, h->st>>>((const cx<R>*)b.uhat, g, b.L.n1s, b.L.i1, kf2,
                                                   cnt0, K0, cnt2, b.dscal);
  PF_SCUDA(h, launched());
  return PF_OK;
}

template <typename R> int pass_chk(pf_slab* h, cudaError_t e, const char* what) {
  if (e != cudaSuccess) return sfail(h, PF_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return PF_OK;
}

// One time step of every slab held here (simulation.py:205-217 per step).
template <typename R> int slab_step(pf_slab* h) {
  const Scheme sc = scheme_for(h->cfg.integrator);
  const bool cfl = h->cfg.cfl > 0.0;
  const bool forcing = h->cfg.forcing_eps > 0.0;
  const bool noise = h->cfg.noise_mag != 0.0;
  int rc;
  for (int s = 0; s < sc.nstages; ++s) {
    const bool want_max = s == 0 && cfl;
    for (auto& b : h->sl) {
      if (want_max) PF_SCUDA(h, cudaMemsetAsync(b.maxbits, 0, sizeof(unsigned long long), h->st));
      if ((rc = pass_chk<R>(h, slab_p1<R>(b.fc, b.uhat, h->st), "slab pass 1"))) return rc;
    }
    if ((rc = barrier(h))) return rc;
    for (auto& b : h->sl) {
      for (int p = 2; p <= 3; ++p)
        if ((rc = pass_chk<R>(h, fused_pass(b.pp, p, nullptr, b.nl, (want_max && p == 3) ? b.maxbits : nullptr, h->st),
                              "slab pass 2/3")))
          return rc;
      if ((rc = pass_chk<R>(h, slab_p4<R>(b.fp, b.nl, h->st), "slab pass 4"))) return rc;
    }
    if ((rc = barrier(h))) return rc;
    if (forcing)
      for (auto& b : h->sl)
        if ((rc = band_energy<R>(h, b))) return rc;
    if ((rc = reduce_scalars(h, want_max, forcing))) return rc;
    if (want_max)
      for (auto& b : h->sl) PF_SCUDA(h, launch_set_dt(b.dscal, b.maxbits, h->cfg.cfl, h->st));
    for (auto& b : h->sl) {
      UpdateArgs<R> A;
      memset(&A, 0, sizeof(A));
      A.uhat = (cx<R>*)b.uhat;
      A.u0 = (cx<R>*)b.u0;
      A.nl = (const cx<R>*)b.nlx;
      A.dscal = b.dscal;
      A.g = h->g;
      A.coef = sc.st[s];
      A.nu = h->cfg.viscosity;
      A.noise_mag = h->cfg.noise_mag;
      A.noise_norm = 1.0 / std::sqrt((double)h->g.nphys) / std::sqrt(2.0 - 2.0 / 3.0);
      A.f_eps = h->cfg.forcing_eps;
      A.f_kf2 = h->cfg.forcing_kf * h->cfg.forcing_kf;
      A.seed = h->cfg.seed;
      A.step = (uint64_t)(h->step + 1);
      A.noise_src = noise ? kNoisePhilox : kNoiseNone;
      A.noise_type = h->cfg.noise_type;
      A.save_u0 = s == 0;
      A.nyq_mask = h->cfg.mask_nyquist;
      A.forcing = forcing;
      A.mstride = 3 * h->g.nspec;
      if ((rc = pass_chk<R>(h, slab_p5<R>(b.fc, A, b.nlx, h->st), "slab pass 5"))) return rc;
    }
  }
  if (!cfl)
    for (auto& b : h->sl) PF_SCUDA(h, launch_advance_time(b.dscal, 1, h->st));
  ++h->step;
  return PF_OK;
}

int check_err_words(pf_slab* h) {
  for (auto& b : h->sl) {
    const int v = fused_device_error(b.pp);
    if (v != 0)
      return sfail(h, PF_ERR_CUDA, "a bounded device wait gave up (code " + std::to_string(v) +
                                       "): results of the step are invalid");
  }
  return PF_OK;
}

// FP64 <-> state precision (FP32 states)
__global__ void k_slab_from64(float* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}
__global__ void k_slab_to64(double* __restrict__ dst, const float* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}
unsigned conv_blocks(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 4096); }

// Record one step of the group as a graph (captured on a private stream).
int record_step(pf_slab* h) {
  if (!h->gst) PF_SCUDA(h, cudaStreamCreateWithFlags(&h->gst, cudaStreamNonBlocking));
  cudaStream_t user = h->st;
  const long long step0 = h->step;
  h->st = h->gst;
  cudaError_t e = cudaStreamBeginCapture(h->gst, cudaStreamCaptureModeThreadLocal);
  int rc = PF_OK;
  if (e == cudaSuccess) {
    rc = h->prec == PF_FP64 ? slab_step<double>(h) : slab_step<float>(h);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(h->gst, &graph);
    if (rc == PF_OK && ee == cudaSuccess)
      e = cudaGraphInstantiate(&h->gexec, graph, 0);
    else if (ee != cudaSuccess)
      e = ee;
    if (graph) cudaGraphDestroy(graph);
  }
  h->st = user;
  h->step = step0;
  if (rc) return rc;
  PF_SCUDA(h, e);
  // the capture stream's launches are ordered after the caller's work by the
  // replays on the caller's stream
  return PF_OK;
}

SlabBuf* local(pf_slab* h, int slab) {
  if (!h || slab < h->first || slab >= h->first + h->nloc) return nullptr;
  return &h->sl[slab - h->first];
}

}  // namespace
}  // namespace pf

extern "C" {

int pf_slab_layout(int n0, int n1, int slabs, int slab, int* out6) {
  if (!out6 || slabs < 1 || slabs > kMaxSlabs || slab < 0 || slab >= slabs || n0 % slabs ||
      n1 % slabs || n0 < 1 || n1 < 1)
    return sfail(nullptr, PF_ERR_INVALID, "pf_slab_layout: bad argument");
  const SlabLayout L = slab_layout(n0, n1, slabs, slab);
  const int v[6] = {L.n0s, L.n1s, L.x0, L.i1, L.c0, L.nc};
  memcpy(out6, v, sizeof(v));
  return PF_OK;
}

int pf_slab_create_group(const pf_config* cfg, int slabs, pf_slab** out) {
  return make_handle(cfg, slabs, 0, slabs, false, out);
}

int pf_slab_create(const pf_config* cfg, int slabs, int slab, pf_slab** out) {
  if (slab < 0 || slab >= slabs) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_create: bad slab");
  return make_handle(cfg, slabs, slab, 1, true, out);
}

int pf_slab_export(const pf_slab* h, void* out, size_t cap, size_t* used) {
  const size_t need = 2 * sizeof(cudaIpcMemHandle_t);
  if (used) *used = need;
  if (!h || !out) return sfail(const_cast<pf_slab*>(h), PF_ERR_INVALID, "pf_slab_export: null argument");
  if (!h->peer) return sfail(const_cast<pf_slab*>(h), PF_ERR_INVALID, "pf_slab_export: a group needs no export");
  if (cap < need) return sfail(const_cast<pf_slab*>(h), PF_ERR_INVALID, "pf_slab_export: buffer too small");
  pf_slab* m = const_cast<pf_slab*>(h);
  cudaIpcMemHandle_t ha, hn;
  PF_SCUDA(m, cudaIpcGetMemHandle(&ha, h->sl[0].pp->A));
  PF_SCUDA(m, cudaIpcGetMemHandle(&hn, h->sl[0].nlx));
  memcpy(out, &ha, sizeof(ha));
  memcpy((char*)out + sizeof(ha), &hn, sizeof(hn));
  return PF_OK;
}

int pf_slab_nccl_id(void* out, size_t cap) {
  if (!out || cap < sizeof(ncclUniqueId))
    return sfail(nullptr, PF_ERR_INVALID, "pf_slab_nccl_id: buffer of 128 bytes needed");
  const Nccl& n = nccl();
  if (!n.ok) return sfail(nullptr, PF_ERR_UNSUPPORTED, n.why);
  ncclUniqueId id;
  const ncclResult_t r = n.GetUniqueId(&id);
  if (r != ncclSuccess) return sfail(nullptr, PF_ERR_CUDA, std::string("ncclGetUniqueId: ") + n.GetErrorString(r));
  memcpy(out, &id, sizeof(id));
  return PF_OK;
}

int pf_slab_connect(pf_slab* h, const void* exports, const void* nccl_id) {
  if (!h || !exports || !nccl_id) return sfail(h, PF_ERR_INVALID, "pf_slab_connect: null argument");
  if (!h->peer || h->connected) return sfail(h, PF_ERR_INVALID, "pf_slab_connect: not a lone unconnected slab");
  const Nccl& n = nccl();
  if (!n.ok) return sfail(h, PF_ERR_UNSUPPORTED, n.why);
  const size_t one = 2 * sizeof(cudaIpcMemHandle_t);
  std::vector<void*> A(h->S), nlx(h->S);
  for (int s = 0; s < h->S; ++s) {
    if (s == h->first) {
      A[s] = h->sl[0].pp->A;
      nlx[s] = h->sl[0].nlx;
      continue;
    }
    cudaIpcMemHandle_t ha, hn;
    memcpy(&ha, (const char*)exports + s * one, sizeof(ha));
    memcpy(&hn, (const char*)exports + s * one + sizeof(ha), sizeof(hn));
    PF_SCUDA(h, cudaIpcOpenMemHandle(&A[s], ha, cudaIpcMemLazyEnablePeerAccess));
    h->opened.push_back(A[s]);
    PF_SCUDA(h, cudaIpcOpenMemHandle(&nlx[s], hn, cudaIpcMemLazyEnablePeerAccess));
    h->opened.push_back(nlx[s]);
  }
  set_dst(h->sl[0], A, nlx);
  PF_SCUDA(h, cudaMalloc(&h->bar, sizeof(int)));
  PF_SCUDA(h, cudaMemset(h->bar, 0, sizeof(int)));
  ncclUniqueId id;
  memcpy(&id, nccl_id, sizeof(id));
  PF_SNCCL(h, n.CommInitRank(&h->comm, h->S, id, h->first));
  h->connected = true;
  return PF_OK;
}

int pf_slab_destroy(pf_slab* h) {
  if (!h) return PF_OK;
  cudaDeviceSynchronize();
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->gst) cudaStreamDestroy(h->gst);
  if (h->comm) nccl().CommDestroy(h->comm);
  for (void* p : h->opened) cudaIpcCloseMemHandle(p);
  if (h->bar) cudaFree(h->bar);
  for (auto& b : h->sl) free_slab(b);
  delete h;
  return PF_OK;
}

const char* pf_slab_last_error(const pf_slab* h) { return h ? h->err.c_str() : g_slab_err.c_str(); }

int pf_slab_set_stream(pf_slab* h, void* stream) {
  if (!h) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_set_stream: null handle");
  h->st = (cudaStream_t)stream;
  return PF_OK;
}

int pf_slab_sizes(const pf_slab* h, int* first, int* count, long long* nspec) {
  if (!h) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_sizes: null handle");
  if (first) *first = h->first;
  if (count) *count = h->nloc;
  if (nspec) *nspec = h->g.nspec;
  return PF_OK;
}

// u_hat of slab `slab` ([3][n0][n1/S][nh] complex128) from / to the host
// (where = 0) or the device (1).
int pf_slab_set_fourier(pf_slab* h, int slab, const double* u_hat, int where) {
  SlabBuf* b = local(h, slab);
  if (!b || !u_hat) return sfail(h, PF_ERR_INVALID, "pf_slab_set_fourier: slab not held here or null data");
  const size_t n = 2 * 3 * (size_t)h->g.nspec;
  double* tmp = nullptr;
  PF_SCUDA(h, cudaMalloc(&tmp, sizeof(double) * n));
  cudaError_t e = cudaMemcpyAsync(tmp, u_hat, sizeof(double) * n,
                                  where ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->st);
  if (e == cudaSuccess) {
    if (h->prec == PF_FP64) {
      e = cudaMemcpyAsync(b->uhat, tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st);
    } else {
      k_slab_from64<<<conv_blocks(n), 256, 0, h->st>>>((float*)b->uhat, tmp, (long long)n);
      e = launched();
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  PF_SCUDA(h, e);
  return PF_OK;
}

int pf_slab_get_fourier(pf_slab* h, int slab, double* u_hat, int where) {
  SlabBuf* b = local(h, slab);
  if (!b || !u_hat) return sfail(h, PF_ERR_INVALID, "pf_slab_get_fourier: slab not held here or null data");
  const size_t n = 2 * 3 * (size_t)h->g.nspec;
  double* tmp = nullptr;
  PF_SCUDA(h, cudaMalloc(&tmp, sizeof(double) * n));
  cudaError_t e;
  if (h->prec == PF_FP64) {
    e = cudaMemcpyAsync(tmp, b->uhat, sizeof(double) * n, cudaMemcpyDeviceToDevice, h->st);
  } else {
    k_slab_to64<<<conv_blocks(n), 256, 0, h->st>>>(tmp, (const float*)b->uhat, (long long)n);
    e = launched();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(u_hat, tmp, sizeof(double) * n,
                        where ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
  cudaFree(tmp);
  PF_SCUDA(h, e);
  return check_err_words(h);
}

int pf_slab_step(pf_slab* h, int nsteps) {
  if (!h) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_step: null handle");
  if (!h->connected) return sfail(h, PF_ERR_INVALID, "pf_slab_step: connect the slab first");
  // A noise-free group replays one recorded step (the step index only feeds
  // the noise draws); the per-process form launches plainly.
  if (!h->peer && nsteps >= 2 && h->cfg.noise_mag == 0.0) {
    if (!h->gexec) {
      int rc = record_step(h);
      if (rc) return rc;
    }
    for (int i = 0; i < nsteps; ++i) {
      PF_SCUDA(h, cudaGraphLaunch(h->gexec, h->st));
      ++h->step;
    }
    return PF_OK;
  }
  for (int i = 0; i < nsteps; ++i) {
    const int rc = h->prec == PF_FP64 ? slab_step<double>(h) : slab_step<float>(h);
    if (rc) return rc;
  }
  return PF_OK;
}

int pf_slab_sync(pf_slab* h) {
  if (!h) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_sync: null handle");
  PF_SCUDA(h, cudaStreamSynchronize(h->st));
  return check_err_words(h);
}

int pf_slab_get_time(pf_slab* h, double* t, long long* step, double* dt) {
  if (!h) return sfail(nullptr, PF_ERR_INVALID, "pf_slab_get_time: null handle");
  double ds[kScalCount];
  PF_SCUDA(h, cudaMemcpyAsync(ds, h->sl[0].dscal, sizeof(ds), cudaMemcpyDeviceToHost, h->st));
  PF_SCUDA(h, cudaStreamSynchronize(h->st));
  if (t) *t = ds[kScalTime];
  if (dt) *dt = ds[kScalDt];
  if (step) *step = h->step;
  return PF_OK;
}

// This slab's part of E = 1/2 sum w |u|^2 and Z = 1/2 sum w |k|^2 |u|^2
// (the box's sums are the sums over the slabs).
int pf_slab_energy(pf_slab* h, int slab, double* energy, double* enstrophy) {
  SlabBuf* b = local(h, slab);
  if (!b) return sfail(h, PF_ERR_INVALID, "pf_slab_energy: slab not held here");
  PF_SCUDA(h, cudaMemsetAsync(b->e2, 0, 2 * sizeof(double), h->st));
  const unsigned blocks = (unsigned)std::min<long long>((h->g.nspec + 255) / 256, 1024);
  if (h->prec == PF_FP64)
    k_slab_energy<double><<<blocks, 256, 0, h->st>>>((const cx<double>*)b->uhat, h->g, b->L.n1s,
                                                     b->L.i1, b->e2);
  else
    k_slab_energy<float><<<blocks, 256, 0, h->st>>>((const cx<float>*)b->uhat, h->g, b->L.n1s,
                                                    b->L.i1, b->e2);
  PF_SCUDA(h, launched());
  double e2[2];
  PF_SCUDA(h, cudaMemcpyAsync(e2, b->e2, sizeof(e2), cudaMemcpyDeviceToHost, h->st));
  PF_SCUDA(h, cudaStreamSynchronize(h->st));
  if (energy) *energy = e2[0];
  if (enstrophy) *enstrophy = e2[1];
  return PF_OK;
}

}  // extern "C"
