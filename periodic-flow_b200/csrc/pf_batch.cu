// Ensembles: many independent linear (fluctuating Stokes) boxes of mixed
// sizes and dimensions advanced together, one kernel launch for all members
// and all steps, optionally replayed from a CUDA graph.
//
// Every mode of a linear box evolves on its own (the operator is diagonal in
// k), so one thread owns one mode of one member for the whole launch and keeps
// its state in registers across stages and steps, drawing its Philox noise in
// registers.  Members' mode ranges are padded to whole CTAs, so a CTA serves a
// single member and looks its descriptor up once.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/periodicflow_b200.h"
#include "pf_kernels.h"
#include "pf_update.cuh"

namespace pf {

constexpr int kBatchBlock = 256;

struct BatchItem {
  Geo g;
  void* uhat;
  const void* lop;
  const void* corr;
  double* dscal;
  double nu, noise_mag, noise_norm, dt;
  uint64_t seed;
  long long block_begin;  // first CTA of this member
  int noise_src;
  int pad;
};

template <typename R, int D, int NC>
PF_D void batch_mode(const BatchItem& it, long long m, uint64_t step0, int nsteps,
                     const Scheme& sc, int noise_type) {
  using C = cx<R>;
  const Geo& g = it.g;
  cx<R>* uh = (cx<R>*)it.uhat;
  const ModeK<R, D> mk_ = mode_k<R, D>(g, m);
  C u[D];
#pragma unroll
  for (int a = 0; a < D; ++a) u[a] = uh[a * g.nspec + m];
  const R L = it.lop ? ((const R*)it.lop)[m] : (R)(-it.nu) * mk_.k2;
  const R corr = it.corr ? ((const R*)it.corr)[m] : R(0);
  const DrawSite site = draw_site(g, mk_.ix.i0, mk_.ix.i1, mk_.ix.i2);
  const R nf = mk_.k2 == R(0) ? R(0) : (R)it.noise_norm;
  const R dt = (R)it.dt, sqdt = (R)sqrt(it.dt);
  // zero noise amplitude at this mode: xi = 0, no draws needed (counter-based)
  const bool philox = it.noise_src == kNoisePhilox && nf != R(0) &&
                      (noise_type == kThermal || corr != R(0));
  // the implicit predictor is dead work without a nonlinear term
  const int first = sc.st[0].implicit ? 1 : 0;
  for (int s = 0; s < nsteps; ++s) {
    const uint64_t step = step0 + (uint64_t)s;
    C w1[NC], w2[NC];
    if (philox) {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        w1[c] = cscale(draw_value<R>(site, c, it.seed, step), nf);
        w2[c] = cscale(draw_value<R>(site, NC + c, it.seed, step), nf);
      }
    }
    C u0[D];
#pragma unroll
    for (int a = 0; a < D; ++a) u0[a] = u[a];
    for (int st = first; st < sc.nstages; ++st) {
      const StageCoef& cf = sc.st[st];
      C xi[D];
      if (philox) {
        noise_term<R, D, NC>(xi, w1, w2, (R)cf.a, noise_type, mk_.k, mk_.k2, corr,
                             (R)it.noise_mag);
      } else {
#pragma unroll
        for (int a = 0; a < D; ++a) xi[a] = czero<C>();
      }
#pragma unroll
      for (int a = 0; a < D; ++a)
        u[a] = stage_update<R>(cf, dt, sqdt, L, u0[a], u[a], czero<C>(), xi[a]);
    }
  }
#pragma unroll
  for (int a = 0; a < D; ++a) uh[a * g.nspec + m] = u[a];
}

// NT: noise type of the whole batch (thermal: NC = D*D, correlated: NC = D)
template <typename R, int NT>
__global__ void __launch_bounds__(kBatchBlock)
k_stokes_batch(const BatchItem* __restrict__ items, int count,
               const unsigned long long* __restrict__ steps, Scheme sc, int nsteps) {
  __shared__ int s_item;
  if (threadIdx.x == 0) {
    // last member whose first CTA is <= this CTA
    int lo = 0, hi = count - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (items[mid].block_begin <= (long long)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_item = lo;
  }
  __syncthreads();
  const int i = s_item;
  const BatchItem it = items[i];
  const long long m = ((long long)blockIdx.x - it.block_begin) * kBatchBlock + threadIdx.x;
  if (m >= it.g.nspec) return;
  const uint64_t step0 = steps[i] + 1;
  if (it.g.dim == 3) {
    if (NT == kThermal) batch_mode<R, 3, 9>(it, m, step0, nsteps, sc, NT);
    else batch_mode<R, 3, 3>(it, m, step0, nsteps, sc, NT);
  } else {
    if (NT == kThermal) batch_mode<R, 2, 4>(it, m, step0, nsteps, sc, NT);
    else batch_mode<R, 2, 2>(it, m, step0, nsteps, sc, NT);
  }
}

// per member: step counter += nsteps, t += dt nsteps times (as the reference
// accumulates t step by step)
__global__ void k_batch_advance(const BatchItem* __restrict__ items, int count,
                                unsigned long long* __restrict__ steps, int nsteps) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    steps[i] += (unsigned long long)nsteps;
    double t = items[i].dscal[kScalTime];
    const double dt = items[i].dt;
    for (int s = 0; s < nsteps; ++s) t += dt;
    items[i].dscal[kScalTime] = t;
  }
}

}  // namespace pf

using namespace pf;

struct pf_batch {
  std::vector<pf_solver*> members;
  std::vector<BatchItem> host_items;
  BatchItem* items = nullptr;
  unsigned long long* steps = nullptr;
  long long blocks = 0;
  int prec = 0, noise_type = 0;
  Scheme scheme;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_steps = 0;
  std::string err;
};

static int bfail(pf_batch* b, int code, const std::string& m) {
  if (b) b->err = m;
  return set_static_error(code, m);
}

static cudaError_t batch_launch(pf_batch* b, int nsteps) {
  const unsigned grid = (unsigned)b->blocks;
  const int n = (int)b->members.size();
  if (b->prec == PF_FP64) {
    if (b->noise_type == kThermal)
      k_stokes_batch<double, kThermal><<<grid, kBatchBlock, 0, b->st>>>(b->items, n, b->steps, b->scheme, nsteps);
    else
      k_stokes_batch<double, kCorrelated><<<grid, kBatchBlock, 0, b->st>>>(b->items, n, b->steps, b->scheme, nsteps);
  } else {
    if (b->noise_type == kThermal)
      k_stokes_batch<float, kThermal><<<grid, kBatchBlock, 0, b->st>>>(b->items, n, b->steps, b->scheme, nsteps);
    else
      k_stokes_batch<float, kCorrelated><<<grid, kBatchBlock, 0, b->st>>>(b->items, n, b->steps, b->scheme, nsteps);
  }
  cudaError_t e = launched();
  if (e != cudaSuccess) return e;
  k_batch_advance<<<(n + 127) / 128, 128, 0, b->st>>>(b->items, n, b->steps, nsteps);
  return launched();
}

extern "C" {

int pf_batch_create(pf_solver* const* members, int count, pf_batch** out) {
  if (!members || count <= 0 || !out) return bfail(nullptr, PF_ERR_INVALID, "pf_batch_create: no members");
  *out = nullptr;
  pf_batch* b = new pf_batch();
  long long blocks = 0;
  for (int i = 0; i < count; ++i) {
    if (!members[i]) { delete b; return bfail(nullptr, PF_ERR_INVALID, "pf_batch_create: null member"); }
    const SolverView v = solver_view(members[i]);
    if (!v.linear_only) {
      delete b;
      return bfail(nullptr, PF_ERR_UNSUPPORTED,
                   "pf_batch_create: members must be linear (is_nonlinear=0, no forcing, fixed dt)");
    }
    if (v.noise_src == 2) {
      delete b;
      return bfail(nullptr, PF_ERR_UNSUPPORTED, "pf_batch_create: injected noise is per solver only");
    }
    if (i == 0) {
      b->prec = v.prec;
      b->noise_type = v.noise_type;
      b->scheme = scheme_for(v.integrator);
    } else if (v.prec != b->prec || v.noise_type != b->noise_type ||
               v.integrator != solver_view(members[0]).integrator) {
      delete b;
      return bfail(nullptr, PF_ERR_INVALID,
                   "pf_batch_create: members must share precision, noise type and integrator");
    }
    BatchItem it;
    memset(&it, 0, sizeof(it));
    it.g = v.g;
    it.uhat = v.uhat;
    it.lop = v.lop;
    it.corr = v.corr;
    it.dscal = v.dscal;
    it.nu = v.nu;
    it.noise_mag = v.noise_mag;
    it.noise_norm = v.noise_norm;
    it.dt = v.dt;
    it.seed = v.seed;
    it.noise_src = v.noise_src;
    it.block_begin = blocks;
    blocks += (v.g.nspec + kBatchBlock - 1) / kBatchBlock;
    b->host_items.push_back(it);
    b->members.push_back(members[i]);
  }
  b->blocks = blocks;
  if (blocks > 0x7fffffffLL) { delete b; return bfail(nullptr, PF_ERR_INVALID, "pf_batch_create: too many modes"); }
  std::vector<unsigned long long> st(count);
  for (int i = 0; i < count; ++i) st[i] = (unsigned long long)solver_view(members[i]).step;
  if (cudaMalloc(&b->items, sizeof(BatchItem) * count) != cudaSuccess ||
      cudaMalloc(&b->steps, sizeof(unsigned long long) * count) != cudaSuccess ||
      cudaMemcpy(b->items, b->host_items.data(), sizeof(BatchItem) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->steps, st.data(), sizeof(unsigned long long) * count, cudaMemcpyHostToDevice) != cudaSuccess) {
    std::string m = std::string("pf_batch_create: ") + cudaGetErrorString(cudaGetLastError());
    pf_batch_destroy(b);
    return bfail(nullptr, PF_ERR_NOMEM, m);
  }
  *out = b;
  return PF_OK;
}

int pf_batch_destroy(pf_batch* b) {
  if (!b) return PF_OK;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->items) cudaFree(b->items);
  if (b->steps) cudaFree(b->steps);
  delete b;
  return PF_OK;
}

int pf_batch_set_stream(pf_batch* b, void* stream) {
  if (!b) return bfail(nullptr, PF_ERR_INVALID, "null batch");
  b->st = (cudaStream_t)stream;
  return PF_OK;
}

const char* pf_batch_last_error(const pf_batch* b) { return b ? b->err.c_str() : ""; }

int pf_batch_step(pf_batch* b, int nsteps) {
  if (!b) return bfail(nullptr, PF_ERR_INVALID, "null batch");
  if (nsteps < 0) return bfail(b, PF_ERR_INVALID, "nsteps must be >= 0");
  if (nsteps == 0) return PF_OK;
  // members may have been stepped on their own since: refresh the counters
  std::vector<unsigned long long> st(b->members.size());
  for (size_t i = 0; i < st.size(); ++i) st[i] = (unsigned long long)solver_view(b->members[i]).step;
  cudaError_t e = cudaMemcpyAsync(b->steps, st.data(), sizeof(unsigned long long) * st.size(),
                                  cudaMemcpyHostToDevice, b->st);
  if (e == cudaSuccess) e = batch_launch(b, nsteps);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) return bfail(b, PF_ERR_CUDA, std::string("pf_batch_step: ") + cudaGetErrorString(e));
  for (pf_solver* m : b->members) solver_add_steps(m, nsteps);
  return PF_OK;
}

int pf_batch_capture(pf_batch* b, int nsteps) {
  if (!b) return bfail(nullptr, PF_ERR_INVALID, "null batch");
  if (nsteps <= 0) return bfail(b, PF_ERR_INVALID, "nsteps must be > 0");
  if (!b->st) return bfail(b, PF_ERR_INVALID, "pf_batch_capture: set a non-default stream first");
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  // the counters the graph starts from
  std::vector<unsigned long long> st(b->members.size());
  for (size_t i = 0; i < st.size(); ++i) st[i] = (unsigned long long)solver_view(b->members[i]).step;
  cudaError_t e = cudaMemcpy(b->steps, st.data(), sizeof(unsigned long long) * st.size(),
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t le = batch_launch(b, nsteps);
    e = cudaStreamEndCapture(b->st, &b->graph);
    if (le != cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) return bfail(b, PF_ERR_CUDA, std::string("pf_batch_capture: ") + cudaGetErrorString(e));
  b->graph_steps = nsteps;
  return PF_OK;
}

int pf_batch_replay(pf_batch* b) {
  if (!b || !b->exec) return bfail(b, PF_ERR_INVALID, "pf_batch_replay: nothing captured");
  cudaError_t e = cudaGraphLaunch(b->exec, b->st);
  if (e != cudaSuccess) return bfail(b, PF_ERR_CUDA, std::string("pf_batch_replay: ") + cudaGetErrorString(e));
  count_launch();
  count_launch();
  for (pf_solver* m : b->members) solver_add_steps(m, b->graph_steps);
  return PF_OK;
}

int pf_batch_sync(pf_batch* b) {
  if (!b) return bfail(nullptr, PF_ERR_INVALID, "null batch");
  cudaError_t e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) return bfail(b, PF_ERR_CUDA, std::string("pf_batch_sync: ") + cudaGetErrorString(e));
  return PF_OK;
}

}  // extern "C"
