// Plans of the fused pencil passes of the 3D nonlinear term (buffers, launch
// variants, autotuner) and the dispatch to the instantiation units; the
// kernels and their launch templates are in pf_fused_impl.cuh.
#include "pf_fused_impl.cuh"

namespace pf {

static bool pow2(int n) { return n >= 16 && (n & (n - 1)) == 0; }
// 3 * 2^b with 48 <= n
static bool three_pow2(int n) {
  const int m = n / 3;
  return n % 3 == 0 && n >= 48 && (m & (m - 1)) == 0;
}

// Launch variants picked by fused_autotune, per geometry (precision, rule,
// sides); a later plan of the same geometry starts from them.
using TuneKey = std::tuple<int, int, int, int, int>;
static std::mutex g_tune_mu;
static std::map<TuneKey, std::array<int, 12>> g_tuned;
static TuneKey tune_key(const FusedPlan* p) {
  return TuneKey(p->prec, p->pad ? 1 : 0, p->f.n0, p->f.n1, p->f.n2);
}

static FusedPlan* fused_create_2d(const Geo& g, int precision, int nmem) {
  if (!fused2d_side(g.n[0]) || !fused2d_side(g.n[1])) return nullptr;
  FusedPlan* p = new FusedPlan();
  p->g = g;
  p->prec = precision;
  p->dim = 2;
  p->f2 = fused2d_geo(g);
  p->f2.nmem = nmem;
  p->cap = nmem;
  const size_t cb = precision == 0 ? 8 : 16;
  if (cudaMalloc(&p->A, cb * nmem * fused2d_scratch_elems(p->f2)) != cudaSuccess ||
      cudaMalloc(&p->err, sizeof(int)) != cudaSuccess ||
      cudaMemset(p->err, 0, sizeof(int)) != cudaSuccess) {
    fused_destroy(p);
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

// slabs > 1: the pencil plan of one slab of the box (passes 2-4 on its
// n0 / slabs planes; pf_slab.cu)
static FusedPlan* create3d(const Geo& g, int precision, int dealias, int nmem, int slabs) {
  if (g.dim != 3) return nullptr;
  const bool pad = dealias == 1;
  // FP32 2/3 rule: sides 2^b 16..512 (the last up to 256) and 3 * 2^b
  // 48..384; 3/2 rule (FP32, FP64) and FP64 2/3 rule: sides 2^b 16..256
  // (3/2 transform lengths 24..384)
  const bool t32 = precision == 0 && !pad;
  for (int a = 0; a < 3; ++a) {
    const bool ok = (pow2(g.n[a]) && g.n[a] <= ((pad || precision == 1) ? 256 : 512)) ||
                    (t32 && three_pow2(g.n[a]) && g.n[a] <= 384);
    if (!ok) return nullptr;
  }
  if (g.n[2] > (t32 && three_pow2(g.n[2]) ? 384 : 256)) return nullptr;
  FusedPlan* p = new FusedPlan();
  p->g = g;
  p->prec = precision;
  p->pad = pad;
  FGeo& f = p->f;
  f.n0 = g.n[0]; f.n1 = g.n[1]; f.n2 = g.n[2]; f.nh = g.nh;
  f.kmax0 = g.kmax[0]; f.kmax1 = g.kmax[1]; f.kmax2 = g.kmax[2];
  if (pad) {
    f.t0 = 3 * f.n0 / 2; f.t1 = 3 * f.n1 / 2; f.t2 = 3 * f.n2 / 2;
    f.c1 = f.n1;  // every N-grid k1 and k2 feeds the padded grid
    f.c2 = f.nh;
  } else {
    f.t0 = f.n0; f.t1 = f.n1; f.t2 = f.n2;
    f.c1 = 2 * f.kmax1 + 1;
    f.c2 = f.kmax2 + 1;
  }
  f.nlrow = f.t1 * f.nh;
  f.nlcomp = (long long)f.t0 * f.t1 * f.nh;
  f.ks0 = g.kscale[0]; f.ks1 = g.kscale[1]; f.ks2 = g.kscale[2];
  f.cflw0 = g.n[0] * g.kscale[0] / (2.0 * M_PI);
  f.cflw1 = g.n[1] * g.kscale[1] / (2.0 * M_PI);
  f.cflw2 = g.n[2] * g.kscale[2] / (2.0 * M_PI);
  f.nspec = g.nspec;
  if (slabs > 1) {
    if (pad || nmem != 1 || f.n0 % slabs != 0) {
      delete p;
      return nullptr;
    }
    p->slabs = slabs;
    f.n0 = f.t0 = f.n0 / slabs;
    f.nlcomp = (long long)f.t0 * f.t1 * f.nh;
    f.nspec = f.nlcomp;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find(tune_key(p));
    if (it != g_tuned.end()) {
      for (int i = 0; i < 6; ++i) {
        p->var[i] = it->second[i];
        p->var384[i] = it->second[6 + i];
      }
    }
  }

  if (const char* v = getenv("PF_FUSED_VARIANT")) {
    // "p1:1,p2:2,p4:1"
    for (const char* c = v; *c; ++c)
      if (c[0] == 'p' && c[1] >= '1' && c[1] <= '5' && c[2] == ':') {
        const int v = atoi(c + 3);
        (v >= 11 ? p->var384 : p->var)[c[1] - '0'] = v;
      }
  }
  if (const char* v = getenv("PF_FUSED_FP64_ROWS")) p->fp64_rows = atoi(v) != 0;
  // the CTAs of one column tile together (measured at 256^3: FP32 2/3 rule
  // 1.717 vs 1.723 ms per RK3 step, 3/2 rule 8.09 vs 8.24, FP64 3.74 vs 3.81)
  p->f.ilv = 1;
  if (const char* v = getenv("PF_FUSED_ILV")) p->f.ilv = atoi(v) != 0;
  if (const char* v = getenv("PF_FUSED_SPLIT")) {
    for (const char* c = v; *c; ++c)
      if (c[0] == 'p' && (c[1] == '1' || c[1] == '2') && c[2] == ':') {
        const int k = atoi(c + 3), pass = c[1] - '0';
        if (k == 1 || k == (pass == 1 ? 3 : 2)) p->split[pass] = k;
      }
  }

  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, dev);
  const size_t cb = precision == 0 ? 8 : 16;
  f.nmem = nmem;
  p->cap = nmem;
  const size_t a_el = 5ull * f.t0 * f.c1 * f.c2 * nmem, b_el = 6ull * f.t0 * f.t1 * f.c2 * nmem;
  if (cudaMalloc(&p->A, cb * a_el) != cudaSuccess || cudaMalloc(&p->B, cb * b_el) != cudaSuccess ||
      (pad && cudaMalloc(&p->nlM, cb * (size_t)(3 * f.nlcomp) * nmem) != cudaSuccess) ||
      cudaMalloc(&p->err, sizeof(int)) != cudaSuccess ||
      cudaMemset(p->err, 0, sizeof(int)) != cudaSuccess) {
    fused_destroy(p);
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

FusedPlan* fused_create(const Geo& g, int precision, int dealias, int nmem) {
  if ((precision != 0 && precision != 1) || (dealias != 0 && dealias != 1) || nmem < 1)
    return nullptr;
  // 2D: 2/3 rule, sides 2^b 16..1024, FP32 and FP64
  if (g.dim == 2) return dealias == 0 ? fused_create_2d(g, precision, nmem) : nullptr;
  return create3d(g, precision, dealias, nmem, 1);
}

FusedPlan* fused_create_pencil(const Geo& g, int precision, int slabs) {
  if ((precision != 0 && precision != 1) || slabs < 2) return nullptr;
  return create3d(g, precision, 0, 1, slabs);
}

void fused_set_members(FusedPlan* p, int active) {
  if (!p || active < 1 || active > p->cap) return;
  p->f.nmem = active;
  p->f2.nmem = active;
}

void fused_destroy(FusedPlan* p) {
  if (!p) return;
  if (p->A) cudaFree(p->A);
  if (p->B) cudaFree(p->B);
  if (p->nlM) cudaFree(p->nlM);
  if (p->err) cudaFree(p->err);
  delete p;
}

// 2D plans: pass 1 is Q1, pass 3 is Q2 (into the caller's nl), 2 and 4 have
// nothing to do.
template <typename R>
static cudaError_t pass_2d(FusedPlan* p, int pass, const void* uhat, void* nl,
                           unsigned long long* maxbits, cudaStream_t st) {
  switch (pass) {
    case 1: return fused2d_inverse<R>(p->f2, (const cx<R>*)uhat, (cx<R>*)p->A, st);
    case 3: return fused2d_products<R>(p->f2, (const cx<R>*)p->A, (cx<R>*)nl, maxbits, st);
    case 2:
    case 4: return cudaSuccess;
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t fused_pass(FusedPlan* p, int pass, const void* uhat, void* nl,
                       unsigned long long* maxbits, cudaStream_t st) {
  if (!p) return cudaErrorNotReady;
  if (p->dim == 2)
    return p->prec == 0 ? pass_2d<float>(p, pass, uhat, nl, maxbits, st)
                        : pass_2d<double>(p, pass, uhat, nl, maxbits, st);
  if (p->prec == 0) {
    if (!tw_base<float>()) return cudaErrorNotReady;
    return p->pad ? fused_pass_f32_pad(p, pass, uhat, maxbits, st)
                  : fused_pass_f32_trunc(p, pass, uhat, nl, maxbits, st);
  }
  if (!tw_base<double>()) return cudaErrorNotReady;
  return p->pad ? fused_pass_f64_pad(p, pass, uhat, maxbits, st)
                : fused_pass_f64_trunc(p, pass, uhat, nl, maxbits, st);
}

cudaError_t fused_update(FusedPlan* p, const UpdateArgs<float>& U, int ncomp, const void* nl,
                         cudaStream_t st) {
  if (!p || p->prec != 0 || !tw_base<float>()) return cudaErrorNotReady;
  if (p->dim == 2) return fused2d_update<float>(p->f2, U, ncomp, (const float2*)nl, st);
  return p->pad ? fused_update_f32_pad(p, U, ncomp, st)
                : fused_update_f32_trunc(p, U, ncomp, nl, st);
}

cudaError_t fused_update(FusedPlan* p, const UpdateArgs<double>& U, int ncomp, const void* nl,
                         cudaStream_t st) {
  if (!p || p->prec != 1 || !tw_base<double>()) return cudaErrorNotReady;
  if (p->dim == 2) return fused2d_update<double>(p->f2, U, ncomp, (const double2*)nl, st);
  return p->pad ? fused_update_f64_pad(p, U, ncomp, st)
                : fused_update_f64_trunc(p, U, ncomp, nl, st);
}

// Candidate launch variants of pass `pass` for this plan (the first is the
// current choice); empty when the pass has only one.
static std::vector<int> candidates(const FusedPlan* p, int pass, bool& is384) {
  std::vector<int> c;
  is384 = false;
  if (p->prec != 0 || p->dim != 3) return c;
  const FGeo& f = p->f;
  if (pass == 3) {
    if (!p->pad && f.n2 == 256) c = {0, 1, 2, 3, 4, 5};
    if (!p->pad && f.n2 == 128) c = {0, 4};
    return c;
  }
  if (f.nmem > 1) return c;  // members use one launch form for passes 1, 2 and 4
  const int len = pass == 1 ? f.t0 : f.t1;
  if (len == 256) {
    c = {0, 1, 2, 3, 4, 5, 6};
    if (pass == 2) c.insert(c.end(), {7, 8, 9});
    if (pass == 2 && !p->pad && p2t_supported(f)) c.push_back(10);
    if (pass == 1) c.insert(c.end(), {7, 9});
  } else if (len == 384) {
    is384 = true;
    c = {0, 11, 12, 13, 14, 15, 16};
    if (pass == 2) c.insert(c.end(), {17, 18, 19});
    if (pass == 1) c.insert(c.end(), {17, 18});
  }
  return c;
}

cudaError_t fused_autotune(FusedPlan* p, const void* uhat, void* nl, cudaStream_t st,
                           int* picks) {
  if (!p) return cudaErrorInvalidValue;
  if (p->dim != 3) {  // the 2D schedule has one launch form per pass
    if (picks) fused_variants(p, picks);
    return cudaSuccess;
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return cudaGetLastError();
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return cudaGetLastError();
  }
  cudaError_t err = cudaSuccess;
  // Each candidate of a pass is timed inside the whole chain of passes 1-4
  // (they write only plan scratch and nl), so the measurement includes what
  // the pass leaves in L2 for the next one and what it inherits from the
  // previous one; the passes are tuned in order.
  auto chain = [&]() {
    cudaError_t e = cudaSuccess;
    for (int q = 1; q <= 4 && e == cudaSuccess; ++q) e = fused_pass(p, q, uhat, nl, nullptr, st);
    return e;
  };
  for (int pass = 1; pass <= 4 && err == cudaSuccess; ++pass) {
    bool is384;
    const std::vector<int> cand = candidates(p, pass, is384);
    int* slot = is384 ? &p->var384[pass] : &p->var[pass];
    const int keep = *slot;
    // three rounds over all candidates, each candidate's best round counts
    // (variants a few microseconds apart are otherwise picked by noise)
    std::vector<float> best(cand.size(), 1e30f);
    for (int round = 0; round < 3 && err == cudaSuccess; ++round) {
      for (size_t i = 0; i < cand.size() && err == cudaSuccess; ++i) {
        *slot = cand[i];
        err = chain();  // warm-up: first use of the variant, L2 state of the chain
        if (err != cudaSuccess) break;
        float ms = 0.f;
        cudaEventRecord(e0, st);
        for (int r = 0; r < 4 && err == cudaSuccess; ++r) err = chain();
        cudaEventRecord(e1, st);
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
        if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
        if (err == cudaSuccess && ms < best[i]) best[i] = ms;
      }
    }
    int pick = keep;
    float bmin = 1e30f;
    for (size_t i = 0; i < cand.size(); ++i)
      if (best[i] < bmin) {
        bmin = best[i];
        pick = cand[i];
      }
    *slot = err == cudaSuccess ? pick : keep;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess) return err;
  std::array<int, 12> a;
  for (int i = 0; i < 6; ++i) {
    a[i] = p->var[i];
    a[6 + i] = p->var384[i];
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[tune_key(p)] = a;
  }
  if (picks)
    for (int i = 0; i < 12; ++i) picks[i] = a[i];
  return cudaSuccess;
}

void fused_variants(const FusedPlan* p, int* out) {
  for (int i = 0; i < 6; ++i) {
    out[i] = p ? p->var[i] : 0;
    out[6 + i] = p ? p->var384[i] : 0;
  }
}

int fused_device_error(FusedPlan* p) {
  if (!p || !p->err) return 0;
  int v = 0;
  if (cudaMemcpy(&v, p->err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  return v;
}

}  // namespace pf
