// Per-mode stage update shared by the stand-alone update kernel and the fused
// last pass (forward FFT along axis 0 + update): Leray projection and Nyquist
// mask of the nonlinear term, forcing, noise, linear term, integrator rule,
// optional E / Z sums (space_solver.py:240-310, time_integrator.py:36-318).
#pragma once
#include "pf_kernels.h"
#include "pf_mode.cuh"

namespace pf {

// FP64 block reduction of two partial sums, stored into gl[0], gl[1] by one
// thread (block_store2: the block's own slots) or added to them atomically
// (block_add2).  Every thread of the block must call it.
template <bool ADD>
PF_D void block_reduce2(double a, double b, double* gl) {
  __shared__ double sa[32], sb[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int w = tid >> 5, l = tid & 31;
  if (l == 0) { sa[w] = a; sb[w] = b; }
  __syncthreads();
  if (w == 0) {
    const int nw = (nthreads + 31) >> 5;
    a = l < nw ? sa[l] : 0.0;
    b = l < nw ? sb[l] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (l == 0) {
      if constexpr (ADD) { atomicAdd(gl, a); atomicAdd(gl + 1, b); }
      else { gl[0] = a; gl[1] = b; }
    }
  }
}
PF_D void block_store2(double a, double b, double* gl) { block_reduce2<false>(a, b, gl); }

PF_D void block_add2(double a, double b, double* gl) { block_reduce2<true>(a, b, gl); }

// Member mb of a launch over boxes laid out member after member: its state
// is at uhat / u0 + mo (mo = mb * mstride), its scalars at dscal + mb *
// kScalCount, its E/Z sums at diag + 2 mb, and it draws noise with key seed +
// mb.  L(k) and C(k) arrays are shared.
struct Member {
  long long mo;
  int mb;
};
template <typename R> PF_D Member member_of(const UpdateArgs<R>& A, int mb) {
  Member r;
  r.mb = mb;
  r.mo = (long long)mb * A.mstride;
  return r;
}

template <typename R, int D> struct ModeK {
  R k[D];
  R k2;
  KInt<D> ki;
  ModeIdx ix;
};

template <typename R, int D> PF_D ModeK<R, D> mode_k(const Geo& g, long long m) {
  ModeK<R, D> r;
  r.ix = mode_index(g, m);
  r.ki = kint_of<D>(g, r.ix);
  double k2 = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double ka = g.kscale[a] * (double)r.ki.k[a];
    r.k[a] = (R)ka;
    k2 += ka * ka;
  }
  r.k2 = (R)k2;
  return r;
}

PF_D double half_weight(const Geo& g, const ModeIdx& ix) {
  const int il = g.dim == 3 ? ix.i2 : ix.i1;
  const int nl = g.n[g.dim - 1];
  return (il == 0 || ((nl % 2 == 0) && il == nl / 2)) ? 1.0 : 2.0;
}

// w1, w2 of one mode: injected arrays or Philox draws times the normal factor
// mask(k != 0) / sqrt(prod N) / sqrt(2 - 2/d) (space_solver.py:143-145, 227-238)
template <typename R, int D, int NC>
PF_D void load_noise(const UpdateArgs<R>& A, long long m, const ModeK<R, D>& mk_,
                     cx<R> (&w1)[NC], cx<R> (&w2)[NC], int mb = 0) {
  if (A.noise_src == kNoiseInjected) {
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      w1[c] = A.winj[(long long)c * A.g.nspec + m];
      w2[c] = A.winj[(long long)(NC + c) * A.g.nspec + m];
    }
  } else {
    const DrawSite s = draw_site(A.g, mk_.ix.i0, mk_.ix.i1, mk_.ix.i2);
    const R nf = mk_.k2 == R(0) ? R(0) : (R)A.noise_norm;
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      w1[c] = cscale(draw_value<R>(s, c, A.seed + (uint64_t)mb, A.step), nf);
      w2[c] = cscale(draw_value<R>(s, NC + c, A.seed + (uint64_t)mb, A.step), nf);
    }
  }
}

template <typename R> struct StageScalars { R dt, sqdt, fcoef; };

template <typename R> PF_D StageScalars<R> stage_scalars(const UpdateArgs<R>& A, int mb = 0) {
  const double* ds = A.dscal + (long long)mb * kScalCount;
  StageScalars<R> s;
  s.dt = (R)ds[kScalDt];
  s.sqdt = (R)sqrt(ds[kScalDt]);
  s.fcoef = R(0);
  if (A.forcing) {
    const double ef = ds[kScalBandE];
    s.fcoef = ef > 0.0 ? (R)(A.f_eps / (2.0 * ef)) : R(0);
  }
  return s;
}

// Update of mode m from preloaded state un (current) and u0v (start of step)
// and its unprojected nonlinear term nv (ignored when !has_nl); writes the new
// state through uh (and u0 at the first stage unless A.uout takes the new
// state), adds to the E/Z sums.  NOISE = false compiles the noise path out
// (noise_mag == 0).  uh, u0: the member's write targets (A.uout or A.uhat,
// and A.u0, offset by the member), mb its member index.
template <typename R, int D, int NC, bool NOISE>
PF_D void update_core(const UpdateArgs<R>& A, long long m, const ModeK<R, D>& mk_,
                      cx<R> (&nv)[D], bool has_nl, cx<R> (&un)[D], const cx<R> (&u0v)[D],
                      const StageScalars<R>& sc, double& accE, double& accZ,
                      cx<R>* __restrict__ uh, cx<R>* __restrict__ u0, int mb) {
  using C = cx<R>;
  const Geo& g = A.g;
  C xi[D];
  if (A.save_u0 && !A.uout) {
#pragma unroll
    for (int a = 0; a < D; ++a) u0[a * g.nspec + m] = un[a];
  }
  // nonlinear term: Leray projection, optional Nyquist mask (space_solver.py:297-300)
  if (has_nl) {
    leray<R, D>(nv, mk_.k, mk_.k2);
    if (A.nyq_mask && is_nyquist<D>(g, mk_.ix)) {
#pragma unroll
      for (int a = 0; a < D; ++a) nv[a] = czero<C>();
    }
  } else {
#pragma unroll
    for (int a = 0; a < D; ++a) nv[a] = czero<C>();
  }
  // linear band forcing: eps / (2 E_band) u on 0 < |k|^2 <= kf^2
  if (A.forcing && mk_.k2 > R(0) && (double)mk_.k2 <= A.f_kf2) {
#pragma unroll
    for (int a = 0; a < D; ++a) nv[a] = cadd(nv[a], cscale(un[a], sc.fcoef));
  }
  if (NOISE && A.noise_src != kNoiseNone) {
    C w1[NC], w2[NC];
    load_noise<R, D, NC>(A, m, mk_, w1, w2, mb);
    const R corr = A.corr ? A.corr[m] : R(0);
    noise_term<R, D, NC>(xi, w1, w2, (R)A.coef.a, A.noise_type, mk_.k, mk_.k2, corr,
                         (R)A.noise_mag);
  } else {
#pragma unroll
    for (int a = 0; a < D; ++a) xi[a] = czero<C>();
  }
  const R L = A.lop ? A.lop[m] : (R)(-A.nu) * mk_.k2;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const C r = stage_update<R>(A.coef, sc.dt, sc.sqdt, L, u0v[a], un[a], nv[a], xi[a]);
    uh[a * g.nspec + m] = r;
    un[a] = r;
  }
  if (A.diag) {
    double e = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) e += (double)un[a].x * un[a].x + (double)un[a].y * un[a].y;
    const double w = half_weight(g, mk_.ix);
    accE += 0.5 * w * e;
    accZ += 0.5 * w * e * (double)mk_.k2;
  }
}

// Loads the state of mode m and updates it (stand-alone update kernel).
template <typename R, int D, int NC>
PF_D void update_mode(const UpdateArgs<R>& A, long long m, const ModeK<R, D>& mk_,
                      cx<R> (&nv)[D], bool has_nl, const StageScalars<R>& sc, double& accE,
                      double& accZ) {
  cx<R> un[D], u0v[D];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    un[a] = A.uhat[a * A.g.nspec + m];
    u0v[a] = A.save_u0 ? un[a] : A.u0[a * A.g.nspec + m];
  }
  update_core<R, D, NC, true>(A, m, mk_, nv, has_nl, un, u0v, sc, accE, accZ,
                              A.uout ? A.uout : A.uhat, A.u0, 0);
}

}  // namespace pf
