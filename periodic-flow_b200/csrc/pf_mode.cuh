// Per-mode physics shared by the update kernels and the fused passes:
// wavenumbers, Leray projection, noise assembly and the stage update rules of
// the five integrators.
#pragma once
#include "pf_common.cuh"
#include "pf_philox.cuh"

namespace pf {

enum Integrator { kExplicitPC = 0, kImplicitPC = 1, kRK2 = 2, kRK3 = 3, kRK4 = 4 };
enum NoiseType { kThermal = 0, kCorrelated = 1 };
enum NoiseSrc { kNoiseNone = 0, kNoisePhilox = 1, kNoiseInjected = 2 };

// One stage of an integrator, dt factored out:
//   base = cu0 u0 + cun unew + cd dt (N + f) + cL dt L (L_on_u0 ? u0 : unew)
//          + cx sqrt(dt) xi
//   unew = implicit ? base / (1 - dt/2 L) : base
// (time_integrator.py:51-56, 111-119, 178-180, 236-241, 292-293)
struct StageCoef {
  double cu0, cun, cd, cL, cx, a;  // a = noise factor of the stage
  int L_on_u0, implicit;
};

struct Scheme {
  int nstages;
  StageCoef st[4];
};

// Mode index decomposition and wavenumbers.
struct ModeIdx { int i0, i1, i2; };

PF_D ModeIdx mode_index(const Geo& g, long long m) {
  ModeIdx r;
  if (g.dim == 3) {
    r.i2 = (int)(m % g.nh);
    const long long t = m / g.nh;
    r.i1 = (int)(t % g.s[1]);
    r.i0 = (int)(t / g.s[1]);
  } else {
    r.i1 = (int)(m % g.nh);
    r.i0 = (int)(m / g.nh);
    r.i2 = 0;
  }
  return r;
}

template <int D> struct KInt { int k[D]; };

template <int D> PF_D KInt<D> kint_of(const Geo& g, const ModeIdx& ix) {
  KInt<D> r;
  if constexpr (D == 3) {
    r.k[0] = kfreq(ix.i0, g.n[0]);
    r.k[1] = kfreq(ix.i1, g.n[1]);
    r.k[2] = ix.i2;
  } else {
    r.k[0] = kfreq(ix.i0, g.n[0]);
    r.k[1] = ix.i1;
  }
  return r;
}

template <int D> PF_D bool keep_dealias(const Geo& g, const KInt<D>& ki) {
  bool keep = true;
#pragma unroll
  for (int a = 0; a < D; ++a) keep = keep && (abs(ki.k[a]) <= g.kmax[a]);
  return keep;
}

template <int D> PF_D bool is_nyquist(const Geo& g, const ModeIdx& ix) {
  const int idx[3] = {ix.i0, ix.i1, ix.i2};
  bool nyq = false;
#pragma unroll
  for (int a = 0; a < D; ++a) nyq = nyq || ((g.n[a] % 2 == 0) && idx[a] == g.n[a] / 2);
  return nyq;
}

template <int D> PF_D bool self_conjugate_plane(const Geo& g, const ModeIdx& ix) {
  const int il = (D == 3) ? ix.i2 : ix.i1;
  const int nl = g.n[D - 1];
  return il == 0 || ((nl % 2 == 0) && il == nl / 2);
}

// Leray projection of a D-vector: p = (k/k^2).v ; v -= p k (math.py:71-100).
// Returns p (the reference's p_hat output).
template <typename R, int D>
PF_D cx<R> leray(cx<R> (&v)[D], const R (&k)[D], R k2) {
  const R inv = k2 == R(0) ? R(0) : R(1) / k2;
  cx<R> p = czero<cx<R>>();
#pragma unroll
  for (int a = 0; a < D; ++a) p = cadd(p, cscale(v[a], k[a] * inv));
#pragma unroll
  for (int a = 0; a < D; ++a) v[a] = csub(v[a], cscale(p, k[a]));
  return p;
}

// Unprojected, unscaled noise of one stage from w = w1 + a w2
// (space_solver.py:240-265).  thermal: xi_a = i sum_b k_b (W_ab + W_ba)
// sqrt(1/2); correlated: C w.
template <typename R, int D, int NC>
PF_D void noise_raw(cx<R> (&xi)[D], const cx<R> (&w1)[NC], const cx<R> (&w2)[NC], R a,
                    int noise_type, const R (&k)[D], R corr) {
  if (noise_type == kThermal) {
    const R f = R(0.70710678118654752440);
#pragma unroll
    for (int i = 0; i < D; ++i) {
      cx<R> acc = czero<cx<R>>();
#pragma unroll
      for (int b = 0; b < D; ++b) {
        if (i * D + b < NC && b * D + i < NC) {
          const cx<R> wib = cadd(w1[i * D + b], cscale(w2[i * D + b], a));
          const cx<R> wbi = cadd(w1[b * D + i], cscale(w2[b * D + i], a));
          acc = cadd(acc, cscale(cadd(wib, wbi), f * k[b]));
        }
      }
      xi[i] = cmuli(acc);
    }
  } else {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      if (i < NC) xi[i] = cscale(cadd(w1[i], cscale(w2[i], a)), corr);
      else xi[i] = czero<cx<R>>();
    }
  }
}

// Noise of one stage: noise_raw, Leray projection, times noise_mag.
template <typename R, int D, int NC>
PF_D void noise_term(cx<R> (&xi)[D], const cx<R> (&w1)[NC], const cx<R> (&w2)[NC], R a,
                     int noise_type, const R (&k)[D], R k2, R corr, R mag) {
  noise_raw<R, D, NC>(xi, w1, w2, a, noise_type, k, corr);
  leray<R, D>(xi, k, k2);
#pragma unroll
  for (int i = 0; i < D; ++i) xi[i] = cscale(xi[i], mag);
}

// Stage update of one component.
template <typename R>
PF_D cx<R> stage_update(const StageCoef& c, R dt, R sqdt, R L, cx<R> u0, cx<R> unew,
                        cx<R> nf /* N + f */, cx<R> xi) {
  const cx<R> lu = cscale(c.L_on_u0 ? u0 : unew, L);
  cx<R> base = cscale(u0, (R)c.cu0);
  if (c.cun != 0.0) base = cadd(base, cscale(unew, (R)c.cun));
  base = cadd(base, cscale(nf, (R)c.cd * dt));
  base = cadd(base, cscale(lu, (R)c.cL * dt));
  if (c.cx != 0.0) base = cadd(base, cscale(xi, (R)c.cx * sqdt));
  if (c.implicit) base = cscale(base, R(1) / (R(1) - dt * R(0.5) * L));
  return base;
}

}  // namespace pf
