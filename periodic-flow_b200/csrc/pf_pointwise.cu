// Pointwise kernels of the solver:
//   * k_update      : one fused stage of any integrator for every mode
//                     (Leray projection and Nyquist mask of N, linear term,
//                     noise assembly, forcing, update rule, optional E/Z sums);
//   * k_stokes      : whole steps of the linear (Stokes) problem with the
//                     state in registers and in-register Philox noise;
//   * k_mask_copy / k_curl_masked / k_cross : pieces of the per-operator
//                     nonlinear term;
//   * reductions    : forcing-band energy, max |u|/dx for CFL, E and Z,
//                     shell spectrum.
#include <cstdio>

#include "pf_kernels.h"
#include "pf_update.cuh"

namespace pf {

constexpr int kBlock = 256;

static unsigned grid_for(long long n, int per_block = kBlock, long long cap = 148LL * 16) {
  long long b = (n + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

template <typename R, int D, int NC>
__global__ void __launch_bounds__(kBlock) k_update(UpdateArgs<R> A) {
  using C = cx<R>;
  const Geo& g = A.g;
  const StageScalars<R> sc = stage_scalars<R>(A);
  double accE = 0.0, accZ = 0.0;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<R, D> mk_ = mode_k<R, D>(g, m);
    C nv[D];
#pragma unroll
    for (int a = 0; a < D; ++a) nv[a] = A.nl ? A.nl[a * g.nspec + m] : czero<C>();
    update_mode<R, D, NC>(A, m, mk_, nv, A.nl != nullptr, sc, accE, accZ);
  }
  if (A.diag) block_add2(accE, accZ, A.diag);
}

// Whole steps of the Stokes problem (no nonlinear term, no forcing): the
// state of a mode stays in registers across stages and steps.
template <typename R, int D, int NC>
__global__ void __launch_bounds__(kBlock) k_stokes(StokesArgs<R> A) {
  using C = cx<R>;
  const Geo& g = A.g;
  const R dt = (R)A.dt;
  const R sqdt = (R)sqrt(A.dt);
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<R, D> mk_ = mode_k<R, D>(g, m);
    C u[D];
#pragma unroll
    for (int a = 0; a < D; ++a) u[a] = A.uhat[a * g.nspec + m];
    const R L = A.lop ? A.lop[m] : (R)(-A.nu) * mk_.k2;
    const R corr = A.corr ? A.corr[m] : R(0);
    const DrawSite site = draw_site(g, mk_.ix.i0, mk_.ix.i1, mk_.ix.i2);
    const R nf = mk_.k2 == R(0) ? R(0) : (R)A.noise_norm;
    // A mode whose noise amplitude is exactly zero (k = 0, or a correlation
    // function that vanishes there) gets xi = 0 whatever the draws are, and
    // counter-based draws of other modes do not depend on it: skip them.
    const bool philox = A.noise_src == kNoisePhilox && nf != R(0) &&
                        (A.noise_type == kThermal || corr != R(0));
    const bool noisy = philox || A.noise_src == kNoiseInjected;
    for (int s = 0; s < A.nsteps; ++s) {
      const uint64_t step = A.step0 + (uint64_t)s;
      C w1[NC], w2[NC];
      if (philox) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          w1[c] = cscale(draw_value<R>(site, c, A.seed, step), nf);
          w2[c] = cscale(draw_value<R>(site, NC + c, A.seed, step), nf);
        }
      } else if (A.noise_src == kNoiseInjected) {
#pragma unroll
        for (int c = 0; c < NC; ++c) {
          w1[c] = A.winj[(long long)c * g.nspec + m];
          w2[c] = A.winj[(long long)(NC + c) * g.nspec + m];
        }
      }
      C u0[D];
#pragma unroll
      for (int a = 0; a < D; ++a) u0[a] = u[a];
      // first_stage = 1 skips the implicit predictor, whose result the
      // corrector never reads when there is no nonlinear term or forcing
      for (int st = A.first_stage; st < A.scheme.nstages; ++st) {
        const StageCoef& cf = A.scheme.st[st];
        C xi[D];
        if (noisy) {
          noise_term<R, D, NC>(xi, w1, w2, (R)cf.a, A.noise_type, mk_.k, mk_.k2, corr,
                               (R)A.noise_mag);
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
    for (int a = 0; a < D; ++a) A.uhat[a * g.nspec + m] = u[a];
  }
}

// dst = mask_2/3(src), ncomp fields
template <typename R, int D>
__global__ void k_mask_copy(cx<R>* __restrict__ dst, const cx<R>* __restrict__ src, Geo g,
                            int ncomp) {
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeIdx ix = mode_index(g, m);
    const bool keep = keep_dealias<D>(g, kint_of<D>(g, ix));
    for (int c = 0; c < ncomp; ++c)
      dst[c * g.nspec + m] = keep ? src[c * g.nspec + m] : czero<cx<R>>();
  }
}

// dst = mask_2/3(i k x u)  (math.py:31-49)
template <typename R, int D>
__global__ void k_curl_masked(cx<R>* __restrict__ dst, const cx<R>* __restrict__ u, Geo g) {
  using C = cx<R>;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<R, D> q = mode_k<R, D>(g, m);
    const bool keep = keep_dealias<D>(g, q.ki);
    if constexpr (D == 2) {
      const C a0 = u[m], a1 = u[g.nspec + m];
      C w = cmuli(csub(cscale(a1, q.k[0]), cscale(a0, q.k[1])));
      dst[m] = keep ? w : czero<C>();
    } else {
      const C a0 = u[m], a1 = u[g.nspec + m], a2 = u[2 * g.nspec + m];
      C w0 = cmuli(csub(cscale(a2, q.k[1]), cscale(a1, q.k[2])));
      C w1 = cmuli(csub(cscale(a0, q.k[2]), cscale(a2, q.k[0])));
      C w2 = cmuli(csub(cscale(a1, q.k[0]), cscale(a0, q.k[1])));
      dst[m] = keep ? w0 : czero<C>();
      dst[g.nspec + m] = keep ? w1 : czero<C>();
      dst[2 * g.nspec + m] = keep ? w2 : czero<C>();
    }
  }
}

// u <- u x w in place (math.py:4-28); optional max of sum |u_i| / dx_i
template <typename R, int D>
__global__ void k_cross(R* __restrict__ u, const R* __restrict__ w, Geo g,
                        unsigned long long* __restrict__ maxbits) {
  double mx = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < g.nphys;
       p += (long long)gridDim.x * blockDim.x) {
    if constexpr (D == 2) {
      const R a0 = u[p], a1 = u[g.nphys + p], b = w[p];
      if (maxbits) {
        const double s = fabs((double)a0) * g.n[0] / (2.0 * M_PI / g.kscale[0]) +
                         fabs((double)a1) * g.n[1] / (2.0 * M_PI / g.kscale[1]);
        mx = fmax(mx, s);
      }
      u[p] = a1 * b;
      u[g.nphys + p] = -a0 * b;
    } else {
      const R a0 = u[p], a1 = u[g.nphys + p], a2 = u[2 * g.nphys + p];
      const R b0 = w[p], b1 = w[g.nphys + p], b2 = w[2 * g.nphys + p];
      if (maxbits) {
        const double s = fabs((double)a0) * g.n[0] * g.kscale[0] / (2.0 * M_PI) +
                         fabs((double)a1) * g.n[1] * g.kscale[1] / (2.0 * M_PI) +
                         fabs((double)a2) * g.n[2] * g.kscale[2] / (2.0 * M_PI);
        mx = fmax(mx, s);
      }
      u[p] = a1 * b2 - a2 * b1;
      u[g.nphys + p] = a2 * b0 - a0 * b2;
      u[2 * g.nphys + p] = a0 * b1 - a1 * b0;
    }
  }
  if (maxbits) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    // non-negative doubles order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
  }
}

// dscal[dt] = cfl / max, from the double bits written by k_cross or P3 (one
// thread per member); the word is reset to zero for the next maximum
__global__ void k_set_dt(double* dscal, unsigned long long* maxbits, double cfl, int nmem) {
  for (int m = threadIdx.x; m < nmem; m += blockDim.x) {
    double* d = dscal + (long long)m * kScalCount;
    const double mx = __longlong_as_double((long long)maxbits[m]);
    maxbits[m] = 0ull;
    if (mx > 0.0) d[kScalDt] = cfl / mx;
    d[kScalTime] += d[kScalDt];
  }
}

// t += dt, n times (the reference accumulates t step by step, simulation.py:206)
__global__ void k_advance_time(double* dscal, int n, int nmem) {
  for (int m = threadIdx.x; m < nmem; m += blockDim.x) {
    double* d = dscal + (long long)m * kScalCount;
    for (int i = 0; i < n; ++i) d[kScalTime] += d[kScalDt];
  }
}

// E_band = 1/2 sum_{0<|k|^2<=kf^2} w |u|^2  -> dscal[kScalBandE].  Visits only
// the index box that can hold the band: per axis cnt[a] slots, slot s maps to
// index s when the whole axis is needed, else to wavenumber s - K (mod n).
struct BandBox { int cnt[3], K[3], full[3]; long long total; };

// single: one CTA per member stores the sum (no zeroed slot needed);
// otherwise CTAs add into a zeroed slot.
template <typename R, int D, bool SINGLE = false>
__global__ void k_band_energy(const cx<R>* __restrict__ u, Geo g, double kf2, BandBox bx,
                              double* dscal) {
  // member blockIdx.y of boxes laid out one after another
  u += (long long)blockIdx.y * D * g.nspec;
  dscal += (long long)blockIdx.y * kScalCount;
  double acc = 0.0;
  for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < bx.total;
       b += (long long)gridDim.x * blockDim.x) {
    int idx[3] = {0, 0, 0};
    long long r = b;
    for (int a = D - 1; a >= 0; --a) {
      const int s = (int)(r % bx.cnt[a]);
      r /= bx.cnt[a];
      if (a == D - 1 || bx.full[a]) idx[a] = s;
      else idx[a] = ((s - bx.K[a]) % g.n[a] + g.n[a]) % g.n[a];
    }
    long long m = idx[0];
    for (int a = 1; a < D; ++a) m = m * g.s[a] + idx[a];
    const ModeK<double, D> q = mode_k<double, D>(g, m);
    if (q.k2 > 0.0 && q.k2 <= kf2) {
      double e = 0.0;
      for (int a = 0; a < D; ++a) {
        const cx<R> z = u[a * g.nspec + m];
        e += (double)z.x * z.x + (double)z.y * z.y;
      }
      acc += 0.5 * half_weight(g, q.ix) * e;
    }
  }
  if constexpr (SINGLE) block_store2(acc, 0.0, dscal + kScalBandE);
  else block_add2(acc, 0.0, dscal + kScalBandE);
}

template <typename R, int D>
__global__ void k_energy(const cx<R>* __restrict__ u, Geo g, double* out2) {
  double accE = 0.0, accZ = 0.0;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<double, D> q = mode_k<double, D>(g, m);
    double e = 0.0;
    for (int a = 0; a < D; ++a) {
      const cx<R> z = u[a * g.nspec + m];
      e += (double)z.x * z.x + (double)z.y * z.y;
    }
    const double w = half_weight(g, q.ix);
    accE += 0.5 * w * e;
    accZ += 0.5 * w * e * q.k2;
  }
  block_add2(accE, accZ, out2);
}

template <typename R, int D>
__global__ void k_spectrum(const cx<R>* __restrict__ u, Geo g, double* out, int nbins,
                           double kunit) {
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < g.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<double, D> q = mode_k<double, D>(g, m);
    double e = 0.0;
    for (int a = 0; a < D; ++a) {
      const cx<R> z = u[a * g.nspec + m];
      e += (double)z.x * z.x + (double)z.y * z.y;
    }
    const int b = (int)floor(sqrt(q.k2) / kunit + 0.5);
    if (b < nbins) atomicAdd(out + b, 0.5 * half_weight(g, q.ix) * e);
  }
}

// ------------------------------------------------- 3/2 padding / truncation
// Grid M = 3N/2 per axis.  Padding writes the trigonometric polynomial of an
// N-grid spectrum onto the M grid: a Nyquist mode of an even side is split in
// half between +N/2 and -N/2 (complex axes) or halved (last axis, whose -N/2
// partner is implied by Hermitian symmetry).  Truncation is the matching fold:
// modes |k| < N/2 are copied, Nyquist modes sum their +N/2 and -N/2 partners.
struct AxisMap { int j[2]; int n; };

PF_D AxisMap pad_targets(int i, int N, int M) {
  AxisMap a;
  if ((N % 2 == 0) && i == N / 2) {
    a.n = 2; a.j[0] = N / 2; a.j[1] = M - N / 2;
  } else {
    const int k = kfreq(i, N);
    a.n = 1; a.j[0] = k >= 0 ? k : M + k; a.j[1] = 0;
  }
  return a;
}

template <typename R, int D>
__global__ void k_pad(cx<R>* __restrict__ dst, const cx<R>* __restrict__ src, Geo gN, Geo gM,
                      int ncomp, int curl) {
  using C = cx<R>;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < gN.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeK<R, D> q = mode_k<R, D>(gN, m);
    C val[3];
    int nout = ncomp;
    if (curl) {
      // i k x u on the N grid (math.py:31-49), then padded
      if constexpr (D == 2) {
        const C a0 = src[m], a1 = src[gN.nspec + m];
        val[0] = cmuli(csub(cscale(a1, q.k[0]), cscale(a0, q.k[1])));
        nout = 1;
      } else {
        const C a0 = src[m], a1 = src[gN.nspec + m], a2 = src[2 * gN.nspec + m];
        val[0] = cmuli(csub(cscale(a2, q.k[1]), cscale(a1, q.k[2])));
        val[1] = cmuli(csub(cscale(a0, q.k[2]), cscale(a2, q.k[0])));
        val[2] = cmuli(csub(cscale(a1, q.k[0]), cscale(a0, q.k[1])));
        nout = 3;
      }
    } else {
      for (int c = 0; c < ncomp; ++c) val[c] = src[c * gN.nspec + m];
    }
    const int il = D == 3 ? q.ix.i2 : q.ix.i1;
    const int nl = gN.n[D - 1];
    const R fl = ((nl % 2 == 0) && il == nl / 2) ? R(0.5) : R(1);
    const AxisMap a0 = pad_targets(q.ix.i0, gN.n[0], gM.n[0]);
    AxisMap a1;
    if constexpr (D == 3) a1 = pad_targets(q.ix.i1, gN.n[1], gM.n[1]);
    else { a1.n = 1; a1.j[0] = 0; }
    const R f0 = a0.n == 2 ? R(0.5) : R(1), f1 = a1.n == 2 ? R(0.5) : R(1);
    for (int s0 = 0; s0 < a0.n; ++s0)
      for (int s1 = 0; s1 < a1.n; ++s1) {
        const long long dm = D == 3 ? ((long long)a0.j[s0] * gM.s[1] + a1.j[s1]) * gM.nh + il
                                    : (long long)a0.j[s0] * gM.nh + il;
        for (int c = 0; c < nout; ++c) dst[c * gM.nspec + dm] = cscale(val[c], f0 * f1 * fl);
      }
  }
}

template <typename R, int D>
__global__ void k_truncate(cx<R>* __restrict__ dst, const cx<R>* __restrict__ src, Geo gN,
                           Geo gM, int ncomp) {
  using C = cx<R>;
  for (long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x; m < gN.nspec;
       m += (long long)gridDim.x * blockDim.x) {
    const ModeIdx ix = mode_index(gN, m);
    const int il = D == 3 ? ix.i2 : ix.i1;
    const int nl = gN.n[D - 1];
    const bool nyq_last = (nl % 2 == 0) && il == nl / 2;
    const AxisMap a0 = pad_targets(ix.i0, gN.n[0], gM.n[0]);
    AxisMap a1;
    if constexpr (D == 3) a1 = pad_targets(ix.i1, gN.n[1], gM.n[1]);
    else { a1.n = 1; a1.j[0] = 0; }
    for (int c = 0; c < ncomp; ++c) {
      C acc = czero<C>();
      for (int s0 = 0; s0 < a0.n; ++s0)
        for (int s1 = 0; s1 < a1.n; ++s1) {
          const int j0 = a0.j[s0], j1 = a1.j[s1];
          const long long sm = D == 3 ? ((long long)j0 * gM.s[1] + j1) * gM.nh + il
                                      : (long long)j0 * gM.nh + il;
          acc = cadd(acc, src[c * gM.nspec + sm]);
          if (nyq_last) {  // the -N/2 partner: conjugate of the mirror mode
            const int r0 = (gM.n[0] - j0) % gM.n[0];
            const int r1 = D == 3 ? (gM.n[1] - j1) % gM.n[1] : 0;
            const long long mm = D == 3 ? ((long long)r0 * gM.s[1] + r1) * gM.nh + il
                                        : (long long)r0 * gM.nh + il;
            acc = cadd(acc, cconj(src[c * gM.nspec + mm]));
          }
        }
      dst[c * gN.nspec + m] = acc;
    }
  }
}

template <typename R>
cudaError_t launch_pad(cx<R>* dst, const cx<R>* src, const Geo& gN, const Geo& gM, int ncomp,
                       int curl, cudaStream_t st) {
  const int nout = curl ? (gN.dim == 3 ? 3 : 1) : ncomp;
  cudaError_t e = cudaMemsetAsync(dst, 0, sizeof(cx<R>) * (size_t)nout * gM.nspec, st);
  if (e != cudaSuccess) return e;
  if (gN.dim == 3) k_pad<R, 3><<<grid_for(gN.nspec), kBlock, 0, st>>>(dst, src, gN, gM, ncomp, curl);
  else k_pad<R, 2><<<grid_for(gN.nspec), kBlock, 0, st>>>(dst, src, gN, gM, ncomp, curl);
  return launched();
}

template <typename R>
cudaError_t launch_truncate(cx<R>* dst, const cx<R>* src, const Geo& gN, const Geo& gM,
                            int ncomp, cudaStream_t st) {
  if (gN.dim == 3) k_truncate<R, 3><<<grid_for(gN.nspec), kBlock, 0, st>>>(dst, src, gN, gM, ncomp);
  else k_truncate<R, 2><<<grid_for(gN.nspec), kBlock, 0, st>>>(dst, src, gN, gM, ncomp);
  return launched();
}

template cudaError_t launch_pad<float>(float2*, const float2*, const Geo&, const Geo&, int, int,
                                       cudaStream_t);
template cudaError_t launch_pad<double>(double2*, const double2*, const Geo&, const Geo&, int,
                                        int, cudaStream_t);
template cudaError_t launch_truncate<float>(float2*, const float2*, const Geo&, const Geo&, int,
                                            cudaStream_t);
template cudaError_t launch_truncate<double>(double2*, const double2*, const Geo&, const Geo&,
                                             int, cudaStream_t);

// -------------------------------------------------------------- launchers
template <typename R>
cudaError_t launch_update(const UpdateArgs<R>& A, int ncomp, cudaStream_t st) {
  const unsigned grid = grid_for(A.g.nspec);
  if (A.g.dim == 3) {
    if (ncomp == 9) k_update<R, 3, 9><<<grid, kBlock, 0, st>>>(A);
    else k_update<R, 3, 3><<<grid, kBlock, 0, st>>>(A);
  } else {
    if (ncomp == 4) k_update<R, 2, 4><<<grid, kBlock, 0, st>>>(A);
    else k_update<R, 2, 2><<<grid, kBlock, 0, st>>>(A);
  }
  return launched();
}

template <typename R>
cudaError_t launch_stokes(const StokesArgs<R>& A, int ncomp, cudaStream_t st) {
  const unsigned grid = grid_for(A.g.nspec, kBlock, 148LL * 64);
  if (A.g.dim == 3) {
    if (ncomp == 9) k_stokes<R, 3, 9><<<grid, kBlock, 0, st>>>(A);
    else k_stokes<R, 3, 3><<<grid, kBlock, 0, st>>>(A);
  } else {
    if (ncomp == 4) k_stokes<R, 2, 4><<<grid, kBlock, 0, st>>>(A);
    else k_stokes<R, 2, 2><<<grid, kBlock, 0, st>>>(A);
  }
  return launched();
}

template <typename R>
cudaError_t launch_mask_copy(cx<R>* dst, const cx<R>* src, const Geo& g, int ncomp,
                             cudaStream_t st) {
  if (g.dim == 3) k_mask_copy<R, 3><<<grid_for(g.nspec), kBlock, 0, st>>>(dst, src, g, ncomp);
  else k_mask_copy<R, 2><<<grid_for(g.nspec), kBlock, 0, st>>>(dst, src, g, ncomp);
  return launched();
}

template <typename R>
cudaError_t launch_curl_masked(cx<R>* dst, const cx<R>* u, const Geo& g, cudaStream_t st) {
  if (g.dim == 3) k_curl_masked<R, 3><<<grid_for(g.nspec), kBlock, 0, st>>>(dst, u, g);
  else k_curl_masked<R, 2><<<grid_for(g.nspec), kBlock, 0, st>>>(dst, u, g);
  return launched();
}

template <typename R>
cudaError_t launch_cross(R* u, const R* w, const Geo& g, unsigned long long* maxbits,
                         cudaStream_t st) {
  if (g.dim == 3) k_cross<R, 3><<<grid_for(g.nphys), kBlock, 0, st>>>(u, w, g, maxbits);
  else k_cross<R, 2><<<grid_for(g.nphys), kBlock, 0, st>>>(u, w, g, maxbits);
  return launched();
}

cudaError_t launch_set_dt(double* dscal, unsigned long long* maxbits, double cfl,
                          cudaStream_t st, int nmem) {
  k_set_dt<<<1, nmem < 256 ? (nmem < 32 ? 32 : nmem) : 256, 0, st>>>(dscal, maxbits, cfl, nmem);
  return launched();
}

cudaError_t launch_advance_time(double* dscal, int n, cudaStream_t st, int nmem) {
  k_advance_time<<<1, nmem < 256 ? (nmem < 32 ? 32 : nmem) : 256, 0, st>>>(dscal, n, nmem);
  return launched();
}

template <typename R>
cudaError_t launch_band_energy(const cx<R>* u, const Geo& g, double kf2, double* dscal,
                               cudaStream_t st, int nmem) {
  BandBox bx;
  bx.total = 1;
  const double kf = sqrt(kf2);
  for (int a = 0; a < 3; ++a) { bx.cnt[a] = 1; bx.K[a] = 0; bx.full[a] = 0; }
  for (int a = 0; a < g.dim; ++a) {
    const int K = (int)floor(kf / g.kscale[a] + 1e-9);
    if (a == g.dim - 1) {
      bx.cnt[a] = (K < g.nh - 1 ? K : g.nh - 1) + 1;
    } else if (2 * K + 1 >= g.n[a]) {
      bx.full[a] = 1;
      bx.cnt[a] = g.n[a];
    } else {
      bx.K[a] = K;
      bx.cnt[a] = 2 * K + 1;
    }
    bx.total *= bx.cnt[a];
  }
  if (bx.total <= 64 * kBlock) {  // one CTA per member stores its sum
    const dim3 grid(1, (unsigned)nmem);
    if (g.dim == 3) k_band_energy<R, 3, true><<<grid, kBlock, 0, st>>>(u, g, kf2, bx, dscal);
    else k_band_energy<R, 2, true><<<grid, kBlock, 0, st>>>(u, g, kf2, bx, dscal);
    return launched();
  }
  // zero each member's band-energy slot (dscal rows of kScalCount doubles)
  cudaError_t e = cudaMemset2DAsync(dscal + kScalBandE, sizeof(double) * kScalCount, 0,
                                    sizeof(double), (size_t)nmem, st);
  if (e != cudaSuccess) return e;
  const dim3 grid(grid_for(bx.total), (unsigned)nmem);
  if (g.dim == 3) k_band_energy<R, 3><<<grid, kBlock, 0, st>>>(u, g, kf2, bx, dscal);
  else k_band_energy<R, 2><<<grid, kBlock, 0, st>>>(u, g, kf2, bx, dscal);
  return launched();
}

template <typename R>
cudaError_t launch_energy(const cx<R>* u, const Geo& g, double* out2, cudaStream_t st) {
  if (g.dim == 3) k_energy<R, 3><<<grid_for(g.nspec), kBlock, 0, st>>>(u, g, out2);
  else k_energy<R, 2><<<grid_for(g.nspec), kBlock, 0, st>>>(u, g, out2);
  return launched();
}

template <typename R>
cudaError_t launch_spectrum(const cx<R>* u, const Geo& g, double* out, int nbins,
                            double kunit, cudaStream_t st) {
  if (g.dim == 3) k_spectrum<R, 3><<<grid_for(g.nspec), kBlock, 0, st>>>(u, g, out, nbins, kunit);
  else k_spectrum<R, 2><<<grid_for(g.nspec), kBlock, 0, st>>>(u, g, out, nbins, kunit);
  return launched();
}

#define PF_INST(R)                                                                          \
  template cudaError_t launch_update<R>(const UpdateArgs<R>&, int, cudaStream_t);           \
  template cudaError_t launch_stokes<R>(const StokesArgs<R>&, int, cudaStream_t);           \
  template cudaError_t launch_mask_copy<R>(cx<R>*, const cx<R>*, const Geo&, int,           \
                                           cudaStream_t);                                   \
  template cudaError_t launch_curl_masked<R>(cx<R>*, const cx<R>*, const Geo&,              \
                                             cudaStream_t);                                 \
  template cudaError_t launch_cross<R>(R*, const R*, const Geo&, unsigned long long*,       \
                                       cudaStream_t);                                       \
  template cudaError_t launch_band_energy<R>(const cx<R>*, const Geo&, double, double*,     \
                                             cudaStream_t, int);                            \
  template cudaError_t launch_energy<R>(const cx<R>*, const Geo&, double*, cudaStream_t);   \
  template cudaError_t launch_spectrum<R>(const cx<R>*, const Geo&, double*, int, double,   \
                                          cudaStream_t);
PF_INST(float)
PF_INST(double)
#undef PF_INST

}  // namespace pf
