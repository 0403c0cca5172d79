// Fused passes of the 2D nonlinear term with the 2/3 rule (the 2D branch of
// space_solver.py:280-300 with math.py:4-49: omega = i (k0 u1 - k1 u0),
// u x omega = (u1 omega, -u0 omega)).
//
// Only columns k1 <= kmax1 and rows |k0| <= kmax0 feed u and omega, so:
//   Q1  inverse FFT along axis 0 of the kept columns of u_hat
//       -> A[3][x0][c1]: u0, u1, D = F0^-1(i k0 u1)
//   Q2  per pair of x0 lines: omega = D - i k1 u0 per column, C2R of u0, u1,
//       omega (the two lines packed as z = a + i b), the products u1 omega and
//       -u0 omega in registers (optional CFL max), R2C scaled by 1 / (n0 n1)
//       -> nl[2][x0][k1]
//   Q3  forward FFT along axis 0 of both nl components, then the stage update
//       of every mode of the column (Leray, Nyquist mask, forcing, noise, L,
//       integrator); the nonlinear term never returns to HBM.
// Per stage that is 2/3 of 2U read + 3 n0 c1 written (Q1), the same read and
// 2U written (Q2), 2U + state read and written (Q3), U = n0 (n1/2+1) complex.
#include <cstdlib>

#include "pf_fft.cuh"
#include "pf_fused2d.h"
#include "pf_update.cuh"

namespace pf {

// V = 1 halves the values per thread (twice the threads per line, one more
// radix stage): these grids are too small to fill the SMs, so more threads in
// flight can beat fewer exchanges.
template <int N, typename R, int V = 0> struct Tune2 {
  static constexpr bool D = sizeof(R) == 8;
  // strided passes Q1, Q3: values per thread, threads per line, columns per CTA
  static constexpr int ES0 = D ? (N <= 8 ? N : 8) : (N <= 16 ? N : (N <= 64 ? 8 : 16));
  static constexpr int ES = ES0 >> V;
  static constexpr int GS = N / ES;
  // four columns (one 32-byte sector per FP32 row) up to 512 threads per CTA
  static constexpr int T = GS >= 512 ? 1 : (GS >= 256 ? 2 : 4);
  // Q3 holds two transformed columns and the update in registers: at most
  // 256 threads per CTA keeps the 255-register budget
  static constexpr int TU = GS >= 256 ? 1 : (GS >= 128 ? 2 : 4);
  // contiguous pass Q2: one line pair per GC threads, 256 threads per CTA
  static constexpr int EC = 8 >> V;
  static constexpr int GC = N / EC;
  static constexpr int LP = GC >= 256 ? 1 : 256 / GC;
  // exchange buffer of one line pair: +1 value per 16 (FP32) or 8 (FP64)
  static constexpr int SHP = D ? 3 : 4;
  static constexpr int BUF = N + (N >> SHP) + 1;
  static PF_HD int sw(int p) { return p + (p >> SHP); }
};

// Exchange buffer of the strided passes: position p of column t, T padding
// values after every 16 positions.
template <int T> PF_HD int colp(int p, int t) { return p * T + t + T * (p >> 4); }
template <int N, int T, typename R> constexpr size_t colp_bytes() {
  return sizeof(cx<R>) * (size_t)(N * T + T * (N >> 4));
}

// ---------------------------------------------------------------------- Q1
template <typename R, int N, int V, bool MEMB = false>
__global__ void __launch_bounds__(Tune2<N, R, V>::T * Tune2<N, R, V>::GS)
k_q1(const cx<R>* __restrict__ uh, cx<R>* __restrict__ A, F2 f, const cx<R>* __restrict__ tw) {
  using TN = Tune2<N, R, V>;
  constexpr int E = TN::ES, G = TN::GS, T = TN::T;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int t = threadIdx.x, j = threadIdx.y;
  const int q = blockIdx.x * T + t;  // kept column k1 in [0, c1)
  const bool active = q < f.c1;
  const int fld = blockIdx.y;        // 0: u0, 1: u1, 2: D
  if constexpr (MEMB) {  // member blockIdx.z of boxes laid out one after another
    uh += (long long)blockIdx.z * 2 * f.nspec;
    A += (long long)blockIdx.z * 3 * f.n0 * f.c1;
  }
  const C* src = uh + (fld == 0 ? 0 : f.nspec);
  C v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int i = j + G * e;
    const int kf = kfreq(i, N);
    C z = czero<C>();
    if (active && abs(kf) <= f.kmax0) z = src[(long long)i * f.nh + q];
    if (fld == 2) z = cmuli(cscale(z, (R)(f.ks0 * kf)));
    v[e] = z;
  }
  fft<N, E, +1>(v, j, tw, [&](int p) -> C& { return sm[colp<T>(p, t)]; },
                [] { __syncthreads(); });
  if (active) {
    C* dst = A + (long long)fld * N * f.c1 + q;
#pragma unroll
    for (int e = 0; e < E; ++e) dst[(long long)(j + G * e) * f.c1] = v[e];
  }
}

// ---------------------------------------------------------------------- Q2
template <typename R, int N, int V, bool MEMB = false>
__global__ void __launch_bounds__(Tune2<N, R, V>::GC * Tune2<N, R, V>::LP)
k_q2(const cx<R>* __restrict__ A, cx<R>* __restrict__ nl, F2 f, const cx<R>* __restrict__ tw,
     unsigned long long* __restrict__ maxbits, R scale) {
  using TN = Tune2<N, R, V>;
  constexpr int E = TN::EC, G = TN::GC, H = N / 2;
  static_assert(G > 32 || 32 % G == 0, "a line pair inside one warp, or whole warps");
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int j = threadIdx.x, lp = threadIdx.y;
  if constexpr (MEMB) {  // member blockIdx.y
    A += (long long)blockIdx.y * 3 * f.n0 * f.c1;
    nl += (long long)blockIdx.y * 2 * f.nspec;
    if (maxbits) maxbits += blockIdx.y;
  }
  const int pair = blockIdx.x * TN::LP + lp;
  const bool active = pair < (f.n0 >> 1);
  const int la = 2 * pair;
  C* ex = reinterpret_cast<C*>(smraw) + lp * TN::BUF;
  auto smf = [&](int p) -> C& { return ex[TN::sw(p)]; };
  auto sync = [] {
    if constexpr (G <= 32) __syncwarp();
    else __syncthreads();
  };
  const long long fsA = (long long)f.n0 * f.c1;
  // lines la, la + 1 of field fld as z = a + i b on the full length-N circle
  // (fld 2: omega = D - i k1 u0); DC imaginary parts dropped as a C2R does
  auto unpack = [&](int fld, C (&z)[E]) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int m = j + G * e;
      const int k = m <= H ? m : N - m;
      C a = czero<C>(), b = czero<C>();
      if (active && k < f.c1) {
        const long long o = (long long)la * f.c1 + k;
        if (fld < 2) {
          a = A[fld * fsA + o];
          b = A[fld * fsA + o + f.c1];
        } else {
          const R kk = (R)(f.ks1 * k);
          a = csub(A[2 * fsA + o], cmuli(cscale(A[o], kk)));
          b = csub(A[2 * fsA + o + f.c1], cmuli(cscale(A[o + f.c1], kk)));
        }
      }
      if (m == 0) { a.y = 0; b.y = 0; }
      C r;
      if (m <= H) { r.x = a.x - b.y; r.y = a.y + b.x; }
      else { r.x = a.x + b.y; r.y = b.x - a.y; }
      z[e] = r;
    }
  };
  C u0[E], u1[E], w[E];
  unpack(0, u0);
  fft<N, E, +1>(u0, j, tw, smf, sync);
  unpack(1, u1);
  fft<N, E, +1>(u1, j, tw, smf, sync);
  unpack(2, w);
  fft<N, E, +1>(w, j, tw, smf, sync);
  double mx = 0.0;
  if (maxbits) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      // CFL sums in the state's precision, the running maximum in FP64
      const R sa = fabs(u0[e].x) * (R)f.cflw0 + fabs(u1[e].x) * (R)f.cflw1;
      const R sb = fabs(u0[e].y) * (R)f.cflw0 + fabs(u1[e].y) * (R)f.cflw1;
      mx = fmax(mx, (double)fmax(sa, sb));
    }
  }
  // line a in the real parts, line b in the imaginary parts:
  // nl0 = u1 omega (into u1), nl1 = -u0 omega (into u0)
#pragma unroll
  for (int e = 0; e < E; ++e) {
    u1[e].x *= w[e].x;  u1[e].y *= w[e].y;
    u0[e].x = -u0[e].x * w[e].x;  u0[e].y = -u0[e].y * w[e].y;
  }
  const R h = R(0.5) * scale;
  auto store = [&](C (&c)[E], int comp) {
    fft<N, E, -1>(c, j, tw, smf, sync);
#pragma unroll
    for (int e = 0; e < E; ++e) smf(j + G * e) = c[e];
    sync();
    if (active) {
      C* oa = nl + comp * f.nspec + (long long)la * f.nh;
      C* ob = oa + f.nh;
#pragma unroll
      for (int e = 0; e <= E / 2; ++e) {
        const int k = j + G * e;
        if (k <= H) {
          const C zk = smf(k);
          const C zn = smf(k == 0 ? 0 : N - k);
          C Av, Bv;
          Av.x = (zk.x + zn.x) * h; Av.y = (zk.y - zn.y) * h;
          Bv.x = (zk.y + zn.y) * h; Bv.y = -(zk.x - zn.x) * h;
          oa[k] = Av;
          ob[k] = Bv;
        }
      }
    }
    sync();
  };
  store(u1, 0);
  store(u0, 1);
  if (maxbits) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x + blockDim.x * threadIdx.y) % 32 == 0)
      atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
  }
}

// ---------------------------------------------------------------------- Q3
template <typename R, int N, int V, int NC, bool NOISE, bool MEMB = false>
__global__ void __launch_bounds__(Tune2<N, R, V>::TU * Tune2<N, R, V>::GS)
k_q3(UpdateArgs<R> U, const cx<R>* __restrict__ nl, F2 f, const cx<R>* __restrict__ tw) {
  using TN = Tune2<N, R, V>;
  const Member mem = member_of(U, MEMB ? (int)blockIdx.y : 0);  // member blockIdx.y
  if constexpr (MEMB) nl += (long long)blockIdx.y * 2 * f.nspec;
  constexpr int E = TN::ES, G = TN::GS, T = TN::TU;
  constexpr int CH0 = sizeof(R) == 8 ? 2 : 4;  // rows per thread whose state loads are in flight
  constexpr int CH = E < CH0 ? E : CH0;
  static_assert(E % CH == 0, "whole chunks of rows");
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int t = threadIdx.x, j = threadIdx.y;
  const int q = blockIdx.x * T + t;  // column k1 in [0, nh)
  const bool active = q < f.nh;
  auto smf = [&](int p) -> C& { return sm[colp<T>(p, t)]; };
  auto sync = [] { __syncthreads(); };
  C v0[E], v1[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const long long m = (long long)(j + G * e) * f.nh + q;
    v0[e] = active ? nl[m] : czero<C>();
    v1[e] = active ? nl[f.nspec + m] : czero<C>();
  }
  fft<N, E, -1>(v0, j, tw, smf, sync);
  fft<N, E, -1>(v1, j, tw, smf, sync);
  const StageScalars<R> sc = stage_scalars<R>(U, mem.mb);
  double accE = 0.0, accZ = 0.0;
  if (active) {
    const R k1 = (R)(f.ks1 * q);
    const cx<R>* __restrict__ uh = U.uhat + mem.mo;
    cx<R>* __restrict__ uo = (U.uout ? U.uout : U.uhat) + mem.mo;  // new state
    cx<R>* __restrict__ u0p = U.u0 + mem.mo;
    const long long ns = f.nspec;
#pragma unroll
    for (int e0 = 0; e0 < E; e0 += CH) {
      C un[CH][2], u0v[CH][2];
#pragma unroll
      for (int cc = 0; cc < CH; ++cc) {
        const long long m = (long long)(j + G * (e0 + cc)) * f.nh + q;
#pragma unroll
        for (int a = 0; a < 2; ++a) {
          un[cc][a] = uh[a * ns + m];
          u0v[cc][a] = U.save_u0 ? un[cc][a] : u0p[a * ns + m];
        }
      }
#pragma unroll
      for (int cc = 0; cc < CH; ++cc) {
        const int i0 = j + G * (e0 + cc);
        const long long m = (long long)i0 * f.nh + q;
        ModeK<R, 2> mk_;
        mk_.ix.i0 = i0; mk_.ix.i1 = q; mk_.ix.i2 = 0;
        const R k0 = (R)(f.ks0 * kfreq(i0, f.n0));
        mk_.k[0] = k0; mk_.k[1] = k1;
        mk_.k2 = k0 * k0 + k1 * k1;
        C nv[2] = {v0[e0 + cc], v1[e0 + cc]};
        update_core<R, 2, NC, NOISE>(U, m, mk_, nv, true, un[cc], u0v[cc], sc, accE, accZ, uo, u0p,
                                     mem.mb);
      }
    }
  }
  if (U.diag) block_add2(accE, accZ, U.diag + 2 * mem.mb);
}

// ------------------------------------------------------------------ host side
bool fused2d_side(int n) { return n >= 16 && n <= 1024 && (n & (n - 1)) == 0; }

F2 fused2d_geo(const Geo& g) {
  F2 f;
  f.n0 = g.n[0]; f.n1 = g.n[1]; f.nh = g.nh;
  f.kmax0 = g.kmax[0]; f.kmax1 = g.kmax[1];
  f.c1 = g.kmax[1] + 1;
  f.nspec = g.nspec;
  f.ks0 = g.kscale[0]; f.ks1 = g.kscale[1];
  f.cflw0 = g.n[0] * g.kscale[0] / (2.0 * M_PI);
  f.cflw1 = g.n[1] * g.kscale[1] / (2.0 * M_PI);
  f.nmem = 1;
  // measured on B200 (RK3, FP32 and FP64): the halved radix is faster at
  // sides 256 and 512 (256^2 FP32 43 vs 60 us per step), slower at 1024
  f.var[0] = 0;
  f.var[1] = f.var[3] = f.n0 <= 512 ? 1 : 0;  // Q1, Q3 transform along axis 0
  f.var[2] = f.n1 <= 512 ? 1 : 0;             // Q2 along axis 1
  if (const char* v = getenv("PF_FUSED2D_VARIANT")) {
    // "q1:1,q2:1,q3:1"
    for (const char* c = v; *c; ++c)
      if (c[0] == 'q' && c[1] >= '1' && c[1] <= '3' && c[2] == ':') f.var[c[1] - '0'] = atoi(c + 3);
  }
  return f;
}

size_t fused2d_scratch_elems(const F2& f) { return 3ull * f.n0 * f.c1; }

template <typename K> static cudaError_t smem_limit(K kern, size_t bytes) {
  if (bytes + 1024 > 48 * 1024)
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

#define PF_SWITCH_2D(n, CALL)     \
  switch (n) {                    \
    case 16: return CALL(16);     \
    case 32: return CALL(32);     \
    case 64: return CALL(64);     \
    case 128: return CALL(128);   \
    case 256: return CALL(256);   \
    case 512: return CALL(512);   \
    case 1024: return CALL(1024); \
    default: return cudaErrorInvalidValue; \
  }

template <typename R, int N, int V>
static cudaError_t q1_run(const F2& f, const cx<R>* uh, cx<R>* A, cudaStream_t st) {
  using TN = Tune2<N, R, V>;
  const size_t sm = colp_bytes<N, TN::T, R>();
  const dim3 grid((unsigned)((f.c1 + TN::T - 1) / TN::T), 3, (unsigned)f.nmem);
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  cudaError_t e;
  if (f.nmem > 1) {
    e = smem_limit(k_q1<R, N, V, true>, sm);
    if (e != cudaSuccess) return e;
    k_q1<R, N, V, true><<<grid, dim3(TN::T, TN::GS), sm, st>>>(uh, A, f, tw);
  } else {
    e = smem_limit(k_q1<R, N, V>, sm);
    if (e != cudaSuccess) return e;
    k_q1<R, N, V><<<grid, dim3(TN::T, TN::GS), sm, st>>>(uh, A, f, tw);
  }
  return launched();
}

template <typename R, int N, int V>
static cudaError_t q2_run(const F2& f, const cx<R>* A, cx<R>* nl, unsigned long long* maxbits,
                          cudaStream_t st) {
  using TN = Tune2<N, R, V>;
  const size_t sm = sizeof(cx<R>) * (size_t)TN::LP * TN::BUF;
  const int npairs = f.n0 / 2;
  const dim3 grid((unsigned)((npairs + TN::LP - 1) / TN::LP), (unsigned)f.nmem);
  const R scale = (R)(1.0 / ((double)f.n0 * (double)f.n1));
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  cudaError_t e;
  if (f.nmem > 1) {
    e = smem_limit(k_q2<R, N, V, true>, sm);
    if (e != cudaSuccess) return e;
    k_q2<R, N, V, true><<<grid, dim3(TN::GC, TN::LP), sm, st>>>(A, nl, f, tw, maxbits, scale);
  } else {
    e = smem_limit(k_q2<R, N, V>, sm);
    if (e != cudaSuccess) return e;
    k_q2<R, N, V><<<grid, dim3(TN::GC, TN::LP), sm, st>>>(A, nl, f, tw, maxbits, scale);
  }
  return launched();
}

// the single-box or the member form of Q3
template <typename R, int N, int V, int NC, bool NOISE>
static cudaError_t q3_go(const F2& f, const UpdateArgs<R>& U, const cx<R>* nl, dim3 grid,
                         dim3 block, size_t sm, const cx<R>* tw, cudaStream_t st) {
  cudaError_t e;
  if (f.nmem > 1) {
    e = smem_limit(k_q3<R, N, V, NC, NOISE, true>, sm);
    if (e != cudaSuccess) return e;
    k_q3<R, N, V, NC, NOISE, true><<<grid, block, sm, st>>>(U, nl, f, tw);
  } else {
    e = smem_limit(k_q3<R, N, V, NC, NOISE>, sm);
    if (e != cudaSuccess) return e;
    k_q3<R, N, V, NC, NOISE><<<grid, block, sm, st>>>(U, nl, f, tw);
  }
  return cudaSuccess;
}

template <typename R, int N, int V>
static cudaError_t q3_run(const F2& f, const UpdateArgs<R>& U, int ncomp, const cx<R>* nl,
                          cudaStream_t st) {
  using TN = Tune2<N, R, V>;
  const size_t sm = colp_bytes<N, TN::TU, R>();
  const dim3 grid((unsigned)((f.nh + TN::TU - 1) / TN::TU), (unsigned)f.nmem),
      block(TN::TU, TN::GS);
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  cudaError_t e;
  if (U.noise_src == kNoiseNone) e = q3_go<R, N, V, 2, false>(f, U, nl, grid, block, sm, tw, st);
  else if (ncomp == 4) e = q3_go<R, N, V, 4, true>(f, U, nl, grid, block, sm, tw, st);
  else e = q3_go<R, N, V, 2, true>(f, U, nl, grid, block, sm, tw, st);
  return e != cudaSuccess ? e : launched();
}

// Variant v of a pass at side N: the halved-radix form exists for N >= 256.
#define PF_Q_VAR(RUN, NN, V, ...) \
  (((NN) >= 256 && (V) == 1) ? RUN<R, NN, ((NN) >= 256 ? 1 : 0)>(__VA_ARGS__) \
                             : RUN<R, NN, 0>(__VA_ARGS__))

template <typename R>
cudaError_t fused2d_inverse(const F2& f, const cx<R>* uhat, cx<R>* A, cudaStream_t st) {
  if (!tw_base<R>()) return cudaErrorNotReady;
#define PF_CALL(NN) PF_Q_VAR(q1_run, NN, f.var[1], f, uhat, A, st)
  PF_SWITCH_2D(f.n0, PF_CALL)
#undef PF_CALL
}

template <typename R>
cudaError_t fused2d_products(const F2& f, const cx<R>* A, cx<R>* nl,
                             unsigned long long* maxbits, cudaStream_t st) {
  if (!tw_base<R>()) return cudaErrorNotReady;
#define PF_CALL(NN) PF_Q_VAR(q2_run, NN, f.var[2], f, A, nl, maxbits, st)
  PF_SWITCH_2D(f.n1, PF_CALL)
#undef PF_CALL
}

template <typename R>
cudaError_t fused2d_update(const F2& f, const UpdateArgs<R>& U, int ncomp, const cx<R>* nl,
                           cudaStream_t st) {
  if (!tw_base<R>()) return cudaErrorNotReady;
#define PF_CALL(NN) PF_Q_VAR(q3_run, NN, f.var[3], f, U, ncomp, nl, st)
  PF_SWITCH_2D(f.n0, PF_CALL)
#undef PF_CALL
}

template cudaError_t fused2d_inverse<float>(const F2&, const float2*, float2*, cudaStream_t);
template cudaError_t fused2d_inverse<double>(const F2&, const double2*, double2*, cudaStream_t);
template cudaError_t fused2d_products<float>(const F2&, const float2*, float2*,
                                             unsigned long long*, cudaStream_t);
template cudaError_t fused2d_products<double>(const F2&, const double2*, double2*,
                                              unsigned long long*, cudaStream_t);
template cudaError_t fused2d_update<float>(const F2&, const UpdateArgs<float>&, int,
                                           const float2*, cudaStream_t);
template cudaError_t fused2d_update<double>(const F2&, const UpdateArgs<double>&, int,
                                            const double2*, cudaStream_t);

}  // namespace pf
