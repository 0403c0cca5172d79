// Generic axis passes of the 2D/3D real FFTs (used by forward()/backward(),
// initialisation, output and the per-operator right-hand side):
//   * k_fft_strided : in-place C2C along a strided axis, one CTA per tile of
//                     T consecutive columns (coalesced rows of T complex);
//   * k_c2r_last    : C2R along the contiguous axis, two lines per complex
//                     FFT (z = a + i b);
//   * k_r2c_last    : R2C along the contiguous axis, two lines per complex FFT,
//                     split with A_k = (Z_k + conj Z_{N-k}) / 2,
//                     B_k = (Z_k - conj Z_{N-k}) / 2i.
#include "pf_fft.cuh"
#include "pf_internal.h"

namespace pf {

template <int N> struct Tune {
  // powers of two: 8 or 16 values per thread; 3 * 2^b: 12 or 24 (a radix-3
  // stage needs E divisible by 3)
  static constexpr int E = (N % 3 == 0) ? (N <= 24 ? N : (N <= 96 ? 12 : 24))
                                        : (N <= 16 ? N : (N <= 64 ? 8 : 16));
  static constexpr int G = N / E;
  static constexpr int T = (256 / G) < 4 ? 4 : ((256 / G) > 64 ? 64 : 256 / G);
  static constexpr int L = (128 / G) < 1 ? 1 : 128 / G;  // line pairs per CTA
};

template <typename R> struct Pad { static constexpr int shift = 4; };
template <> struct Pad<double> { static constexpr int shift = 3; };

template <typename R, int N, int DIR>
__global__ void __launch_bounds__(Tune<N>::T * Tune<N>::G)
k_fft_strided(cx<R>* __restrict__ data, long long ncols, long long ntotal,
              long long plane_stride, long long line_stride, R scale, int use_scale,
              const cx<R>* __restrict__ tw) {
  constexpr int E = Tune<N>::E, G = Tune<N>::G, T = Tune<N>::T;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int t = threadIdx.x, j = threadIdx.y;
  const long long q = (long long)blockIdx.x * T + t;
  const bool active = q < ntotal;
  long long base = 0;
  if (active) {
    const long long p = q / ncols;
    base = p * plane_stride + (q - p * ncols);
  }
  C v[E];
#pragma unroll
  for (int e = 0; e < E; ++e)
    v[e] = active ? data[base + (long long)(j + G * e) * line_stride] : czero<C>();
  fft<N, E, DIR, false>(v, j, tw, [&](int pos) -> C& { return sm[pos * T + t]; },
                 [] { __syncthreads(); });
  if (active) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      C z = use_scale ? cscale(v[e], scale) : v[e];
      data[base + (long long)(j + G * e) * line_stride] = z;
    }
  }
}

template <typename R, int N>
__global__ void __launch_bounds__(Tune<N>::L * Tune<N>::G)
k_c2r_last(const cx<R>* __restrict__ in, R* __restrict__ out, long long nlines,
           long long in_stride, long long out_stride, const cx<R>* __restrict__ tw) {
  constexpr int E = Tune<N>::E, G = Tune<N>::G, L = Tune<N>::L;
  constexpr int H = N / 2;
  constexpr int SH = Pad<R>::shift;
  constexpr int BUF = N + (N >> SH) + 1;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw) + threadIdx.y * BUF;
  const int j = threadIdx.x;
  const long long pair = (long long)blockIdx.x * L + threadIdx.y;
  const long long la = 2 * pair, lb = la + 1;
  const bool hasA = la < nlines, hasB = lb < nlines;
  const C* A = in + la * in_stride;
  const C* B = in + lb * in_stride;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int m = j + G * e;
    const int k = m <= H ? m : N - m;
    C a = hasA ? A[k] : czero<C>();
    C b = hasB ? B[k] : czero<C>();
    if (m == 0 || m == H) { a.y = 0; b.y = 0; }
    C z;
    if (m <= H) { z.x = a.x - b.y; z.y = a.y + b.x; }
    else { z.x = a.x + b.y; z.y = b.x - a.y; }
    v[e] = z;
  }
  auto smf = [&](int pos) -> C& { return sm[pos + (pos >> SH)]; };
  if constexpr (G <= 32) fft<N, E, +1, false>(v, j, tw, smf, [] { __syncwarp(); });
  else fft<N, E, +1, false>(v, j, tw, smf, [] { __syncthreads(); });
  R* oa = out + la * out_stride;
  R* ob = out + lb * out_stride;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = j + G * e;
    if (hasA) oa[n] = v[e].x;
    if (hasB) ob[n] = v[e].y;
  }
}

template <typename R, int N>
__global__ void __launch_bounds__(Tune<N>::L * Tune<N>::G)
k_r2c_last(const R* __restrict__ in, cx<R>* __restrict__ out, long long nlines,
           long long in_stride, long long out_stride, R scale, const cx<R>* __restrict__ tw) {
  constexpr int E = Tune<N>::E, G = Tune<N>::G, L = Tune<N>::L;
  constexpr int H = N / 2;
  constexpr int SH = Pad<R>::shift;
  constexpr int BUF = N + (N >> SH) + 1;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw) + threadIdx.y * BUF;
  const int j = threadIdx.x;
  const long long pair = (long long)blockIdx.x * L + threadIdx.y;
  const long long la = 2 * pair, lb = la + 1;
  const bool hasA = la < nlines, hasB = lb < nlines;
  const R* a = in + la * in_stride;
  const R* b = in + lb * in_stride;
  C v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int n = j + G * e;
    v[e].x = hasA ? a[n] : R(0);
    v[e].y = hasB ? b[n] : R(0);
  }
  auto smf = [&](int pos) -> C& { return sm[pos + (pos >> SH)]; };
  auto sync = [] { if constexpr (G <= 32) __syncwarp(); else __syncthreads(); };
  fft<N, E, -1, false>(v, j, tw, smf, sync);
#pragma unroll
  for (int e = 0; e < E; ++e) smf(j + G * e) = v[e];
  sync();
  C* oa = out + la * out_stride;
  C* ob = out + lb * out_stride;
  const R h = R(0.5) * scale;
#pragma unroll
  for (int e = 0; e <= E / 2; ++e) {
    const int k = j + G * e;
    if (k <= H) {
      const C zk = smf(k);
      const C zn = smf(k == 0 ? 0 : N - k);
      C A, Bv;
      A.x = (zk.x + zn.x) * h; A.y = (zk.y - zn.y) * h;
      // (zk - conj zn) / 2i
      Bv.x = (zk.y + zn.y) * h; Bv.y = -(zk.x - zn.x) * h;
      if (hasA) oa[k] = A;
      if (hasB) ob[k] = Bv;
    }
  }
}

// ------------------------------------------------------------------ launchers
template <typename K> static cudaError_t set_smem(K kern, size_t bytes) {
  if (bytes > 48 * 1024)
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

template <typename R, int N>
static cudaError_t launch_strided(cx<R>* data, int dir, long long ncols, long long nplanes,
                                  long long ps, long long ls, double scale, cudaStream_t st) {
  using TN = Tune<N>;
  const cx<R>* twb = tw_base<R>();
  if (!twb) return cudaErrorNotReady;  // tables not built on this device
  const cx<R>* tw = twb + tw_offset(N);
  const long long ntotal = ncols * nplanes;
  if (ntotal == 0) return cudaSuccess;
  dim3 block(TN::T, TN::G);
  dim3 grid((unsigned)((ntotal + TN::T - 1) / TN::T));
  // exchange buffer whenever the plan has more than one stage (a 3 * 2^b
  // length with one thread per line still exchanges between its stages)
  size_t sm = Plan<N, TN::E, false>::stages() > 1 ? sizeof(cx<R>) * N * TN::T : 0;
  const int us = scale != 1.0;
  cudaError_t e;
  if (dir < 0) {
    e = set_smem(k_fft_strided<R, N, -1>, sm);
    if (e != cudaSuccess) return e;
    k_fft_strided<R, N, -1><<<grid, block, sm, st>>>(data, ncols, ntotal, ps, ls, (R)scale, us, tw);
  } else {
    e = set_smem(k_fft_strided<R, N, +1>, sm);
    if (e != cudaSuccess) return e;
    k_fft_strided<R, N, +1><<<grid, block, sm, st>>>(data, ncols, ntotal, ps, ls, (R)scale, us, tw);
  }
  return launched();
}

template <typename R, int N>
static cudaError_t launch_c2r(const cx<R>* in, R* out, long long nlines, long long is,
                              long long os, cudaStream_t st) {
  using TN = Tune<N>;
  const cx<R>* twb = tw_base<R>();
  if (!twb) return cudaErrorNotReady;  // tables not built on this device
  const cx<R>* tw = twb + tw_offset(N);
  const long long npairs = (nlines + 1) / 2;
  if (npairs == 0) return cudaSuccess;
  dim3 block(TN::G, TN::L);
  dim3 grid((unsigned)((npairs + TN::L - 1) / TN::L));
  size_t sm = sizeof(cx<R>) * TN::L * (N + (N >> Pad<R>::shift) + 1);
  cudaError_t e = set_smem(k_c2r_last<R, N>, sm);
  if (e != cudaSuccess) return e;
  k_c2r_last<R, N><<<grid, block, sm, st>>>(in, out, nlines, is, os, tw);
  return launched();
}

template <typename R, int N>
static cudaError_t launch_r2c(const R* in, cx<R>* out, long long nlines, long long is,
                              long long os, double scale, cudaStream_t st) {
  using TN = Tune<N>;
  const cx<R>* twb = tw_base<R>();
  if (!twb) return cudaErrorNotReady;  // tables not built on this device
  const cx<R>* tw = twb + tw_offset(N);
  const long long npairs = (nlines + 1) / 2;
  if (npairs == 0) return cudaSuccess;
  dim3 block(TN::G, TN::L);
  dim3 grid((unsigned)((npairs + TN::L - 1) / TN::L));
  size_t sm = sizeof(cx<R>) * TN::L * (N + (N >> Pad<R>::shift) + 1);
  cudaError_t e = set_smem(k_r2c_last<R, N>, sm);
  if (e != cudaSuccess) return e;
  k_r2c_last<R, N><<<grid, block, sm, st>>>(in, out, nlines, is, os, (R)scale, tw);
  return launched();
}

bool fft_length_supported(int n) {
  if (n >= 4 && n <= kMaxFFT && (n & (n - 1)) == 0) return true;
  if (n % 3 != 0) return false;
  const int m = n / 3;  // 3 * 2^b, 12..768
  return n >= 12 && n <= kMax3FFT && (m & (m - 1)) == 0;
}

#define PF_SWITCH_N(n, CALL)                     \
  switch (n) {                                   \
    case 4: return CALL(4);                      \
    case 8: return CALL(8);                      \
    case 16: return CALL(16);                    \
    case 32: return CALL(32);                    \
    case 64: return CALL(64);                    \
    case 128: return CALL(128);                  \
    case 256: return CALL(256);                  \
    case 512: return CALL(512);                  \
    case 1024: return CALL(1024);                \
    case 12: return CALL(12);                    \
    case 24: return CALL(24);                    \
    case 48: return CALL(48);                    \
    case 96: return CALL(96);                    \
    case 192: return CALL(192);                  \
    case 384: return CALL(384);                  \
    case 768: return CALL(768);                  \
    default: return cudaErrorInvalidValue;       \
  }

template <typename R>
cudaError_t fft_strided(cx<R>* data, int n, int dir, long long ncols, long long nplanes,
                        long long plane_stride, long long line_stride, double scale,
                        cudaStream_t st) {
#define PF_CALL(NN) launch_strided<R, NN>(data, dir, ncols, nplanes, plane_stride, line_stride, scale, st)
  PF_SWITCH_N(n, PF_CALL)
#undef PF_CALL
}

template <typename R>
cudaError_t fft_c2r_last(const cx<R>* in, R* out, int n, long long nlines, long long in_stride,
                         long long out_stride, cudaStream_t st) {
#define PF_CALL(NN) launch_c2r<R, NN>(in, out, nlines, in_stride, out_stride, st)
  PF_SWITCH_N(n, PF_CALL)
#undef PF_CALL
}

template <typename R>
cudaError_t fft_r2c_last(const R* in, cx<R>* out, int n, long long nlines, long long in_stride,
                         long long out_stride, double scale, cudaStream_t st) {
#define PF_CALL(NN) launch_r2c<R, NN>(in, out, nlines, in_stride, out_stride, scale, st)
  PF_SWITCH_N(n, PF_CALL)
#undef PF_CALL
}

template cudaError_t fft_strided<float>(float2*, int, int, long long, long long, long long,
                                        long long, double, cudaStream_t);
template cudaError_t fft_strided<double>(double2*, int, int, long long, long long, long long,
                                         long long, double, cudaStream_t);
template cudaError_t fft_c2r_last<float>(const float2*, float*, int, long long, long long,
                                         long long, cudaStream_t);
template cudaError_t fft_c2r_last<double>(const double2*, double*, int, long long, long long,
                                          long long, cudaStream_t);
template cudaError_t fft_r2c_last<float>(const float*, float2*, int, long long, long long,
                                         long long, double, cudaStream_t);
template cudaError_t fft_r2c_last<double>(const double*, double2*, int, long long, long long,
                                          long long, double, cudaStream_t);

}  // namespace pf
