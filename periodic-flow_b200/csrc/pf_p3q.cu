// P3 of the fused 2/3-rule schedule (FP32, contiguous sides 128 and 256)
// with one shared-memory exchange per line FFT.
//
// A pair of (x0, x1) lines is packed as z = a + i b and owned by G = N / 16
// lanes holding sixteen values each (lane j: positions j + G e).  A line FFT
// is two Stockham stages: radix 16 on the lane's own values, one exchange
// through shared memory, then radix G with twiddles W_N^(r jv) that depend
// only on the lane -- computed once per kernel and kept in registers, so the
// loop loads no twiddles.  Against the eight-value form (k_p3 in
// pf_fused.cu: three stages, two exchanges, table twiddles) this halves the
// exchange traffic of the nine line FFTs of a pair, the part of P3 that
// shared-memory bandwidth bounds.
//
// Per group of PW line pairs (one warp): the six input fields arrive by one
// bulk copy per field into the warp's staging buffer (mbarrier, bounded
// wait), refilled for the next group as soon as the last field is read; u
// goes to lane-private shared slots after its C2R and omega is transformed
// one field at a time, accumulating u x omega in registers; the three R2C
// outputs are split into the two lines' spectra.  The split pairs value k
// with N - k, which lane G - j of the same pair holds, so it is fetched by
// warp shuffles instead of a shared-memory round trip.  CFL sums are FP32;
// the maximum leaves as FP64 bits (atomicMax on the bit pattern).
#include "pf_fft.cuh"
#include "pf_fgeo.h"
#include "pf_internal.h"
#include "pf_tma.cuh"

namespace pf {

template <int N> struct TuneQ {
  static_assert(N == 128 || N == 256, "sides 128 and 256");
  static constexpr int E = 16;
  static constexpr int G = N / E;      // lanes per line pair: 16 (256) or 8 (128)
  static constexpr int PW = 32 / G;    // line pairs per warp
  static constexpr int R1 = G;         // radix of the second stage
  static constexpr int Q1 = E / R1;    // its butterflies per lane
  static constexpr int BUF = N + 8;    // exchange buffer of a pair (complex values)
  static constexpr int UST = 3 * N + 8;  // u slots of a pair
  // Exchange position p lives at p ^ ((p >> 4) & 15): the radix-16 stores
  // (positions 16 j + r) and the strided loads (j + G e) of one pair fall on
  // distinct banks; the +8 pads give neighbouring pairs (N = 128) the other
  // half of the banks.
  static PF_HD int sw(int p) { return p ^ ((p >> 4) & 15); }
  static constexpr int warp_complex(int c2) {
    return (6 * 2 * PW * c2 + PW * BUF + PW * UST + 15) & ~15;
  }
};

template <int N> using TwQ = float2[TuneQ<N>::Q1][TuneQ<N>::R1 - 1];

// Line FFT of the pair whose exchange buffer is ex (DIR +1 inverse, -1
// forward); input and output in natural order, position j + G e in v[e].
template <int N, int DIR>
PF_D void fft_q(float2 (&v)[16], int j, const TwQ<N>& tq, float2* ex) {
  using T = TuneQ<N>;
  constexpr int E = T::E, G = T::G, R1 = T::R1, Q1 = T::Q1;
  // stage 1: radix 16 over the lane's own positions j + G r (Ns = 1), output
  // position 16 j + r
  dft16<DIR>(v);
#pragma unroll
  for (int r = 0; r < E; ++r) ex[T::sw(E * j + r)] = v[r];
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = ex[T::sw(j + G * e)];
  __syncwarp();
  // stage 2: radix R1 (Ns = 16), butterfly q reads positions jv + r N / R1,
  // jv = j + q G, twiddled by W_N^(r jv); output position jv + 16 r, i.e.
  // j + G e for e = q + r Q1: natural order in the lane's own registers
#pragma unroll
  for (int q = 0; q < Q1; ++q) {
    float2 b[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) b[r] = v[q + r * Q1];
#pragma unroll
    for (int r = 1; r < R1; ++r) {
      float2 w = tq[q][r - 1];
      if (DIR > 0) w.y = -w.y;
      b[r] = cmul(b[r], w);
    }
    dft<R1, DIR>(b);
#pragma unroll
    for (int r = 0; r < R1; ++r) v[q + r * Q1] = b[r];
  }
}

template <int N, int W>
__global__ void __launch_bounds__(32 * W, 1)
k_p3q(const float2* __restrict__ B, float2* __restrict__ nl, FGeo f,
      const float2* __restrict__ tw, unsigned long long* __restrict__ maxbits, float scale,
      int* __restrict__ err, long long ngroups) {
  using T = TuneQ<N>;
  constexpr int E = T::E, G = T::G, PW = T::PW, R1 = T::R1, Q1 = T::Q1;
  constexpr int H = N / 2;
  static_assert(W <= 16, "mbarriers fit the 128-byte header");
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pw = lane / G, j = lane % G;
  const int fb = 2 * PW * f.c2;  // complex values of one field of a group
  const int SC = 6 * fb;
  const int WC = T::warp_complex(f.c2);
  const uint32_t fbytes = (uint32_t)(fb * sizeof(float2));
  const long long fs_in = (long long)f.n0 * f.n1 * f.c2;
  const long long gpm = (long long)f.n0 * f.n1 / (2 * PW);  // groups per member
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw) + warp;
  float2* wbase = reinterpret_cast<float2*>(smraw + 128) + (long long)warp * WC;
  float2* ex = wbase + SC + pw * T::BUF;
  float2* ur = wbase + SC + PW * T::BUF + pw * T::UST;  // u of this pair, lane-private slots
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  TwQ<N> tq;
#pragma unroll
  for (int q = 0; q < Q1; ++q)
#pragma unroll
    for (int r = 1; r < R1; ++r) tq[q][r - 1] = __ldg(tw + r * (j + q * G));
  auto issue = [&](long long grp) {
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(bar, 6 * fbytes);
      const long long mem = grp / gpm;  // member of the group
      const float2* src = B + mem * 6 * fs_in + (grp - mem * gpm) * fb;
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) bulk_g2s(wbase + fld * fb, src + fld * fs_in, fbytes, bar);
    }
  };
  // two adjacent half-spectrum lines a, b of one field packed as z = a + i b
  // on the full length-N circle (DC imaginary parts dropped)
  auto unpack = [&](const float2* pa, float2 (&z)[E]) {
    const float2* pb = pa + f.c2;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int m = j + G * e;
      const int k = m <= H ? m : N - m;
      const bool kin = k < f.c2;
      float2 a = kin ? pa[k] : make_float2(0.f, 0.f);
      float2 b = kin ? pb[k] : make_float2(0.f, 0.f);
      if (m == 0) { a.y = 0.f; b.y = 0.f; }
      float2 r;
      if (m <= H) { r.x = a.x - b.y; r.y = a.y + b.x; }
      else { r.x = a.x + b.y; r.y = b.x - a.y; }
      z[e] = r;
    }
  };
  const float cw0 = (float)f.cflw0, cw1 = (float)f.cflw1, cw2 = (float)f.cflw2;
  const float h = 0.5f * scale;
  // lane of this pair holding position N - k for k = j + G e (j > 0)
  const int mirror = (lane & ~(G - 1)) | ((G - j) & (G - 1));
  const long long TW = (long long)gridDim.x * W;
  long long g = (long long)blockIdx.x * W + warp;
  if (g < ngroups) issue(g);
  float mx = 0.f;
  long long curm = -1;  // member whose CFL maximum mx holds
  // warp maximum into member m's slot as FP64 bits
  auto flush = [&](long long m) {
    double d = (double)mx;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    if (lane == 0) atomicMax(maxbits + m, (unsigned long long)__double_as_longlong(d));
    mx = 0.f;
  };
  for (int it = 0; g < ngroups; g += TW, ++it) {
    const long long mem = g / gpm;
    if (maxbits && mem != curm) {
      if (curm >= 0) flush(curm);
      curm = mem;
    }
    const bool more = g + TW < ngroups;
    const bool ok = mbar_wait_bounded(bar, (uint32_t)(it & 1));
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(err, kErrWaitP3);
      return;
    }
    const float2* in = wbase + 2 * pw * f.c2;
    float2 v[E];
#pragma unroll
    for (int fld = 0; fld < 3; ++fld) {
      unpack(in + fld * fb, v);
      fft_q<N, +1>(v, j, tq, ex);
#pragma unroll
      for (int e = 0; e < E; ++e) ur[fld * N + j + G * e] = v[e];
    }
    if (maxbits) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 u0 = ur[j + G * e], u1 = ur[N + j + G * e], u2 = ur[2 * N + j + G * e];
        const float sa = fabsf(u0.x) * cw0 + fabsf(u1.x) * cw1 + fabsf(u2.x) * cw2;
        const float sb = fabsf(u0.y) * cw0 + fabsf(u1.y) * cw1 + fabsf(u2.y) * cw2;
        mx = fmaxf(mx, fmaxf(sa, sb));
      }
    }
    float2 c[3][E];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int e = 0; e < E; ++e) c[i][e] = make_float2(0.f, 0.f);
#pragma unroll
    for (int wc = 0; wc < 3; ++wc) {
      unpack(in + (3 + wc) * fb, v);
      if (wc == 2) {
        __syncwarp();  // every lane has read the group: the buffer takes the next one
        if (more) issue(g + TW);
      }
      fft_q<N, +1>(v, j, tq, ex);
      // c0 = u1 w2 - u2 w1, c1 = u2 w0 - u0 w2, c2 = u0 w1 - u1 w0 (math.py:4-28):
      // field wc adds u[wc+2] w to c[wc+1] and subtracts u[wc+1] w from c[wc+2];
      // real parts are line a, imaginary parts line b
      const int ia = (wc + 1) % 3, ib = (wc + 2) % 3;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float2 ua = ur[ia * N + j + G * e], ub = ur[ib * N + j + G * e];
        c[ia][e].x += ub.x * v[e].x;  c[ia][e].y += ub.y * v[e].y;
        c[ib][e].x -= ua.x * v[e].x;  c[ib][e].y -= ua.y * v[e].y;
      }
    }
    const long long la = 2 * ((g - mem * gpm) * PW + pw);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      fft_q<N, -1>(c[i], j, tq, ex);
      float2* oa = nl + (mem * 3 + i) * f.nlcomp + la * f.nh;
      float2* ob = oa + f.nh;
#pragma unroll
      for (int e = 0; e <= E / 2; ++e) {
        // N - k = (G - j) + G (E - 1 - e) for j > 0 (lane `mirror`), G (E - e) for j = 0
        float2 zn;
        zn.x = __shfl_sync(0xffffffffu, c[i][E - 1 - e].x, mirror);
        zn.y = __shfl_sync(0xffffffffu, c[i][E - 1 - e].y, mirror);
        if (j == 0) zn = c[i][(E - e) & (E - 1)];
        const float2 zk = c[i][e];
        const int k = j + G * e;
        if (k <= H) {
          float2 Av, Bv;
          Av.x = (zk.x + zn.x) * h; Av.y = (zk.y - zn.y) * h;
          Bv.x = (zk.y + zn.y) * h; Bv.y = -(zk.x - zn.x) * h;
          oa[k] = Av;
          ob[k] = Bv;
        }
      }
    }
  }
  if (maxbits && curm >= 0) flush(curm);
}

template <int N, int W>
static size_t p3q_smem(int c2) {
  return 128 + sizeof(float2) * (size_t)W * TuneQ<N>::warp_complex(c2);
}

template <int N, int W>
static cudaError_t p3q_run(const float2* B, float2* nl, const FGeo& f, const float2* tw,
                           unsigned long long* maxbits, float scale, int* err, long long ngroups,
                           int nsm, cudaStream_t st) {
  const size_t sm = p3q_smem<N, W>(f.c2);
  if (sm > 227 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_p3q<N, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sm);
  if (e != cudaSuccess) return e;
  long long blocks = (ngroups + W - 1) / W;
  if (blocks > nsm) blocks = nsm;
  k_p3q<N, W><<<(unsigned)blocks, 32 * W, sm, st>>>(B, nl, f, tw, maxbits, scale, err, ngroups);
  return launched();
}

bool p3q_supported(int n2, int W) {
  const int c2 = (n2 - 1) / 3 + 1;
  if (n2 == 256) return (W == 6 && p3q_smem<256, 6>(c2) <= 227 * 1024) ||
                        (W == 7 && p3q_smem<256, 7>(c2) <= 227 * 1024);
  if (n2 == 128) return W == 6 && p3q_smem<128, 6>(c2) <= 227 * 1024;
  return false;
}

cudaError_t p3q_launch(int n2, int W, const float2* B, float2* nl, const FGeo& f,
                       const float2* tw, unsigned long long* maxbits, float scale, int* err,
                       long long ngroups, int nsm, cudaStream_t st) {
  if (n2 != f.n2 || f.c2 != f.kmax2 + 1 || !p3q_supported(n2, W)) return cudaErrorInvalidValue;
  if (n2 == 256)
    return W == 6 ? p3q_run<256, 6>(B, nl, f, tw, maxbits, scale, err, ngroups, nsm, st)
                  : p3q_run<256, 7>(B, nl, f, tw, maxbits, scale, err, ngroups, nsm, st);
  return p3q_run<128, 6>(B, nl, f, tw, maxbits, scale, err, ngroups, nsm, st);
}

}  // namespace pf
