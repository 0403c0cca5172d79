// Register-resident Stockham FFT engine (lengths 2^b and 3 * 2^b).
//
// A line of N complex values is owned by G = N / E threads; thread j holds
// x[j + G*e] for e in [0, E) ("natural strided" mapping).  Each radix-R stage
// is the Stockham autosort iteration of Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors" (SC'08): butterfly jv
// reads positions jv + r*N/R, twiddles by W_{Ns R}^{r (jv mod Ns)}, does a
// radix-R DFT and writes positions (jv/Ns)*Ns*R + jv mod Ns + r*Ns.  With the
// natural strided mapping the reads of every stage are the thread's own
// registers, and the writes of the last stage land on the thread's own
// positions again, so an S-stage transform costs S-1 exchanges through shared
// memory and both input and output are in natural order.  For contiguous
// lines that mapping is also the coalesced one; for strided lines consecutive
// threads own consecutive columns.
#pragma once
#include "pf_common.cuh"

namespace pf {

// ---- twiddle tables ---------------------------------------------------------
// A table for length N holds exp(-2 pi i m / N), m in [0, N), rounded from
// FP64; kernels receive its device address (tables live in pf_tables.cu).
// Lengths with tables: 2^b (2..1024) and 3 * 2^b (12..768).
constexpr int kMaxFFT = 1024;
constexpr int kMax3FFT = 768;
constexpr int kTwPow2 = 2 * kMaxFFT - 2;        // sum of 2^b tables
constexpr int kTwSize = kTwPow2 + 2 * kMax3FFT - 12;
// offset of the table of length n (2^b: n - 2; 12 * 2^m: kTwPow2 + n - 12)
PF_HD int tw_offset(int n) { return (n % 3 == 0) ? kTwPow2 + n - 12 : n - 2; }

template <typename C> PF_D C ldtw(const C* p) { return __ldg(p); }

// ---- small DFTs in registers (DIR = -1 forward, +1 inverse) -----------------
// multiply by the 16th root of unity W^m, W = exp(DIR * 2 pi i / 16), exact
// constants of cos/sin(m pi / 8)
template <int DIR, int M, typename C> PF_D C w16(C a) {
  using R = decltype(a.x);
  constexpr int m = ((M % 16) + 16) % 16;
  const R c1 = R(0.92387953251128675613), s1 = R(0.38268343236508977173);
  const R h = R(0.70710678118654752440);
  R cr, ci;  // cos(2 pi m/16), DIR*sin(2 pi m/16)
  switch (m) {
    case 0: return a;
    case 4: { C z; z.x = -DIR * a.y; z.y = DIR * a.x; return z; }
    case 8: { C z; z.x = -a.x; z.y = -a.y; return z; }
    case 12: { C z; z.x = DIR * a.y; z.y = -DIR * a.x; return z; }
    case 2: cr = h; ci = DIR * h; break;
    case 6: cr = -h; ci = DIR * h; break;
    case 10: cr = -h; ci = -DIR * h; break;
    case 14: cr = h; ci = -DIR * h; break;
    case 1: cr = c1; ci = DIR * s1; break;
    case 3: cr = s1; ci = DIR * c1; break;
    case 5: cr = -s1; ci = DIR * c1; break;
    case 7: cr = -c1; ci = DIR * s1; break;
    case 9: cr = -c1; ci = -DIR * s1; break;
    case 11: cr = -s1; ci = -DIR * c1; break;
    case 13: cr = s1; ci = -DIR * c1; break;
    default: cr = c1; ci = -DIR * s1; break;  // 15
  }
  C z; z.x = a.x * cr - a.y * ci; z.y = a.x * ci + a.y * cr; return z;
}

template <int DIR, typename C> PF_D void dft2(C& a, C& b) {
  C t = a; a = cadd(t, b); b = csub(t, b);
}

// in: x0..x3 (stride S in array v starting at o); out natural order
template <int DIR, typename C> PF_D void dft4(C& x0, C& x1, C& x2, C& x3) {
  C a0 = cadd(x0, x2), a1 = csub(x0, x2), a2 = cadd(x1, x3), d = csub(x1, x3);
  // a3 = d * (DIR * i)
  C a3; a3.x = -DIR * d.y; a3.y = DIR * d.x;
  x0 = cadd(a0, a2); x2 = csub(a0, a2); x1 = cadd(a1, a3); x3 = csub(a1, a3);
}

template <int DIR, typename C> PF_D void dft8(C* v) {
  // even / odd radix-4 DFTs, then combine with W8^k = W16^(2k)
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  o1 = w16<DIR, 2>(o1); o2 = w16<DIR, 4>(o2); o3 = w16<DIR, 6>(o3);
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int DIR, typename C> PF_D void dft16(C* v) {
  // X[k1 + 4 k2] = sum_n2 W4^(n2 k2) W16^(n2 k1) sum_n1 x[4 n1 + n2] W4^(n1 k1)
  C y[16];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    C a = v[n2], b = v[4 + n2], c = v[8 + n2], d = v[12 + n2];
    dft4<DIR>(a, b, c, d);
    y[n2 * 4 + 0] = a; y[n2 * 4 + 1] = b; y[n2 * 4 + 2] = c; y[n2 * 4 + 3] = d;
  }
  y[1 * 4 + 1] = w16<DIR, 1>(y[5]);  y[1 * 4 + 2] = w16<DIR, 2>(y[6]);
  y[1 * 4 + 3] = w16<DIR, 3>(y[7]);  y[2 * 4 + 1] = w16<DIR, 2>(y[9]);
  y[2 * 4 + 2] = w16<DIR, 4>(y[10]); y[2 * 4 + 3] = w16<DIR, 6>(y[11]);
  y[3 * 4 + 1] = w16<DIR, 3>(y[13]); y[3 * 4 + 2] = w16<DIR, 6>(y[14]);
  y[3 * 4 + 3] = w16<DIR, 9>(y[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C a = y[k1], b = y[4 + k1], c = y[8 + k1], d = y[12 + k1];
    dft4<DIR>(a, b, c, d);
    v[k1] = a; v[k1 + 4] = b; v[k1 + 8] = c; v[k1 + 12] = d;
  }
}

// radix 3: W = exp(DIR 2 pi i / 3) = -1/2 + i DIR sqrt(3)/2
template <int DIR, typename C> PF_D void dft3(C& a, C& b, C& c) {
  using R = decltype(a.x);
  const R s = R(DIR) * R(0.86602540378443864676);
  const C t = cadd(b, c), d = csub(b, c);
  C m;  // a - t/2
  m.x = a.x - R(0.5) * t.x;
  m.y = a.y - R(0.5) * t.y;
  a = cadd(a, t);
  C sd;  // i s d
  sd.x = -s * d.y;
  sd.y = s * d.x;
  b = cadd(m, sd);
  c = csub(m, sd);
}

template <int R, int DIR, typename C> PF_D void dft(C* v) {
  if constexpr (R == 1) {
  } else if constexpr (R == 3) {
    dft3<DIR>(v[0], v[1], v[2]);
  } else if constexpr (R == 2) {
    dft2<DIR>(v[0], v[1]);
  } else if constexpr (R == 4) {
    dft4<DIR>(v[0], v[1], v[2], v[3]);
  } else if constexpr (R == 8) {
    dft8<DIR>(v);
  } else {
    static_assert(R == 16, "radix");
    dft16<DIR>(v);
  }
}

// ---- stage plan -------------------------------------------------------------
// N = 2^b or 3 * 2^b.  A factor 3 goes into the first stage (E a multiple
// of 3): with M3 a radix 3 R2 DFT in registers (dft3x: R2 = min(E2, N / 3)),
// without it a radix-3 stage of its own; the rest of the power-of-two part
// takes greedy radices E2, E2, ..., remainder with E2 the power-of-two part
// of E.  Ns(s) = product of earlier radices.  Every radix divides E.
template <int N, int E, bool M3 = true> struct Plan {
  static constexpr int P3 = (N % 3 == 0) ? 1 : 0;
  static constexpr int E2 = (E % 3 == 0) ? E / 3 : E;
  static_assert(!P3 || E % 3 == 0, "a radix-3 stage needs E divisible by 3");
  // first radix (the factor 3)
  static constexpr int R0 = P3 ? (M3 ? 3 * ((N / 3) < E2 ? (N / 3) : E2) : 3) : 1;
  static constexpr int radix(int s) {
    if (P3 && s == 0) return R0;
    int rem = P3 ? N / R0 : N, r = 1;
    for (int t = P3; t <= s; ++t) { r = rem < E2 ? rem : E2; rem /= r; }
    return r;
  }
  static constexpr int ns(int s) {
    int p = 1;
    for (int t = 0; t < s; ++t) p *= radix(t);
    return p;
  }
  static constexpr int stages() {
    int s = 0, p = 1;
    while (p < N) { p *= radix(s); ++s; }
    return s;
  }
};

// Radix R = 3 R2 in registers (Cooley-Tukey, 3 x R2): 3-point DFTs over n1
// of v[R2 n1 + n2], twiddles W_R^(k1 n2), R2-point DFTs over n2; output k =
// k1 + 3 k2 in natural order.  W_R^m = exp(DIR 2 pi i m / R) is entry
// m N / R of the length-N table (conjugated for DIR > 0).
template <int N, int R2, int DIR, typename C>
PF_D void dft3x(C* v, const C* __restrict__ tw) {
  constexpr int R = 3 * R2;
  static_assert(N % R == 0, "the table of length N holds W_R");
  C y[3][R2];
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) {
    C a = v[n2], b = v[R2 + n2], c = v[2 * R2 + n2];
    dft3<DIR>(a, b, c);
    y[0][n2] = a;
    y[1][n2] = b;
    y[2][n2] = c;
  }
#pragma unroll
  for (int k1 = 1; k1 < 3; ++k1) {
#pragma unroll
    for (int n2 = 1; n2 < R2; ++n2) {
      C w = ldtw(tw + (k1 * n2) * (N / R));
      if (DIR > 0) w.y = -w.y;
      y[k1][n2] = cmul(y[k1][n2], w);
    }
  }
#pragma unroll
  for (int k1 = 0; k1 < 3; ++k1) {
    dft<R2, DIR>(y[k1]);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + 3 * k2] = y[k1][k2];
  }
}

// One Stockham stage on the thread's E registers.  Returns with v holding the
// stage output at positions given by dst(); the caller exchanges or stops.
template <int N, int E, int R, int NS, int DIR, typename C>
PF_D void stage_compute(C (&v)[E], int j, const C* __restrict__ tw) {
  constexpr int G = N / E;
  constexpr int Q = E / R;  // butterflies per thread
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    C b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) b[r] = v[q + r * Q];
    if constexpr (NS > 1) {
      const int jv = j + q * G;
      const int m = jv % NS;
      constexpr int step = N / (NS * R);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        C w = ldtw(tw + r * m * step);
        if (DIR > 0) w.y = -w.y;
        b[r] = cmul(b[r], w);
      }
    }
    if constexpr (R % 3 == 0 && R > 3) dft3x<N, R / 3, DIR>(b, tw);
    else dft<R, DIR>(b);
#pragma unroll
    for (int r = 0; r < R; ++r) v[q + r * Q] = b[r];
  }
}

// Position written by element e (= q + r*Q) of thread j in a stage (R, NS).
template <int N, int E, int R, int NS> PF_D int stage_dst(int j, int e) {
  constexpr int G = N / E;
  constexpr int Q = E / R;
  const int q = e % Q, r = e / Q;
  const int jv = j + q * G;
  return (jv / NS) * NS * R + (jv % NS) + r * NS;
}

template <int N, int E, int DIR, int s, int S, bool M3, typename C, typename SMF, typename SYNCF>
PF_D void fft_stages(C (&v)[E], int j, const C* tw, SMF& sm, SYNCF& sync) {
  if constexpr (s < S) {
    using P = Plan<N, E, M3>;
    constexpr int R = P::radix(s);
    constexpr int NS = P::ns(s);
    stage_compute<N, E, R, NS, DIR>(v, j, tw);
    if constexpr (s + 1 < S) {
      constexpr int G = N / E;
#pragma unroll
      for (int e = 0; e < E; ++e) sm(stage_dst<N, E, R, NS>(j, e)) = v[e];
      sync();
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = sm(j + G * e);
      sync();
    }
    fft_stages<N, E, DIR, s + 1, S, M3>(v, j, tw, sm, sync);
  }
}

// Full FFT.  SM(pos) -> C& addresses the exchange buffer of this line; SYNC()
// synchronises all threads sharing the buffer.  Called by every thread of the
// group (no divergence around it).
template <int N, int E, int DIR, bool M3 = true, typename C, typename SMF, typename SYNCF>
PF_D void fft(C (&v)[E], int j, const C* __restrict__ tw, SMF sm, SYNCF sync) {
  using P = Plan<N, E, M3>;
  constexpr int S = P::stages();
  static_assert(N % E == 0, "E divides N");
  fft_stages<N, E, DIR, 0, S, M3>(v, j, tw, sm, sync);
}

}  // namespace pf
