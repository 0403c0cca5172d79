// Kernels and launch templates of the fused pencil passes of the 3D nonlinear
// term (included by the plan unit pf_fused.cu and by the instantiation units
// pf_fused_f32t/f32p/f64t/f64p.cu, one per precision and rule, which the
// build compiles in parallel).
//
// 2/3 rule:
//
// Only modes with |k_i| <= kmax_i = (n_i - 1) / 3 feed u and omega, so the
// inverse passes work on compact "kept" index ranges:  along a complex axis
// the kept indices are [0, kmax] and [n - kmax, n), compacted to [0, c) with
// c = 2 kmax + 1; along the last axis they are [0, kmax2], c2 = kmax2 + 1.
//
//   P1  inverse FFT along axis 0 of the kept (k1, k2) columns of u_hat
//       -> A[5][x0][k1c][k2c]: u0, u1, u2, D1 = F0^-1(i k0 u1), D2 = F0^-1(i k0 u2)
//   P2  omega = i k x u assembled per (k1, k2) (omega1 = i k2 u0 - D2,
//       omega2 = D1 - i k1 u0), inverse FFT along axis 1
//       -> B[6][x0][x1][k2c]: u0, u1, u2, w0, w1, w2
//   P3  per pair of (x0, x1) lines: C2R of the six fields (z = a + i b),
//       u x omega in registers (optional CFL max), R2C of the three products,
//       scaled by 1 / (n0 n1 n2) -> nl[3][x0][x1][k2]
//   P4  forward FFT along axis 1 of nl (generic strided pass)
//   P5  forward FFT along axis 0 of nl, then the stage update of every mode
//       of the column (Leray, Nyquist mask, forcing, noise, L, integrator)
//       writing u_hat: the nonlinear term never returns to HBM.
#pragma once
#include <array>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "pf_fft.cuh"
#include "pf_fgeo.h"
#include "pf_fused.h"
#include "pf_fused2d.h"
#include "pf_tma.cuh"
#include "pf_update.cuh"

namespace pf {

// Transform lengths are 2^b (2/3 rule) or 3 * 2^b (3/2 rule, M = 3n/2); a
// radix-3 first stage needs E divisible by 3.
// FP64 (R = double) halves the values per lane of the FP32 choices (a complex
// double takes four registers).
template <int N, typename R = float> struct TuneS {  // strided passes P1, P2, P4 (T measured best at 128 / G)
  static constexpr bool D = sizeof(R) == 8;
  static constexpr int E = N % 3 == 0 ? 12
                           : (D ? (N <= 8 ? N : 8) : (N <= 16 ? N : (N <= 64 ? 8 : 16)));
  static constexpr int G = N / E;
  static constexpr int T = (128 / G) < 8 ? 8 : ((128 / G) > 64 ? 64 : 128 / G);
};
template <int N, typename R = float> struct TuneU {  // P5 (FFT + update, three fields staged in smem)
  static constexpr int E = TuneS<N, R>::E;
  static constexpr int G = N / E;
  static constexpr int T0 = (256 / G) < 4 ? 4 : ((256 / G) > 64 ? 64 : 256 / G);
  // the staging tile (3 N T values) kept near 100 KB
  static constexpr int T = 3 * N * T0 * (int)sizeof(cx<R>) > 100 * 1024 ? T0 / 2 : T0;
};
template <int N, typename R = float> struct TuneC {  // contiguous pass P3: 8 (2^b) or 12 (3 * 2^b) values per lane
  static constexpr int E = N % 3 == 0 ? 12 : 8;
  static constexpr int G = N / E;   // lanes per line pair, <= 32 for N <= 256 / 384
  static constexpr int PW = 32 / G; // line pairs per warp
  static constexpr int W = 8;       // warps per CTA
  // exchange buffer of one line pair (8-byte values): position p lives at
  // p ^ ((p >> 3) & 15), which spreads the radix-8 stage stores (stride 8)
  // over all banks; the pair stride shifts neighbouring pairs' banks.  The
  // sides up to 16 and 3 * 2^b use a plain +1 per 16 padding instead.
  static constexpr bool PLAIN = N <= 16 || N % 3 == 0 || sizeof(R) == 8;
  static constexpr int SHP = sizeof(R) == 8 ? 3 : 4;  // FP64: +1 per 8 (16-byte values)
  static constexpr int BUF = PLAIN ? N + (N >> SHP) + 1 : (N == 32 ? N + 4 : (N == 64 ? N + 8 : N));
  static PF_HD int sw(int p) { return PLAIN ? p + (p >> SHP) : p ^ ((p >> 3) & 15); }
  // FP64 P3 runs the streamed-omega kernel: 6 warps fit its shared memory
  static constexpr int WS = sizeof(R) == 8 ? 6 : 8;
};

// Exchange buffer of the strided passes: position p of column t.  Eight
// padding values after every 16 positions put the radix-16 stage stores of
// neighbouring threadIdx.y rows (positions 16 apart) on different banks when
// T = 8.
template <int T> PF_HD int col_pos(int p, int t) { return p * T + t + 8 * (p >> 4); }
template <int N, int T, typename R = float> constexpr size_t col_buf_bytes() {
  return sizeof(cx<R>) * (size_t)(N * T + 8 * (N >> 4));
}


// Row i of a length-t inverse transform along an axis whose N-grid side is n:
// its weight (0, 1/2 or 1) and the N-grid wavenumber index kf of its input.
// 2/3 rule (PAD false, t == n): rows with |k| <= kmax are kept.  3/2 rule
// (PAD true, t = 3n/2): the N-grid spectrum embedded in the t grid, the even
// side's Nyquist row (wavenumber -n/2) split half to +n/2 and half to -n/2
// (basis.py:80-81 padding).  Its N-grid row index is kf mod n.
template <bool PAD> PF_D float row_weight(int i, int t, int n, int kmax, int& kf) {
  if constexpr (!PAD) {
    kf = kfreq(i, t);
    return abs(kf) <= kmax ? 1.f : 0.f;
  } else {
    const int h = n >> 1, k = kfreq(i, t);
    if (abs(k) < h) { kf = k; return 1.f; }
    kf = -h;
    return abs(k) == h ? 0.5f : 0.f;
  }
}

// Forward direction of the 3/2 rule: N-grid row i of a complex axis takes
// transform row src, plus row t - n/2 for the Nyquist row (the +n/2 and -n/2
// wavenumbers fold into one).
PF_D int fold_src(int i, int t, int n) {
  const int h = n >> 1;
  return i <= h ? i : t - (n - i);
}

struct FusedPlan {
  Geo g;
  FGeo f{};
  int prec;
  void* A = nullptr;  // 5 * t0 * c1 * c2 complex
  void* B = nullptr;  // 6 * t0 * t1 * c2 complex
  void* nlM = nullptr;  // 3/2 rule: 3 * t0 * t1 * nh complex (nl on the padded x0, x1 grid)
  bool pad = false;
  int dim = 3;        // 2: the three-pass 2D schedule of pf_fused2d.cu on f2 (A its scratch)
  F2 f2;
  int* err = nullptr; // device error word (bounded waits that gave up)
  int cap = 1;        // members the buffers hold (f.nmem / f2.nmem: members launched)
  int slabs = 1;      // pencil plan of one slab (pf_slab.cu): f.n0 = f.t0 = planes per slab
  int nsm = 148;
  // launch variant per pass (used where that pass's axis has 256 points):
  // measured best on B200 at 256^3 are P1 one output field per CTA row
  // (16, 8), P2 (16, 8) at >= 4 CTAs per SM, P3 one staging buffer, 8 warps
  // x 1 CTA (162 us against 175 us for 4 warps x 3 CTAs once the R2C split
  // moved to warp shuffles: the 255-register budget holds the output phase)
  int var[6] = {0, 7, 5, 3, 0, 0};
  // the same for 384-point passes (3/2 rule at n = 256), variants 11..19:
  // P1 one output field per CTA row at 24 values, P2 the same at twelve
  // values, P4 24 values
  int var384[6] = {0, 17, 18, 0, 13, 0};
  // CTA rows per column tile of P1 (1 or 3) and P2 (1 or 2): one per group
  // of fields (PF_FUSED_SPLIT="p1:v,p2:v" overrides)
  int split[6] = {1, 3, 2, 1, 1, 1};
  // FP64: P1 / P2 with one output field per CTA row (sides >= 64; measured
  // 3.9 vs 4.2 ms per RK3 step at 256^3; PF_FUSED_FP64_ROWS=0 turns it off)
  bool fp64_rows = true;
};

// CFL maximum of a warp into member m's slot (double bits, atomicMax on the
// bit pattern of a non-negative double); every lane calls it.
PF_D void flush_max(unsigned long long* maxbits, long long m, double& mx) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits + m, (unsigned long long)__double_as_longlong(mx));
  mx = 0.0;
}

// Destination slab s of a slab pass's store: selects among the (kernel
// parameter) pointers with constant indices.
template <typename C> PF_D C* slab_dst(const FGeo& f, int s) {
  void* p = f.sl_dst[0];
#pragma unroll
  for (int i = 1; i < kMaxSlabs; ++i)
    if (s == i) p = f.sl_dst[i];
  return reinterpret_cast<C*>(p);
}

// ---------------------------------------------------------------------- P1
// SLAB (with FIVE, 2/3 rule): one slab's kept compact rows; plane x0 of the
// output goes to slab x0 / sl_n0's pass-1 buffer [5][sl_n0][c1][c2].
template <typename R, int N, int E, int T, int MB, bool PAD, bool FIVE = false, bool MEMB = false,
          bool SLAB = false>
__global__ void __launch_bounds__(T * (N / E), MB)
k_p1(const cx<R>* __restrict__ uh, cx<R>* __restrict__ A, FGeo f,
     const cx<R>* __restrict__ tw) {
  constexpr int G = N / E;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  // 32-bit offsets inside a box: every fused index space is below 2^31 for
  // sides <= 512; MEMB: member blockIdx.z
  if constexpr (MEMB) {
    uh += (long long)blockIdx.z * 3 * f.nspec;
    A += (long long)blockIdx.z * 5 * f.t0 * f.c1 * f.c2;
  }
  static_assert(!SLAB || (FIVE && !PAD && !MEMB), "slab P1: one field per CTA row, 2/3 rule");
  const int t = threadIdx.x, j = threadIdx.y;
  const int ncols = (SLAB ? f.sl_nc : f.c1) * f.c2;
  const int tile = (FIVE && f.ilv) ? (int)blockIdx.x / 5 : (int)blockIdx.x;
  const int q = tile * T + t;
  const bool active = q < ncols;
  int in_off = 0;
  if (active) {
    int k1c = q / f.c2;
    const int k2c = q - k1c * f.c2;
    if constexpr (SLAB) k1c += f.sl_c0;
    const int i1 = k1c <= f.kmax1 ? k1c : k1c + (f.n1 - f.c1);
    in_off = (SLAB ? i1 - f.sl_i1 : i1) * f.nh + k2c;
  }
  const int row_in = (SLAB ? f.sl_n1 : f.n1) * f.nh;
  const int fs_out = N * ncols;
  const int fs_in = (int)f.nspec;
  auto smf = [&](int pos) -> C& { return sm[col_pos<T>(pos, t)]; };
  auto sync = [] { __syncthreads(); };
  // row e of the column: weight, N-grid wavenumber index and source row
  // (recomputed, not stored)
  auto rowin = [&](int e, int& kf, int& src) {
    const float w = active ? row_weight<PAD>(j + G * e, N, f.n0, f.kmax0, kf) : 0.f;
    src = PAD ? (kf < 0 ? kf + f.n0 : kf) : j + G * e;
    return w;
  };
  auto load = [&](int c, int e, int& kf) {
    int src;
    const float w = rowin(e, kf, src);
    C z = w != 0.f ? uh[c * fs_in + src * row_in + in_off] : czero<C>();
    if constexpr (PAD) z = cscale(z, (R)w);
    return z;
  };
  // gridDim.y == 3: block row y transforms field y alone (u0; u1 and D1;
  // u2 and D2), which triples the CTAs without extra traffic
  const int part = gridDim.y == 1 ? -1 : (int)blockIdx.y;
  if constexpr (FIVE) {
    // FIVE: block row y makes output field y alone (u0, u1, u2, D1, D2) with
    // one line buffer; the derivative rows re-read u1, u2
    const int fld = f.ilv ? (int)blockIdx.x - tile * 5 : (int)blockIdx.y;
    const int c = fld < 3 ? fld : fld - 2;
    C w[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      int kf;
      w[e] = load(c, e, kf);
      if (fld >= 3) w[e] = cmuli(cscale(w[e], (R)(f.ks0 * kf)));
    }
    fft<N, E, +1>(w, j, tw, smf, sync);
    if constexpr (SLAB) {
      const int plane = f.c1 * f.c2;
      const long long fsd = (long long)f.sl_n0 * plane;
      const int col = f.sl_c0 * f.c2 + q;
      if (active) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int x0 = j + G * e, s = x0 / f.sl_n0;
          slab_dst<C>(f, s)[fld * fsd + (long long)(x0 - s * f.sl_n0) * plane + col] = w[e];
        }
      }
      // the stores may go to peer memory: visible before the exchange barrier
      __threadfence_system();
    } else if (active) {
#pragma unroll
      for (int e = 0; e < E; ++e) A[fld * fs_out + (j + G * e) * ncols + q] = w[e];
    }
    return;
  }
  C v[E], w[E];
  if (part <= 0) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      int kf;
      v[e] = load(0, e, kf);
    }
    fft<N, E, +1>(v, j, tw, smf, sync);
    if (active) {
#pragma unroll
      for (int e = 0; e < E; ++e) A[(j + G * e) * ncols + q] = v[e];
    }
  }
#pragma unroll
  for (int c = 1; c <= 2; ++c) {
    if (part >= 0 && part != c) continue;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      int kf;
      v[e] = load(c, e, kf);
      w[e] = cmuli(cscale(v[e], (R)(f.ks0 * kf)));
    }
    fft<N, E, +1>(v, j, tw, smf, sync);
    fft<N, E, +1>(w, j, tw, smf, sync);
    if (active) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        A[c * fs_out + (j + G * e) * ncols + q] = v[e];
        A[(2 + c) * fs_out + (j + G * e) * ncols + q] = w[e];
      }
    }
  }
}

// ---------------------------------------------------------------------- P2
template <typename R, int N, int E, int T, int MB, bool PAD, bool SIX = false, bool MEMB = false>
__global__ void __launch_bounds__(T * (N / E), MB)
k_p2(const cx<R>* __restrict__ A, cx<R>* __restrict__ B, FGeo f,
     const cx<R>* __restrict__ tw) {
  constexpr int G = N / E;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  if constexpr (MEMB) {  // member blockIdx.z
    A += (long long)blockIdx.z * 5 * f.t0 * f.c1 * f.c2;
    B += (long long)blockIdx.z * 6 * f.t0 * f.t1 * f.c2;
  }
  const int t = threadIdx.x, j = threadIdx.y;
  const int ncols = f.t0 * f.c2;
  const int tile = (SIX && f.ilv) ? (int)blockIdx.x / 6 : (int)blockIdx.x;
  const int q = tile * T + t;
  const bool active = q < ncols;
  int in_base = 0, out_base = 0;
  R k2 = 0;
  if (active) {
    const int x0 = q / f.c2;
    const int k2c = q - x0 * f.c2;
    in_base = x0 * f.c1 * f.c2 + k2c;
    out_base = x0 * N * f.c2 + k2c;
    k2 = (R)(f.ks2 * k2c);
  }
  const int fs_in = f.t0 * f.c1 * f.c2;
  const int fs_out = f.t0 * N * f.c2;
  auto smf = [&](int pos) -> C& { return sm[col_pos<T>(pos, t)]; };
  auto sync = [] { __syncthreads(); };
  // per element e of the line (recomputed, not stored): weight, k1 and the
  // compact input row
  auto wt = [&](int e, int& kf) {
    return active ? row_weight<PAD>(j + G * e, N, f.n1, f.kmax1, kf) : 0.f;
  };
  auto k1 = [&](int e) {
    int kf;
    wt(e, kf);
    return (R)(f.ks1 * kf);
  };
  auto ld = [&](int fld, int e) {
    int kf;
    const float w = wt(e, kf);
    if (w == 0.f) return czero<C>();
    int row;
    if constexpr (PAD) {
      row = kf < 0 ? kf + f.n1 : kf;
    } else {
      const int i1 = j + G * e;
      row = i1 <= f.kmax1 ? i1 : i1 - (N - f.c1);
    }
    C z = A[fld * fs_in + in_base + row * f.c2];
    if constexpr (PAD) z = cscale(z, (R)w);
    return z;
  };
  auto store = [&](int fld, const C (&v)[E]) {
    if (active) {
#pragma unroll
      for (int e = 0; e < E; ++e) B[fld * fs_out + out_base + (j + G * e) * f.c2] = v[e];
    }
  };
  // gridDim.y == 2: block row 0 makes omega0, u1, u2 (reads u1, u2), row 1
  // omega2, omega1, u0 (reads u0, D1, D2); twice the CTAs, no extra traffic
  const int part = gridDim.y == 1 ? -1 : (int)blockIdx.y;
  if constexpr (SIX) {
    // SIX: block row y makes output field y' alone with one line buffer
    // (omega fields read their two inputs): one FFT per CTA, fewer registers,
    // at the cost of re-reading u0, u1, u2
    C w[E];
    const int row = f.ilv ? (int)blockIdx.x - tile * 6 : (int)blockIdx.y;
    switch (row) {
      case 0:  // omega0 = i (k1 u2 - k2 u1)
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = cmuli(csub(cscale(ld(2, e), k1(e)), cscale(ld(1, e), k2)));
        fft<N, E, +1>(w, j, tw, smf, sync);
        store(3, w);
        break;
      case 1:
      case 2:
      case 5: {  // u1, u2, u0
        const int fld = row == 5 ? 0 : row;
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = ld(fld, e);
        fft<N, E, +1>(w, j, tw, smf, sync);
        store(fld, w);
        break;
      }
      case 3:  // omega2 = D1 - i k1 u0
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = csub(ld(3, e), cmuli(cscale(ld(0, e), k1(e))));
        fft<N, E, +1>(w, j, tw, smf, sync);
        store(5, w);
        break;
      default:  // omega1 = i k2 u0 - D2
#pragma unroll
        for (int e = 0; e < E; ++e) w[e] = csub(cmuli(cscale(ld(0, e), k2)), ld(4, e));
        fft<N, E, +1>(w, j, tw, smf, sync);
        store(4, w);
        break;
    }
    return;
  }
  C a[E], b[E], w[E];
  if (part <= 0) {
    // omega0 = i (k1 u2 - k2 u1); u1; u2
#pragma unroll
    for (int e = 0; e < E; ++e) {
      a[e] = ld(1, e);
      b[e] = ld(2, e);
      w[e] = cmuli(csub(cscale(b[e], k1(e)), cscale(a[e], k2)));
    }
    fft<N, E, +1>(w, j, tw, smf, sync);
    store(3, w);
    fft<N, E, +1>(a, j, tw, smf, sync);
    store(1, a);
    fft<N, E, +1>(b, j, tw, smf, sync);
    store(2, b);
  }
  if (part != 0) {
    // omega2 = D1 - i k1 u0; omega1 = i k2 u0 - D2; u0
#pragma unroll
    for (int e = 0; e < E; ++e) {
      a[e] = ld(0, e);
      b[e] = ld(3, e);
      w[e] = csub(b[e], cmuli(cscale(a[e], k1(e))));
    }
    fft<N, E, +1>(w, j, tw, smf, sync);
    store(5, w);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      b[e] = ld(4, e);
      w[e] = csub(cmuli(cscale(a[e], k2)), b[e]);
    }
    fft<N, E, +1>(w, j, tw, smf, sync);
    store(4, w);
    fft<N, E, +1>(a, j, tw, smf, sync);
    store(0, a);
  }
}

// ---------------------------------------------------------------------- P3
// Persistent: every warp walks groups of PW = 32 / G line pairs (one pair per
// G lanes).  A group's six input fields are two adjacent lines each, so one
// bulk copy per field lands a group in shared memory; the copy of the next
// group (other stage) is in flight while the current one is transformed.
// MEMB: more than one member (the member of a group is its index / gpm).
template <typename R, int N, int NB, int W, int MB, bool MEMB = false>
__global__ void __launch_bounds__(32 * W, MB)
k_p3(const cx<R>* __restrict__ B, cx<R>* __restrict__ nl, FGeo f,
     const cx<R>* __restrict__ tw, unsigned long long* __restrict__ maxbits, R scale,
     int* __restrict__ err, long long ngroups) {
  constexpr int E = TuneC<N>::E, G = TuneC<N>::G, PW = TuneC<N>::PW;
  constexpr int H = N / 2;
  constexpr int BUF = TuneC<N>::BUF;
  static_assert(G <= 32 && 32 % G == 0, "line pairs tile a warp");
  static_assert(NB == 1 || NB == 2, "one or two staging buffers per warp");
  static_assert(NB * W <= 16, "mbarriers fit the 128-byte header");
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];  // mbarriers 8 B, bulk copies 16 B
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pw = lane / G, j = lane % G;
  const int fb = 2 * PW * f.c2;        // complex values of one field of a group
  const int SC = 6 * fb;               // one staging buffer
  const int WC = ((NB * SC + PW * BUF) + 15) & ~15;
  const uint32_t fbytes = (uint32_t)(fb * sizeof(C));
  const long long fs_in = (long long)f.n0 * f.n1 * f.c2;
  const long long gpm = (long long)f.t0 * f.t1 / (2 * PW);  // groups per member (MEMB)
  uint64_t* bars = reinterpret_cast<uint64_t*>(smraw) + NB * warp;
  C* wbase = reinterpret_cast<C*>(smraw + 128) + (long long)warp * WC;
  C* ex = wbase + NB * SC + pw * BUF;
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NB; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
  }
  __syncwarp();
  auto issue = [&](long long grp, int s) {
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(&bars[s], 6 * fbytes);
      const C* src = B + grp * fb;
      if constexpr (MEMB) {  // member mem's fields start at mem * 6 * fs_in
        const long long mem = grp / gpm;
        src = B + mem * 6 * fs_in + (grp - mem * gpm) * fb;
      }
      C* dst = wbase + s * SC;
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) bulk_g2s(dst + fld * fb, src + fld * fs_in, fbytes, &bars[s]);
    }
  };
  auto smf = [&](int pos) -> C& { return ex[TuneC<N>::sw(pos)]; };
  auto sync = [] { __syncwarp(); };
  // line pair of one field: two adjacent half-spectrum lines a, b packed as
  // z = a + i b on the full length-N circle (DC imaginary parts dropped)
  auto unpack = [&](const C* pa, C (&z)[E]) {
    const C* pb = pa + f.c2;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int m = j + G * e;
      const int k = m <= H ? m : N - m;
      const bool kin = k < f.c2;
      C a = kin ? pa[k] : czero<C>();
      C b = kin ? pb[k] : czero<C>();
      if (m == 0) { a.y = 0; b.y = 0; }
      C r;
      if (m <= H) { r.x = a.x - b.y; r.y = a.y + b.x; }
      else { r.x = a.x + b.y; r.y = b.x - a.y; }
      z[e] = r;
    }
  };
  const long long TW = (long long)gridDim.x * W;
  long long g = (long long)blockIdx.x * W + warp;
  if (g < ngroups) issue(g, 0);
  double mx = 0.0;
  [[maybe_unused]] long long curm = -1;  // member whose CFL maximum mx holds (MEMB)
  const R h = R(0.5) * scale;
  const R cw0 = (R)f.cflw0, cw1 = (R)f.cflw1, cw2 = (R)f.cflw2;
  static_assert((E & (E - 1)) == 0, "power-of-two values per lane");
  // lane of this pair holding bin N - k for k = j + G e (j > 0)
  const int mirror = (lane & ~(G - 1)) | ((G - j) & (G - 1));
  R mxr = R(0);  // running CFL maximum (as FP64 bits into maxbits when flushed)
  for (int it = 0; g < ngroups; g += TW, ++it) {
    long long mem = 0;
    if constexpr (MEMB) {
      mem = g / gpm;
      if (maxbits && mem != curm) {
        if (curm >= 0) {
          mx = (double)mxr;
          mxr = R(0);
          flush_max(maxbits, curm, mx);
        }
        curm = mem;
      }
    }
    const int s = NB == 2 ? (it & 1) : 0;
    const bool more = g + TW < ngroups;
    if (NB == 2 && more) {
      __syncwarp();
      issue(g + TW, s ^ 1);
    }
    const uint32_t par = NB == 2 ? (uint32_t)((it >> 1) & 1) : (uint32_t)(it & 1);
    const bool ok = mbar_wait_bounded(&bars[s], par);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(err, kErrWaitP3);
      if (NB == 2 && more) mbar_wait_bounded(&bars[s ^ 1], (uint32_t)(((it + 1) >> 1) & 1));
      return;
    }
    const C* in = wbase + s * SC + 2 * pw * f.c2;
    C z[6][E];
    if constexpr (NB == 1) {
      // all six fields into registers, then the buffer takes the next group
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) unpack(in + fld * fb, z[fld]);
      __syncwarp();
      if (more) issue(g + TW, 0);
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) fft<N, E, +1>(z[fld], j, tw, smf, sync);
    } else {
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) {
        unpack(in + fld * fb, z[fld]);
        fft<N, E, +1>(z[fld], j, tw, smf, sync);
      }
    }
    // u x omega for both lines (real parts: line a, imaginary parts: line b)
    C c[3][E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const C u0 = z[0][e], u1 = z[1][e], u2 = z[2][e];
      const C w0 = z[3][e], w1 = z[4][e], w2 = z[5][e];
      c[0][e].x = u1.x * w2.x - u2.x * w1.x;  c[0][e].y = u1.y * w2.y - u2.y * w1.y;
      c[1][e].x = u2.x * w0.x - u0.x * w2.x;  c[1][e].y = u2.y * w0.y - u0.y * w2.y;
      c[2][e].x = u0.x * w1.x - u1.x * w0.x;  c[2][e].y = u0.y * w1.y - u1.y * w0.y;
      if (maxbits) {  // CFL sums and their running maximum in the state's precision
        const R sa = fabs(u0.x) * cw0 + fabs(u1.x) * cw1 + fabs(u2.x) * cw2;
        const R sb = fabs(u0.y) * cw0 + fabs(u1.y) * cw1 + fabs(u2.y) * cw2;
        mxr = fmax(mxr, fmax(sa, sb));
      }
    }
    const long long la = 2 * ((g - mem * gpm) * PW + pw);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      fft<N, E, -1>(c[i], j, tw, smf, sync);
      C* oa = nl + i * f.nspec + la * f.nh;
      if constexpr (MEMB) oa += mem * 3 * f.nlcomp;
      C* ob = oa + f.nh;
      // R2C split of the two lines: bin k = j + G e is this lane's register
      // e; its mirror N - k is register E - 1 - e of lane G - j of the pair
      // (register (E - e) mod E of this lane when j = 0), fetched by warp
      // shuffles instead of a shared-memory round trip
#pragma unroll
      for (int e = 0; e <= E / 2; ++e) {
        C zn;
        zn.x = __shfl_sync(0xffffffffu, c[i][E - 1 - e].x, mirror);
        zn.y = __shfl_sync(0xffffffffu, c[i][E - 1 - e].y, mirror);
        if (j == 0) zn = c[i][(E - e) & (E - 1)];
        const C zk = c[i][e];
        const int k = j + G * e;
        if (k <= H) {
          C Av, Bv;
          Av.x = (zk.x + zn.x) * h; Av.y = (zk.y - zn.y) * h;
          Bv.x = (zk.y + zn.y) * h; Bv.y = -(zk.x - zn.x) * h;
          oa[k] = Av;
          ob[k] = Bv;
        }
      }
    }
  }
  mx = (double)mxr;
  if constexpr (MEMB) {
    if (maxbits && curm >= 0) flush_max(maxbits, curm, mx);
  } else if (maxbits) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
  }
}

// P3 with omega streamed: u goes to thread-private shared-memory slots after
// its C2R and omega is transformed one field at a time, accumulating u x
// omega in registers, for when six whole fields would not fit the registers
// (twelve values per lane on 3/2-rule lines, or FP64).  One staging buffer
// per warp, refilled once the group's last field is in registers.
// PAD (3/2 rule): padded lines of t2 = 3 n2 / 2 points, inputs k2 <= n2/2
// (the Nyquist column halved), outputs k2 <= n2/2 (the Nyquist entry plus
// its -n2/2 partner, the conjugate).  2/3 rule: inputs k2 <= kmax2, every
// output k2 <= n2/2.
template <typename R, int N, int W, bool PAD, bool MEMB = false>
__global__ void __launch_bounds__(32 * W, 1)
k_p3s(const cx<R>* __restrict__ B, cx<R>* __restrict__ nl, FGeo f,
        const cx<R>* __restrict__ tw, unsigned long long* __restrict__ maxbits, R scale,
        int* __restrict__ err, long long ngroups) {
  constexpr int E = TuneC<N, R>::E, G = TuneC<N, R>::G, PW = TuneC<N, R>::PW;
  constexpr int H = N / 2;
  constexpr int BUF = TuneC<N, R>::BUF;
  static_assert(G <= 32 && 32 % G == 0, "line pairs tile a warp");
  static_assert(W <= 16, "mbarriers fit the 128-byte header");
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pw = lane / G, j = lane % G;
  const int fb = 2 * PW * f.c2;
  const int SC = 6 * fb;
  const int WC = ((SC + PW * BUF + PW * 3 * N) + 15) & ~15;
  const uint32_t fbytes = (uint32_t)(fb * sizeof(C));
  const long long fs_in = (long long)f.t0 * f.t1 * f.c2;
  const long long gpm = (long long)f.t0 * f.t1 / (2 * PW);  // groups per member (MEMB)
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw) + warp;
  C* wbase = reinterpret_cast<C*>(smraw + 128) + (long long)warp * WC;
  C* ex = wbase + SC + pw * BUF;
  C* ur = wbase + SC + PW * BUF + pw * 3 * N;  // u on the padded line, own slots
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  auto issue = [&](long long grp) {
    if (lane == 0) {
      fence_proxy_async_smem();
      mbar_arrive_expect_tx(bar, 6 * fbytes);
      const C* src = B + grp * fb;
      if constexpr (MEMB) {  // member mem's fields start at mem * 6 * fs_in
        const long long mem = grp / gpm;
        src = B + mem * 6 * fs_in + (grp - mem * gpm) * fb;
      }
#pragma unroll
      for (int fld = 0; fld < 6; ++fld) bulk_g2s(wbase + fld * fb, src + fld * fs_in, fbytes, bar);
    }
  };
  auto smf = [&](int pos) -> C& { return ex[TuneC<N, R>::sw(pos)]; };
  auto sync = [] { __syncwarp(); };
  auto unpack = [&](const C* pa, C (&z)[E]) {
    const C* pb = pa + f.c2;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int m = j + G * e;
      const int k = m <= H ? m : N - m;
      const bool kin = k < f.c2;
      C a = kin ? pa[k] : czero<C>();
      C b = kin ? pb[k] : czero<C>();
      if (PAD && k == f.c2 - 1) { a = cscale(a, R(0.5)); b = cscale(b, R(0.5)); }
      if (m == 0) { a.y = 0; b.y = 0; }
      C r;
      if (m <= H) { r.x = a.x - b.y; r.y = a.y + b.x; }
      else { r.x = a.x + b.y; r.y = b.x - a.y; }
      z[e] = r;
    }
  };
  // line a in the real parts, line b in the imaginary parts
  auto mul = [](C p, C q) { C r; r.x = p.x * q.x; r.y = p.y * q.y; return r; };
  const long long TW = (long long)gridDim.x * W;
  long long g = (long long)blockIdx.x * W + warp;
  if (g < ngroups) issue(g);
  double mx = 0.0;
  [[maybe_unused]] long long curm = -1;  // member whose CFL maximum mx holds (MEMB)
  const R h = R(0.5) * scale;
  const R cw0 = (R)f.cflw0, cw1 = (R)f.cflw1, cw2 = (R)f.cflw2;
  for (int it = 0; g < ngroups; g += TW, ++it) {
    long long mem = 0;
    if constexpr (MEMB) {
      mem = g / gpm;
      if (maxbits && mem != curm) {
        if (curm >= 0) flush_max(maxbits, curm, mx);
        curm = mem;
      }
    }
    const bool more = g + TW < ngroups;
    const bool ok = mbar_wait_bounded(bar, (uint32_t)(it & 1));
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) atomicExch(err, kErrWaitP3);
      return;
    }
    const C* in = wbase + 2 * pw * f.c2;
    C v[E];
#pragma unroll
    for (int fld = 0; fld < 3; ++fld) {
      unpack(in + fld * fb, v);
      fft<N, E, +1>(v, j, tw, smf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) ur[fld * N + j + G * e] = v[e];
    }
    if (maxbits) {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const C u0 = ur[j + G * e], u1 = ur[N + j + G * e], u2 = ur[2 * N + j + G * e];
        // CFL sums in the state's precision, the running maximum in FP64
        const R sa = fabs(u0.x) * cw0 + fabs(u1.x) * cw1 + fabs(u2.x) * cw2;
        const R sb = fabs(u0.y) * cw0 + fabs(u1.y) * cw1 + fabs(u2.y) * cw2;
        mx = fmax(mx, (double)fmax(sa, sb));
      }
    }
    C c[3][E];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int e = 0; e < E; ++e) c[i][e] = czero<C>();
#pragma unroll
    for (int wc = 0; wc < 3; ++wc) {
      unpack(in + (3 + wc) * fb, v);
      if (wc == 2) {
        __syncwarp();  // every lane has read the group
        if (more) issue(g + TW);
      }
      fft<N, E, +1>(v, j, tw, smf, sync);
      // c0 = u1 w2 - u2 w1, c1 = u2 w0 - u0 w2, c2 = u0 w1 - u1 w0: field wc
      // adds u[wc+2] w to c[wc+1] and subtracts u[wc+1] w from c[wc+2]
      const int ia = (wc + 1) % 3, ib = (wc + 2) % 3;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const C ua = ur[ia * N + j + G * e], ub = ur[ib * N + j + G * e];
        c[ia][e] = cadd(c[ia][e], mul(ub, v[e]));
        c[ib][e] = csub(c[ib][e], mul(ua, v[e]));
      }
    }
    const long long la = 2 * ((g - mem * gpm) * PW + pw);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      fft<N, E, -1>(c[i], j, tw, smf, sync);
#pragma unroll
      for (int e = 0; e < E; ++e) smf(j + G * e) = c[i][e];
      sync();
      C* oa = nl + i * f.nlcomp + la * f.nh;
      if constexpr (MEMB) oa += mem * 3 * f.nlcomp;
      C* ob = oa + f.nh;
#pragma unroll
      for (int e = 0; e <= E / 2; ++e) {
        const int k = j + G * e;
        if (k < f.nh) {
          const C zk = smf(k);
          const C zn = smf(k == 0 ? 0 : N - k);
          C Av, Bv;
          Av.x = (zk.x + zn.x) * h; Av.y = (zk.y - zn.y) * h;
          Bv.x = (zk.y + zn.y) * h; Bv.y = -(zk.x - zn.x) * h;
          if (PAD && k == f.nh - 1) {
            Av.x *= R(2); Av.y = R(0);
            Bv.x *= R(2); Bv.y = R(0);
          }
          oa[k] = Av;
          ob[k] = Bv;
        }
      }
      sync();
    }
  }
  if constexpr (MEMB) {
    if (maxbits && curm >= 0) flush_max(maxbits, curm, mx);
  } else if (maxbits) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
  }
}

// ---------------------------------------------------------------------- P4
// In-place forward FFT along axis 1 of nl[3][x0][x1][k2]: column q = (plane,
// k2) with plane = comp * t0 + x0.  3/2 rule: the t1 transform rows are then
// truncated to the n1 N-grid rows (+n1/2 and -n1/2 folded into the Nyquist
// row), written to the first n1 rows of the column.
// SLAB (2/3 rule): out of place, row k1 of the column to slab k1 / sl_n1's
// nonlinear buffer [3][sl_N0][sl_n1][nh] at plane sl_x0 + x0.
template <typename R, int N, int E, int T, int MB, bool PAD, bool MEMB = false, bool SLAB = false>
__global__ void __launch_bounds__(T * (N / E), MB)
k_p4(cx<R>* __restrict__ nl, FGeo f, const cx<R>* __restrict__ tw) {
  constexpr int G = N / E;
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  if constexpr (MEMB) nl += (long long)blockIdx.y * 3 * f.nlcomp;  // member blockIdx.y
  const int t = threadIdx.x, j = threadIdx.y;
  const long long ncols = (long long)3 * f.t0 * f.nh;
  const long long q = (long long)blockIdx.x * T + t;
  const bool active = q < ncols;
  long long base = 0;
  if (active) {
    const long long pl = q / f.nh;
    base = pl * N * f.nh + (q - pl * f.nh);
  }
  C v[E];
#pragma unroll
  for (int e = 0; e < E; ++e)
    v[e] = active ? nl[base + (long long)(j + G * e) * f.nh] : czero<C>();
  fft<N, E, -1>(v, j, tw, [&](int pos) -> C& { return sm[col_pos<T>(pos, t)]; },
                [] { __syncthreads(); });
  if constexpr (SLAB) {
    static_assert(!PAD && !MEMB, "slab P4: 2/3 rule");
    if (active) {
      const long long pl = q / f.nh;
      const int c = (int)(pl / f.t0), xl = (int)(pl - (long long)c * f.t0);
      const long long rows = (long long)f.sl_n1 * f.nh;
      const long long bd = c * (long long)f.sl_N0 * rows + (long long)(f.sl_x0 + xl) * rows +
                           (q - pl * f.nh);
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int i = j + G * e, r = i / f.sl_n1;
        slab_dst<C>(f, r)[bd + (long long)(i - r * f.sl_n1) * f.nh] = v[e];
      }
    }
    __threadfence_system();
  } else if constexpr (!PAD) {
    if (active) {
#pragma unroll
      for (int e = 0; e < E; ++e) nl[base + (long long)(j + G * e) * f.nh] = v[e];
    }
  } else {
    // the FFT's last exchange was read before its closing barrier
#pragma unroll
    for (int e = 0; e < E; ++e) sm[col_pos<T>(j + G * e, t)] = v[e];
    __syncthreads();
    constexpr int EU = 2 * E / 3;  // n1 = 2 N / 3 rows, G per step
    const int h = f.n1 >> 1;
    if (active) {
#pragma unroll
      for (int e = 0; e < EU; ++e) {
        const int i = j + G * e;
        C z = sm[col_pos<T>(fold_src(i, N, f.n1), t)];
        if (i == h) z = cadd(z, sm[col_pos<T>(N - h, t)]);
        nl[base + (long long)i * f.nh] = z;
      }
    }
  }
}

// ---------------------------------------------------------------------- P5
// The three FFT outputs of a column tile are parked in shared memory (one
// N x T buffer per component, also the FFT's exchange buffer) so the update
// phase holds only a chunk of modes in registers; u_hat / u0 of a chunk are
// loaded before any of its stores.
// SLAB: the columns of one slab's k1 rows [sl_i1, sl_i1 + sl_n1) (state and
// nl in the slab's layout; wavenumbers and noise sites of the whole box).
// MB5 > 0: at least MB5 CTAs per SM (register cap) instead of the default.
// S0: the first stage of a step (u0 is the state itself, nothing to load for
// it), with 8 rows of state loads in flight.
template <typename R, int N, int NC, bool NOISE, int CHU, bool PAD, bool MEMB = false,
          bool SLAB = false, int MB5 = 0, bool S0 = false>
__global__ void __launch_bounds__(TuneU<N, R>::T * TuneU<N, R>::G,
                                  MB5 ? MB5 : (sizeof(R) == 8 ? 1 : 2))
k_p5(UpdateArgs<R> U, const cx<R>* __restrict__ nl, FGeo f, const cx<R>* __restrict__ tw) {
  constexpr int E = TuneU<N, R>::E, G = TuneU<N, R>::G, T = TuneU<N, R>::T;
  const Member mem = member_of(U, MEMB ? (int)blockIdx.y : 0);  // member blockIdx.y
  if (MEMB) nl += (long long)blockIdx.y * 3 * f.nlcomp;
  // rows per thread whose state loads are in flight
  constexpr int CH = S0 ? (E < 8 ? E : 8) : (E < CHU ? E : CHU);
  using C = cx<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* S = reinterpret_cast<C*>(smraw);
  const int t = threadIdx.x, j = threadIdx.y;
  const int ncols = (SLAB ? f.sl_n1 : f.n1) * f.nh;
  const int q = blockIdx.x * T + t;
  const bool active = q < ncols;
  const long long fs = f.nlcomp;  // nl: [3][t0][rows of nlrow]; 2/3 rule: the state layout
  auto sync = [] { __syncthreads(); };
  // component c + 1 is loaded while component c is transformed
  C v[E], nx[E];
#pragma unroll
  for (int e = 0; e < E; ++e) nx[e] = active ? nl[(j + G * e) * f.nlrow + q] : czero<C>();
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C* Sc = S + c * N * T;
    auto smf = [&](int pos) -> C& { return Sc[pos * T + t]; };
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = nx[e];
    if (c < 2) {
#pragma unroll
      for (int e = 0; e < E; ++e)
        nx[e] = active ? nl[(c + 1) * fs + (j + G * e) * f.nlrow + q] : czero<C>();
    }
    fft<N, E, -1>(v, j, tw, smf, sync);
#pragma unroll
    for (int e = 0; e < E; ++e) Sc[(j + G * e) * T + t] = v[e];
  }
  // 3/2 rule: the update reads the folded rows, written by other threads
  if constexpr (PAD) __syncthreads();
  // N-grid rows per thread: all E (2/3 rule) or the n0 = 2N/3 of the t0 = N
  // transform rows (3/2 rule)
  constexpr int EU = PAD ? 2 * E / 3 : E;
  static_assert(EU % CH == 0, "whole chunks of rows");
  const int h0 = f.n0 >> 1;
  auto nhat = [&](int a, int i0) {
    if constexpr (!PAD) {
      return S[a * N * T + i0 * T + t];
    } else {
      C z = S[a * N * T + fold_src(i0, N, f.n0) * T + t];
      if (i0 == h0) z = cadd(z, S[a * N * T + (N - h0) * T + t]);
      return z;
    }
  };
  const StageScalars<R> sc = stage_scalars<R>(U, mem.mb);
  double accE = 0.0, accZ = 0.0;
  if (active) {
    const int i1l = q / f.nh, i2 = q - i1l * f.nh;
    const int i1 = SLAB ? i1l + f.sl_i1 : i1l;
    const R k1 = (R)(f.ks1 * kfreq(i1, f.n1)), k2 = (R)(f.ks2 * i2);
    const cx<R>* __restrict__ uh = U.uhat + mem.mo;
    cx<R>* __restrict__ uo = (U.uout ? U.uout : U.uhat) + mem.mo;  // new state
    cx<R>* __restrict__ u0p = U.u0 + mem.mo;
    const long long ns = f.nspec;
#pragma unroll
    for (int e0 = 0; e0 < EU; e0 += CH) {
      C un[CH][3], u0v[CH][3];
#pragma unroll
      for (int cc = 0; cc < CH; ++cc) {
        const long long m = (long long)(j + G * (e0 + cc)) * ncols + q;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          un[cc][a] = uh[a * ns + m];
          u0v[cc][a] = (S0 || U.save_u0) ? un[cc][a] : u0p[a * ns + m];
        }
      }
#pragma unroll
      for (int cc = 0; cc < CH; ++cc) {
        const int i0 = j + G * (e0 + cc);
        const long long m = (long long)i0 * ncols + q;
        ModeK<R, 3> mk_;
        mk_.ix.i0 = i0; mk_.ix.i1 = i1; mk_.ix.i2 = i2;
        const R k0 = (R)(f.ks0 * kfreq(i0, f.n0));
        mk_.k[0] = k0; mk_.k[1] = k1; mk_.k[2] = k2;
        mk_.k2 = k0 * k0 + k1 * k1 + k2 * k2;
        C nv[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) nv[a] = nhat(a, i0);
        update_core<R, 3, NC, NOISE>(U, m, mk_, nv, true, un[cc], u0v[cc], sc, accE, accZ, uo, u0p,
                                     mem.mb);
      }
    }
  }
  if (U.diag) block_add2(accE, accZ, U.diag + 2 * mem.mb);
}

// ------------------------------------------------------------------ plan / launch
// Raise the dynamic shared-memory limit when dynamic plus the kernel's static
// shared memory (up to 1 KB here) could pass the 48 KB default.
template <typename K> static cudaError_t set_smem(K kern, size_t bytes) {
  if (bytes + 1024 > 48 * 1024)
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return cudaSuccess;
}

#define PF_SWITCH_S(n, CALL)      \
  switch (n) {                    \
    case 16: return CALL(16);     \
    case 32: return CALL(32);     \
    case 64: return CALL(64);     \
    case 128: return CALL(128);   \
    case 256: return CALL(256);   \
    case 512: return CALL(512);   \
    default: return cudaErrorInvalidValue; \
  }
// FP32 2/3-rule sides: powers of two and 3 * 2^b (48..384)
#define PF_SWITCH_T(n, CALL)      \
  switch (n) {                    \
    case 16: return CALL(16);     \
    case 32: return CALL(32);     \
    case 48: return CALL(48);     \
    case 64: return CALL(64);     \
    case 96: return CALL(96);     \
    case 128: return CALL(128);   \
    case 192: return CALL(192);   \
    case 256: return CALL(256);   \
    case 384: return CALL(384);   \
    case 512: return CALL(512);   \
    default: return cudaErrorInvalidValue; \
  }
// transform lengths of the 3/2 rule (N-grid sides 16..256)
#define PF_SWITCH_M(n, CALL)      \
  switch (n) {                    \
    case 24: return CALL(24);     \
    case 48: return CALL(48);     \
    case 96: return CALL(96);     \
    case 192: return CALL(192);   \
    case 384: return CALL(384);   \
    default: return cudaErrorInvalidValue; \
  }

// Launch variants (radix width E, columns per CTA T, minimum CTAs per SM MB
// that caps registers; 0: no cap) of the FP32 strided passes; variant 0 is
// the TuneS default, 1..6 exist for n = 256 and 11..16 for 384, and P1 / P2
// also have one-output-field-per-CTA-row forms (7..9 at 256; 17..19 at 384;
// tuning knob PF_FUSED_VARIANT="p1:v,p2:v,p3:v,p4:v", which overrides
// FusedPlan::var).
// FP64 uses the TuneS defaults.  The 3/2 rule always needs the exchange
// buffer (P4 folds through it).
template <typename R, int N, int E, int T, bool PAD>
constexpr size_t strided_smem() {
  return (PAD || Plan<N, E>::stages() > 1) ? col_buf_bytes<N, T, R>() : 0;
}

template <typename R, bool PAD, int N, int E, int T, int MB = 0, bool MEMB = false>
static cudaError_t p1_run(FusedPlan* p, const cx<R>* uh, cudaStream_t st) {
  constexpr int G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)p->f.c1 * p->f.c2;
  const size_t sm = strided_smem<R, N, E, T, PAD>();
  cudaError_t e = set_smem(k_p1<R, N, E, T, MB, PAD, false, MEMB>, sm);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((ncols + T - 1) / T), (unsigned)p->split[1], MEMB ? (unsigned)p->f.nmem : 1u);
  k_p1<R, N, E, T, MB, PAD, false, MEMB><<<grid, dim3(T, G), sm, st>>>(uh, (cx<R>*)p->A, p->f, tw);
  return launched();
}

template <typename R, bool PAD, int N, int E, int T, int MB = 0, bool MEMB = false>
static cudaError_t p2_run(FusedPlan* p, cudaStream_t st) {
  constexpr int G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)p->f.t0 * p->f.c2;
  const size_t sm = strided_smem<R, N, E, T, PAD>();
  cudaError_t e = set_smem(k_p2<R, N, E, T, MB, PAD, false, MEMB>, sm);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((ncols + T - 1) / T), (unsigned)p->split[2], MEMB ? (unsigned)p->f.nmem : 1u);
  k_p2<R, N, E, T, MB, PAD, false, MEMB><<<grid, dim3(T, G), sm, st>>>(
      (const cx<R>*)p->A, (cx<R>*)p->B, p->f, tw);
  return launched();
}

template <typename R, bool PAD, int N, int E, int T, int MB = 0, bool MEMB = false>
static cudaError_t p4_run(FusedPlan* p, cx<R>* nl, cudaStream_t st) {
  constexpr int G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)3 * p->f.t0 * p->f.nh;
  const size_t sm = strided_smem<R, N, E, T, PAD>();
  cudaError_t e = set_smem(k_p4<R, N, E, T, MB, PAD, MEMB>, sm);
  if (e != cudaSuccess) return e;
  const dim3 grid((unsigned)((ncols + T - 1) / T), MEMB ? (unsigned)p->f.nmem : 1u);
  k_p4<R, N, E, T, MB, PAD, MEMB><<<grid, dim3(T, G), sm, st>>>(nl, p->f, tw);
  return launched();
}

#define PF_VARIANTS(RUN, N, ...)                                        \
  if constexpr (sizeof(R) == 4 && N == 384) {                           \
    switch (var384) {                                                   \
      case 11: return RUN<R, PAD, 384, 12, 8, 2>(__VA_ARGS__);          \
      case 12: return RUN<R, PAD, 384, 12, 16, 1>(__VA_ARGS__);         \
      case 13: return RUN<R, PAD, 384, 24, 8>(__VA_ARGS__);             \
      case 14: return RUN<R, PAD, 384, 24, 8, 3>(__VA_ARGS__);          \
      case 15: return RUN<R, PAD, 384, 24, 8, 4>(__VA_ARGS__);          \
      case 16: return RUN<R, PAD, 384, 24, 16, 2>(__VA_ARGS__);         \
      default: break;                                                   \
    }                                                                   \
  }                                                                     \
  if constexpr (sizeof(R) == 4 && N == 256) {                           \
    switch (var) {                                                      \
      case 1: return RUN<R, PAD, 256, 8, 16>(__VA_ARGS__);              \
      case 2: return RUN<R, PAD, 256, 8, 32>(__VA_ARGS__);              \
      case 3: return RUN<R, PAD, 256, 16, 8>(__VA_ARGS__);              \
      case 4: return RUN<R, PAD, 256, 16, 8, 3>(__VA_ARGS__);           \
      case 5: return RUN<R, PAD, 256, 16, 8, 4>(__VA_ARGS__);           \
      case 6: return RUN<R, PAD, 256, 16, 16, 2>(__VA_ARGS__);          \
      default: break;                                                   \
    }                                                                   \
  }                                                                     \
  return RUN<R, PAD, N, TuneS<N, R>::E, TuneS<N, R>::T>(__VA_ARGS__);

// P1 with one output field per CTA row (five rows)
template <typename R, bool PAD, int N, int E, int T, int MB = 0, bool MEMB = false>
static cudaError_t p1five_run(FusedPlan* p, const cx<R>* uh, cudaStream_t st) {
  constexpr int G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)p->f.c1 * p->f.c2;
  const size_t sm = strided_smem<R, N, E, T, PAD>();
  cudaError_t e = set_smem(k_p1<R, N, E, T, MB, PAD, true, MEMB>, sm);
  if (e != cudaSuccess) return e;
  const unsigned tiles = (unsigned)((ncols + T - 1) / T);
  const dim3 grid(p->f.ilv ? 5 * tiles : tiles, p->f.ilv ? 1u : 5u, MEMB ? (unsigned)p->f.nmem : 1u);
  k_p1<R, N, E, T, MB, PAD, true, MEMB><<<grid, dim3(T, G), sm, st>>>(uh, (cx<R>*)p->A, p->f, tw);
  return launched();
}

template <typename R, int N, bool PAD>
static cudaError_t p1_n(FusedPlan* p, const cx<R>* uh, cudaStream_t st) {
  const int var = p->var[1], var384 = p->var384[1];
  (void)var; (void)var384;
  if (p->f.nmem > 1) {
    // members: the form a single box takes by default (one output field per
    // CTA row for FP32 at 256 points and FP64 from 48), so a member's
    // arithmetic is the single box's
    using TS = TuneS<N, R>;
    constexpr bool five = sizeof(R) == 8 ? N >= 48 : N == 256;
    if constexpr (five) return p1five_run<R, PAD, N, TS::E, TS::T, 0, true>(p, uh, st);
    else return p1_run<R, PAD, N, TS::E, TS::T, 0, true>(p, uh, st);
  }
  if constexpr (sizeof(R) == 4 && N == 384) {
    switch (var384) {
      case 17: return p1five_run<R, PAD, 384, 24, 8>(p, uh, st);
      case 18: return p1five_run<R, PAD, 384, 12, 8>(p, uh, st);
      default: break;
    }
  }
  if constexpr (sizeof(R) == 4 && N == 256) {
    switch (var) {
      case 7: return p1five_run<R, PAD, 256, 16, 8>(p, uh, st);
      case 9: return p1five_run<R, PAD, 256, 16, 16>(p, uh, st);
      default: break;
    }
  }
  if constexpr (sizeof(R) == 8 && N >= 48) {
    if (p->fp64_rows) return p1five_run<R, PAD, N, TuneS<N, R>::E, TuneS<N, R>::T>(p, uh, st);
  }
  PF_VARIANTS(p1_run, N, p, uh, st)
}
// P2 with one output field per CTA row (six rows)
template <typename R, bool PAD, int N, int E, int T, int MB = 0, bool MEMB = false>
static cudaError_t p2six_run(FusedPlan* p, cudaStream_t st) {
  constexpr int G = N / E;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)p->f.t0 * p->f.c2;
  const size_t sm = strided_smem<R, N, E, T, PAD>();
  cudaError_t e = set_smem(k_p2<R, N, E, T, MB, PAD, true, MEMB>, sm);
  if (e != cudaSuccess) return e;
  const unsigned tiles = (unsigned)((ncols + T - 1) / T);
  const dim3 grid(p->f.ilv ? 6 * tiles : tiles, p->f.ilv ? 1u : 6u, MEMB ? (unsigned)p->f.nmem : 1u);
  k_p2<R, N, E, T, MB, PAD, true, MEMB><<<grid, dim3(T, G), sm, st>>>(
      (const cx<R>*)p->A, (cx<R>*)p->B, p->f, tw);
  return launched();
}

template <typename R, int N, bool PAD> static cudaError_t p2_n(FusedPlan* p, cudaStream_t st) {
  const int var = p->var[2], var384 = p->var384[2];
  (void)var; (void)var384;
  if (p->f.nmem > 1) {  // members: the default tile (FP64 from 48 points: one field per row)
    using TS = TuneS<N, R>;
    if constexpr (sizeof(R) == 8 && N >= 48) return p2six_run<R, PAD, N, TS::E, TS::T, 0, true>(p, st);
    else return p2_run<R, PAD, N, TS::E, TS::T, 0, true>(p, st);
  }
  if constexpr (sizeof(R) == 4 && N == 384) {
    switch (var384) {
      case 17: return p2six_run<R, PAD, 384, 24, 8>(p, st);
      case 18: return p2six_run<R, PAD, 384, 12, 8>(p, st);
      case 19: return p2six_run<R, PAD, 384, 24, 16>(p, st);
      default: break;
    }
  }
  if constexpr (sizeof(R) == 4 && N == 256) {
    switch (var) {
      case 7: return p2six_run<R, PAD, 256, 16, 8>(p, st);
      case 8: return p2six_run<R, PAD, 256, 16, 8, 4>(p, st);
      case 9: return p2six_run<R, PAD, 256, 16, 16>(p, st);
      case 10:  // input tiles by tiled bulk tensor copies (pf_p2t.cu)
        if constexpr (!PAD) {
          if (p2t_supported(p->f))
            return p2t_launch((const float2*)p->A, (float2*)p->B, p->f,
                              tw_base<float>() + tw_offset(256), p->err, st);
        }
        break;
      default: break;
    }
  }
  if constexpr (sizeof(R) == 8 && N >= 48) {
    if (p->fp64_rows) return p2six_run<R, PAD, N, TuneS<N, R>::E, TuneS<N, R>::T>(p, st);
  }
  PF_VARIANTS(p2_run, N, p, st)
}
template <typename R, int N, bool PAD>
static cudaError_t p4_n(FusedPlan* p, cx<R>* nl, cudaStream_t st) {
  const int var = p->var[4], var384 = p->var384[4];
  (void)var; (void)var384;
  if (p->f.nmem > 1)  // members: the default tile
    return p4_run<R, PAD, N, TuneS<N, R>::E, TuneS<N, R>::T, 0, true>(p, nl, st);
  PF_VARIANTS(p4_run, N, p, nl, st)
}

// P3 with omega streamed (3/2 rule; FP64)
template <typename R, bool PAD, int N, int W>
static cudaError_t p3s_run(FusedPlan* p, cx<R>* nl, unsigned long long* maxbits,
                           cudaStream_t st) {
  using TN = TuneC<N, R>;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ngroups = (long long)p->f.nmem * p->f.t0 * p->f.t1 / (2 * TN::PW);
  const int fb = 2 * TN::PW * p->f.c2;
  const int WC = ((6 * fb + TN::PW * TN::BUF + TN::PW * 3 * N) + 15) & ~15;
  const size_t sm = 128 + sizeof(cx<R>) * (size_t)W * WC;
  cudaError_t e = set_smem(k_p3s<R, N, W, PAD>, sm);
  if (e != cudaSuccess) return e;
  const R scale = (R)(1.0 / ((double)p->f.t0 * p->slabs * p->f.t1 * p->f.t2));
  long long blocks = (ngroups + W - 1) / W;
  if (blocks > (long long)p->nsm) blocks = p->nsm;
  if (p->f.nmem > 1) {
    e = set_smem(k_p3s<R, N, W, PAD, true>, sm);
    if (e != cudaSuccess) return e;
    k_p3s<R, N, W, PAD, true><<<(unsigned)blocks, 32 * W, sm, st>>>(
        (const cx<R>*)p->B, nl, p->f, tw, maxbits, scale, p->err, ngroups);
  } else {
    k_p3s<R, N, W, PAD><<<(unsigned)blocks, 32 * W, sm, st>>>(
        (const cx<R>*)p->B, nl, p->f, tw, maxbits, scale, p->err, ngroups);
  }
  return launched();
}

// FP32 2/3 rule: six fields in registers
template <int N, int NB, int W, int MB>
static cudaError_t p3_run(FusedPlan* p, float2* nl, unsigned long long* maxbits, cudaStream_t st) {
  using TN = TuneC<N>;
  const float2* tw = tw_base<float>() + tw_offset(N);
  const long long ngroups = (long long)p->f.nmem * p->f.n0 * p->f.n1 / (2 * TN::PW);
  const int fb = 2 * TN::PW * p->f.c2;
  const int WC = ((NB * 6 * fb + TN::PW * TN::BUF) + 15) & ~15;
  const size_t sm = 128 + sizeof(float2) * (size_t)W * WC;
  cudaError_t e = set_smem(k_p3<float, N, NB, W, MB>, sm);
  if (e != cudaSuccess) return e;
  const float scale = (float)(1.0 / ((double)p->f.n0 * p->slabs * p->f.n1 * p->f.n2));
  long long blocks = (ngroups + W - 1) / W;
  if (blocks > (long long)p->nsm * MB) blocks = (long long)p->nsm * MB;
  if (p->f.nmem > 1) {
    e = set_smem(k_p3<float, N, NB, W, MB, true>, sm);
    if (e != cudaSuccess) return e;
    k_p3<float, N, NB, W, MB, true><<<(unsigned)blocks, 32 * W, sm, st>>>(
        (const float2*)p->B, nl, p->f, tw, maxbits, scale, p->err, ngroups);
  } else {
    k_p3<float, N, NB, W, MB><<<(unsigned)blocks, 32 * W, sm, st>>>(
        (const float2*)p->B, nl, p->f, tw, maxbits, scale, p->err, ngroups);
  }
  return launched();
}

// The one-exchange form of pf_p3q.cu (sixteen values per lane, twiddles in
// registers, shuffled output split) with W warps per CTA.
static inline cudaError_t p3q_go(FusedPlan* p, int n, int W, float2* nl, unsigned long long* maxbits,
                          cudaStream_t st) {
  const float2* tw = tw_base<float>() + tw_offset(n);
  const int pw = 32 / (n / 16);
  const long long ngroups = (long long)p->f.nmem * p->f.n0 * p->f.n1 / (2 * pw);
  const float scale = (float)(1.0 / ((double)p->f.n0 * p->slabs * p->f.n1 * p->f.n2));
  return p3q_launch(n, W, (const float2*)p->B, nl, p->f, tw, maxbits, scale, p->err, ngroups,
                    p->nsm, st);
}

// FP32 2/3 rule, variant 0: two staging buffers per warp, 8 warps, one CTA
// per SM; 1..3 (n2 = 256): one staging buffer refilled as soon as the group
// is in registers, with 8 warps x 2 CTAs, 4 warps x 3 CTAs or 8 warps x 1
// CTA; 4, 5 (n2 = 256) and 4 (n2 = 128): the one-exchange form with 6 or 7
// warps.  3/2 rule, FP64 and 3 * 2^b sides: the streamed-omega kernel.
template <typename R, int N, bool PAD>
static cudaError_t p3_n(FusedPlan* p, cx<R>* nl, unsigned long long* maxbits, cudaStream_t st) {
  if constexpr (PAD || sizeof(R) == 8 || N % 3 == 0) {
    if constexpr (N > 384 || (!PAD && N % 3 != 0 && N > 256)) return cudaErrorInvalidValue;
    else if constexpr (sizeof(R) == 8 && PAD)
      return p3s_run<R, PAD, N, 4>(p, nl, maxbits, st);  // 50-53 KB of shared memory per warp
    else return p3s_run<R, PAD, N, TuneC<N, R>::WS>(p, nl, maxbits, st);
  } else if constexpr (N > 256) {
    return cudaErrorInvalidValue;
  } else {
    if constexpr (N == 256) {
      switch (p->var[3]) {
        case 1: return p3_run<256, 1, 8, 2>(p, nl, maxbits, st);
        case 2: return p3_run<256, 1, 4, 3>(p, nl, maxbits, st);
        case 3: return p3_run<256, 1, 8, 1>(p, nl, maxbits, st);
        case 4: return p3q_go(p, 256, 6, nl, maxbits, st);
        case 5: return p3q_go(p, 256, 7, nl, maxbits, st);
        default: break;
      }
    }
    if constexpr (N == 128) {
      if (p->var[3] == 4) return p3q_go(p, 128, 6, nl, maxbits, st);
    }
    return p3_run<N, 2, TuneC<N>::W, 1>(p, nl, maxbits, st);
  }
}

// the single-box or the member form of P5
template <typename R, bool PAD, int N, int CH, int NC, bool NOISE, int MB5 = 0, bool S0 = false>
static cudaError_t p5_go(FusedPlan* p, const UpdateArgs<R>& U, const cx<R>* nl, dim3 grid,
                         dim3 block, size_t sm, const cx<R>* tw, cudaStream_t st) {
  cudaError_t e;
  if constexpr (S0) {  // one box, first stage
    e = set_smem(k_p5<R, N, NC, NOISE, CH, PAD, false, false, MB5, true>, sm);
    if (e != cudaSuccess) return e;
    k_p5<R, N, NC, NOISE, CH, PAD, false, false, MB5, true><<<grid, block, sm, st>>>(U, nl, p->f, tw);
    return cudaSuccess;
  }
  if constexpr (MB5 > 0) {  // one box
    e = set_smem(k_p5<R, N, NC, NOISE, CH, PAD, false, false, MB5>, sm);
    if (e != cudaSuccess) return e;
    k_p5<R, N, NC, NOISE, CH, PAD, false, false, MB5><<<grid, block, sm, st>>>(U, nl, p->f, tw);
    return cudaSuccess;
  }
  if (p->f.nmem > 1) {
    e = set_smem(k_p5<R, N, NC, NOISE, CH, PAD, true>, sm);
    if (e != cudaSuccess) return e;
    k_p5<R, N, NC, NOISE, CH, PAD, true><<<grid, block, sm, st>>>(U, nl, p->f, tw);
  } else {
    e = set_smem(k_p5<R, N, NC, NOISE, CH, PAD>, sm);
    if (e != cudaSuccess) return e;
    k_p5<R, N, NC, NOISE, CH, PAD><<<grid, block, sm, st>>>(U, nl, p->f, tw);
  }
  return cudaSuccess;
}

template <typename R, bool PAD, int N, int CH, int MB5 = 0, bool S0 = false>
static cudaError_t p5_run(FusedPlan* p, const UpdateArgs<R>& U, int ncomp, const cx<R>* nl,
                          cudaStream_t st) {
  using TN = TuneU<N, R>;
  const cx<R>* tw = tw_base<R>() + tw_offset(N);
  const long long ncols = (long long)p->f.n1 * p->f.nh;
  const size_t sm = sizeof(cx<R>) * 3 * N * TN::T;
  const dim3 grid((unsigned)((ncols + TN::T - 1) / TN::T), (unsigned)p->f.nmem),
      block(TN::T, TN::G);
  if ((MB5 > 0 || S0) && p->f.nmem > 1) return cudaErrorInvalidValue;
  cudaError_t e;
  if (U.noise_src == kNoiseNone) e = p5_go<R, PAD, N, CH, 3, false, MB5, S0>(p, U, nl, grid, block, sm, tw, st);
  else if (ncomp == 9) e = p5_go<R, PAD, N, CH, 9, true, MB5>(p, U, nl, grid, block, sm, tw, st);
  else e = p5_go<R, PAD, N, CH, 3, true, MB5>(p, U, nl, grid, block, sm, tw, st);
  return e != cudaSuccess ? e : launched();
}

// Variant 0 keeps the state loads of 4 rows per thread in flight (FP64: 2);
// 1, 2 (FP32, n0 = 256) use 2 and 8; FP64 from 128 points runs two CTAs per
// SM unless variant 4.
template <typename R, int N, bool PAD>
static cudaError_t p5_n(FusedPlan* p, const UpdateArgs<R>& U, int ncomp, const cx<R>* nl,
                        cudaStream_t st) {
  if constexpr (sizeof(R) == 4 && N == 256) {
    switch (p->var[5]) {
      case 1: return p5_run<R, PAD, 256, 2>(p, U, ncomp, nl, st);
      case 2: return p5_run<R, PAD, 256, 8>(p, U, ncomp, nl, st);
      default: break;
    }
    if constexpr (!PAD) {
      // first stage, one box, no noise: 8 rows of state loads in flight
      // (variant 5 keeps the general form)
      if (p->var[5] != 5 && U.save_u0 && p->f.nmem == 1 && U.noise_src == kNoiseNone)
        return p5_run<R, PAD, 256, 4, 0, true>(p, U, ncomp, nl, st);
    }
  }
  if constexpr (sizeof(R) == 8 && !PAD && N >= 128) {
    // FP64, one box, no noise: two CTAs per SM (registers capped at 128, 16
    // bytes spilled at 256) instead of one at 158 registers -- 3.54 against
    // 3.76 ms per RK3 step at 256^3; variant 4 keeps one CTA per SM
    if (p->var[5] != 4 && p->f.nmem == 1 && U.noise_src == kNoiseNone)
      return p5_run<R, PAD, N, 2, 2>(p, U, ncomp, nl, st);
  }
  return p5_run<R, PAD, N, sizeof(R) == 8 ? 2 : 4>(p, U, ncomp, nl, st);
}

// 3/2 rule: passes 3 and 4 work in the plan's padded-grid buffer, which
// pass 5 reads.
template <typename R>
static cudaError_t pass_pad(FusedPlan* p, int pass, const void* uhat,
                            unsigned long long* maxbits, cudaStream_t st) {
  using C = cx<R>;
  C* nlp = (C*)p->nlM;
  switch (pass) {
    case 1: {
#define PF_CALL(NN) p1_n<R, NN, true>(p, (const C*)uhat, st)
      PF_SWITCH_M(p->f.t0, PF_CALL)
#undef PF_CALL
    }
    case 2: {
#define PF_CALL(NN) p2_n<R, NN, true>(p, st)
      PF_SWITCH_M(p->f.t1, PF_CALL)
#undef PF_CALL
    }
    case 3: {
#define PF_CALL(NN) p3_n<R, NN, true>(p, nlp, maxbits, st)
      PF_SWITCH_M(p->f.t2, PF_CALL)
#undef PF_CALL
    }
    case 4: {
#define PF_CALL(NN) p4_n<R, NN, true>(p, nlp, st)
      PF_SWITCH_M(p->f.t1, PF_CALL)
#undef PF_CALL
    }
    default:
      return cudaErrorInvalidValue;
  }
}

// 2/3 rule: nl is the caller's buffer in the state layout.  FP32 sides are
// powers of two and 3 * 2^b, FP64 powers of two.
template <typename R>
static cudaError_t pass_trunc(FusedPlan* p, int pass, const void* uhat, void* nl,
                              unsigned long long* maxbits, cudaStream_t st) {
  using C = cx<R>;
  C* nlp = (C*)nl;
  if constexpr (sizeof(R) == 4) {
    switch (pass) {
      case 1: {
#define PF_CALL(NN) p1_n<R, NN, false>(p, (const C*)uhat, st)
        PF_SWITCH_T(p->f.n0, PF_CALL)
#undef PF_CALL
      }
      case 2: {
#define PF_CALL(NN) p2_n<R, NN, false>(p, st)
        PF_SWITCH_T(p->f.n1, PF_CALL)
#undef PF_CALL
      }
      case 3: {
#define PF_CALL(NN) p3_n<R, NN, false>(p, nlp, maxbits, st)
        PF_SWITCH_T(p->f.n2, PF_CALL)
#undef PF_CALL
      }
      case 4: {
#define PF_CALL(NN) p4_n<R, NN, false>(p, nlp, st)
        PF_SWITCH_T(p->f.n1, PF_CALL)
#undef PF_CALL
      }
      default:
        return cudaErrorInvalidValue;
    }
  } else {
    switch (pass) {
      case 1: {
#define PF_CALL(NN) p1_n<R, NN, false>(p, (const C*)uhat, st)
        PF_SWITCH_S(p->f.n0, PF_CALL)
#undef PF_CALL
      }
      case 2: {
#define PF_CALL(NN) p2_n<R, NN, false>(p, st)
        PF_SWITCH_S(p->f.n1, PF_CALL)
#undef PF_CALL
      }
      case 3: {
#define PF_CALL(NN) p3_n<R, NN, false>(p, nlp, maxbits, st)
        PF_SWITCH_S(p->f.n2, PF_CALL)
#undef PF_CALL
      }
      case 4: {
#define PF_CALL(NN) p4_n<R, NN, false>(p, nlp, st)
        PF_SWITCH_S(p->f.n1, PF_CALL)
#undef PF_CALL
      }
      default:
        return cudaErrorInvalidValue;
    }
  }
}

template <typename R>
static cudaError_t update_pad(FusedPlan* p, const UpdateArgs<R>& U, int ncomp, cudaStream_t st) {
#define PF_CALL(NN) p5_n<R, NN, true>(p, U, ncomp, (const cx<R>*)p->nlM, st)
  PF_SWITCH_M(p->f.t0, PF_CALL)
#undef PF_CALL
}

template <typename R>
static cudaError_t update_trunc(FusedPlan* p, const UpdateArgs<R>& U, int ncomp, const void* nl,
                                cudaStream_t st) {
#define PF_CALL(NN) p5_n<R, NN, false>(p, U, ncomp, (const cx<R>*)nl, st)
  if constexpr (sizeof(R) == 4) {
    PF_SWITCH_T(p->f.n0, PF_CALL)
  } else {
    PF_SWITCH_S(p->f.n0, PF_CALL)
  }
#undef PF_CALL
}

// entry points of the instantiation units
#define PF_UNIT_DECL(R, S)                                                                       \
  cudaError_t fused_pass_##S##_trunc(FusedPlan* p, int pass, const void* uhat, void* nl,        \
                                     unsigned long long* maxbits, cudaStream_t st);              \
  cudaError_t fused_pass_##S##_pad(FusedPlan* p, int pass, const void* uhat,                    \
                                   unsigned long long* maxbits, cudaStream_t st);                \
  cudaError_t fused_update_##S##_trunc(FusedPlan* p, const UpdateArgs<R>& U, int ncomp,         \
                                       const void* nl, cudaStream_t st);                        \
  cudaError_t fused_update_##S##_pad(FusedPlan* p, const UpdateArgs<R>& U, int ncomp,           \
                                     cudaStream_t st);
PF_UNIT_DECL(float, f32)
PF_UNIT_DECL(double, f64)
#undef PF_UNIT_DECL

}  // namespace pf
