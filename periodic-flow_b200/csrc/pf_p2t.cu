// P2 of the fused 2/3-rule schedule (FP32, axis-1 length 256) with its input
// tiles brought in by tiled bulk tensor copies (TMA).
//
// P2 reads the pass-1 buffer A[5][x0][k1c][k2c] column by column: a CTA owns
// 8 columns k2c of one plane x0 and needs, per input field, the 171 kept k1c
// rows of those columns -- one 3D box {8 complex, c1 rows, 1 plane} of the
// tensor A seen as [5 t0][c1][c2].  A's rows are c2 = 86 complex (688 bytes,
// a multiple of 16), which tiled copies require; the state layout's rows of
// n/2 + 1 = 129 complex (1032 bytes) are not, so the other strided passes
// (P1, P4, P5) cannot take their tiles this way.  One thread issues the boxes
// of the CTA's fields (two or three, per the split of P2's outputs over two
// CTA rows) into 128-byte-aligned shared slots; every thread waits on the
// CTA's mbarrier (bounded) and then runs P2's FFTs from shared memory.  The
// columns past c2 in the plane's last tile are filled with zeros by the copy
// and not stored.  No multicast: each CTA loads its own boxes.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "pf_fft.cuh"
#include "pf_fgeo.h"
#include "pf_internal.h"
#include "pf_tma.cuh"

namespace pf {

namespace {

constexpr int kN = 256, kE = 16, kG = kN / kE, kT = 8;  // axis length, values/thread, threads/column, columns/CTA
constexpr int kSlotBytes = 11008;   // one box (8 x 171 complex = 10944 B) rounded to 128 B
constexpr int kMaxRows = 171;       // c1 at n1 = 256
constexpr int kBoxes = 3;           // CTA row 1 reads u0, D1, D2

// exchange buffer position of the strided FFT (as the other strided passes)
PF_D int colq(int p, int t) { return p * kT + t + 8 * (p >> 4); }
constexpr size_t kExBytes = sizeof(float2) * (size_t)(kN * kT + 8 * (kN >> 4));
constexpr size_t kSmem = 128 + (size_t)kBoxes * kSlotBytes + kExBytes;

PF_D void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

__global__ void __launch_bounds__(kT * kG, 4)
k_p2t(const __grid_constant__ CUtensorMap tmA, float2* __restrict__ B, FGeo f,
      const float2* __restrict__ tw, int* __restrict__ err, int tiles_per_plane) {
  using C = float2;
  extern __shared__ __align__(128) unsigned char smraw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  C* slot0 = reinterpret_cast<C*>(smraw + 128);
  C* sm = reinterpret_cast<C*>(smraw + 128 + kBoxes * kSlotBytes);
  const int t = threadIdx.x, j = threadIdx.y;
  const int x0 = blockIdx.x / tiles_per_plane;
  const int k2c0 = (blockIdx.x - x0 * tiles_per_plane) * kT;
  const int k2c = k2c0 + t;
  const bool active = k2c < f.c2;
  const int part = blockIdx.y;  // 0: reads u1, u2; 1: reads u0, D1, D2
  const int nbox = part == 0 ? 2 : 3;
  const uint32_t box_bytes = (uint32_t)(kT * f.c1 * sizeof(C));
  if (t == 0 && j == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (t == 0 && j == 0) {
    mbar_arrive_expect_tx(bar, nbox * box_bytes);
    for (int b = 0; b < nbox; ++b) {
      const int fld = part == 0 ? 1 + b : (b == 0 ? 0 : 2 + b);  // {1, 2} or {0, 3, 4}
      tma_load_3d(reinterpret_cast<unsigned char*>(slot0) + b * kSlotBytes, &tmA, 2 * k2c0, 0,
                  fld * f.t0 + x0, bar);
    }
  }
  const bool ok = mbar_wait_bounded(bar, 0);
  if (!__syncthreads_and(ok)) {
    if (t == 0 && j == 0) atomicExch(err, kErrWaitP2);
    return;
  }
  auto slot = [&](int b) -> const C* {
    return reinterpret_cast<const C*>(reinterpret_cast<const unsigned char*>(slot0) + b * kSlotBytes);
  };
  const float k2 = (float)(f.ks2 * k2c);
  // element e of the thread's column from box b: zero outside the kept rows
  // |k1| <= kmax1, else compact row i1 (or i1 - (n - c1) for negative k1)
  auto val = [&](int b, int e, float& k1) {
    const int i1 = j + kG * e;
    const int kf = kfreq(i1, kN);
    k1 = (float)(f.ks1 * kf);
    if (abs(kf) > f.kmax1) return czero<C>();
    const int row = i1 <= f.kmax1 ? i1 : i1 - (kN - f.c1);
    return slot(b)[row * kT + t];
  };
  auto smf = [&](int pos) -> C& { return sm[colq(pos, t)]; };
  auto sync = [] { __syncthreads(); };
  const long long fs_out = (long long)f.t0 * kN * f.c2;
  const long long out_base = (long long)x0 * kN * f.c2 + k2c;
  auto store = [&](int fld, const C (&v)[kE]) {
    if (active) {
#pragma unroll
      for (int e = 0; e < kE; ++e) B[fld * fs_out + out_base + (long long)(j + kG * e) * f.c2] = v[e];
    }
  };
  C a[kE], b[kE], w[kE];
  if (part == 0) {
    // omega0 = i (k1 u2 - k2 u1); u1; u2
#pragma unroll
    for (int e = 0; e < kE; ++e) {
      float k1;
      a[e] = val(0, e, k1);
      b[e] = val(1, e, k1);
      w[e] = cmuli(csub(cscale(b[e], k1), cscale(a[e], k2)));
    }
    fft<kN, kE, +1>(w, j, tw, smf, sync);
    store(3, w);
    fft<kN, kE, +1>(a, j, tw, smf, sync);
    store(1, a);
    fft<kN, kE, +1>(b, j, tw, smf, sync);
    store(2, b);
  } else {
    // omega2 = D1 - i k1 u0; omega1 = i k2 u0 - D2; u0
#pragma unroll
    for (int e = 0; e < kE; ++e) {
      float k1;
      a[e] = val(0, e, k1);
      b[e] = val(1, e, k1);
      w[e] = csub(b[e], cmuli(cscale(a[e], k1)));
    }
    fft<kN, kE, +1>(w, j, tw, smf, sync);
    store(5, w);
#pragma unroll
    for (int e = 0; e < kE; ++e) {
      float k1;
      b[e] = val(2, e, k1);
      w[e] = csub(cmuli(cscale(a[e], k2)), b[e]);
    }
    fft<kN, kE, +1>(w, j, tw, smf, sync);
    store(4, w);
    fft<kN, kE, +1>(a, j, tw, smf, sync);
    store(0, a);
  }
}

}  // namespace

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

bool p2t_supported(const FGeo& f) {
  // axis-1 length 256 with the 2/3 rule (c1 = 171 kept rows), one box per
  // field of a tile; A's row stride must be a multiple of 16 bytes
  return f.t1 == kN && f.n1 == kN && f.c1 == kMaxRows && f.nmem == 1 &&
         (2 * f.c2 * (int)sizeof(float)) % 16 == 0 && encode_fn() != nullptr;
}

cudaError_t p2t_launch(const float2* A, float2* B, const FGeo& f, const float2* tw, int* err,
                       cudaStream_t st) {
  if (!p2t_supported(f)) return cudaErrorInvalidValue;
  CUtensorMap map;
  // A as floats: x = 2 c2 (a complex is two floats), y = c1 rows, z = 5 t0 planes
  const cuuint64_t dims[3] = {(cuuint64_t)(2 * f.c2), (cuuint64_t)f.c1,
                              (cuuint64_t)(5 * f.t0)};
  const cuuint64_t strides[2] = {(cuuint64_t)(2 * f.c2) * sizeof(float),
                                 (cuuint64_t)(2 * f.c2) * f.c1 * sizeof(float)};
  const cuuint32_t box[3] = {2 * kT, (cuuint32_t)f.c1, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(A),
                                 dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(k_p2t, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSmem);
  if (e != cudaSuccess) return e;
  const int tiles = (f.c2 + kT - 1) / kT;
  const dim3 grid((unsigned)(tiles * f.t0), 2);
  k_p2t<<<grid, dim3(kT, kG), kSmem, st>>>(map, B, f, tw, err, tiles);
  return launched();
}

}  // namespace pf
