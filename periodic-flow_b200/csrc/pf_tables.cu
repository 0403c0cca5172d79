// Twiddle tables of the FFT engine, one static copy per device.
#include <atomic>
#include <cmath>
#include <mutex>
#include <vector>

#include "pf_fft.cuh"
#include "pf_internal.h"

namespace pf {

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_total() { return g_launches.load(std::memory_order_relaxed); }

static __device__ float2 g_tw_f32[kTwSize];
static __device__ double2 g_tw_f64[kTwSize];

// Device addresses of the tables, one slot per device.  Fixed arrays of
// atomics: tw_base() reads a slot without the set-up mutex while another host
// thread may be setting up a different device, so nothing here is ever
// reallocated.
constexpr int kMaxDevices = 64;
static std::atomic<const float2*> s_tw32[kMaxDevices];
static std::atomic<const double2*> s_tw64[kMaxDevices];

// exp(-2 pi i m / n) in FP64, evaluated on the first octant and mapped by
// symmetry so every entry is as accurate as the host sin/cos near zero.
static void root_of_unity(long m, long n, double* c, double* s) {
  // reduce m/n to [0, 1/8] and reflect
  long a = (8 * m) / n;  // octant
  double ang;
  const double t = 2.0 * M_PI / (double)n;
  long mm = m;
  double cc, ss;
  switch (a) {
    case 0: ang = t * mm; cc = cos(ang); ss = sin(ang); break;
    case 1: ang = t * ((double)n / 4 - mm); cc = sin(ang); ss = cos(ang); break;
    case 2: ang = t * (mm - (double)n / 4); cc = -sin(ang); ss = cos(ang); break;
    case 3: ang = t * ((double)n / 2 - mm); cc = -cos(ang); ss = sin(ang); break;
    case 4: ang = t * (mm - (double)n / 2); cc = -cos(ang); ss = -sin(ang); break;
    case 5: ang = t * (3.0 * n / 4 - mm); cc = -sin(ang); ss = -cos(ang); break;
    case 6: ang = t * (mm - 3.0 * n / 4); cc = sin(ang); ss = -cos(ang); break;
    default: ang = t * ((double)n - mm); cc = cos(ang); ss = -sin(ang); break;
  }
  *c = cc;
  *s = -ss;  // exp(-i theta)
}

cudaError_t ensure_tables() {
  static std::mutex mu;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (s_tw32[dev].load(std::memory_order_acquire) && s_tw64[dev].load(std::memory_order_acquire))
    return cudaSuccess;
  std::vector<float2> f(kTwSize);
  std::vector<double2> d(kTwSize);
  auto fill = [&](int n) {
    const int off = tw_offset(n);
    for (int m = 0; m < n; ++m) {
      double c, s;
      root_of_unity(m, n, &c, &s);
      d[off + m] = make_double2(c, s);
      f[off + m] = make_float2((float)c, (float)s);
    }
  };
  for (int n = 2; n <= kMaxFFT; n *= 2) fill(n);
  for (int n = 12; n <= kMax3FFT; n *= 2) fill(n);
  e = cudaMemcpyToSymbol(g_tw_f32, f.data(), sizeof(float2) * kTwSize);
  if (e != cudaSuccess) return e;
  e = cudaMemcpyToSymbol(g_tw_f64, d.data(), sizeof(double2) * kTwSize);
  if (e != cudaSuccess) return e;
  void* p32 = nullptr;
  void* p64 = nullptr;
  e = cudaGetSymbolAddress(&p32, g_tw_f32);
  if (e != cudaSuccess) return e;
  e = cudaGetSymbolAddress(&p64, g_tw_f64);
  if (e != cudaSuccess) return e;
  s_tw64[dev].store((const double2*)p64, std::memory_order_release);
  s_tw32[dev].store((const float2*)p32, std::memory_order_release);
  return cudaSuccess;
}

template <> const float2* tw_base<float>() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  return s_tw32[dev].load(std::memory_order_acquire);
}
template <> const double2* tw_base<double>() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  return s_tw64[dev].load(std::memory_order_acquire);
}

}  // namespace pf
