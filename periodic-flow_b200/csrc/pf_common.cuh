// Common device helpers for the periodicflow B200 kernels: complex arithmetic,
// grid descriptors, wavenumbers and mode predicates.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PF_HD __host__ __device__ __forceinline__
#define PF_D __device__ __forceinline__

namespace pf {

template <typename R> struct CT;
template <> struct CT<float> { using T = float2; };
template <> struct CT<double> { using T = double2; };
template <typename R> using cx = typename CT<R>::T;

template <typename R> PF_HD cx<R> mk(R a, R b) { cx<R> z; z.x = a; z.y = b; return z; }
template <typename C> PF_HD C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> PF_HD C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> PF_HD C cmul(C a, C b) {
  C z; z.x = a.x * b.x - a.y * b.y; z.y = a.x * b.y + a.y * b.x; return z;
}
// a * conj(b)
template <typename C> PF_HD C cmulc(C a, C b) {
  C z; z.x = a.x * b.x + a.y * b.y; z.y = a.y * b.x - a.x * b.y; return z;
}
template <typename C, typename R> PF_HD C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
template <typename C> PF_HD C cconj(C a) { a.y = -a.y; return a; }
// multiply by i
template <typename C> PF_HD C cmuli(C a) { C z; z.x = -a.y; z.y = a.x; return z; }
template <typename C> PF_HD C czero() { C z; z.x = 0; z.y = 0; return z; }

// Box geometry shared by all kernels.  Spectral arrays use the reference's
// layout (comp, n0, n1, n2/2+1) in 3D and (comp, n0, n1/2+1) in 2D, dense.
struct Geo {
  int dim;        // 2 or 3
  int n[3];       // physical points per axis (2D: n[0], n[1]; n[2] = 1)
  int nh;         // last-axis spectral extent n_last/2 + 1
  int s[3];       // spectral extents per axis (last one = nh)
  long long nspec;  // modes per scalar spectral field
  long long nphys;  // points per scalar physical field
  double kscale[3]; // 2 pi / L_i
  int kmax[3];      // 2/3 rule: keep |k_i| <= kmax[i]  (3|k| < n)
};

// signed integer wavenumber of index i along a complex (fftfreq) axis
PF_HD int kfreq(int i, int n) { return (i <= (n - 1) / 2) ? i : i - n; }

}  // namespace pf
