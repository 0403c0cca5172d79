// Fused passes of the 2D nonlinear term (u x omega with the 2/3 rule).
#pragma once
#include "pf_kernels.h"

namespace pf {

// Geometry of one 2D box as the fused passes see it.
struct F2 {
  int n0, n1, nh;       // physical sides, nh = n1 / 2 + 1
  int kmax0, kmax1;     // 2/3 rule: |k_i| <= kmax_i feed u and omega
  int c1;               // kept columns along the last axis (kmax1 + 1)
  long long nspec;      // n0 * nh
  double ks0, ks1;      // 2 pi / L_i
  double cflw0, cflw1;  // n_i / L_i
  int var[4];           // launch form of Q1..Q3 (0: default, 1: halved radix, sides >= 256)
  int nmem;             // members laid out one after another (state and nl 2 nspec,
                        // pass-1 buffer 3 n0 c1 complex values each), one launch per pass
};

// Sides with a fused 2D schedule: powers of two 16..1024 (FP32 and FP64).
bool fused2d_side(int n);
F2 fused2d_geo(const Geo& g);
size_t fused2d_scratch_elems(const F2& f);  // complex values of the pass-1 buffer

// Q1: inverse FFT along axis 0 of the kept columns of uhat -> A (scratch)
template <typename R>
cudaError_t fused2d_inverse(const F2& f, const cx<R>* uhat, cx<R>* A, cudaStream_t st);
// Q2: per pair of x0 lines, omega, C2R, u x omega (optional CFL max as double
// bits into maxbits), R2C scaled by 1 / (n0 n1) -> nl[2][n0][nh]
template <typename R>
cudaError_t fused2d_products(const F2& f, const cx<R>* A, cx<R>* nl,
                             unsigned long long* maxbits, cudaStream_t st);
// Q3: forward FFT along axis 0 of nl fused with the stage update
template <typename R>
cudaError_t fused2d_update(const F2& f, const UpdateArgs<R>& U, int ncomp, const cx<R>* nl,
                           cudaStream_t st);

}  // namespace pf
