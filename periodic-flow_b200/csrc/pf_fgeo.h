// Geometry of the fused 3D pencil schedule, shared by pf_fused.cu and the
// separately compiled pass kernels (pf_p3q.cu).
#pragma once
#include "pf_common.cuh"

namespace pf {

struct FGeo {
  int n0, n1, n2, nh;          // N grid (the state's grid)
  int t0, t1, t2;              // transform lengths: n_i (2/3 rule) or 3 n_i / 2 (3/2 rule)
  int c1, c2;                  // compact inverse-input extents along axes 1, 2
  int kmax0, kmax1, kmax2;
  double ks0, ks1, ks2;
  double cflw0, cflw1, cflw2;  // n_i / L_i
  long long nspec;
  int nlrow;                   // nl row stride along axis 0 (t1 nh)
  long long nlcomp;            // nl component stride (t0 t1 nh)
  // Members: boxes of this geometry laid out one after another in every
  // buffer (state 3 nspec, nl 3 nlcomp, A 5 t0 c1 c2, B 6 t0 t1 c2 complex
  // values per member); each pass covers all of them in one launch.
  int nmem;
  // P1's five-row and P2's six-row forms: 1 numbers a CTA's output field
  // fastest (blockIdx.x = tile * fields + field), so the CTAs of one column
  // tile run together and their shared input rows are re-read from L2; 0:
  // the field is blockIdx.y
  int ilv;
  // Slab decomposition of one box over sl_S slabs (pf_slab.cu; unused by the
  // whole-box passes): slab r holds the spectral rows k1 in [r sl_n1,
  // (r + 1) sl_n1) of every (k0, k2) and, between the two exchanges, the
  // physical planes x0 in [r sl_n0, (r + 1) sl_n0).  P1 of a slab transforms
  // its kept compact rows [sl_c0, sl_c0 + sl_nc) and stores plane x0 straight
  // into slab x0 / sl_n0's pass-1 buffer sl_dst[x0 / sl_n0]; P4 stores row k1
  // into slab k1 / sl_n1's nonlinear buffer.  sl_dst may be another GPU's
  // memory (peer mapping): plain stores only.
  int sl_S, sl_n0, sl_n1, sl_x0, sl_i1, sl_c0, sl_nc, sl_N0;
  void* sl_dst[8];
};
constexpr int kMaxSlabs = 8;

// P3 of the 2/3 rule in FP32 with one shared-memory exchange per line FFT
// (pf_p3q.cu): contiguous sides n2 = 128 or 256, W warps per CTA (6 or 7),
// one CTA per SM, at most nsm CTAs.  B, nl, maxbits, err as for the other P3
// forms.
cudaError_t p3q_launch(int n2, int W, const float2* B, float2* nl, const FGeo& f,
                       const float2* tw, unsigned long long* maxbits, float scale, int* err,
                       long long ngroups, int nsm, cudaStream_t st);
bool p3q_supported(int n2, int W);

// P2 of the 2/3 rule in FP32 at axis-1 length 256 with tiled bulk tensor
// copies of its input tiles (pf_p2t.cu); one box: single-box plans only.
cudaError_t p2t_launch(const float2* A, float2* B, const FGeo& f, const float2* tw, int* err,
                       cudaStream_t st);
bool p2t_supported(const FGeo& f);

}  // namespace pf
