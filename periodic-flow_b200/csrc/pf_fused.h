// Fused pencil passes of the nonlinear term (u x omega): 3D five-pass
// schedule, 2D three-pass schedule (pf_fused2d.cu).
#pragma once
#include "pf_kernels.h"

namespace pf {

struct FusedPlan;

// Returns nullptr when no fused schedule is built for this geometry (3D:
// FP32 2/3 rule, sides 2^b 16..512 with n2 <= 256 and 3 * 2^b 48..384; 3/2
// rule (FP32, FP64) and FP64 2/3 rule, sides 2^b 16..256; 2D: 2/3 rule, FP32
// and FP64, sides 2^b 16..1024).  2D plans run passes 1 and 3 and the update;
// passes 2 and 4 are no-ops there.
// nmem > 1: buffers and launches for nmem boxes of this geometry laid out one
// after another (state, nl and the device scalars of the caller likewise).
FusedPlan* fused_create(const Geo& g, int precision, int dealias, int nmem = 1);
// The pencil plan of one of `slabs` slabs of a 3D box (2/3 rule): passes 2-4
// on n0 / slabs planes x0 (pass-1 buffer A [5][n0/slabs][c1][c2], nl in the
// layout [3][n0/slabs][n1][nh]); pass 3 scales by 1 / (n0 n1 n2).  nullptr
// where fused_create(g, precision, 0) has no plan or slabs does not divide n0.
FusedPlan* fused_create_pencil(const Geo& g, int precision, int slabs);
void fused_destroy(FusedPlan* p);
// Launches of the plan cover members [0, active) (active <= the plan's members).
void fused_set_members(FusedPlan* p, int active);
// Pass 1..4 of the nonlinear term of uhat (unprojected) into nl; pass 3
// writes max(sum_i |u_i| / dx_i) as double bits into maxbits when non-null.
cudaError_t fused_pass(FusedPlan* p, int pass, const void* uhat, void* nl,
                       unsigned long long* maxbits, cudaStream_t st);
// Pass 5: forward FFT along axis 0 of nl fused with the stage update.
cudaError_t fused_update(FusedPlan* p, const UpdateArgs<float>& U, int ncomp, const void* nl,
                         cudaStream_t st);
cudaError_t fused_update(FusedPlan* p, const UpdateArgs<double>& U, int ncomp, const void* nl,
                         cudaStream_t st);

// Times every launch variant of passes 1-4 inside the chain of passes 1-4 on
// this plan's buffers (each pass writes only plan scratch and nl) and keeps
// the fastest; the picks (var[6], var384[6]) also seed later plans of the
// same geometry.  Synchronous.
cudaError_t fused_autotune(FusedPlan* p, const void* uhat, void* nl, cudaStream_t st, int* picks);
void fused_variants(const FusedPlan* p, int* out12);

// Error word of bounded device waits (0: none; synchronous read).
int fused_device_error(FusedPlan* p);

}  // namespace pf
