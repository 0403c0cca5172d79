// Fused pencil passes of the nonlinear term (u x omega with 2/3 truncation).
#pragma once
#include "pf_internal.h"

namespace pf {

struct FusedPlan;

// Returns nullptr when no fused schedule is built for this geometry.
FusedPlan* fused_create(const Geo& g, int precision, int dealias);
void fused_destroy(FusedPlan* p);
// Unprojected nonlinear term of uhat into nl; optional max(sum |u_i|/dx_i)
// as float bits into maxbits.
cudaError_t fused_nonlinear(FusedPlan* p, const void* uhat, void* nl, unsigned long long* maxbits,
                            cudaStream_t st);

}  // namespace pf
