// Instantiation unit of the fused 3D passes: FP32, 2/3 rule.
#include "pf_fused_impl.cuh"

namespace pf {

cudaError_t fused_pass_f32_trunc(FusedPlan* p, int pass, const void* uhat, void* nl,
                                 unsigned long long* maxbits, cudaStream_t st) {
  return pass_trunc<float>(p, pass, uhat, nl, maxbits, st);
}

cudaError_t fused_update_f32_trunc(FusedPlan* p, const UpdateArgs<float>& U, int ncomp,
                                   const void* nl, cudaStream_t st) {
  return update_trunc<float>(p, U, ncomp, nl, st);
}

}  // namespace pf
