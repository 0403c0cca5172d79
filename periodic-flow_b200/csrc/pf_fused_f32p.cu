// Instantiation unit of the fused 3D passes: FP32, 3/2 rule.
#include "pf_fused_impl.cuh"

namespace pf {

cudaError_t fused_pass_f32_pad(FusedPlan* p, int pass, const void* uhat,
                               unsigned long long* maxbits, cudaStream_t st) {
  return pass_pad<float>(p, pass, uhat, maxbits, st);
}

cudaError_t fused_update_f32_pad(FusedPlan* p, const UpdateArgs<float>& U, int ncomp,
                                 cudaStream_t st) {
  return update_pad<float>(p, U, ncomp, st);
}

}  // namespace pf
