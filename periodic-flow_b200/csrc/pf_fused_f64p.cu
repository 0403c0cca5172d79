// Instantiation unit of the fused 3D passes: FP64, 3/2 rule.
#include "pf_fused_impl.cuh"

namespace pf {

cudaError_t fused_pass_f64_pad(FusedPlan* p, int pass, const void* uhat,
                               unsigned long long* maxbits, cudaStream_t st) {
  return pass_pad<double>(p, pass, uhat, maxbits, st);
}

cudaError_t fused_update_f64_pad(FusedPlan* p, const UpdateArgs<double>& U, int ncomp,
                                 cudaStream_t st) {
  return update_pad<double>(p, U, ncomp, st);
}

}  // namespace pf
