// Instantiation unit of the fused 3D passes: FP64, 2/3 rule.
#include "pf_fused_impl.cuh"

namespace pf {

cudaError_t fused_pass_f64_trunc(FusedPlan* p, int pass, const void* uhat, void* nl,
                                 unsigned long long* maxbits, cudaStream_t st) {
  return pass_trunc<double>(p, pass, uhat, nl, maxbits, st);
}

cudaError_t fused_update_f64_trunc(FusedPlan* p, const UpdateArgs<double>& U, int ncomp,
                                   const void* nl, cudaStream_t st) {
  return update_trunc<double>(p, U, ncomp, nl, st);
}

}  // namespace pf
