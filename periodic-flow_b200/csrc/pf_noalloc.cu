// Backward transform for callers that must not allocate device memory.
//
// Some callers of this library cannot call cudaMalloc: code that runs in a
// pre-sized memory budget (an embedding application that hands the library a
// fixed pool), hosts whose allocator must not be entered from the calling
// thread (a real-time or callback context), or integrations where every
// device allocation has to be accounted for up front.  pf_backward_noalloc
// gives them the backward transform (spectral -> physical, the reference's
// V.backward) without any allocation: the spectral work copy that the
// transform destroys in place lives in a file-scope device array of fixed size
// that every GPU loading this library holds until the process exits.
//
// Rules of use:
//  * at most kNoAllocScratchBytes (32 MiB) of work copy: dim * nspec complex
//    values of the requested precision; larger requests are rejected;
//  * the first call on a device (with that device current) looks up the
//    array's device address with cudaGetSymbolAddress and fills the FFT
//    twiddle tables; make that first call before any stream capture;
//  * all calls share the one array: calls that overlap on the GPU (different
//    streams, or the same array from several host threads) race; serialise
//    them on one stream;
//  * the array keeps the previous call's contents; the transform overwrites
//    every element it reads, so nothing has to start at zero.
#include <mutex>
#include <string>
#include <vector>

#include "../../include/periodicflow_b200.h"
#include "pf_internal.h"

namespace pf {

static constexpr size_t kNoAllocScratchBytes = 32ull << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// device address of g_noalloc_scratch per device (host code may not use the
// symbol itself as a device pointer)
static std::mutex s_mu;
static std::vector<void*> s_scratch;

static int scratch_for_device(void** out, std::string* err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return PF_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lk(s_mu);
  if ((int)s_scratch.size() > dev && s_scratch[dev]) {
    *out = s_scratch[dev];
    return PF_OK;
  }
  e = ensure_tables();
  if (e != cudaSuccess) {
    *err = std::string("twiddle tables: ") + cudaGetErrorString(e);
    return PF_ERR_CUDA;
  }
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) {
    *err = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
    return PF_ERR_CUDA;
  }
  if ((int)s_scratch.size() <= dev) s_scratch.resize(dev + 1, nullptr);
  s_scratch[dev] = p;
  *out = p;
  return PF_OK;
}

template <typename R>
static cudaError_t backward_into(int dim, const int* n, const cx<R>* u_hat, R* u, cx<R>* X,
                                 long long nspec, cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(X, u_hat, sizeof(cx<R>) * (size_t)dim * nspec,
                                  cudaMemcpyDeviceToDevice, st);
  if (e != cudaSuccess) return e;
  if (dim == 3) {
    const int nh = n[2] / 2 + 1;
    const long long plane = (long long)n[1] * nh;
    e = fft_strided<R>(X, n[0], +1, plane, dim, nspec, plane, 1.0, st);
    if (e != cudaSuccess) return e;
    e = fft_strided<R>(X, n[1], +1, nh, (long long)dim * n[0], plane, nh, 1.0, st);
    if (e != cudaSuccess) return e;
    return fft_c2r_last<R>(X, u, n[2], (long long)dim * n[0] * n[1], nh, n[2], st);
  }
  const int nh = n[1] / 2 + 1;
  e = fft_strided<R>(X, n[0], +1, nh, dim, nspec, nh, 1.0, st);
  if (e != cudaSuccess) return e;
  return fft_c2r_last<R>(X, u, n[1], (long long)dim * n[0], nh, n[1], st);
}

}  // namespace pf

using namespace pf;

extern "C" int pf_backward_noalloc(int precision, int dim, const int* n, const void* u_hat,
                                   void* u, void* stream) {
  if (precision != PF_FP32 && precision != PF_FP64)
    return set_static_error(PF_ERR_INVALID, "pf_backward_noalloc: precision must be PF_FP32 or PF_FP64");
  if ((dim != 2 && dim != 3) || !n)
    return set_static_error(PF_ERR_INVALID, "pf_backward_noalloc: dim must be 2 or 3 with n given");
  if (!u_hat || !u) return set_static_error(PF_ERR_INVALID, "pf_backward_noalloc: null array");
  long long nspec = 1;
  for (int a = 0; a < dim; ++a) {
    if (!fft_length_supported(n[a]))
      return set_static_error(PF_ERR_UNSUPPORTED,
                              "pf_backward_noalloc: grid size " + std::to_string(n[a]) +
                                  " not built: sides 2^b from 4 to 1024 and 3 * 2^b from 12 to 768 are supported");
    nspec *= (a == dim - 1) ? (n[a] / 2 + 1) : n[a];
  }
  const size_t cbytes = precision == PF_FP64 ? 16 : 8;
  const size_t need = cbytes * (size_t)dim * (size_t)nspec;
  if (need > kNoAllocScratchBytes)
    return set_static_error(PF_ERR_INVALID,
                            "pf_backward_noalloc: needs " + std::to_string(need) +
                                " bytes of work space, more than the fixed " +
                                std::to_string(kNoAllocScratchBytes) +
                                "-byte scratch; use pf_get_physical on a solver handle");
  void* scratch = nullptr;
  std::string err;
  int rc = scratch_for_device(&scratch, &err);
  if (rc) return set_static_error(rc, "pf_backward_noalloc: " + err);
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e =
      precision == PF_FP64
          ? backward_into<double>(dim, n, (const double2*)u_hat, (double*)u, (double2*)scratch, nspec, st)
          : backward_into<float>(dim, n, (const float2*)u_hat, (float*)u, (float2*)scratch, nspec, st);
  if (e != cudaSuccess)
    return set_static_error(PF_ERR_CUDA, std::string("pf_backward_noalloc: ") + cudaGetErrorString(e));
  return PF_OK;
}
