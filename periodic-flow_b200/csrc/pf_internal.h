// Host-side internal interface between the C-ABI layer and the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "pf_common.cuh"

struct pf_config;

namespace pf {

// Record the message returned by pf_last_error(NULL); returns code.
int set_static_error(int code, const std::string& msg);
// The checks pf_create applies to a configuration (PF_OK or an error code,
// message via pf_last_error(NULL)), and the box geometry it describes.
int config_validate(const ::pf_config* c);
Geo config_geo(const ::pf_config* c);

struct SolverView;

// kernel launch accounting: every launcher of this library reports here
void count_launch();
void add_launches(long long n);
long long launch_total();
inline cudaError_t launched() {
  count_launch();
  return cudaGetLastError();
}

// twiddle tables: filled once per device before any FFT launch
cudaError_t ensure_tables();
// device address of the concatenated tables of the current device; the table
// of length N starts at tw_base<R>() + (N - 2)
template <typename R> const cx<R>* tw_base();

// ---------------------------------------------------------------- FFT passes
// In-place complex FFT along a strided axis.  Column q in [0, nplanes*ncols)
// addresses base + (q / ncols) * plane_stride + (q % ncols); line element i is
// at + i * line_stride (strides in complex elements).
template <typename R>
cudaError_t fft_strided(cx<R>* data, int n, int dir, long long ncols, long long nplanes,
                        long long plane_stride, long long line_stride, double scale,
                        cudaStream_t st);

// Complex-to-real along the contiguous last axis: nlines lines of n/2+1 complex
// (row stride in_stride) -> nlines lines of n reals (row stride out_stride).
template <typename R>
cudaError_t fft_c2r_last(const cx<R>* in, R* out, int n, long long nlines,
                         long long in_stride, long long out_stride, cudaStream_t st);

// Real-to-complex along the last axis, result multiplied by scale.
template <typename R>
cudaError_t fft_r2c_last(const R* in, cx<R>* out, int n, long long nlines,
                         long long in_stride, long long out_stride, double scale,
                         cudaStream_t st);

bool fft_length_supported(int n);

}  // namespace pf
