// Operator entry points with the reference functions' semantics on device
// arrays (math.py:4-100, space_solver.py:15-64, time_integrator.py:36-318).
#include <cmath>
#include <string>

#include "../../include/periodicflow_b200.h"
#include "pf_common.cuh"

using namespace pf;

namespace {

unsigned nblk(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

#define GRID_LOOP(i, n)                                                          \
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (n); \
       i += (long long)gridDim.x * blockDim.x)

template <typename R>
__global__ void k_op_cross(R* c, const R* a, const R* b, long long P, int d) {
  GRID_LOOP(p, P) {
    if (d == 2) {
      const R w = b[p];
      const R a0 = a[p], a1 = a[P + p];
      c[p] = a1 * w;
      c[P + p] = -a0 * w;
    } else {
      const R a0 = a[p], a1 = a[P + p], a2 = a[2 * P + p];
      const R b0 = b[p], b1 = b[P + p], b2 = b[2 * P + p];
      c[p] = a1 * b2 - a2 * b1;
      c[P + p] = a2 * b0 - a0 * b2;
      c[2 * P + p] = a0 * b1 - a1 * b0;
    }
  }
}

template <typename R>
__global__ void k_op_curl(cx<R>* c, const R* k, const cx<R>* a, long long P, int d) {
  GRID_LOOP(p, P) {
    if (d == 2) {
      c[p] = cmuli(csub(cscale(a[P + p], k[p]), cscale(a[p], k[P + p])));
    } else {
      const R k0 = k[p], k1 = k[P + p], k2 = k[2 * P + p];
      const cx<R> a0 = a[p], a1 = a[P + p], a2 = a[2 * P + p];
      c[p] = cmuli(csub(cscale(a2, k1), cscale(a1, k2)));
      c[P + p] = cmuli(csub(cscale(a0, k2), cscale(a2, k0)));
      c[2 * P + p] = cmuli(csub(cscale(a1, k0), cscale(a0, k1)));
    }
  }
}

template <typename R>
__global__ void k_op_linop(cx<R>* Lu, const R* L, const cx<R>* u, long long P, int nc) {
  GRID_LOOP(p, P) {
    const R l = L[p];
    for (int i = 0; i < nc; ++i) Lu[i * P + p] = cscale(u[i * P + p], l);
  }
}

template <typename R>
__global__ void k_op_leray(cx<R>* u, const R* k, const R* kk2, cx<R>* ph, long long P, int d) {
  GRID_LOOP(p, P) {
    cx<R> s = czero<cx<R>>();
    for (int i = 0; i < d; ++i) s = cadd(s, cscale(u[i * P + p], kk2[i * P + p]));
    if (ph) ph[p] = s;
    for (int i = 0; i < d; ++i) u[i * P + p] = csub(u[i * P + p], cscale(s, k[i * P + p]));
  }
}

template <typename R>
__global__ void k_op_sym(cx<R>* ws, const cx<R>* w, long long P, int d) {
  const R f = (R)0.70710678118654752440;
  GRID_LOOP(p, P) {
    for (int a = 0; a < d; ++a)
      for (int b = 0; b < d; ++b)
        ws[(a * d + b) * P + p] = cscale(cadd(w[(a * d + b) * P + p], w[(b * d + a) * P + p]), f);
  }
}

template <typename R>
__global__ void k_op_ndiv(cx<R>* noise, const cx<R>* ws, const R* k, long long P, int d) {
  GRID_LOOP(p, P) {
    for (int a = 0; a < d; ++a) {
      cx<R> acc = czero<cx<R>>();
      for (int b = 0; b < d; ++b) acc = cadd(acc, cscale(ws[(a * d + b) * P + p], k[b * P + p]));
      noise[a * P + p] = cmuli(acc);
    }
  }
}

template <typename R>
__global__ void k_op_step(int integ, int stage, R dt, long long n, long long npc, cx<R>* unew,
                          const cx<R>* u0, const cx<R>* Nl, cx<R>* Lu, const cx<R>* f,
                          const cx<R>* xi, const R* L) {
  GRID_LOOP(i, n) {
    const cx<R> a0 = u0[i], N = Nl[i], fo = f[i];
    const cx<R> z = xi ? xi[i] : czero<cx<R>>();
    cx<R> r;
    switch (integ) {
      case PF_EXPLICIT_PC: {  // time_integrator.py:51-56
        const R a = stage == 0 ? R(0.5) : R(1.0);
        r = cadd(cadd(a0, cscale(cadd(cadd(N, Lu[i]), fo), a * dt)), cscale(z, sqrt(R(0.5) * dt)));
        break;
      }
      case PF_IMPLICIT_PC: {  // time_integrator.py:111-119
        const R a = stage == 0 ? R(0.5) : R(1.0), b = stage == 0 ? R(0.0) : R(0.5);
        const R l = L[i % npc];
        if (stage == 1) Lu[i] = cscale(a0, l);
        const R ainv = R(1) / (R(1) - dt / R(2) * l);
        cx<R> s = cadd(a0, cscale(cadd(N, fo), a * dt));
        s = cadd(s, cscale(Lu[i], b * dt));
        s = cadd(s, cscale(z, sqrt(R(0.5) * dt)));
        r = cscale(s, ainv);
        break;
      }
      case PF_RK2: {  // time_integrator.py:178-180
        const R a = stage == 0 ? R(0.0) : R(0.5), b = stage == 0 ? R(1.0) : R(0.5);
        r = cadd(cscale(a0, a), cscale(cadd(unew[i], cscale(cadd(cadd(N, Lu[i]), fo), dt)), b));
        break;
      }
      case PF_RK3: {  // time_integrator.py:236-241
        const R as[3] = {R(0), R(0.75), R(1.0 / 3.0)}, bs[3] = {R(1), R(0.25), R(2.0 / 3.0)};
        const R a = as[stage], b = bs[stage];
        cx<R> s = cadd(unew[i], cscale(cadd(cadd(N, Lu[i]), fo), dt));
        s = cadd(s, cscale(z, sqrt(dt)));
        r = cadd(cscale(a0, a), cscale(s, b));
        break;
      }
      default: {  // PF_RK4, time_integrator.py:292-293
        const R al[4] = {R(0.25), R(1.0 / 3.0), R(0.5), R(1.0)};
        r = cadd(a0, cscale(cadd(cadd(N, Lu[i]), fo), al[stage] * dt));
        break;
      }
    }
    unew[i] = r;
  }
}

long long prod(int dim, const long long* shape) {
  long long p = 1;
  for (int i = 0; i < dim; ++i) p *= shape[i];
  return p;
}

int check(int precision, int dim, const long long* shape) {
  if (precision != PF_FP32 && precision != PF_FP64) return PF_ERR_INVALID;
  if (dim != 2 && dim != 3) return PF_ERR_INVALID;
  if (!shape) return PF_ERR_INVALID;
  for (int i = 0; i < dim; ++i)
    if (shape[i] <= 0) return PF_ERR_INVALID;
  return PF_OK;
}

int status() { return cudaGetLastError() == cudaSuccess ? PF_OK : PF_ERR_CUDA; }

}  // namespace

extern "C" {

int pf_op_cross(int prec, int dim, const long long* shape, void* c, const void* a, const void* b,
                void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_cross<double><<<nblk(P), 256, 0, st>>>((double*)c, (const double*)a, (const double*)b, P, dim);
  else k_op_cross<float><<<nblk(P), 256, 0, st>>>((float*)c, (const float*)a, (const float*)b, P, dim);
  return status();
}

int pf_op_curl(int prec, int dim, const long long* shape, void* c, const void* k, const void* a,
               void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_curl<double><<<nblk(P), 256, 0, st>>>((double2*)c, (const double*)k, (const double2*)a, P, dim);
  else k_op_curl<float><<<nblk(P), 256, 0, st>>>((float2*)c, (const float*)k, (const float2*)a, P, dim);
  return status();
}

int pf_op_apply_linear_operator(int prec, int dim, const long long* shape, void* Lu,
                                const void* L, const void* u, void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_linop<double><<<nblk(P), 256, 0, st>>>((double2*)Lu, (const double*)L, (const double2*)u, P, dim);
  else k_op_linop<float><<<nblk(P), 256, 0, st>>>((float2*)Lu, (const float*)L, (const float2*)u, P, dim);
  return status();
}

int pf_op_leray_projection(int prec, int dim, const long long* shape, void* u, const void* k,
                           const void* kk2, void* p_hat, void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_leray<double><<<nblk(P), 256, 0, st>>>((double2*)u, (const double*)k, (const double*)kk2, (double2*)p_hat, P, dim);
  else k_op_leray<float><<<nblk(P), 256, 0, st>>>((float2*)u, (const float*)k, (const float*)kk2, (float2*)p_hat, P, dim);
  return status();
}

int pf_op_symmetrize(int prec, int dim, const long long* shape, void* ws, const void* w,
                     void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_sym<double><<<nblk(P), 256, 0, st>>>((double2*)ws, (const double2*)w, P, dim);
  else k_op_sym<float><<<nblk(P), 256, 0, st>>>((float2*)ws, (const float2*)w, P, dim);
  return status();
}

int pf_op_noise_divergence(int prec, int dim, const long long* shape, void* noise,
                           const void* ws, const void* k, void* stream) {
  if (int rc = check(prec, dim, shape)) return rc;
  const long long P = prod(dim, shape);
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64) k_op_ndiv<double><<<nblk(P), 256, 0, st>>>((double2*)noise, (const double2*)ws, (const double*)k, P, dim);
  else k_op_ndiv<float><<<nblk(P), 256, 0, st>>>((float2*)noise, (const float2*)ws, (const float*)k, P, dim);
  return status();
}

int pf_op_stepping(int prec, int integ, int stage, double dt, long long n, void* unew,
                   const void* u0, const void* Nl, void* Lu, const void* f, const void* xi,
                   const void* L, long long npc, void* stream) {
  if (prec != PF_FP32 && prec != PF_FP64) return PF_ERR_INVALID;
  if (integ < PF_EXPLICIT_PC || integ > PF_RK4 || stage < 0) return PF_ERR_INVALID;
  const int nst[5] = {2, 2, 2, 3, 4};
  if (stage >= nst[integ]) return PF_ERR_INVALID;
  if (integ == PF_IMPLICIT_PC && (!L || npc <= 0)) return PF_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (prec == PF_FP64)
    k_op_step<double><<<nblk(n), 256, 0, st>>>(integ, stage, dt, n, npc, (double2*)unew, (const double2*)u0,
                                               (const double2*)Nl, (double2*)Lu, (const double2*)f,
                                               (const double2*)xi, (const double*)L);
  else
    k_op_step<float><<<nblk(n), 256, 0, st>>>(integ, stage, (float)dt, n, npc, (float2*)unew, (const float2*)u0,
                                              (const float2*)Nl, (float2*)Lu, (const float2*)f,
                                              (const float2*)xi, (const float*)L);
  return status();
}

}  // extern "C"
