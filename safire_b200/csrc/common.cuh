// Shared definitions for the B200 AFQMC walker-step kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "afqmc_c.h"

namespace afqmc {

// complex128 storage: layout-compatible with std::complex<double> and the C-ABI afqmc_c128.
using c128 = double2;

__host__ __device__ __forceinline__ c128 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ c128 cadd(c128 a, c128 b) { return cmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ c128 csub(c128 a, c128 b) { return cmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ c128 cmul(c128 a, c128 b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ c128 cscale(c128 a, double s) { return cmk(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ c128 cconj(c128 a) { return cmk(a.x, -a.y); }
__host__ __device__ __forceinline__ double cabs1(c128 a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ double cabs(c128 a) { return hypot(a.x, a.y); }
// a / b with Smith's scaling
__host__ __device__ __forceinline__ c128 cdiv(c128 a, c128 b) {
  if (fabs(b.x) >= fabs(b.y)) {
    double r = b.y / b.x, d = b.x + r * b.y;
    return cmk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
  } else {
    double r = b.x / b.y, d = b.x * r + b.y;
    return cmk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
  }
}
// principal complex log
__host__ __device__ __forceinline__ c128 clog(c128 a) { return cmk(log(hypot(a.x, a.y)), atan2(a.y, a.x)); }
__host__ __device__ __forceinline__ c128 cexp(c128 a) {
  double e = exp(a.x);
  return cmk(e * cos(a.y), e * sin(a.y));
}

// Error state shared by the C-ABI entry points (thread-local detail string).
void set_error_detail(const char* fmt, ...);
const char* error_detail();

#define AFQMC_CUDA_TRY(expr)                                                               \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      ::afqmc::set_error_detail("%s:%d %s: %s", __FILE__, __LINE__, #expr,                 \
                                cudaGetErrorString(e_));                                   \
      return AFQMC_ERR_CUDA;                                                               \
    }                                                                                      \
  } while (0)

#define AFQMC_CHECK_ARG(cond, ...)                                                         \
  do {                                                                                     \
    if (!(cond)) {                                                                         \
      ::afqmc::set_error_detail(__VA_ARGS__);                                              \
      return AFQMC_ERR_ARG;                                                                \
    }                                                                                      \
  } while (0)

#define AFQMC_TRY(expr)                                                                    \
  do {                                                                                     \
    int s_ = (expr);                                                                       \
    if (s_ != AFQMC_OK) return s_;                                                         \
  } while (0)

// count of kernels launched by this library (exported as afqmc_kernel_launches)
void count_launch();

inline int launch_status(const char* what) {
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error_detail("launch of %s failed: %s", what, cudaGetErrorString(e));
    return AFQMC_ERR_CUDA;
  }
  return AFQMC_OK;
}

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace afqmc
