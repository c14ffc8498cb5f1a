// Force-bias auxiliary fields: X = probit(u) + i (clamp(vbias) - clamp(vMF)), the hybrid weight
// HW[w] = sum_n -vdiff (X - vdiff/2) and the mean-field factor mf[w] = -Re(vMF.vMF)/2 +
// i sum_n X vMF, fused into one pass over the [W][Nc] fields.
//
// Reference: construct_X_impl (src/AFQMC/Propagators/construct_X_kernel.hpp:20-89, continuous
// charge fields, no force-bias projection), assemble_X (Propagators/AFQMCBasePropagator.cpp:
// 686-733), meanfield_factor (AFQMCBasePropagator.cpp:334-336) and probit (src/AFQMC/Utilities/
// probit.h:57-135, Acklam's rational approximation of the inverse normal CDF).  The reference
// reduces HW with atomics; here each walker's row is one CTA and the sums are block reductions.
//
// Field uniforms come either from a caller buffer (the reference's host-generated RNGbuff) or from
// a counter-based Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw, SC'11) evaluated in place,
// so no uniform buffer is written to or read from HBM.
#include "fields.cuh"

namespace afqmc {
namespace {

__device__ __forceinline__ double probit(double p) {
  // coefficients of Acklam's published approximation
  const double a0 = -3.969683028665376e+01, a1 = 2.209460984245205e+02,
               a2 = -2.759285104469687e+02, a3 = 1.383577518672690e+02,
               a4 = -3.066479806614716e+01, a5 = 2.506628277459239e+00;
  const double b0 = -5.447609879822406e+01, b1 = 1.615858368580409e+02,
               b2 = -1.556989798598866e+02, b3 = 6.680131188771972e+01,
               b4 = -1.328068155288572e+01;
  const double c0 = -7.784894002430293e-03, c1 = -3.223964580411365e-01,
               c2 = -2.400758277161838e+00, c3 = -2.549732539343734e+00,
               c4 = 4.374664141464968e+00, c5 = 2.938163982698783e+00;
  const double d0 = 7.784695709041462e-03, d1 = 3.224671290700398e-01,
               d2 = 2.445134137142996e+00, d3 = 3.754408661907416e+00;
  if (p < 0 || p > 1) return 0.0;
  if (p == 0) return -HUGE_VAL;
  if (p == 1) return HUGE_VAL;
  if (p < 0.02425) {
    double q = sqrt(-2 * log(p));
    return (((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
           ((((d0 * q + d1) * q + d2) * q + d3) * q + 1);
  }
  if (p > 0.97575) {
    double q = sqrt(-2 * log(1 - p));
    return -(((((c0 * q + c1) * q + c2) * q + c3) * q + c4) * q + c5) /
           ((((d0 * q + d1) * q + d2) * q + d3) * q + 1);
  }
  double q = p - 0.5, r = q * q;
  return (((((a0 * r + a1) * r + a2) * r + a3) * r + a4) * r + a5) * q /
         (((((b0 * r + b1) * r + b2) * r + b3) * r + b4) * r + 1);
}

__device__ __forceinline__ c128 clamp_mag(c128 v, double bound) {
  double a = cabs(v);
  return a > bound ? cscale(v, bound / a) : v;
}

constexpr int FX_THREADS = 256;

template <bool DEVICE_RNG>
__global__ void __launch_bounds__(FX_THREADS)
    construct_x_kernel(const c128* __restrict__ vbias, long ldv, const double* __restrict__ u,
                       long ldu, const c128* __restrict__ vMF, c128* __restrict__ X, long ldx,
                       c128* __restrict__ HW, c128* __restrict__ mf, int Nc, double vbias_bound,
                       double half_re_vmf2, unsigned long long seed,
                       const unsigned long long* __restrict__ counter) {
  const long w = blockIdx.x;
  const c128* vb = vbias + w * ldv;
  c128* Xw = X + w * ldx;
  c128 hw = cmk(0, 0), xv = cmk(0, 0);
  const unsigned long long step = DEVICE_RNG ? *counter : 0ull;
  for (int n2 = threadIdx.x; 2 * n2 < Nc; n2 += FX_THREADS) {
    double uu[2];
    if constexpr (DEVICE_RNG) {
      philox_uniform2(seed, step, (unsigned)w, (unsigned)n2, uu);
    } else {
      uu[0] = u[w * ldu + 2 * n2];
      uu[1] = (2 * n2 + 1 < Nc) ? u[w * ldu + 2 * n2 + 1] : 0.5;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = 2 * n2 + h;
      if (n >= Nc) break;
      const c128 vmf0 = vMF[n];
      const c128 vmf_t = clamp_mag(vmf0, vbias_bound);
      const c128 vb_t = clamp_mag(vb[n], vbias_bound);
      const c128 vdiff = cmul(cmk(0, 1), csub(vb_t, vmf_t));
      const c128 x = cadd(cmk(probit(uu[h]), 0.0), vdiff);
      Xw[n] = x;
      hw = cadd(hw, cmul(cmk(-vdiff.x, -vdiff.y), csub(x, cscale(vdiff, 0.5))));
      xv = cadd(xv, cmul(x, vmf0));
    }
  }
  __shared__ double red[4][FX_THREADS / 32];
  double vals[4] = {hw.x, hw.y, xv.x, xv.y};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double v = vals[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q)
      for (int k = 0; k < FX_THREADS / 32; ++k) t[q] += red[q][k];
    HW[w] = cmk(t[0], t[1]);
    // mf = -0.5 Re(vMF.vMF) + im * (X.vMF)
    mf[w] = cmk(half_re_vmf2 - t[3], t[2]);
  }
}

__global__ void advance_counter_kernel(unsigned long long* counter) { *counter += 1ull; }

}  // namespace

int construct_x(cudaStream_t s, const c128* vbias, long ldv, const double* u, long ldu,
                const c128* vMF, c128* X, long ldx, c128* HW, c128* mf, int W, int Nc,
                double vbias_bound, double half_re_vmf2, unsigned long long seed,
                unsigned long long* counter) {
  if (W <= 0) return AFQMC_OK;
  if (u) {
    construct_x_kernel<false><<<W, FX_THREADS, 0, s>>>(vbias, ldv, u, ldu, vMF, X, ldx, HW, mf,
                                                       Nc, vbias_bound, half_re_vmf2, 0ull,
                                                       nullptr);
  } else {
    if (!counter) {
      set_error_detail("construct_x: device RNG needs a counter");
      return AFQMC_ERR_ARG;
    }
    construct_x_kernel<true><<<W, FX_THREADS, 0, s>>>(vbias, ldv, nullptr, 0, vMF, X, ldx, HW, mf,
                                                      Nc, vbias_bound, half_re_vmf2, seed,
                                                      counter);
    AFQMC_TRY(launch_status("construct_x_kernel"));
    advance_counter_kernel<<<1, 1, 0, s>>>(counter);
  }
  return launch_status("construct_x_kernel");
}

}  // namespace afqmc
