// Walker-property kernels: the phaseless hybrid update, the weight cap, population-control row
// copies and the estimator sums.
//
// Reference: walker_update / bound_local_energy / bound_walker_weights
// (src/AFQMC/Propagators/WalkerSetUpdate.hpp:46-58, 69-191, 198-218) run there as a host loop
// after staging the properties to the host every step; here the same per-walker formula runs on
// the device, one thread per walker, so a whole step stays on the GPU (and in one CUDA graph).
// population_control (src/AFQMC/Walkers/population_control.hpp:218-255), EnergyEstimator::measure
// (src/AFQMC/Estimators/EnergyEstimator.h:51-100) and averagePseudoEnergy
// (src/AFQMC/Drivers/average_energy.hpp:53-63).
#include "update.cuh"

namespace afqmc {
namespace {

__global__ void walker_update_kernel(c128* __restrict__ buf, long walker_size, long prop0, int W,
                                     const c128* __restrict__ new_ovlp,
                                     const c128* __restrict__ mf, const c128* __restrict__ hw,
                                     double dt, double Eshift_host,
                                     const double* __restrict__ Eshift_dev, double E0,
                                     double lower_cut, double upper_cut, double max_weight,
                                     unsigned long long* __restrict__ stats) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  const double Eshift = Eshift_dev ? *Eshift_dev : Eshift_host;
  c128* p = buf + long(i) * walker_size + prop0;
  const c128 old_ovlp = p[AFQMC_OVLP];
  const c128 old_eloc = p[AFQMC_PSEUDO_ELOC];
  c128 weight = p[AFQMC_WEIGHT];
  c128 phase = p[AFQMC_PHASE];
  const c128 nov = new_ovlp[i];
  const c128 mfi = mf[i];

  const double delta_theta = nov.y - old_ovlp.y - mfi.y;
  const double scale = fmax(0.0, cos(delta_theta));
  // eloc = (mf - hw - (new_ovlp - old_ovlp)) / dt + E0
  c128 eloc = cadd(cscale(csub(csub(mfi, hw[i]), csub(nov, old_ovlp)), 1.0 / dt), cmk(E0, 0.0));
  unsigned long long n_total = 0, n_up = 0, n_lo = 0;
  if (!isfinite(eloc.x)) {
    weight = cmk(0, 0);
    phase = cmk(0, 0);
    eloc = old_eloc;
  } else {
    const double hi = Eshift + upper_cut * sqrt(2.0 / dt);
    const double lo = Eshift - lower_cut * sqrt(2.0 / dt);
    n_total = 1;
    if (eloc.x > hi) n_up = 1;
    else if (eloc.x < lo) n_lo = 1;
    eloc.x = fmin(fmax(eloc.x, lo), hi);
    // w = exp(-dt (eloc - Eshift)); weight *= scale |w|; phase *= w / |w|
    const c128 arg = cscale(cmk(eloc.x - Eshift, eloc.y), -dt);
    const double mag = exp(arg.x);
    const c128 ph = cmk(cos(arg.y), sin(arg.y));
    weight = cscale(weight, scale * mag);
    phase = cmul(phase, ph);
  }
  // bound_walker_weights
  unsigned long long nw_up = 0;
  const double aw = cabs(weight);
  if (aw > max_weight) {
    weight = cscale(weight, max_weight / aw);
    nw_up = 1;
  }
  p[AFQMC_WEIGHT] = weight;
  p[AFQMC_PHASE] = phase;
  p[AFQMC_PSEUDO_ELOC] = eloc;
  p[AFQMC_OVLP] = nov;
  p[AFQMC_THETA] = cmk(delta_theta, 0.0);
  if (stats) {
    if (n_total) atomicAdd(&stats[0], n_total);
    if (n_up) atomicAdd(&stats[1], n_up);
    if (n_lo) atomicAdd(&stats[2], n_lo);
    atomicAdd(&stats[3], 1ull);
    if (nw_up) atomicAdd(&stats[4], nw_up);
  }
}

__global__ void copy_rows_kernel(c128* __restrict__ buf, long walker_size,
                                 const int* __restrict__ dst, const int* __restrict__ src) {
  const int j = blockIdx.x;
  const c128* s = buf + long(src[j]) * walker_size;
  c128* d = buf + long(dst[j]) * walker_size;
  for (long e = threadIdx.x; e < walker_size; e += blockDim.x) d[e] = s[e];
}

__global__ void pack_rows_kernel(const c128* __restrict__ buf, long walker_size,
                                 const int* __restrict__ idx, c128* __restrict__ out) {
  const int j = blockIdx.x;
  const c128* s = buf + long(idx[j]) * walker_size;
  c128* d = out + long(j) * walker_size;
  for (long e = threadIdx.x; e < walker_size; e += blockDim.x) d[e] = s[e];
}

__global__ void unpack_rows_kernel(c128* __restrict__ buf, long walker_size,
                                   const int* __restrict__ idx, const c128* __restrict__ in) {
  const int j = blockIdx.x;
  c128* d = buf + long(idx[j]) * walker_size;
  const c128* s = in + long(j) * walker_size;
  for (long e = threadIdx.x; e < walker_size; e += blockDim.x) d[e] = s[e];
}

__global__ void normalize_weights_kernel(c128* __restrict__ buf, long walker_size, long prop0,
                                         int W) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W) return;
  c128* p = buf + long(i) * walker_size + prop0 + AFQMC_WEIGHT;
  c128 w = *p;
  *p = cscale(w, 1.0 / cabs(w));
}

__global__ void gather_property_kernel(const c128* __restrict__ buf, long walker_size, long off,
                                       int W, c128* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < W) out[i] = buf[long(i) * walker_size + off];
}

__global__ void scatter_property_kernel(c128* __restrict__ buf, long walker_size, long off, int W,
                                        const c128* __restrict__ in) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < W) buf[long(i) * walker_size + off] = in[i];
}

// Weighted sums over walkers in a fixed order (one CTA, deterministic).
template <int NV>
__global__ void __launch_bounds__(1024)
    weighted_sums_kernel(const c128* __restrict__ buf, long walker_size, long prop0, int W,
                         const c128* __restrict__ E, int mode, double dt,
                         c128* __restrict__ out) {
  // mode 0: {w E1, w EXX, w EJ, w} from E [W][3];  mode 1: {w exp(dt eloc), w}
  double acc[2 * NV];
#pragma unroll
  for (int q = 0; q < 2 * NV; ++q) acc[q] = 0.0;
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    const c128* p = buf + long(i) * walker_size + prop0;
    const c128 w = p[AFQMC_WEIGHT];
    c128 v[NV];
    if (mode == 0) {
      for (int q = 0; q < 3 && q < NV; ++q) v[q] = cmul(w, E[long(i) * 3 + q]);
    } else {
      v[0] = cmul(w, cexp(cscale(p[AFQMC_PSEUDO_ELOC], dt)));
    }
    v[NV - 1] = w;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      acc[2 * q] += v[q].x;
      acc[2 * q + 1] += v[q].y;
    }
  }
  __shared__ double red[2 * NV][32];
#pragma unroll
  for (int q = 0; q < 2 * NV; ++q) {
    double v = acc[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 2 * NV) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; ++k) t += red[threadIdx.x][k];
    reinterpret_cast<double*>(out)[threadIdx.x] = t;
  }
}

}  // namespace

int walker_update(cudaStream_t s, c128* buf, long walker_size, long prop0, int W,
                  const c128* new_ovlp, const c128* mf, const c128* hw, double dt, double Eshift,
                  const double* Eshift_dev, double E0, double lower_cut, double upper_cut,
                  double max_weight, unsigned long long* stats) {
  if (W <= 0) return AFQMC_OK;
  walker_update_kernel<<<ceil_div(W, 128), 128, 0, s>>>(buf, walker_size, prop0, W, new_ovlp, mf,
                                                        hw, dt, Eshift, Eshift_dev, E0, lower_cut,
                                                        upper_cut, max_weight, stats);
  return launch_status("walker_update_kernel");
}

int copy_rows(cudaStream_t s, c128* buf, long walker_size, const int* dst, const int* src, int n) {
  if (n <= 0) return AFQMC_OK;
  copy_rows_kernel<<<n, 256, 0, s>>>(buf, walker_size, dst, src);
  return launch_status("copy_rows_kernel");
}

int pack_rows(cudaStream_t s, const c128* buf, long walker_size, const int* idx, int n, c128* out) {
  if (n <= 0) return AFQMC_OK;
  pack_rows_kernel<<<n, 256, 0, s>>>(buf, walker_size, idx, out);
  return launch_status("pack_rows_kernel");
}

int unpack_rows(cudaStream_t s, c128* buf, long walker_size, const int* idx, int n, const c128* in) {
  if (n <= 0) return AFQMC_OK;
  unpack_rows_kernel<<<n, 256, 0, s>>>(buf, walker_size, idx, in);
  return launch_status("unpack_rows_kernel");
}

int normalize_weights(cudaStream_t s, c128* buf, long walker_size, long prop0, int W) {
  if (W <= 0) return AFQMC_OK;
  normalize_weights_kernel<<<ceil_div(W, 128), 128, 0, s>>>(buf, walker_size, prop0, W);
  return launch_status("normalize_weights_kernel");
}

int gather_property(cudaStream_t s, const c128* buf, long walker_size, long off, int W, c128* out) {
  if (W <= 0) return AFQMC_OK;
  gather_property_kernel<<<ceil_div(W, 128), 128, 0, s>>>(buf, walker_size, off, W, out);
  return launch_status("gather_property_kernel");
}

int scatter_property(cudaStream_t s, c128* buf, long walker_size, long off, int W, const c128* in) {
  if (W <= 0) return AFQMC_OK;
  scatter_property_kernel<<<ceil_div(W, 128), 128, 0, s>>>(buf, walker_size, off, W, in);
  return launch_status("scatter_property_kernel");
}

int energy_sums(cudaStream_t s, const c128* buf, long walker_size, long prop0, int W,
                const c128* E, c128* out4) {
  weighted_sums_kernel<4><<<1, 1024, 0, s>>>(buf, walker_size, prop0, W, E, 0, 0.0, out4);
  return launch_status("weighted_sums_kernel");
}

int pseudo_energy_sums(cudaStream_t s, const c128* buf, long walker_size, long prop0, int W,
                       double dt, c128* out2) {
  weighted_sums_kernel<2><<<1, 1024, 0, s>>>(buf, walker_size, prop0, W, nullptr, 1, dt, out2);
  return launch_status("weighted_sums_kernel");
}

}  // namespace afqmc
