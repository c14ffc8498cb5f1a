// Particle-hole multi-Slater-determinant (PHMSD) energy kernels.
//
// Reference: src/AFQMC/Wavefunctions/detail/phmsd_impl.hpp
//   ph_excited_2body_energy_dense_cholesky (lines 33-153) and ph_excited_1body_energy (156-193).
// The reference walks the determinants of one walker per launch; here one launch covers every
// (determinant, walker) pair: a CTA per pair, its threads over the Cholesky index n, every
// per-n dot product over the active orbitals done by one thread from its own rows of Twina.
//
// Layouts (C order):
//   iexcit [ndet][2][nex] holes (electron indices into refc), then particles (active orbitals)
//   Twina  [nw][nelec][nchol][nact], R [nw][ndet][nex][nact], wgt [ndet][nw], S [nw][nelec][nact]
//   EX, EJ, E [nw] (accumulated), KE [ndet][nw][nchol] (written)
#include <vector>

#include "common.cuh"

namespace afqmc {
namespace {

constexpr int PH_THREADS = 256;
constexpr int PH_NEX_MAX = 8;

__device__ __forceinline__ c128 dot_row(const c128* __restrict__ t, const c128* __restrict__ r,
                                        int nact) {
  double re = 0.0, im = 0.0;
  for (int a = 0; a < nact; ++a) {
    const c128 x = t[a], y = r[a];
    re = fma(x.x, y.x, fma(-x.y, y.y, re));
    im = fma(x.x, y.y, fma(x.y, y.x, im));
  }
  return cmk(re, im);
}

__device__ __forceinline__ void block_sum3(c128& a, c128& b, c128& c, double* red) {
  // red: [PH_THREADS / 32][6]
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a.x += __shfl_xor_sync(0xffffffffu, a.x, off);
    a.y += __shfl_xor_sync(0xffffffffu, a.y, off);
    b.x += __shfl_xor_sync(0xffffffffu, b.x, off);
    b.y += __shfl_xor_sync(0xffffffffu, b.y, off);
    c.x += __shfl_xor_sync(0xffffffffu, c.x, off);
    c.y += __shfl_xor_sync(0xffffffffu, c.y, off);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[warp * 6 + 0] = a.x; red[warp * 6 + 1] = a.y;
    red[warp * 6 + 2] = b.x; red[warp * 6 + 3] = b.y;
    red[warp * 6 + 4] = c.x; red[warp * 6 + 5] = c.y;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int w = 0; w < int(blockDim.x >> 5); ++w)
      for (int k = 0; k < 6; ++k) s[k] += red[w * 6 + k];
    a = cmk(s[0], s[1]);
    b = cmk(s[2], s[3]);
    c = cmk(s[4], s[5]);
  }
}

__global__ void __launch_bounds__(PH_THREADS) ph_excited_2body_kernel(
    const int* __restrict__ iexcit, const int* __restrict__ refc, const c128* __restrict__ Twina,
    const c128* __restrict__ R, const c128* __restrict__ wgt, int nw, int ndet, int nex, int nact,
    int nelec, int nchol, c128* EX, c128* EJ, c128* __restrict__ KE) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c128* Rs = reinterpret_cast<c128*>(smem_raw);                 // [nex][nact]
  int* occ = reinterpret_cast<int*>(Rs + size_t(nex) * nact);    // [nelec]
  int* ref = occ + nelec;                                        // [nelec]
  __shared__ double red[PH_THREADS / 32 * 6];
  __shared__ int hole[PH_NEX_MAX], part[PH_NEX_MAX];

  const int d = blockIdx.x, w = blockIdx.y;
  const int* iex = iexcit + size_t(d) * 2 * nex;
  if (threadIdx.x < nex) {
    hole[threadIdx.x] = iex[threadIdx.x];
    part[threadIdx.x] = iex[nex + threadIdx.x];
  }
  const c128* Rw = R + (size_t(w) * ndet + d) * nex * nact;
  for (int k = threadIdx.x; k < nex * nact; k += blockDim.x) Rs[k] = Rw[k];
  __syncthreads();
  // occupied orbital of every electron in this determinant (phmsd_impl.hpp:71-80)
  for (int i = threadIdx.x; i < nelec; i += blockDim.x) {
    int o = refc[i];
    for (int e = 0; e < nex; ++e)
      if (hole[e] == i) {
        o = part[e];
        break;
      }
    occ[i] = o;
    ref[i] = refc[i];
  }
  __syncthreads();

  const c128* Tw = Twina + size_t(w) * nelec * nchol * nact;
  c128 ex = cmk(0, 0), ej = cmk(0, 0), ej0 = cmk(0, 0);
  for (int n = threadIdx.x; n < nchol; n += blockDim.x) {
    auto row = [&](int j) { return Tw + (size_t(j) * nchol + n) * nact; };
    c128 kn = cmk(0, 0), f0 = cmk(0, 0);
    // R[e] . T[hole e]: the e1 == e2 terms and the excited part of K
    for (int e = 0; e < nex; ++e) {
      const c128 f = dot_row(row(hole[e]), Rs + e * nact, nact);
      ex = cadd(ex, cmul(f, f));
      kn = cadd(kn, f);
    }
    // 2 (T[hole e2] . R[e1]) (T[hole e1] . R[e2]), e1 < e2
    for (int e1 = 0; e1 < nex; ++e1)
      for (int e2 = e1 + 1; e2 < nex; ++e2) {
        const c128 fa = dot_row(row(hole[e2]), Rs + e1 * nact, nact);
        const c128 fb = dot_row(row(hole[e1]), Rs + e2 * nact, nact);
        ex = cadd(ex, cmul(cmk(2.0, 0.0), cmul(fa, fb)));
      }
    // 2 sum_j T[hole e1][n][occ j] (T[j][n][:] . R[e1])
    for (int e1 = 0; e1 < nex; ++e1) {
      const c128* tp = row(hole[e1]);
      for (int j = 0; j < nelec; ++j) {
        const c128 fa = dot_row(row(j), Rs + e1 * nact, nact);
        ex = cadd(ex, cmul(cmk(2.0, 0.0), cmul(tp[occ[j]], fa)));
      }
    }
    // diagonal-diagonal terms of the changed electrons (phmsd_impl.hpp:123-137)
    for (int i = 0; i < nelec; ++i) {
      const int oi = occ[i], ri = ref[i];
      const c128* ti = row(i);
      if (oi != ri) ex = cadd(ex, csub(cmul(ti[oi], ti[oi]), cmul(ti[ri], ti[ri])));
      for (int j = i + 1; j < nelec; ++j) {
        const int oj = occ[j], rj = ref[j];
        if (oi != ri || oj != rj) {
          const c128* tj = row(j);
          const c128 v = csub(cmul(ti[oj], tj[oi]), cmul(ti[rj], tj[ri]));
          ex = cadd(ex, cmul(cmk(2.0, 0.0), v));
        }
      }
      kn = cadd(kn, ti[oi]);
      f0 = cadd(f0, ti[ri]);
    }
    KE[(size_t(d) * nw + w) * nchol + n] = kn;
    ej = cadd(ej, cmul(kn, kn));
    ej0 = cadd(ej0, cmul(f0, f0));
  }
  block_sum3(ex, ej, ej0, red);
  if (threadIdx.x == 0) {
    const c128 h = cmul(cmk(0.5, 0.0), wgt[size_t(d) * nw + w]);
    const c128 dx = cmul(h, ex);
    const c128 dj = cmul(h, csub(ej, ej0));
    atomicAdd(&EX[w].x, -dx.x);
    atomicAdd(&EX[w].y, -dx.y);
    atomicAdd(&EJ[w].x, dj.x);
    atomicAdd(&EJ[w].y, dj.y);
  }
}

__global__ void __launch_bounds__(PH_THREADS) ph_excited_1body_kernel(
    const int* __restrict__ iexcit, const int* __restrict__ refc, const c128* __restrict__ S,
    const c128* __restrict__ R, const c128* __restrict__ wgt, int nw, int ndet, int nex, int nact,
    int nelec, c128* E) {
  __shared__ double red[PH_THREADS / 32 * 6];
  const int d = blockIdx.x, w = blockIdx.y;
  const int* iex = iexcit + size_t(d) * 2 * nex;
  const c128* Sw = S + size_t(w) * nelec * nact;
  const c128* Rw = R + (size_t(w) * ndet + d) * nex * nact;
  c128 s = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (int k = threadIdx.x; k < nex * nact; k += blockDim.x) {
    const int p = k / nact, a = k - p * nact;
    s = cadd(s, cmul(Sw[size_t(iex[p]) * nact + a], Rw[k]));
  }
  block_sum3(s, z1, z2, red);
  if (threadIdx.x == 0) {
    for (int p = 0; p < nex; ++p) {
      const int ip = iex[p];
      s = cadd(s, csub(Sw[size_t(ip) * nact + iex[nex + p]], Sw[size_t(ip) * nact + refc[ip]]));
    }
    const c128 v = cmul(wgt[size_t(d) * nw + w], s);
    atomicAdd(&E[w].x, v.x);
    atomicAdd(&E[w].y, v.y);
  }
}

int check_dims(const char* who, int nw, int ndet, int nex, int nact, int nelec) {
  if (nw < 0 || ndet < 0 || nex < 1 || nex > PH_NEX_MAX || nact < 1 || nelec < 1) {
    set_error_detail("%s: nw=%d ndet=%d nex=%d (1..%d) nact=%d nelec=%d", who, nw, ndet, nex,
                     PH_NEX_MAX, nact, nelec);
    return AFQMC_ERR_SHAPE;
  }
  return AFQMC_OK;
}

// Copies the (small) excitation lists to the host and checks every index before a launch reads
// with them: holes in [0, nelec), particles and the reference orbitals in [0, nact).
int check_indices(const char* who, cudaStream_t s, const int* iexcit, const int* refc, int ndet,
                  int nex, int nact, int nelec) {
  std::vector<int> ie(size_t(ndet) * 2 * nex), rc(nelec);
  AFQMC_CUDA_TRY(cudaMemcpyAsync(ie.data(), iexcit, ie.size() * sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(rc.data(), refc, rc.size() * sizeof(int), cudaMemcpyDeviceToHost,
                                 s));
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  for (int i = 0; i < nelec; ++i)
    if (rc[i] < 0 || rc[i] >= nact) {
      set_error_detail("%s: refc[%d] = %d outside [0, %d)", who, i, rc[i], nact);
      return AFQMC_ERR_ARG;
    }
  for (int d = 0; d < ndet; ++d)
    for (int e = 0; e < nex; ++e) {
      const int h = ie[size_t(d) * 2 * nex + e], p = ie[size_t(d) * 2 * nex + nex + e];
      if (h < 0 || h >= nelec || p < 0 || p >= nact) {
        set_error_detail("%s: determinant %d excitation %d: hole %d (< %d), particle %d (< %d)",
                         who, d, e, h, nelec, p, nact);
        return AFQMC_ERR_ARG;
      }
    }
  return AFQMC_OK;
}

}  // namespace
}  // namespace afqmc

using namespace afqmc;

extern "C" int afqmc_ph_excited_2body_energy(const int* iexcit, const int* refc,
                                             const afqmc_c128* Twina, const afqmc_c128* R,
                                             const afqmc_c128* wgt, int nw, int ndet, int nex,
                                             int nact, int nelec, int nchol, afqmc_c128* EX,
                                             afqmc_c128* EJ, afqmc_c128* KE,
                                             afqmc_stream stream) {
  AFQMC_CHECK_ARG(iexcit && refc && Twina && R && wgt && EX && EJ && KE,
                  "afqmc_ph_excited_2body_energy: null argument");
  AFQMC_TRY(check_dims("afqmc_ph_excited_2body_energy", nw, ndet, nex, nact, nelec));
  if (nchol < 1) {
    set_error_detail("afqmc_ph_excited_2body_energy: nchol=%d", nchol);
    return AFQMC_ERR_SHAPE;
  }
  if (nw == 0 || ndet == 0) return AFQMC_OK;
  AFQMC_TRY(check_indices("afqmc_ph_excited_2body_energy", reinterpret_cast<cudaStream_t>(stream),
                          iexcit, refc, ndet, nex, nact, nelec));
  const size_t smem = size_t(nex) * nact * sizeof(c128) + 2 * size_t(nelec) * sizeof(int);
  if (smem > 200 * 1024) {
    set_error_detail("afqmc_ph_excited_2body_energy: nex*nact too large (%d x %d)", nex, nact);
    return AFQMC_ERR_UNSUPPORTED;
  }
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(ph_excited_2body_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  dim3 grid(ndet, nw);
  ph_excited_2body_kernel<<<grid, PH_THREADS, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      iexcit, refc, reinterpret_cast<const c128*>(Twina), reinterpret_cast<const c128*>(R),
      reinterpret_cast<const c128*>(wgt), nw, ndet, nex, nact, nelec, nchol,
      reinterpret_cast<c128*>(EX), reinterpret_cast<c128*>(EJ), reinterpret_cast<c128*>(KE));
  return launch_status("ph_excited_2body_kernel");
}

extern "C" int afqmc_ph_excited_1body_energy(const int* iexcit, const int* refc,
                                             const afqmc_c128* S, const afqmc_c128* R,
                                             const afqmc_c128* wgt, int nw, int ndet, int nex,
                                             int nact, int nelec, afqmc_c128* E,
                                             afqmc_stream stream) {
  AFQMC_CHECK_ARG(iexcit && refc && S && R && wgt && E,
                  "afqmc_ph_excited_1body_energy: null argument");
  AFQMC_TRY(check_dims("afqmc_ph_excited_1body_energy", nw, ndet, nex, nact, nelec));
  if (nw == 0 || ndet == 0) return AFQMC_OK;
  AFQMC_TRY(check_indices("afqmc_ph_excited_1body_energy", reinterpret_cast<cudaStream_t>(stream),
                          iexcit, refc, ndet, nex, nact, nelec));
  dim3 grid(ndet, nw);
  ph_excited_1body_kernel<<<grid, PH_THREADS, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      iexcit, refc, reinterpret_cast<const c128*>(S), reinterpret_cast<const c128*>(R),
      reinterpret_cast<const c128*>(wgt), nw, ndet, nex, nact, nelec, reinterpret_cast<c128*>(E));
  return launch_status("ph_excited_1body_kernel");
}
