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
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <type_traits>
#include <memory>
#include <vector>

#include "common.cuh"
#include "detops.cuh"
#include "mixed.cuh"
#include "zgemm.cuh"

namespace afqmc {
namespace {

constexpr int PH_THREADS = 256;
constexpr int PH_NEX_MAX = 8;

// complex arithmetic in single precision for the mixed-precision energy tables (the complex128
// helpers of common.cuh, restated for float2)
using c64 = float2;
using afqmc::cadd;
using afqmc::cmul;
using afqmc::cscale;
using afqmc::csub;
__device__ __forceinline__ c64 cadd(c64 a, c64 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ c64 csub(c64 a, c64 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ c64 cmul(c64 a, c64 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ c64 cscale(c64 a, float s) { return make_float2(a.x * s, a.y * s); }
template <typename R> struct CxOf;
template <> struct CxOf<double> { using T = c128; };
template <> struct CxOf<float> { using T = c64; };
template <typename C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ c128 czero<c128>() { return cmk(0, 0); }
template <> __device__ __forceinline__ c64 czero<c64>() { return make_float2(0.f, 0.f); }
template <typename C> __device__ __forceinline__ C to_cx(c128 x);
template <> __device__ __forceinline__ c128 to_cx<c128>(c128 x) { return x; }
template <> __device__ __forceinline__ c64 to_cx<c64>(c128 x) {
  return make_float2(float(x.x), float(x.y));
}
template <typename C> __device__ __forceinline__ C to_cx(c64 x);
template <> __device__ __forceinline__ c128 to_cx<c128>(c64 x) {
  return cmk(double(x.x), double(x.y));
}
// o += v, component-wise atomics in o's precision
__device__ __forceinline__ void atomic_add_cx(c128* o, c128 v) {
  atomicAdd(&o->x, v.x);
  atomicAdd(&o->y, v.y);
}
__device__ __forceinline__ void atomic_add_cx(c64* o, c128 v) {
  atomicAdd(&o->x, float(v.x));
  atomicAdd(&o->y, float(v.y));
}

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

// TNN[w][i][:] = TMN[w][refc[i]][:]  (Log_OverlapForWoodbury's copy_select of the reference rows)
__global__ void gather_ref_rows_kernel(const c128* __restrict__ TMN, const int* __restrict__ refc,
                                       c128* __restrict__ TNN, int nact, int N) {
  const int w = blockIdx.x;
  for (int k = threadIdx.x; k < N * N; k += blockDim.x) {
    const int i = k / N, j = k - i * N;
    TNN[size_t(w) * N * N + k] = TMN[(size_t(w) * nact + refc[i]) * N + j];
  }
}

// ov[w][u] = det(QQ0[w][particles_u][holes_u]) for every unique excitation u >= 1 (ov[w][0] = 1):
// partial-pivoting LU of the nex x nex block in registers / local memory (nex <= PH_NEX_MAX).
__global__ void excitation_det_kernel(const c128* __restrict__ QQ0, const int* __restrict__ uoff,
                                      const int* __restrict__ unex, const int* __restrict__ uexc,
                                      int nuniq, int W, int nact, int N, c128* __restrict__ ov) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nuniq) * W) return;
  const int w = int(t / nuniq), u = int(t - long(w) * nuniq);
  if (u == 0) {
    ov[t] = cmk(1.0, 0.0);
    return;
  }
  const int n = unex[u];
  const int* e = uexc + uoff[u];
  const c128* Q = QQ0 + size_t(w) * nact * N;
  c128 a[PH_NEX_MAX][PH_NEX_MAX];
  for (int p = 0; p < n; ++p)
    for (int q = 0; q < n; ++q) a[p][q] = Q[size_t(e[n + p]) * N + e[q]];
  c128 det = cmk(1.0, 0.0);
  for (int k = 0; k < n; ++k) {
    int piv = k;
    double best = cabs1(a[k][k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = cabs1(a[i][k]);
      if (v > best) {
        best = v;
        piv = i;
      }
    }
    if (!(best > 0.0)) {
      det = cmk(0.0, 0.0);
      break;
    }
    if (piv != k) {
      for (int j = 0; j < n; ++j) {
        const c128 x = a[k][j];
        a[k][j] = a[piv][j];
        a[piv][j] = x;
      }
      det = cmk(-det.x, -det.y);
    }
    det = cmul(det, a[k][k]);
    const c128 dinv = cdiv(cmk(1.0, 0.0), a[k][k]);
    for (int i = k + 1; i < n; ++i) {
      const c128 f = cmul(a[i][k], dinv);
      for (int j = k + 1; j < n; ++j) a[i][j] = csub(a[i][j], cmul(f, a[k][j]));
    }
  }
  ov[t] = det;
}

// ovlp[w] = log(sum_k c_k ov_up[w][det_up k] ov_dn[w][det_dn k]) + logov[w]  (PHMSD.cpp:884-896)
__global__ void __launch_bounds__(PH_THREADS) phmsd_combine_kernel(
    const c128* __restrict__ ov_up, const c128* __restrict__ ov_dn, int nu_up, int nu_dn,
    const int* __restrict__ det_up, const int* __restrict__ det_dn, const c128* __restrict__ coef,
    int ndet, const c128* __restrict__ logov, c128* __restrict__ ovlp) {
  __shared__ double red[PH_THREADS / 32 * 6];
  const int w = blockIdx.x;
  const c128* ou = ov_up + size_t(w) * nu_up;
  const c128* od = ov_dn + size_t(w) * nu_dn;
  c128 s = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (int k = threadIdx.x; k < ndet; k += blockDim.x)
    s = cadd(s, cmul(coef[k], cmul(ou[det_up[k]], od[det_dn[k]])));
  block_sum3(s, z1, z2, red);
  if (threadIdx.x == 0) ovlp[w] = cadd(clog(s), logov[w]);
}

// Lnak[n][a][k] <- tmp[a][k][n]  (rows of OrbMat * L viewed as M x (M Nc))
__global__ void lnak_act_reorder_kernel(const c128* __restrict__ in, c128* __restrict__ out,
                                        int nact, int M, int Nc) {
  const long e = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= long(nact) * M * Nc) return;
  const int n = int(e % Nc);
  const long r = e / Nc;
  const int k = int(r % M), a = int(r / M);
  out[(long(n) * nact + a) * M + k] = in[e];
}

// wgt[u][w] = scale_u(w) * sum over the determinants k of unique excitation u (CSR row u) of
// c_k v_other[w][other_k]; scale = ov_self[w][u] when ov_self is given (energy_alg1's
// "W *= ovlp_ratio" steps)
__global__ void couple_kernel(const int* __restrict__ rowptr, const int* __restrict__ kidx,
                              const int* __restrict__ det_other, const c128* __restrict__ coef,
                              const c128* __restrict__ v_other, int nu_other,
                              const c128* __restrict__ ov_self, int nu, int W,
                              c128* __restrict__ wgt) {
  // one warp per (u, w): the row of the reference (u = 0) holds a large share of the
  // determinants, so its entries are split over the lanes
  const long t = (long(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= long(nu) * W) return;
  const int u = int(t / W), w = int(t - long(u) * W);
  c128 acc = cmk(0, 0);
  for (int j = rowptr[u] + lane; j < rowptr[u + 1]; j += 32) {
    const int k = kidx[j];
    acc = cadd(acc, cmul(coef[k], v_other[size_t(w) * nu_other + det_other[k]]));
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
    acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
  }
  if (lane == 0) {
    if (ov_self) acc = cmul(acc, ov_self[size_t(w) * nu + u]);
    wgt[t] = acc;
  }
}

// out[w][u] = in[u][w]  (nu x W)
__global__ void transpose_uw_kernel(const c128* __restrict__ in, int nu, int W,
                                    c128* __restrict__ out) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nu) * W) return;
  const int w = int(t / nu), u = int(t - long(w) * nu);
  out[t] = in[size_t(u) * W + w];
}

// Ov[w] = sum_u wgt[u][w] ov[w][u]   (before the weights are scaled by the overlaps)
__global__ void __launch_bounds__(PH_THREADS) total_overlap_kernel(
    const c128* __restrict__ wgt, const c128* __restrict__ ov, int nu, int W,
    c128* __restrict__ Ov) {
  __shared__ double red[PH_THREADS / 32 * 6];
  const int w = blockIdx.x;
  c128 s = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (int u = threadIdx.x; u < nu; u += blockDim.x)
    s = cadd(s, cmul(wgt[size_t(u) * W + w], ov[size_t(w) * nu + u]));
  block_sum3(s, z1, z2, red);
  if (threadIdx.x == 0) Ov[w] = s;
}

// ph_reference_energy (Real3IndexFactorization.hpp:212-235, 612-690): per walker
//   e1 = (E0) + sum_i Swia[i][refc_i],  ex = -1/2 sum_{i,j,n} T[i][n][refc_j] T[j][n][refc_i],
//   Kl[n] = sum_i T[i][n][refc_i],  ej = 1/2 Kl.Kl;  E[w] += Ov[w] (e1, ex, ej)
__global__ void __launch_bounds__(PH_THREADS) ph_reference_kernel(
    const c128* __restrict__ Swia, const c128* __restrict__ Twina, const int* __restrict__ refc,
    int nel, int nchol, int nact, double E0, const c128* __restrict__ Ov, c128* __restrict__ E,
    c128* __restrict__ Kl) {
  __shared__ double red[PH_THREADS / 32 * 6];
  const int w = blockIdx.x;
  const c128* T = Twina + size_t(w) * nel * nchol * nact;
  c128 ex = cmk(0, 0), ej = cmk(0, 0), e1 = cmk(0, 0);
  for (int n = threadIdx.x; n < nchol; n += blockDim.x) {
    c128 kn = cmk(0, 0);
    for (int i = 0; i < nel; ++i) {
      const c128* ti = T + (size_t(i) * nchol + n) * nact;
      kn = cadd(kn, ti[refc[i]]);
      for (int j = 0; j < nel; ++j) {
        const c128* tj = T + (size_t(j) * nchol + n) * nact;
        ex = cadd(ex, cmul(ti[refc[j]], tj[refc[i]]));
      }
    }
    Kl[size_t(w) * nchol + n] = kn;
    ej = cadd(ej, cmul(kn, kn));
  }
  for (int i = threadIdx.x; i < nel; i += blockDim.x)
    e1 = cadd(e1, Swia[(size_t(w) * nel + i) * nact + refc[i]]);
  block_sum3(ex, ej, e1, red);
  if (threadIdx.x == 0) {
    const c128 o = Ov[w];
    const c128 v1 = cmul(o, cmk(e1.x + E0, e1.y));
    const c128 vx = cmul(o, cmul(cmk(-0.5, 0), ex));
    const c128 vj = cmul(o, cmul(cmk(0.5, 0), ej));
    E[w * 3 + 0] = cadd(E[w * 3 + 0], v1);
    E[w * 3 + 1] = cadd(E[w * 3 + 1], vx);
    E[w * 3 + 2] = cadd(E[w * 3 + 2], vj);
  }
}

// Inverse of the excitation block a[p][q] = QQ0[particle_p][hole_q] (nex x nex, e = holes then
// particles) by Gauss-Jordan with partial pivoting; false for a singular block.
__device__ bool woodbury_block_inverse(const c128* __restrict__ Q0, const int* __restrict__ e,
                                       int nex, int nel, c128 (&inv)[PH_NEX_MAX][PH_NEX_MAX]) {
  c128 a[PH_NEX_MAX][PH_NEX_MAX];
  for (int p = 0; p < nex; ++p)
    for (int q = 0; q < nex; ++q) {
      a[p][q] = Q0[size_t(e[nex + p]) * nel + e[q]];
      inv[p][q] = cmk(p == q ? 1.0 : 0.0, 0.0);
    }
  for (int k = 0; k < nex; ++k) {
    int piv = k;
    double best = cabs1(a[k][k]);
    for (int i = k + 1; i < nex; ++i)
      if (cabs1(a[i][k]) > best) {
        best = cabs1(a[i][k]);
        piv = i;
      }
    if (!(best > 0.0)) return false;
    if (piv != k)
      for (int j = 0; j < nex; ++j) {
        c128 x = a[k][j]; a[k][j] = a[piv][j]; a[piv][j] = x;
        x = inv[k][j]; inv[k][j] = inv[piv][j]; inv[piv][j] = x;
      }
    const c128 dinv = cdiv(cmk(1.0, 0.0), a[k][k]);
    for (int j = 0; j < nex; ++j) {
      a[k][j] = cmul(a[k][j], dinv);
      inv[k][j] = cmul(inv[k][j], dinv);
    }
    for (int i = 0; i < nex; ++i)
      if (i != k) {
        const c128 f = a[i][k];
        for (int j = 0; j < nex; ++j) {
          a[i][j] = csub(a[i][j], cmul(f, a[k][j]));
          inv[i][j] = csub(inv[i][j], cmul(f, inv[k][j]));
        }
      }
  }
  return true;
}

// get_compact_ph_R_matrices (phmsd_helpers.hpp:311-398): R[w][d][p][:] from the inverse Q of the
// excitation block QQ0[particles][holes]; orbs = the determinant's occupied active orbitals:
//   R[p][orbs_i] -= Q[p][q] QQ0[part_q][i]  (all electrons i),  R[p][orbs(hole_q)] += Q[p][q]
// R must be zero on entry; a singular block leaves its rows zero (as the reference).
__global__ void compact_R_kernel(const c128* __restrict__ QQ0, const int* __restrict__ iexcit,
                                 const int* __restrict__ refc, int ndet, int nex, int W, int nact,
                                 int nel, c128* __restrict__ R) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(W) * ndet) return;
  const int w = int(t / ndet), d = int(t - long(w) * ndet);
  const int* e = iexcit + size_t(d) * 2 * nex;
  const c128* Q0 = QQ0 + size_t(w) * nact * nel;
  c128 inv[PH_NEX_MAX][PH_NEX_MAX];
  // a singular block leaves this determinant's R zero (as the reference)
  if (!woodbury_block_inverse(Q0, e, nex, nel, inv)) return;
  c128* Rw = R + (size_t(w) * ndet + d) * nex * nact;
  for (int p = 0; p < nex; ++p) {
    c128* Rp = Rw + size_t(p) * nact;
    for (int q = 0; q < nex; ++q) {
      const c128 ipq = inv[p][q];
      const c128* Tq = Q0 + size_t(e[nex + q]) * nel;
      for (int i = 0; i < nel; ++i) {
        int oi = refc[i];
        for (int h = 0; h < nex; ++h)
          if (e[h] == i) oi = e[nex + h];
        Rp[oi] = csub(Rp[oi], cmul(ipq, Tq[i]));
      }
      int oh = e[nex + q];  // orbital of hole q's electron in this determinant
      Rp[oh] = cadd(Rp[oh], ipq);
    }
  }
}

// INV[w][uinv[u] ...] = inverse of the excitation block of every unique excitation u >= 1
// (row-major nex x nex), zeros for a singular block: the Q matrices of the Woodbury R.
__global__ void woodbury_inverses_kernel(const c128* __restrict__ QQ0, const int* __restrict__ uoff,
                                         const int* __restrict__ unex,
                                         const int* __restrict__ uexc,
                                         const int* __restrict__ uinv, int nuniq, int W, int nact,
                                         int nel, int ninv, c128* __restrict__ INV,
                                         float2* __restrict__ INV32,
                                         const int4* __restrict__ uhdrs) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(nuniq - 1) * W) return;
  const int w = int(t / (nuniq - 1)), u = 1 + int(t - long(w) * (nuniq - 1));
  const int nex = unex[u];
  c128 inv[PH_NEX_MAX][PH_NEX_MAX];
  const bool ok = woodbury_block_inverse(QQ0 + size_t(w) * nact * nel, uexc + uoff[u], nex, nel,
                                         inv);
  c128* o = INV + size_t(w) * ninv + uinv[u];
  for (int p = 0; p < nex; ++p)
    for (int q = 0; q < nex; ++q) o[p * nex + q] = ok ? inv[p][q] : cmk(0.0, 0.0);
  if (INV32) {  // structure-of-arrays within the shell: entry k at base + k cnt
    const int4 hs = uhdrs[u];
    float2* o32 = INV32 + size_t(w) * ninv + hs.z;
    for (int p = 0; p < nex; ++p)
      for (int q = 0; q < nex; ++q)
        o32[size_t(p * nex + q) * hs.w] = ok ? make_float2(float(inv[p][q].x), float(inv[p][q].y))
                                             : make_float2(0.f, 0.f);
  }
}

// The 1-body energies of every unique excitation u >= 1 for walker blockIdx.x, from the
// Woodbury inverses Qi (INV, uhdr) instead of R rows (ph_excited_1body_kernel over compact_R's
// rows, PHMSD.cpp:376-546): with R_u[p] = sum_q Qi[p][q] (e_{part_q} - sum_i QQ0[part_q][i]
// e_{o_u(i)}), o_u(i) the orbital of electron i in determinant u (its particle for a hole, else
// refc[i]),
//   e1_u = sum_p (S[i_p] . R_u[p] + S[i_p][part_p] - S[i_p][refc[i_p]]),
// and E[w] += sum_u wgt[u][w] e1_u.  Because Qi inverts M[q][x] = QQ0[part_q][i_x], the terms at
// the holes' reference orbitals cancel and e1_u = sum_{p,q} Qi[p][q] Sf1[i_p][c_q] with the
// per-walker table Sf1[i][c] = S[i][v_c] - sum_j S[i][refc_j] QQ0[v_c][j] (v_c the virtual
// orbitals, c_q the particle columns).  A singular block has Qi = 0, so e1_u = 0 (as the
// reference).  Grid (walkers, parts): each CTA builds Sf1 and takes every gridDim.y-th excitation.
__global__ void __launch_bounds__(PH_THREADS) excited_1body_all_kernel(
    const c128* __restrict__ S, const c128* __restrict__ QQ0, const int* __restrict__ refc,
    const int* __restrict__ vl, int nv, const int4* __restrict__ uhdr,
    const int* __restrict__ uexc4, const c128* __restrict__ INV, int ninv,
    const c128* __restrict__ wgt, int nuniq, int W, int nel, int nact, c128* __restrict__ E) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  c128* sf1 = reinterpret_cast<c128*>(smem_raw);  // [nel][nv]
  __shared__ double red[PH_THREADS / 32 * 6];
  const int w = blockIdx.x;
  const c128* Sw = S + size_t(w) * nel * nact;
  const c128* Q0 = QQ0 + size_t(w) * nact * nel;
  const c128* Iw = INV + size_t(w) * ninv;
  for (int k = threadIdx.x; k < nel * nv; k += blockDim.x) {
    const int i = k / nv, c = k - i * nv;
    const c128* Si = Sw + size_t(i) * nact;
    const c128* Qc = Q0 + size_t(vl[c]) * nel;
    c128 t = Si[vl[c]];
    for (int j = 0; j < nel; ++j) t = csub(t, cmul(Si[refc[j]], Qc[j]));
    sf1[k] = t;
  }
  __syncthreads();
  c128 acc = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (int u = 1 + blockIdx.y * blockDim.x + threadIdx.x; u < nuniq;
       u += gridDim.y * blockDim.x) {
    const int4 hd = uhdr[u];
    const int n = hd.x;
    const int* e4 = uexc4 + hd.y;  // holes, particles, hole rows, particle columns
    const c128* Qi = Iw + hd.z;
    c128 e1 = cmk(0, 0);
    for (int p = 0; p < n; ++p) {
      const c128* row = sf1 + e4[p] * nv;
      for (int q = 0; q < n; ++q) e1 = cadd(e1, cmul(Qi[p * n + q], row[e4[3 * n + q]]));
    }
    acc = cadd(acc, cmul(wgt[size_t(u) * W + w], e1));
  }
  block_sum3(acc, z1, z2, red);
  if (threadIdx.x == 0) {
    atomicAdd(&E[w].x, acc.x);
    atomicAdd(&E[w].y, acc.y);
  }
}

// The 2-body energy terms of one excited determinant at one Cholesky index n, from per-walker
// tables instead of its R rows.  With t_j = T[j][n][:] (rows of the half-rotated Twina), the
// reference orbitals r_i, the virtual orbitals v_c, the determinant's holes h_a (electrons),
// their hole rows k_a and particle columns c_a (its particles p_a = v_{c_a}), Q = INV (the
// inverse of the excitation block M[q][x] = QQ0[p_q][h_x]), and the compact
// R_b[x] = sum_q Q[b][q] (delta(x, p_q) - sum_i delta(x, occ_i) QQ0[p_q][i]), the terms of
// ph_excited_2body_energy_dense_cholesky (detail/phmsd_impl.hpp:33-153) summed in closed form
// over the electrons are
//   F[a][b] = t_{h_a} . R_b,  D[a] = U[h_a] . R_a  with U[h][x] = sum_j t_h[r_j] t_j[x],
//   kn = f0 + sum_a (F[a][a] + t_{h_a}[p_a] - t_{h_a}[r_a]),  f0 = sum_i t_i[r_i],
//   ex = sum_{a,b} F[a][b] F[b][a] + sum_{a,x} (t_{h_a}[p_x] t_{h_x}[p_a] - t_{h_a}[r_x] t_{h_x}[r_a])
//        + 2 sum_a (D[a] + sum_x (t_{h_a}[p_x] - t_{h_a}[r_x]) F[x][a]
//                   + U[h_a][p_a] - U[h_a][r_a] - sum_x t_{h_a}[r_x] (t_{h_x}[p_a] - t_{h_x}[r_a])).
// Because Q M = 1, F = P - (t_{h_a}[p_b] - t_{h_a}[r_b]) with P[a][b] = sum_q Sf[h_a][c_q] Q[b][q],
// and every term at the holes' reference columns cancels, which leaves
//   kn = f0 + tr P,   ex = tr(P P) + 2 sum_{a,q} Q[a][q] SU[k_a][c_q],
//   Sf[j][c] = t_j[v_c] - sum_i t_j[r_i] QQ0[v_c][i],   SU[k][c] = sum_j t_{h_k}[r_j] Sf[j][c].
// Table layout: Sf [nel][nv] (all electrons' rows), SU [nh][nv] (hole rows), one pair per
// Cholesky index g of the block's group (strides sfs, sus).  e4 = the determinant's holes,
// particles, hole rows k and particle columns c.  The determinant's Q and indices are read once
// for the ng indices of the group: exg[g], kng[g].
template <int NEX, int NG, typename C>
__device__ __forceinline__ void excited_terms(const int* __restrict__ e4,
                                              const C* __restrict__ Qg, int es, const C* Sf,
                                              const C* SU, int nv, int sfs, int sus, int ng,
                                              const C* f0, C* exg, C* kng) {
  using R = decltype(f0[0].x);
  C Qi[NEX * NEX];  // the determinant's Woodbury inverse, in the working precision
#pragma unroll
  for (int k = 0; k < NEX * NEX; ++k) Qi[k] = Qg[k * es];
  int so[NEX], uo[NEX], pc[NEX];
#pragma unroll
  for (int a = 0; a < NEX; ++a) {
    so[a] = e4[a * es] * nv;
    uo[a] = e4[(2 * NEX + a) * es] * nv;
    pc[a] = e4[(3 * NEX + a) * es];
  }
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    if (g >= ng) break;
    const C* Sg = Sf + g * sfs;
    const C* Ug = SU + g * sus;
    C P[NEX][NEX];
    C d = czero<C>();
#pragma unroll
    for (int a = 0; a < NEX; ++a) {
      C sv[NEX];
#pragma unroll
      for (int q = 0; q < NEX; ++q) {
        sv[q] = Sg[so[a] + pc[q]];
        d = cadd(d, cmul(Qi[a * NEX + q], Ug[uo[a] + pc[q]]));
      }
#pragma unroll
      for (int b = 0; b < NEX; ++b) {
        C acc = czero<C>();
#pragma unroll
        for (int q = 0; q < NEX; ++q) acc = cadd(acc, cmul(sv[q], Qi[b * NEX + q]));
        P[a][b] = acc;
      }
    }
    C tr = czero<C>(), pp = czero<C>(), off = czero<C>();
#pragma unroll
    for (int a = 0; a < NEX; ++a) {
      tr = cadd(tr, P[a][a]);
      pp = cadd(pp, cmul(P[a][a], P[a][a]));
#pragma unroll
      for (int b = a + 1; b < NEX; ++b) off = cadd(off, cmul(P[a][b], P[b][a]));
    }
    exg[g] = cadd(cadd(pp, cscale(off, R(2))), cscale(d, R(2)));
    kng[g] = cadd(f0[g], tr);
  }
}

// nex > 4 is rare: out of line, so that its larger frame stays out of the common path
template <int NEX, int NG, typename C>
__device__ __noinline__ void excited_terms_rare(const int* e4, const C* Qi, int es, const C* Sf,
                                                const C* SU, int nv, int sfs, int sus, int ng,
                                                const C* f0, C* exg, C* kng) {
  excited_terms<NEX, NG, C>(e4, Qi, es, Sf, SU, nv, sfs, sus, ng, f0, exg, kng);
}

// One product of the tables: out[k][c] = sum_j a[r_k][sel_j] b[j][c] over the rows k < nrows
// (r_k = rows[k], or k when rows is null), c < ncol.  A thread owns RT rows and the columns
// t and t + half (half = ceil(ncol / 2)) of them, so that every shared-memory read of a feeds
// two products and every read of b feeds RT; neighbouring threads read neighbouring columns of b.
// With sub: out[k][c] = sub[k][subcols_c] - (the product) instead.
template <int RT, typename C>
__device__ __forceinline__ void table_product(const C* a, int lda, const int* rows, int nrows,
                                              const int* sel, int nsum, const C* b, int ldb,
                                              int ncol, C* out, int ldo, const C* sub = nullptr,
                                              int ldsub = 0, const int* subcols = nullptr) {
  const int half = (ncol + 1) / 2;
  const int nrt = (nrows + RT - 1) / RT;
  for (int t = threadIdx.x; t < nrt * half; t += blockDim.x) {
    const int rt = t / half, ct = t - rt * half;
    const bool two = ct + half < ncol;
    const C* ar[RT];
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int k = rt * RT + r;
      ar[r] = a + (k < nrows ? (rows ? rows[k] : k) : 0) * lda;  // a row past the end: row 0
    }
    C acc0[RT], acc1[RT];
#pragma unroll
    for (int r = 0; r < RT; ++r) acc0[r] = acc1[r] = czero<C>();
    for (int j = 0; j < nsum; ++j) {
      const int sj = sel[j];
      const C b0 = b[j * ldb + ct];
      const C b1 = two ? b[j * ldb + ct + half] : czero<C>();
#pragma unroll
      for (int r = 0; r < RT; ++r) {
        const C x = ar[r][sj];
        acc0[r] = cadd(acc0[r], cmul(x, b0));
        acc1[r] = cadd(acc1[r], cmul(x, b1));
      }
    }
#pragma unroll
    for (int r = 0; r < RT; ++r) {
      const int k = rt * RT + r;
      if (k >= nrows) break;
      if (sub) {
        acc0[r] = csub(sub[k * ldsub + subcols[ct]], acc0[r]);
        if (two) acc1[r] = csub(sub[k * ldsub + subcols[ct + half]], acc1[r]);
      }
      out[k * ldo + ct] = acc0[r];
      if (two) out[k * ldo + ct + half] = acc1[r];
    }
  }
}

// Excited-determinant 2-body energies of one spin for walker blockIdx.y at the NG Cholesky
// indices n = NG blockIdx.x + g, all unique excitations in one launch (the work of
// ph_excited_energies_first_step / second_step, phmsd_helpers.hpp:401-527, for every shell): the
// per-(walker, n) tables Sf and SU in shared memory, built one index at a time, then one thread
// per excited determinant over the group's indices (its Q, indices and weight read once).
// EXacc[w] -= wgt ex / 2, EJacc[w] += wgt (kn^2 - f0^2) / 2; KE[u][w][n] = kn, or with `cross`
// E[w].EJ += cross . kn.  The reference determinant's terms come from the same tables
// (ph_reference_energy, Real3IndexFactorization.hpp:212-233, 598-696): Kref[w][n] = f0,
// REF[w] += (sum_ij t_i[r_j] t_j[r_i], f0^2).
// R = double: complex128 tables and per-determinant sums (the reference's arithmetic); R = float:
// complex64 tables and per-determinant sums, for the mixed-precision energy (half the shared
// memory, twice the FP32 rate); the sums over determinants, the reference determinant's terms
// and every output stay FP64.
constexpr int PHX_THREADS = 256;

// asynchronous global -> shared copies of 8 or 16 bytes (cp.async, completion per commit group)
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// TW: the element type of Twina (complex128, or complex64 from the mixed half rotation).  When
// it is the working type C the rows t_j come in by asynchronous copies, the next index's while
// the current one's tables are built (nbuf = 2), else by converting loads.  INVc holds the
// Woodbury inverses in the working type; uhdr[u] = {nex, base of u in uexc4, base of u in INVc,
// stride es}: field entry k of excitation u at base + k es (es = 1: one excitation's entries
// together; es = the shell's size: structure-of-arrays, consecutive excitations adjacent).
template <typename R, int NG, typename TW>
__global__ void __launch_bounds__(PHX_THREADS, sizeof(R) == 4 ? 2 : 1) excited_energy_tables_kernel(
    const TW* __restrict__ Twina, const c128* __restrict__ QQ0, const int* __restrict__ refc,
    const int* __restrict__ hl, const int* __restrict__ vl, int nh, int nv,
    const int4* __restrict__ uhdr, const int* __restrict__ uexc4,
    const typename CxOf<R>::T* __restrict__ INVc, int ninv,
    const c128* __restrict__ wgtT, int nuniq, int W, int nel, int nact, int nchol, int nbuf,
    c128* __restrict__ EXacc, c128* __restrict__ EJacc, TW* __restrict__ KE,
    const TW* __restrict__ cross, c128* __restrict__ E, TW* __restrict__ Kref,
    c128* __restrict__ REF) {
  using C = typename CxOf<R>::T;
  constexpr bool ASYNC = sizeof(TW) == sizeof(C);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Tb0 = reinterpret_cast<C*>(smem_raw);                // [nbuf][nel][nact]
  C* Tb1 = Tb0 + (nbuf - 1) * nel * nact;
  C* Qv = Tb0 + nbuf * nel * nact;                        // [nel][nv]
  C* Sf = Qv + nel * nv;                                  // [NG][nel][nv]
  C* SU = Sf + NG * nel * nv;                             // [NG][nh][nv]
  int* refs = reinterpret_cast<int*>(SU + NG * nh * nv);  // [nel]
  int* hls = refs + nel;                                  // [nh]
  int* vls = hls + nh;                                    // [nv]
  __shared__ double red[PHX_THREADS / 32 * 6];
  const int n0 = blockIdx.x * NG, w = blockIdx.y;
  const int ng = min(NG, nchol - n0);
  const int sfs = nel * nv, sus = nh * nv;
  const TW* Tw = Twina + size_t(w) * nel * nchol * nact;
  const c128* Qw = QQ0 + size_t(w) * nact * nel;
  auto load_t = [&](int g, C* dst) {
    const int n = n0 + g;
    for (int k = threadIdx.x; k < nel * nact; k += blockDim.x) {
      const int j = k / nact, x = k - j * nact;
      const TW* src = Tw + (size_t(j) * nchol + n) * nact + x;
      if constexpr (ASYNC)
        cp_async<int(sizeof(C))>(dst + k, src);
      else
        dst[k] = to_cx<C>(*src);
    }
    if constexpr (ASYNC) cp_async_commit();
  };
  load_t(0, Tb0);
  for (int k = threadIdx.x; k < nel * nv; k += blockDim.x) {
    const int i = k / nv, c = k - i * nv;
    Qv[k] = to_cx<C>(Qw[size_t(vl[c]) * nel + i]);
  }
  for (int i = threadIdx.x; i < nel; i += blockDim.x) refs[i] = refc[i];
  for (int k = threadIdx.x; k < nh; k += blockDim.x) hls[k] = hl[k];
  for (int c = threadIdx.x; c < nv; c += blockDim.x) vls[c] = vl[c];
  C f0w[NG];
  c128 f00[NG];
  c128 ex0 = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0), f00s = cmk(0, 0);
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    f0w[g] = czero<C>();
    f00[g] = cmk(0, 0);
    if (g >= ng) break;
    const int n = n0 + g;
    C* Tn = (g & 1) ? Tb1 : Tb0;
    C* Sg = Sf + g * sfs;
    C* Ug = SU + g * sus;
    if (nbuf == 2 && g + 1 < ng) {
      load_t(g + 1, (g & 1) ? Tb0 : Tb1);  // the other buffer, free since the last barrier
      if constexpr (ASYNC) cp_async_wait<1>();
    } else {
      if constexpr (ASYNC) cp_async_wait<0>();
    }
    __syncthreads();
    // Sf = t[:, v] - t[:, r] Qv
    table_product<3, C>(Tn, nact, nullptr, nel, refs, nel, Qv, nv, nv, Sg, nv, Tn, nact, vls);
    // the reference determinant: f0 = sum_i t_i[r_i], ex0 = sum_ij t_i[r_j] t_j[r_i] (summed
    // over the group's indices, reduced over the block after the loop)
    for (int k = threadIdx.x; k < nel * nel; k += blockDim.x) {
      const int i = k / nel, j = k - i * nel;
      ex0 = cadd(ex0,
                 cmul(to_cx<c128>(Tn[i * nact + refs[j]]), to_cx<c128>(Tn[j * nact + refs[i]])));
    }
    __syncthreads();
    // SU = t[hole rows, r] Sf
    table_product<3, C>(Tn, nact, hls, nh, refs, nel, Sg, nv, nv, Ug, nv);
    c128 f0 = cmk(0, 0);
    for (int i = 0; i < nel; ++i) f0 = cadd(f0, to_cx<c128>(Tn[i * nact + refs[i]]));
    f0w[g] = to_cx<C>(f0);
    f00[g] = cmul(f0, f0);
    if (threadIdx.x == 0 && Kref) {
      Kref[size_t(w) * nchol + n] = to_cx<TW>(f0);
      f00s = cadd(f00s, f00[g]);
    }
    __syncthreads();  // SU complete; Tn free for the next index's rows
    if (nbuf == 1 && g + 1 < ng) load_t(g + 1, Tb0);
  }
  block_sum3(ex0, z1, z2, red);
  if (threadIdx.x == 0 && Kref) {
    atomicAdd(&REF[2 * w].x, ex0.x);
    atomicAdd(&REF[2 * w].y, ex0.y);
    atomicAdd(&REF[2 * w + 1].x, f00s.x);
    atomicAdd(&REF[2 * w + 1].y, f00s.y);
  }
  __syncthreads();
  c128 exs = cmk(0, 0), ejs = cmk(0, 0), ejc = cmk(0, 0);
  const C* Iw = INVc + size_t(w) * ninv;
  const c128* wgw = wgtT + size_t(w) * nuniq;  // this walker's weights, consecutive in u
  for (int u = 1 + threadIdx.x; u < nuniq; u += blockDim.x) {
    const int4 hd = uhdr[u];
    const c128 wu = wgw[u];
    const int* e4 = uexc4 + hd.y;
    const C* Qi = Iw + hd.z;
    C exw[NG], knw[NG];
    switch (hd.x) {
      case 1: excited_terms<1, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 2: excited_terms<2, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 3: excited_terms<3, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 4: excited_terms<4, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 5: excited_terms_rare<5, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 6: excited_terms_rare<6, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      case 7: excited_terms_rare<7, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
      default: excited_terms_rare<8, NG, C>(e4, Qi, hd.w, Sf, SU, nv, sfs, sus, ng, f0w, exw, knw); break;
    }
    c128 exu = cmk(0, 0), eju = cmk(0, 0);
    const size_t o = (size_t(u) * W + w) * nchol + n0;
#pragma unroll
    for (int g = 0; g < NG; ++g) {
      if (g >= ng) break;
      const c128 kn = to_cx<c128>(knw[g]);
      exu = cadd(exu, to_cx<c128>(exw[g]));
      eju = cadd(eju, csub(cmul(kn, kn), f00[g]));
      if (cross)
        ejc = cadd(ejc, cmul(to_cx<c128>(cross[o + g]), kn));
      else
        KE[o + g] = to_cx<TW>(kn);
    }
    exs = cadd(exs, cmul(wu, exu));
    ejs = cadd(ejs, cmul(wu, eju));
  }
  block_sum3(exs, ejs, ejc, red);
  if (threadIdx.x == 0) {
    atomicAdd(&EXacc[w].x, -0.5 * exs.x);
    atomicAdd(&EXacc[w].y, -0.5 * exs.y);
    atomicAdd(&EJacc[w].x, 0.5 * ejs.x);
    atomicAdd(&EJacc[w].y, 0.5 * ejs.y);
    if (cross) {
      atomicAdd(&E[w * 3 + 2].x, ejc.x);
      atomicAdd(&E[w * 3 + 2].y, ejc.y);
    }
  }
}

// The reference determinant's energy from the table sums (ph_reference_kernel's result):
// E[w] += Ov (E0 + sum_i S[i][r_i], -ex0 / 2, f0^2 / 2)
__global__ void reference_from_tables_kernel(const c128* __restrict__ Swia,
                                             const int* __restrict__ refc, int nel, int nact,
                                             double E0, const c128* __restrict__ Ov,
                                             const c128* __restrict__ REF, int W,
                                             c128* __restrict__ E) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  c128 e1 = cmk(E0, 0);
  for (int i = 0; i < nel; ++i) e1 = cadd(e1, Swia[(size_t(w) * nel + i) * nact + refc[i]]);
  const c128 o = Ov[w];
  E[w * 3 + 0] = cadd(E[w * 3 + 0], cmul(o, e1));
  E[w * 3 + 1] = cadd(E[w * 3 + 1], cmul(o, cscale(REF[2 * w], -0.5)));
  E[w * 3 + 2] = cadd(E[w * 3 + 2], cmul(o, cscale(REF[2 * w + 1], 0.5)));
}

// KEd[d][w][n] = ov_dn[w][d] sum_{k in CSR row d} c_k ov_up[w][up_k] KEr[up_k][w][n]
// The determinants of CSR row d are split into segments of at most KE_SEG (rows with many
// determinants, such as the reference down-spin excitation, would otherwise serialise one CTA);
// segment g = (d, j0, j1).  A row of one segment stores its result, longer rows add into KEd,
// which is zeroed first.
// KT: the element type of the K vectors (complex64 in the mixed energy's tables path).
constexpr int KE_SEG = 16;
template <typename KT>
__global__ void couple_ke_kernel(const int* __restrict__ seg, const int* __restrict__ kidx,
                                 const int* __restrict__ det_up, const c128* __restrict__ coef,
                                 const KT* __restrict__ KEr, const c128* __restrict__ ov_up,
                                 int nu_up, const c128* __restrict__ ov_dn, int nu_dn, int W,
                                 int nchol, KT* __restrict__ KEd) {
  __shared__ c128 f[KE_SEG];
  __shared__ int uu[KE_SEG];
  const int g = blockIdx.x, w = blockIdx.y;
  const int d = seg[4 * g], j0 = seg[4 * g + 1], j1 = seg[4 * g + 2], single = seg[4 * g + 3];
  const c128 od = ov_dn[size_t(w) * nu_dn + d];
  for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
    const int k = kidx[j], u = det_up[k];
    uu[j - j0] = u;
    f[j - j0] = cmul(od, cmul(coef[k], ov_up[size_t(w) * nu_up + u]));
  }
  __syncthreads();
  for (int n = threadIdx.x; n < nchol; n += blockDim.x) {
    c128 acc = cmk(0, 0);
    for (int j = 0; j < j1 - j0; ++j)
      acc = cadd(acc, cmul(f[j], to_cx<c128>(KEr[(size_t(uu[j]) * W + w) * nchol + n])));
    KT* o = KEd + (size_t(d) * W + w) * nchol + n;
    if (single)
      *o = to_cx<KT>(acc);
    else
      atomic_add_cx(o, acc);
  }
}

// the KEd rows of the CSR rows split over several segments (krow) set to zero before their
// segments add into them
template <typename KT>
__global__ void zero_k_rows_kernel(const int* __restrict__ krow, int W, int nchol,
                                   KT* __restrict__ KEd) {
  KT* o = KEd + (size_t(krow[blockIdx.x]) * W + blockIdx.y) * nchol;
  for (int n = threadIdx.x; n < nchol; n += blockDim.x) o[n] = to_cx<KT>(cmk(0, 0));
}

// E[w][2] += sum_{d, n} A[d][w][n] B[d][w][n]  (the cross-spin Coulomb products)
template <typename KT>
__global__ void __launch_bounds__(PH_THREADS) cross_ej_kernel(const KT* __restrict__ A,
                                                              const KT* __restrict__ B, int nd,
                                                              int W, int nchol,
                                                              c128* __restrict__ E) {
  __shared__ double red[PH_THREADS / 32 * 6];
  const int w = blockIdx.x;
  c128 s = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (long k = threadIdx.x; k < long(nd) * nchol; k += blockDim.x) {
    const int d = int(k / nchol), n = int(k - long(d) * nchol);
    const size_t o = (size_t(d) * W + w) * nchol + n;
    s = cadd(s, cmul(to_cx<c128>(A[o]), to_cx<c128>(B[o])));
  }
  block_sum3(s, z1, z2, red);
  if (threadIdx.x == 0) E[w * 3 + 2] = cadd(E[w * 3 + 2], s);
}

// E[w] += (e1[w], ex[w], ej[w])
__global__ void add_components_kernel(const c128* __restrict__ e1, const c128* __restrict__ ex,
                                      const c128* __restrict__ ej, int W, c128* __restrict__ E) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  E[w * 3 + 0] = cadd(E[w * 3 + 0], e1[w]);
  E[w * 3 + 1] = cadd(E[w * 3 + 1], ex[w]);
  E[w * 3 + 2] = cadd(E[w * 3 + 2], ej[w]);
}

// ovlp[w] = log Ov[w] + logov[w]
__global__ void phmsd_combine_log_kernel(const c128* __restrict__ Ov, const c128* __restrict__ logov,
                                         int W, c128* __restrict__ ovlp) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w < W) ovlp[w] = cadd(clog(Ov[w]), logov[w]);
}

// E[w] /= Ov[w];  ovlp[w] = log Ov[w] + logov[w]
__global__ void finish_energy_kernel(const c128* __restrict__ Ov, const c128* __restrict__ logov,
                                     int W, c128* __restrict__ E, c128* __restrict__ ovlp) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const c128 r = cdiv(cmk(1.0, 0.0), Ov[w]);
  for (int c = 0; c < 3; ++c) E[w * 3 + c] = cmul(E[w * 3 + c], r);
  ovlp[w] = cadd(clog(Ov[w]), logov[w]);
}

// The full R of calculate_R (phmsd_helpers.hpp:200-309) for walker blockIdx.x, all unique
// excitations at once, accumulated in shared memory.  Determinant u (weight wu, holes h, particles
// p, reference orbitals r, Q = INV) adds to row h_a, with c[q] = wu Q[a][q]:
//   + c[q] at p_q,  + wu at p_a,  - wu at r_a            (its compact R row and the identity shift)
//   - sum_q c[q] QQ0[p_q][i] at occ_i for every electron i
// The last term is summed as A QQ0 (A[h][b] = sum of c over (u, a, q) with h_a = h, p_q = b) onto
// the reference orbitals r_i, and the hole electrons' share is moved from r_{h_e} to p_e per
// determinant.  Every electron row also gets sum_u wu at r_i (the identity of every determinant).
// Shared-memory atomics order the sums differently from run to run (the reference reduces R with
// atomics too).
constexpr int PHR_THREADS = 256;
__global__ void __launch_bounds__(PHR_THREADS) phmsd_R_kernel(
    const c128* __restrict__ QQ0, const int* __restrict__ refc, const int* __restrict__ uoff,
    const int* __restrict__ unex, const int* __restrict__ uexc, const int* __restrict__ uinv,
    const c128* __restrict__ INV, int ninv, const c128* __restrict__ wgt, int nuniq, int W,
    int nel, int nact, c128* __restrict__ R) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NA = nel * nact;
  c128* Rs = reinterpret_cast<c128*>(smem_raw);  // [nel][nact]
  c128* As = Rs + NA;                             // [nel][nact]
  c128* Qs = As + NA;                             // [nact][nel]
  __shared__ double red[PHR_THREADS / 32 * 6];
  __shared__ c128 wsum;
  const int w = blockIdx.x;
  const c128* Qw = QQ0 + size_t(w) * nact * nel;
  for (int k = threadIdx.x; k < NA; k += blockDim.x) {
    Rs[k] = cmk(0, 0);
    As[k] = cmk(0, 0);
    Qs[k] = Qw[k];
  }
  c128 ws = cmk(0, 0), z1 = cmk(0, 0), z2 = cmk(0, 0);
  for (int u = threadIdx.x; u < nuniq; u += blockDim.x) ws = cadd(ws, wgt[size_t(u) * W + w]);
  block_sum3(ws, z1, z2, red);
  if (threadIdx.x == 0) wsum = ws;
  __syncthreads();
  auto add = [](c128* x, c128 v) {
    atomicAdd(&x->x, v.x);
    atomicAdd(&x->y, v.y);
  };
  const c128* Iw = INV + size_t(w) * ninv;
  for (int u = 1 + threadIdx.x; u < nuniq; u += blockDim.x) {
    const c128 wu = wgt[size_t(u) * W + w];
    if (wu.x == 0.0 && wu.y == 0.0) continue;
    const int nex = unex[u];
    const int* e = uexc + uoff[u];
    const c128* Qi = Iw + uinv[u];
    for (int a = 0; a < nex; ++a) {
      const int ha = e[a], pa = e[nex + a];
      c128* Ra = Rs + ha * nact;
      c128* Aa = As + ha * nact;
      add(Ra + pa, wu);
      add(Ra + refc[ha], cmk(-wu.x, -wu.y));
      for (int q = 0; q < nex; ++q) {
        const c128 c = cmul(wu, Qi[a * nex + q]);
        add(Ra + e[nex + q], c);
        add(Aa + e[nex + q], c);
      }
      for (int x = 0; x < nex; ++x) {
        const int hx = e[x];
        c128 sx = cmk(0, 0);
        for (int q = 0; q < nex; ++q)
          sx = cadd(sx, cmul(cmul(wu, Qi[a * nex + q]), Qs[e[nex + q] * nel + hx]));
        add(Ra + refc[hx], sx);
        add(Ra + e[nex + x], cmk(-sx.x, -sx.y));
      }
    }
  }
  __syncthreads();
  // R[h][r_i] += delta(h, i) sum_u wu - (A QQ0)[h][i]  (each (h, r_i) once: refc is one-to-one)
  for (int k = threadIdx.x; k < nel * nel; k += blockDim.x) {
    const int hh = k / nel, i = k - hh * nel;
    const c128* Ah = As + hh * nact;
    c128 v = hh == i ? wsum : cmk(0, 0);
    for (int b = 0; b < nact; ++b) v = csub(v, cmul(Ah[b], Qs[b * nel + i]));
    c128* t = Rs + hh * nact + refc[i];
    *t = cadd(*t, v);
  }
  __syncthreads();
  c128* Rw = R + size_t(w) * NA;
  for (int k = threadIdx.x; k < NA; k += blockDim.x) Rw[k] = Rs[k];
}

// x[w][...] *= 1 / Ov[w]
__global__ void scale_by_overlap_kernel(c128* __restrict__ x, long per_w, long stride_w,
                                        const c128* __restrict__ Ov, int W) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= long(W) * per_w) return;
  const int w = int(t / per_w);
  const long e = t - long(w) * per_w;
  c128* v = x + long(w) * stride_w + e;
  *v = cmul(*v, cdiv(cmk(1.0, 0.0), Ov[w]));
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

// ---------------------------------------------------------------------------------------------
// PHMSD trial handle and its log overlap (PHMSD::Log_Overlap, Wavefunctions/PHMSD.cpp:804-900)
// ---------------------------------------------------------------------------------------------
struct afqmc_phmsd_s {
  int device = 0, M = 0, nel[2] = {0, 0}, nact[2] = {0, 0}, nuniq[2] = {0, 0}, ndet = 0;
  int precision = AFQMC_PREC_FP64;  // of the energy's per-(walker, vector) tables
  c128* orbmat[2] = {nullptr, nullptr};
  int* refc[2] = {nullptr, nullptr};
  int* uoff[2] = {nullptr, nullptr};
  int* unex[2] = {nullptr, nullptr};
  int* uexc[2] = {nullptr, nullptr};
  int* det[2] = {nullptr, nullptr};
  c128* coef = nullptr;
  int capW = 0;
  c128 *TMN = nullptr, *TNN = nullptr, *QQ0 = nullptr, *ov[2] = {nullptr, nullptr};
  c128* logov = nullptr;
  // determinants grouped by unique excitation of each spin (CSR rows u, entries = determinant k)
  int* rowptr[2] = {nullptr, nullptr};
  int* kidx[2] = {nullptr, nullptr};
  // excitation shells (equal nex, contiguous unique indices): first index, count, nex
  std::vector<int> sh_k0[2], sh_nd[2], sh_nex[2];
  std::vector<int> uoff_h[2];
  c128* Rfull = nullptr;
  // offset of every unique excitation's inverse block (nex^2 entries) and the total per walker
  int* uinv[2] = {nullptr, nullptr};
  int ninv[2] = {0, 0};
  // energy tables: hole rows (electrons that are a hole of some excitation) and virtual columns
  // (active orbitals outside the reference); per excitation its holes, particles, hole rows and
  // particle columns (uexc4 from uoff4)
  int* hl[2] = {nullptr, nullptr};
  int* vl[2] = {nullptr, nullptr};
  int nh[2] = {0, 0}, nv[2] = {0, 0};
  int* uexc4[2] = {nullptr, nullptr};
  int* uoff4[2] = {nullptr, nullptr};
  bool tables_ok[2] = {false, false};
  // segments {d, j0, j1, single} of the down-spin CSR rows for couple_ke_kernel
  int* kseg = nullptr;
  int nkseg = 0;
  int* krow = nullptr;  // the CSR rows split over several segments (their KEd rows are zeroed)
  int nkrow = 0;
  c128* INV = nullptr;
  // mixed precision: the same inverses in complex64 (float2, half the bytes of INV's buffer)
  c128* INV32 = nullptr;
  // per unique excitation {nex, uoff4, uinv, 0} (one load in the energy tables kernel)
  int4* uhdr[2] = {nullptr, nullptr};
  // the tables kernel's view: within each run of equal nex (a shell of cnt excitations), the
  // fields of uexc4 and the entries of the complex64 inverses INV32 are stored structure-of-
  // arrays (element k of excitation u at base + k cnt + (u - u0)), so that the threads of a
  // warp, which take consecutive excitations, read consecutive addresses; uhdrs[u] = {nex,
  // uexc4s base of u, INV32 base of u, cnt}
  int4* uhdrs[2] = {nullptr, nullptr};
  int* uexc4s[2] = {nullptr, nullptr};
  // Twina holds complex64 elements (the mixed tensor-core half rotation feeding the tables)
  bool twina64[2] = {false, false};
  // the K vectors KEr, KEd, Kdn hold complex64 (the mixed tables path on both spins)
  bool ke64 = false;
  // energy: the Hamiltonian half-rotated with the active orbitals
  bool has_ham = false;
  int Nc = 0;
  double E0 = 0.0;
  c128* lnak[2] = {nullptr, nullptr};  // [Nc][nact][M]
  c128* haj[2] = {nullptr, nullptr};   // [nact][M]
  // mixed precision: Lnak in FP16 split planes for the tensor-core half rotation, made at the
  // first mixed energy (state 0 untried, 1 ready, -1 Lnak complex: the complex128 GEMM runs)
  TcGemmRB* tc_lnak[2] = {nullptr, nullptr};
  int tc_lnak_state[2] = {0, 0};
  void free_tc_lnak() {
    for (int s = 0; s < 2; ++s) {
      tcgemm_rb_destroy(tc_lnak[s]);
      tc_lnak[s] = nullptr;
      tc_lnak_state[s] = 0;
    }
  }
  // energy scratch for a block of walkers
  int capWb = 0;
  c128 *eG[2] = {nullptr, nullptr}, *eQ[2] = {nullptr, nullptr}, *eov[2] = {nullptr, nullptr};
  c128 *eTMN = nullptr, *eTNN = nullptr, *elogov = nullptr, *eOv = nullptr;
  c128 *wgt = nullptr, *Swia = nullptr, *Twina = nullptr, *KEr = nullptr, *KEd = nullptr;
  c128* wgtT = nullptr;  // wgt transposed, [w][u], for the tables kernel
  c128 *KEl = nullptr, *Kdn = nullptr, *R = nullptr, *el = nullptr;
  size_t R_elems = 0, KEl_elems = 0;
  int capCore = 0;  // walkers the Woodbury factors / density-matrix buffers hold
  void free_energy_scratch() {
    for (c128** q : {&Swia, &Twina, &KEr, &KEd, &KEl, &Kdn, &R, &el})
      if (*q) {
        cudaFree(*q);
        *q = nullptr;
      }
    capWb = 0;
  }
  void free_core_scratch() {
    for (c128** q : {&eG[0], &eG[1], &eQ[0], &eQ[1], &eov[0], &eov[1], &eTMN, &eTNN, &elogov,
                     &eOv, &wgt, &wgtT, &Rfull, &INV, &INV32})
      if (*q) {
        cudaFree(*q);
        *q = nullptr;
      }
    capCore = 0;
  }
  void free_scratch() {
    for (c128** p : {&TMN, &TNN, &QQ0, &ov[0], &ov[1], &logov})
      if (*p) {
        cudaFree(*p);
        *p = nullptr;
      }
    capW = 0;
  }
  ~afqmc_phmsd_s() {
    free_scratch();
    free_energy_scratch();
    free_core_scratch();
    free_tc_lnak();
    for (int s = 0; s < 2; ++s) {
      cudaFree(rowptr[s]);
      cudaFree(kidx[s]);
      cudaFree(uinv[s]);
      cudaFree(hl[s]);
      cudaFree(vl[s]);
      cudaFree(uexc4[s]);
      cudaFree(uoff4[s]);
      cudaFree(uhdr[s]);
      cudaFree(uhdrs[s]);
      cudaFree(uexc4s[s]);
      cudaFree(lnak[s]);
      cudaFree(haj[s]);
      cudaFree(orbmat[s]);
      cudaFree(refc[s]);
      cudaFree(uoff[s]);
      cudaFree(unex[s]);
      cudaFree(uexc[s]);
      cudaFree(det[s]);
    }
    cudaFree(coef);
    cudaFree(kseg);
    cudaFree(krow);
  }
};

namespace {

template <typename T>
int to_device(T** dst, const T* src, size_t n) {
  if (n == 0) n = 1;
  AFQMC_CUDA_TRY(cudaMalloc(dst, n * sizeof(T)));
  if (src) AFQMC_CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return AFQMC_OK;
}

int phmsd_scratch(afqmc_phmsd h, int W) {
  if (h->capW >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  h->free_scratch();
  const int na = h->nact[0] > h->nact[1] ? h->nact[0] : h->nact[1];
  const int ne = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  AFQMC_CUDA_TRY(cudaMalloc(&h->TMN, sizeof(c128) * size_t(W) * na * ne));
  AFQMC_CUDA_TRY(cudaMalloc(&h->QQ0, sizeof(c128) * size_t(W) * na * ne));
  AFQMC_CUDA_TRY(cudaMalloc(&h->TNN, sizeof(c128) * size_t(W) * ne * ne));
  for (int s = 0; s < 2; ++s)
    AFQMC_CUDA_TRY(cudaMalloc(&h->ov[s], sizeof(c128) * size_t(W) * h->nuniq[s]));
  AFQMC_CUDA_TRY(cudaMalloc(&h->logov, sizeof(c128) * size_t(W)));
  h->capW = W;
  return AFQMC_OK;
}

}  // namespace

extern "C" int afqmc_phmsd_create(int M, int nup, int ndn, int nact_up, int nact_dn,
                                  const afqmc_c128* orbmat_up, const afqmc_c128* orbmat_dn,
                                  const int* refc_up, const int* refc_dn, int nuniq_up,
                                  const int* nex_up, const int* exc_up, int nuniq_dn,
                                  const int* nex_dn, const int* exc_dn, int ndet,
                                  const int* det_up, const int* det_dn, const afqmc_c128* coef,
                                  afqmc_phmsd* out) {
  AFQMC_CHECK_ARG(out && orbmat_up && orbmat_dn && refc_up && refc_dn && det_up && det_dn && coef,
                  "afqmc_phmsd_create: null argument");
  *out = nullptr;
  AFQMC_CHECK_ARG(M > 0 && nup > 0 && ndn > 0 && nact_up >= nup && nact_dn >= ndn &&
                      nact_up <= M && nact_dn <= M && nuniq_up >= 1 && nuniq_dn >= 1 && ndet >= 1,
                  "afqmc_phmsd_create: bad sizes (M=%d nup=%d ndn=%d nact=%d/%d nuniq=%d/%d "
                  "ndet=%d)", M, nup, ndn, nact_up, nact_dn, nuniq_up, nuniq_dn, ndet);
  const int nel[2] = {nup, ndn}, nact[2] = {nact_up, nact_dn}, nuniq[2] = {nuniq_up, nuniq_dn};
  const int* refc[2] = {refc_up, refc_dn};
  const int* nexs[2] = {nex_up, nex_dn};
  const int* excs[2] = {exc_up, exc_dn};
  // host validation of every index the kernels will read with
  std::vector<int> off[2], nex[2];
  for (int s = 0; s < 2; ++s) {
    for (int i = 0; i < nel[s]; ++i)
      AFQMC_CHECK_ARG(refc[s][i] >= 0 && refc[s][i] < nact[s],
                      "afqmc_phmsd_create: refc[%d][%d] = %d outside [0, %d)", s, i, refc[s][i],
                      nact[s]);
    AFQMC_CHECK_ARG(nuniq[s] == 1 || (nexs[s] && excs[s]),
                    "afqmc_phmsd_create: null excitation list");
    off[s].assign(nuniq[s], 0);
    nex[s].assign(nuniq[s], 0);
    int pos = 0;
    for (int u = 1; u < nuniq[s]; ++u) {
      const int n = nexs[s][u - 1];
      AFQMC_CHECK_ARG(n >= 1 && n <= PH_NEX_MAX && n <= nel[s],
                      "afqmc_phmsd_create: excitation %d of spin %d has nex = %d (1..%d)", u, s,
                      n, PH_NEX_MAX);
      off[s][u] = pos;
      nex[s][u] = n;
      for (int q = 0; q < n; ++q) {
        const int hole = excs[s][pos + q], part = excs[s][pos + n + q];
        AFQMC_CHECK_ARG(hole >= 0 && hole < nel[s] && part >= 0 && part < nact[s],
                        "afqmc_phmsd_create: excitation %d of spin %d: hole %d (< %d), particle "
                        "%d (< %d)", u, s, hole, nel[s], part, nact[s]);
      }
      pos += 2 * n;
    }
  }
  for (int s = 0; s < 2; ++s)
    for (int u = 2; u < nuniq[s]; ++u)
      AFQMC_CHECK_ARG(nex[s][u] >= nex[s][u - 1],
                      "afqmc_phmsd_create: unique excitations of spin %d must be ordered by "
                      "excitation number (u = %d has %d after %d)", s, u, nex[s][u],
                      nex[s][u - 1]);
  for (int k = 0; k < ndet; ++k)
    AFQMC_CHECK_ARG(det_up[k] >= 0 && det_up[k] < nuniq_up && det_dn[k] >= 0 &&
                        det_dn[k] < nuniq_dn,
                    "afqmc_phmsd_create: determinant %d couples (%d, %d) outside (%d, %d)", k,
                    det_up[k], det_dn[k], nuniq_up, nuniq_dn);
  // Internal order of the unique excitations: by excitation number, then holes, then particles
  // (a permutation that changes no result).  Neighbouring threads of the energy kernels then
  // evaluate determinants with the same holes and nearby particles, whose table reads fall on
  // neighbouring shared-memory words.
  std::vector<int> exc_sorted[2], det_sorted[2];
  const int* det_in[2] = {det_up, det_dn};
  for (int s = 0; s < 2; ++s) {
    std::vector<int> order(nuniq[s] > 1 ? nuniq[s] - 1 : 0);
    for (size_t j = 0; j < order.size(); ++j) order[j] = int(j) + 1;
    auto key_less = [&](int a, int b) {
      if (nex[s][a] != nex[s][b]) return nex[s][a] < nex[s][b];
      const int n = nex[s][a];
      return std::lexicographical_compare(excs[s] + off[s][a], excs[s] + off[s][a] + 2 * n,
                                          excs[s] + off[s][b], excs[s] + off[s][b] + 2 * n);
    };
    std::stable_sort(order.begin(), order.end(), key_less);
    std::vector<int> newidx(nuniq[s], 0), noff(nuniq[s], 0), nnex(nuniq[s], 0);
    int pos = 0;
    for (size_t j = 0; j < order.size(); ++j) {
      const int u = order[j], v = int(j) + 1, n = nex[s][u];
      newidx[u] = v;
      noff[v] = pos;
      nnex[v] = n;
      exc_sorted[s].insert(exc_sorted[s].end(), excs[s] + off[s][u], excs[s] + off[s][u] + 2 * n);
      pos += 2 * n;
    }
    det_sorted[s].resize(ndet);
    for (int k = 0; k < ndet; ++k) det_sorted[s][k] = newidx[det_in[s][k]];
    off[s] = noff;
    nex[s] = nnex;
    excs[s] = exc_sorted[s].data();
  }
  det_up = det_sorted[0].data();
  det_dn = det_sorted[1].data();
  std::unique_ptr<afqmc_phmsd_s> h(new afqmc_phmsd_s);
  cudaGetDevice(&h->device);
  h->M = M;
  h->ndet = ndet;
  const afqmc_c128* orb[2] = {orbmat_up, orbmat_dn};
  for (int s = 0; s < 2; ++s) {
    h->nel[s] = nel[s];
    h->nact[s] = nact[s];
    h->nuniq[s] = nuniq[s];
    AFQMC_TRY(to_device(&h->orbmat[s], reinterpret_cast<const c128*>(orb[s]),
                        size_t(nact[s]) * M));
    AFQMC_TRY(to_device(&h->refc[s], refc[s], size_t(nel[s])));
    AFQMC_TRY(to_device(&h->uoff[s], off[s].data(), off[s].size()));
    AFQMC_TRY(to_device(&h->unex[s], nex[s].data(), nex[s].size()));
    size_t nexc = 0;
    for (int u = 1; u < nuniq[s]; ++u) nexc += 2 * size_t(nex[s][u]);
    AFQMC_TRY(to_device(&h->uexc[s], nuniq[s] > 1 ? excs[s] : nullptr, nexc));
  }
  AFQMC_TRY(to_device(&h->det[0], det_up, size_t(ndet)));
  AFQMC_TRY(to_device(&h->det[1], det_dn, size_t(ndet)));
  AFQMC_TRY(to_device(&h->coef, reinterpret_cast<const c128*>(coef), size_t(ndet)));
  const int* dets[2] = {det_up, det_dn};
  for (int s = 0; s < 2; ++s) {
    // CSR of the determinants by this spin's unique excitation, in determinant order
    std::vector<int> rp(nuniq[s] + 1, 0), ki(ndet);
    for (int k = 0; k < ndet; ++k) ++rp[dets[s][k] + 1];
    for (int u = 0; u < nuniq[s]; ++u) rp[u + 1] += rp[u];
    std::vector<int> pos(rp.begin(), rp.end() - 1);
    for (int k = 0; k < ndet; ++k) ki[pos[dets[s][k]]++] = k;
    AFQMC_TRY(to_device(&h->rowptr[s], rp.data(), rp.size()));
    AFQMC_TRY(to_device(&h->kidx[s], ki.data(), ki.size()));
    if (s == 1) {
      std::vector<int> sg;
      for (int u = 0; u < nuniq[1]; ++u) {
        const bool single = rp[u + 1] - rp[u] <= KE_SEG;
        for (int j = rp[u]; j < rp[u + 1] || j == rp[u]; j += KE_SEG) {
          sg.insert(sg.end(), {u, j, std::min(j + KE_SEG, rp[u + 1]), single ? 1 : 0});
          if (rp[u + 1] == rp[u]) break;
        }
      }
      h->nkseg = int(sg.size() / 4);
      AFQMC_TRY(to_device(&h->kseg, sg.data(), sg.size()));
      std::vector<int> kr;
      for (int u = 0; u < nuniq[1]; ++u)
        if (rp[u + 1] - rp[u] > KE_SEG) kr.push_back(u);
      h->nkrow = int(kr.size());
      AFQMC_TRY(to_device(&h->krow, kr.data(), kr.size()));
    }
    // shells of equal excitation number
    for (int u = 1; u < nuniq[s]; ++u) {
      if (h->sh_nex[s].empty() || h->sh_nex[s].back() != nex[s][u]) {
        h->sh_k0[s].push_back(u);
        h->sh_nd[s].push_back(0);
        h->sh_nex[s].push_back(nex[s][u]);
      }
      ++h->sh_nd[s].back();
    }
    h->uoff_h[s] = off[s];
    std::vector<int> io(nuniq[s], 0);
    for (int u = 1; u < nuniq[s]; ++u) {
      io[u] = h->ninv[s];
      h->ninv[s] += nex[s][u] * nex[s][u];
    }
    AFQMC_TRY(to_device(&h->uinv[s], io.data(), io.size()));
    // table indexing of the excitations
    std::vector<int> hrow(nel[s], -1), vcol(nact[s], -1), hlv, vlv;
    for (int u = 1; u < nuniq[s]; ++u)
      for (int a = 0; a < nex[s][u]; ++a) hrow[excs[s][off[s][u] + a]] = 0;
    for (int i = 0; i < nel[s]; ++i)
      if (hrow[i] == 0) {
        hrow[i] = int(hlv.size());
        hlv.push_back(i);
      }
    std::vector<char> isref(nact[s], 0);
    for (int i = 0; i < nel[s]; ++i) isref[refc[s][i]] = 1;
    for (int x = 0; x < nact[s]; ++x)
      if (!isref[x]) {
        vcol[x] = int(vlv.size());
        vlv.push_back(x);
      }
    std::vector<int> e4, o4(nuniq[s], 0);
    bool ok = true;
    for (int u = 1; u < nuniq[s]; ++u) {
      const int n = nex[s][u], *e = excs[s] + off[s][u];
      o4[u] = int(e4.size());
      for (int a = 0; a < 2 * n; ++a) e4.push_back(e[a]);
      for (int a = 0; a < n; ++a) e4.push_back(hrow[e[a]]);
      for (int a = 0; a < n; ++a) {
        e4.push_back(vcol[e[n + a]]);
        ok = ok && vcol[e[n + a]] >= 0;  // a particle inside the reference: R-row kernels
      }
    }
    h->nh[s] = int(hlv.size());
    h->nv[s] = int(vlv.size());
    h->tables_ok[s] = ok;
    AFQMC_TRY(to_device(&h->hl[s], hlv.data(), hlv.size()));
    AFQMC_TRY(to_device(&h->vl[s], vlv.data(), vlv.size()));
    AFQMC_TRY(to_device(&h->uexc4[s], e4.data(), e4.size()));
    AFQMC_TRY(to_device(&h->uoff4[s], o4.data(), o4.size()));
    std::vector<int4> hd(nuniq[s], make_int4(0, 0, 0, 0));
    for (int u = 1; u < nuniq[s]; ++u) hd[u] = make_int4(nex[s][u], o4[u], io[u], 1);
    AFQMC_TRY(to_device(&h->uhdr[s], hd.data(), hd.size()));
    // structure-of-arrays copies per shell (runs of equal nex, nex non-decreasing in u)
    std::vector<int4> hs(nuniq[s], make_int4(0, 0, 0, 1));
    std::vector<int> e4s(e4.size() > 0 ? e4.size() : 1, 0);
    for (int u0 = 1; u0 < nuniq[s];) {
      const int n = nex[s][u0];
      int cnt = 0;
      while (u0 + cnt < nuniq[s] && nex[s][u0 + cnt] == n) ++cnt;
      const int ebase = o4[u0], qbase = io[u0];
      for (int t = 0; t < cnt; ++t) {
        const int u = u0 + t;
        hs[u] = make_int4(n, ebase + t, qbase + t, cnt);
        for (int f = 0; f < 4 * n; ++f) e4s[size_t(ebase) + size_t(f) * cnt + t] = e4[o4[u] + f];
      }
      u0 += cnt;
    }
    AFQMC_TRY(to_device(&h->uhdrs[s], hs.data(), hs.size()));
    AFQMC_TRY(to_device(&h->uexc4s[s], e4s.data(), e4s.size()));
  }
  *out = h.release();
  return AFQMC_OK;
}

extern "C" int afqmc_phmsd_destroy(afqmc_phmsd h) {
  if (h) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(h->device);
    delete h;
    cudaSetDevice(prev);
  }
  return AFQMC_OK;
}

extern "C" int afqmc_phmsd_set_precision(afqmc_phmsd h, int precision) {
  AFQMC_CHECK_ARG(h && (precision == AFQMC_PREC_FP64 || precision == AFQMC_PREC_MIXED),
                  "afqmc_phmsd_set_precision: precision must be FP64 or MIXED");
  h->precision = precision;
  return AFQMC_OK;
}

extern "C" int afqmc_phmsd_info(afqmc_phmsd h, int* dims) {
  AFQMC_CHECK_ARG(h && dims, "afqmc_phmsd_info: null argument");
  dims[0] = h->M;
  dims[1] = h->nel[0];
  dims[2] = h->nel[1];
  dims[3] = h->nact[0];
  dims[4] = h->nact[1];
  dims[5] = h->has_ham ? h->Nc : 0;
  return AFQMC_OK;
}

extern "C" int afqmc_phmsd_log_overlap(afqmc_phmsd h, const afqmc_c128* wbuf, long ldS,
                                       afqmc_c128* ovlp, int W, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && wbuf && ovlp, "afqmc_phmsd_log_overlap: null argument");
  AFQMC_CHECK_ARG(W >= 0 && ldS >= long(h->M) * (h->nel[0] + h->nel[1]),
                  "afqmc_phmsd_log_overlap: W=%d, walker stride %ld < M (nup + ndn)", W, ldS);
  if (W == 0) return AFQMC_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  AFQMC_TRY(phmsd_scratch(h, W));
  AFQMC_CUDA_TRY(cudaMemsetAsync(h->logov, 0, sizeof(c128) * W, s));
  const c128* S = reinterpret_cast<const c128*>(wbuf);
  for (int sp = 0; sp < 2; ++sp) {
    const int N = h->nel[sp], na = h->nact[sp];
    const c128* Ss = S + (sp == 0 ? 0 : long(h->M) * h->nel[0]);
    // TMN = A S   (math::product(A,B,TMN), density_matrix.hpp:510)
    GemmParams p{};
    p.m = na; p.n = N; p.k = h->M;
    p.A = h->orbmat[sp]; p.lda = h->M; p.strideA = 0;
    p.B = Ss; p.ldb = N; p.strideB = ldS;
    p.C = h->TMN; p.ldc = N; p.strideC = long(na) * N;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, W, GN, false, GN, false, p));
    gather_ref_rows_kernel<<<W, 128, 0, s>>>(h->TMN, h->refc[sp], h->TNN, na, N);
    AFQMC_TRY(launch_status("gather_ref_rows_kernel"));
    // log det TNN accumulated, TNN <- TNN^{-1}
    AFQMC_TRY(batched_logdet_inverse(s, h->TNN, long(N) * N, h->TNN, long(N) * N, h->logov, W, N,
                                     true, cmk(1, 0), cmk(0, 0)));
    // QQ0 = TMN TNN^{-1}
    GemmParams q{};
    q.m = na; q.n = N; q.k = N;
    q.A = h->TMN; q.lda = N; q.strideA = long(na) * N;
    q.B = h->TNN; q.ldb = N; q.strideB = long(N) * N;
    q.C = h->QQ0; q.ldc = N; q.strideC = long(na) * N;
    q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, W, GN, false, GN, false, q));
    const long nt = long(h->nuniq[sp]) * W;
    excitation_det_kernel<<<unsigned((nt + 127) / 128), 128, 0, s>>>(
        h->QQ0, h->uoff[sp], h->unex[sp], h->uexc[sp], h->nuniq[sp], W, na, N, h->ov[sp]);
    AFQMC_TRY(launch_status("excitation_det_kernel"));
  }
  phmsd_combine_kernel<<<W, PH_THREADS, 0, s>>>(h->ov[0], h->ov[1], h->nuniq[0], h->nuniq[1],
                                                h->det[0], h->det[1], h->coef, h->ndet, h->logov,
                                                reinterpret_cast<c128*>(ovlp));
  return launch_status("phmsd_combine_kernel");
}

// ---------------------------------------------------------------------------------------------
// PHMSD energy (PHMSD::energy_alg1, Wavefunctions/PHMSD.cpp:376-546, COLLINEAR walkers)
// ---------------------------------------------------------------------------------------------
extern "C" int afqmc_phmsd_set_hamiltonian(afqmc_phmsd h, const double* Likn, int nspin_H2,
                                           const afqmc_c128* hij, int nspin_H1, int Nc,
                                           double E0) {
  AFQMC_CHECK_ARG(h && Likn && hij, "afqmc_phmsd_set_hamiltonian: null argument");
  AFQMC_CHECK_ARG(Nc > 0 && (nspin_H2 == 1 || nspin_H2 == 2) && (nspin_H1 == 1 || nspin_H1 == 2),
                  "afqmc_phmsd_set_hamiltonian: Nc=%d nspin_H2=%d nspin_H1=%d", Nc, nspin_H2,
                  nspin_H1);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  const long M = h->M, MM = M * M;
  double* L = nullptr;
  c128 *hd = nullptr, *tmp = nullptr;
  int st = AFQMC_OK;
  auto fail = [&](int code) {
    cudaFree(L);
    cudaFree(hd);
    cudaFree(tmp);
    cudaSetDevice(prev);
    return code;
  };
  if (cudaMalloc(&L, sizeof(double) * nspin_H2 * MM * Nc) != cudaSuccess ||
      cudaMalloc(&hd, sizeof(c128) * nspin_H1 * MM) != cudaSuccess) {
    set_error_detail("afqmc_phmsd_set_hamiltonian: out of device memory");
    return fail(AFQMC_ERR_ALLOC);
  }
  cudaMemcpy(L, Likn, sizeof(double) * nspin_H2 * MM * Nc, cudaMemcpyHostToDevice);
  cudaMemcpy(hd, hij, sizeof(c128) * nspin_H1 * MM, cudaMemcpyHostToDevice);
  h->free_tc_lnak();
  for (int sp = 0; sp < 2; ++sp) {
    const int na = h->nact[sp];
    cudaFree(h->lnak[sp]);
    cudaFree(h->haj[sp]);
    h->lnak[sp] = h->haj[sp] = nullptr;
    if (cudaMalloc(&h->lnak[sp], sizeof(c128) * size_t(Nc) * na * M) != cudaSuccess ||
        cudaMalloc(&h->haj[sp], sizeof(c128) * size_t(na) * M) != cudaSuccess ||
        cudaMalloc(&tmp, sizeof(c128) * size_t(na) * MM * Nc) != cudaSuccess) {
      set_error_detail("afqmc_phmsd_set_hamiltonian: out of device memory");
      return fail(AFQMC_ERR_ALLOC);
    }
    // tmp[a][(k, n)] = sum_i OrbMat[a][i] L[i][(k, n)]  -> Lnak[n][a][k]
    GemmParams p{};
    p.m = na; p.n = int(M * Nc); p.k = int(M);
    p.A = h->orbmat[sp]; p.lda = M; p.strideA = 0;
    p.B = L + size_t(sp % nspin_H2) * MM * Nc; p.ldb = M * Nc; p.strideB = 0;
    p.C = tmp; p.ldc = M * Nc; p.strideC = 0;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    if ((st = zgemm(nullptr, 1, GN, false, GN, true, p))) return fail(st);
    const long tot = long(na) * M * Nc;
    lnak_act_reorder_kernel<<<unsigned((tot + 255) / 256), 256>>>(tmp, h->lnak[sp], na, int(M),
                                                                   Nc);
    if ((st = launch_status("lnak_act_reorder_kernel"))) return fail(st);
    // haj = OrbMat h1
    GemmParams q{};
    q.m = na; q.n = int(M); q.k = int(M);
    q.A = h->orbmat[sp]; q.lda = M;
    q.B = hd + size_t(sp % nspin_H1) * MM; q.ldb = M;
    q.C = h->haj[sp]; q.ldc = M;
    q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
    if ((st = zgemm(nullptr, 1, GN, false, GN, false, q))) return fail(st);
    if (cudaDeviceSynchronize() != cudaSuccess) {
      set_error_detail("afqmc_phmsd_set_hamiltonian: %s", cudaGetErrorString(cudaGetLastError()));
      return fail(AFQMC_ERR_CUDA);
    }
    cudaFree(tmp);
    tmp = nullptr;
  }
  h->free_energy_scratch();  // sized for the previous number of Cholesky vectors
  h->Nc = Nc;
  h->E0 = E0;
  h->has_ham = true;
  return fail(AFQMC_OK);
}

namespace {

int scratch_alloc(c128** p, size_t n) {
  if (cudaMalloc(p, sizeof(c128) * (n ? n : 1)) != cudaSuccess) {
    set_error_detail("PHMSD scratch: out of device memory (%zu bytes)", sizeof(c128) * n);
    return AFQMC_ERR_ALLOC;
  }
  return AFQMC_OK;
}

// per-block buffers of the Woodbury factors, excitation overlaps, weights and R (density matrix
// and energy), for Wb walkers
int phmsd_core_scratch(afqmc_phmsd h, int Wb) {
  if (h->capCore >= Wb) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  h->free_core_scratch();
  const size_t na = std::max(h->nact[0], h->nact[1]), ne = std::max(h->nel[0], h->nel[1]);
  const size_t M = h->M, nu = std::max(h->nuniq[0], h->nuniq[1]);
  for (int s = 0; s < 2; ++s) {
    AFQMC_TRY(scratch_alloc(&h->eG[s], size_t(Wb) * ne * M));
    AFQMC_TRY(scratch_alloc(&h->eQ[s], size_t(Wb) * na * ne));
    AFQMC_TRY(scratch_alloc(&h->eov[s], size_t(Wb) * h->nuniq[s]));
  }
  AFQMC_TRY(scratch_alloc(&h->eTMN, size_t(Wb) * na * ne));
  AFQMC_TRY(scratch_alloc(&h->eTNN, size_t(Wb) * ne * ne));
  AFQMC_TRY(scratch_alloc(&h->elogov, Wb));
  AFQMC_TRY(scratch_alloc(&h->eOv, Wb));
  AFQMC_TRY(scratch_alloc(&h->wgt, nu * Wb));
  AFQMC_TRY(scratch_alloc(&h->wgtT, nu * Wb));
  AFQMC_TRY(scratch_alloc(&h->Rfull, size_t(Wb) * ne * na));
  AFQMC_TRY(scratch_alloc(&h->INV, size_t(Wb) * std::max(h->ninv[0], h->ninv[1])));
  AFQMC_TRY(scratch_alloc(&h->INV32, (size_t(Wb) * std::max(h->ninv[0], h->ninv[1]) + 1) / 2));
  h->capCore = Wb;
  return AFQMC_OK;
}

// the energy's additional per-block buffers (half-rotated tensors, K vectors, R rows)
int phmsd_energy_scratch(afqmc_phmsd h, int Wb) {
  AFQMC_TRY(phmsd_core_scratch(h, Wb));
  if (h->capWb >= Wb) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  h->free_energy_scratch();
  const size_t na = std::max(h->nact[0], h->nact[1]), ne = std::max(h->nel[0], h->nel[1]);
  const size_t Nc = h->Nc;
  int maxnd = 1;
  size_t maxR = 1;
  for (int s = 0; s < 2; ++s)
    for (size_t j = 0; j < h->sh_nd[s].size(); ++j) {
      maxnd = std::max(maxnd, h->sh_nd[s][j]);
      maxR = std::max(maxR, size_t(h->sh_nd[s][j]) * h->sh_nex[s][j] * h->nact[s]);
    }
  AFQMC_TRY(scratch_alloc(&h->Swia, size_t(Wb) * ne * na));
  AFQMC_TRY(scratch_alloc(&h->Twina, size_t(Wb) * ne * Nc * na));
  AFQMC_TRY(scratch_alloc(&h->KEr, size_t(h->nuniq[0]) * Wb * Nc));
  AFQMC_TRY(scratch_alloc(&h->KEd, size_t(h->nuniq[1]) * Wb * Nc));
  AFQMC_TRY(scratch_alloc(&h->KEl, size_t(maxnd) * Wb * Nc));
  AFQMC_TRY(scratch_alloc(&h->Kdn, size_t(Wb) * Nc));
  AFQMC_TRY(scratch_alloc(&h->R, maxR * Wb));
  AFQMC_TRY(scratch_alloc(&h->el, 5 * size_t(Wb)));
  h->capWb = Wb;
  return AFQMC_OK;
}

// density matrix, Woodbury factors and excitation overlaps of spin sp for walkers [w0, w0+nb)
int phmsd_spin_factors(afqmc_phmsd h, cudaStream_t s, int sp, const c128* S, long ldS, int nb) {
  const int N = h->nel[sp], na = h->nact[sp];
  GemmParams p{};
  p.m = na; p.n = N; p.k = h->M;
  p.A = h->orbmat[sp]; p.lda = h->M; p.strideA = 0;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = h->eTMN; p.ldc = N; p.strideC = long(na) * N;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, nb, GN, false, GN, false, p));
  gather_ref_rows_kernel<<<nb, 128, 0, s>>>(h->eTMN, h->refc[sp], h->eTNN, na, N);
  AFQMC_TRY(launch_status("gather_ref_rows_kernel"));
  AFQMC_TRY(batched_logdet_inverse(s, h->eTNN, long(N) * N, h->eTNN, long(N) * N, h->elogov, nb,
                                   N, true, cmk(1, 0), cmk(0, 0)));
  // QQ0 = TAB TNN^{-1};  G = TNN^{-T} S^T  (compact, density_matrix.hpp:696-703)
  GemmParams q{};
  q.m = na; q.n = N; q.k = N;
  q.A = h->eTMN; q.lda = N; q.strideA = long(na) * N;
  q.B = h->eTNN; q.ldb = N; q.strideB = long(N) * N;
  q.C = h->eQ[sp]; q.ldc = N; q.strideC = long(na) * N;
  q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, nb, GN, false, GN, false, q));
  GemmParams g{};
  g.m = N; g.n = h->M; g.k = N;
  g.A = h->eTNN; g.lda = N; g.strideA = long(N) * N;
  g.B = S; g.ldb = N; g.strideB = ldS;
  g.C = h->eG[sp]; g.ldc = h->M; g.strideC = long(N) * h->M;
  g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, nb, GT, false, GT, false, g));
  const long nt = long(h->nuniq[sp]) * nb;
  excitation_det_kernel<<<unsigned((nt + 127) / 128), 128, 0, s>>>(
      h->eQ[sp], h->uoff[sp], h->unex[sp], h->uexc[sp], h->nuniq[sp], nb, na, N, h->eov[sp]);
  return launch_status("excitation_det_kernel");
}

// Swia = G haj^T, Twina = G Lnak^T for spin sp
// shared memory of excited_energy_tables_kernel: nbuf buffers of the rows t_j, Qv, and ng
// pairs of tables Sf, SU, in elements of elem bytes
size_t excited_tables_smem(afqmc_phmsd h, int sp, size_t elem, int ng, int nbuf) {
  const size_t N = h->nel[sp], na = h->nact[sp], nv = h->nv[sp], nh = h->nh[sp];
  return (size_t(nbuf) * N * na + N * nv + size_t(ng) * (N * nv + nh * nv)) * elem +
         (N + nh + nv) * sizeof(int);
}

// the energy of spin sp runs the per-(walker, n) tables kernel (else the per-shell R rows)
bool phmsd_tables(afqmc_phmsd h, int sp) {
  const size_t esz = h->precision == AFQMC_PREC_MIXED ? sizeof(c64) : sizeof(c128);
  return h->tables_ok[sp] && excited_tables_smem(h, sp, esz, 1, 1) <= 200 * 1024;
}

// the FP16 split planes of Lnak for the mixed half rotation, made at the first mixed energy
// (state 1 ready, -1 Lnak complex or K not a multiple of 8: the complex128 GEMM runs)
int phmsd_tc_prepare(afqmc_phmsd h, cudaStream_t s, int sp) {
  if (h->tc_lnak_state[sp] != 0) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  const int st = tcgemm_rb_create(&h->tc_lnak[sp], h->lnak[sp], long(h->Nc) * h->nact[sp],
                                  h->M, h->M);
  if (st != AFQMC_OK && st != AFQMC_ERR_UNSUPPORTED) return st;
  h->tc_lnak_state[sp] = st == AFQMC_OK ? 1 : -1;
  return AFQMC_OK;
}

int phmsd_half_rotated(afqmc_phmsd h, cudaStream_t s, int sp, int nb) {
  const int N = h->nel[sp], na = h->nact[sp];
  GemmParams p{};
  p.m = nb * N; p.n = na; p.k = h->M;
  p.A = h->eG[sp]; p.lda = h->M;
  p.B = h->haj[sp]; p.ldb = h->M;
  p.C = h->Swia; p.ldc = na;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, 1, GN, false, GT, false, p));
  if (h->precision == AFQMC_PREC_MIXED) {
    // mixed precision: the FP16 split on the tensor cores when Lnak is real
    AFQMC_TRY(phmsd_tc_prepare(h, s, sp));
    if (h->tc_lnak_state[sp] == 1) {
      // complex64 output where only the tables kernels read it (both spins, h->ke64)
      h->twina64[sp] = h->ke64;
      return tcgemm_rb_run(s, h->tc_lnak[sp], h->eG[sp], h->M, nb * N, h->Twina,
                           long(h->Nc) * na, h->twina64[sp]);
    }
  }
  h->twina64[sp] = false;
  GemmParams q{};
  q.m = nb * N; q.n = h->Nc * na; q.k = h->M;
  q.A = h->eG[sp]; q.lda = h->M;
  q.B = h->lnak[sp]; q.ldb = h->M;
  q.C = h->Twina; q.ldc = long(h->Nc) * na;
  q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
  return zgemm(s, 1, GN, false, GT, false, q);
}

// The reference determinant's and the excited determinants' energies of spin sp
// (PHMSD.cpp:438-531): Kref [W][Nc] receives the reference K vector; KEout the excited ones
// [u][W][Nc] (first spin), or `cross` [u][W][Nc] is contracted with them (second spin).
int phmsd_reference_and_excited(afqmc_phmsd h, cudaStream_t s, int sp, int nb, double E0,
                                c128* Kref, c128* KEout, const c128* cross, c128* E) {
  const int N = h->nel[sp], na = h->nact[sp], Nc = h->Nc;
  // the 2-body terms from per-(walker, n) tables when they fit in shared memory, else per shell
  // from the R rows (the reference kernel's formulation)
  const bool mixed = h->precision == AFQMC_PREC_MIXED;
  const bool tables = phmsd_tables(h, sp);
  if (!tables) {
    ph_reference_kernel<<<nb, PH_THREADS, 0, s>>>(h->Swia, h->Twina, h->refc[sp], N, Nc, na, E0,
                                                  h->eOv, E, Kref);
    AFQMC_TRY(launch_status("ph_reference_kernel"));
  }
  AFQMC_CUDA_TRY(cudaMemsetAsync(h->el, 0, sizeof(c128) * 5 * nb, s));
  // per shell (the R-row formulation) only without the tables; with them every unique
  // excitation's 1-body term comes from its Woodbury inverse in one launch below
  for (size_t j = 0; j < h->sh_k0[sp].size() && !tables; ++j) {
    const int k0 = h->sh_k0[sp][j], nd = h->sh_nd[sp][j], nex = h->sh_nex[sp][j];
    const int* iex = h->uexc[sp] + h->uoff_h[sp][k0];
    const size_t Rn = size_t(nb) * nd * nex * na;
    AFQMC_CUDA_TRY(cudaMemsetAsync(h->R, 0, sizeof(c128) * Rn, s));
    const long nt = long(nb) * nd;
    compact_R_kernel<<<unsigned((nt + 127) / 128), 128, 0, s>>>(h->eQ[sp], iex, h->refc[sp], nd,
                                                                nex, nb, na, N, h->R);
    AFQMC_TRY(launch_status("compact_R_kernel"));
    const c128* w = h->wgt + size_t(k0) * nb;
    dim3 grid(nd, nb);
    ph_excited_1body_kernel<<<grid, PH_THREADS, 0, s>>>(iex, h->refc[sp], h->Swia, h->R, w, nb,
                                                        nd, nex, na, N, h->el);
    AFQMC_TRY(launch_status("ph_excited_1body_kernel"));
    c128* KE = cross ? h->KEl : KEout + size_t(k0) * nb * Nc;
    const size_t smem = size_t(nex) * na * sizeof(c128) + 2 * size_t(N) * sizeof(int);
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(ph_excited_2body_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    ph_excited_2body_kernel<<<grid, PH_THREADS, smem, s>>>(iex, h->refc[sp], h->Twina, h->R, w,
                                                          nb, nd, nex, na, N, Nc, h->el + nb,
                                                          h->el + 2 * nb, KE);
    AFQMC_TRY(launch_status("ph_excited_2body_kernel"));
    if (cross) {
      cross_ej_kernel<c128><<<nb, PH_THREADS, 0, s>>>(cross + size_t(k0) * nb * Nc, h->KEl, nd,
                                                      nb, Nc, E);
      AFQMC_TRY(launch_status("cross_ej_kernel"));
    }
  }
  if (tables) {
    if (h->nuniq[sp] > 1) {
      const long nt = long(h->nuniq[sp] - 1) * nb;
      woodbury_inverses_kernel<<<unsigned((nt + 127) / 128), 128, 0, s>>>(
          h->eQ[sp], h->uoff[sp], h->unex[sp], h->uexc[sp], h->uinv[sp], h->nuniq[sp], nb, na, N,
          h->ninv[sp], h->INV, mixed ? reinterpret_cast<float2*>(h->INV32) : nullptr,
          h->uhdrs[sp]);
      AFQMC_TRY(launch_status("woodbury_inverses_kernel"));
      const size_t sm1 = size_t(N) * h->nv[sp] * sizeof(c128);
      AFQMC_CUDA_TRY(cudaFuncSetAttribute(excited_1body_all_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm1)));
      excited_1body_all_kernel<<<dim3(nb, 4), PH_THREADS, sm1, s>>>(
          h->Swia, h->eQ[sp], h->refc[sp], h->vl[sp], h->nv[sp], h->uhdr[sp], h->uexc4[sp],
          h->INV, h->ninv[sp], h->wgt, h->nuniq[sp], nb, N, na, h->el);
      AFQMC_TRY(launch_status("excited_1body_all_kernel"));
    }
    c128* REF = h->el + 3 * nb;  // [nb][2]: sum_n ex0, sum_n f0^2
    {
      const long nt = long(h->nuniq[sp]) * nb;
      transpose_uw_kernel<<<unsigned((nt + 255) / 256), 256, 0, s>>>(h->wgt, h->nuniq[sp], nb,
                                                                     h->wgtT);
      AFQMC_TRY(launch_status("transpose_uw_kernel"));
    }
    // four Cholesky indices per CTA where their tables fit (each determinant's Q, indices and
    // weight are then read once per four indices), the next index's rows loaded while the
    // current tables are built where a second row buffer fits
    const size_t esz = mixed ? sizeof(c64) : sizeof(c128);
    const size_t lim = size_t(mixed ? 110 : 200) * 1024;
    int ngr = 4, nbuf = 2;
    if (excited_tables_smem(h, sp, esz, 4, 2) > lim) nbuf = 1;
    if (excited_tables_smem(h, sp, esz, 4, nbuf) > lim) ngr = nbuf = 1;
    const size_t smem = excited_tables_smem(h, sp, esz, ngr, nbuf);
    const dim3 grid((Nc + ngr - 1) / ngr, nb);
    // the K vectors have Twina's element type (complex64 in the mixed energy's tables path)
    auto go = [&](auto kern, const auto* tw, const auto* inv) -> int {
      using KT = std::remove_const_t<std::remove_pointer_t<decltype(tw)>>;
      AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(smem)));
      kern<<<grid, PHX_THREADS, smem, s>>>(
          tw, h->eQ[sp], h->refc[sp], h->hl[sp], h->vl[sp], h->nh[sp], h->nv[sp],
          mixed ? h->uhdrs[sp] : h->uhdr[sp], mixed ? h->uexc4s[sp] : h->uexc4[sp], inv,
          h->ninv[sp], h->wgtT, h->nuniq[sp], nb, N, na, Nc, nbuf, h->el + nb,
          h->el + 2 * nb, cross ? nullptr : reinterpret_cast<KT*>(KEout),
          reinterpret_cast<const KT*>(cross), E, reinterpret_cast<KT*>(Kref), REF);
      return AFQMC_OK;
    };
    const c64* inv32 = reinterpret_cast<const c64*>(h->INV32);
    const c64* tw64 = reinterpret_cast<const c64*>(h->Twina);
    if (mixed && h->twina64[sp])
      AFQMC_TRY(ngr == 4 ? go(excited_energy_tables_kernel<float, 4, c64>, tw64, inv32)
                         : go(excited_energy_tables_kernel<float, 1, c64>, tw64, inv32));
    else if (mixed)
      AFQMC_TRY(ngr == 4 ? go(excited_energy_tables_kernel<float, 4, c128>, h->Twina, inv32)
                         : go(excited_energy_tables_kernel<float, 1, c128>, h->Twina, inv32));
    else
      AFQMC_TRY(ngr == 4 ? go(excited_energy_tables_kernel<double, 4, c128>, h->Twina, h->INV)
                         : go(excited_energy_tables_kernel<double, 1, c128>, h->Twina, h->INV));
    AFQMC_TRY(launch_status("excited_energy_tables_kernel"));
    reference_from_tables_kernel<<<(nb + 127) / 128, 128, 0, s>>>(h->Swia, h->refc[sp], N, na, E0,
                                                                  h->eOv, REF, nb, E);
    AFQMC_TRY(launch_status("reference_from_tables_kernel"));
  }
  add_components_kernel<<<(nb + 127) / 128, 128, 0, s>>>(h->el, h->el + nb, h->el + 2 * nb, nb,
                                                          E);
  return launch_status("add_components_kernel");
}

}  // namespace

extern "C" int afqmc_phmsd_energy(afqmc_phmsd h, const afqmc_c128* wbuf, long ldS,
                                  afqmc_c128* E_out, afqmc_c128* ovlp, int W, int block,
                                  afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && wbuf && E_out && ovlp, "afqmc_phmsd_energy: null argument");
  AFQMC_CHECK_ARG(h->has_ham, "afqmc_phmsd_energy: no Hamiltonian (afqmc_phmsd_set_hamiltonian)");
  AFQMC_CHECK_ARG(W >= 0 && ldS >= long(h->M) * (h->nel[0] + h->nel[1]),
                  "afqmc_phmsd_energy: W=%d, walker stride %ld < M (nup + ndn)", W, ldS);
  if (W == 0) return AFQMC_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int Wb = block > 0 ? (block < W ? block : W) : (W < 64 ? W : 64);
  int st = phmsd_energy_scratch(h, Wb);
  if (st) {
    cudaSetDevice(prev);
    return st;
  }
  const int Nc = h->Nc;
  const c128* S = reinterpret_cast<const c128*>(wbuf);
  c128* Eall = reinterpret_cast<c128*>(E_out);
  c128* Oall = reinterpret_cast<c128*>(ovlp);
  auto run = [&]() -> int {
    // complex64 half-rotated rows and K vectors when both spins run the mixed tables kernels
    h->ke64 = false;
    if (h->precision == AFQMC_PREC_MIXED && phmsd_tables(h, 0) && phmsd_tables(h, 1)) {
      AFQMC_TRY(phmsd_tc_prepare(h, s, 0));
      AFQMC_TRY(phmsd_tc_prepare(h, s, 1));
      h->ke64 = h->tc_lnak_state[0] == 1 && h->tc_lnak_state[1] == 1;
    }
    for (int w0 = 0; w0 < W; w0 += Wb) {
      const int nb = (W - w0 < Wb) ? W - w0 : Wb;
      const c128* Sb = S + long(w0) * ldS;
      c128* E = Eall + size_t(w0) * 3;
      AFQMC_CUDA_TRY(cudaMemsetAsync(E, 0, sizeof(c128) * 3 * nb, s));
      AFQMC_CUDA_TRY(cudaMemsetAsync(h->elogov, 0, sizeof(c128) * nb, s));
      AFQMC_TRY(phmsd_spin_factors(h, s, 0, Sb, ldS, nb));
      AFQMC_TRY(phmsd_spin_factors(h, s, 1, Sb + long(h->M) * h->nel[0], ldS, nb));
      const int nu0 = h->nuniq[0], nu1 = h->nuniq[1];
      auto couple = [&](int sp, const c128* v_other, int nu_other, const c128* ov_self) -> int {
        const long nt = long(h->nuniq[sp]) * nb;
        couple_kernel<<<unsigned((nt + 3) / 4), 128, 0, s>>>(
            h->rowptr[sp], h->kidx[sp], h->det[1 - sp], h->coef, v_other, nu_other, ov_self,
            h->nuniq[sp], nb, h->wgt);
        return launch_status("couple_kernel");
      };
      // spin up: weights, total overlap, reference and excited energies (PHMSD.cpp:438-470)
      AFQMC_TRY(couple(0, h->eov[1], nu1, nullptr));
      total_overlap_kernel<<<nb, PH_THREADS, 0, s>>>(h->wgt, h->eov[0], nu0, nb, h->eOv);
      AFQMC_TRY(launch_status("total_overlap_kernel"));
      AFQMC_TRY(couple(0, h->eov[1], nu1, h->eov[0]));
      AFQMC_TRY(phmsd_half_rotated(h, s, 0, nb));
      AFQMC_TRY(phmsd_reference_and_excited(h, s, 0, nb, h->E0, h->KEr, h->KEr, nullptr, E));
      // K vectors coupled to the down-spin excitations (PHMSD.cpp:472-494)
      {
        if (h->nkrow > 0) {
          if (h->ke64)
            zero_k_rows_kernel<c64><<<dim3(h->nkrow, nb), 256, 0, s>>>(
                h->krow, nb, Nc, reinterpret_cast<c64*>(h->KEd));
          else
            zero_k_rows_kernel<c128><<<dim3(h->nkrow, nb), 256, 0, s>>>(h->krow, nb, Nc, h->KEd);
          AFQMC_TRY(launch_status("zero_k_rows_kernel"));
        }
        dim3 grid(h->nkseg, nb);
        if (h->ke64)
          couple_ke_kernel<c64><<<grid, 128, 0, s>>>(
              h->kseg, h->kidx[1], h->det[0], h->coef, reinterpret_cast<const c64*>(h->KEr),
              h->eov[0], nu0, h->eov[1], nu1, nb, Nc, reinterpret_cast<c64*>(h->KEd));
        else
          couple_ke_kernel<c128><<<grid, 128, 0, s>>>(h->kseg, h->kidx[1], h->det[0], h->coef,
                                                      h->KEr, h->eov[0], nu0, h->eov[1], nu1, nb,
                                                      Nc, h->KEd);
        AFQMC_TRY(launch_status("couple_ke_kernel"));
      }
      // spin down (PHMSD.cpp:497-531)
      AFQMC_TRY(couple(1, h->eov[0], nu0, h->eov[1]));
      AFQMC_TRY(phmsd_half_rotated(h, s, 1, nb));
      AFQMC_TRY(phmsd_reference_and_excited(h, s, 1, nb, 0.0, h->Kdn, nullptr, h->KEd, E));
      if (h->ke64)
        cross_ej_kernel<c64><<<nb, PH_THREADS, 0, s>>>(reinterpret_cast<const c64*>(h->KEd),
                                                       reinterpret_cast<const c64*>(h->Kdn), 1,
                                                       nb, Nc, E);
      else
        cross_ej_kernel<c128><<<nb, PH_THREADS, 0, s>>>(h->KEd, h->Kdn, 1, nb, Nc, E);
      AFQMC_TRY(launch_status("cross_ej_kernel"));
      finish_energy_kernel<<<(nb + 127) / 128, 128, 0, s>>>(h->eOv, h->elogov, nb, E,
                                                            Oall + w0);
      AFQMC_TRY(launch_status("finish_energy_kernel"));
    }
    return AFQMC_OK;
  };
  st = run();
  cudaSetDevice(prev);
  return st;
}

// ---------------------------------------------------------------------------------------------
// PHMSD mixed density matrix (PHMSD::MixedDensityMatrix, compact, PHMSD.cpp:684-795) and vbias
// ---------------------------------------------------------------------------------------------
extern "C" int afqmc_phmsd_density_matrix(afqmc_phmsd h, const afqmc_c128* wbuf, long ldS,
                                          afqmc_c128* G_out, afqmc_c128* ovlp, int W, int block,
                                          afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && wbuf && G_out && ovlp, "afqmc_phmsd_density_matrix: null argument");
  AFQMC_CHECK_ARG(W >= 0 && ldS >= long(h->M) * (h->nel[0] + h->nel[1]),
                  "afqmc_phmsd_density_matrix: W=%d, walker stride %ld < M (nup + ndn)", W, ldS);
  if (W == 0) return AFQMC_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  // the density matrix needs only the per-walker Woodbury buffers (~0.5 MB per walker at
  // nel = 30, nact = 70, 2000 excitations): blocks of up to 512 walkers
  const int Wb = block > 0 ? (block < W ? block : W) : (W < 512 ? W : 512);
  int st = phmsd_core_scratch(h, Wb);
  if (st) {
    cudaSetDevice(prev);
    return st;
  }
  const c128* S = reinterpret_cast<const c128*>(wbuf);
  c128* Gall = reinterpret_cast<c128*>(G_out);
  c128* Oall = reinterpret_cast<c128*>(ovlp);
  const long rowsG = long(h->nact[0]) + h->nact[1];
  auto run = [&]() -> int {
    for (int w0 = 0; w0 < W; w0 += Wb) {
      const int nb = (W - w0 < Wb) ? W - w0 : Wb;
      const c128* Sb = S + long(w0) * ldS;
      AFQMC_CUDA_TRY(cudaMemsetAsync(h->elogov, 0, sizeof(c128) * nb, s));
      AFQMC_TRY(phmsd_spin_factors(h, s, 0, Sb, ldS, nb));
      AFQMC_TRY(phmsd_spin_factors(h, s, 1, Sb + long(h->M) * h->nel[0], ldS, nb));
      for (int sp = 0; sp < 2; ++sp) {
        const int N = h->nel[sp], na = h->nact[sp], nu = h->nuniq[sp];
        const long nt = long(nu) * nb;
        // wgt[u][w] (PHMSD.cpp:717-724, 754-760)
        if (sp == 0) {
          couple_kernel<<<unsigned((nt + 3) / 4), 128, 0, s>>>(
              h->rowptr[0], h->kidx[0], h->det[1], h->coef, h->eov[1], h->nuniq[1], nullptr, nu,
              nb, h->wgt);
          AFQMC_TRY(launch_status("couple_kernel"));
          total_overlap_kernel<<<nb, PH_THREADS, 0, s>>>(h->wgt, h->eov[0], nu, nb, h->eOv);
          AFQMC_TRY(launch_status("total_overlap_kernel"));
        }
        couple_kernel<<<unsigned((nt + 3) / 4), 128, 0, s>>>(
            h->rowptr[sp], h->kidx[sp], h->det[1 - sp], h->coef, h->eov[1 - sp],
            h->nuniq[1 - sp], h->eov[sp], nu, nb, h->wgt);
        AFQMC_TRY(launch_status("couple_kernel"));
        // full R (calculate_R): the inverse of every excitation block, then all determinants'
        // rows accumulated per walker
        if (nu > 1) {
          const long ni = long(nu - 1) * nb;
          woodbury_inverses_kernel<<<unsigned((ni + 127) / 128), 128, 0, s>>>(
              h->eQ[sp], h->uoff[sp], h->unex[sp], h->uexc[sp], h->uinv[sp], nu, nb, na, N,
              h->ninv[sp], h->INV, nullptr, nullptr);
          AFQMC_TRY(launch_status("woodbury_inverses_kernel"));
        }
        const size_t rsm = 3 * size_t(N) * na * sizeof(c128);
        AFQMC_CHECK_ARG(rsm <= 200 * 1024,
                        "afqmc_phmsd_density_matrix: nel x nact = %d x %d exceeds shared memory",
                        N, na);
        AFQMC_CUDA_TRY(cudaFuncSetAttribute(phmsd_R_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, int(rsm)));
        phmsd_R_kernel<<<nb, PHR_THREADS, rsm, s>>>(h->eQ[sp], h->refc[sp], h->uoff[sp],
                                                    h->unex[sp], h->uexc[sp], h->uinv[sp], h->INV,
                                                    h->ninv[sp], h->wgt, nu, nb, N, na, h->Rfull);
        AFQMC_TRY(launch_status("phmsd_R_kernel"));
        // G_s = R^T G_ref  (rows of this spin's active orbitals)
        GemmParams p{};
        p.m = na; p.n = h->M; p.k = N;
        p.A = h->Rfull; p.lda = na; p.strideA = long(N) * na;
        p.B = h->eG[sp]; p.ldb = h->M; p.strideB = long(N) * h->M;
        p.C = Gall + long(w0) * rowsG * h->M + (sp == 0 ? 0 : long(h->nact[0]) * h->M);
        p.ldc = h->M; p.strideC = rowsG * h->M;
        p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
        AFQMC_TRY(zgemm(s, nb, GT, false, GN, false, p));
      }
      const long per = rowsG * h->M;
      scale_by_overlap_kernel<<<unsigned((per * nb + 255) / 256), 256, 0, s>>>(
          Gall + long(w0) * per, per, per, h->eOv, nb);
      AFQMC_TRY(launch_status("scale_by_overlap_kernel"));
      phmsd_combine_log_kernel<<<(nb + 127) / 128, 128, 0, s>>>(h->eOv, h->elogov, nb,
                                                                Oall + w0);
      AFQMC_TRY(launch_status("phmsd_combine_log_kernel"));
    }
    return AFQMC_OK;
  };
  st = run();
  cudaSetDevice(prev);
  return st;
}

extern "C" int afqmc_phmsd_vbias(afqmc_phmsd h, const afqmc_c128* G, afqmc_c128* v, int W,
                                 double dt, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && G && v, "afqmc_phmsd_vbias: null argument");
  AFQMC_CHECK_ARG(h->has_ham, "afqmc_phmsd_vbias: no Hamiltonian (afqmc_phmsd_set_hamiltonian)");
  if (W <= 0) return AFQMC_OK;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long rowsG = long(h->nact[0]) + h->nact[1];
  int st = AFQMC_OK;
  // v[w][n] = sqrt(dt) sum_s sum_{a,k} G_s[w][a][k] Lnak_s[n][a][k]  (Real3Index vbias, COLLINEAR)
  for (int sp = 0; sp < 2 && !st; ++sp) {
    GemmParams p{};
    p.m = W; p.n = h->Nc; p.k = h->nact[sp] * h->M;
    p.A = reinterpret_cast<const c128*>(G) + (sp == 0 ? 0 : long(h->nact[0]) * h->M);
    p.lda = rowsG * h->M;
    p.B = h->lnak[sp]; p.ldb = long(h->nact[sp]) * h->M;
    p.C = reinterpret_cast<c128*>(v); p.ldc = h->Nc;
    p.alpha = cmk(std::sqrt(dt), 0); p.beta = cmk(sp == 0 ? 0.0 : 1.0, 0);
    st = zgemm(s, 1, GN, false, GT, false, p);
  }
  cudaSetDevice(prev);
  return st;
}

// ---------------------------------------------------------------------------------------------
// Particle-hole structure of a determinant expansion given as occupation lists (what the
// PHMSD factory builds into ph_excitations from the wavefunction file, Wavefunction.cpp:349-495,
// Excitations.hpp:207-554): host logic.
// ---------------------------------------------------------------------------------------------
namespace {
// parity of the permutation that sorts v (number of inversions mod 2)
int parity(const std::vector<int>& v) {
  int inv = 0;
  for (size_t i = 0; i < v.size(); ++i)
    for (size_t j = i + 1; j < v.size(); ++j) inv += v[i] > v[j];
  return inv & 1;
}
}  // namespace

extern "C" int afqmc_phmsd_excitations(int nact, int nel, const int* refc, int ndet,
                                       const int* occ, int* det_index, double* sign, int* nuniq,
                                       int* nex, int* exc) {
  AFQMC_CHECK_ARG(nact > 0 && nel >= 0 && nel <= nact && ndet >= 0 && refc && nuniq && nex &&
                      (ndet == 0 || (occ && det_index && sign && exc)),
                  "afqmc_phmsd_excitations: bad argument");
  std::vector<int> where(nact, -1);  // electron of each reference orbital
  for (int i = 0; i < nel; ++i) {
    AFQMC_CHECK_ARG(refc[i] >= 0 && refc[i] < nact && where[refc[i]] < 0,
                    "afqmc_phmsd_excitations: reference orbital %d of electron %d invalid or "
                    "repeated", refc[i], i);
    where[refc[i]] = i;
  }
  std::vector<int> ref(refc, refc + nel);
  // unique excitations per excitation number, in order of first appearance
  std::vector<std::map<std::vector<int>, int>> seen;
  std::vector<std::vector<std::vector<int>>> lists;
  std::vector<std::pair<int, int>> key(ndet);  // (n, position in lists[n])
  std::vector<char> mark(nact);
  for (int k = 0; k < ndet; ++k) {
    const int* o = occ + size_t(k) * nel;
    std::fill(mark.begin(), mark.end(), 0);
    for (int i = 0; i < nel; ++i) {
      AFQMC_CHECK_ARG(o[i] >= 0 && o[i] < nact && !mark[o[i]],
                      "afqmc_phmsd_excitations: determinant %d: orbital %d invalid or repeated",
                      k, o[i]);
      mark[o[i]] = 1;
    }
    std::vector<int> holes, parts;
    for (int i = 0; i < nel; ++i)
      if (!mark[refc[i]]) holes.push_back(i);
    for (int x = 0; x < nact; ++x)
      if (mark[x] && where[x] < 0) parts.push_back(x);
    const int n = int(holes.size());
    AFQMC_CHECK_ARG(n <= PH_NEX_MAX, "afqmc_phmsd_excitations: determinant %d is a %d-fold "
                                      "excitation (at most %d)", k, n, PH_NEX_MAX);
    // the Woodbury determinant: reference columns with hole h_e replaced by particle p_e (both
    // ascending); its sign relative to the determinant in the given column order
    std::vector<int> L = ref;
    for (int e = 0; e < n; ++e) L[holes[e]] = parts[e];
    std::vector<int> given(o, o + nel);
    sign[k] = ((parity(L) + parity(given)) & 1) ? -1.0 : 1.0;
    if (int(seen.size()) <= n) {
      seen.resize(n + 1);
      lists.resize(n + 1);
    }
    std::vector<int> e = holes;
    e.insert(e.end(), parts.begin(), parts.end());
    auto it = seen[n].find(e);
    if (it == seen[n].end()) {
      it = seen[n].emplace(e, int(lists[n].size())).first;
      lists[n].push_back(e);
    }
    key[k] = {n, it->second};
  }
  // unique index: 0 the reference, then by excitation number
  std::vector<int> first(lists.size() + 1, 1);
  int u = 1, pos = 0;
  for (size_t n = 1; n < lists.size(); ++n) {
    first[n] = u;
    for (const auto& e : lists[n]) {
      nex[u - 1] = int(n);
      std::copy(e.begin(), e.end(), exc + pos);
      pos += int(e.size());
      ++u;
    }
  }
  *nuniq = u;
  for (int k = 0; k < ndet; ++k)
    det_index[k] = key[k].first == 0 ? 0 : first[key[k].first] + key[k].second;
  return AFQMC_OK;
}

