// Tensor-hypercontraction (THC) Hamiltonian operations, complex128 on the FP64 tensor path.
//
// Reference: THCOps (src/AFQMC/HamiltonianOperations/THCOps.hpp), the second implementation of
// the HamiltonianOperations interface next to Real3IndexFactorization.  The two-electron
// integrals are factorised over nu interpolation points u:
//   L_n[i][k] = sum_u X[i][u] X[k][u] Luv[u][n]      (n < nv, the "Cholesky" index)
//   sum_n L_n[i][l] L_n[k][j] = sum_{u,v} X[i][u] X[l][u] Z[u][v] X[k][v] X[j][v],  Z = Luv Luv^T
// with X = Piu [M][nu] (real) and the trial-rotated points Y[a][u] = sum_i PsiT[a][i] X[i][u]
// (rotcXau; PsiT the conjugate-transposed trial, the half rotation of the library's compact G:
// G_full[i][k] = sum_a PsiT[a][i] G[a][k]).  Per walker w:
//   Guu[u]      = a sum_s sum_a (G_s X)[a][u] Y_s[a][u]                     (Guu_from_compact,
//                                                                            THCOps.hpp:636-703)
//   vbias[n]    = sqrt(dt) sum_u Luv[u][n] Guu[u]                           (vbias, :571-615)
//   vHS[i][k]   = sqrt(dt) sum_u X[i][u] X[k][u] sum_n Luv[u][n] x[n]       (vHS, :462-569)
//   Guv_s[u][v] = sum_a Y_s[a][u] (G_s X)[a][v]                             (Guv_Guu, :755-835)
//   EXX         = -scl/2 sum_s sum_{u,v} Z[u][v] Guv_s[u][v] Guv_s[v][u]     (energy, :149-293)
//   EJ          = scl^2/2 sum_{u,v} g[u] Z[u][v] g[v],  g[u] = sum_s Guv_s[u][u]
//   E1          = E0 + scl sum_{a,k} G[a][k] haj[a][k]
// a = scl = 2 for CLOSED walkers, else 1.  The reference reaches EXX through two more GEMMs
// ((Guv o Z) Y^T, then X times that, contracted with G); the sum above is the same quantity,
// formed directly from Guv (nu^2 per walker instead of 2 nu^2 nel + nu nel M).
// vHS runs as one GEMM over all walkers against the precomputed products XX[(i,k)][u] =
// X[i][u] X[k][u]; the walker's fields enter through T[w][u] = sum_n Luv[u][n] x[w][n].
#include <cmath>
#include <memory>
#include <new>
#include <vector>

#include "common.cuh"
#include "thc.cuh"
#include "zgemm.cuh"

namespace afqmc {

namespace {

constexpr int THC_THREADS = 256;

// Guu[w][u] (+)= a sum_a T1[w][a][u] Y[a][u]
__global__ void thc_guu_kernel(const c128* __restrict__ T1, const c128* __restrict__ Y, int nel,
                               int nu, int W, double a, int accumulate, c128* __restrict__ Guu) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= long(W) * nu) return;
  const int w = int(e / nu), u = int(e - long(w) * nu);
  const c128* t = T1 + size_t(w) * nel * nu + u;
  c128 s = cmk(0, 0);
  for (int k = 0; k < nel; ++k) s = cadd(s, cmul(t[size_t(k) * nu], Y[size_t(k) * nu + u]));
  s = cmk(a * s.x, a * s.y);
  Guu[e] = accumulate ? cadd(Guu[e], s) : s;
}

__device__ __forceinline__ c128 block_sum(c128 v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) {
    red[2 * warp] = v.x;
    red[2 * warp + 1] = v.y;
  }
  __syncthreads();
  c128 s = cmk(0, 0);
  if (threadIdx.x == 0)
    for (int k = 0; k < int(blockDim.x >> 5); ++k) s = cadd(s, cmk(red[2 * k], red[2 * k + 1]));
  return s;  // thread 0
}

// one CTA per walker w of the block: EXX[w] += -scl/2 sum_{u,v} Z[u][v] Guv[u][v] Guv[v][u] and
// g[w][u] (+)= Guv[u][u]
__global__ void __launch_bounds__(THC_THREADS) thc_exx_kernel(const c128* __restrict__ Guv,
                                                              const double* __restrict__ Z,
                                                              int nu, double scl,
                                                              int accumulate_g,
                                                              c128* __restrict__ g,
                                                              c128* __restrict__ E) {
  __shared__ double red[2 * THC_THREADS / 32];
  const int w = blockIdx.x;
  const c128* Gw = Guv + size_t(w) * nu * nu;
  c128 s = cmk(0, 0);
  for (long e = threadIdx.x; e < long(nu) * nu; e += blockDim.x) {
    const int u = int(e / nu), v = int(e - long(u) * nu);
    const double z = Z[e];
    if (z != 0.0) s = cadd(s, cmul(cmk(z, 0), cmul(Gw[e], Gw[size_t(v) * nu + u])));
  }
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    const c128 d = Gw[size_t(u) * nu + u];
    c128* gu = g + size_t(w) * nu + u;
    *gu = accumulate_g ? cadd(*gu, d) : d;
  }
  const c128 t = block_sum(s, red);
  if (threadIdx.x == 0) E[size_t(w) * 3 + 1] = cadd(E[size_t(w) * 3 + 1], cmk(-0.5 * scl * t.x, -0.5 * scl * t.y));
}

// one CTA per walker: EJ[w] = scl^2/2 sum_{u,v} g[u] Z[u][v] g[v]
__global__ void __launch_bounds__(THC_THREADS) thc_ej_kernel(const c128* __restrict__ g,
                                                             const double* __restrict__ Z, int nu,
                                                             double sclj, c128* __restrict__ E) {
  __shared__ double red[2 * THC_THREADS / 32];
  const int w = blockIdx.x;
  const c128* gw = g + size_t(w) * nu;
  c128 s = cmk(0, 0);
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    c128 zg = cmk(0, 0);
    for (int v = 0; v < nu; ++v) {
      const double z = Z[size_t(u) * nu + v];
      zg = cmk(zg.x + z * gw[v].x, zg.y + z * gw[v].y);
    }
    s = cadd(s, cmul(gw[u], zg));
  }
  const c128 t = block_sum(s, red);
  if (threadIdx.x == 0) E[size_t(w) * 3 + 2] = cadd(E[size_t(w) * 3 + 2], cmk(0.5 * sclj * t.x, 0.5 * sclj * t.y));
}

// E[w][0] = E0 + scl sum_{a,k} G[w][a][k] haj[a][k]
__global__ void __launch_bounds__(THC_THREADS) thc_e1_kernel(const c128* __restrict__ G, long ldG,
                                                             const c128* __restrict__ haj, long n,
                                                             double E0, double scl,
                                                             c128* __restrict__ E) {
  __shared__ double red[2 * THC_THREADS / 32];
  const int w = blockIdx.x;
  const c128* Gw = G + size_t(w) * ldG;
  c128 s = cmk(0, 0);
  for (long e = threadIdx.x; e < n; e += blockDim.x) s = cadd(s, cmul(Gw[e], haj[e]));
  const c128 t = block_sum(s, red);
  if (threadIdx.x == 0) E[size_t(w) * 3] = cmk(E0 + scl * t.x, scl * t.y);
}

// XX[(i,k)][u] = X[i][u] X[k][u]
__global__ void thc_xx_kernel(const double* __restrict__ X, int M, int nu, double* __restrict__ XX) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= long(M) * M * nu) return;
  const int u = int(e % nu);
  const long ik = e / nu;
  const int i = int(ik / M), k = int(ik - long(i) * M);
  XX[e] = X[size_t(i) * nu + u] * X[size_t(k) * nu + u];
}

int thc_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return AFQMC_OK;
  set_error_detail("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? AFQMC_ERR_ALLOC : AFQMC_ERR_CUDA;
}

}  // namespace

struct ThcData {
  int M = 0, nu = 0, nv = 0, nspin = 1, nel[2] = {0, 0}, el_off[2] = {0, 0};
  double* X = nullptr;   // [M][nu]
  double* XX = nullptr;  // [M*M][nu]
  double* L = nullptr;   // [nu][nv]
  double* Z = nullptr;   // [nu][nu]
  c128* Y = nullptr;     // [nel_tot][nu]
  // workspace
  long cap_w = 0;
  c128 *T1 = nullptr, *Guu = nullptr, *Tw = nullptr, *Guv = nullptr, *g = nullptr;
  long cap_guv = 0;
  ~ThcData() {
    for (void* p : {(void*)X, (void*)XX, (void*)L, (void*)Z, (void*)Y, (void*)T1, (void*)Guu,
                    (void*)Tw, (void*)Guv, (void*)g})
      if (p) cudaFree(p);
  }
};

namespace {
int ensure(ThcData* t, int W) {
  if (t->cap_w >= W) return AFQMC_OK;
  AFQMC_TRY(thc_cuda(cudaDeviceSynchronize(), "thc workspace"));
  for (c128** p : {&t->T1, &t->Guu, &t->Tw, &t->g})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  const int nmax = t->nel[0] > t->nel[1] ? t->nel[0] : t->nel[1];
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->T1, sizeof(c128) * size_t(W) * nmax * t->nu), "thc T1"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->Guu, sizeof(c128) * size_t(W) * t->nu), "thc Guu"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->Tw, sizeof(c128) * size_t(W) * t->nu), "thc T"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->g, sizeof(c128) * size_t(W) * t->nu), "thc g"));
  t->cap_w = W;
  return AFQMC_OK;
}

// T1[w][a][u] = sum_k G_s[w][a][k] X[k][u] for spin block s of walkers [0, W)
int thc_t1(cudaStream_t s, ThcData* t, const c128* G, long ldG, int sp, int W) {
  GemmParams p{};
  p.m = t->nel[sp]; p.n = t->nu; p.k = t->M;
  p.A = G + long(t->el_off[sp]) * t->M; p.lda = t->M; p.strideA = ldG;
  p.B = t->X; p.ldb = t->nu; p.strideB = 0;
  p.C = t->T1; p.ldc = t->nu; p.strideC = long(t->nel[sp]) * t->nu;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  return zgemm(s, W, GN, false, GN, true, p);
}
}  // namespace

int thc_create(ThcData** out, int walker_type, int M, int nup, int ndn, int nu, int nv,
               const double* X, const double* L, const double* Z, const c128* PsiT_dev) {
  *out = nullptr;
  std::unique_ptr<ThcData> t(new (std::nothrow) ThcData());
  if (!t) return AFQMC_ERR_ALLOC;
  t->M = M; t->nu = nu; t->nv = nv;
  t->nspin = walker_type == AFQMC_COLLINEAR ? 2 : 1;
  t->nel[0] = nup;
  t->nel[1] = walker_type == AFQMC_COLLINEAR ? ndn : 0;
  t->el_off[0] = 0;
  t->el_off[1] = nup;
  const int nel_tot = t->nel[0] + t->nel[1];
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->X, sizeof(double) * size_t(M) * nu), "thc X"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->XX, sizeof(double) * size_t(M) * M * nu), "thc XX"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->L, sizeof(double) * size_t(nu) * nv), "thc L"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->Z, sizeof(double) * size_t(nu) * nu), "thc Z"));
  AFQMC_TRY(thc_cuda(cudaMalloc(&t->Y, sizeof(c128) * size_t(nel_tot > 0 ? nel_tot : 1) * nu),
                     "thc Y"));
  cudaMemcpy(t->X, X, sizeof(double) * size_t(M) * nu, cudaMemcpyHostToDevice);
  cudaMemcpy(t->L, L, sizeof(double) * size_t(nu) * nv, cudaMemcpyHostToDevice);
  if (Z) {
    cudaMemcpy(t->Z, Z, sizeof(double) * size_t(nu) * nu, cudaMemcpyHostToDevice);
  } else {
    // Z = Luv Luv^T on the host (set-up)
    std::vector<double> z(size_t(nu) * nu, 0.0);
    for (int u = 0; u < nu; ++u)
      for (int v = 0; v <= u; ++v) {
        double acc = 0.0;
        for (int n = 0; n < nv; ++n) acc += L[size_t(u) * nv + n] * L[size_t(v) * nv + n];
        z[size_t(u) * nu + v] = z[size_t(v) * nu + u] = acc;
      }
    cudaMemcpy(t->Z, z.data(), sizeof(double) * z.size(), cudaMemcpyHostToDevice);
  }
  const long nxx = long(M) * M * nu;
  thc_xx_kernel<<<unsigned((nxx + 255) / 256), 256>>>(t->X, M, nu, t->XX);
  AFQMC_TRY(launch_status("thc_xx_kernel"));
  // Y[a][u] = sum_i PsiT[a][i] X[i][u]
  if (nel_tot > 0) {
    GemmParams p{};
    p.m = nel_tot; p.n = nu; p.k = M;
    p.A = PsiT_dev; p.lda = M; p.strideA = 0;
    p.B = t->X; p.ldb = nu; p.strideB = 0;
    p.C = t->Y; p.ldc = nu; p.strideC = 0;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(nullptr, 1, GN, false, GN, true, p));
  }
  AFQMC_TRY(thc_cuda(cudaDeviceSynchronize(), "thc_create"));
  *out = t.release();
  return AFQMC_OK;
}

void thc_destroy(ThcData* t) { delete t; }

int thc_vbias(cudaStream_t s, ThcData* t, const c128* G, long ldG, c128* v, int W, double dt,
              double a_occ) {
  if (W <= 0) return AFQMC_OK;
  AFQMC_TRY(ensure(t, W));
  bool first = true;
  for (int sp = 0; sp < t->nspin; ++sp) {
    if (t->nel[sp] == 0) continue;
    AFQMC_TRY(thc_t1(s, t, G, ldG, sp, W));
    const long n = long(W) * t->nu;
    thc_guu_kernel<<<unsigned((n + 255) / 256), 256, 0, s>>>(
        t->T1, t->Y + size_t(t->el_off[sp]) * t->nu, t->nel[sp], t->nu, W, a_occ, first ? 0 : 1,
        t->Guu);
    AFQMC_TRY(launch_status("thc_guu_kernel"));
    first = false;
  }
  if (first) return thc_cuda(cudaMemsetAsync(v, 0, sizeof(c128) * size_t(W) * t->nv, s), "vbias");
  GemmParams p{};
  p.m = W; p.n = t->nv; p.k = t->nu;
  p.A = t->Guu; p.lda = t->nu; p.strideA = 0;
  p.B = t->L; p.ldb = t->nv; p.strideB = 0;
  p.C = v; p.ldc = t->nv; p.strideC = 0;
  p.alpha = cmk(std::sqrt(dt), 0); p.beta = cmk(0, 0);
  return zgemm(s, 1, GN, false, GN, true, p);
}

int thc_vhs(cudaStream_t s, ThcData* t, const c128* X, c128* V, int W, double dt) {
  if (W <= 0) return AFQMC_OK;
  AFQMC_TRY(ensure(t, W));
  // T[w][u] = sum_n x[w][n] Luv[u][n]
  GemmParams p{};
  p.m = W; p.n = t->nu; p.k = t->nv;
  p.A = X; p.lda = t->nv; p.strideA = 0;
  p.B = t->L; p.ldb = t->nv; p.strideB = 0;
  p.C = t->Tw; p.ldc = t->nu; p.strideC = 0;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, 1, GN, false, GT, true, p));
  // V[w][(i,k)] = sqrt(dt) sum_u T[w][u] XX[(i,k)][u]
  const long MM = long(t->M) * t->M;
  GemmParams q{};
  q.m = W; q.n = int(MM); q.k = t->nu;
  q.A = t->Tw; q.lda = t->nu; q.strideA = 0;
  q.B = t->XX; q.ldb = t->nu; q.strideB = 0;
  q.C = V; q.ldc = MM; q.strideC = 0;
  q.alpha = cmk(std::sqrt(dt), 0); q.beta = cmk(0, 0);
  return zgemm(s, 1, GN, false, GT, true, q);
}

int thc_energy(cudaStream_t s, ThcData* t, const c128* G, long ldG, const c128* haj, double E0,
               double scl, double sclj, c128* E, int W, bool addH1, bool addEJ, bool addEXX) {
  if (W <= 0) return AFQMC_OK;
  AFQMC_TRY(ensure(t, W));
  AFQMC_TRY(thc_cuda(cudaMemsetAsync(E, 0, sizeof(c128) * 3 * size_t(W), s), "energy"));
  const int nel_tot = t->nel[0] + t->nel[1];
  if (addH1) {
    thc_e1_kernel<<<W, THC_THREADS, 0, s>>>(G, ldG, haj, long(nel_tot) * t->M, E0, scl, E);
    AFQMC_TRY(launch_status("thc_e1_kernel"));
  }
  if (!(addEJ || addEXX)) return AFQMC_OK;
  // Guv blocks of at most 2^25 complex elements (512 MB)
  const long per = long(t->nu) * t->nu;
  long wb = (1l << 25) / (per > 0 ? per : 1);
  if (wb < 1) wb = 1;
  if (wb > W) wb = W;
  if (t->cap_guv < wb * per) {
    AFQMC_TRY(thc_cuda(cudaStreamSynchronize(s), "thc Guv"));
    if (t->Guv) cudaFree(t->Guv);
    t->Guv = nullptr;
    t->cap_guv = 0;
    AFQMC_TRY(thc_cuda(cudaMalloc(&t->Guv, sizeof(c128) * size_t(wb * per)), "thc Guv"));
    t->cap_guv = wb * per;
  }
  for (long w0 = 0; w0 < W; w0 += wb) {
    const int nb = int(W - w0 < wb ? W - w0 : wb);
    bool first = true;
    for (int sp = 0; sp < t->nspin; ++sp) {
      if (t->nel[sp] == 0) continue;
      AFQMC_TRY(thc_t1(s, t, G + w0 * ldG, ldG, sp, nb));
      // Guv_w = Y_s^T T1_w
      GemmParams p{};
      p.m = t->nu; p.n = t->nu; p.k = t->nel[sp];
      p.A = t->Y + size_t(t->el_off[sp]) * t->nu; p.lda = t->nu; p.strideA = 0;
      p.B = t->T1; p.ldb = t->nu; p.strideB = long(t->nel[sp]) * t->nu;
      p.C = t->Guv; p.ldc = t->nu; p.strideC = per;
      p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
      AFQMC_TRY(zgemm(s, nb, GT, false, GN, false, p));
      thc_exx_kernel<<<nb, THC_THREADS, 0, s>>>(t->Guv, t->Z, t->nu, addEXX ? scl : 0.0,
                                                first ? 0 : 1, t->g, E + w0 * 3);
      AFQMC_TRY(launch_status("thc_exx_kernel"));
      first = false;
    }
    if (addEJ && !first) {
      thc_ej_kernel<<<nb, THC_THREADS, 0, s>>>(t->g, t->Z, t->nu, sclj, E + w0 * 3);
      AFQMC_TRY(launch_status("thc_ej_kernel"));
    }
  }
  return AFQMC_OK;
}

int thc_sizes(const ThcData* t, int* nu, int* nv) {
  *nu = t->nu;
  *nv = t->nv;
  return AFQMC_OK;
}

}  // namespace afqmc
