// Local energy of the Real3Index factorisation: one-body E1, exchange EXX and Coulomb EJ.
//
// Reference: Real3IndexFactorization::energy / energy_impl
// (src/AFQMC/HamiltonianOperations/Real3IndexFactorization.hpp:138-174, 476-590):
//   E1[w]  = E0 + scl sum_{a,j} G[w,a,j] haj[a,j]
//   T[w,b,n,a] = sum_k G[w,b,k] Lnak[n,a,k]
//   EXX[w] = -scl/2 sum_{a,b,n} T[w,a,n,b] T[w,b,n,a]
//   Kl[w,n] = sum_a T[w,a,n,a];   EJ[w] = sclj/2 sum_n Kl[w,n]^2
// with scl = 2 (CLOSED) or 1, sclj = 4 (CLOSED) or 1.  The reference materialises T in chunks of
// Cholesky vectors sized by max_memory_MB; the complex128 path here materialises it in chunks of
// walkers (one DMMA GEMM per chunk) and reduces each N x N block of T with one CTA.
#include "energy.cuh"
#include "mixed.cuh"
#include "zgemm.cuh"

namespace afqmc {
namespace {

// One CTA per (walker, Cholesky vector): trace(T_n T_n) and trace(T_n) of the N x N block.
__global__ void __launch_bounds__(128)
    exchange_block_kernel(const c128* __restrict__ T, int N, int Nc, int w_first,
                          c128* __restrict__ exx_part, c128* __restrict__ Kl) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int pitch = N | 1;
  c128* t = reinterpret_cast<c128*>(smem_raw);
  const int n = blockIdx.x, wl = blockIdx.y;
  const long row_stride = long(Nc) * N;
  const c128* Tb = T + long(wl) * N * row_stride + long(n) * N;
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    int b = e / N, a = e % N;
    t[b * pitch + a] = Tb[long(b) * row_stride + a];
  }
  __syncthreads();
  c128 acc = cmk(0, 0), tr = cmk(0, 0);
  for (int e = threadIdx.x; e < N * N; e += blockDim.x) {
    int b = e / N, a = e % N;
    acc = cadd(acc, cmul(t[b * pitch + a], t[a * pitch + b]));
    if (a == b) tr = cadd(tr, t[b * pitch + a]);
  }
  __shared__ double red[4][4];
  double v[4] = {acc.x, acc.y, tr.x, tr.y};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q)
      for (int k = 0; k < (int)blockDim.x / 32; ++k) s[q] += red[q][k];
    const long w = w_first + wl;
    exx_part[w * Nc + n] = cadd(exx_part[w * Nc + n], cmk(s[0], s[1]));
    Kl[w * Nc + n] = cadd(Kl[w * Nc + n], cmk(s[2], s[3]));
  }
}

// One CTA per walker: E1 (per spin block accumulate), final EXX / EJ assembly.
__global__ void __launch_bounds__(256)
    e1_kernel(const c128* __restrict__ G, long ldG, const c128* __restrict__ haj, int NM,
              double scl, c128* __restrict__ E) {
  const long w = blockIdx.x;
  const c128* Gw = G + w * ldG;
  c128 acc = cmk(0, 0);
  for (int e = threadIdx.x; e < NM; e += blockDim.x) acc = cadd(acc, cmul(Gw[e], haj[e]));
  __shared__ double red[2][8];
  double v[2] = {acc.x, acc.y};
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[2] = {0, 0};
    for (int q = 0; q < 2; ++q)
      for (int k = 0; k < (int)blockDim.x / 32; ++k) s[q] += red[q][k];
    E[w * 3 + 0] = cadd(E[w * 3 + 0], cscale(cmk(s[0], s[1]), scl));
  }
}

__global__ void __launch_bounds__(256)
    finish_kernel(const c128* __restrict__ exx_part, const c128* __restrict__ Kl, int Nc,
                  double scl_x, double scl_j, int addEXX, int addEJ, c128* __restrict__ E) {
  const long w = blockIdx.x;
  c128 ex = cmk(0, 0), ej = cmk(0, 0);
  for (int n = threadIdx.x; n < Nc; n += blockDim.x) {
    if (addEXX) ex = cadd(ex, exx_part[w * Nc + n]);
    if (addEJ) {
      c128 k = Kl[w * Nc + n];
      ej = cadd(ej, cmul(k, k));
    }
  }
  __shared__ double red[4][8];
  double v[4] = {ex.x, ex.y, ej.x, ej.y};
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[4] = {0, 0, 0, 0};
    for (int q = 0; q < 4; ++q)
      for (int k = 0; k < (int)blockDim.x / 32; ++k) s[q] += red[q][k];
    if (addEXX) E[w * 3 + 1] = cadd(E[w * 3 + 1], cscale(cmk(s[0], s[1]), scl_x));
    if (addEJ) E[w * 3 + 2] = cadd(E[w * 3 + 2], cscale(cmk(s[2], s[3]), scl_j));
  }
}

__global__ void init_energy_kernel(c128* E, int W, double E0, int addH1) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < W) {
    E[i * 3 + 0] = cmk(addH1 ? E0 : 0.0, 0.0);
    E[i * 3 + 1] = cmk(0, 0);
    E[i * 3 + 2] = cmk(0, 0);
  }
}

}  // namespace

int energy_fp64(cudaStream_t s, const EnergyArgs& a, c128* E, int W, bool addH1, bool addEJ,
                bool addEXX, c128* workT, long workT_elems, c128* exx_part, c128* Kl,
                MixedHam* tc) {
  if (W <= 0) return AFQMC_OK;
  init_energy_kernel<<<ceil_div(W, 128), 128, 0, s>>>(E, W, a.E0, addH1 ? 1 : 0);
  AFQMC_TRY(launch_status("init_energy_kernel"));
  const bool need_T = addEXX || addEJ;
  if (need_T) {
    AFQMC_CUDA_TRY(cudaMemsetAsync(exx_part, 0, sizeof(c128) * size_t(W) * a.Nc, s));
    AFQMC_CUDA_TRY(cudaMemsetAsync(Kl, 0, sizeof(c128) * size_t(W) * a.Nc, s));
  }
  for (int sp = 0; sp < a.nspin; ++sp) {
    const int Ns = a.nel[sp];
    if (Ns == 0) continue;
    const c128* Gs = a.G + long(a.el_off[sp]) * a.M;  // spin block inside each walker's row
    if (addH1) {
      e1_kernel<<<W, 256, 0, s>>>(Gs, a.ldG, a.haj + long(a.el_off[sp]) * a.M, Ns * a.M, a.scl, E);
      AFQMC_TRY(launch_status("e1_kernel"));
    }
    if (!need_T) continue;
    if (tc && exchange_fused_ok(tc, sp)) {
      AFQMC_TRY(exchange_fused(s, tc, sp, W, exx_part, Kl));
      continue;
    }
    // chunk of walkers whose T [Wc*Ns][Nc*Ns] fits the workspace
    const long per_walker = long(Ns) * a.Nc * Ns;
    int Wc = int(workT_elems / per_walker);
    if (Wc < 1) {
      set_error_detail("energy: workspace too small for one walker's exchange tensor");
      return AFQMC_ERR_ALLOC;
    }
    Wc = Wc > W ? W : Wc;
    const int pitch = Ns | 1;
    const size_t smem = size_t(Ns) * pitch * sizeof(c128);
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(exchange_block_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    for (int w0 = 0; w0 < W; w0 += Wc) {
      const int wc = (W - w0) < Wc ? (W - w0) : Wc;
      // T[(w,b)][(n,a)] = sum_k G[w,b,k] Lnak[n,a,k]; rows of G are strided by ldG per walker,
      // so one GEMM per walker in the chunk (batched, shared Lnak)
      if (tc) {
        AFQMC_TRY(exchange_T_tc(s, tc, sp, w0, wc, workT));
        exchange_block_kernel<<<dim3(a.Nc, wc), 128, smem, s>>>(workT, Ns, a.Nc, w0, exx_part, Kl);
        AFQMC_TRY(launch_status("exchange_block_kernel"));
        continue;
      }
      GemmParams p{};
      p.m = Ns; p.n = a.Nc * Ns; p.k = a.M;
      p.A = Gs + long(w0) * a.ldG; p.lda = a.M; p.strideA = a.ldG;
      p.B = a.Lnak_real[sp] ? (const void*)a.Lnak_real[sp] : (const void*)a.Lnak[sp];
      p.ldb = a.M; p.strideB = 0;
      p.C = workT; p.ldc = long(a.Nc) * Ns; p.strideC = per_walker;
      p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
      AFQMC_TRY(zgemm(s, wc, GN, false, GT, a.Lnak_real[sp] != nullptr, p));
      exchange_block_kernel<<<dim3(a.Nc, wc), 128, smem, s>>>(workT, Ns, a.Nc, w0, exx_part, Kl);
      AFQMC_TRY(launch_status("exchange_block_kernel"));
    }
  }
  if (tc && addEJ && a.coulomb_fp64) {
    // Kl[w][n] = sum_s sum_{a,k} G[w][a][k] Lnak_s[n][a][k] in complex128 (DMMA), in place of the
    // traces of the TF32-split exchange tiles
    bool first = true;
    for (int sp = 0; sp < a.nspin; ++sp) {
      const int Ns = a.nel[sp];
      if (Ns == 0) continue;
      GemmParams p{};
      p.m = W; p.n = a.Nc; p.k = Ns * a.M;
      p.A = a.G + long(a.el_off[sp]) * a.M; p.lda = a.ldG; p.strideA = 0;
      p.B = a.Lnak_real[sp] ? (const void*)a.Lnak_real[sp] : (const void*)a.Lnak[sp];
      p.ldb = long(Ns) * a.M; p.strideB = 0;
      p.C = Kl; p.ldc = a.Nc; p.strideC = 0;
      p.alpha = cmk(1, 0); p.beta = first ? cmk(0, 0) : cmk(1, 0);
      AFQMC_TRY(zgemm(s, 1, GN, false, GT, a.Lnak_real[sp] != nullptr, p));
      first = false;
    }
  }
  if (need_T) {
    finish_kernel<<<W, 256, 0, s>>>(exx_part, Kl, a.Nc, -0.5 * a.scl, 0.5 * a.sclj, addEXX ? 1 : 0,
                                    addEJ ? 1 : 0, E);
    AFQMC_TRY(launch_status("finish_kernel"));
  }
  return AFQMC_OK;
}

}  // namespace afqmc
