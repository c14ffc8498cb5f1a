// Learned exchange-energy control variate: a small MLP (features -> H -> H -> 1, GELU) trained
// and evaluated by this library's own BF16 tensor-core kernels (tcgen05.mma kind::f16 with BF16
// operands and an FP32 accumulator in tensor memory, one 128 x 64 output tile per CTA), FP32
// master weights and Adam.
//
// It has no counterpart in the reference: the exact exchange energy (Real3IndexFactorization
// energy_impl, Real3IndexFactorization.hpp:476-590) stays the reference value.  The estimator that uses it
// evaluates the exact exchange on a random subset of walkers and the network on all of them, so
// its expectation over the subset is the exact weighted average whatever the network predicts.
//
// Layout: features X [B][D] FP32 (row-major) are standardised with per-feature mean / inverse
// std into Xn [B][D] BF16; W1 [H][D], W2 [H][H], w3 [H] (row-major, out x in); activations
// Z (pre-GELU, FP32) and A (post-GELU, BF16) [B][H].
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <random>
#include <vector>

#include "common.cuh"
#include "tc.cuh"

namespace afqmc {
namespace {

using bf16 = __nv_bfloat16;

// GEMM tiles: 128 output rows (the tcgen05 M) x 64 columns, K in chunks of 64 BF16 (one 128-byte
// swizzle row per operand row), two chunks in flight
constexpr int TMB = 128, TNB = 64, TKB = 64, MLP_THREADS = 128;
constexpr int MA_TILE = TMB * 128, MB_TILE = TNB * 128, M_STAGE = MA_TILE + MB_TILE;
constexpr size_t MLP_SMEM = 2 * size_t(M_STAGE) + 1024 + 64;
constexpr int MLP_MAX_SPLIT = 4;

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
  // d/dz [z Phi(z)] = Phi(z) + z phi(z)
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
         z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ float to_f(bf16 x) { return __bfloat162float(x); }
__device__ __forceinline__ float to_f(float x) { return x; }

enum Epi { EPI_STORE = 0, EPI_BIAS_GELU = 1, EPI_GELU_GRAD = 2 };

// Instruction descriptor: kind::f16 with BF16 A and B, F32 D, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// byte offset of BF16 element (r, k) of a K-major tile in the 128-byte swizzle layout the UMMA
// descriptor expects (the layout TMA writes): 16-byte unit k/8 of row r sits at unit (k/8) ^ (r%8)
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
  return uint32_t(r) * 128u + ((uint32_t(k >> 3) ^ uint32_t(r & 7)) << 4) + uint32_t(k & 7) * 2u;
}

// rows x TKB of op(element) into a swizzled tile; elem(r, k) = P[r sr + k sk]; the thread walk
// follows the contiguous index for coalesced reads
template <typename T>
__device__ __forceinline__ void fill_tile(unsigned char* tile, int rows, int r0, int R, int k0,
                                          int K, const T* __restrict__ P, long sr, long sk) {
  const bool k_fast = (sk == 1);
  for (int idx = threadIdx.x; idx < rows * TKB; idx += MLP_THREADS) {
    int r, k;
    if (k_fast) {
      r = idx / TKB;
      k = idx - r * TKB;
    } else {
      k = idx / rows;
      r = idx - k * rows;
    }
    const int gr = r0 + r, gk = k0 + k;
    const float v = (gr < R && gk < K) ? to_f(P[gr * sr + gk * sk]) : 0.f;
    *reinterpret_cast<bf16*>(tile + sw128_off(r, k)) = __float2bfloat16(v);
  }
}

// C[m][n] = sum_k A(m, k) B(k, n), A(m, k) = A[m sam + k sak], B(k, n) = B[k sbk + n sbn],
// operands rounded to BF16 in shared memory, FP32 accumulation in tensor memory:
//   EPI_STORE:     Cf[m][n] = acc                                   (FP32, ldc)
//   EPI_BIAS_GELU: Z = acc + bias[n]; Cf = Z (FP32); Cb = gelu(Z) (BF16)
//   EPI_GELU_GRAD: Cb = acc * gelu'(Zin[m][n])                      (BF16)
// All 128 threads convert the next K chunk into the free stage while one thread's MMAs run on
// the other (an mbarrier per stage tells when those MMAs have read it); the four warps then
// read their 32 accumulator rows from tensor memory.  Waits are bounded (error word err).
// Split K (gridDim.z > 1): CTA z sums the chunks [z per, (z + 1) per) and stores its partial
// sum (EPI_STORE) at Cf + z * split_stride; splitk_reduce_kernel adds them in order.
template <typename TA, typename TB, int EPI>
__global__ void __launch_bounds__(MLP_THREADS, 1) mlp_gemm_kernel(
    int M, int N, int K, const TA* __restrict__ A, long sam, long sak, const TB* __restrict__ B,
    long sbk, long sbn, float* __restrict__ Cf, bf16* __restrict__ Cb, long ldc,
    const float* __restrict__ bias, const float* __restrict__ Zin, long split_stride,
    unsigned* err) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* done = reinterpret_cast<uint64_t*>(base + 2 * M_STAGE);  // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int m0 = blockIdx.y * TMB, n0 = blockIdx.x * TNB;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    tc::mbar_init(&done[0], 1);
    tc::mbar_init(&done[1], 1);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tmem_slot, TNB);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t taddr = *tmem_slot;
  constexpr uint32_t ID = idesc_bf16(TMB, TNB);
  const int nk_all = (K + TKB - 1) / TKB;
  const int per = (nk_all + int(gridDim.z) - 1) / int(gridDim.z);
  const int kbeg = int(blockIdx.z) * per;
  const int nk = max(0, min(nk_all, kbeg + per) - kbeg);  // this CTA's chunks
  if (gridDim.z > 1) Cf += long(blockIdx.z) * split_stride;
  for (int j = 0; j < nk; ++j) {
    const int s = j & 1, kc = kbeg + j;
    unsigned char* st = base + s * M_STAGE;
    // the MMAs of chunk j - 2 read this stage
    if (j >= 2) tc::mbar_wait(&done[s], unsigned((j - 2) >> 1) & 1u, err, abort_flag);
    fill_tile(st, TMB, m0, M, kc * TKB, K, A, sam, sak);
    fill_tile(st + MA_TILE, TNB, n0, N, kc * TKB, K, B, sbn, sbk);
    // the generic-proxy stores above become visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0 && !*abort_flag) {
      tc::tc_fence_after();
      const uint32_t sa = tc::smem_u32(st), sb = tc::smem_u32(st + MA_TILE);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        if (kc * TKB + kk * 16 >= K) break;
        mma_bf16(taddr, tc::sdesc_sw128(sa) + uint64_t(2 * kk), tc::sdesc_sw128(sb) + uint64_t(2 * kk),
                 ID, (j > 0 || kk > 0) ? 1u : 0u);
      }
      tc::mma_commit(&done[s]);
    }
  }
  // the last commit completes after every earlier MMA of this thread
  const int last = nk - 1;
  const bool mine = nk > 0 && !*abort_flag &&
                    tc::mbar_wait(&done[last & 1], unsigned(last >> 1) & 1u, err, abort_flag);
  // every thread takes the same branch: the tensor-memory loads below are warp-collective
  const bool ok = __syncthreads_and(mine) != 0;
  tc::tc_fence_after();
  if (nk == 0 && gridDim.z > 1) {
    // a split without chunks (K shorter than the splits): its partial sum is zero
    const int m = m0 + warp * 32 + lane;
    if (m < M)
      for (int n = n0; n < min(N, n0 + TNB); ++n) Cf[long(m) * ldc + n] = 0.f;
  }
  if (ok) {
    const int m = m0 + warp * 32 + lane;
    const uint32_t trow = taddr + (uint32_t(warp * 32) << 16);
#pragma unroll 1
    for (int c0 = 0; c0 < TNB; c0 += 16) {
      float v[16];
      tc::tmem_ld16(trow + c0, v);
      tc::tmem_ld_wait();
      if (m >= M) continue;
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int n = n0 + c0 + j;
        if (n >= N) break;
        const long o = long(m) * ldc + n;
        float x = v[j];
        if (EPI == EPI_STORE) {
          Cf[o] = x;
        } else if (EPI == EPI_BIAS_GELU) {
          x += bias[n];
          Cf[o] = x;
          Cb[o] = __float2bfloat16(gelu(x));
        } else {
          Cb[o] = __float2bfloat16(x * gelu_grad(Zin[o]));
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, TNB);
}

// the split-K partial sums P[z][m][n] (z < nsplit, ld N) added in order, then the epilogue
template <int EPI>
__global__ void splitk_reduce_kernel(const float* __restrict__ P, int nsplit, int M, int N,
                                     float* __restrict__ Cf, bf16* __restrict__ Cb, long ldc,
                                     const float* __restrict__ bias,
                                     const float* __restrict__ Zin) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= long(M) * N) return;
  const int m = int(i / N), n = int(i - long(m) * N);
  float x = 0.f;
  for (int z = 0; z < nsplit; ++z) x += P[long(z) * M * N + i];
  const long o = long(m) * ldc + n;
  if (EPI == EPI_STORE) {
    Cf[o] = x;
  } else if (EPI == EPI_BIAS_GELU) {
    x += bias[n];
    Cf[o] = x;
    Cb[o] = __float2bfloat16(gelu(x));
  } else {
    Cb[o] = __float2bfloat16(x * gelu_grad(Zin[o]));
  }
}

// Xn[b][d] = bf16((X[b][d] - mean[d]) * istd[d])
__global__ void standardize_kernel(const float* __restrict__ X, const float* __restrict__ mean,
                                   const float* __restrict__ istd, int B, int D,
                                   bf16* __restrict__ Xn) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= long(B) * D) return;
  const int d = int(i % D);
  Xn[i] = __float2bfloat16((X[i] - mean[d]) * istd[d]);
}

// y[b] = A[b] . w3 + b3 (one warp per row); with target: the Huber loss of r = y - t with
// threshold HUBER (r^2 / 2 inside, HUBER (|r| - HUBER / 2) outside) averaged over the batch into
// loss[0] and its derivative clamp(r, -HUBER, HUBER) / B into dy[b]: heavy-tailed exchange
// energies then cannot blow up a step
constexpr float HUBER = 2.0f;
__global__ void head_kernel(const bf16* __restrict__ A, const float* __restrict__ w3,
                            const float* __restrict__ b3, int B, int H, float* __restrict__ y,
                            const float* __restrict__ target, float* __restrict__ dy,
                            float* __restrict__ loss) {
  const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (b >= B) return;
  float s = 0.f;
  for (int j = lane; j < H; j += 32) s += __bfloat162float(A[long(b) * H + j]) * w3[j];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) {
    const float v = s + b3[0];
    if (y) y[b] = v;
    if (target) {
      const float r = v - target[b];
      const float a = fabsf(r);
      dy[b] = fminf(fmaxf(r, -HUBER), HUBER) / B;
      atomicAdd(loss, (a <= HUBER ? 0.5f * r * r : HUBER * (a - 0.5f * HUBER)) / B);
    }
  }
}

// dZ2[b][j] = dy[b] w3[j] gelu'(Z2[b][j]) (BF16)
__global__ void head_backward_kernel(const float* __restrict__ dy, const float* __restrict__ w3,
                                     const float* __restrict__ Z, int B, int H,
                                     bf16* __restrict__ dZ) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= long(B) * H) return;
  const int j = int(i % H);
  dZ[i] = __float2bfloat16(dy[i / H] * w3[j] * gelu_grad(Z[i]));
}

// out[j] = sum_b X[b][j] s[b] (s = nullptr: 1), column sums over the batch
template <typename T>
__global__ void column_sum_kernel(const T* __restrict__ X, const float* __restrict__ s, int B,
                                  int H, float* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= H) return;
  float acc = 0.f;
  for (int b = 0; b < B; ++b) acc += to_f(X[long(b) * H + j]) * (s ? s[b] : 1.f);
  out[j] = acc;
}

__global__ void sum_kernel(const float* __restrict__ x, int n, float* __restrict__ out) {
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t += red[w];
    out[0] = t;
  }
}

// Adam (bias-corrected) on FP32 master weights; the BF16 copy follows (when present)
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, long n, float lr,
                            float b1, float b2, float eps, float c1, float c2,
                            bf16* __restrict__ pb) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (pb) pb[i] = __float2bfloat16(pi);
}

__global__ void to_bf16_kernel(const float* __restrict__ x, long n, bf16* __restrict__ y) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16(x[i]);
}

// X[w] = [Re vbias (Nc), Im vbias (Nc), Re G[a][a] (a < N), Im G[a][a], and with E:
// Re E1, Im E1, Re EJ, Im EJ] for each walker
__global__ void exchange_features_kernel(const c128* __restrict__ vb, long ldv,
                                         const c128* __restrict__ G, long ldG, int N, int M,
                                         int Nc, int W, const c128* __restrict__ E,
                                         float* __restrict__ X) {
  const int w = blockIdx.x;
  const int D = 2 * Nc + 2 * N + (E ? 4 : 0);
  float* x = X + long(w) * D;
  if (E && threadIdx.x == 0) {
    x[2 * Nc + 2 * N + 0] = float(E[w * 3 + 0].x);
    x[2 * Nc + 2 * N + 1] = float(E[w * 3 + 0].y);
    x[2 * Nc + 2 * N + 2] = float(E[w * 3 + 2].x);
    x[2 * Nc + 2 * N + 3] = float(E[w * 3 + 2].y);
  }
  for (int i = threadIdx.x; i < Nc; i += blockDim.x) {
    const c128 v = vb[long(w) * ldv + i];
    x[i] = float(v.x);
    x[Nc + i] = float(v.y);
  }
  for (int a = threadIdx.x; a < N; a += blockDim.x) {
    const c128 v = G[long(w) * ldG + long(a) * M + a];
    x[2 * Nc + a] = float(v.x);
    x[2 * Nc + N + a] = float(v.y);
  }
}

// y <- y a + b
__global__ void affine_kernel(float* __restrict__ y, long n, float a, float b) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) y[i] = y[i] * a + b;
}

// out[b] = (t[b] - mean) * inv
__global__ void normalize_target_kernel(const float* __restrict__ t, long n, float mean,
                                        float inv, float* __restrict__ out) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (t[i] - mean) * inv;
}

unsigned grid1(long n, int t) { return unsigned((n + t - 1) / t); }

}  // namespace
}  // namespace afqmc

using namespace afqmc;

struct afqmc_mlp_s {
  int device = 0;
  int D = 0, H = 0, cap = 0;
  long step = 0;
  float y_mean = 0.f, y_std = 1.f;
  // parameters (FP32 masters), their BF16 copies, gradients and Adam moments; one block each:
  // [W1 (H D) | b1 (H) | W2 (H H) | b2 (H) | w3 (H) | b3 (1)]
  float *P = nullptr, *Gr = nullptr, *Mo = nullptr, *Vo = nullptr;
  bf16* Pb = nullptr;  // BF16 W1 | W2 (same offsets as P for W1; W2 after H D)
  float *mean = nullptr, *istd = nullptr;
  // batch workspace (cap rows)
  bf16 *Xn = nullptr, *A1 = nullptr, *A2 = nullptr, *dZ2 = nullptr, *dZ1 = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *y = nullptr, *dy = nullptr, *loss = nullptr;
  float* ws = nullptr;  // split-K partial sums (ws_cap floats)
  long ws_cap = 0;
  unsigned* err = nullptr;  // bounded-wait error word of the GEMM kernels (bit 0: timeout)
  long nparam() const { return long(H) * D + H + long(H) * H + H + H + 1; }
  long oW1() const { return 0; }
  long ob1() const { return long(H) * D; }
  long oW2() const { return ob1() + H; }
  long ob2() const { return oW2() + long(H) * H; }
  long ow3() const { return ob2() + H; }
  long ob3() const { return ow3() + H; }
  void free_batch() {
    for (void* p : {(void*)Xn, (void*)A1, (void*)A2, (void*)dZ2, (void*)dZ1, (void*)Z1,
                    (void*)Z2, (void*)y, (void*)dy, (void*)ws})
      if (p) cudaFree(p);
    Xn = A1 = A2 = dZ2 = dZ1 = nullptr;
    Z1 = Z2 = y = dy = ws = nullptr;
    cap = 0;
    ws_cap = 0;
  }
  ~afqmc_mlp_s() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    free_batch();
    for (void* p : {(void*)P, (void*)Gr, (void*)Mo, (void*)Vo, (void*)Pb, (void*)mean,
                    (void*)istd, (void*)loss, (void*)err})
      if (p) cudaFree(p);
    cudaSetDevice(prev);
  }
};

namespace {

int mlp_batch(afqmc_mlp h, int B) {
  if (h->cap >= B) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  h->free_batch();
  const size_t bh = size_t(B) * h->H;
  AFQMC_CUDA_TRY(cudaMalloc(&h->Xn, sizeof(bf16) * size_t(B) * h->D));
  AFQMC_CUDA_TRY(cudaMalloc(&h->A1, sizeof(bf16) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->A2, sizeof(bf16) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->dZ2, sizeof(bf16) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->dZ1, sizeof(bf16) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Z1, sizeof(float) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Z2, sizeof(float) * bh));
  AFQMC_CUDA_TRY(cudaMalloc(&h->y, sizeof(float) * B));
  AFQMC_CUDA_TRY(cudaMalloc(&h->dy, sizeof(float) * B));
  // split-K partial sums of the GEMMs with few output tiles: up to MLP_MAX_SPLIT x (B or H) x H
  h->ws_cap = long(MLP_MAX_SPLIT) * std::max(B, h->H) * h->H;
  AFQMC_CUDA_TRY(cudaMalloc(&h->ws, sizeof(float) * size_t(h->ws_cap)));
  h->cap = B;
  return AFQMC_OK;
}

int g_mlp_sms = 0;

// C = epilogue(A B).  With fewer output tiles than half the SMs and a long K, the K range is
// split over up to MLP_MAX_SPLIT CTAs per tile whose partial sums (in the handle's workspace) a
// second kernel adds in a fixed order: deterministic, and the SMs stay busy.
template <typename TA, typename TB, int EPI>
int gemm(afqmc_mlp h, cudaStream_t s, int M, int N, int K, const TA* A, long sam, long sak,
         const TB* B, long sbk, long sbn, float* Cf, bf16* Cb, long ldc,
         const float* bias = nullptr, const float* Zin = nullptr) {
  if (M <= 0 || N <= 0) return AFQMC_OK;
  if (g_mlp_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_mlp_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  dim3 grid((N + TNB - 1) / TNB, (M + TMB - 1) / TMB);
  const long tiles = long(grid.x) * grid.y;
  const int nk = (K + TKB - 1) / TKB;
  int nsplit = 1;
  if (2 * tiles < g_mlp_sms && nk >= 8) {
    nsplit = int(std::min<long>(MLP_MAX_SPLIT, g_mlp_sms / tiles));
    nsplit = std::min(nsplit, nk / 4);
    if (long(nsplit) * M * N > h->ws_cap) nsplit = 1;
  }
  if (nsplit > 1) {
    auto kern = mlp_gemm_kernel<TA, TB, EPI_STORE>;
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        int(MLP_SMEM)));
    grid.z = nsplit;
    kern<<<grid, MLP_THREADS, MLP_SMEM, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, h->ws, nullptr, N,
                                             nullptr, nullptr, long(M) * N, h->err);
    AFQMC_TRY(launch_status("mlp_gemm_kernel"));
    splitk_reduce_kernel<EPI><<<grid1(long(M) * N, 256), 256, 0, s>>>(h->ws, nsplit, M, N, Cf,
                                                                      Cb, ldc, bias, Zin);
    return launch_status("splitk_reduce_kernel");
  }
  auto kern = mlp_gemm_kernel<TA, TB, EPI>;
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(MLP_SMEM)));
  kern<<<grid, MLP_THREADS, MLP_SMEM, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, Cf, Cb, ldc, bias,
                                           Zin, 0, h->err);
  return launch_status("mlp_gemm_kernel");
}

// forward pass of B rows: Xn, Z1/A1, Z2/A2, y (normalised units)
int mlp_forward(afqmc_mlp h, const float* X, int B, cudaStream_t s) {
  const int D = h->D, H = h->H;
  standardize_kernel<<<grid1(long(B) * D, 256), 256, 0, s>>>(X, h->mean, h->istd, B, D, h->Xn);
  AFQMC_TRY(launch_status("standardize_kernel"));
  // Z1 = Xn W1^T + b1
  AFQMC_TRY((gemm<bf16, bf16, EPI_BIAS_GELU>(h, s, B, H, D, h->Xn, D, 1, h->Pb + h->oW1(), 1, D,
                                             h->Z1, h->A1, H, h->P + h->ob1())));
  // Z2 = A1 W2^T + b2
  AFQMC_TRY((gemm<bf16, bf16, EPI_BIAS_GELU>(h, s, B, H, H, h->A1, H, 1, h->Pb + h->oW2(), 1, H,
                                             h->Z2, h->A2, H, h->P + h->ob2())));
  return AFQMC_OK;
}

// gradients of the mean squared error (normalised units) for the batch of the last forward pass
int mlp_backward(afqmc_mlp h, int B, cudaStream_t s) {
  const int D = h->D, H = h->H;
  float* g = h->Gr;
  // head: dw3 = A2^T dy, db3 = sum dy, dZ2 = dy w3 gelu'(Z2)
  column_sum_kernel<bf16><<<grid1(H, 128), 128, 0, s>>>(h->A2, h->dy, B, H, g + h->ow3());
  AFQMC_TRY(launch_status("column_sum_kernel"));
  sum_kernel<<<1, 256, 0, s>>>(h->dy, B, g + h->ob3());
  AFQMC_TRY(launch_status("sum_kernel"));
  head_backward_kernel<<<grid1(long(B) * H, 256), 256, 0, s>>>(h->dy, h->P + h->ow3(), h->Z2, B,
                                                               H, h->dZ2);
  AFQMC_TRY(launch_status("head_backward_kernel"));
  // dW2 = dZ2^T A1, db2 = column sums of dZ2
  AFQMC_TRY((gemm<bf16, bf16, EPI_STORE>(h, s, H, H, B, h->dZ2, 1, H, h->A1, H, 1, g + h->oW2(),
                                         nullptr, H)));
  column_sum_kernel<bf16><<<grid1(H, 128), 128, 0, s>>>(h->dZ2, nullptr, B, H, g + h->ob2());
  AFQMC_TRY(launch_status("column_sum_kernel"));
  // dZ1 = (dZ2 W2) gelu'(Z1)
  AFQMC_TRY((gemm<bf16, bf16, EPI_GELU_GRAD>(h, s, B, H, H, h->dZ2, H, 1, h->Pb + h->oW2(), H, 1,
                                             nullptr, h->dZ1, H, nullptr, h->Z1)));
  // dW1 = dZ1^T Xn, db1 = column sums of dZ1
  AFQMC_TRY((gemm<bf16, bf16, EPI_STORE>(h, s, H, D, B, h->dZ1, 1, H, h->Xn, D, 1, g + h->oW1(),
                                         nullptr, D)));
  column_sum_kernel<bf16><<<grid1(H, 128), 128, 0, s>>>(h->dZ1, nullptr, B, H, g + h->ob1());
  return launch_status("column_sum_kernel");
}

}  // namespace

extern "C" int afqmc_mlp_create(int D, int H, unsigned long long seed, afqmc_mlp* out) {
  AFQMC_CHECK_ARG(out && D > 0 && H > 0 && H % 8 == 0 && D % 2 == 0,
                  "afqmc_mlp_create: D=%d (even), H=%d (multiple of 8)", D, H);
  *out = nullptr;
  std::unique_ptr<afqmc_mlp_s> h(new (std::nothrow) afqmc_mlp_s());
  AFQMC_CHECK_ARG(h, "afqmc_mlp_create: out of host memory");
  cudaGetDevice(&h->device);
  h->D = D;
  h->H = H;
  const long np = h->nparam();
  // He-style uniform initialisation for GELU layers, small output layer, zero biases
  std::vector<float> p(np, 0.f);
  std::mt19937_64 rng(seed);
  auto fill = [&](long off, long n, float bound) {
    std::uniform_real_distribution<float> u(-bound, bound);
    for (long i = 0; i < n; ++i) p[off + i] = u(rng);
  };
  fill(h->oW1(), long(H) * D, std::sqrt(6.f / D));
  fill(h->oW2(), long(H) * H, std::sqrt(6.f / H));
  fill(h->ow3(), H, std::sqrt(3.f / H));
  AFQMC_CUDA_TRY(cudaMalloc(&h->P, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Gr, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Mo, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Vo, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMalloc(&h->Pb, sizeof(bf16) * np));
  AFQMC_CUDA_TRY(cudaMalloc(&h->mean, sizeof(float) * D));
  AFQMC_CUDA_TRY(cudaMalloc(&h->istd, sizeof(float) * D));
  AFQMC_CUDA_TRY(cudaMalloc(&h->loss, sizeof(float)));
  AFQMC_CUDA_TRY(cudaMalloc(&h->err, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaMemset(h->err, 0, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaMemcpy(h->P, p.data(), sizeof(float) * np, cudaMemcpyHostToDevice));
  AFQMC_CUDA_TRY(cudaMemset(h->Gr, 0, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMemset(h->Mo, 0, sizeof(float) * np));
  AFQMC_CUDA_TRY(cudaMemset(h->Vo, 0, sizeof(float) * np));
  std::vector<float> z(D, 0.f), o(D, 1.f);
  AFQMC_CUDA_TRY(cudaMemcpy(h->mean, z.data(), sizeof(float) * D, cudaMemcpyHostToDevice));
  AFQMC_CUDA_TRY(cudaMemcpy(h->istd, o.data(), sizeof(float) * D, cudaMemcpyHostToDevice));
  to_bf16_kernel<<<grid1(np, 256), 256>>>(h->P, np, h->Pb);
  AFQMC_TRY(launch_status("to_bf16_kernel"));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = h.release();
  return AFQMC_OK;
}

extern "C" int afqmc_mlp_destroy(afqmc_mlp h) {
  delete h;
  return AFQMC_OK;
}

extern "C" int afqmc_mlp_set_normalization(afqmc_mlp h, const float* mean, const float* istd,
                                           float y_mean, float y_std) {
  AFQMC_CHECK_ARG(h && mean && istd && y_std > 0.f, "afqmc_mlp_set_normalization: bad argument");
  AFQMC_CUDA_TRY(cudaMemcpy(h->mean, mean, sizeof(float) * h->D, cudaMemcpyHostToDevice));
  AFQMC_CUDA_TRY(cudaMemcpy(h->istd, istd, sizeof(float) * h->D, cudaMemcpyHostToDevice));
  h->y_mean = y_mean;
  h->y_std = y_std;
  return AFQMC_OK;
}

extern "C" int afqmc_mlp_params(afqmc_mlp h, int which, float* host, int to_device) {
  AFQMC_CHECK_ARG(h && host && which >= 0 && which <= 1, "afqmc_mlp_params: bad argument");
  AFQMC_CHECK_ARG(!(which == 1 && to_device), "afqmc_mlp_params: gradients are read-only");
  float* d = which == 0 ? h->P : h->Gr;
  const long np = h->nparam();
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  if (to_device) {
    AFQMC_CUDA_TRY(cudaMemcpy(d, host, sizeof(float) * np, cudaMemcpyHostToDevice));
    to_bf16_kernel<<<grid1(np, 256), 256>>>(h->P, np, h->Pb);
    AFQMC_TRY(launch_status("to_bf16_kernel"));
    AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  } else {
    AFQMC_CUDA_TRY(cudaMemcpy(host, d, sizeof(float) * np, cudaMemcpyDeviceToHost));
  }
  return AFQMC_OK;
}

extern "C" long afqmc_mlp_num_params(afqmc_mlp h) { return h ? h->nparam() : 0; }

extern "C" int afqmc_mlp_predict(afqmc_mlp h, const float* X, int B, float* y,
                                 afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && X && y && B >= 0, "afqmc_mlp_predict: bad argument");
  if (B == 0) return AFQMC_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  AFQMC_TRY(mlp_batch(h, B));
  AFQMC_TRY(mlp_forward(h, X, B, s));
  head_kernel<<<grid1(B, 4), 128, 0, s>>>(h->A2, h->P + h->ow3(), h->P + h->ob3(), B, h->H, y,
                                          nullptr, nullptr, nullptr);
  AFQMC_TRY(launch_status("head_kernel"));
  // back to the target's units
  affine_kernel<<<grid1(B, 256), 256, 0, s>>>(y, B, h->y_std, h->y_mean);
  return launch_status("affine_kernel");
}

// forward + loss + backward for a batch: gradients left in the handle, loss (device, may be
// NULL) = mean (y - t)^2 / 2 in normalised units; t in the target's units
static int mlp_grad(afqmc_mlp h, const float* X, const float* t, int B, float* loss,
                    cudaStream_t s) {
  AFQMC_TRY(mlp_batch(h, B));
  AFQMC_TRY(mlp_forward(h, X, B, s));
  // normalised target into dy's buffer first, then the head overwrites dy with the residual
  normalize_target_kernel<<<grid1(B, 256), 256, 0, s>>>(t, B, h->y_mean, 1.f / h->y_std, h->dy);
  AFQMC_TRY(launch_status("normalize_target_kernel"));
  AFQMC_CUDA_TRY(cudaMemsetAsync(h->loss, 0, sizeof(float), s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(h->y, h->dy, sizeof(float) * B, cudaMemcpyDeviceToDevice, s));
  head_kernel<<<grid1(B, 4), 128, 0, s>>>(h->A2, h->P + h->ow3(), h->P + h->ob3(), B, h->H,
                                          nullptr, h->y, h->dy, h->loss);
  AFQMC_TRY(launch_status("head_kernel"));
  AFQMC_TRY(mlp_backward(h, B, s));
  if (loss)
    AFQMC_CUDA_TRY(cudaMemcpyAsync(loss, h->loss, sizeof(float), cudaMemcpyDeviceToDevice, s));
  return AFQMC_OK;
}

extern "C" int afqmc_mlp_gradients(afqmc_mlp h, const float* X, const float* t, int B,
                                   float* loss, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && X && t && B > 0, "afqmc_mlp_gradients: bad argument");
  return mlp_grad(h, X, t, B, loss, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int afqmc_mlp_train_step(afqmc_mlp h, const float* X, const float* t, int B, float lr,
                                    float* loss, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && X && t && B > 0 && lr > 0.f, "afqmc_mlp_train_step: bad argument");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  AFQMC_TRY(mlp_grad(h, X, t, B, loss, s));
  ++h->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, float(h->step)), c2 = 1.f - std::pow(b2, float(h->step));
  const long np = h->nparam();
  adam_kernel<<<grid1(np, 256), 256, 0, s>>>(h->P, h->Gr, h->Mo, h->Vo, np, lr, b1, b2, 1e-8f,
                                             c1, c2, h->Pb);
  return launch_status("adam_kernel");
}

extern "C" int afqmc_exchange_features(const afqmc_c128* vbias, long ldv, const afqmc_c128* G,
                                       long ldG, int N, int M, int Nc, int W,
                                       const afqmc_c128* E, float* X, afqmc_stream stream) {
  AFQMC_CHECK_ARG(vbias && G && X && N > 0 && M >= N && Nc > 0 && W >= 0,
                  "afqmc_exchange_features: bad argument");
  if (W == 0) return AFQMC_OK;
  exchange_features_kernel<<<W, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const c128*>(vbias), ldv, reinterpret_cast<const c128*>(G), ldG, N, M, Nc,
      W, reinterpret_cast<const c128*>(E), X);
  return launch_status("exchange_features_kernel");
}
