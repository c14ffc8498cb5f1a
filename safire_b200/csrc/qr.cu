// Batched re-orthonormalisation of the walkers' Slater matrices.
//
// Reference: det_ops::orthogonalize (src/AFQMC/SlaterDeterminantOperations/orthogonalize.hpp:
// 131-169) calls LAPACK geqrf + ungqr on each S_w (M x N) and multiplies column i of Q by
// scl_i = sign(Re R_ii) (log_determinant_from_geqrf, numerics/operations/determinants_impl.hpp:
// 77-108).  The result is the unique Q whose R has a real positive diagonal, so any stable QR gives
// the same walker.  Here: CholeskyQR2 — the Gram matrices S^H S and the products S R^{-1} run as
// batched DMMA GEMMs, the N x N Cholesky factorisations and triangular inverses in one CTA per
// walker; two passes make Q orthonormal to rounding for the well-conditioned matrices that periodic
// re-orthogonalisation keeps.
#include "detops.cuh"
#include "zgemm.cuh"

namespace afqmc {
namespace {

// ---------------------------------------------------------------------------------------------
// CholeskyQR: G = S^H S = R^H R (R upper, real positive diagonal), Rinv = R^{-1}; one CTA per
// walker, the N x N matrices in shared memory.  logdetR[w] += sum_i log R_ii.
// ---------------------------------------------------------------------------------------------
constexpr int CH_THREADS = 256;

__global__ void __launch_bounds__(CH_THREADS)
    chol_inv_kernel(const c128* __restrict__ Gram, c128* __restrict__ Rinv, c128* __restrict__ logdetR,
                    int N) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int PP = N | 1;
  c128* a = reinterpret_cast<c128*>(smem_raw);  // [N][PP]  -> R (upper)
  c128* x = a + size_t(N) * PP;                 // [N][PP]  -> R^{-1}
  double* dg = reinterpret_cast<double*>(x + size_t(N) * PP);  // [N] R_ii
  const long w = blockIdx.x;
  const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
  const c128* Gw = Gram + w * long(N) * N;
  for (int i = ty; i < N; i += CH_THREADS / 32)
    for (int j = tx; j < N; j += 32) {
      a[i * PP + j] = Gw[long(i) * N + j];
      x[i * PP + j] = cmk(0, 0);
    }
  __syncthreads();
  // right-looking Cholesky on the upper triangle: row j <- row j / sqrt(a_jj); trailing update
  for (int j = 0; j < N; ++j) {
    double d = a[j * PP + j].x;
    d = d > 1e-300 ? sqrt(d) : 1e-150;
    const double dinv = 1.0 / d;
    __syncthreads();
    if (tid == 0) dg[j] = d;
    for (int l = j + 1 + tid; l < N; l += CH_THREADS) a[j * PP + l] = cscale(a[j * PP + l], dinv);
    __syncthreads();
    // A_il -= conj(R_ji) R_jl  for j < i <= l
    for (int i = j + 1 + ty; i < N; i += CH_THREADS / 32) {
      const c128 rji = cconj(a[j * PP + i]);
      for (int l = i + tx; l < N; l += 32) a[i * PP + l] = csub(a[i * PP + l], cmul(rji, a[j * PP + l]));
    }
    __syncthreads();
  }
  // R^{-1}: back substitution row by row, thread = column c
  for (int i = N - 1; i >= 0; --i) {
    for (int c = i + tid; c < N; c += CH_THREADS) {
      c128 acc = cmk(i == c ? 1.0 : 0.0, 0.0);
      for (int l = i + 1; l <= c; ++l) acc = csub(acc, cmul(a[i * PP + l], x[l * PP + c]));
      x[i * PP + c] = cscale(acc, 1.0 / dg[i]);
    }
    __syncthreads();
  }
  c128* Rw = Rinv + w * long(N) * N;
  for (int i = ty; i < N; i += CH_THREADS / 32)
    for (int j = tx; j < N; j += 32) Rw[long(i) * N + j] = x[i * PP + j];
  if (ty == 0) {
    double sr = 0.0;
    for (int i = tx; i < N; i += 32) sr += log(dg[i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sr += __shfl_xor_sync(0xffffffffu, sr, off);
    if (tx == 0) logdetR[w] = cadd(logdetR[w], cmk(sr, 0.0));
  }
}

}  // namespace

// One CholeskyQR pass: Q = S R^{-1} written to Q (ldQ), R from the Gram matrix of S.
static int cholqr_pass(cudaStream_t s, const c128* S, long ldS, c128* Q, long ldQ, c128* logdetR,
                       int W, int M, int N, c128* gram, c128* rinv) {
  GemmParams g{};
  g.m = N; g.n = N; g.k = M;
  g.A = S; g.lda = N; g.strideA = ldS;  // A^H with A stored [M][N]
  g.B = S; g.ldb = N; g.strideB = ldS;
  g.C = gram; g.ldc = N; g.strideC = long(N) * N;
  g.alpha = cmk(1, 0); g.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, W, GH, false, GN, false, g));
  const int PP = N | 1;
  const size_t smem = 2 * size_t(N) * PP * sizeof(c128) + N * sizeof(double);
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(chol_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(smem)));
  chol_inv_kernel<<<W, CH_THREADS, smem, s>>>(gram, rinv, logdetR, N);
  AFQMC_TRY(launch_status("chol_inv_kernel"));
  GemmParams q{};
  q.m = M; q.n = N; q.k = N;
  q.A = S; q.lda = N; q.strideA = ldS;
  q.B = rinv; q.ldb = N; q.strideB = long(N) * N;
  q.C = Q; q.ldc = N; q.strideC = ldQ;
  q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
  return zgemm(s, W, GN, false, GN, false, q);
}

// det_ops::orthogonalize by CholeskyQR2: two passes give Q orthonormal to rounding for the
// well-conditioned walkers that the periodic re-orthogonalisation keeps; R = R2 R1 has a real
// positive diagonal, so Q is the same unique factor as geqrf + ungqr + sign fix.
int orthogonalize(cudaStream_t s, c128* S, long ldS, c128* logdetR, int W, int M, int N,
                  c128* work) {
  if (W <= 0 || N <= 0 || M <= 0) return AFQMC_OK;
  if (N > M) {
    set_error_detail("orthogonalize: N = %d > M = %d", N, M);
    return AFQMC_ERR_SHAPE;
  }
  if (2 * size_t(N | 1) * N * sizeof(c128) > 227 * 1024) {
    set_error_detail("orthogonalize: N = %d exceeds the shared-memory Cholesky kernel", N);
    return AFQMC_ERR_UNSUPPORTED;
  }
  const size_t nQ = size_t(W) * M * N, nG = size_t(W) * N * N;
  void* buf = work;
  if (!buf) AFQMC_CUDA_TRY(cudaMallocAsync(&buf, sizeof(c128) * (nQ + 2 * nG), s));
  c128* Q = static_cast<c128*>(buf);
  c128* gram = Q + nQ;
  c128* rinv = gram + nG;
  int st = cholqr_pass(s, S, ldS, Q, long(M) * N, logdetR, W, M, N, gram, rinv);
  if (!st) st = cholqr_pass(s, Q, long(M) * N, S, ldS, logdetR, W, M, N, gram, rinv);
  if (!work) cudaFreeAsync(buf, s);
  return st;
}

}  // namespace afqmc
