// Batched Householder QR re-orthonormalisation of the walkers' Slater matrices.
//
// Reference: det_ops::orthogonalize (src/AFQMC/SlaterDeterminantOperations/orthogonalize.hpp:
// 131-169) calls LAPACK geqrf + ungqr on each S_w (M x N) and multiplies column i of Q by
// scl_i = sign(Re R_ii) (log_determinant_from_geqrf, numerics/operations/determinants_impl.hpp:
// 77-108).  The result is the unique Q whose R has a real positive diagonal, so any stable QR gives
// the same walker; this kernel restates geqrf's reflectors (zlarfg convention: beta real,
// H = I - tau v v^H with v_0 = 1) and ungqr's backward accumulation (zung2r) in shared memory.
// One CTA per walker; the whole M x N matrix lives in shared memory (M*N <= 13.5k elements).
#include "detops.cuh"

namespace afqmc {
namespace {

constexpr int QR_THREADS = 256;
constexpr int QR_WARPS = QR_THREADS / 32;

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int q = 0; q < QR_WARPS; ++q) t += red[q];
    red[QR_WARPS] = t;
  }
  __syncthreads();
  return red[QR_WARPS];
}

// A(k:M, k+1:N) <- (I - ctau v v^H) A(k:M, k+1:N), v = [1, a(k+1:M, k)]
__device__ void apply_reflector(c128* a, int pitch, int M, int N, int k, c128 ctau, c128* wbuf) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int j = k + 1 + warp; j < N; j += QR_WARPS) {
    c128 acc = cmk(0, 0);
    for (int i = k + lane; i < M; i += 32) {
      c128 v = (i == k) ? cmk(1, 0) : a[i * pitch + k];
      acc = cadd(acc, cmul(cconj(v), a[i * pitch + j]));
    }
    for (int off = 16; off > 0; off >>= 1) {
      acc.x += __shfl_down_sync(0xffffffffu, acc.x, off);
      acc.y += __shfl_down_sync(0xffffffffu, acc.y, off);
    }
    if (lane == 0) wbuf[j] = cmul(ctau, acc);
  }
  __syncthreads();
  const int ncol = N - k - 1, nrow = M - k;
  for (int e = threadIdx.x; e < ncol * nrow; e += QR_THREADS) {
    int i = k + e / ncol, j = k + 1 + e % ncol;
    c128 v = (i == k) ? cmk(1, 0) : a[i * pitch + k];
    a[i * pitch + j] = csub(a[i * pitch + j], cmul(v, wbuf[j]));
  }
  __syncthreads();
}

__global__ void __launch_bounds__(QR_THREADS)
    qr_orthogonalize_kernel(c128* __restrict__ S, long ldS, c128* __restrict__ logdetR, int M,
                            int N) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int pitch = N | 1;  // odd pitch: conflict-free column walks of 16-byte elements
  c128* a = reinterpret_cast<c128*>(smem_raw);
  // 16-byte arrays first, the 8-byte diagonal last (keeps every c128 16-byte aligned)
  c128* tau = a + size_t(M) * pitch;                    // [N]
  c128* wbuf = tau + N;                                 // [N]
  double* rdiag = reinterpret_cast<double*>(wbuf + N);  // [N]
  __shared__ double red[QR_WARPS + 1];

  const long w = blockIdx.x;
  c128* Sw = S + w * ldS;
  for (int e = threadIdx.x; e < M * N; e += QR_THREADS) a[(e / N) * pitch + e % N] = Sw[e];
  __syncthreads();

  // ---- geqrf (zgeqr2): reflectors stored below the diagonal ----
  for (int k = 0; k < N; ++k) {
    double part = 0.0;
    for (int i = k + 1 + threadIdx.x; i < M; i += QR_THREADS) {
      c128 x = a[i * pitch + k];
      part += x.x * x.x + x.y * x.y;
    }
    const double xnorm2 = block_sum(part, red);
    const c128 alpha = a[k * pitch + k];
    c128 t = cmk(0, 0);
    double beta = alpha.x;
    if (!(xnorm2 == 0.0 && alpha.y == 0.0)) {
      beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2), alpha.x);
      t = cmk((beta - alpha.x) / beta, -alpha.y / beta);
      const c128 scal = cdiv(cmk(1, 0), cmk(alpha.x - beta, alpha.y));
      for (int i = k + 1 + threadIdx.x; i < M; i += QR_THREADS)
        a[i * pitch + k] = cmul(a[i * pitch + k], scal);
    }
    if (threadIdx.x == 0) {
      tau[k] = t;
      rdiag[k] = beta;
    }
    __syncthreads();
    // apply H^H = I - conj(tau) v v^H to the trailing columns
    if (k < N - 1 && (t.x != 0.0 || t.y != 0.0)) apply_reflector(a, pitch, M, N, k, cconj(t), wbuf);
  }

  // ---- log det R with the sign fix ----
  if (threadIdx.x == 0) {
    const double small = 2.2250738585072014e-308;
    c128 res = logdetR[w];
    for (int k = 0; k < N; ++k) {
      double scl = rdiag[k] < 0.0 ? -1.0 : 1.0;
      res = cadd(res, clog(cmk(scl * rdiag[k] + small, 0.0)));
    }
    logdetR[w] = res;
  }

  // ---- ungqr (zung2r): form Q in place, backward over the reflectors ----
  for (int k = N - 1; k >= 0; --k) {
    const c128 t = tau[k];
    if (k < N - 1 && (t.x != 0.0 || t.y != 0.0)) apply_reflector(a, pitch, M, N, k, t, wbuf);
    // column k of Q: [0..k-1] = 0, [k] = 1 - tau, [k+1..M-1] = -tau v
    for (int i = threadIdx.x; i < M; i += QR_THREADS) {
      c128 q;
      if (i < k) q = cmk(0, 0);
      else if (i == k) q = cmk(1.0 - t.x, -t.y);
      else q = cmul(cmk(-t.x, -t.y), a[i * pitch + k]);
      a[i * pitch + k] = q;
    }
    __syncthreads();
  }

  // S <- Q diag(scl)
  for (int e = threadIdx.x; e < M * N; e += QR_THREADS) {
    int i = e / N, j = e % N;
    double scl = rdiag[j] < 0.0 ? -1.0 : 1.0;
    Sw[e] = cscale(a[i * pitch + j], scl);
  }
}

}  // namespace

int orthogonalize(cudaStream_t s, c128* S, long ldS, c128* logdetR, int W, int M, int N) {
  if (W <= 0 || N <= 0 || M <= 0) return AFQMC_OK;
  if (N > M) {
    set_error_detail("orthogonalize: N = %d > M = %d", N, M);
    return AFQMC_ERR_SHAPE;
  }
  const int pitch = N | 1;
  size_t smem = size_t(M) * pitch * sizeof(c128) + N * (2 * sizeof(c128) + sizeof(double));
  if (smem > 227 * 1024) {
    set_error_detail("orthogonalize: M*N = %d x %d exceeds the shared-memory QR kernel", M, N);
    return AFQMC_ERR_UNSUPPORTED;
  }
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(qr_orthogonalize_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  qr_orthogonalize_kernel<<<W, QR_THREADS, smem, s>>>(S, ldS, logdetR, M, N);
  return launch_status("qr_orthogonalize_kernel");
}

}  // namespace afqmc
