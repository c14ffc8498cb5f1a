// det_ops on the device: batched overlap matrices, LU log-determinants, inverses, mixed density
// matrices, Taylor propagation and QR re-orthonormalisation.
//
// Reference: src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp (log_overlap_impl 113-156,
// MixedDensityMatrix 535-601, inverse_logdet 43-111), determinants_impl.hpp (log-det conventions),
// propagate.hpp (apply_expM 41-70, propagate_impl 238-298), orthogonalize.hpp (131-169).
#include "detops.cuh"
#include "zgemm.cuh"

namespace afqmc {

__device__ __forceinline__ c128 wrap_imag(c128 z) {
  const double pi = 3.14159265358979323846;
  double im = z.y;
  if (im > pi) {
    while (im > pi) im -= 2 * pi;
  } else if (im < -pi) {
    while (im < -pi) im += 2 * pi;
  }
  return cmk(z.x, im);
}

// log(d + DBL_MIN) or log(-1*d + DBL_MIN), as log_determinant_from_getrf_impl writes it
__device__ __forceinline__ c128 log_pivot(c128 d, bool swapped) {
  const double small = 2.2250738585072014e-308;
  c128 v = swapped ? cmul(cmk(-1.0, 0.0), d) : d;
  return clog(cmk(v.x + small, v.y + 0.0));
}

// ---------------------------------------------------------------------------------------------
// Gauss-Jordan elimination with partial pivoting (pivot = first max |re|+|im|, as izamax) on
// [A | I] in shared memory.  The pivots are the U diagonal of getrf with the same row
// interchanges, so the log-determinant follows log_determinant_from_getrf; the right half ends as
// A^{-1} (zero for a singular A, as getri_or_zero).  One CTA per matrix.
// ---------------------------------------------------------------------------------------------
template <bool INVERT>
__global__ void __launch_bounds__(256) gj_logdet_kernel(const c128* __restrict__ A, long strideA,
                                                         c128* __restrict__ Ainv, long strideInv,
                                                         c128* __restrict__ ovlp, int N,
                                                         c128 post_scale, c128 post_add) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int P = INVERT ? 2 * N : N;  // row length of the augmented matrix
  c128* a = reinterpret_cast<c128*>(smem_raw);      // [N][P]
  c128* piv_val = a + size_t(N) * P;                 // [N]
  int* piv_swapped = reinterpret_cast<int*>(piv_val + N);
  __shared__ int s_piv;
  __shared__ int s_singular;
  __shared__ double s_red_v[8];
  __shared__ int s_red_i[8];

  const long w = blockIdx.x;
  const c128* Aw = A + w * strideA;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < N * N; e += nt) {
    int i = e / N, j = e % N;
    a[i * P + j] = Aw[e];
  }
  if (INVERT) {
    for (int e = tid; e < N * N; e += nt) {
      int i = e / N, j = e % N;
      a[i * P + N + j] = cmk(i == j ? 1.0 : 0.0, 0.0);
    }
  }
  if (tid == 0) s_singular = 0;
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    // pivot search in column k, rows k..N-1 (first maximal |re|+|im|)
    double best = -1.0;
    int bi = N;
    for (int i = k + tid; i < N; i += nt) {
      double v = cabs1(a[i * P + k]);
      if (v > best) {
        best = v;
        bi = i;
      }
    }
    for (int off = 16; off > 0; off >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, best, off);
      int oi = __shfl_down_sync(0xffffffffu, bi, off);
      if (ov > best || (ov == best && oi < bi)) {
        best = ov;
        bi = oi;
      }
    }
    if ((tid & 31) == 0) {
      s_red_v[tid >> 5] = best;
      s_red_i[tid >> 5] = bi;
    }
    __syncthreads();
    if (tid == 0) {
      double bv = s_red_v[0];
      int b = s_red_i[0];
      for (int q = 1; q < (nt + 31) / 32; ++q)
        if (s_red_v[q] > bv || (s_red_v[q] == bv && s_red_i[q] < b)) {
          bv = s_red_v[q];
          b = s_red_i[q];
        }
      s_piv = b;
      piv_swapped[k] = (b != k);
      if (!(bv > 0.0)) s_singular = 1;
    }
    __syncthreads();
    const int p = s_piv;
    if (p != k) {
      for (int j = tid; j < P; j += nt) {
        c128 t = a[k * P + j];
        a[k * P + j] = a[p * P + j];
        a[p * P + j] = t;
      }
      __syncthreads();
    }
    const c128 d = a[k * P + k];
    if (tid == 0) piv_val[k] = d;
    const bool zero = (d.x == 0.0 && d.y == 0.0);
    if (!zero) {
      // eliminate column k: below the diagonal (LU part) and, for the inverse, above it too
      const int r0 = INVERT ? 0 : k + 1;
      const int nrows = N - r0;
      const int ncols = P - (k + 1);
      const c128 dinv = cdiv(cmk(1.0, 0.0), d);
      // multipliers stored in column k of each row before the update
      for (int i = r0 + tid; i < N; i += nt) {
        if (i == k) continue;
        a[i * P + k] = cmul(a[i * P + k], dinv);
      }
      __syncthreads();
      for (int e = tid; e < nrows * ncols; e += nt) {
        int i = r0 + e / ncols, j = k + 1 + e % ncols;
        if (i == k) continue;
        a[i * P + j] = csub(a[i * P + j], cmul(a[i * P + k], a[k * P + j]));
      }
      __syncthreads();
      if (INVERT) {
        // row k scaled by 1/d so the left block becomes the identity
        for (int j = k + 1 + tid; j < P; j += nt) a[k * P + j] = cmul(a[k * P + j], dinv);
        __syncthreads();
      }
    }
  }

  if (tid == 0) {
    c128 res = ovlp[w];
    for (int k = 0; k < N; ++k) res = cadd(res, log_pivot(piv_val[k], piv_swapped[k] != 0));
    res = wrap_imag(res);
    ovlp[w] = cadd(cmul(post_scale, res), post_add);
  }
  if (INVERT) {
    c128* Iw = Ainv + w * strideInv;
    const bool sing = s_singular != 0;
    for (int e = tid; e < N * N; e += nt) {
      int i = e / N, j = e % N;
      Iw[e] = sing ? cmk(0.0, 0.0) : a[i * P + N + j];
    }
  }
}

int batched_logdet_inverse(cudaStream_t s, const c128* A, long strideA, c128* Ainv, long strideInv,
                           c128* ovlp, int W, int N, bool invert, c128 post_scale, c128 post_add) {
  if (W <= 0 || N <= 0) return AFQMC_OK;
  const int P = invert ? 2 * N : N;
  size_t smem = size_t(N) * P * sizeof(c128) + N * sizeof(c128) + N * sizeof(int);
  if (smem > 227 * 1024) {
    set_error_detail("batched_logdet_inverse: N = %d exceeds the shared-memory kernel (max 84)", N);
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (invert) {
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(gj_logdet_kernel<true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    gj_logdet_kernel<true><<<W, 256, smem, s>>>(A, strideA, Ainv, strideInv, ovlp, N, post_scale,
                                                post_add);
  } else {
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(gj_logdet_kernel<false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    gj_logdet_kernel<false><<<W, 256, smem, s>>>(A, strideA, nullptr, 0, ovlp, N, post_scale,
                                                 post_add);
  }
  return launch_status("gj_logdet_kernel");
}

// ---------------------------------------------------------------------------------------------
// Mixed density matrix / log overlap
// ---------------------------------------------------------------------------------------------
int overlap_matrices(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* T, int W,
                     int M, int N) {
  // T_w = PsiT (N x M) * S_w (M x N)   (math::product(A,B,TNN), density_matrix.hpp:142)
  GemmParams p{};
  p.m = N; p.n = N; p.k = M;
  p.A = PsiT; p.lda = M; p.strideA = 0;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = T; p.ldc = N; p.strideC = long(N) * N;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  return zgemm(s, W, GN, false, GN, false, p);
}

int log_overlap(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* ovlp, int W,
                int M, int N, c128* work_T, c128 post_scale, c128 post_add) {
  if (N == 0) return AFQMC_OK;
  AFQMC_TRY(overlap_matrices(s, PsiT, S, ldS, work_T, W, M, N));
  return batched_logdet_inverse(s, work_T, long(N) * N, nullptr, 0, ovlp, W, N, false, post_scale,
                                post_add);
}

int mixed_density_matrix(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* G,
                         long ldG, c128* ovlp, int W, int M, int N, bool compact, c128* work_T,
                         c128* work_NM, c128 post_scale, c128 post_add) {
  if (N == 0) return AFQMC_OK;
  AFQMC_TRY(overlap_matrices(s, PsiT, S, ldS, work_T, W, M, N));
  AFQMC_TRY(batched_logdet_inverse(s, work_T, long(N) * N, work_T, long(N) * N, ovlp, W, N, true,
                                   post_scale, post_add));
  // C = TNN^T * S^T  (product<'T','T'>, density_matrix.hpp:576): [N x M]
  c128* Cc = compact ? G : work_NM;
  long ldc_w = compact ? ldG : long(N) * M;
  GemmParams p{};
  p.m = N; p.n = M; p.k = N;
  p.A = work_T; p.lda = N; p.strideA = long(N) * N;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = Cc; p.ldc = M; p.strideC = ldc_w;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, W, GT, false, GT, false, p));
  if (compact) return AFQMC_OK;
  // full G = PsiT^T * C  (product<'T'>(A,TNM,C), density_matrix.hpp:584): [M x M]
  GemmParams q{};
  q.m = M; q.n = M; q.k = N;
  q.A = PsiT; q.lda = M; q.strideA = 0;
  q.B = work_NM; q.ldb = M; q.strideB = long(N) * M;
  q.C = G; q.ldc = M; q.strideC = ldG;
  q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
  return zgemm(s, W, GT, false, GN, false, q);
}

// ---------------------------------------------------------------------------------------------
// Taylor propagation: S <- P1 exp_T(i V) P1 S  (propagate.hpp:41-70, 238-298)
// work1/work2/work3: [W][M][N] each.
// ---------------------------------------------------------------------------------------------
int propagate(cudaStream_t s, const void* P1, bool p1_real, const c128* V, long strideV, c128* S,
              long ldS, int W, int M, int N, int order, c128* work1, c128* work2, c128* work3) {
  if (N == 0 || W == 0) return AFQMC_OK;
  const long sMN = long(M) * N;
  // T0 = P1 * S into work2, and the running sum TMN = T0 into work1
  GemmParams p{};
  p.m = M; p.n = N; p.k = M;
  p.A = P1; p.lda = M; p.strideA = 0;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = work2; p.ldc = N; p.strideC = sMN;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  p.D = work1; p.ldd = N; p.strideD = sMN; p.d_store = true;
  AFQMC_TRY(zgemm(s, W, GN, p1_real, GN, false, p));
  // T_n = (i/n) V T_{n-1};  TMN += T_n   (apply_expM<'N'>)
  c128* Tprev = work2;
  c128* Tnext = work3;
  for (int n = 1; n <= order; ++n) {
    GemmParams q{};
    q.m = M; q.n = N; q.k = M;
    q.A = V; q.lda = M; q.strideA = strideV;
    q.B = Tprev; q.ldb = N; q.strideB = sMN;
    q.C = Tnext; q.ldc = N; q.strideC = sMN;
    q.alpha = cmk(0.0, 1.0 / double(n)); q.beta = cmk(0, 0);
    q.D = work1; q.ldd = N; q.strideD = sMN; q.d_store = false;
    AFQMC_TRY(zgemm(s, W, GN, false, GN, false, q));
    c128* t = Tprev;
    Tprev = Tnext;
    Tnext = t;
  }
  // S = P1 * TMN
  GemmParams r{};
  r.m = M; r.n = N; r.k = M;
  r.A = P1; r.lda = M; r.strideA = 0;
  r.B = work1; r.ldb = N; r.strideB = sMN;
  r.C = S; r.ldc = N; r.strideC = ldS;
  r.alpha = cmk(1, 0); r.beta = cmk(0, 0);
  return zgemm(s, W, GN, p1_real, GN, false, r);
}

}  // namespace afqmc
