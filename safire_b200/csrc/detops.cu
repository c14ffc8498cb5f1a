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
// A^{-1} (zero for a singular A, as getri_or_zero).  Without the inverse only the trailing
// submatrix is eliminated (plain LU) and the matrix needs a quarter of the shared memory, so more
// matrices share an SM.  One CTA per matrix, 8 warps: warp 0 finds the pivot, the pivot row, the
// old row k and the scaled multipliers are snapshotted, then every thread updates its
// (rows ty+8r) x (cols k+1+tx+32c) elements from the snapshots only: three barriers per step and
// no element read after another thread wrote it in the same phase.
// ---------------------------------------------------------------------------------------------
constexpr int GJ_THREADS = 256;

template <bool INVERT>
__global__ void __launch_bounds__(GJ_THREADS) gj_logdet_kernel(const c128* __restrict__ A,
                                                                long strideA,
                                                                c128* __restrict__ Ainv,
                                                                long strideInv,
                                                                c128* __restrict__ ovlp, int N,
                                                                c128 post_scale, c128 post_add) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int P = INVERT ? 2 * N : N;  // columns of the augmented matrix
  const int PP = P | 1;              // odd pitch: conflict-free column walks
  c128* a = reinterpret_cast<c128*>(smem_raw);  // [N][PP]
  c128* rbuf = a + size_t(N) * PP;              // pivot row (post-swap row k) [P]
  c128* kbuf = rbuf + P;                        // old row k [P]
  c128* mbuf = kbuf + P;                        // scaled multipliers of the post-swap rows [N]
  c128* piv_val = mbuf + N;                     // [N]
  int* piv_swapped = reinterpret_cast<int*>(piv_val + N);
  __shared__ int s_piv;
  __shared__ int s_singular;
  __shared__ c128 s_dinv;

  const long w = blockIdx.x;
  const c128* Aw = A + w * strideA;
  const int tid = threadIdx.x;
  const int tx = tid & 31, ty = tid >> 5;
  for (int i = ty; i < N; i += GJ_THREADS / 32) {
    for (int j = tx; j < N; j += 32) a[i * PP + j] = Aw[long(i) * N + j];
    if (INVERT)
      for (int j = tx; j < N; j += 32) a[i * PP + N + j] = cmk(i == j ? 1.0 : 0.0, 0.0);
  }
  if (tid == 0) s_singular = 0;
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    // 1. pivot search in column k, rows k..N-1 (warp 0)
    if (ty == 0) {
      double best = -1.0;
      int bi = N;
      for (int i = k + tx; i < N; i += 32) {
        const double v = cabs1(a[i * PP + k]);
        if (v > best) {
          best = v;
          bi = i;
        }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, best, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (ov > best || (ov == best && oi < bi)) {
          best = ov;
          bi = oi;
        }
      }
      if (tx == 0) {
        if (bi >= N) bi = k;  // a column of NaNs: zero pivot at row k
        s_piv = bi;
        piv_swapped[k] = (bi != k);
        const c128 d = a[bi * PP + k];
        piv_val[k] = d;
        if (!(best > 0.0)) {
          s_singular = 1;
          s_dinv = cmk(0, 0);
        } else {
          s_dinv = cdiv(cmk(1.0, 0.0), d);
        }
      }
    }
    __syncthreads();
    const int p = s_piv;
    const c128 dinv = s_dinv;
    const bool zero = (dinv.x == 0.0 && dinv.y == 0.0);
    // 2. snapshots: pivot row, old row k, multipliers (column k of the post-swap rows) * dinv
    for (int j = k + tid; j < P; j += GJ_THREADS) {
      rbuf[j] = a[p * PP + j];
      kbuf[j] = a[k * PP + j];
    }
    for (int i = (INVERT ? 0 : k) + tid; i < N; i += GJ_THREADS) {
      const c128 c = (i == k) ? a[p * PP + k] : ((i == p) ? a[k * PP + k] : a[i * PP + k]);
      mbuf[i] = cmul(c, dinv);
    }
    __syncthreads();
    // 3. row swap + elimination (+ pivot-row scaling for the inverse)
    const int r0 = INVERT ? 0 : k;
    for (int i = r0 + ty; i < N; i += GJ_THREADS / 32) {
      if (i == k) {
        for (int j = k + 1 + tx; j < P; j += 32)
          a[k * PP + j] = (INVERT && !zero) ? cmul(rbuf[j], dinv) : rbuf[j];
      } else {
        const c128 m = mbuf[i];
        const bool from_k = (i == p);
        for (int j = k + 1 + tx; j < P; j += 32) {
          const c128 src = from_k ? kbuf[j] : a[i * PP + j];
          a[i * PP + j] = zero ? src : csub(src, cmul(m, rbuf[j]));
        }
      }
    }
    __syncthreads();
  }

  // log det: sum_k log(+-U_kk + DBL_MIN), accumulated onto ovlp, imaginary part wrapped
  if (ty == 0) {
    double sr = 0.0, si = 0.0;
    for (int k = tx; k < N; k += 32) {
      const c128 l = log_pivot(piv_val[k], piv_swapped[k] != 0);
      sr += l.x;
      si += l.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, off);
      si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    if (tx == 0) {
      c128 res = cadd(ovlp[w], cmk(sr, si));
      res = wrap_imag(res);
      ovlp[w] = cadd(cmul(post_scale, res), post_add);
    }
  }
  if (INVERT) {
    c128* Iw = Ainv + w * strideInv;
    const bool sing = s_singular != 0;
    for (int i = ty; i < N; i += GJ_THREADS / 32)
      for (int j = tx; j < N; j += 32) Iw[long(i) * N + j] = sing ? cmk(0.0, 0.0) : a[i * PP + N + j];
  }
}

// ---------------------------------------------------------------------------------------------
// Register-resident Gauss-Jordan / LU for N <= 64 (the production sizes).  One CTA of 64 C threads
// per matrix (C = 2 column classes up to N = 32, else 4); thread t holds row
// i = t % 64 and the columns j = h + C q of class h = t / 64 in registers (q < QMAX), so a step
// touches shared memory only for the pivot column, the pivot row and the row that moves in the
// interchange.
// Step k: every warp finds the pivot p (first max |re|+|im| in column k, rows k..N-1, as izamax)
// from the column buffer; the owners of row p write it as it stands with 1 in column k, the owners
// of row k write the old row k; after one barrier every row i != k subtracts g_i times the pivot
// row, g_i = f_i / pivot with f_i its column-k element before the interchange (the multiplier in
// getf2's rounding order), and row p takes the old row k first.  Column k is moved to the column
// buffer and zeroed in the registers at the end of step k-1, so the update leaves -g_i there (the
// in-place Gauss-Jordan inverse); row k becomes the pivot row / pivot.  Without the inverse only
// rows below k are eliminated (plain LU, the same U diagonal).  The row interchanges permute the
// columns of the in-place inverse; they are undone on the way out (columns swapped in reverse step
// order).  Two barriers a step.
// ---------------------------------------------------------------------------------------------
template <int QMAX, int C, bool INVERT>
__global__ void __launch_bounds__(64 * C, C == 2 ? 3 : (QMAX <= 13 ? 2 : 1)) gj_reg_kernel(const c128* __restrict__ A,
                                                               long strideA,
                                                               c128* __restrict__ Ainv,
                                                               long strideInv,
                                                               c128* __restrict__ ovlp, int N,
                                                               c128 post_scale, c128 post_add) {
  __shared__ c128 rowbuf[64];     // pivot row, column k = 1
  __shared__ c128 kbuf[64];       // old row k (moves to row p)
  __shared__ c128 colbuf[2][64];  // column k of every row at step k (buffer k & 1)
  __shared__ c128 piv_val[64];
  __shared__ int perm[64];
  __shared__ int pos[64];
  __shared__ int s_singular;

  const int t = threadIdx.x;
  const int i = t & 63;
  const int h = t >> 6;  // column class: columns j = h + C q
  const int lane = t & 31;
  const bool row_ok = i < N;
  const long w = blockIdx.x;
  const c128* Aw = A + w * strideA;

  c128 a[QMAX];
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int j = h + C * q;
    a[q] = (row_ok && j < N) ? Aw[long(i) * N + j] : cmk(0.0, 0.0);
  }
  if (h == 0) {
    if (row_ok) colbuf[0][i] = a[0];
    a[0] = cmk(0.0, 0.0);
  }
  if (t == 0) s_singular = 0;
  __syncthreads();

  for (int k = 0; k < N; ++k) {
    const c128* col = colbuf[k & 1];
    // pivot: first max |re|+|im| in column k, rows k..N-1.  Non-negative doubles order as their
    // bit patterns, so the maximum is two warp max-reductions (high, then low word); NaN and rows
    // outside k..N-1 take key 0.  The first row holding the maximum comes from two ballots.
    const int r0 = k + lane, r1 = k + lane + 32;
    const double v0 = r0 < N ? cabs1(col[r0]) : 0.0;
    const double v1 = r1 < N ? cabs1(col[r1]) : 0.0;
    const unsigned long long k0 = (v0 == v0) ? static_cast<unsigned long long>(__double_as_longlong(v0)) : 0ull;
    const unsigned long long k1 = (v1 == v1) ? static_cast<unsigned long long>(__double_as_longlong(v1)) : 0ull;
    const unsigned long long kl = k1 > k0 ? k1 : k0;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, unsigned(kl >> 32));
    const unsigned mlo = __reduce_max_sync(0xffffffffu, unsigned(kl >> 32) == mhi ? unsigned(kl) : 0u);
    const unsigned long long kmax = (static_cast<unsigned long long>(mhi) << 32) | mlo;
    const bool zero = (kmax == 0ull);
    const unsigned b0 = __ballot_sync(0xffffffffu, r0 < N && k0 == kmax);
    const unsigned b1 = __ballot_sync(0xffffffffu, r1 < N && k1 == kmax);
    // a zero (or NaN) column: zero pivot at row k, no interchange
    const int p = zero ? k : (b0 ? k + __ffs(b0) - 1 : k + 32 + __ffs(b1) - 1);
    const c128 piv = col[p];
    // 1/pivot = conj(pivot) / |pivot|^2
    const double rden = 1.0 / (piv.x * piv.x + piv.y * piv.y);
    const c128 dinv = cmk(piv.x * rden, -piv.y * rden);
    if (t == 0) {
      perm[k] = p;
      piv_val[k] = piv;
      if (zero) s_singular = 1;
    }
    if (!zero) {
      // pivot row as it stands (its column k was zeroed in the registers) with 1 in column k
      if (i == p) {
#pragma unroll
        for (int q = 0; q < QMAX; ++q) {
          const int j = h + C * q;
          if (j < N) rowbuf[j] = a[q];
        }
        if (h == (k % C)) rowbuf[k] = cmk(1.0, 0.0);
      }
      if (i == k && p != k) {
#pragma unroll
        for (int q = 0; q < QMAX; ++q) {
          const int j = h + C * q;
          if (j < N) kbuf[j] = a[q];
        }
      }
    }
    __syncthreads();
    c128* nxt = colbuf[(k + 1) & 1];
    const int kn = k + 1;
    if (!zero && row_ok) {
      if (i == k) {
        // row k <- pivot row / pivot (column k: 1/pivot)
        if (INVERT) {
#pragma unroll
          for (int q = 0; q < QMAX; ++q) {
            const int j = h + C * q;
            if (j < N) a[q] = cmul(rowbuf[j], dinv);
          }
        }
      } else if (INVERT || i > k) {
        // row i -= g * pivot row, g = f / pivot (column k: 0 - g = -f/pivot)
        const c128 f = (i == p) ? col[k] : col[i];
        const c128 g = cmul(f, dinv);
        if (i == p) {
#pragma unroll
          for (int q = 0; q < QMAX; ++q) {
            const int j = h + C * q;
            if (j < N) a[q] = kbuf[j];
          }
        }
        const c128 ng = cmk(-g.x, -g.y);
#pragma unroll
        for (int q = 0; q < QMAX; ++q) {
          const int j = h + C * q;
          if (j < N) {
            const c128 r = rowbuf[j];
            a[q].x = fma(ng.x, r.x, fma(g.y, r.y, a[q].x));
            a[q].y = fma(ng.x, r.y, fma(ng.y, r.x, a[q].y));
          }
          // keep the pivot-row loads in groups of eight (bounds the registers they hold)
          if ((q & 7) == 7) asm volatile("" ::: "memory");
        }
      }
    }
    // column k+1 moves to the column buffer for the next pivot search and is zeroed in the
    // registers (warp-uniform branch to its register)
    if (kn < N && h == (kn % C)) {
      switch (kn / C) {
#define GR_CASE(Q)                          \
  case Q:                                   \
    if (Q < QMAX) {                         \
      constexpr int QQ = Q < QMAX ? Q : 0;  \
      if (row_ok) nxt[i] = a[QQ];           \
      a[QQ] = cmk(0.0, 0.0);                \
    }                                       \
    break;
        GR_CASE(0) GR_CASE(1) GR_CASE(2) GR_CASE(3) GR_CASE(4) GR_CASE(5) GR_CASE(6) GR_CASE(7)
        GR_CASE(8) GR_CASE(9) GR_CASE(10) GR_CASE(11) GR_CASE(12) GR_CASE(13) GR_CASE(14)
        GR_CASE(15)
#undef GR_CASE
        default:
          break;
      }
    }
    __syncthreads();
  }

  if (t < 32) {
    double sr = 0.0, si = 0.0;
    for (int k = t; k < N; k += 32) {
      const c128 l = log_pivot(piv_val[k], perm[k] != k);
      sr += l.x;
      si += l.y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sr += __shfl_xor_sync(0xffffffffu, sr, off);
      si += __shfl_xor_sync(0xffffffffu, si, off);
    }
    if (t == 0) {
      c128 res = cadd(ovlp[w], cmk(sr, si));
      res = wrap_imag(res);
      ovlp[w] = cadd(cmul(post_scale, res), post_add);
    }
  }
  if (INVERT) {
    // at[c] = column of the in-place result that ends in column c (kept in kbuf's memory,
    // free after the last step); pos is its inverse
    int* at = reinterpret_cast<int*>(kbuf);
    if (t < N) at[t] = t;
    __syncthreads();
    if (t == 0)
      for (int k = N - 1; k >= 0; --k) {
        const int q = perm[k];
        const int x = at[k];
        at[k] = at[q];
        at[q] = x;
      }
    __syncthreads();
    if (t < N) pos[at[t]] = t;
    __syncthreads();
    const bool sing = s_singular != 0;
    if (row_ok) {
      c128* Iw = Ainv + w * strideInv + long(i) * N;
#pragma unroll
      for (int q = 0; q < QMAX; ++q) {
        const int j = h + C * q;
        if (j < N) Iw[pos[j]] = sing ? cmk(0.0, 0.0) : a[q];
      }
    }
  }
}

template <int QMAX, int C>
void launch_gj_reg(cudaStream_t s, const c128* A, long strideA, c128* Ainv, long strideInv,
                   c128* ovlp, int W, int N, bool invert, c128 post_scale, c128 post_add) {
  if (invert)
    gj_reg_kernel<QMAX, C, true><<<W, 64 * C, 0, s>>>(A, strideA, Ainv, strideInv, ovlp, N,
                                                      post_scale, post_add);
  else
    gj_reg_kernel<QMAX, C, false><<<W, 64 * C, 0, s>>>(A, strideA, nullptr, 0, ovlp, N,
                                                       post_scale, post_add);
}

int batched_logdet_inverse(cudaStream_t s, const c128* A, long strideA, c128* Ainv, long strideInv,
                           c128* ovlp, int W, int N, bool invert, c128 post_scale, c128 post_add) {
  if (W <= 0 || N <= 0) return AFQMC_OK;
  if (N <= 64) {
    if (N <= 8)
      launch_gj_reg<4, 2>(s, A, strideA, Ainv, strideInv, ovlp, W, N, invert, post_scale, post_add);
    else if (N <= 16)
      launch_gj_reg<8, 2>(s, A, strideA, Ainv, strideInv, ovlp, W, N, invert, post_scale, post_add);
    else if (N <= 32)
      launch_gj_reg<16, 2>(s, A, strideA, Ainv, strideInv, ovlp, W, N, invert, post_scale,
                           post_add);
    else if (N <= 52)
      launch_gj_reg<13, 4>(s, A, strideA, Ainv, strideInv, ovlp, W, N, invert, post_scale,
                           post_add);
    else
      launch_gj_reg<16, 4>(s, A, strideA, Ainv, strideInv, ovlp, W, N, invert, post_scale,
                           post_add);
    return launch_status("gj_reg_kernel");
  }
  const int P = invert ? 2 * N : N;
  const int PP = P | 1;
  size_t smem = (size_t(N) * PP + 2 * size_t(P) + 2 * size_t(N)) * sizeof(c128) + N * sizeof(int);
  if (smem > 227 * 1024) {
    set_error_detail("batched_logdet_inverse: N = %d exceeds the shared-memory kernel", N);
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (invert) {
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(gj_logdet_kernel<true>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    gj_logdet_kernel<true><<<W, GJ_THREADS, smem, s>>>(A, strideA, Ainv, strideInv, ovlp, N,
                                                       post_scale, post_add);
  } else {
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(gj_logdet_kernel<false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    gj_logdet_kernel<false><<<W, GJ_THREADS, smem, s>>>(A, strideA, nullptr, 0, ovlp, N,
                                                        post_scale, post_add);
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
