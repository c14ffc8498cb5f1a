// Device det_ops (see detops.cu / qr.cu).
#pragma once

#include "common.cuh"

namespace afqmc {

// ovlp[w] = post_scale * wrap(ovlp[w] + log det A_w) + post_add; Ainv_w = A_w^{-1} when invert.
int batched_logdet_inverse(cudaStream_t s, const c128* A, long strideA, c128* Ainv, long strideInv,
                           c128* ovlp, int W, int N, bool invert, c128 post_scale, c128 post_add);

// T_w = PsiT * S_w   ([W][N][N])
int overlap_matrices(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* T, int W,
                     int M, int N);

// det_ops::Log_Overlap with the post affine map (work_T: [W][N][N])
int log_overlap(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* ovlp, int W,
                int M, int N, c128* work_T, c128 post_scale, c128 post_add);

// det_ops::MixedDensityMatrix (work_T: [W][N][N]; work_NM: [W][N][M], only for !compact)
int mixed_density_matrix(cudaStream_t s, const c128* PsiT, const c128* S, long ldS, c128* G,
                         long ldG, c128* ovlp, int W, int M, int N, bool compact, c128* work_T,
                         c128* work_NM, c128 post_scale, c128 post_add);

// S <- P1 exp_T(i V) P1 S.  work1..3: [W][M][N] each.
int propagate(cudaStream_t s, const void* P1, bool p1_real, const c128* V, long strideV, c128* S,
              long ldS, int W, int M, int N, int order, c128* work1, c128* work2, c128* work3);

// det_ops::orthogonalize: S_w <- Q_w diag(sign(Re R_ii)), logdetR[w] += sum log(|R_ii|).
// work: [W*M*N + 2*W*N*N] complex, or nullptr to take it from the stream-ordered allocator.
int orthogonalize(cudaStream_t s, c128* S, long ldS, c128* logdetR, int W, int M, int N,
                  c128* work = nullptr);

}  // namespace afqmc
