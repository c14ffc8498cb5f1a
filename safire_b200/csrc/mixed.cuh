// Mixed-precision (tensor-core) contractions of the walker step (see mixed.cu).
#pragma once

#include "common.cuh"
#include "energy.cuh"

namespace afqmc {

struct MixedHam;  // split-TF32 copies of the Hamiltonian tensors + operand planes

int mixed_ham_create(MixedHam** out, const EnergyArgs& a, cudaStream_t s);
void mixed_ham_destroy(MixedHam* m);
// v [W][Nc] (complex128) = a * G Lnak^T
int vbias_mixed(cudaStream_t s, MixedHam* m, const c128* G, long ldG, c128* v, int W, double a);
// split planes of a * X L^T kept in m; V != nullptr also receives them as complex128 [W][M][M]
int vhs_mixed(cudaStream_t s, MixedHam* m, const c128* X, c128* V, int W, double a);
// S <- P1 exp_T(iV) P1 S with V from the last vhs_mixed call (P1 real float64 [M][M])
int propagate_mixed(cudaStream_t s, MixedHam* m, const void* P1, bool p1_real, c128* S, long ldS,
                    int W, int M, int N, int order);
// 0: one batched GEMM launch per Taylor product; 1 (default): all products of a walker in one
// persistent kernel (M <= 256, N <= 64), one or two walkers in flight per CTA chosen by the walker
// count; 2 / 3: the persistent kernel with one / two walkers in flight; 4 / 5: the same in the
// FP16 split (vHS then writes FP16 V planes)
int mixed_set_taylor_mode(MixedHam* m, int mode);
// the FP16 Taylor variants (4, 5) are available for these shapes
bool mixed_taylor_f16_ok(MixedHam* m);
// split planes of G for the exchange-energy GEMMs
int mixed_prepare_G(cudaStream_t s, MixedHam* m, const c128* G, long ldG, int W);
// T [(w,b)][(n,a)] for walkers [w0, w0+wc) of spin block sp (complex128, the chunk layout of
// energy_fp64)
int exchange_T_tc(cudaStream_t s, MixedHam* m, int sp, int w0, int wc, c128* workT);
// fused T-free exchange for spin block sp (real trial, N <= 50): exx/kl [W][Nc] +=
bool exchange_fused_ok(MixedHam* m, int sp);
int exchange_fused(cudaStream_t s, MixedHam* m, int sp, int W, c128* exx, c128* kl);
// vHS over the i <= k pairs only when every Cholesky vector is symmetric (enable = 1, the
// default) or over all pairs (0); *active tells whether the symmetric form runs
int mixed_set_vhs_symmetry(MixedHam* m, int enable, int* active);
// operand format of vbias, vHS and the exchange contraction: 0 auto (FP16 split when the shapes
// allow it), 1 TF32 split, 2 FP16 split (an error when the shapes do not allow it);
// *active_f16 tells whether the FP16 split runs
int mixed_set_split_format(MixedHam* m, int format, int* active_f16);
// 3: 3xTF32 (default), 1: single TF32 product in the exchange contraction
int mixed_set_exchange_split(MixedHam* m, int nsplit);
// tile shapes and orders that leave every result bit for bit the same: the vbias CTA tile width
// (128 or 64 Cholesky vectors) and the exchange kernel's L2 block (vector pairs per block of its
// tile order)
int mixed_set_tiles(MixedHam* m, int vbias_bn, int exch_nblk);
int mixed_get_tiles(MixedHam* m, int* vbias_bn, int* exch_nblk);
// one bounded device wait that nothing completes, with a budget of `budget` cycles (at most the
// kernels' own): AFQMC_ERR_TIMEOUT and bit 0 of the error word when it gave up
int mixed_wait_selftest(cudaStream_t s, MixedHam* m, long long budget);
int mixed_clear_error(MixedHam* m);
// first device-side wait timeout reported by the tensor-core kernels (0 = none)
int mixed_error_flag(MixedHam* m, unsigned* flag);

// C [rows_a][cols of B] (complex128, ldc) = A B^T with A complex128 [rows_a][K] (lda) and B real,
// given as complex128 [rows_b][K] (ldb) with zero imaginary parts: FP16 split products on the
// tensor cores, FP32 accumulation (B split once at creation; AFQMC_ERR_UNSUPPORTED when B has an
// imaginary part or K is not a multiple of 8)
struct TcGemmRB;
int tcgemm_rb_create(TcGemmRB** out, const c128* B, long rows_b, long K, long ldb);
void tcgemm_rb_destroy(TcGemmRB* g);
// c64_out: C holds complex64 (float2) elements, ldc counted in them
int tcgemm_rb_run(cudaStream_t s, TcGemmRB* g, const c128* A, long lda, int rows_a, c128* C,
                  long ldc, bool c64_out = false);

}  // namespace afqmc
