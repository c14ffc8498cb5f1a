/*
 * afqmc_c.h — C ABI of the B200-native batched AFQMC walker step.
 *
 * Drop-in boundary for the hot path of bkesk/SAFIRE (paths below are relative to that repository):
 *   - HamiltonianOperations (Real3IndexFactorization alternative):
 *       src/AFQMC/HamiltonianOperations/HamiltonianOperations.h:33-103,
 *       src/AFQMC/HamiltonianOperations/Real3IndexFactorization.hpp
 *   - det_ops free functions: src/AFQMC/SlaterDeterminantOperations/{density_matrix,orthogonalize,
 *       propagate}.hpp
 *   - the single-determinant NOMSD trial: src/AFQMC/Wavefunctions/NOMSD.{hpp,cpp}
 *   - the hybrid phaseless propagator step and comb population control:
 *       src/AFQMC/Propagators/AFQMCBasePropagator.{h,cpp}, Propagators/WalkerSetUpdate.hpp,
 *       src/AFQMC/Walkers/population_control.hpp
 *
 * Conventions
 *   - complex128 is afqmc_c128 {re, im}, layout-compatible with std::complex<double>.
 *   - All arrays are C-ordered (row-major) like the reference's nda views.  Device arrays are
 *     caller-owned device pointers unless a parameter says "host".
 *   - Every function returns an AFQMC_* status; 0 is success.  afqmc_last_error() gives a
 *     human-readable detail for the calling thread.  No C++ exception crosses the ABI.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are asynchronous with
 *     respect to the host unless documented otherwise.
 *   - Where the reference accumulates into an output (log-overlaps), so do these functions.
 */
#ifndef AFQMC_C_H
#define AFQMC_C_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afqmc_c128 {
  double re, im;
} afqmc_c128;

typedef struct CUstream_st* afqmc_stream; /* == cudaStream_t */

/* status codes (the reference throws; these replace its utils::check / APP_ABORT paths) */
#define AFQMC_OK 0
#define AFQMC_ERR_ARG 1         /* invalid argument / null pointer */
#define AFQMC_ERR_SHAPE 2       /* shape or size mismatch (utils::check "Size mismatch") */
#define AFQMC_ERR_CUDA 3        /* CUDA runtime error */
#define AFQMC_ERR_NONFINITE 4   /* non-finite value where the reference would abort */
#define AFQMC_ERR_TIMEOUT 5     /* a bounded device wait gave up */
#define AFQMC_ERR_ALLOC 6       /* device allocation failed */
#define AFQMC_ERR_UNSUPPORTED 7 /* configuration outside what the library implements */
#define AFQMC_ERR_COLLAPSE 8    /* total walker weight collapsed (population_control.hpp:39) */

/* walker types (reference enum WALKER_TYPES, src/AFQMC/config.h:46-52) */
#define AFQMC_CLOSED 1
#define AFQMC_COLLINEAR 2

/* precision of the contraction kernels */
#define AFQMC_PREC_FP64 0  /* complex128 throughout (the drop-in) */
#define AFQMC_PREC_MIXED 1 /* 3xTF32 tensor-core contractions, FP64 LU/QR/weights/energy sums */

/* walker_data scalar properties, in walker-row order (src/AFQMC/Walkers/WalkerConfig.hpp:28-48,
 * WalkerSetBase.cpp:88-110) */
#define AFQMC_WEIGHT 0
#define AFQMC_PHASE 1
#define AFQMC_PSEUDO_ELOC 2
#define AFQMC_E1 3
#define AFQMC_EXX 4
#define AFQMC_EJ 5
#define AFQMC_OVLP 6
#define AFQMC_LOGSCL_UP 7
#define AFQMC_LOGSCL_DN 8
#define AFQMC_IS_UNITARY 9
#define AFQMC_THETA 10
#define AFQMC_NPROP 11

const char* afqmc_status_string(int status);
const char* afqmc_last_error(void);
int afqmc_version(void);
/* number of kernels this library has launched in the process (instrumentation) */
unsigned long long afqmc_kernel_launches(void);

/* =========================================================================================
 * det_ops (src/AFQMC/SlaterDeterminantOperations/density_matrix.hpp, orthogonalize.hpp,
 * propagate.hpp).  S is [W][M][N] with a walker stride of ldS elements (>= M*N), so a walker
 * buffer row (Slater block followed by properties) can be passed directly.
 * ========================================================================================= */

/* det_ops::Log_Overlap(A=PsiT [N][M], B=S, ovlp) — density_matrix.hpp:431-447.
 * ovlp[w] += log det(PsiT * S_w), imaginary part wrapped to [-pi, pi] after accumulation
 * (numerics/operations/determinants_impl.hpp:32-75). */
int afqmc_log_overlap(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS, afqmc_c128* ovlp,
                      int W, int M, int N, afqmc_stream stream);

/* afqmc_log_overlap without any device allocation.  No counterpart in the reference: it exists
 * for callers that cannot allocate device memory (an application that reserves all device memory
 * for its own pool and treats a later cudaMalloc as an error, or one already at its memory limit).
 * Same arguments and result as afqmc_log_overlap; its scratch is a fixed 8 MiB device array inside
 * the library, so W*N*N must not exceed 524288 (larger calls return AFQMC_ERR_SHAPE).  All calls on
 * a device share that array: calls that overlap on the GPU race.  The first call on a device
 * looks up the array's address with that device current; make it before any stream capture. */
int afqmc_log_overlap_noalloc(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS,
                              afqmc_c128* ovlp, int W, int M, int N, afqmc_stream stream);

/* det_ops::MixedDensityMatrix(A=PsiT, B=S, C=G, ovlp, compact, herm=true) —
 * density_matrix.hpp:535-601.  compact != 0: G [W][N][M] = (PsiT S_w)^{-T} S_w^T;
 * compact == 0: G [W][M][M] = PsiT^T (PsiT S_w)^{-T} S_w^T.  ldG = walker stride of G.
 * A singular PsiT S_w gives a zero inverse (getri_or_zero, numerics/nda_functions.hpp:422). */
int afqmc_mixed_density_matrix(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS,
                               afqmc_c128* G, long ldG, afqmc_c128* ovlp, int W, int M, int N,
                               int compact, afqmc_stream stream);

/* det_ops::MixedDensityMatrix with a bra per walker (A [W][M][N], walker stride ldA) —
 * density_matrix.hpp:603-649, the overload BackPropEstimator and MixedEstimator call with the
 * back-propagated references (Estimators/BackPropEstimator.hpp:105-107).  T_w = A_w^H S_w,
 * ovlp[w] += log det T_w; compact != 0: G [W][N][M] = T_w^{-T} S_w^T; compact == 0:
 * G [W][M][M] = (S_w T_w^{-1} A_w^H)^T.  A singular T_w gives a zero inverse. */
int afqmc_mixed_density_matrix_batched(const afqmc_c128* A, long ldA, const afqmc_c128* S,
                                       long ldS, afqmc_c128* G, long ldG, afqmc_c128* ovlp, int W,
                                       int M, int N, int compact, afqmc_stream stream);

/* det_ops::detail::inverse_logdet (batched) — density_matrix.hpp:80-111.
 * Ainv [W][N][N] = A^{-1} (zero if singular), logdet[w] += log det A_w. */
int afqmc_inverse_logdet(const afqmc_c128* A, afqmc_c128* Ainv, afqmc_c128* logdet, int W, int N,
                         afqmc_stream stream);

/* det_ops::orthogonalize(A=S, log_detR) — orthogonalize.hpp:131-169.  In place: S_w <- Q_w with
 * R's diagonal made real-positive; logdetR[w] += sum_i log(|R_ii|) (the sign-fixed QR log det). */
int afqmc_orthogonalize(afqmc_c128* S, long ldS, afqmc_c128* logdetR, int W, int M, int N,
                        afqmc_stream stream);

/* det_ops::detail::propagate_impl<'N'>(npol=1, S, P1, V, order) — propagate.hpp:238-298.
 * S_w <- P1 * sum_{n=0..order} (i V_w)^n/n! * P1 * S_w.  P1 [M][M] (shared), V [W][M][M]. */
int afqmc_propagate(const afqmc_c128* P1, const afqmc_c128* V, afqmc_c128* S, long ldS, int W,
                    int M, int N, int order, afqmc_stream stream);

/* =========================================================================================
 * HamiltonianOperations, Real3IndexFactorization alternative (ndet = 1, npol = 1).
 * ========================================================================================= */
typedef struct afqmc_ham_s* afqmc_ham;

/* Builds the device tensors of RealDenseHamiltonian::getHamiltonianOperations
 * (src/AFQMC/Hamiltonians/RealDenseHamiltonian.cpp:36-184): Likn, Lnak = PsiT L, haj = PsiT h
 * (HamiltonianOperations/detail/one_body.hpp:124-153) and v0 = -1/2 sum L L.
 *   Likn  host float64 [nspin_H2][M][M][Nc]   (Hamiltonian/DenseFactorized/L)
 *   hij   host complex [nspin_H1][M][M]       (Hamiltonian/hcore)
 *   PsiT  host complex [nup][M] (+ [ndn][M] for COLLINEAR): the trial's conjugate transpose
 * The handle is bound to the device current at creation. */
int afqmc_ham_create(int walker_type, int M, int nup, int ndn, int Nc, const double* Likn,
                     int nspin_H2, const afqmc_c128* hij, int nspin_H1, double E0,
                     const afqmc_c128* PsiT, afqmc_ham* out);
/* The tensor-hypercontraction factorisation behind the same handle — THCOps
 * (HamiltonianOperations/THCOps.hpp:50-105, the constructor; vbias :571-615, vHS :462-569,
 * energy :149-293).  The two-electron integrals are L_n[i][k] = sum_u X[i][u] X[k][u] L[u][n]:
 *   X     host float64 [M][nu]   (Piu: the orbitals at the nu interpolation points)
 *   L     host float64 [nu][nv]  (Luv; nv plays the part of N_chol: vbias [W][nv], X [W][nv])
 *   Z     host float64 [nu][nu]  (rotMuv = L L^T; NULL: computed from L)
 *   hij   host complex [nspin_H1][M][M];  v0 host float64 [M][M] (NULL: computed from X, Z)
 *   PsiT  as afqmc_ham_create (the trial-rotated points Y = PsiT X are built from it)
 * Every afqmc_ham_* operation and the propagator then use the THC contractions, in complex128
 * only (a mixed-precision call returns AFQMC_ERR_UNSUPPORTED); one determinant (as THCOps). */
int afqmc_ham_create_thc(int walker_type, int M, int nup, int ndn, int nu, int nv,
                         const double* X, const double* L, const double* Z,
                         const afqmc_c128* hij, int nspin_H1, const double* v0, double E0,
                         const afqmc_c128* PsiT, afqmc_ham* out);
/* nu and nv of a THC handle (0, 0 for a Cholesky one) */
int afqmc_ham_thc_info(afqmc_ham ham, int* nu, int* nv);
int afqmc_ham_destroy(afqmc_ham ham);
/* number_of_cholesky_vectors / energy_offset / walker type (Real3IndexFactorization.hpp:432-438) */
int afqmc_ham_info(afqmc_ham ham, int* walker_type, int* M, int* nup, int* ndn, int* Nc,
                   double* E0);
/* Copies of the built tensors (for tests): Lnak [nspin][Nc][N_s][M], haj [nel][M],
 * vexx [nspin_H2][M][M] (all host). Any pointer may be NULL. */
int afqmc_ham_get_tensors(afqmc_ham ham, afqmc_c128* Lnak, afqmc_c128* haj, double* vexx);

/* Real3IndexFactorization::vbias — Real3IndexFactorization.hpp:328-428 (half-rotated G).
 * G [W][nel*M], v [W][Nc]: v = sqrt(dt) (x2 if CLOSED) sum_{a,k} G[w,a,k] Lnak[n,a,k]. */
int afqmc_ham_vbias(afqmc_ham ham, const afqmc_c128* G, afqmc_c128* v, int W, double dt,
                    int precision, afqmc_stream stream);

/* Real3IndexFactorization::vHS — Real3IndexFactorization.hpp:282-326.  X [W][Nc];
 * V [nspin_vHS][W][M][M] (caller-owned; the reference returns a pooled buffer):
 * V[s,w,i,k] = sqrt(dt) sum_n L_s[i,k,n] X[w,n]. */
int afqmc_ham_vhs(afqmc_ham ham, const afqmc_c128* X, afqmc_c128* V, int W, double dt,
                  int precision, afqmc_stream stream);

/* Real3IndexFactorization::energy — Real3IndexFactorization.hpp:138-174, 476-590.
 * E [W][3] = (E1, EXX, EJ) from the half-rotated G [W][nel*M]. */
int afqmc_ham_energy(afqmc_ham ham, const afqmc_c128* G, afqmc_c128* E, int W, int addH1,
                     int addEJ, int addEXX, int precision, afqmc_stream stream);

/* TF32 products per real product in the mixed-precision exchange contraction: 3 (3xTF32, the
 * default) or 1 (plain TF32, for runs whose energy tolerance allows it). */
int afqmc_ham_set_exchange_split(afqmc_ham ham, int nsplit);

/* Mixed-precision vHS over symmetric Cholesky vectors.  When every L_n is symmetric (to 1e-10 of
 * the largest |L|, checked once on the device; real orbitals make it so), V_w = sum_n X_n L_n is
 * complex symmetric and the tensor-core vHS computes only the (i, k) pairs with i <= k, writing
 * each value to V[w][i][k] and V[w][k][i].  enable = 1 (default) uses that form when the vectors
 * qualify, 0 always computes all M^2 pairs (the reference's contraction,
 * Real3IndexFactorization.hpp:282-326, computes all of them).  *active (optional) receives 1 when
 * the symmetric form runs. */
int afqmc_ham_set_vhs_symmetry(afqmc_ham ham, int enable, int* active);

/* Operand format of the mixed-precision vbias, vHS and exchange contractions.  Both keep 22
 * significant bits of each operand in two terms, x = hi + lo, and multiply with three products
 * (hi*hi + hi*lo + lo*hi) accumulated in FP32:
 *   AFQMC_SPLIT_TF32  TF32 terms (kind::tf32 MMAs, 4 bytes per term);
 *   AFQMC_SPLIT_FP16  FP16 terms of operands scaled by powers of two (per walker row for G and
 *                     X, one scale per static tensor), the scales undone exactly in the
 *                     epilogue: twice the tensor rate and half the operand bytes of TF32;
 *   AFQMC_SPLIT_AUTO  FP16 when the shapes allow it (M and N_chol multiples of 8, one spin block
 *                     of Cholesky vectors, a real trial, CLOSED walkers with 1..50 electrons),
 *                     else TF32 (the default).
 * AFQMC_SPLIT_FP16 on shapes that do not allow it returns AFQMC_ERR_UNSUPPORTED.  *active_f16
 * (optional) receives 1 when the FP16 split runs.  The Taylor propagation always uses TF32. */
#define AFQMC_SPLIT_AUTO 0
#define AFQMC_SPLIT_TF32 1
#define AFQMC_SPLIT_FP16 2
int afqmc_ham_set_split_format(afqmc_ham ham, int format, int* active_f16);

/* Mixed-precision Taylor propagation.  0 launches one batched GEMM per product; the others run
 * all order + 2 products of each walker in one persistent tensor-core kernel (M <= 256 orbitals,
 * N <= 64 electrons per spin): 2 / 3 in the TF32 split with one / two walkers in flight per CTA,
 * 4 / 5 the same in the FP16 split (afqmc_ham_set_split_format; every Taylor term stored with its
 * own power-of-two scale), 6 / 7 (TF32 / FP16) one walker in flight with the running sum in
 * tensor memory.  With one walker in flight (2, 4) the small split products (hi*lo, lo*hi) get
 * their own FP32 accumulator, added to the main one (hi*hi) in the epilogue: the tensor core's
 * FP32 accumulation truncates toward zero at every update, and a third of the updates in the
 * main accumulator shrinks that bias threefold.  1 (and the default) is 2.  All compute the
 * same sums. */
int afqmc_ham_set_taylor_fused(afqmc_ham ham, int fused);
/* Which operations a mixed-precision call runs on the TF32 tensor cores (the rest in complex128):
 * AFQMC_MIXED_VBIAS the step's vbias, AFQMC_MIXED_PROPAGATION its vHS and Taylor propagation,
 * AFQMC_MIXED_ENERGY the energy's exchange / Coulomb contraction.  Default AFQMC_MIXED_ALL. */
#define AFQMC_MIXED_VBIAS 1
#define AFQMC_MIXED_PROPAGATION 2
#define AFQMC_MIXED_ENERGY 4
#define AFQMC_MIXED_ALL 7
/* Attribution only: the step's vHS on the tensor cores with the Taylor propagation in complex128
 * (without AFQMC_MIXED_PROPAGATION). */
#define AFQMC_MIXED_VHS 8
int afqmc_ham_set_mixed_ops(afqmc_ham ham, int mask);
/* Mixed-precision energy: 1 takes EJ's Coulomb vector Kl = sum_{a,k} G Lnak from a complex128
 * GEMM (one DMMA GEMM per measurement, ~4% of a 10-step block at M=200), 0 (default) from the
 * traces of the tensor-core exchange tiles. */
int afqmc_ham_set_coulomb_fp64(afqmc_ham ham, int on);

/* Error word of the tensor-core kernels' bounded device waits (bit 0: a wait on a TMA or MMA
 * completion gave up after about 2 s and the kernel returned without finishing).  0 = none, or
 * the mixed-precision path was never used.  Synchronous. */
int afqmc_ham_device_error(afqmc_ham ham, unsigned* flag);

/* Clears the error word of afqmc_ham_device_error.  Synchronous. */
int afqmc_ham_clear_device_error(afqmc_ham ham);

/* Self-test of the bounded device waits (no counterpart in the reference): one kernel waits on
 * an mbarrier that nothing arrives at, with the wait routine of the tensor-core kernels and a
 * budget of budget_cycles (at most the kernels' own, about 2 s; <= 0 selects that).  The wait
 * gives up, sets bit 0 of the Hamiltonian's error word and the kernel returns, leaving the
 * context usable.  Returns AFQMC_ERR_TIMEOUT when the wait gave up (the expected outcome).
 * Synchronous. */
int afqmc_ham_wait_selftest(afqmc_ham ham, long long budget_cycles, afqmc_stream stream);

/* getOneBodyPropagatorMatrix — Real3IndexFactorization.hpp:99-124 with add_one_body_shifts
 * (detail/one_body.hpp:65-85).  vMF host [Nc]; H1 host [nspin][M][M] = dt (h + v0) + vHS(vMF).
 * Synchronous. */
int afqmc_ham_one_body_propagator(afqmc_ham ham, double dt, const afqmc_c128* vMF,
                                  afqmc_c128* H1);

/* =========================================================================================
 * Walker set: device buffer of rows [S_alpha (M*nup) | S_beta (M*ndn) | 11 properties]
 * (WalkerSetBase.cpp:44-125).  For CLOSED walkers ndn is not stored.
 * ========================================================================================= */
typedef struct afqmc_wset_s* afqmc_wset;

int afqmc_wset_create(int walker_type, int M, int nup, int ndn, int W, afqmc_wset* out);
int afqmc_wset_destroy(afqmc_wset ws);
/* device pointer to the walker buffer and the row length in complex elements */
int afqmc_wset_buffer(afqmc_wset ws, afqmc_c128** data, long* walker_size, int* W);
/* property column <-> host [W] (WalkerSetBase.h:463-481 getProperty/setProperty); synchronous */
int afqmc_wset_get_property(afqmc_wset ws, int prop, afqmc_c128* host_out);
int afqmc_wset_set_property(afqmc_wset ws, int prop, const afqmc_c128* host_in);
/* every walker = the trial (NOMSD::initial_guess, NOMSD.cpp:131-153), weight = phase = 1 */
int afqmc_wset_init_from_trial(afqmc_wset ws, afqmc_ham ham, afqmc_stream stream);

/* =========================================================================================
 * Single-determinant NOMSD trial on a walker set (Wavefunctions/NOMSD.cpp)
 * ========================================================================================= */

/* NOMSD::MixedDensityMatrix / DensityMatrix (compact) — NOMSD.hpp:293-343:
 * G [W][nel*M], ovlp [W] (overwritten; CLOSED doubles the single-spin log overlap). */
int afqmc_wfn_density_matrix(afqmc_ham ham, afqmc_wset ws, afqmc_c128* G, afqmc_c128* ovlp,
                             afqmc_stream stream);
/* NOMSD::Log_Overlap — NOMSD.cpp:280-301 (+ log conj(ci), ci = 1). ovlp [W] overwritten. */
int afqmc_wfn_log_overlap(afqmc_ham ham, afqmc_wset ws, afqmc_c128* ovlp, afqmc_stream stream);
/* NOMSD::Energy — NOMSD.cpp:159-182: E [W][3], ovlp [W] (device, overwritten).
 * set_properties != 0 also stores OVLP, E1, EXX, EJ on the walkers (NOMSD.cpp:67-79). */
int afqmc_wfn_energy(afqmc_ham ham, afqmc_wset ws, afqmc_c128* E, afqmc_c128* ovlp,
                     int set_properties, int precision, afqmc_stream stream);
/* The OneRDM observable of the MixedEstimator (Estimators/Observables/onerdm.hpp:39-64,
 * MixedEstimator.hpp:42-108), single reference: rdm [nspin][M][M] (device, written) =
 * sum_w w_w G_w with G_w[i][k] = sum_a PsiT[a][i] Gc_w[a][k] the full mixed density matrix built
 * from the compact one G [W][ldG] of afqmc_wfn_density_matrix, w the walkers' weights; the caller
 * divides by the weight sum (as the reference's Measurements do).  No RotationMatrix. */
int afqmc_wfn_onerdm(afqmc_ham ham, afqmc_wset ws, const afqmc_c128* G, long ldG,
                     afqmc_c128* rdm, afqmc_stream stream);
/* NOMSD with several determinants (ci.size() > 1; NOMSD.cpp:93-333): one Hamiltonian handle per
 * determinant (afqmc_ham_create with that determinant's PsiT: its half-rotated Lnak / haj; the
 * handles must outlive the trial) and the coefficients ci [ndet] (host). */
typedef struct afqmc_nomsd_s* afqmc_nomsd;
int afqmc_nomsd_create(int ndet, const afqmc_ham* hams, const afqmc_c128* ci, afqmc_nomsd* out);
int afqmc_nomsd_destroy(afqmc_nomsd trial);
/* NOMSD::Log_Overlap (NOMSD.cpp:281-333): ovlp [W] (device) = log sum_d conj(c_d) ov_d,
 * summed relative to the largest determinant */
int afqmc_nomsd_log_overlap(afqmc_nomsd trial, afqmc_wset ws, afqmc_c128* ovlp,
                            afqmc_stream stream);
/* NOMSD::Energy (NOMSD.cpp:159-217): E [W][3] = sum_d conj(c_d) e^{ov_d} E_d / sum_d
 * conj(c_d) e^{ov_d}, ovlp [W] its log.  Synchronous. */
int afqmc_nomsd_energy(afqmc_nomsd trial, afqmc_wset ws, afqmc_c128* E, afqmc_c128* ovlp,
                       int precision, afqmc_stream stream);
/* NOMSD::MixedDensityMatrix, compact = false (NOMSD.cpp:220-279): G [W][nspin][M][M] (device) =
 * sum_d w_d G_d / sum_d w_d with w_d = conj(c_d) exp(ov_d - OVLP) (the walkers' OVLP property);
 * ovlp [W] = sum_d w_d + OVLP, as the reference returns it. */
int afqmc_nomsd_density_matrix(afqmc_nomsd trial, afqmc_wset ws, afqmc_c128* G,
                               afqmc_c128* ovlp, afqmc_stream stream);
/* Real3IndexFactorization::vbias on a full G (the ndet > 1 branch, hpp:389-427):
 * v [W][Nc] = sqrt(dt) (x2 CLOSED) sum_s sum_{ik} L_s[ik][n] G[w][s][ik] */
int afqmc_nomsd_vbias(afqmc_nomsd trial, const afqmc_c128* G, afqmc_c128* v, int W, double dt,
                      afqmc_stream stream);
/* NOMSD::vMF — NOMSD.cpp:437-465: vbias of the trial's own density matrix.  host [Nc]. */
int afqmc_wfn_vmf(afqmc_ham ham, double dt, afqmc_c128* vMF_host);

/* =========================================================================================
 * Propagator (AFQMCBasePropagator, hybrid force bias, dense vHS, single determinant)
 * ========================================================================================= */
typedef struct afqmc_prop_params {
  double dt;
  int taylor_n;                 /* 6 */
  double vbias_bound;           /* 50 */
  double upper_cutoff_scale;    /* 10 */
  double lower_cutoff_scale;    /* 1 */
  double weight_bound_floor;    /* 100 */
  double weight_bound_fraction; /* 0.1 */
  int denseP1;                  /* 0: P1 truncated at |x| > 1e-8 like the reference's CSR copy */
  int precision;                /* AFQMC_PREC_* */
} afqmc_prop_params;

typedef struct afqmc_prop_s* afqmc_prop;

/* Fills the reference defaults for a non-model Hamiltonian (parameters.hpp:103-131,
 * parameter_defaults.cpp:274-289). */
void afqmc_prop_params_default(afqmc_prop_params* p);

/* AFQMCBasePropagator construction + generateP1 (AFQMCBasePropagator.cpp:42-214):
 * vMF (imag zeroed), H1, hermitize, P1 = exp(-H1/2), CSR-like truncation.  Allocates the step
 * workspace for up to max_walkers walkers.  Synchronous. */
int afqmc_prop_create(afqmc_ham ham, const afqmc_prop_params* params, int max_walkers,
                      afqmc_prop* out);
int afqmc_prop_destroy(afqmc_prop prop);
/* Runs the propagator's steps with a multi-determinant trial (AFQMCBasePropagator over a
 * PHMSD wavefunction, Wavefunction.hpp's variant): vbias from afqmc_phmsd_density_matrix and
 * afqmc_phmsd_vbias, overlaps (step and orthogonalisation) from afqmc_phmsd_log_overlap.  Needs
 * COLLINEAR walkers and a trial whose Hamiltonian has been set.  With AFQMC_PREC_MIXED the vHS
 * and the Taylor propagation of both spin blocks run on the tensor cores (split precision; the
 * trial's vbias and overlaps stay complex128).  vMF (host [Nc],
 * may be NULL) replaces the mean field and regenerates P1 (generateP1 with the trial's vMF,
 * PHMSD.cpp:1329-1572, computed by the caller).  trial NULL detaches.  Synchronous.  The trial
 * must outlive its use by the propagator. */
typedef struct afqmc_phmsd_s* afqmc_phmsd;
int afqmc_prop_set_phmsd(afqmc_prop prop, afqmc_phmsd trial, const afqmc_c128* vMF);
/* The same for a NOMSD trial with several determinants (afqmc_nomsd_create): vbias from the
 * combined full density matrix (afqmc_nomsd_density_matrix / afqmc_nomsd_vbias), overlaps from
 * afqmc_nomsd_log_overlap; FP64; vMF (host [Nc], may be NULL) as for PHMSD (NOMSD::vMF for
 * several determinants, NOMSD.cpp:466-520, is the caller's). */
int afqmc_prop_set_nomsd(afqmc_prop prop, afqmc_nomsd trial, const afqmc_c128* vMF);
/* host copies: P1 [nspin][M][M], vMF [Nc] (either may be NULL) */
int afqmc_prop_get_p1(afqmc_prop prop, afqmc_c128* P1, afqmc_c128* vMF);

/* One phaseless step, AFQMCBasePropagator::Propagate (AFQMCBasePropagator.cpp:289-392):
 * vbias -> X (construct_X) -> vHS -> propagate -> Log_Overlap -> walker_update ->
 * bound_walker_weights, all on the device (the walker update is the reference's host loop,
 * restated as a kernel with the same formula).
 *   uniforms: device [W][Nc] field uniforms (the reference's RNGbuff, rng_block_size = Nc), or
 *             NULL to draw them on the device from the propagator's counter-based generator.
 * Capturable in a CUDA graph when uniforms == NULL or points to a fixed device buffer. */
int afqmc_prop_step(afqmc_prop prop, afqmc_wset ws, double Eshift, const double* uniforms,
                    afqmc_stream stream);
/* Same as afqmc_prop_step but Eshift is read from device memory at run time (graph friendly). */
int afqmc_prop_step_dev(afqmc_prop prop, afqmc_wset ws, const double* Eshift_dev,
                        const double* uniforms, afqmc_stream stream);
/* Step with explicit reuse of the density matrix between steps (Eshift from device memory).
 * AFQMC_STEP_KEEP_G: the new overlaps are computed together with the density matrix of the
 *   propagated walkers (same product, LU and log det, plus the inverse and G), kept in the
 *   propagator for the next step.
 * AFQMC_STEP_G_READY: the propagator holds the density matrix of exactly these walkers (the last
 *   step ran with KEEP_G on this walker set and nothing has changed its Slater matrices since:
 *   no orthogonalisation, population control, row copy or direct write), so the step skips
 *   recomputing it.  The caller owns this promise; results are identical to a step that
 *   recomputes G when it holds. */
#define AFQMC_STEP_G_READY 1
#define AFQMC_STEP_KEEP_G 2
int afqmc_prop_step_flags(afqmc_prop prop, afqmc_wset ws, const double* Eshift_dev,
                          const double* uniforms, int flags, afqmc_stream stream);
/* Autotuner: times the mixed-precision step on these walkers with each Taylor propagation
 * variant of afqmc_ham_set_taylor_fused (0, 2, 3, 4, 5, 6, 7) and keeps for the Hamiltonian the
 * faster of the two with separate accumulators for the small split products (2, 4); walkers,
 * field counter and bound statistics are restored, so the run continues as if it had not been
 * called.  *best = chosen mode (-1: FP64 or PHMSD,
 * nothing to tune); ms [7] (may be NULL) = the step time of variants 0, 2, 3, 4, 5, 6, 7 (0 for
 * a variant not tried: 4, 5 and 7 need the FP16 split).  Synchronous. */
int afqmc_prop_autotune(afqmc_prop prop, afqmc_wset ws, int* best, float* ms,
                        afqmc_stream stream);
/* Tile shapes and orders of the mixed-precision contractions that leave every result bit for
 * bit the same, timed on the live walkers with their state restored (no reference counterpart:
 * the reference's GEMMs are library calls): the vbias CTA tile width (128 / 64 Cholesky
 * vectors), the vHS form (i <= k pairs mirrored / all pairs) and the exchange kernel's L2 block
 * (16 / 32 / 64 / 128 vector pairs of its tile order).  choice [3] = the kept (width, symmetric,
 * block), -1 where nothing was tuned (complex128 or multi-determinant propagators); ms [8] = the
 * candidates' times in that order (ms per step, then ms per energy evaluation), may be NULL. */
int afqmc_prop_autotune_tiles(afqmc_prop prop, afqmc_wset ws, int* choice, float* ms,
                              afqmc_stream stream);
/* the same choices by hand / as they stand (defaults 128 and 64) */
int afqmc_ham_set_tiles(afqmc_ham ham, int vbias_bn, int exchange_block);
int afqmc_ham_get_tiles(afqmc_ham ham, int* vbias_bn, int* exchange_block);
/* AFQMCBasePropagator::Orthogonalize (cpp:735-741): QR re-orthonormalisation then OVLP refresh. */
int afqmc_prop_orthogonalize(afqmc_prop prop, afqmc_wset ws, afqmc_stream stream);
/* Seeds / advances the device field generator (Philox4x32-10, counter = step). */
int afqmc_prop_set_field_seed(afqmc_prop prop, unsigned long long seed);
/* Last step's intermediates, device pointers valid until the next step: vbias [W][Nc],
 * X [W][Nc], HW [W], mf [W], new_ovlp [W].  Any output may be NULL. */
int afqmc_prop_last_step(afqmc_prop prop, const afqmc_c128** vbias, const afqmc_c128** X,
                         const afqmc_c128** hw, const afqmc_c128** mf,
                         const afqmc_c128** new_ovlp);
/* Per-phase device timing of a step, the analogue of the reference's AFQMCTimers
 * (src/AFQMC/Utilities/AFQMCTimer.h:25-63): phases G_for_vbias, vbias, assemble_X, vHS,
 * propagate, pseudo_energy (overlap), extra (walker update).  afqmc_prop_timings waits for and
 * returns the milliseconds of the last step run with timing enabled. */
#define AFQMC_NPHASE 7
int afqmc_prop_set_timing(afqmc_prop prop, int enable);
int afqmc_prop_timings(afqmc_prop prop, double* ms);
/* bound statistics (AFQMCBasePropagator.h:199-237): counts[6] = eloc {total, upper, lower},
 * weight {total, upper, lower}; synchronous */
int afqmc_prop_bound_stats(afqmc_prop prop, long long* counts);

/* =========================================================================================
 * Population control and estimators (host + device)
 * ========================================================================================= */
typedef struct afqmc_host_rng_s* afqmc_host_rng;

/* split_seed (src/utilities/Random.cpp:7-20) */
unsigned long long afqmc_split_seed(int seed, int rank, unsigned stream);
/* HostRandomGenerator (src/utilities/Random.hpp:37-51): std::mt19937 + uniform_real_distribution */
int afqmc_host_rng_create(unsigned long long seed, afqmc_host_rng* out);
int afqmc_host_rng_destroy(afqmc_host_rng rng);
int afqmc_host_rng_uniform(afqmc_host_rng rng, double* out, long n);

/* ---------------------------------------------------------------------------------------
 * PHMSD (particle-hole multi-determinant) energy kernels
 * -------------------------------------------------------------------------------------- */
/* ph_excited_2body_energy_dense_cholesky (Wavefunctions/detail/phmsd_impl.hpp:33-153): for every
 * walker w and determinant d of one excitation shell (nex holes -> nex particles),
 *   EX[w] -= 1/2 wgt[d][w] eX(w,d),  EJ[w] += 1/2 wgt[d][w] (sum_n KE[d][w][n]^2 - eJ0(w)),
 * KE[d][w][n] written.  Device arrays: iexcit [ndet][2][nex] (holes = electron indices into
 * refc, then particles = active orbitals), refc [nelec], Twina [nw][nelec][nchol][nact],
 * R [nw][ndet][nex][nact], wgt [ndet][nw], EX/EJ [nw], KE [ndet][nw][nchol].  nex <= 8.
 * The excitation lists are validated on the host first (synchronous copy of iexcit, refc). */
int afqmc_ph_excited_2body_energy(const int* iexcit, const int* refc, const afqmc_c128* Twina,
                                  const afqmc_c128* R, const afqmc_c128* wgt, int nw, int ndet,
                                  int nex, int nact, int nelec, int nchol, afqmc_c128* EX,
                                  afqmc_c128* EJ, afqmc_c128* KE, afqmc_stream stream);
/* ph_excited_1body_energy (phmsd_impl.hpp:156-193): E[w] += sum_d wgt[d][w] sum_p
 * (S[w][hole_p] . R[w][d][p] + S[w][hole_p][particle_p] - S[w][hole_p][refc[hole_p]]).
 * S [nw][nelec][nact]; other layouts as above. */
int afqmc_ph_excited_1body_energy(const int* iexcit, const int* refc, const afqmc_c128* S,
                                  const afqmc_c128* R, const afqmc_c128* wgt, int nw, int ndet,
                                  int nex, int nact, int nelec, afqmc_c128* E,
                                  afqmc_stream stream);

/* PHMSD trial (Wavefunctions/PHMSD.hpp:60-120, Excitations.hpp:207-554) in explicit arrays, all
 * on the host: orbmat_s [nact_s][M] the active orbitals conjugate-transposed; refc_s [N_s] the
 * active orbital of every electron in the reference; unique excitations u = 1..nuniq_s-1 of each
 * spin (u = 0 is the reference): nex_s[u-1] holes/particles each, their lists concatenated in
 * exc_s as [holes (electron indices), particles (active orbitals)]; determinant k couples unique
 * excitations det_up[k], det_dn[k] with coupling coef[k] = conj(c_k) for the trial
 * sum_k c_k |D_k> (the reference's determinant couplings hold the conjugated CI coefficients,
 * Wavefunction.cpp:458-464), so the overlap is sum_k coef[k] <D_k|phi>.  Every index is
 * validated.
 * (afqmc_phmsd is declared with the propagator above.) */
int afqmc_phmsd_create(int M, int nup, int ndn, int nact_up, int nact_dn,
                       const afqmc_c128* orbmat_up, const afqmc_c128* orbmat_dn,
                       const int* refc_up, const int* refc_dn, int nuniq_up, const int* nex_up,
                       const int* exc_up, int nuniq_dn, const int* nex_dn, const int* exc_dn,
                       int ndet, const int* det_up, const int* det_dn, const afqmc_c128* coef,
                       afqmc_phmsd* out);
int afqmc_phmsd_destroy(afqmc_phmsd trial);
/* PHMSD::Log_Overlap (PHMSD.cpp:804-900), COLLINEAR walkers: ovlp[w] (device, written) =
 * log(sum_k c_k ov_up,k ov_dn,k) + log det of the reference blocks, with the Woodbury
 * evaluation of every excitation overlap.  wbuf: walker rows [W][ldS], S_up [M][nup] then
 * S_dn [M][ndn] at the start of each row (the walker-buffer layout). */
int afqmc_phmsd_log_overlap(afqmc_phmsd trial, const afqmc_c128* wbuf, long ldS,
                            afqmc_c128* ovlp, int W, afqmc_stream stream);

/* The particle-hole structure of one spin of a determinant expansion given as occupation lists
 * (the ph_excitations that PHMSD's factory builds, Excitations.hpp:207-554), host only:
 * occ [ndet][nel] holds each determinant's occupied active orbitals in the column order its
 * coefficient refers to; refc [nel] the reference (electron i in orbital refc[i]).  Outputs:
 * det_index [ndet] (0 = the reference, else the unique excitation), sign [ndet] (+-1: multiply the
 * coefficient by it for afqmc_phmsd_create, whose determinants replace hole h_e by particle p_e
 * in place, holes and particles ascending), *nuniq, nex [ndet] (excitation number of unique
 * excitations 1..nuniq-1) and exc [ndet * 2 * nel] (their holes then particles), ordered by
 * excitation number and first appearance. */
int afqmc_phmsd_excitations(int nact, int nel, const int* refc, int ndet, const int* occ,
                            int* det_index, double* sign, int* nuniq, int* nex, int* exc);
/* dims[6] = {M, nup, ndn, nact_up, nact_dn, Nc (0 before afqmc_phmsd_set_hamiltonian)} */
int afqmc_phmsd_info(afqmc_phmsd trial, int* dims);
/* Arithmetic of afqmc_phmsd_energy's excited-determinant 2-body terms: AFQMC_PREC_FP64 (default)
 * complex128 per-(walker, Cholesky vector) tables and per-determinant sums; AFQMC_PREC_MIXED
 * the same in complex64 (half the shared memory, the FP32 rate), the sums over determinants, the
 * reference determinant's terms and every output in complex128. */
int afqmc_phmsd_set_precision(afqmc_phmsd trial, int precision);

/* The Real3IndexFactorization tensors of a PHMSD trial: Likn [nspin_H2][M][M][Nc] (real) and
 * hij [nspin_H1][M][M] on the host, half-rotated on the device with the active orbitals
 * (the HamiltonianOperations a PHMSD wavefunction builds). */
int afqmc_phmsd_set_hamiltonian(afqmc_phmsd trial, const double* Likn, int nspin_H2,
                                const afqmc_c128* hij, int nspin_H1, int Nc, double E0);
/* PHMSD::energy_alg1 (PHMSD.cpp:376-546), COLLINEAR walkers: E [W][3] (E1, EXX, EJ, device,
 * written) and the log overlap [W] (device, written) of the multi-determinant trial, by the
 * Woodbury evaluation of every excited determinant.  Walkers are processed in blocks of `block`
 * (<= 0: 64); the excitation lists must be ordered by excitation number. */
int afqmc_phmsd_energy(afqmc_phmsd trial, const afqmc_c128* wbuf, long ldS, afqmc_c128* E,
                       afqmc_c128* ovlp, int W, int block, afqmc_stream stream);
/* PHMSD::MixedDensityMatrix, compact COLLINEAR (PHMSD.cpp:684-795): G [W][nact_up +
 * nact_dn][M] (device, written) = (R_s^T G_s^ref) / Ov per spin block, with R the coefficient-
 * weighted Woodbury matrices of every excited determinant (calculate_R,
 * phmsd_helpers.hpp:200-309); ovlp [W] (device, written) the log overlap.  Blocks of `block`
 * walkers (<= 0: 512). */
int afqmc_phmsd_density_matrix(afqmc_phmsd trial, const afqmc_c128* wbuf, long ldS,
                               afqmc_c128* G, afqmc_c128* ovlp, int W, int block,
                               afqmc_stream stream);
/* PHMSD::vbias (PHMSD.cpp:54-72) over Real3IndexFactorization::vbias
 * (Real3IndexFactorization.hpp:328-384): v [W][Nc] (device, written) = sqrt(dt) sum_s Lnak_s . G_s
 * with G from afqmc_phmsd_density_matrix and the active-space Lnak of
 * afqmc_phmsd_set_hamiltonian. */
int afqmc_phmsd_vbias(afqmc_phmsd trial, const afqmc_c128* G, afqmc_c128* v, int W, double dt,
                      afqmc_stream stream);

/* comb (population_control.hpp:34-65): host arrays; draws one uniform from rng. */
int afqmc_comb(afqmc_host_rng rng, const double* weights, int n, int num_target, int* offspring);
/* plan_walker_exchange (population_control.hpp:87-133): pure host logic. plan holds up to
 * max_plan entries of {src, walker, dst, copies}; *nplan receives the count. */
int afqmc_plan_walker_exchange(const int* offspring, const int* counts, int nranks, int* plan,
                               int max_plan, int* nplan);
/* population_control on one rank (population_control.hpp:218-255): |w| to host, comb, row
 * copies on the device in the reference's slot order, weights <- w/|w|.  Synchronous.
 * offspring (host [W]) may be NULL. */
int afqmc_population_control(afqmc_wset ws, afqmc_host_rng rng, int* offspring,
                             afqmc_stream stream);
/* Row gather: dst row j <- src row src_index[j] (device int array) for j in [0, n); rows of
 * walker_size elements.  Building block for the multi-rank exchange. */
int afqmc_wset_copy_rows(afqmc_wset ws, const int* dst_slots, const int* src_slots, int n,
                         afqmc_stream stream);
/* pack rows idx[0..n) into buf [n][walker_size] / unpack buf rows into slots idx (device) */
int afqmc_wset_pack_rows(afqmc_wset ws, const int* idx, int n, afqmc_c128* buf,
                         afqmc_stream stream);
int afqmc_wset_unpack_rows(afqmc_wset ws, const int* idx, int n, const afqmc_c128* buf,
                           afqmc_stream stream);
/* weights <- w/|w| for all walkers (end of population_control) */
int afqmc_wset_normalize_weights(afqmc_wset ws, afqmc_stream stream);

/* EnergyEstimator::measure sums (EnergyEstimator.h:51-100): out4 (device) =
 * {sum_w w E1, sum_w w EXX, sum_w w EJ, sum_w w} */
int afqmc_energy_sums(afqmc_wset ws, const afqmc_c128* E, afqmc_c128* out4, afqmc_stream stream);
/* averagePseudoEnergy numerator/denominator (Drivers/average_energy.hpp:53-63): out2 (device) =
 * {sum w exp(dt*eloc), sum w} */
int afqmc_pseudo_energy_sums(afqmc_wset ws, double dt, afqmc_c128* out2, afqmc_stream stream);

/* =========================================================================================
 * Learned exchange-energy control variate (no reference counterpart; the exact exchange of
 * afqmc_ham_energy stays the reference value).  An MLP features (D) -> H -> H -> 1 with GELU, trained and
 * evaluated by BF16 tensor-core kernels with FP32 accumulation, FP32 master weights and Adam.
 * Parameters are one FP32 block [W1 (H x D) | b1 (H) | W2 (H x H) | b2 (H) | w3 (H) | b3 (1)],
 * row-major (out x in).  Features and targets are device FP32; targets in physical units, the
 * network works on standardised features and targets (afqmc_mlp_set_normalization).
 * ========================================================================================= */
typedef struct afqmc_mlp_s* afqmc_mlp;
/* D even, H a multiple of 8; uniform He initialisation from `seed` (host) */
int afqmc_mlp_create(int D, int H, unsigned long long seed, afqmc_mlp* out);
int afqmc_mlp_destroy(afqmc_mlp mlp);
long afqmc_mlp_num_params(afqmc_mlp mlp);
/* host arrays: mean, istd [D]; the target's mean and standard deviation */
int afqmc_mlp_set_normalization(afqmc_mlp mlp, const float* mean, const float* istd,
                                float y_mean, float y_std);
/* which = 0: parameters (read or write), 1: gradients of the last afqmc_mlp_gradients /
 * afqmc_mlp_train_step (read); host FP32 [afqmc_mlp_num_params].  Synchronous. */
int afqmc_mlp_params(afqmc_mlp mlp, int which, float* host, int to_device);
/* y [B] (device) = prediction for features X [B][D] (device) */
int afqmc_mlp_predict(afqmc_mlp mlp, const float* X, int B, float* y, afqmc_stream stream);
/* forward + backward of the Huber loss (threshold 2: r^2 / 2 inside, 2 (|r| - 1) outside, r =
 * y - t) averaged over the batch in standardised units for X [B][D], t [B]; gradients kept in the
 * handle; loss (device float, may be NULL) */
int afqmc_mlp_gradients(afqmc_mlp mlp, const float* X, const float* t, int B, float* loss,
                        afqmc_stream stream);
/* afqmc_mlp_gradients followed by one Adam step (beta 0.9 / 0.999, eps 1e-8) */
int afqmc_mlp_train_step(afqmc_mlp mlp, const float* X, const float* t, int B, float lr,
                         float* loss, afqmc_stream stream);
/* features of W walkers: X [W][D] = [Re vbias, Im vbias, Re G[a][a], Im G[a][a] (a < N)] from
 * vbias [W][ldv] and the compact density matrix G [W][ldG] ([N][M] per spin block), D = 2 Nc +
 * 2 N; with E [W][3] (E1, EXX, EJ; may be NULL) also Re E1, Im E1, Re EJ, Im EJ (D + 4) */
int afqmc_exchange_features(const afqmc_c128* vbias, long ldv, const afqmc_c128* G, long ldG,
                            int N, int M, int Nc, int W, const afqmc_c128* E, float* X,
                            afqmc_stream stream);

#ifdef __cplusplus
}
#endif

#endif /* AFQMC_C_H */
