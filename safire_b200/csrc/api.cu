// C ABI of the walker step (include/afqmc_c.h): handles for the Hamiltonian operations, the walker
// set and the propagator, and the extern "C" entry points that sequence the kernels.
#include <algorithm>
#include <atomic>
#include <complex>
#include <numeric>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <random>
#include <string>
#include <vector>

#include "common.cuh"
#include "detops.cuh"
#include "energy.cuh"
#include "fields.cuh"
#include "mixed.cuh"
#include "update.cuh"
#include "thc.cuh"
#include "zgemm.cuh"

namespace afqmc {

static thread_local std::string g_err;

void set_error_detail(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
}
const char* error_detail() { return g_err.c_str(); }

static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

using cplx = std::complex<double>;

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

template <class T>
int dalloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) return AFQMC_OK;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
  if (e != cudaSuccess) {
    set_error_detail("cudaMalloc of %zu bytes failed: %s", n * sizeof(T), cudaGetErrorString(e));
    return AFQMC_ERR_ALLOC;
  }
  return AFQMC_OK;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}


}  // namespace
}  // namespace afqmc

using namespace afqmc;

// ---------------------------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------------------------
struct afqmc_ham_s {
  int device = 0;
  int walker_type = AFQMC_CLOSED, M = 0, nup = 0, ndn = 0, Nc = 0;
  int nspin = 1, nspin_H2 = 1, nspin_H1 = 1;
  int nel[2] = {0, 0}, el_off[2] = {0, 0}, nel_tot = 0;
  double E0 = 0;
  bool trial_real = false;
  bool coulomb_fp64 = false;  // mixed precision: EJ's Coulomb vector from a complex128 GEMM
  int mixed_ops = AFQMC_MIXED_ALL;  // which operations a mixed-precision call runs on TF32
  double* Likn = nullptr;               // [nspin_H2][M][M][Nc]
  c128* Lnak[2] = {nullptr, nullptr};   // [Nc][nel_s][M]
  double* Lnak_r[2] = {nullptr, nullptr};
  c128* haj = nullptr;                  // [nel_tot][M]
  c128* PsiT = nullptr;                 // [nel_tot][M]
  c128* PsiH = nullptr;                 // [M][nel_s] per spin, concatenated (initial walker)
  std::vector<c128> hij_h;              // [nspin_H1][M][M]
  std::vector<double> vexx_h;           // [nspin_H2][M][M]
  MixedHam* mixed = nullptr;            // tensor-core copies (built on first mixed call)
  ThcData* thc = nullptr;               // THC factorisation instead of Likn (afqmc_ham_create_thc)
  ~afqmc_ham_s() {
    DeviceGuard g(device);
    if (thc) thc_destroy(thc);
    dfree(Likn);
    for (int s = 0; s < 2; ++s) {
      dfree(Lnak[s]);
      dfree(Lnak_r[s]);
    }
    dfree(haj);
    dfree(PsiT);
    dfree(PsiH);
    if (mixed) mixed_ham_destroy(mixed);
  }
};

struct afqmc_wset_s {
  int device = 0;
  int walker_type = AFQMC_CLOSED, M = 0, nup = 0, ndn = 0, W = 0;
  long walker_size = 0, prop0 = 0;
  c128* buf = nullptr;
  ~afqmc_wset_s() {
    DeviceGuard g(device);
    dfree(buf);
  }
  long offS(int spin) const { return spin == 0 ? 0 : long(M) * nup; }
};

struct afqmc_prop_s {
  int device = 0;
  afqmc_ham_s* ham = nullptr;
  afqmc_prop_params p{};
  int maxW = 0;
  bool p1_real = false;
  int nspin_P1 = 1, nspin_V = 1;
  c128* P1 = nullptr;        // [nspin][M][M]
  double* P1r = nullptr;     // real copy when real
  c128* vMF = nullptr;       // [Nc]
  std::vector<c128> P1_h, vMF_h;
  double mf0 = 0;            // -Re(vMF.vMF)/2
  // step workspace
  c128 *G = nullptr, *vb = nullptr, *X = nullptr, *HW = nullptr, *mf = nullptr;
  c128 *newov = nullptr, *ovtmp = nullptr, *T = nullptr, *V = nullptr;
  c128 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
  c128* ortho_work = nullptr;
  double* Eshift_d = nullptr;
  unsigned long long* counter = nullptr;
  unsigned long long* stats = nullptr;
  unsigned long long seed = 0x5AF1E5EEDull;
  // multi-determinant trial used in place of the Hamiltonian's single determinant
  afqmc_phmsd ph = nullptr;
  c128* Gph = nullptr;       // [maxW][nact_up + nact_dn][M]
  afqmc_nomsd md = nullptr;  // several-determinant NOMSD trial
  c128* Gfull = nullptr;     // [maxW][nspin][M][M]
  // per-phase CUDA events of the last timed step (AFQMCTimers analogue)
  bool timing = false;
  cudaEvent_t ev[AFQMC_NPHASE + 1] = {};
  ~afqmc_prop_s() {
    DeviceGuard g(device);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    dfree(P1); dfree(P1r); dfree(vMF);
    dfree(G); dfree(vb); dfree(X); dfree(HW); dfree(mf); dfree(newov); dfree(ovtmp);
    dfree(T); dfree(V); dfree(w1); dfree(w2); dfree(w3); dfree(ortho_work);
    dfree(Eshift_d); dfree(counter); dfree(stats); dfree(Gph); dfree(Gfull);
  }
};

struct afqmc_host_rng_s {
  std::mt19937 rng;
};

// NOMSD with several determinants (NOMSD.hpp / NOMSD.cpp, ci.size() > 1): one Hamiltonian
// handle per determinant (its half-rotated tensors), the coefficients ci.
// The propagation step batches over the determinants: PsiTall holds every determinant's
// PsiT stacked per spin ([nd][N_s][M] at nd * el_off[s] * M), so one GEMM per walker forms the
// overlap matrices of all determinants, one Gauss-Jordan launch inverts them, and one GEMM
// with K = nd * N_s sums the weighted full density matrices.  Walkers go in chunks of wchunk
// (the batched launches' grid limit and a bounded workspace): Tb and Ttb
// [wchunk][nd][N_s][N_s] and Gcb [wchunk][nd][N_s][M] per spin, ovd / wdd [wchunk][nd].
struct afqmc_nomsd_s {
  int device = 0;
  std::vector<afqmc_ham_s*> hams;
  std::vector<c128> ci;
  c128 *PsiTall = nullptr, *dcc = nullptr, *dlc = nullptr;  // conj(ci), log conj(ci)
  c128 *Gc = nullptr, *ov = nullptr, *T = nullptr, *Ed = nullptr;  // energy (per determinant)
  c128 *Tb = nullptr, *Ttb = nullptr, *Gcb = nullptr, *ovd = nullptr, *wdd = nullptr;
  int capW = 0, wchunk = 0;
  void free_bufs() {
    dfree(Gc); dfree(ov); dfree(T); dfree(Ed);
    dfree(Tb); dfree(Ttb); dfree(Gcb); dfree(ovd); dfree(wdd);
    capW = 0;
    wchunk = 0;
  }
  ~afqmc_nomsd_s() {
    DeviceGuard g(device);
    free_bufs();
    dfree(PsiTall); dfree(dcc); dfree(dlc);
  }
};

// ---------------------------------------------------------------------------------------------
// status
// ---------------------------------------------------------------------------------------------
extern "C" const char* afqmc_status_string(int status) {
  switch (status) {
    case AFQMC_OK: return "ok";
    case AFQMC_ERR_ARG: return "invalid argument";
    case AFQMC_ERR_SHAPE: return "shape mismatch";
    case AFQMC_ERR_CUDA: return "CUDA error";
    case AFQMC_ERR_NONFINITE: return "non-finite value";
    case AFQMC_ERR_TIMEOUT: return "device wait timed out";
    case AFQMC_ERR_ALLOC: return "allocation failed";
    case AFQMC_ERR_UNSUPPORTED: return "unsupported configuration";
    case AFQMC_ERR_COLLAPSE: return "total walker weight collapsed";
    default: return "unknown status";
  }
}
extern "C" const char* afqmc_last_error(void) { return error_detail(); }
extern "C" int afqmc_version(void) { return 1; }
extern "C" unsigned long long afqmc_kernel_launches(void) { return g_launches.load(); }

// ---------------------------------------------------------------------------------------------
// det_ops
// ---------------------------------------------------------------------------------------------
namespace {
// Scratch of the stream-ordered allocator.  The device's default pool keeps freed blocks for reuse
// (release threshold raised once per device), so repeated calls do not map and unmap memory.
void retain_pool_memory() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  std::lock_guard<std::mutex> lock(mu);
  if (done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  done[dev] = true;
}

struct Scratch {
  void* p = nullptr;
  cudaStream_t s = nullptr;
  ~Scratch() {
    if (p) cudaFreeAsync(p, s);
  }
  int get(size_t bytes, cudaStream_t st) {
    s = st;
    if (bytes == 0) return AFQMC_OK;
    retain_pool_memory();
    cudaError_t e = cudaMallocAsync(&p, bytes, st);
    if (e != cudaSuccess) {
      set_error_detail("cudaMallocAsync(%zu) failed: %s", bytes, cudaGetErrorString(e));
      p = nullptr;
      return AFQMC_ERR_ALLOC;
    }
    return AFQMC_OK;
  }
};
}  // namespace

extern "C" int afqmc_log_overlap(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS,
                                 afqmc_c128* ovlp, int W, int M, int N, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0, "afqmc_log_overlap: negative size");
  if (W == 0 || N == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(PsiT && S && ovlp, "afqmc_log_overlap: null pointer");
  AFQMC_CHECK_ARG(ldS >= long(M) * N, "afqmc_log_overlap: ldS < M*N");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Scratch T;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(W) * N * N, s));
  return log_overlap(s, (const c128*)PsiT, (const c128*)S, ldS, (c128*)ovlp, W, M, N,
                     (c128*)T.p, cmk(1, 0), cmk(0, 0));
}

extern "C" int afqmc_mixed_density_matrix(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS,
                                          afqmc_c128* G, long ldG, afqmc_c128* ovlp, int W, int M,
                                          int N, int compact, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0, "afqmc_mixed_density_matrix: negative size");
  if (W == 0) return AFQMC_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long gsize = compact ? long(N) * M : long(M) * M;
  AFQMC_CHECK_ARG(G && ovlp && (N == 0 || (PsiT && S)), "afqmc_mixed_density_matrix: null pointer");
  AFQMC_CHECK_ARG(ldG >= gsize, "afqmc_mixed_density_matrix: ldG too small");
  if (N == 0) {
    // empty sector: overlap factor 1, density matrix zero (density_matrix.hpp:561-567)
    if (!compact && gsize > 0)
      AFQMC_CUDA_TRY(cudaMemset2DAsync(G, ldG * sizeof(c128), 0, gsize * sizeof(c128), W, s));
    return AFQMC_OK;
  }
  AFQMC_CHECK_ARG(ldS >= long(M) * N, "afqmc_mixed_density_matrix: ldS < M*N");
  Scratch T, NMw;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(W) * N * N, s));
  if (!compact) AFQMC_TRY(NMw.get(sizeof(c128) * size_t(W) * N * M, s));
  return mixed_density_matrix(s, (const c128*)PsiT, (const c128*)S, ldS, (c128*)G, ldG,
                              (c128*)ovlp, W, M, N, compact != 0, (c128*)T.p, (c128*)NMw.p,
                              cmk(1, 0), cmk(0, 0));
}

extern "C" int afqmc_mixed_density_matrix_batched(const afqmc_c128* A, long ldA,
                                                  const afqmc_c128* S, long ldS, afqmc_c128* G,
                                                  long ldG, afqmc_c128* ovlp, int W, int M, int N,
                                                  int compact, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0, "afqmc_mixed_density_matrix_batched: negative size");
  if (W == 0) return AFQMC_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const long gsize = compact ? long(N) * M : long(M) * M;
  AFQMC_CHECK_ARG(G && ovlp && (N == 0 || (A && S)),
                  "afqmc_mixed_density_matrix_batched: null pointer");
  AFQMC_CHECK_ARG(ldG >= gsize, "afqmc_mixed_density_matrix_batched: ldG too small");
  if (N == 0) {
    if (!compact && gsize > 0)
      AFQMC_CUDA_TRY(cudaMemset2DAsync(G, ldG * sizeof(c128), 0, gsize * sizeof(c128), W, s));
    return AFQMC_OK;
  }
  AFQMC_CHECK_ARG(ldA >= long(M) * N && ldS >= long(M) * N,
                  "afqmc_mixed_density_matrix_batched: ldA or ldS < M*N");
  const long NN = long(N) * N;
  Scratch T, Ti, NMw;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(W) * NN, s));
  AFQMC_TRY(Ti.get(sizeof(c128) * size_t(W) * NN, s));
  if (!compact) AFQMC_TRY(NMw.get(sizeof(c128) * size_t(W) * N * M, s));
  // T_w = A_w^H S_w  (N x N)
  GemmParams p{};
  p.m = N; p.n = N; p.k = M;
  p.A = A; p.lda = N; p.strideA = ldA;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = (c128*)T.p; p.ldc = N; p.strideC = NN;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, W, GH, false, GN, false, p));
  // T_w^{-1} and ovlp[w] += log det T_w
  AFQMC_TRY(batched_logdet_inverse(s, (const c128*)T.p, NN, (c128*)Ti.p, NN, (c128*)ovlp, W, N,
                                   true, cmk(1, 0), cmk(0, 0)));
  if (compact) {
    // G_w = T_w^{-T} S_w^T  (N x M)
    p = GemmParams{};
    p.m = N; p.n = M; p.k = N;
    p.A = Ti.p; p.lda = N; p.strideA = NN;
    p.B = S; p.ldb = N; p.strideB = ldS;
    p.C = (c128*)G; p.ldc = M; p.strideC = ldG;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    return zgemm(s, W, GT, false, GT, false, p);
  }
  // X_w = T_w^{-1} A_w^H (N x M); G_w = X_w^T S_w^T = (S_w T_w^{-1} A_w^H)^T  (M x M)
  p = GemmParams{};
  p.m = N; p.n = M; p.k = N;
  p.A = Ti.p; p.lda = N; p.strideA = NN;
  p.B = A; p.ldb = N; p.strideB = ldA;
  p.C = (c128*)NMw.p; p.ldc = M; p.strideC = long(N) * M;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  AFQMC_TRY(zgemm(s, W, GN, false, GH, false, p));
  p = GemmParams{};
  p.m = M; p.n = M; p.k = N;
  p.A = NMw.p; p.lda = M; p.strideA = long(N) * M;
  p.B = S; p.ldb = N; p.strideB = ldS;
  p.C = (c128*)G; p.ldc = M; p.strideC = ldG;
  p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
  return zgemm(s, W, GT, false, GT, false, p);
}

extern "C" int afqmc_inverse_logdet(const afqmc_c128* A, afqmc_c128* Ainv, afqmc_c128* logdet,
                                    int W, int N, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && N >= 0, "afqmc_inverse_logdet: negative size");
  if (W == 0 || N == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(A && Ainv && logdet, "afqmc_inverse_logdet: null pointer");
  return batched_logdet_inverse(reinterpret_cast<cudaStream_t>(stream), (const c128*)A,
                                long(N) * N, (c128*)Ainv, long(N) * N, (c128*)logdet, W, N, true,
                                cmk(1, 0), cmk(0, 0));
}

extern "C" int afqmc_orthogonalize(afqmc_c128* S, long ldS, afqmc_c128* logdetR, int W, int M,
                                   int N, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0, "afqmc_orthogonalize: negative size");
  if (W == 0 || N == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(S && logdetR, "afqmc_orthogonalize: null pointer");
  AFQMC_CHECK_ARG(ldS >= long(M) * N, "afqmc_orthogonalize: ldS < M*N");
  return orthogonalize(reinterpret_cast<cudaStream_t>(stream), (c128*)S, ldS, (c128*)logdetR, W,
                       M, N);
}

extern "C" int afqmc_propagate(const afqmc_c128* P1, const afqmc_c128* V, afqmc_c128* S,
                               long ldS, int W, int M, int N, int order, afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0 && order >= 0, "afqmc_propagate: negative size");
  if (W == 0 || N == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(P1 && V && S, "afqmc_propagate: null pointer");
  AFQMC_CHECK_ARG(ldS >= long(M) * N, "afqmc_propagate: ldS < M*N");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  Scratch w;
  const size_t one = size_t(W) * M * N;
  AFQMC_TRY(w.get(sizeof(c128) * one * 3, s));
  c128* b = (c128*)w.p;
  return propagate(s, P1, false, (const c128*)V, long(M) * M, (c128*)S, ldS, W, M, N, order, b,
                   b + one, b + 2 * one);
}

// ---------------------------------------------------------------------------------------------
// Hamiltonian operations
// ---------------------------------------------------------------------------------------------
namespace api_kernels {

__global__ void lnak_reorder_kernel(const c128* __restrict__ in, c128* __restrict__ out,
                                    double* __restrict__ out_r, int Ns, int M, int Nc) {
  // in [a][k][n] (row a of PsiT * L viewed as M x (M*Nc)), out [n][a][k]
  long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  long total = long(Ns) * M * Nc;
  if (e >= total) return;
  int n = int(e % Nc);
  long r = e / Nc;
  int k = int(r % M);
  int a = int(r / M);
  c128 v = in[e];
  long o = (long(n) * Ns + a) * M + k;
  out[o] = v;
  if (out_r) out_r[o] = v.x;
}

}  // namespace api_kernels

namespace {

int ham_vbias(afqmc_ham_s* h, cudaStream_t s, const c128* G, long ldG, c128* v, int W, double dt) {
  if (h->thc) return thc_vbias(s, h->thc, G, ldG, v, W, dt, h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0);
  const double a = std::sqrt(dt) * (h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0);
  bool first = true;
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    if (Ns == 0) continue;
    GemmParams p{};
    p.m = W; p.n = h->Nc; p.k = Ns * h->M;
    p.A = G + long(h->el_off[sp]) * h->M; p.lda = ldG; p.strideA = 0;
    p.B = h->trial_real ? (const void*)h->Lnak_r[sp] : (const void*)h->Lnak[sp];
    p.ldb = long(Ns) * h->M; p.strideB = 0;
    p.C = v; p.ldc = h->Nc; p.strideC = 0;
    p.alpha = cmk(a, 0); p.beta = first ? cmk(0, 0) : cmk(1, 0);
    AFQMC_TRY(zgemm(s, 1, GN, false, GT, h->trial_real, p));
    first = false;
  }
  if (first) AFQMC_CUDA_TRY(cudaMemsetAsync(v, 0, sizeof(c128) * size_t(W) * h->Nc, s));
  return AFQMC_OK;
}

int ham_vhs(afqmc_ham_s* h, cudaStream_t s, const c128* X, c128* V, int W, double dt) {
  if (h->thc) return thc_vhs(s, h->thc, X, V, W, dt);
  const int nst = h->walker_type == AFQMC_COLLINEAR ? h->nspin_H2 : 1;
  const long MM = long(h->M) * h->M;
  for (int is = 0; is < nst; ++is) {
    GemmParams p{};
    p.m = W; p.n = int(MM); p.k = h->Nc;
    p.A = X; p.lda = h->Nc; p.strideA = 0;
    p.B = h->Likn + size_t(is % h->nspin_H2) * MM * h->Nc; p.ldb = h->Nc; p.strideB = 0;
    p.C = V + size_t(is) * W * MM; p.ldc = MM; p.strideC = 0;
    p.alpha = cmk(std::sqrt(dt), 0); p.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, 1, GN, false, GT, true, p));
  }
  return AFQMC_OK;
}

EnergyArgs energy_args(afqmc_ham_s* h, const c128* G, long ldG) {
  EnergyArgs a{};
  a.G = G; a.ldG = ldG; a.M = h->M; a.Nc = h->Nc; a.nspin = h->nspin;
  for (int s = 0; s < 2; ++s) {
    a.nel[s] = h->nel[s];
    a.el_off[s] = h->el_off[s];
    a.Lnak[s] = h->Lnak[s];
    a.Lnak_real[s] = h->trial_real ? h->Lnak_r[s] : nullptr;
  }
  a.haj = h->haj;
  a.E0 = h->E0;
  a.scl = h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0;
  a.sclj = h->walker_type == AFQMC_CLOSED ? 4.0 : 1.0;
  a.Likn = h->Likn;
  a.nspin_H2 = h->nspin_H2;
  a.coulomb_fp64 = h->coulomb_fp64;
  return a;
}

// exchange-tensor chunk budget (complex elements): 256 MiB, at least one walker
long energy_chunk_elems(afqmc_ham_s* h, int W) {
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  long per = long(nmax) * h->Nc * nmax;
  long budget = (256l << 20) / long(sizeof(c128));
  long nw = budget / (per > 0 ? per : 1);
  if (nw < 1) nw = 1;
  if (nw > W) nw = W;
  return nw * per;
}

int ham_energy(afqmc_ham_s* h, cudaStream_t s, const c128* G, long ldG, c128* E, int W, bool addH1,
               bool addEJ, bool addEXX, int precision) {
  if (h->thc) {
    if (precision == AFQMC_PREC_MIXED) {
      set_error_detail("THC Hamiltonian: complex128 only (no mixed-precision path)");
      return AFQMC_ERR_UNSUPPORTED;
    }
    const double scl = h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0;
    return thc_energy(s, h->thc, G, ldG, h->haj, h->E0, scl, scl * scl, E, W, addH1, addEJ,
                      addEXX);
  }
  EnergyArgs a = energy_args(h, G, ldG);
  MixedHam* tc = nullptr;
  if (precision == AFQMC_PREC_MIXED && (h->mixed_ops & AFQMC_MIXED_ENERGY)) {
    if (!h->mixed) AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    tc = h->mixed;
    AFQMC_TRY(mixed_prepare_G(s, tc, G, ldG, W));
  }
  Scratch wT, ex, kl;
  bool fused = tc != nullptr;
  for (int sp = 0; sp < h->nspin && fused; ++sp)
    if (h->nel[sp] > 0 && !exchange_fused_ok(tc, sp)) fused = false;
  const long chunk = fused ? 0 : energy_chunk_elems(h, W);
  if (!fused) AFQMC_TRY(wT.get(sizeof(c128) * size_t(chunk), s));
  AFQMC_TRY(ex.get(sizeof(c128) * size_t(W) * h->Nc, s));
  AFQMC_TRY(kl.get(sizeof(c128) * size_t(W) * h->Nc, s));
  return energy_fp64(s, a, E, W, addH1, addEJ, addEXX, (c128*)wT.p, chunk, (c128*)ex.p,
                     (c128*)kl.p, tc);
}

}  // namespace

namespace {

// the trial-dependent part of a Hamiltonian handle: PsiT, PsiH (the initial walker), haj
int ham_trial_setup(afqmc_ham_s* h, const afqmc_c128* hij, int nspin_H1, const c128* psi) {
  const int M = h->M;
  const long MM = long(M) * M;
  bool real = true;
  for (long e = 0; e < long(h->nel_tot) * M; ++e) real = real && psi[e].y == 0.0;
  h->trial_real = real;
  cudaStream_t s = nullptr;
  AFQMC_TRY(dalloc(&h->PsiT, size_t(h->nel_tot) * M));
  if (h->nel_tot)
    AFQMC_CUDA_TRY(cudaMemcpy(h->PsiT, psi, sizeof(c128) * h->nel_tot * M, cudaMemcpyHostToDevice));
  // PsiH: per spin [M][nel_s] = conj(PsiT_s)^T, concatenated spin blocks
  {
    std::vector<c128> ph(size_t(h->nel_tot) * M);
    long off = 0;
    for (int sp = 0; sp < h->nspin; ++sp) {
      const int Ns = h->nel[sp];
      for (int i = 0; i < M; ++i)
        for (int a = 0; a < Ns; ++a) {
          c128 v = psi[long(h->el_off[sp] + a) * M + i];
          ph[off + long(i) * Ns + a] = cmk(v.x, -v.y);
        }
      off += long(M) * Ns;
    }
    AFQMC_TRY(dalloc(&h->PsiH, ph.size()));
    if (!ph.empty())
      AFQMC_CUDA_TRY(cudaMemcpy(h->PsiH, ph.data(), sizeof(c128) * ph.size(), cudaMemcpyHostToDevice));
  }
  // haj = PsiT_s * h_s
  c128* hij_d = nullptr;
  AFQMC_TRY(dalloc(&hij_d, size_t(nspin_H1) * MM));
  AFQMC_CUDA_TRY(cudaMemcpy(hij_d, hij, sizeof(c128) * nspin_H1 * MM, cudaMemcpyHostToDevice));
  AFQMC_TRY(dalloc(&h->haj, size_t(h->nel_tot) * M));
  for (int sp = 0; sp < h->nspin; ++sp) {
    if (h->nel[sp] == 0) continue;
    GemmParams p{};
    p.m = h->nel[sp]; p.n = M; p.k = M;
    p.A = h->PsiT + long(h->el_off[sp]) * M; p.lda = M;
    p.B = hij_d + (sp % nspin_H1) * MM; p.ldb = M;
    p.C = h->haj + long(h->el_off[sp]) * M; p.ldc = M;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    int st = zgemm(s, 1, GN, false, GN, false, p);
    if (st) { dfree(hij_d); return st; }
  }
  dfree(hij_d);
  return AFQMC_OK;
}
}  // namespace

extern "C" int afqmc_ham_create(int walker_type, int M, int nup, int ndn, int Nc,
                                const double* Likn, int nspin_H2, const afqmc_c128* hij,
                                int nspin_H1, double E0, const afqmc_c128* PsiT,
                                afqmc_ham* out) {
  AFQMC_CHECK_ARG(out, "afqmc_ham_create: null out");
  *out = nullptr;
  AFQMC_CHECK_ARG(walker_type == AFQMC_CLOSED || walker_type == AFQMC_COLLINEAR,
                  "afqmc_ham_create: walker_type must be CLOSED (1) or COLLINEAR (2)");
  AFQMC_CHECK_ARG(M > 0 && Nc > 0 && nup >= 0 && ndn >= 0, "afqmc_ham_create: bad sizes");
  AFQMC_CHECK_ARG(nup <= M && ndn <= M, "afqmc_ham_create: more electrons than orbitals");
  AFQMC_CHECK_ARG(Likn && hij && PsiT, "afqmc_ham_create: null input");
  AFQMC_CHECK_ARG(nspin_H2 == 1 || nspin_H2 == 2, "afqmc_ham_create: nspin_H2 must be 1 or 2");
  AFQMC_CHECK_ARG(nspin_H1 == 1 || nspin_H1 == 2, "afqmc_ham_create: nspin_H1 must be 1 or 2");
  if (walker_type == AFQMC_CLOSED) {
    AFQMC_CHECK_ARG(nspin_H2 == 1 && nspin_H1 == 1,
                    "afqmc_ham_create: CLOSED walkers take a spin-independent Hamiltonian");
  }
  std::unique_ptr<afqmc_ham_s> h(new (std::nothrow) afqmc_ham_s());
  AFQMC_CHECK_ARG(h, "afqmc_ham_create: out of host memory");
  cudaGetDevice(&h->device);
  h->walker_type = walker_type;
  h->M = M; h->nup = nup; h->ndn = ndn; h->Nc = Nc;
  h->nspin = walker_type == AFQMC_COLLINEAR ? 2 : 1;
  h->nspin_H2 = nspin_H2; h->nspin_H1 = nspin_H1;
  h->nel[0] = nup;
  h->nel[1] = walker_type == AFQMC_COLLINEAR ? ndn : 0;
  h->el_off[0] = 0;
  h->el_off[1] = nup;
  h->nel_tot = h->nel[0] + h->nel[1];
  h->E0 = E0;
  const long MM = long(M) * M;
  h->hij_h.assign((const c128*)hij, (const c128*)hij + nspin_H1 * MM);
  const c128* psi = (const c128*)PsiT;

  cudaStream_t s = nullptr;
  AFQMC_TRY(dalloc(&h->Likn, size_t(nspin_H2) * MM * Nc));
  AFQMC_CUDA_TRY(cudaMemcpy(h->Likn, Likn, sizeof(double) * nspin_H2 * MM * Nc,
                            cudaMemcpyHostToDevice));
  AFQMC_TRY(ham_trial_setup(h.get(), hij, nspin_H1, psi));
  const bool real = h->trial_real;
  // Lnak_s[n][a][k] = sum_i PsiT_s[a][i] L_s[i][k][n]: one GEMM PsiT_s (N x M) * L_s (M x M*Nc)
  // into [a][k][n], then a reorder to [n][a][k]
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    if (Ns == 0) continue;
    c128* tmp = nullptr;
    AFQMC_TRY(dalloc(&tmp, size_t(Ns) * M * Nc));
    AFQMC_TRY(dalloc(&h->Lnak[sp], size_t(Ns) * M * Nc));
    if (real) AFQMC_TRY(dalloc(&h->Lnak_r[sp], size_t(Ns) * M * Nc));
    GemmParams p{};
    p.m = Ns; p.n = int(long(M) * Nc); p.k = M;
    p.A = h->PsiT + long(h->el_off[sp]) * M; p.lda = M;
    p.B = h->Likn + size_t(sp % nspin_H2) * MM * Nc; p.ldb = long(M) * Nc;
    p.C = tmp; p.ldc = long(M) * Nc;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    int st = zgemm(s, 1, GN, false, GN, true, p);
    if (st) { dfree(tmp); return st; }
    long total = long(Ns) * M * Nc;
    api_kernels::lnak_reorder_kernel<<<ceil_div(total, 256), 256, 0, s>>>(tmp, h->Lnak[sp], h->Lnak_r[sp], Ns,
                                                            M, Nc);
    st = launch_status("lnak_reorder_kernel");
    cudaDeviceSynchronize();
    dfree(tmp);
    if (st) return st;
  }
  // v0[i][l] = -1/2 sum_{j,n} L[i][j][n] L[l][j][n]  (host copy, as the reference keeps it)
  {
    c128* v0 = nullptr;
    AFQMC_TRY(dalloc(&v0, size_t(nspin_H2) * MM));
    h->vexx_h.assign(size_t(nspin_H2) * MM, 0.0);
    std::vector<c128> tmp(static_cast<size_t>(MM));
    for (int isp = 0; isp < nspin_H2; ++isp) {
      GemmParams p{};
      p.m = M; p.n = M; p.k = int(long(M) * Nc);
      p.A = h->Likn + size_t(isp) * MM * Nc; p.lda = long(M) * Nc;
      p.B = h->Likn + size_t(isp) * MM * Nc; p.ldb = long(M) * Nc;
      p.C = v0 + size_t(isp) * MM; p.ldc = M;
      p.alpha = cmk(-0.5, 0); p.beta = cmk(0, 0);
      int st = zgemm(s, 1, GN, true, GT, true, p);
      if (st) { dfree(v0); return st; }
      cudaMemcpy(tmp.data(), v0 + size_t(isp) * MM, sizeof(c128) * MM, cudaMemcpyDeviceToHost);
      for (long e = 0; e < MM; ++e) h->vexx_h[size_t(isp) * MM + e] = tmp[e].x;
    }
    dfree(v0);
  }
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = h.release();
  return AFQMC_OK;
}

// THC Hamiltonian operations behind the same handle (THCOps, HamiltonianOperations/THCOps.hpp:
// the constructor's factors Piu = X, Luv = L, rotMuv = Z, the half-rotated haj and v0)
extern "C" int afqmc_ham_create_thc(int walker_type, int M, int nup, int ndn, int nu, int nv,
                                    const double* X, const double* L, const double* Z,
                                    const afqmc_c128* hij, int nspin_H1, const double* v0,
                                    double E0, const afqmc_c128* PsiT, afqmc_ham* out) {
  AFQMC_CHECK_ARG(out, "afqmc_ham_create_thc: null out");
  *out = nullptr;
  AFQMC_CHECK_ARG(walker_type == AFQMC_CLOSED || walker_type == AFQMC_COLLINEAR,
                  "afqmc_ham_create_thc: walker_type must be CLOSED (1) or COLLINEAR (2)");
  AFQMC_CHECK_ARG(M > 0 && nu > 0 && nv > 0 && nup >= 0 && ndn >= 0,
                  "afqmc_ham_create_thc: bad sizes");
  AFQMC_CHECK_ARG(nup <= M && ndn <= M, "afqmc_ham_create_thc: more electrons than orbitals");
  AFQMC_CHECK_ARG(X && L && hij && PsiT, "afqmc_ham_create_thc: null input");
  AFQMC_CHECK_ARG(nspin_H1 == 1 || nspin_H1 == 2, "afqmc_ham_create_thc: nspin_H1 must be 1 or 2");
  if (walker_type == AFQMC_CLOSED)
    AFQMC_CHECK_ARG(nspin_H1 == 1,
                    "afqmc_ham_create_thc: CLOSED walkers take a spin-independent Hamiltonian");
  std::unique_ptr<afqmc_ham_s> h(new (std::nothrow) afqmc_ham_s());
  AFQMC_CHECK_ARG(h, "afqmc_ham_create_thc: out of host memory");
  cudaGetDevice(&h->device);
  h->walker_type = walker_type;
  h->M = M; h->nup = nup; h->ndn = ndn; h->Nc = nv;
  h->nspin = walker_type == AFQMC_COLLINEAR ? 2 : 1;
  h->nspin_H2 = 1; h->nspin_H1 = nspin_H1;
  h->nel[0] = nup;
  h->nel[1] = walker_type == AFQMC_COLLINEAR ? ndn : 0;
  h->el_off[0] = 0;
  h->el_off[1] = nup;
  h->nel_tot = h->nel[0] + h->nel[1];
  h->E0 = E0;
  const long MM = long(M) * M;
  h->hij_h.assign((const c128*)hij, (const c128*)hij + nspin_H1 * MM);
  AFQMC_TRY(ham_trial_setup(h.get(), hij, nspin_H1, (const c128*)PsiT));
  AFQMC_TRY(thc_create(&h->thc, walker_type, M, nup, ndn, nu, nv, X, L, Z, h->PsiT));
  h->vexx_h.assign(size_t(MM), 0.0);
  if (v0) {
    std::memcpy(h->vexx_h.data(), v0, sizeof(double) * MM);
  } else {
    // v0[i][l] = -1/2 sum_{j,n} L_n[i][j] L_n[l][j] = -1/2 sum_{u,v} X[i][u] Z[u][v] S[u][v]
    // X[l][v], S[u][v] = sum_j X[j][u] X[j][v], Z = L L^T unless given (host set-up)
    std::vector<double> Zh(size_t(nu) * nu, 0.0), S(size_t(nu) * nu, 0.0), A(size_t(M) * nu, 0.0);
    for (int u = 0; u < nu; ++u)
      for (int v = 0; v < nu; ++v) {
        double z = 0.0, sv = 0.0;
        if (Z) {
          z = Z[size_t(u) * nu + v];
        } else {
          for (int n = 0; n < nv; ++n) z += L[size_t(u) * nv + n] * L[size_t(v) * nv + n];
        }
        for (int j = 0; j < M; ++j) sv += X[size_t(j) * nu + u] * X[size_t(j) * nu + v];
        Zh[size_t(u) * nu + v] = z * sv;
      }
    for (int i = 0; i < M; ++i)
      for (int v = 0; v < nu; ++v) {
        double acc = 0.0;
        for (int u = 0; u < nu; ++u) acc += X[size_t(i) * nu + u] * Zh[size_t(u) * nu + v];
        A[size_t(i) * nu + v] = acc;
      }
    for (int i = 0; i < M; ++i)
      for (int l = 0; l < M; ++l) {
        double acc = 0.0;
        for (int v = 0; v < nu; ++v) acc += A[size_t(i) * nu + v] * X[size_t(l) * nu + v];
        h->vexx_h[size_t(i) * M + l] = -0.5 * acc;
      }
  }
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = h.release();
  return AFQMC_OK;
}

extern "C" int afqmc_ham_thc_info(afqmc_ham h, int* nu, int* nv) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_thc_info: null handle");
  if (!h->thc) {
    if (nu) *nu = 0;
    if (nv) *nv = 0;
    return AFQMC_OK;
  }
  int a = 0, b = 0;
  thc_sizes(h->thc, &a, &b);
  if (nu) *nu = a;
  if (nv) *nv = b;
  return AFQMC_OK;
}

extern "C" int afqmc_ham_destroy(afqmc_ham ham) {
  delete ham;
  return AFQMC_OK;
}

extern "C" int afqmc_ham_info(afqmc_ham h, int* wt, int* M, int* nup, int* ndn, int* Nc,
                              double* E0) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_info: null handle");
  if (wt) *wt = h->walker_type;
  if (M) *M = h->M;
  if (nup) *nup = h->nup;
  if (ndn) *ndn = h->ndn;
  if (Nc) *Nc = h->Nc;
  if (E0) *E0 = h->E0;
  return AFQMC_OK;
}

extern "C" int afqmc_ham_get_tensors(afqmc_ham h, afqmc_c128* Lnak, afqmc_c128* haj,
                                     double* vexx) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_get_tensors: null handle");
  AFQMC_CHECK_ARG(!(Lnak && h->thc), "afqmc_ham_get_tensors: a THC Hamiltonian has no Lnak");
  DeviceGuard g(h->device);
  if (Lnak) {
    long off = 0;
    for (int sp = 0; sp < h->nspin; ++sp) {
      long n = long(h->Nc) * h->nel[sp] * h->M;
      if (n) AFQMC_CUDA_TRY(cudaMemcpy((c128*)Lnak + off, h->Lnak[sp], sizeof(c128) * n,
                                       cudaMemcpyDeviceToHost));
      off += n;
    }
  }
  if (haj && h->nel_tot)
    AFQMC_CUDA_TRY(cudaMemcpy(haj, h->haj, sizeof(c128) * h->nel_tot * h->M, cudaMemcpyDeviceToHost));
  if (vexx) std::memcpy(vexx, h->vexx_h.data(), sizeof(double) * h->vexx_h.size());
  return AFQMC_OK;
}

extern "C" int afqmc_ham_vbias(afqmc_ham h, const afqmc_c128* G, afqmc_c128* v, int W, double dt,
                               int precision, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && W >= 0, "afqmc_ham_vbias: bad argument");
  if (W == 0) return AFQMC_OK;  // no walkers: nothing is read or written
  AFQMC_CHECK_ARG(G && v, "afqmc_ham_vbias: null array");
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == AFQMC_PREC_MIXED && (h->mixed_ops & AFQMC_MIXED_VBIAS)) {
    EnergyArgs a = energy_args(h, (const c128*)G, long(h->nel_tot) * h->M);
    if (!h->mixed) AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    return vbias_mixed(s, h->mixed, (const c128*)G, long(h->nel_tot) * h->M, (c128*)v, W,
                       std::sqrt(dt) * (h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0));
  }
  return ham_vbias(h, s, (const c128*)G, long(h->nel_tot) * h->M, (c128*)v, W, dt);
}

extern "C" int afqmc_ham_vhs(afqmc_ham h, const afqmc_c128* X, afqmc_c128* V, int W, double dt,
                             int precision, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && W >= 0, "afqmc_ham_vhs: bad argument");
  if (W == 0) return AFQMC_OK;  // no walkers: nothing is read or written
  AFQMC_CHECK_ARG(X && V, "afqmc_ham_vhs: null array");
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == AFQMC_PREC_MIXED && (h->mixed_ops & AFQMC_MIXED_PROPAGATION)) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    if (!h->mixed) AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    return vhs_mixed(s, h->mixed, (const c128*)X, (c128*)V, W, std::sqrt(dt));
  }
  return ham_vhs(h, s, (const c128*)X, (c128*)V, W, dt);
}

extern "C" int afqmc_ham_energy(afqmc_ham h, const afqmc_c128* G, afqmc_c128* E, int W, int addH1,
                                int addEJ, int addEXX, int precision, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && W >= 0, "afqmc_ham_energy: bad argument");
  AFQMC_CHECK_ARG(!addEJ || addEXX, "afqmc_ham_energy: addEJ without addEXX is not implemented "
                                    "(as in Real3IndexFactorization.hpp:589)");
  if (W == 0) return AFQMC_OK;  // no walkers: nothing is read or written
  AFQMC_CHECK_ARG(G && E, "afqmc_ham_energy: null array");
  DeviceGuard g(h->device);
  return ham_energy(h, reinterpret_cast<cudaStream_t>(stream), (const c128*)G,
                    long(h->nel_tot) * h->M, (c128*)E, W, addH1 != 0, addEJ != 0, addEXX != 0,
                    precision);
}

extern "C" int afqmc_ham_set_mixed_ops(afqmc_ham h, int mask) {
  AFQMC_CHECK_ARG(h && (mask & ~(AFQMC_MIXED_ALL | AFQMC_MIXED_VHS)) == 0,
                  "afqmc_ham_set_mixed_ops: bad mask");
  h->mixed_ops = mask;
  return AFQMC_OK;
}

extern "C" int afqmc_ham_set_coulomb_fp64(afqmc_ham h, int on) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_coulomb_fp64: null handle");
  h->coulomb_fp64 = on != 0;
  return AFQMC_OK;
}

extern "C" int afqmc_ham_set_exchange_split(afqmc_ham h, int nsplit) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_exchange_split: null handle");
  AFQMC_CHECK_ARG(nsplit == 1 || nsplit == 3, "afqmc_ham_set_exchange_split: nsplit must be 1 or 3");
  DeviceGuard g(h->device);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, nullptr));
  }
  return mixed_set_exchange_split(h->mixed, nsplit);
}

extern "C" int afqmc_ham_set_vhs_symmetry(afqmc_ham h, int enable, int* active) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_vhs_symmetry: null handle");
  DeviceGuard g(h->device);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, nullptr));
  }
  return mixed_set_vhs_symmetry(h->mixed, enable, active);
}

extern "C" int afqmc_ham_set_split_format(afqmc_ham h, int format, int* active_f16) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_split_format: null handle");
  DeviceGuard g(h->device);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, nullptr));
  }
  return mixed_set_split_format(h->mixed, format, active_f16);
}

extern "C" int afqmc_ham_set_taylor_fused(afqmc_ham h, int fused) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_taylor_fused: null handle");
  AFQMC_CHECK_ARG(fused >= 0 && fused <= 7, "afqmc_ham_set_taylor_fused: mode must be 0..7");
  DeviceGuard g(h->device);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, nullptr));
  }
  return mixed_set_taylor_mode(h->mixed, fused);
}

extern "C" int afqmc_ham_device_error(afqmc_ham h, unsigned* flag) {
  AFQMC_CHECK_ARG(h && flag, "afqmc_ham_device_error: null argument");
  DeviceGuard g(h->device);
  *flag = 0;
  if (h->mixed) return mixed_error_flag(h->mixed, flag);
  return AFQMC_OK;
}

extern "C" int afqmc_ham_clear_device_error(afqmc_ham h) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_clear_device_error: null argument");
  DeviceGuard g(h->device);
  if (h->mixed) return mixed_clear_error(h->mixed);
  return AFQMC_OK;
}

extern "C" int afqmc_ham_wait_selftest(afqmc_ham h, long long budget_cycles,
                                       afqmc_stream stream) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_wait_selftest: null argument");
  DeviceGuard g(h->device);
  cudaStream_t s = (cudaStream_t)stream;
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
  }
  return mixed_wait_selftest(s, h->mixed, budget_cycles);
}

extern "C" int afqmc_ham_one_body_propagator(afqmc_ham h, double dt, const afqmc_c128* vMF,
                                             afqmc_c128* H1) {
  AFQMC_CHECK_ARG(h && vMF && H1, "afqmc_ham_one_body_propagator: null argument");
  DeviceGuard g(h->device);
  const long MM = long(h->M) * h->M;
  const int nst = h->walker_type == AFQMC_COLLINEAR ? h->nspin_H2 : 1;
  c128 *x = nullptr, *v = nullptr;
  AFQMC_TRY(dalloc(&x, size_t(h->Nc)));
  int st = dalloc(&v, size_t(nst) * MM);
  if (st) { dfree(x); return st; }
  cudaMemcpy(x, vMF, sizeof(c128) * h->Nc, cudaMemcpyHostToDevice);
  st = ham_vhs(h, nullptr, x, v, 1, dt);
  std::vector<c128> mf(size_t(nst) * MM);
  if (!st) {
    cudaError_t e = cudaMemcpy(mf.data(), v, sizeof(c128) * mf.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      set_error_detail("afqmc_ham_one_body_propagator: %s", cudaGetErrorString(e));
      st = AFQMC_ERR_CUDA;
    }
  }
  dfree(x);
  dfree(v);
  if (st) return st;
  c128* out = (c128*)H1;
  const int nsv = h->nspin_H2;  // vexx spin blocks
  for (int s = 0; s < h->nspin; ++s)
    for (long e = 0; e < MM; ++e) {
      c128 hv = h->hij_h[size_t(s % h->nspin_H1) * MM + e];
      double v0 = h->vexx_h[size_t(s % nsv) * MM + e];
      c128 m = mf[size_t(s % nst) * MM + e];
      out[size_t(s) * MM + e] = cmk(dt * hv.x + dt * v0 + m.x, dt * hv.y + m.y);
    }
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// walker sets
// ---------------------------------------------------------------------------------------------
namespace api_kernels {
__global__ void broadcast_row_kernel(c128* buf, long walker_size, int W, const c128* row) {
  long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  long total = long(W) * walker_size;
  if (e < total) buf[e] = row[e % walker_size];
}
}  // namespace api_kernels

extern "C" int afqmc_wset_create(int walker_type, int M, int nup, int ndn, int W,
                                 afqmc_wset* out) {
  AFQMC_CHECK_ARG(out, "afqmc_wset_create: null out");
  *out = nullptr;
  AFQMC_CHECK_ARG(walker_type == AFQMC_CLOSED || walker_type == AFQMC_COLLINEAR,
                  "afqmc_wset_create: bad walker type");
  AFQMC_CHECK_ARG(M > 0 && nup >= 0 && ndn >= 0 && W > 0, "afqmc_wset_create: bad sizes");
  std::unique_ptr<afqmc_wset_s> ws(new (std::nothrow) afqmc_wset_s());
  AFQMC_CHECK_ARG(ws, "afqmc_wset_create: out of host memory");
  cudaGetDevice(&ws->device);
  ws->walker_type = walker_type;
  ws->M = M; ws->nup = nup; ws->ndn = walker_type == AFQMC_COLLINEAR ? ndn : 0; ws->W = W;
  ws->prop0 = long(M) * (ws->nup + ws->ndn);
  ws->walker_size = ws->prop0 + AFQMC_NPROP;
  AFQMC_TRY(dalloc(&ws->buf, size_t(W) * ws->walker_size));
  AFQMC_CUDA_TRY(cudaMemset(ws->buf, 0, sizeof(c128) * size_t(W) * ws->walker_size));
  *out = ws.release();
  return AFQMC_OK;
}

extern "C" int afqmc_wset_destroy(afqmc_wset ws) {
  delete ws;
  return AFQMC_OK;
}

extern "C" int afqmc_wset_buffer(afqmc_wset ws, afqmc_c128** data, long* walker_size, int* W) {
  AFQMC_CHECK_ARG(ws, "afqmc_wset_buffer: null handle");
  if (data) *data = (afqmc_c128*)ws->buf;
  if (walker_size) *walker_size = ws->walker_size;
  if (W) *W = ws->W;
  return AFQMC_OK;
}

extern "C" int afqmc_wset_get_property(afqmc_wset ws, int prop, afqmc_c128* host_out) {
  AFQMC_CHECK_ARG(ws && host_out && prop >= 0 && prop < AFQMC_NPROP,
                  "afqmc_wset_get_property: bad argument");
  DeviceGuard g(ws->device);
  AFQMC_CUDA_TRY(cudaMemcpy2D(host_out, sizeof(c128), ws->buf + ws->prop0 + prop,
                              ws->walker_size * sizeof(c128), sizeof(c128), ws->W,
                              cudaMemcpyDeviceToHost));
  return AFQMC_OK;
}

extern "C" int afqmc_wset_set_property(afqmc_wset ws, int prop, const afqmc_c128* host_in) {
  AFQMC_CHECK_ARG(ws && host_in && prop >= 0 && prop < AFQMC_NPROP,
                  "afqmc_wset_set_property: bad argument");
  DeviceGuard g(ws->device);
  AFQMC_CUDA_TRY(cudaMemcpy2D(ws->buf + ws->prop0 + prop, ws->walker_size * sizeof(c128), host_in,
                              sizeof(c128), sizeof(c128), ws->W, cudaMemcpyHostToDevice));
  return AFQMC_OK;
}

extern "C" int afqmc_wset_init_from_trial(afqmc_wset ws, afqmc_ham h, afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && h, "afqmc_wset_init_from_trial: null handle");
  AFQMC_CHECK_ARG(ws->M == h->M && ws->nup == h->nel[0] && ws->ndn == h->nel[1] &&
                      ws->walker_type == h->walker_type,
                  "afqmc_wset_init_from_trial: walker set does not match the Hamiltonian");
  DeviceGuard g(ws->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  std::vector<c128> row(static_cast<size_t>(ws->walker_size), cmk(0, 0));
  const long nS = ws->prop0;
  if (nS) AFQMC_CUDA_TRY(cudaMemcpy(row.data(), h->PsiH, sizeof(c128) * nS, cudaMemcpyDeviceToHost));
  row[nS + AFQMC_WEIGHT] = cmk(1, 0);
  row[nS + AFQMC_PHASE] = cmk(1, 0);
  c128* drow = nullptr;
  AFQMC_TRY(dalloc(&drow, row.size()));
  AFQMC_CUDA_TRY(cudaMemcpy(drow, row.data(), sizeof(c128) * row.size(), cudaMemcpyHostToDevice));
  long total = long(ws->W) * ws->walker_size;
  api_kernels::broadcast_row_kernel<<<ceil_div(total, 256), 256, 0, s>>>(ws->buf, ws->walker_size, ws->W, drow);
  int st = launch_status("broadcast_row_kernel");
  cudaStreamSynchronize(s);
  dfree(drow);
  return st;
}

// ---------------------------------------------------------------------------------------------
// NOMSD (single determinant, ci = 1)
// ---------------------------------------------------------------------------------------------
namespace {

int wfn_density_matrix(afqmc_ham_s* h, afqmc_wset_s* ws, cudaStream_t s, c128* G, long ldG,
                       c128* ovlp, c128* workT) {
  const int W = ws->W;
  AFQMC_CUDA_TRY(cudaMemsetAsync(ovlp, 0, sizeof(c128) * W, s));
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    if (Ns == 0) continue;
    const c128 scale = (h->walker_type == AFQMC_CLOSED) ? cmk(2, 0) : cmk(1, 0);
    AFQMC_TRY(mixed_density_matrix(s, h->PsiT + long(h->el_off[sp]) * h->M, ws->buf + ws->offS(sp),
                                   ws->walker_size, G + long(h->el_off[sp]) * h->M, ldG, ovlp, W,
                                   h->M, Ns, true, workT, nullptr, scale, cmk(0, 0)));
  }
  return AFQMC_OK;
}

int wfn_log_overlap(afqmc_ham_s* h, afqmc_wset_s* ws, cudaStream_t s, c128* ovlp, c128* workT) {
  const int W = ws->W;
  AFQMC_CUDA_TRY(cudaMemsetAsync(ovlp, 0, sizeof(c128) * W, s));
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    if (Ns == 0) continue;
    const c128 scale = (h->walker_type == AFQMC_CLOSED) ? cmk(2, 0) : cmk(1, 0);
    AFQMC_TRY(log_overlap(s, h->PsiT + long(h->el_off[sp]) * h->M, ws->buf + ws->offS(sp),
                          ws->walker_size, ovlp, W, h->M, Ns, workT, scale, cmk(0, 0)));
  }
  return AFQMC_OK;
}

bool wset_matches(afqmc_ham_s* h, afqmc_wset_s* ws) {
  return ws->M == h->M && ws->nup == h->nel[0] && ws->ndn == h->nel[1] &&
         ws->walker_type == h->walker_type;
}

}  // namespace

extern "C" int afqmc_wfn_density_matrix(afqmc_ham h, afqmc_wset ws, afqmc_c128* G,
                                        afqmc_c128* ovlp, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && ws && G && ovlp, "afqmc_wfn_density_matrix: null argument");
  AFQMC_CHECK_ARG(wset_matches(h, ws), "afqmc_wfn_density_matrix: walker set / Hamiltonian mismatch");
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  Scratch T;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(ws->W) * nmax * nmax, s));
  return wfn_density_matrix(h, ws, s, (c128*)G, long(h->nel_tot) * h->M, (c128*)ovlp, (c128*)T.p);
}

extern "C" int afqmc_wfn_onerdm(afqmc_ham h, afqmc_wset ws, const afqmc_c128* G, long ldG,
                                afqmc_c128* rdm, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && ws && G && rdm, "afqmc_wfn_onerdm: null argument");
  AFQMC_CHECK_ARG(wset_matches(h, ws), "afqmc_wfn_onerdm: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ldG >= long(h->nel_tot) * h->M, "afqmc_wfn_onerdm: ldG %ld < nel M", ldG);
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int M = h->M, W = ws->W;
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  Scratch Gs;
  AFQMC_TRY(Gs.get(sizeof(c128) * size_t(nmax > 0 ? nmax : 1) * M, s));
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    c128* out = reinterpret_cast<c128*>(rdm) + size_t(sp) * M * M;
    if (Ns == 0) {
      AFQMC_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(c128) * M * M, s));
      continue;
    }
    // Gsum [Ns][M] = sum_w w_w G_w (the weights are the walkers' WEIGHT column)
    GemmParams a{};
    a.m = 1; a.n = Ns * M; a.k = W;
    a.A = ws->buf + ws->prop0 + AFQMC_WEIGHT; a.lda = ws->walker_size;
    a.B = reinterpret_cast<const c128*>(G) + long(h->el_off[sp]) * M; a.ldb = ldG;
    a.C = reinterpret_cast<c128*>(Gs.p); a.ldc = Ns * M;
    a.alpha = cmk(1, 0); a.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, 1, GT, false, GN, false, a));
    // full G [M][M] = PsiT^T Gsum  (G[i][k] = sum_a PsiT[a][i] Gc[a][k])
    GemmParams b{};
    b.m = M; b.n = M; b.k = Ns;
    b.A = h->PsiT + long(h->el_off[sp]) * M; b.lda = M;
    b.B = reinterpret_cast<const c128*>(Gs.p); b.ldb = M;
    b.C = out; b.ldc = M;
    b.alpha = cmk(1, 0); b.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, 1, GT, false, GN, false, b));
  }
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// NOMSD with several determinants (NOMSD.cpp:93-333, 159-217; Real3IndexFactorization.hpp:389-427)
// ---------------------------------------------------------------------------------------------
namespace multidet {
// E[w] = sum_d conj(c_d) E_d e^{ov_d - m} / sum_d conj(c_d) e^{ov_d - m}, Ov = log(den) + m
// (NOMSD.cpp:195-211)
__global__ void multidet_energy_kernel(const c128* __restrict__ Ed, const c128* __restrict__ ov,
                                       const c128* __restrict__ cc, int ndet, int W,
                                       c128* __restrict__ E, c128* __restrict__ Ov) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  c128 m = ov[w];
  for (int d = 1; d < ndet; ++d)
    if (ov[size_t(d) * W + w].x > m.x) m = ov[size_t(d) * W + w];
  c128 den = cmk(0, 0), s[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
  for (int d = 0; d < ndet; ++d) {
    const c128 f = cmul(cc[d], cexp(csub(ov[size_t(d) * W + w], m)));
    den = cadd(den, f);
    for (int q = 0; q < 3; ++q) s[q] = cadd(s[q], cmul(f, Ed[(size_t(d) * W + w) * 3 + q]));
  }
  for (int q = 0; q < 3; ++q) E[w * 3 + q] = cdiv(s[q], den);
  Ov[w] = cadd(clog(den), m);
}

// Workspace bound of one walker chunk of the batched several-determinant step
constexpr size_t NOMSD_CHUNK_BYTES = size_t(1) << 30;

int nomsd_bufs(afqmc_nomsd md, int W) {
  if (md->capW >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  md->free_bufs();
  afqmc_ham_s* h = md->hams[0];
  const long M = h->M, ldG = long(h->nel_tot) * M;
  const int nmax = std::max(h->nel[0], h->nel[1]);
  const size_t nd = md->hams.size();
  AFQMC_TRY(dalloc(&md->Gc, size_t(W) * (ldG > 0 ? ldG : 1)));
  AFQMC_TRY(dalloc(&md->ov, nd * W));
  AFQMC_TRY(dalloc(&md->T, size_t(W) * (nmax > 0 ? nmax * nmax : 1)));
  AFQMC_TRY(dalloc(&md->Ed, nd * W * 3));
  // batched step: chunk of walkers
  const size_t nsq = size_t(h->nel[0]) * h->nel[0] + size_t(h->nel[1]) * h->nel[1];
  const size_t per_walker = nd * (size_t(ldG) + nsq + 2) * sizeof(c128);
  size_t wc = std::min<size_t>(size_t(W), 65535 / nd);
  wc = std::min(wc, std::max<size_t>(1, NOMSD_CHUNK_BYTES / per_walker));
  AFQMC_TRY(dalloc(&md->Tb, wc * nd * (nsq > 0 ? nsq : 1)));
  AFQMC_TRY(dalloc(&md->Ttb, wc * nd * (nsq > 0 ? nsq : 1)));
  AFQMC_TRY(dalloc(&md->Gcb, wc * nd * size_t(ldG > 0 ? ldG : 1)));
  AFQMC_TRY(dalloc(&md->ovd, wc * nd));
  AFQMC_TRY(dalloc(&md->wdd, wc * nd));
  md->wchunk = int(wc);
  md->capW = W;
  return AFQMC_OK;
}

// out[w] = m + log sum_d exp(ovd[w][d] + lc[d] - m), m = the largest real part of the
// ovd[w][d] + lc[d] (NOMSD.cpp:303-331: per-determinant log overlap + log conj(ci))
__global__ void logsumexp_wd_kernel(const c128* __restrict__ ovd, const c128* __restrict__ lc,
                                    int ndet, int W, c128* __restrict__ out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const c128* o = ovd + size_t(w) * ndet;
  c128 m = cadd(o[0], lc[0]);
  for (int d = 1; d < ndet; ++d) {
    const c128 x = cadd(o[d], lc[d]);
    if (x.x > m.x) m = x;
  }
  c128 sum = cmk(0, 0);
  for (int d = 0; d < ndet; ++d) sum = cadd(sum, cexp(csub(cadd(o[d], lc[d]), m)));
  out[w] = cadd(m, clog(sum));
}

// f_d = conj(c_d) exp(ovd[w][d] - ovlp_w) with ovlp_w the walker's stored log overlap;
// wdd[w][d] = f_d / sum_d f_d, Ov[w] = sum_d f_d + ovlp_w (NOMSD.cpp:220-279: the reference
// divides the summed G by the linear sum and then adds the log of the shift to it)
__global__ void multidet_weights_kernel(const c128* __restrict__ ovd, const c128* __restrict__ cc,
                                        int ndet, int W, const c128* __restrict__ wbuf, long ldw,
                                        long prop_ovlp, c128* __restrict__ wdd,
                                        c128* __restrict__ Ov) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  const c128 shift = wbuf[long(w) * ldw + prop_ovlp];
  const c128* o = ovd + size_t(w) * ndet;
  c128* f = wdd + size_t(w) * ndet;
  c128 sum = cmk(0, 0);
  for (int d = 0; d < ndet; ++d) {
    f[d] = cmul(cc[d], cexp(csub(o[d], shift)));
    sum = cadd(sum, f[d]);
  }
  const c128 inv = cdiv(cmk(1, 0), sum);
  for (int d = 0; d < ndet; ++d) f[d] = cmul(f[d], inv);
  Ov[w] = cadd(sum, shift);
}

// Tt[b] = wdd[b] T[b]^T for nb blocks of n x n elements
__global__ void weight_transpose_blocks_kernel(const c128* __restrict__ T, c128* __restrict__ Tt,
                                               int n, long nb, const c128* __restrict__ wdd) {
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const long nsq = long(n) * n;
  if (t >= nsq * nb) return;
  const long b = t / nsq;
  const int e = int(t - b * nsq), i = e / n, j = e - i * n;
  Tt[b * nsq + long(j) * n + i] = cmul(T[t], wdd[b]);
}

// Overlap matrices T[w][d] = PsiT_d S_w of every determinant for walkers w0 .. w0+wc-1 (one
// GEMM per spin), their log determinants summed over spins into ovd[w][d] (CLOSED x2) and,
// with invert, T[w][d] <- T[w][d]^{-1} (one Gauss-Jordan launch per spin)
int nomsd_overlaps(afqmc_nomsd md, afqmc_wset_s* ws, cudaStream_t s, int w0, int wc,
                   bool invert) {
  afqmc_ham_s* h0 = md->hams[0];
  const int nd = int(md->hams.size());
  const long M = h0->M, nb = long(wc) * nd;
  const c128* S0 = ws->buf + long(w0) * ws->walker_size;
  const c128 scale = (h0->walker_type == AFQMC_CLOSED) ? cmk(2, 0) : cmk(1, 0);
  AFQMC_CUDA_TRY(cudaMemsetAsync(md->ovd, 0, sizeof(c128) * nb, s));
  long toff = 0;
  for (int sp = 0; sp < h0->nspin; ++sp) {
    const int Ns = h0->nel[sp];
    if (Ns == 0) continue;
    const long nsq = long(Ns) * Ns;
    c128* Tsp = md->Tb + toff;
    toff += long(md->wchunk) * nd * nsq;
    GemmParams p{};
    p.m = nd * Ns; p.n = Ns; p.k = int(M);
    p.A = md->PsiTall + long(nd) * h0->el_off[sp] * M; p.lda = M; p.strideA = 0;
    p.B = S0 + ws->offS(sp); p.ldb = Ns; p.strideB = ws->walker_size;
    p.C = Tsp; p.ldc = Ns; p.strideC = long(nd) * nsq;
    p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
    AFQMC_TRY(zgemm(s, wc, GN, false, GN, false, p));
    AFQMC_TRY(batched_logdet_inverse(s, Tsp, nsq, invert ? Tsp : nullptr, nsq, md->ovd, int(nb),
                                     Ns, invert, scale, cmk(0, 0)));
  }
  return AFQMC_OK;
}

int nomsd_log_overlap(afqmc_nomsd md, afqmc_wset_s* ws, cudaStream_t s, c128* ovlp) {
  const int W = ws->W, nd = int(md->hams.size());
  AFQMC_TRY(nomsd_bufs(md, W));
  for (int w0 = 0; w0 < W; w0 += md->wchunk) {
    const int wc = std::min(md->wchunk, W - w0);
    AFQMC_TRY(nomsd_overlaps(md, ws, s, w0, wc, false));
    logsumexp_wd_kernel<<<ceil_div(wc, 128), 128, 0, s>>>(md->ovd, md->dlc, nd, wc, ovlp + w0);
    AFQMC_TRY(launch_status("logsumexp_wd_kernel"));
  }
  return AFQMC_OK;
}

// full mixed density matrices of every determinant combined (NOMSD.cpp:220-279, compact=false):
// G[w][s] = sum_d wdd[w][d] PsiT_d^T (T[w][d]^{-1})^T S_w^T, the weight folded into the inverse
// before the compact product and the sum over determinants done by one GEMM with K = nd * N_s
int nomsd_density_matrix(afqmc_nomsd md, afqmc_wset_s* ws, cudaStream_t s, c128* G, c128* Ov) {
  afqmc_ham_s* h0 = md->hams[0];
  const int W = ws->W, nd = int(md->hams.size()), nspin = h0->nspin;
  const long M = h0->M, MM = M * M, per = long(nspin) * MM;
  AFQMC_TRY(nomsd_bufs(md, W));
  for (int w0 = 0; w0 < W; w0 += md->wchunk) {
    const int wc = std::min(md->wchunk, W - w0);
    const long nb = long(wc) * nd;
    const c128* S0 = ws->buf + long(w0) * ws->walker_size;
    c128* Gw = G + long(w0) * per;
    AFQMC_TRY(nomsd_overlaps(md, ws, s, w0, wc, true));
    multidet_weights_kernel<<<ceil_div(wc, 128), 128, 0, s>>>(
        md->ovd, md->dcc, nd, wc, S0, ws->walker_size, ws->prop0 + AFQMC_OVLP, md->wdd, Ov + w0);
    AFQMC_TRY(launch_status("multidet_weights_kernel"));
    long toff = 0;
    for (int sp = 0; sp < nspin; ++sp) {
      const int Ns = h0->nel[sp];
      if (Ns == 0) {
        AFQMC_CUDA_TRY(cudaMemset2DAsync(Gw + sp * MM, per * sizeof(c128), 0, MM * sizeof(c128),
                                         wc, s));
        continue;
      }
      const long nsq = long(Ns) * Ns;
      c128* Tsp = md->Tb + toff;
      c128* Ttsp = md->Ttb + toff;
      toff += long(md->wchunk) * nd * nsq;
      c128* Gcsp = md->Gcb + long(md->wchunk) * nd * h0->el_off[sp] * M;
      weight_transpose_blocks_kernel<<<ceil_div(nsq * nb, 256), 256, 0, s>>>(Tsp, Ttsp, Ns, nb,
                                                                            md->wdd);
      AFQMC_TRY(launch_status("weight_transpose_blocks_kernel"));
      // Gc[w] = [wdd_d (T_d^{-1})^T]_d S_w^T  [nd N_s x M]  (every determinant's compact G,
      // weighted; one product per walker)
      GemmParams p{};
      p.m = nd * Ns; p.n = int(M); p.k = Ns;
      p.A = Ttsp; p.lda = Ns; p.strideA = long(nd) * nsq;
      p.B = S0 + ws->offS(sp); p.ldb = Ns; p.strideB = ws->walker_size;
      p.C = Gcsp; p.ldc = M; p.strideC = long(nd) * Ns * M;
      p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
      AFQMC_TRY(zgemm(s, wc, GN, false, GT, false, p));
      // G[w][s] = PsiTall_s^T Gc[w]  (K = nd * N_s: the sum over determinants)
      GemmParams q{};
      q.m = int(M); q.n = int(M); q.k = nd * Ns;
      q.A = md->PsiTall + long(nd) * h0->el_off[sp] * M; q.lda = M; q.strideA = 0;
      q.B = Gcsp; q.ldb = M; q.strideB = long(nd) * Ns * M;
      q.C = Gw + sp * MM; q.ldc = M; q.strideC = per;
      q.alpha = cmk(1, 0); q.beta = cmk(0, 0);
      AFQMC_TRY(zgemm(s, wc, GT, false, GN, false, q));
    }
  }
  return AFQMC_OK;
}

// vbias from the full G (the ndet > 1 branch, Real3IndexFactorization.hpp:389-427):
// v[w][n] = a sum_s sum_{ik} L_s[ik][n] G[w][s][ik], a = sqrt(dt) (x2 CLOSED)
int nomsd_vbias(afqmc_ham_s* h, cudaStream_t s, const c128* G, c128* v, int W, double dt) {
  const int nspin = h->nspin;
  const long MM = long(h->M) * h->M;
  const double a = std::sqrt(dt) * (h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0);
  for (int sp = 0; sp < nspin; ++sp) {
    GemmParams p{};
    p.m = W; p.n = h->Nc; p.k = int(MM);
    p.A = G + sp * MM; p.lda = nspin * MM; p.strideA = 0;
    p.B = h->Likn + size_t(sp % h->nspin_H2) * MM * h->Nc; p.ldb = h->Nc; p.strideB = 0;
    p.C = v; p.ldc = h->Nc; p.strideC = 0;
    p.alpha = cmk(a, 0); p.beta = sp == 0 ? cmk(0, 0) : cmk(1, 0);
    AFQMC_TRY(zgemm(s, 1, GN, false, GN, true, p));
  }
  return AFQMC_OK;
}
}  // namespace multidet
using namespace multidet;

extern "C" int afqmc_nomsd_create(int ndet, const afqmc_ham* hams, const afqmc_c128* ci,
                                  afqmc_nomsd* out) {
  AFQMC_CHECK_ARG(out && hams && ci && ndet >= 1 && ndet <= 65535,
                  "afqmc_nomsd_create: bad argument");
  *out = nullptr;
  afqmc_ham_s* h0 = hams[0];
  AFQMC_CHECK_ARG(h0, "afqmc_nomsd_create: null Hamiltonian 0");
  for (int d = 0; d < ndet; ++d)
    AFQMC_CHECK_ARG(!hams[d] || !hams[d]->thc,
                    "afqmc_nomsd_create: THC Hamiltonians take one determinant (as THCOps)");
  for (int d = 1; d < ndet; ++d) {
    afqmc_ham_s* h = hams[d];
    AFQMC_CHECK_ARG(h && h->device == h0->device && h->walker_type == h0->walker_type &&
                        h->M == h0->M && h->Nc == h0->Nc && h->nel[0] == h0->nel[0] &&
                        h->nel[1] == h0->nel[1],
                    "afqmc_nomsd_create: determinant %d's Hamiltonian differs in shape", d);
  }
  std::unique_ptr<afqmc_nomsd_s> md(new (std::nothrow) afqmc_nomsd_s());
  AFQMC_CHECK_ARG(md, "afqmc_nomsd_create: out of host memory");
  md->device = h0->device;
  md->hams.assign(hams, hams + ndet);
  md->ci.assign(reinterpret_cast<const c128*>(ci), reinterpret_cast<const c128*>(ci) + ndet);
  DeviceGuard g(md->device);
  // every determinant's PsiT stacked per spin, conj(ci) and log conj(ci) (a coefficient below
  // 1e-12 in modulus enters the log overlap as 1e-12, NOMSD.cpp:303-316)
  const long M = h0->M;
  AFQMC_TRY(dalloc(&md->PsiTall, size_t(ndet) * (h0->nel_tot > 0 ? h0->nel_tot : 1) * M));
  for (int sp = 0; sp < h0->nspin; ++sp) {
    const long rows = long(h0->nel[sp]) * M;
    for (int d = 0; d < ndet && rows > 0; ++d)
      AFQMC_CUDA_TRY(cudaMemcpy(md->PsiTall + long(ndet) * h0->el_off[sp] * M + d * rows,
                                hams[d]->PsiT + long(h0->el_off[sp]) * M, sizeof(c128) * rows,
                                cudaMemcpyDeviceToDevice));
  }
  std::vector<c128> cc(ndet), lc(ndet);
  for (int d = 0; d < ndet; ++d) {
    cc[d] = cconj(md->ci[d]);
    lc[d] = cabs(md->ci[d]) < 1e-12 ? clog(cmk(1e-12, 0)) : clog(cc[d]);
  }
  AFQMC_TRY(dalloc(&md->dcc, size_t(ndet)));
  AFQMC_TRY(dalloc(&md->dlc, size_t(ndet)));
  AFQMC_CUDA_TRY(cudaMemcpy(md->dcc, cc.data(), sizeof(c128) * ndet, cudaMemcpyHostToDevice));
  AFQMC_CUDA_TRY(cudaMemcpy(md->dlc, lc.data(), sizeof(c128) * ndet, cudaMemcpyHostToDevice));
  *out = md.release();
  return AFQMC_OK;
}

extern "C" int afqmc_nomsd_destroy(afqmc_nomsd md) {
  delete md;
  return AFQMC_OK;
}

extern "C" int afqmc_nomsd_log_overlap(afqmc_nomsd md, afqmc_wset ws, afqmc_c128* ovlp,
                                       afqmc_stream stream) {
  AFQMC_CHECK_ARG(md && ws && ovlp, "afqmc_nomsd_log_overlap: null argument");
  AFQMC_CHECK_ARG(wset_matches(md->hams[0], ws), "afqmc_nomsd_log_overlap: mismatch");
  DeviceGuard g(md->device);
  return nomsd_log_overlap(md, ws, reinterpret_cast<cudaStream_t>(stream),
                           reinterpret_cast<c128*>(ovlp));
}

extern "C" int afqmc_nomsd_energy(afqmc_nomsd md, afqmc_wset ws, afqmc_c128* E, afqmc_c128* ovlp,
                                  int precision, afqmc_stream stream) {
  AFQMC_CHECK_ARG(md && ws && E && ovlp, "afqmc_nomsd_energy: null argument");
  AFQMC_CHECK_ARG(wset_matches(md->hams[0], ws), "afqmc_nomsd_energy: mismatch");
  DeviceGuard g(md->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int W = ws->W, nd = int(md->hams.size());
  AFQMC_TRY(nomsd_bufs(md, W));
  const long ldG = long(md->hams[0]->nel_tot) * md->hams[0]->M;
  for (int d = 0; d < nd; ++d) {
    afqmc_ham_s* h = md->hams[d];
    AFQMC_TRY(wfn_density_matrix(h, ws, s, md->Gc, ldG, md->ov + size_t(d) * W, md->T));
    AFQMC_TRY(ham_energy(h, s, md->Gc, ldG, md->Ed + size_t(d) * W * 3, W, true, true, true,
                         precision));
  }
  multidet_energy_kernel<<<ceil_div(W, 128), 128, 0, s>>>(md->Ed, md->ov, md->dcc, nd, W,
                                                          (c128*)E, (c128*)ovlp);
  AFQMC_TRY(launch_status("multidet_energy_kernel"));
  return cudaStreamSynchronize(s) == cudaSuccess ? AFQMC_OK : AFQMC_ERR_CUDA;
}

extern "C" int afqmc_nomsd_density_matrix(afqmc_nomsd md, afqmc_wset ws, afqmc_c128* G,
                                          afqmc_c128* ovlp, afqmc_stream stream) {
  AFQMC_CHECK_ARG(md && ws && G && ovlp, "afqmc_nomsd_density_matrix: null argument");
  AFQMC_CHECK_ARG(wset_matches(md->hams[0], ws), "afqmc_nomsd_density_matrix: mismatch");
  DeviceGuard g(md->device);
  return nomsd_density_matrix(md, ws, reinterpret_cast<cudaStream_t>(stream),
                              reinterpret_cast<c128*>(G), reinterpret_cast<c128*>(ovlp));
}

extern "C" int afqmc_nomsd_vbias(afqmc_nomsd md, const afqmc_c128* G, afqmc_c128* v, int W,
                                 double dt, afqmc_stream stream) {
  AFQMC_CHECK_ARG(md && W >= 0, "afqmc_nomsd_vbias: bad argument");
  if (W == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(G && v, "afqmc_nomsd_vbias: null array");
  DeviceGuard g(md->device);
  return nomsd_vbias(md->hams[0], reinterpret_cast<cudaStream_t>(stream),
                     reinterpret_cast<const c128*>(G), reinterpret_cast<c128*>(v), W, dt);
}

extern "C" int afqmc_wfn_log_overlap(afqmc_ham h, afqmc_wset ws, afqmc_c128* ovlp,
                                     afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && ws && ovlp, "afqmc_wfn_log_overlap: null argument");
  AFQMC_CHECK_ARG(wset_matches(h, ws), "afqmc_wfn_log_overlap: walker set / Hamiltonian mismatch");
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  Scratch T;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(ws->W) * nmax * nmax, s));
  return wfn_log_overlap(h, ws, s, (c128*)ovlp, (c128*)T.p);
}

extern "C" int afqmc_wfn_energy(afqmc_ham h, afqmc_wset ws, afqmc_c128* E, afqmc_c128* ovlp,
                                int set_properties, int precision, afqmc_stream stream) {
  AFQMC_CHECK_ARG(h && ws && E && ovlp, "afqmc_wfn_energy: null argument");
  AFQMC_CHECK_ARG(wset_matches(h, ws), "afqmc_wfn_energy: walker set / Hamiltonian mismatch");
  DeviceGuard g(h->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int W = ws->W;
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  Scratch T, Gb;
  const long ldG = long(h->nel_tot) * h->M;
  AFQMC_TRY(T.get(sizeof(c128) * size_t(W) * nmax * nmax, s));
  AFQMC_TRY(Gb.get(sizeof(c128) * size_t(W) * ldG, s));
  AFQMC_TRY(wfn_density_matrix(h, ws, s, (c128*)Gb.p, ldG, (c128*)ovlp, (c128*)T.p));
  AFQMC_TRY(ham_energy(h, s, (const c128*)Gb.p, ldG, (c128*)E, W, true, true, true, precision));
  // + log(conj(ci)) with ci = 1 adds 0 (NOMSD.cpp:180-182)
  if (set_properties) {
    const c128* Ed = (const c128*)E;
    AFQMC_TRY(scatter_property(s, ws->buf, ws->walker_size, ws->prop0 + AFQMC_OVLP, W,
                               (const c128*)ovlp));
    // E is [W][3]; scatter each column through a strided gather
    for (int q = 0; q < 3; ++q) {
      AFQMC_CUDA_TRY(cudaMemcpy2DAsync(ws->buf + ws->prop0 + AFQMC_E1 + q,
                                       ws->walker_size * sizeof(c128), Ed + q, 3 * sizeof(c128),
                                       sizeof(c128), W, cudaMemcpyDeviceToDevice, s));
    }
  }
  return AFQMC_OK;
}

extern "C" int afqmc_wfn_vmf(afqmc_ham h, double dt, afqmc_c128* vMF_host) {
  AFQMC_CHECK_ARG(h && vMF_host, "afqmc_wfn_vmf: null argument");
  DeviceGuard g(h->device);
  cudaStream_t s = nullptr;
  const long ldG = long(h->nel_tot) * h->M;
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  c128 *G = nullptr, *T = nullptr, *ov = nullptr, *v = nullptr;
  int st = dalloc(&G, size_t(ldG > 0 ? ldG : 1));
  if (!st) st = dalloc(&T, size_t(nmax > 0 ? nmax * nmax : 1));
  if (!st) st = dalloc(&ov, 1);
  if (!st) st = dalloc(&v, size_t(h->Nc));
  if (!st) {
    cudaMemset(ov, 0, sizeof(c128));
    long off = 0;
    for (int sp = 0; sp < h->nspin && !st; ++sp) {
      const int Ns = h->nel[sp];
      if (Ns == 0) continue;
      // G of the trial with itself: S = PsiT^H
      st = mixed_density_matrix(s, h->PsiT + long(h->el_off[sp]) * h->M, h->PsiH + off,
                                long(h->M) * Ns, G + long(h->el_off[sp]) * h->M, ldG, ov, 1, h->M,
                                Ns, true, T, nullptr, cmk(1, 0), cmk(0, 0));
      off += long(h->M) * Ns;
    }
  }
  if (!st) st = ham_vbias(h, s, G, ldG, v, 1, dt);
  if (!st) {
    cudaError_t e = cudaMemcpy(vMF_host, v, sizeof(c128) * h->Nc, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      set_error_detail("afqmc_wfn_vmf: %s", cudaGetErrorString(e));
      st = AFQMC_ERR_CUDA;
    }
  }
  dfree(G); dfree(T); dfree(ov); dfree(v);
  return st;
}

// ---------------------------------------------------------------------------------------------
// propagator
// ---------------------------------------------------------------------------------------------
extern "C" void afqmc_prop_params_default(afqmc_prop_params* p) {
  if (!p) return;
  p->dt = 0.01;
  p->taylor_n = 6;
  p->vbias_bound = 50.0;
  p->upper_cutoff_scale = 10.0;
  p->lower_cutoff_scale = 1.0;
  p->weight_bound_floor = 100.0;
  p->weight_bound_fraction = 0.1;
  p->denseP1 = 0;
  p->precision = AFQMC_PREC_FP64;
}

namespace {

// exp(A) for a small dense complex matrix on the device: Taylor series of A / 2^s to 24 terms
// (||A/2^s||_1 <= 1/2, truncation below 1e-25) followed by s squarings.
int expm_device(const std::vector<c128>& A, int M, std::vector<c128>& out) {
  const long MM = long(M) * M;
  double norm1 = 0;
  for (int j = 0; j < M; ++j) {
    double c = 0;
    for (int i = 0; i < M; ++i) c += cabs(A[size_t(i) * M + j]);
    norm1 = c > norm1 ? c : norm1;
  }
  int sq = 0;
  while (norm1 / std::ldexp(1.0, sq) > 0.5) ++sq;
  const double f = std::ldexp(1.0, -sq);
  std::vector<c128> As(static_cast<size_t>(MM)), Id(size_t(MM), cmk(0, 0));
  for (long e = 0; e < MM; ++e) As[e] = cscale(A[e], f);
  for (int i = 0; i < M; ++i) Id[size_t(i) * M + i] = cmk(1, 0);
  c128 *dA = nullptr, *dE = nullptr, *dT0 = nullptr, *dT1 = nullptr;
  int st = dalloc(&dA, size_t(MM));
  if (!st) st = dalloc(&dE, size_t(MM));
  if (!st) st = dalloc(&dT0, size_t(MM));
  if (!st) st = dalloc(&dT1, size_t(MM));
  if (!st) {
    cudaMemcpy(dA, As.data(), sizeof(c128) * MM, cudaMemcpyHostToDevice);
    cudaMemcpy(dE, Id.data(), sizeof(c128) * MM, cudaMemcpyHostToDevice);
    cudaMemcpy(dT0, Id.data(), sizeof(c128) * MM, cudaMemcpyHostToDevice);
    c128 *prev = dT0, *next = dT1;
    for (int k = 1; k <= 24 && !st; ++k) {
      GemmParams p{};
      p.m = M; p.n = M; p.k = M;
      p.A = prev; p.lda = M; p.B = dA; p.ldb = M; p.C = next; p.ldc = M;
      p.alpha = cmk(1.0 / k, 0); p.beta = cmk(0, 0);
      p.D = dE; p.ldd = M; p.d_store = false;
      st = zgemm(nullptr, 1, GN, false, GN, false, p);
      std::swap(prev, next);
    }
    for (int k = 0; k < sq && !st; ++k) {
      GemmParams p{};
      p.m = M; p.n = M; p.k = M;
      p.A = dE; p.lda = M; p.B = dE; p.ldb = M; p.C = dT0; p.ldc = M;
      p.alpha = cmk(1, 0); p.beta = cmk(0, 0);
      st = zgemm(nullptr, 1, GN, false, GN, false, p);
      if (!st) cudaMemcpy(dE, dT0, sizeof(c128) * MM, cudaMemcpyDeviceToDevice);
    }
    out.resize(size_t(MM));
    if (!st) {
      cudaError_t e = cudaMemcpy(out.data(), dE, sizeof(c128) * MM, cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        set_error_detail("expm_device: %s", cudaGetErrorString(e));
        st = AFQMC_ERR_CUDA;
      }
    }
  }
  dfree(dA); dfree(dE); dfree(dT0); dfree(dT1);
  return st;
}

}  // namespace

// vMF (given on the host, or the trial's own), P1 and their device copies: the setup part of
// AFQMCBasePropagator's constructor and generateP1 (AFQMCBasePropagator.cpp:85-214)
static int prop_mean_field(afqmc_prop_s* pr, const c128* vMF_host) {
  afqmc_ham_s* h = pr->ham;
  const afqmc_prop_params* params = &pr->p;
  const int M = h->M, Nc = h->Nc;
  const long MM = long(M) * M;
  const double dt = params->dt;
  // vMF with the imaginary part zeroed (AFQMCBasePropagator.cpp:85-110)
  pr->vMF_h.resize(Nc);
  if (vMF_host)
    std::copy(vMF_host, vMF_host + Nc, pr->vMF_h.begin());
  else
    AFQMC_TRY(afqmc_wfn_vmf(h, dt, (afqmc_c128*)pr->vMF_h.data()));
  double re2 = 0;
  for (auto& v : pr->vMF_h) {
    v.y = 0.0;
    re2 += v.x * v.x;
  }
  pr->mf0 = -0.5 * re2;
  // H1 = dt (h + v0) + vHS(vMF); hermitize; x(-1/2); P1 = exp  (cpp:119-159)
  const int nspin = h->nspin;
  std::vector<c128> H1(size_t(nspin) * MM);
  AFQMC_TRY(afqmc_ham_one_body_propagator(h, dt, (const afqmc_c128*)pr->vMF_h.data(),
                                          (afqmc_c128*)H1.data()));
  pr->P1_h.resize(size_t(nspin) * MM);
  for (int s = 0; s < nspin; ++s) {
    std::vector<c128> A(H1.begin() + s * MM, H1.begin() + (s + 1) * MM);
    for (int i = 0; i < M; ++i)
      for (int j = i; j < M; ++j) {
        if (i == j) {
          A[size_t(i) * M + i].y = 0.0;
        } else {
          c128 aij = A[size_t(i) * M + j], aji = A[size_t(j) * M + i];
          c128 v = cmk(0.5 * aij.x + 0.5 * aji.x, 0.5 * aij.y - 0.5 * aji.y);
          A[size_t(i) * M + j] = v;
          A[size_t(j) * M + i] = cconj(v);
        }
      }
    for (auto& v : A) v = cscale(v, -0.5);
    std::vector<c128> P;
    AFQMC_TRY(expm_device(A, M, P));
    std::copy(P.begin(), P.end(), pr->P1_h.begin() + s * MM);
  }
  // CSR-like truncation |x| > 1e-8 unless denseP1; a real P1 is applied in real arithmetic
  bool real = true;
  if (!params->denseP1) {
    double vmax = 0, imax = 0;
    for (auto& v : pr->P1_h) {
      if (cabs(v) > 1e-8) {
        vmax = std::max(vmax, cabs(v));
        imax = std::max(imax, std::fabs(v.y));
      } else {
        v = cmk(0, 0);
      }
    }
    real = imax <= 1e-14 * vmax;
    if (real)
      for (auto& v : pr->P1_h) v.y = 0.0;
  } else {
    for (auto& v : pr->P1_h) real = real && v.y == 0.0;
  }
  pr->p1_real = real;
  pr->nspin_P1 = nspin;
  pr->nspin_V = h->walker_type == AFQMC_COLLINEAR ? h->nspin_H2 : 1;
  dfree(pr->P1);
  dfree(pr->P1r);
  dfree(pr->vMF);
  AFQMC_TRY(dalloc(&pr->P1, size_t(nspin) * MM));
  AFQMC_CUDA_TRY(cudaMemcpy(pr->P1, pr->P1_h.data(), sizeof(c128) * nspin * MM,
                            cudaMemcpyHostToDevice));
  if (real) {
    std::vector<double> pr_h(size_t(nspin) * MM);
    for (size_t e = 0; e < pr_h.size(); ++e) pr_h[e] = pr->P1_h[e].x;
    AFQMC_TRY(dalloc(&pr->P1r, pr_h.size()));
    AFQMC_CUDA_TRY(cudaMemcpy(pr->P1r, pr_h.data(), sizeof(double) * pr_h.size(),
                              cudaMemcpyHostToDevice));
  }
  AFQMC_TRY(dalloc(&pr->vMF, size_t(Nc)));
  AFQMC_CUDA_TRY(cudaMemcpy(pr->vMF, pr->vMF_h.data(), sizeof(c128) * Nc, cudaMemcpyHostToDevice));
  return AFQMC_OK;
}

extern "C" int afqmc_prop_create(afqmc_ham h, const afqmc_prop_params* params, int max_walkers,
                                 afqmc_prop* out) {
  AFQMC_CHECK_ARG(h && params && out && max_walkers > 0, "afqmc_prop_create: bad argument");
  *out = nullptr;
  AFQMC_CHECK_ARG(params->dt > 0 && params->taylor_n >= 0, "afqmc_prop_create: bad dt / order");
  AFQMC_CHECK_ARG(params->precision == AFQMC_PREC_FP64 || params->precision == AFQMC_PREC_MIXED,
                  "afqmc_prop_create: unknown precision");
  DeviceGuard g(h->device);
  std::unique_ptr<afqmc_prop_s> pr(new (std::nothrow) afqmc_prop_s());
  AFQMC_CHECK_ARG(pr, "afqmc_prop_create: out of host memory");
  pr->device = h->device;
  pr->ham = h;
  pr->p = *params;
  pr->maxW = max_walkers;
  const int M = h->M, Nc = h->Nc;
  const long MM = long(M) * M;

  AFQMC_TRY(prop_mean_field(pr.get(), nullptr));

  // step workspace
  const int W = max_walkers;
  const long ldG = long(h->nel_tot) * M;
  int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
  AFQMC_TRY(dalloc(&pr->G, size_t(W) * (ldG > 0 ? ldG : 1)));
  AFQMC_TRY(dalloc(&pr->vb, size_t(W) * Nc));
  AFQMC_TRY(dalloc(&pr->X, size_t(W) * Nc));
  AFQMC_TRY(dalloc(&pr->HW, size_t(W)));
  AFQMC_TRY(dalloc(&pr->mf, size_t(W)));
  AFQMC_TRY(dalloc(&pr->newov, size_t(W)));
  AFQMC_TRY(dalloc(&pr->ovtmp, size_t(W)));
  AFQMC_TRY(dalloc(&pr->T, size_t(W) * (nmax > 0 ? nmax * nmax : 1)));
  AFQMC_TRY(dalloc(&pr->V, size_t(pr->nspin_V) * W * MM));
  AFQMC_TRY(dalloc(&pr->w1, size_t(W) * M * (nmax > 0 ? nmax : 1)));
  AFQMC_TRY(dalloc(&pr->w2, size_t(W) * M * (nmax > 0 ? nmax : 1)));
  AFQMC_TRY(dalloc(&pr->w3, size_t(W) * M * (nmax > 0 ? nmax : 1)));
  AFQMC_TRY(dalloc(&pr->ortho_work, size_t(W) * M * (nmax > 0 ? nmax : 1) +
                                        2 * size_t(W) * (nmax > 0 ? nmax * nmax : 1)));
  AFQMC_TRY(dalloc(&pr->Eshift_d, 1));
  AFQMC_TRY(dalloc(&pr->counter, 1));
  AFQMC_TRY(dalloc(&pr->stats, 8));
  AFQMC_CUDA_TRY(cudaMemset(pr->counter, 0, sizeof(unsigned long long)));
  AFQMC_CUDA_TRY(cudaMemset(pr->stats, 0, 8 * sizeof(unsigned long long)));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = pr.release();
  return AFQMC_OK;
}

extern "C" int afqmc_prop_destroy(afqmc_prop prop) {
  delete prop;
  return AFQMC_OK;
}

extern "C" int afqmc_prop_set_phmsd(afqmc_prop pr, afqmc_phmsd trial, const afqmc_c128* vMF) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_set_phmsd: null handle");
  AFQMC_CHECK_ARG(!trial || !pr->ham->thc,
                  "afqmc_prop_set_phmsd: a THC Hamiltonian takes one determinant (as THCOps)");
  DeviceGuard g(pr->device);
  if (!trial) {
    pr->ph = nullptr;
    dfree(pr->Gph);
    return vMF ? prop_mean_field(pr, reinterpret_cast<const c128*>(vMF)) : AFQMC_OK;
  }
  afqmc_ham_s* h = pr->ham;
  int d[6];
  AFQMC_TRY(afqmc_phmsd_info(trial, d));
  AFQMC_CHECK_ARG(h->walker_type == AFQMC_COLLINEAR,
                  "afqmc_prop_set_phmsd: a PHMSD trial needs COLLINEAR walkers");
  AFQMC_CHECK_ARG(d[0] == h->M && d[1] == h->nel[0] && d[2] == h->nel[1],
                  "afqmc_prop_set_phmsd: trial (M=%d, %d+%d) does not match the Hamiltonian "
                  "(M=%d, %d+%d)", d[0], d[1], d[2], h->M, h->nel[0], h->nel[1]);
  AFQMC_CHECK_ARG(d[5] == h->Nc,
                  "afqmc_prop_set_phmsd: trial Hamiltonian has %d Cholesky vectors, the "
                  "propagator %d (afqmc_phmsd_set_hamiltonian first)", d[5], h->Nc);
  AFQMC_CHECK_ARG(!pr->md, "afqmc_prop_set_phmsd: a multi-determinant NOMSD trial is attached");
  dfree(pr->Gph);
  AFQMC_TRY(dalloc(&pr->Gph, size_t(pr->maxW) * (d[3] + d[4]) * h->M));
  if (vMF) AFQMC_TRY(prop_mean_field(pr, reinterpret_cast<const c128*>(vMF)));
  pr->ph = trial;
  return AFQMC_OK;
}

extern "C" int afqmc_prop_set_nomsd(afqmc_prop pr, afqmc_nomsd trial, const afqmc_c128* vMF) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_set_nomsd: null handle");
  DeviceGuard g(pr->device);
  if (!trial) {
    pr->md = nullptr;
    dfree(pr->Gfull);
    return vMF ? prop_mean_field(pr, reinterpret_cast<const c128*>(vMF)) : AFQMC_OK;
  }
  afqmc_ham_s* h = pr->ham;
  afqmc_ham_s* t = trial->hams[0];
  AFQMC_CHECK_ARG(t->walker_type == h->walker_type && t->M == h->M && t->Nc == h->Nc &&
                      t->nel[0] == h->nel[0] && t->nel[1] == h->nel[1],
                  "afqmc_prop_set_nomsd: trial and propagator Hamiltonians differ in shape");
  AFQMC_CHECK_ARG(pr->p.precision == AFQMC_PREC_FP64,
                  "afqmc_prop_set_nomsd: multi-determinant steps run in FP64");
  AFQMC_CHECK_ARG(!pr->ph, "afqmc_prop_set_nomsd: a PHMSD trial is attached");
  dfree(pr->Gfull);
  AFQMC_TRY(dalloc(&pr->Gfull, size_t(pr->maxW) * h->nspin * h->M * h->M));
  if (vMF) AFQMC_TRY(prop_mean_field(pr, reinterpret_cast<const c128*>(vMF)));
  pr->md = trial;
  return AFQMC_OK;
}

extern "C" int afqmc_prop_get_p1(afqmc_prop pr, afqmc_c128* P1, afqmc_c128* vMF) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_get_p1: null handle");
  if (P1) std::memcpy(P1, pr->P1_h.data(), sizeof(c128) * pr->P1_h.size());
  if (vMF) std::memcpy(vMF, pr->vMF_h.data(), sizeof(c128) * pr->vMF_h.size());
  return AFQMC_OK;
}

extern "C" int afqmc_prop_set_field_seed(afqmc_prop pr, unsigned long long seed) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_set_field_seed: null handle");
  DeviceGuard g(pr->device);
  pr->seed = seed;
  AFQMC_CUDA_TRY(cudaMemset(pr->counter, 0, sizeof(unsigned long long)));
  return AFQMC_OK;
}

namespace {

int prop_step(afqmc_prop_s* pr, afqmc_wset_s* ws, double Eshift, const double* Eshift_dev,
              const double* uniforms, int flags, cudaStream_t s) {
  afqmc_ham_s* h = pr->ham;
  auto mark = [&](int i) -> int {
    if (pr->timing) AFQMC_CUDA_TRY(cudaEventRecord(pr->ev[i], s));
    return AFQMC_OK;
  };
  AFQMC_TRY(mark(0));
  const int W = ws->W, M = h->M, Nc = h->Nc;
  const double dt = pr->p.dt;
  const long ldG = long(h->nel_tot) * M;
  const bool mixed_any = pr->p.precision == AFQMC_PREC_MIXED;
  const bool mixed_v = mixed_any && (h->mixed_ops & AFQMC_MIXED_VBIAS);
  const bool mixed = mixed_any && (h->mixed_ops & AFQMC_MIXED_PROPAGATION);
  const bool mixed_vhs_only = mixed_any && !mixed && (h->mixed_ops & AFQMC_MIXED_VHS) &&
                              h->nspin_H2 == 1;
  // 1. vbias: G of the walkers (NOMSD::vbias, NOMSD.cpp:39-61); with AFQMC_STEP_G_READY the
  //    previous step left it for these walkers
  if (pr->md) {
    // NOMSD::vbias with several determinants (NOMSD.cpp:39-61): the full G, then Likn . G
    AFQMC_TRY(nomsd_density_matrix(pr->md, ws, s, pr->Gfull, pr->ovtmp));
    AFQMC_TRY(mark(1));
    AFQMC_TRY(nomsd_vbias(h, s, pr->Gfull, pr->vb, W, dt));
  } else if (pr->ph) {
    // PHMSD::vbias (PHMSD.cpp:54-72): the multi-determinant density matrix, then Lnak . G
    AFQMC_TRY(afqmc_phmsd_density_matrix(pr->ph, (const afqmc_c128*)ws->buf, ws->walker_size,
                                         (afqmc_c128*)pr->Gph, (afqmc_c128*)pr->ovtmp, W, 0,
                                         (afqmc_stream)s));
    AFQMC_TRY(mark(1));
    AFQMC_TRY(afqmc_phmsd_vbias(pr->ph, (const afqmc_c128*)pr->Gph, (afqmc_c128*)pr->vb, W, dt,
                                (afqmc_stream)s));
  } else {
    if (!(flags & AFQMC_STEP_G_READY))
      AFQMC_TRY(wfn_density_matrix(h, ws, s, pr->G, ldG, pr->ovtmp, pr->T));
    AFQMC_TRY(mark(1));
  }
  if (pr->ph || pr->md) {
    // vbias done above
  } else if (mixed_v) {
    EnergyArgs a = energy_args(h, pr->G, ldG);
    if (!h->mixed) AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    AFQMC_TRY(vbias_mixed(s, h->mixed, pr->G, ldG, pr->vb, W,
                          std::sqrt(dt) * (h->walker_type == AFQMC_CLOSED ? 2.0 : 1.0)));
  } else {
    AFQMC_TRY(ham_vbias(h, s, pr->G, ldG, pr->vb, W, dt));
  }
  AFQMC_TRY(mark(2));
  // 2. X, HW, mf
  AFQMC_TRY(construct_x(s, pr->vb, Nc, uniforms, Nc, pr->vMF, pr->X, Nc, pr->HW, pr->mf, W, Nc,
                        pr->p.vbias_bound, pr->mf0, pr->seed, pr->counter));
  AFQMC_TRY(mark(3));
  // 3. vHS
  if (mixed) {
    // (with a multi-determinant trial the vbias above ran through the trial, in complex128, and
    // the mixed tensors may not exist yet)
    if (!h->mixed) {
      EnergyArgs a = energy_args(h, pr->G, ldG);
      AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    }
    AFQMC_TRY(vhs_mixed(s, h->mixed, pr->X, nullptr, W, std::sqrt(dt)));
  } else if (mixed_vhs_only) {
    if (!h->mixed) {
      EnergyArgs a = energy_args(h, pr->G, ldG);
      AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
    }
    AFQMC_TRY(vhs_mixed(s, h->mixed, pr->X, pr->V, W, std::sqrt(dt)));
  } else {
    AFQMC_TRY(ham_vhs(h, s, pr->X, pr->V, W, dt));
  }
  AFQMC_TRY(mark(4));
  // 4. propagate each spin block
  const long MM = long(M) * M;
  for (int sp = 0; sp < h->nspin; ++sp) {
    const int Ns = h->nel[sp];
    if (Ns == 0) continue;
    const void* P1 = pr->p1_real ? (const void*)(pr->P1r + size_t(sp % pr->nspin_P1) * MM)
                                 : (const void*)(pr->P1 + size_t(sp % pr->nspin_P1) * MM);
    const c128* V = pr->V + size_t(sp % pr->nspin_V) * W * MM;
    if (mixed) {
      AFQMC_TRY(propagate_mixed(s, h->mixed, P1, pr->p1_real, ws->buf + ws->offS(sp),
                                ws->walker_size, W, M, Ns, pr->p.taylor_n));
    } else {
      AFQMC_TRY(propagate(s, P1, pr->p1_real, V, MM, ws->buf + ws->offS(sp), ws->walker_size, W, M,
                          Ns, pr->p.taylor_n, pr->w1, pr->w2, pr->w3));
    }
  }
  AFQMC_TRY(mark(5));
  // 5. new overlaps; with AFQMC_STEP_KEEP_G also the density matrix of the propagated walkers
  //    for the next step (the same product, LU and log det, plus the inverse and G)
  if (pr->md)
    AFQMC_TRY(nomsd_log_overlap(pr->md, ws, s, pr->newov));
  else if (pr->ph)
    AFQMC_TRY(afqmc_phmsd_log_overlap(pr->ph, (const afqmc_c128*)ws->buf, ws->walker_size,
                                      (afqmc_c128*)pr->newov, W, (afqmc_stream)s));
  else if (flags & AFQMC_STEP_KEEP_G)
    AFQMC_TRY(wfn_density_matrix(h, ws, s, pr->G, ldG, pr->newov, pr->T));
  else
    AFQMC_TRY(wfn_log_overlap(h, ws, s, pr->newov, pr->T));
  AFQMC_TRY(mark(6));
  // 6-7. walker_update + bound_walker_weights
  const double max_weight = std::max(pr->p.weight_bound_floor, pr->p.weight_bound_fraction * W);
  AFQMC_TRY(walker_update(s, ws->buf, ws->walker_size, ws->prop0, W, pr->newov, pr->mf, pr->HW,
                          dt, Eshift, Eshift_dev, h->E0, pr->p.lower_cutoff_scale,
                          pr->p.upper_cutoff_scale, max_weight, pr->stats));
  return mark(7);
}

}  // namespace

extern "C" int afqmc_prop_step(afqmc_prop pr, afqmc_wset ws, double Eshift, const double* u,
                               afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws, "afqmc_prop_step: null handle");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_step: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ws->W <= pr->maxW, "afqmc_prop_step: %d walkers exceed the propagator's %d",
                  ws->W, pr->maxW);
  DeviceGuard g(pr->device);
  return prop_step(pr, ws, Eshift, nullptr, u, 0, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int afqmc_prop_step_dev(afqmc_prop pr, afqmc_wset ws, const double* Eshift_dev,
                                   const double* u, afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws && Eshift_dev, "afqmc_prop_step_dev: null argument");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_step_dev: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ws->W <= pr->maxW, "afqmc_prop_step_dev: too many walkers");
  DeviceGuard g(pr->device);
  return prop_step(pr, ws, 0.0, Eshift_dev, u, 0, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int afqmc_prop_step_flags(afqmc_prop pr, afqmc_wset ws, const double* Eshift_dev,
                                     const double* u, int flags, afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws && Eshift_dev, "afqmc_prop_step_flags: null argument");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_step_flags: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ws->W <= pr->maxW, "afqmc_prop_step_flags: too many walkers");
  AFQMC_CHECK_ARG((flags & ~(AFQMC_STEP_G_READY | AFQMC_STEP_KEEP_G)) == 0,
                  "afqmc_prop_step_flags: unknown flags %d", flags);
  AFQMC_CHECK_ARG(!((pr->ph || pr->md) && flags),
                  "afqmc_prop_step_flags: no density reuse with a multi-determinant trial");
  DeviceGuard g(pr->device);
  return prop_step(pr, ws, 0.0, Eshift_dev, u, flags, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int afqmc_prop_autotune(afqmc_prop pr, afqmc_wset ws, int* best, float* ms,
                                   afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws && best, "afqmc_prop_autotune: null argument");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_autotune: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ws->W <= pr->maxW, "afqmc_prop_autotune: too many walkers");
  DeviceGuard g(pr->device);
  afqmc_ham_s* h = pr->ham;
  *best = -1;
  if (pr->p.precision != AFQMC_PREC_MIXED || pr->ph || pr->md) return AFQMC_OK;  // no choice
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t nbuf = size_t(ws->W) * ws->walker_size;
  // the state a step changes: walkers (with their properties), the field counter, the bound
  // statistics; saved here and restored after every trial, so that tuning leaves no trace
  Scratch save, aux;
  AFQMC_TRY(save.get(sizeof(c128) * nbuf, s));
  AFQMC_TRY(aux.get(sizeof(unsigned long long) * 9, s));
  unsigned long long* auxp = reinterpret_cast<unsigned long long*>(aux.p);
  AFQMC_CUDA_TRY(cudaMemcpyAsync(save.p, ws->buf, sizeof(c128) * nbuf, cudaMemcpyDeviceToDevice, s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(auxp, pr->counter, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(auxp + 1, pr->stats, 8 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, s));
  auto restore = [&]() -> int {
    AFQMC_CUDA_TRY(cudaMemcpyAsync(ws->buf, save.p, sizeof(c128) * nbuf, cudaMemcpyDeviceToDevice, s));
    AFQMC_CUDA_TRY(cudaMemcpyAsync(pr->counter, auxp, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToDevice, s));
    AFQMC_CUDA_TRY(cudaMemcpyAsync(pr->stats, auxp + 1, 8 * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToDevice, s));
    return AFQMC_OK;
  };
  cudaEvent_t e0, e1;
  AFQMC_CUDA_TRY(cudaEventCreate(&e0));
  AFQMC_CUDA_TRY(cudaEventCreate(&e1));
  // Taylor propagation variants: 0 per-term GEMMs; fused: 2 / 3 TF32 split with one / two
  // walkers in flight per CTA, 4 / 5 the same in the FP16 split (when the shapes allow it), 6 / 7
  // one walker in flight with the running sum in tensor memory.  Every variant is timed; the
  // choice is among 2 and 4, whose small split products have their own accumulator (the others
  // accumulate three times as many updates in one FP32 accumulator, whose truncation toward zero
  // shifts the mixed-estimator energy).
  const int modes[7] = {0, 2, 3, 4, 5, 6, 7};
  float best_ms = 1e30f;
  int st = AFQMC_OK;
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    st = mixed_ham_create(&h->mixed, a, s);
  }
  const bool f16 = !st && mixed_taylor_f16_ok(h->mixed);
  for (int mi = 0; mi < 7; ++mi)
    if (ms) ms[mi] = 0.f;
  for (int mi = 0; mi < 7 && !st; ++mi) {
    const int md = modes[mi];
    if (!f16 && (md == 4 || md == 5 || md == 7)) continue;
    if ((st = mixed_set_taylor_mode(h->mixed, modes[mi]))) break;
    float t = 0.f;
    for (int rep = 0; rep < 3 && !st; ++rep) {  // the first repetition warms up
      if ((st = restore())) break;
      if (rep > 0 && cudaEventRecord(e0, s) != cudaSuccess) st = AFQMC_ERR_CUDA;
      if (!st) st = prop_step(pr, ws, 0.0, nullptr, nullptr, 0, s);
      if (!st && rep > 0) {
        float x = 0.f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&x, e0, e1) != cudaSuccess)
          st = AFQMC_ERR_CUDA;
        t += x;
      }
    }
    if (ms) ms[mi] = t / 2;
    if (!st && (md == 2 || md == 4) && t / 2 < best_ms) {
      best_ms = t / 2;
      *best = md;
    }
  }
  if (!st && *best >= 0) st = mixed_set_taylor_mode(h->mixed, *best);
  const int st2 = restore();
  if (cudaStreamSynchronize(s) != cudaSuccess && !st) st = AFQMC_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st ? st : st2;
}

// Tile shapes and orders of the mixed-precision contractions that leave every result bit for bit
// the same, timed on the live walkers (state restored): the vbias CTA tile width (128 / 64
// Cholesky vectors, one step each), the vHS form (i <= k pairs mirrored / all pairs, when the
// Cholesky vectors are symmetric; one step each) and the exchange kernel's L2 block (16 / 32 / 64
// / 128 vector pairs, one energy evaluation each).  choice [3] = the kept (bn, symmetric, block);
// ms [8] = the times in that order (0 for a candidate not run).
extern "C" int afqmc_prop_autotune_tiles(afqmc_prop pr, afqmc_wset ws, int* choice, float* ms,
                                         afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws && choice, "afqmc_prop_autotune_tiles: null argument");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_autotune_tiles: walker set / Hamiltonian mismatch");
  AFQMC_CHECK_ARG(ws->W <= pr->maxW, "afqmc_prop_autotune_tiles: too many walkers");
  DeviceGuard g(pr->device);
  afqmc_ham_s* h = pr->ham;
  for (int k = 0; k < 8; ++k)
    if (ms) ms[k] = 0.f;
  choice[0] = choice[1] = choice[2] = -1;
  if (pr->p.precision != AFQMC_PREC_MIXED || pr->ph || pr->md) return AFQMC_OK;  // no choice
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, s));
  }
  MixedHam* m = h->mixed;
  const size_t nbuf = size_t(ws->W) * ws->walker_size;
  Scratch save, aux;
  AFQMC_TRY(save.get(sizeof(c128) * nbuf, s));
  AFQMC_TRY(aux.get(sizeof(unsigned long long) * 9, s));
  unsigned long long* auxp = reinterpret_cast<unsigned long long*>(aux.p);
  AFQMC_CUDA_TRY(cudaMemcpyAsync(save.p, ws->buf, sizeof(c128) * nbuf, cudaMemcpyDeviceToDevice, s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(auxp, pr->counter, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, s));
  AFQMC_CUDA_TRY(cudaMemcpyAsync(auxp + 1, pr->stats, 8 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToDevice, s));
  auto restore = [&]() -> int {
    AFQMC_CUDA_TRY(cudaMemcpyAsync(ws->buf, save.p, sizeof(c128) * nbuf, cudaMemcpyDeviceToDevice, s));
    AFQMC_CUDA_TRY(cudaMemcpyAsync(pr->counter, auxp, sizeof(unsigned long long),
                                   cudaMemcpyDeviceToDevice, s));
    AFQMC_CUDA_TRY(cudaMemcpyAsync(pr->stats, auxp + 1, 8 * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToDevice, s));
    return AFQMC_OK;
  };
  cudaEvent_t e0, e1;
  AFQMC_CUDA_TRY(cudaEventCreate(&e0));
  AFQMC_CUDA_TRY(cudaEventCreate(&e1));
  // mean time of `body` over two runs after one warm-up run, each from the restored state
  auto timed = [&](auto&& body, float* out) -> int {
    float t = 0.f;
    for (int rep = 0; rep < 3; ++rep) {
      AFQMC_TRY(restore());
      if (rep > 0 && cudaEventRecord(e0, s) != cudaSuccess) return AFQMC_ERR_CUDA;
      AFQMC_TRY(body());
      if (rep > 0) {
        float x = 0.f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&x, e0, e1) != cudaSuccess)
          return AFQMC_ERR_CUDA;
        t += x;
      }
    }
    *out = t / 2;
    return AFQMC_OK;
  };
  auto step = [&]() -> int { return prop_step(pr, ws, 0.0, nullptr, nullptr, 0, s); };
  int st = AFQMC_OK;
  int bn0 = 128, blk0 = 64;
  mixed_get_tiles(m, &bn0, &blk0);
  // vbias tile width
  {
    const int cand[2] = {128, 64};
    float best = 1e30f;
    for (int k = 0; k < 2 && !st; ++k) {
      float t = 0.f;
      if (!(st = mixed_set_tiles(m, cand[k], blk0)) && !(st = timed(step, &t))) {
        if (ms) ms[k] = t;
        if (t < best) {
          best = t;
          choice[0] = cand[k];
        }
      }
    }
    if (!st) st = mixed_set_tiles(m, choice[0], blk0);
  }
  // vHS form (only when the symmetric one is available)
  if (!st) {
    int active = 0;
    st = mixed_set_vhs_symmetry(m, 1, &active);
    if (!st && active) {
      float t1 = 0.f, t0 = 0.f;
      if (!(st = timed(step, &t1)) && !(st = mixed_set_vhs_symmetry(m, 0, &active)) &&
          !(st = timed(step, &t0))) {
        if (ms) {
          ms[2] = t1;
          ms[3] = t0;
        }
        choice[1] = t1 <= t0 ? 1 : 0;
        st = mixed_set_vhs_symmetry(m, choice[1], &active);
      }
    } else if (!st) {
      choice[1] = 0;
    }
  }
  // exchange L2 block, on the walkers' own density matrix
  if (!st) {
    const int W = ws->W;
    const long ldG = long(h->nel_tot) * h->M;
    const int nmax = h->nel[0] > h->nel[1] ? h->nel[0] : h->nel[1];
    Scratch Gb, Tb, ov, E;
    if (!(st = Gb.get(sizeof(c128) * size_t(W) * ldG, s)) &&
        !(st = Tb.get(sizeof(c128) * size_t(W) * nmax * nmax, s)) &&
        !(st = ov.get(sizeof(c128) * size_t(W), s)) && !(st = E.get(sizeof(c128) * 3 * size_t(W), s)))
      st = wfn_density_matrix(h, ws, s, (c128*)Gb.p, ldG, (c128*)ov.p, (c128*)Tb.p);
    const int cand[4] = {16, 32, 64, 128};
    float best = 1e30f;
    for (int k = 0; k < 4 && !st; ++k) {
      auto energy = [&]() -> int {
        return ham_energy(h, s, (const c128*)Gb.p, ldG, (c128*)E.p, W, true, true, true,
                          AFQMC_PREC_MIXED);
      };
      float t = 0.f;
      if (!(st = mixed_set_tiles(m, choice[0], cand[k])) && !(st = timed(energy, &t))) {
        if (ms) ms[4 + k] = t;
        if (t < best) {
          best = t;
          choice[2] = cand[k];
        }
      }
    }
    if (!st) st = mixed_set_tiles(m, choice[0], choice[2]);
  }
  const int st2 = restore();
  if (cudaStreamSynchronize(s) != cudaSuccess && !st) st = AFQMC_ERR_CUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return st ? st : st2;
}

// the current tile choices of the mixed-precision contractions (vbias tile width, exchange block)
extern "C" int afqmc_ham_get_tiles(afqmc_ham h, int* vbias_bn, int* exchange_block) {
  AFQMC_CHECK_ARG(h && vbias_bn && exchange_block, "afqmc_ham_get_tiles: null argument");
  *vbias_bn = 128;
  *exchange_block = 64;
  if (h->mixed) mixed_get_tiles(h->mixed, vbias_bn, exchange_block);
  return AFQMC_OK;
}

// set the tile choices by hand (bn 128 / 64, block >= 1; results are the same bit for bit)
extern "C" int afqmc_ham_set_tiles(afqmc_ham h, int vbias_bn, int exchange_block) {
  AFQMC_CHECK_ARG(h, "afqmc_ham_set_tiles: null argument");
  DeviceGuard g(h->device);
  if (!h->mixed) {
    EnergyArgs a = energy_args(h, nullptr, 0);
    AFQMC_TRY(mixed_ham_create(&h->mixed, a, nullptr));
  }
  return mixed_set_tiles(h->mixed, vbias_bn, exchange_block);
}

extern "C" int afqmc_prop_orthogonalize(afqmc_prop pr, afqmc_wset ws, afqmc_stream stream) {
  AFQMC_CHECK_ARG(pr && ws, "afqmc_prop_orthogonalize: null handle");
  AFQMC_CHECK_ARG(wset_matches(pr->ham, ws), "afqmc_prop_orthogonalize: mismatch");
  DeviceGuard g(pr->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  afqmc_ham_s* h = pr->ham;
  AFQMC_CUDA_TRY(cudaMemsetAsync(pr->ovtmp, 0, sizeof(c128) * ws->W, s));
  for (int sp = 0; sp < h->nspin; ++sp) {
    if (h->nel[sp] == 0) continue;
    AFQMC_TRY(orthogonalize(s, ws->buf + ws->offS(sp), ws->walker_size, pr->ovtmp, ws->W, h->M,
                            h->nel[sp], pr->ortho_work));
  }
  if (pr->md)
    AFQMC_TRY(nomsd_log_overlap(pr->md, ws, s, pr->newov));
  else if (pr->ph)
    AFQMC_TRY(afqmc_phmsd_log_overlap(pr->ph, (const afqmc_c128*)ws->buf, ws->walker_size,
                                      (afqmc_c128*)pr->newov, ws->W, (afqmc_stream)s));
  else
    AFQMC_TRY(wfn_log_overlap(h, ws, s, pr->newov, pr->T));
  return scatter_property(s, ws->buf, ws->walker_size, ws->prop0 + AFQMC_OVLP, ws->W, pr->newov);
}

extern "C" int afqmc_prop_last_step(afqmc_prop pr, const afqmc_c128** vbias, const afqmc_c128** X,
                                    const afqmc_c128** hw, const afqmc_c128** mf,
                                    const afqmc_c128** new_ovlp) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_last_step: null handle");
  if (vbias) *vbias = (const afqmc_c128*)pr->vb;
  if (X) *X = (const afqmc_c128*)pr->X;
  if (hw) *hw = (const afqmc_c128*)pr->HW;
  if (mf) *mf = (const afqmc_c128*)pr->mf;
  if (new_ovlp) *new_ovlp = (const afqmc_c128*)pr->newov;
  return AFQMC_OK;
}

extern "C" int afqmc_prop_set_timing(afqmc_prop pr, int enable) {
  AFQMC_CHECK_ARG(pr, "afqmc_prop_set_timing: null handle");
  DeviceGuard g(pr->device);
  if (enable && !pr->ev[0])
    for (auto& e : pr->ev) AFQMC_CUDA_TRY(cudaEventCreate(&e));
  pr->timing = enable != 0;
  return AFQMC_OK;
}

extern "C" int afqmc_prop_timings(afqmc_prop pr, double* ms) {
  AFQMC_CHECK_ARG(pr && ms, "afqmc_prop_timings: null argument");
  AFQMC_CHECK_ARG(pr->ev[0], "afqmc_prop_timings: timing was never enabled");
  DeviceGuard g(pr->device);
  AFQMC_CUDA_TRY(cudaEventSynchronize(pr->ev[AFQMC_NPHASE]));
  for (int i = 0; i < AFQMC_NPHASE; ++i) {
    float t = 0;
    AFQMC_CUDA_TRY(cudaEventElapsedTime(&t, pr->ev[i], pr->ev[i + 1]));
    ms[i] = t;
  }
  return AFQMC_OK;
}

extern "C" int afqmc_prop_bound_stats(afqmc_prop pr, long long* counts) {
  AFQMC_CHECK_ARG(pr && counts, "afqmc_prop_bound_stats: null argument");
  DeviceGuard g(pr->device);
  unsigned long long h[8];
  AFQMC_CUDA_TRY(cudaMemcpy(h, pr->stats, sizeof(h), cudaMemcpyDeviceToHost));
  counts[0] = (long long)h[0];
  counts[1] = (long long)h[1];
  counts[2] = (long long)h[2];
  counts[3] = (long long)h[3];
  counts[4] = (long long)h[4];
  counts[5] = 0;
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// population control and estimators
// ---------------------------------------------------------------------------------------------
extern "C" unsigned long long afqmc_split_seed(int seed, int rank, unsigned stream) {
  unsigned long long x = (unsigned long long)(unsigned)seed << 32 |
                         (unsigned long long)stream << 24 | (unsigned)rank;
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

extern "C" int afqmc_host_rng_create(unsigned long long seed, afqmc_host_rng* out) {
  AFQMC_CHECK_ARG(out, "afqmc_host_rng_create: null out");
  *out = new (std::nothrow) afqmc_host_rng_s{std::mt19937(std::mt19937::result_type(seed))};
  AFQMC_CHECK_ARG(*out, "afqmc_host_rng_create: out of host memory");
  return AFQMC_OK;
}

extern "C" int afqmc_host_rng_destroy(afqmc_host_rng rng) {
  delete rng;
  return AFQMC_OK;
}

extern "C" int afqmc_host_rng_uniform(afqmc_host_rng rng, double* out, long n) {
  AFQMC_CHECK_ARG(rng && (out || n == 0), "afqmc_host_rng_uniform: null argument");
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (long i = 0; i < n; ++i) out[i] = dist(rng->rng);
  return AFQMC_OK;
}

extern "C" int afqmc_comb(afqmc_host_rng rng, const double* weights, int n, int num_target,
                          int* offspring) {
  AFQMC_CHECK_ARG(rng && weights && offspring && n > 0 && num_target >= 0,
                  "afqmc_comb: bad argument");
  std::vector<double> cum(static_cast<size_t>(n));
  std::partial_sum(weights, weights + n, cum.begin());
  const double total = cum[size_t(n) - 1];
  if (!(total > 1e-6)) {
    set_error_detail("The total walker weight collapsed to %g.", total);
    return AFQMC_ERR_COLLAPSE;
  }
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  const double r = dist(rng->rng);
  int last = n - 1;
  while (weights[last] <= 0.0) --last;
  std::fill(offspring, offspring + n, 0);
  int iw = 0, ic = 0;
  while (ic < num_target) {
    const double comb = (ic + r) * total / num_target;
    if (comb < cum[size_t(iw)] || iw == last) {
      offspring[iw] += 1;
      ++ic;
    } else {
      ++iw;
    }
  }
  return AFQMC_OK;
}

extern "C" int afqmc_plan_walker_exchange(const int* offspring, const int* counts, int nranks,
                                          int* plan, int max_plan, int* nplan) {
  AFQMC_CHECK_ARG(offspring && counts && nranks > 0 && nplan, "afqmc_plan_walker_exchange: null");
  long ntot = 0, osum = 0;
  for (int r = 0; r < nranks; ++r) ntot += counts[r];
  for (long i = 0; i < ntot; ++i) osum += offspring[i];
  if (osum != ntot) {
    set_error_detail("plan_walker_exchange: offspring does not preserve the population.");
    return AFQMC_ERR_SHAPE;
  }
  struct Exp { int src, walker, copies; };
  std::vector<Exp> exports;
  std::vector<std::pair<int, int>> deficits;
  std::vector<int> order;
  for (int r = 0, first = 0; r < nranks; first += counts[r], ++r) {
    const int nw = counts[r];
    const int* local = offspring + first;
    int excess = -nw;
    for (int i = 0; i < nw; ++i) excess += local[i];
    if (excess < 0) deficits.emplace_back(r, -excess);
    if (excess <= 0) continue;
    order.resize(size_t(nw));
    for (int i = 0; i < nw; ++i) order[size_t(i)] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return local[a] > local[b]; });
    for (int k = 0; excess > 0; ++k) {
      int m = std::min(local[order[size_t(k)]], excess);
      exports.push_back({r, order[size_t(k)], m});
      excess -= m;
    }
  }
  int np = 0;
  size_t d = 0;
  for (auto e : exports) {
    while (e.copies > 0) {
      int n = std::min(e.copies, deficits[d].second);
      if (plan && np < max_plan) {
        plan[4 * np + 0] = e.src;
        plan[4 * np + 1] = e.walker;
        plan[4 * np + 2] = deficits[d].first;
        plan[4 * np + 3] = n;
      }
      ++np;
      e.copies -= n;
      deficits[d].second -= n;
      if (deficits[d].second == 0) ++d;
    }
  }
  *nplan = np;
  if (plan && np > max_plan) {
    set_error_detail("plan_walker_exchange: %d transfers exceed max_plan %d", np, max_plan);
    return AFQMC_ERR_SHAPE;
  }
  return AFQMC_OK;
}

extern "C" int afqmc_population_control(afqmc_wset ws, afqmc_host_rng rng, int* offspring_out,
                                        afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && rng, "afqmc_population_control: null handle");
  DeviceGuard g(ws->device);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int W = ws->W;
  std::vector<c128> w(static_cast<size_t>(W));
  AFQMC_CUDA_TRY(cudaMemcpy2DAsync(w.data(), sizeof(c128), ws->buf + ws->prop0 + AFQMC_WEIGHT,
                                   ws->walker_size * sizeof(c128), sizeof(c128), W,
                                   cudaMemcpyDeviceToHost, s));
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  std::vector<double> absw(static_cast<size_t>(W));
  for (int i = 0; i < W; ++i) absw[size_t(i)] = std::abs(cplx(w[size_t(i)].x, w[size_t(i)].y));
  std::vector<int> off(static_cast<size_t>(W));
  AFQMC_TRY(afqmc_comb(rng, absw.data(), W, W, off.data()));
  if (offspring_out) std::memcpy(offspring_out, off.data(), sizeof(int) * W);
  // single-rank swap_walkers_async: a walker keeps its slot; extra copies fill the slots of the
  // walkers without offspring in increasing order (population_control.hpp:142-209)
  std::vector<int> freeslots;
  for (int i = 0; i < W; ++i)
    if (off[size_t(i)] == 0) freeslots.push_back(i);
  std::vector<int> pairs;  // [dst..., src...]
  std::vector<int> dst, src;
  size_t nxt = 0;
  for (int i = 0; i < W; ++i)
    for (int c = 1; c < off[size_t(i)]; ++c) {
      dst.push_back(freeslots[nxt++]);
      src.push_back(i);
    }
  const int n = int(dst.size());
  if (n > 0) {
    pairs.insert(pairs.end(), dst.begin(), dst.end());
    pairs.insert(pairs.end(), src.begin(), src.end());
    int* d = nullptr;
    AFQMC_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(int) * pairs.size(), s));
    AFQMC_CUDA_TRY(cudaMemcpyAsync(d, pairs.data(), sizeof(int) * pairs.size(),
                                   cudaMemcpyHostToDevice, s));
    int st = copy_rows(s, ws->buf, ws->walker_size, d, d + n, n);
    cudaFreeAsync(d, s);
    if (st) return st;
  }
  AFQMC_TRY(normalize_weights(s, ws->buf, ws->walker_size, ws->prop0, W));
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  return AFQMC_OK;
}

extern "C" int afqmc_wset_copy_rows(afqmc_wset ws, const int* dst, const int* src, int n,
                                    afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && (n == 0 || (dst && src)), "afqmc_wset_copy_rows: null argument");
  DeviceGuard g(ws->device);
  return copy_rows(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size, dst, src, n);
}

extern "C" int afqmc_wset_pack_rows(afqmc_wset ws, const int* idx, int n, afqmc_c128* buf,
                                    afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && (n == 0 || (idx && buf)), "afqmc_wset_pack_rows: null argument");
  DeviceGuard g(ws->device);
  return pack_rows(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size, idx, n,
                   (c128*)buf);
}

extern "C" int afqmc_wset_unpack_rows(afqmc_wset ws, const int* idx, int n, const afqmc_c128* buf,
                                      afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && (n == 0 || (idx && buf)), "afqmc_wset_unpack_rows: null argument");
  DeviceGuard g(ws->device);
  return unpack_rows(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size, idx, n,
                     (const c128*)buf);
}

extern "C" int afqmc_wset_normalize_weights(afqmc_wset ws, afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws, "afqmc_wset_normalize_weights: null handle");
  DeviceGuard g(ws->device);
  return normalize_weights(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size,
                           ws->prop0, ws->W);
}

extern "C" int afqmc_energy_sums(afqmc_wset ws, const afqmc_c128* E, afqmc_c128* out4,
                                 afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && E && out4, "afqmc_energy_sums: null argument");
  DeviceGuard g(ws->device);
  return energy_sums(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size, ws->prop0,
                     ws->W, (const c128*)E, (c128*)out4);
}

extern "C" int afqmc_pseudo_energy_sums(afqmc_wset ws, double dt, afqmc_c128* out2,
                                        afqmc_stream stream) {
  AFQMC_CHECK_ARG(ws && out2, "afqmc_pseudo_energy_sums: null argument");
  DeviceGuard g(ws->device);
  return pseudo_energy_sums(reinterpret_cast<cudaStream_t>(stream), ws->buf, ws->walker_size,
                            ws->prop0, ws->W, dt, (c128*)out2);
}
