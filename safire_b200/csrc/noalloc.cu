// afqmc_log_overlap_noalloc: the batched log-overlap without any device allocation.
//
// afqmc_log_overlap takes its [W][N][N] overlap-matrix scratch from the stream-ordered allocator.
// Some callers cannot allocate device memory at all: an application that reserves all device
// memory for its own pool at start-up and treats any later cudaMalloc as an error, or a process
// that is already at its device-memory limit.  This
// variant uses instead a file-scope device array of fixed size, so a call allocates nothing; the
// caller still passes the inputs and the output.
//
// Limits and sharing:
//   - the scratch holds kNoAllocScratchElems complex128 values (8 MiB): W * N * N must not exceed
//     524288 (for example W <= 209 at N = 50, or W <= 8192 at N = 8); larger calls are rejected
//     with AFQMC_ERR_SHAPE;
//   - every device that loads the library holds this array until the process exits;
//   - all calls on a device share the one array, so calls that overlap on the GPU (different
//     streams, or host threads without ordering between their streams) race on it; calls on one
//     stream are ordered and safe.  Each call overwrites the whole scratch region it uses before
//     reading it, so nothing in it needs to start at zero;
//   - the first call on a device looks the array's device address up (cudaGetSymbolAddress) with
//     that device current; make that first call before any stream capture on that device.  The
//     address is kept with the unique ID of the context it belongs to (cuCtxGetId); a call in a
//     different context of the device (after cudaDeviceReset, which reloads the module) looks it
//     up again, so no call uses an address of a context that no longer exists.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "detops.cuh"

namespace afqmc {
namespace {

constexpr long kNoAllocScratchElems = 1L << 19;  // 8 MiB of complex128

static __device__ __align__(256) c128 g_noalloc_scratch[kNoAllocScratchElems];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
c128* g_scratch_ptr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // cuCtxGetId of the context of the address

// unique ID of the current context (0 if the driver entry points are unavailable)
unsigned long long current_context_id() {
  static PFN_cuCtxGetCurrent_v4000 get_cur = nullptr;
  static PFN_cuCtxGetId_v12000 get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_cur && get_id && get_cur(&ctx) == CUDA_SUCCESS && ctx) get_id(ctx, &id);
  return id;
}

// Device address of the scratch array on the current device, looked up once per device and
// context.
int noalloc_scratch(c128** out) {
  int dev = -1;
  AFQMC_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error_detail("afqmc_log_overlap_noalloc: device %d out of range", dev);
    return AFQMC_ERR_ARG;
  }
  // 0 before the context is current on this thread: then the address is looked up (which makes
  // it current) and again on the next call, when the ID is known
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev] || ctx == 0 || g_scratch_ctx[dev] != ctx) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error_detail("afqmc_log_overlap_noalloc: cudaGetSymbolAddress failed: %s",
                       cudaGetErrorString(e));
      return AFQMC_ERR_CUDA;
    }
    g_scratch_ptr[dev] = static_cast<c128*>(p);
    g_scratch_ctx[dev] = ctx;
  }
  *out = g_scratch_ptr[dev];
  return AFQMC_OK;
}

}  // namespace
}  // namespace afqmc

using namespace afqmc;

extern "C" int afqmc_log_overlap_noalloc(const afqmc_c128* PsiT, const afqmc_c128* S, long ldS,
                                         afqmc_c128* ovlp, int W, int M, int N,
                                         afqmc_stream stream) {
  AFQMC_CHECK_ARG(W >= 0 && M >= 0 && N >= 0, "afqmc_log_overlap_noalloc: negative size");
  if (W == 0 || N == 0) return AFQMC_OK;
  AFQMC_CHECK_ARG(PsiT && S && ovlp, "afqmc_log_overlap_noalloc: null pointer");
  AFQMC_CHECK_ARG(ldS >= long(M) * N, "afqmc_log_overlap_noalloc: ldS < M*N");
  if (long(W) * N * N > kNoAllocScratchElems) {
    set_error_detail("afqmc_log_overlap_noalloc: W*N*N = %ld exceeds the fixed scratch of %ld "
                     "complex elements (8 MiB); split the walkers into smaller calls",
                     long(W) * N * N, kNoAllocScratchElems);
    return AFQMC_ERR_SHAPE;
  }
  c128* T = nullptr;
  AFQMC_TRY(noalloc_scratch(&T));
  return log_overlap(reinterpret_cast<cudaStream_t>(stream), (const c128*)PsiT, (const c128*)S,
                     ldS, (c128*)ovlp, W, M, N, T, cmk(1, 0), cmk(0, 0));
}
