// Mixed-precision contractions of the walker step on the 5th-generation tensor cores.
//
// Every contraction is a (batched) complex GEMM run as real tcgen05.mma kind::tf32 products with
// the 3xTF32 split x = hi + lo (hi = TF32(x), lo = TF32(x - hi)): a*b ~ ahi*bhi + ahi*blo + alo*bhi,
// accumulated in FP32 in tensor memory.  Complex operands are kept as planes
// {re_hi, re_lo, im_hi, im_lo}; the -Im(A)Im(B) term uses the MMA's A-negate bit.  Operand tiles
// arrive by TMA (128-byte swizzle) in a 2-3 stage mbarrier pipeline: warp 0 issues the TMA loads,
// one thread of warp 1 issues the MMAs, warps 2-5 drain the accumulators from TMEM and run the
// epilogue of the calling contraction.  FP64 stays where the method needs it (overlap LU,
// inverse, log-det, QR, weights, energy sums); see the per-function notes below for which
// reference contraction each call replaces.
#include <cudaTypedefs.h>

#include <memory>
#include <mutex>

#include "detops.cuh"
#include "energy.cuh"
#include "mixed.cuh"
#include "tc.cuh"
#include "zgemm.cuh"

namespace afqmc {

namespace {

constexpr int TC_THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int BK = 32;           // K elements per stage (128 bytes of FP32 = one swizzle row)

enum Epi : int {
  EPI_C128 = 0,      // out_c[z][row][col] = alpha * acc                (complex128)
  EPI_PLANES = 1,    // out planes [z][row][col] = split(alpha * acc)    (hi/lo re/im fp32)
  EPI_TAYLOR = 2,    // out planes [z][col][row] = split(alpha*acc); acc planes [z][col][row] (+)=
  EPI_S64 = 3,       // out_c[z][row][col] = alpha * acc (walker Slater matrix, FP64)
  EPI_VHS = 4,       // out planes [z=0][row][ (col/M)*ldv + col%M ] = split(alpha * acc)
};

struct TcParams {
  CUtensorMap a[4];
  CUtensorMap b[4];
  int m, n, k, batch;
  int order;  // tile order (see tc_tile)
  int a_batched, b_batched;
  c128 alpha;
  float* out[4];        // split planes re_hi, re_lo, im_hi, im_lo
  long out_ld, out_bs;  // leading dim / batch stride of the output planes (elements)
  float* acc[2];        // Taylor running sum re, im  (EPI_TAYLOR)
  int acc_init;         // 1: acc = value (first term), 0: acc += value
  float* acc_split[4];  // optional split copy of the updated running sum (last Taylor term)
  c128* out_c;
  long outc_ld, outc_bs;
  int vhs_M;            // EPI_VHS: columns are (i, k) pairs of an M x M matrix
  unsigned* err;
};

template <bool A_CPLX, bool B_CPLX, int BN, int STAGES>
struct TcCfg {
  static constexpr int NA = A_CPLX ? 4 : 2;
  static constexpr int NB = B_CPLX ? 4 : 2;
  static constexpr int A_TILE = 128 * BK * 4;  // bytes per plane tile
  static constexpr int B_TILE = BN * BK * 4;
  static constexpr int STAGE = NA * A_TILE + NB * B_TILE;
  // two accumulators (re, im) x 2 buffers
  static constexpr int TMEM_COLS = (4 * BN <= 128) ? 128 : (4 * BN <= 256) ? 256 : 512;
  static constexpr size_t SMEM = size_t(STAGES) * STAGE + 1024 /*align*/ + 256 /*barriers*/;
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 128, "UMMA N for M=128, double buffered");
  static_assert(SMEM <= 232448, "shared memory");
};

__device__ __forceinline__ void split_store(float v, float* hi, float* lo, long idx) {
  const float h = tc::tf32_hi(v);
  hi[idx] = h;
  lo[idx] = v - h;
}

// tile t -> (m tile, n tile, batch).  order 0: m tiles fastest (consecutive tiles share the B
// tile); order 1: n tiles fastest (consecutive tiles share the A tile).
__device__ __forceinline__ void tc_tile(long t, int MT, int NT, int order, int& mt, int& nt,
                                        int& z) {
  if (order == 0) {
    mt = int(t % MT);
    const long r = t / MT;
    nt = int(r % NT);
    z = int(r / NT);
  } else {
    nt = int(t % NT);
    const long r = t / NT;
    mt = int(r % MT);
    z = int(r / MT);
  }
}

// Persistent tensor-core GEMM: one CTA per SM walks the tiles; the TMA ring runs ahead across
// tiles and the epilogue of tile i overlaps the MMAs of tile i+1 (two TMEM accumulators).
template <bool A_CPLX, bool B_CPLX, int BN, int STAGES, int EPI>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_cgemm_kernel(const __grid_constant__ TcParams p) {
  using K = TcCfg<A_CPLX, B_CPLX, BN, STAGES>;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * K::STAGE);
  uint64_t* empty = full + STAGES;
  uint64_t* acc_full = empty + STAGES;  // [2]
  uint64_t* acc_empty = acc_full + 2;   // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int MT = (p.m + 127) / 128, NT = (p.n + BN - 1) / BN;
  const long ntiles = long(MT) * NT * p.batch;
  const int nk = (p.k + BK - 1) / BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], 128);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
#pragma unroll
    for (int q = 0; q < K::NA; ++q) tc::prefetch_tmap(&p.a[q]);
#pragma unroll
    for (int q = 0; q < K::NB; ++q) tc::prefetch_tmap(&p.b[q]);
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, K::TMEM_COLS);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t taddr = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      long it = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        int mt, nt, z;
        tc_tile(t, MT, NT, p.order, mt, nt, z);
        const int za = p.a_batched ? z : 0, zb = p.b_batched ? z : 0;
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = int(it % STAGES);
          if (it >= STAGES) {
            if (!tc::mbar_wait(&empty[s], unsigned((it / STAGES) - 1) & 1u, p.err, abort_flag)) {
              ok = false;
              break;
            }
          }
          unsigned char* st = base + size_t(s) * K::STAGE;
          tc::mbar_arrive_expect_tx(&full[s], K::STAGE);
#pragma unroll
          for (int q = 0; q < K::NA; ++q)
            tc::tma_load_3d(st + q * K::A_TILE, &p.a[q], &full[s], kc * BK, mt * 128, za);
#pragma unroll
          for (int q = 0; q < K::NB; ++q)
            tc::tma_load_3d(st + K::NA * K::A_TILE + q * K::B_TILE, &p.b[q], &full[s], kc * BK,
                            nt * BN, zb);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_tf32(128, BN, false);
      constexpr uint32_t IDN = tc::idesc_tf32(128, BN, true);
      long it = 0, ti = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++ti) {
        const int buf = int(ti & 1);
        if (ti >= 2) {
          if (!tc::mbar_wait(&acc_empty[buf], unsigned((ti / 2) - 1) & 1u, p.err, abort_flag)) {
            ok = false;
            break;
          }
        }
        tc::tc_fence_after();
        const uint32_t dr = taddr + uint32_t(buf * 2 * BN), di = dr + BN;
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = int(it % STAGES);
          if (!tc::mbar_wait(&full[s], unsigned(it / STAGES) & 1u, p.err, abort_flag)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          unsigned char* st = base + size_t(s) * K::STAGE;
          const uint32_t sa = tc::smem_u32(st);
          const uint32_t sb = tc::smem_u32(st + K::NA * K::A_TILE);
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {
            if (kc * BK + kk * 8 >= p.k) break;  // zero fill past K
            // +32 bytes per K=8 step inside the 128-byte swizzle row (descriptor units of 16 B)
            auto A = [&](int q) { return tc::sdesc_sw128(sa + q * K::A_TILE) + uint64_t(2 * kk); };
            auto B = [&](int q) { return tc::sdesc_sw128(sb + q * K::B_TILE) + uint64_t(2 * kk); };
            const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
            if constexpr (A_CPLX && B_CPLX) {
              // Dr = Ar Br - Ai Bi ; Di = Ar Bi + Ai Br  (planes 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo)
              tc::mma_tf32(dr, A(0), B(0), ID, acc0);
              tc::mma_tf32(dr, A(0), B(1), ID, 1);
              tc::mma_tf32(dr, A(1), B(0), ID, 1);
              tc::mma_tf32(dr, A(2), B(2), IDN, 1);
              tc::mma_tf32(dr, A(2), B(3), IDN, 1);
              tc::mma_tf32(dr, A(3), B(2), IDN, 1);
              tc::mma_tf32(di, A(0), B(2), ID, acc0);
              tc::mma_tf32(di, A(0), B(3), ID, 1);
              tc::mma_tf32(di, A(1), B(2), ID, 1);
              tc::mma_tf32(di, A(2), B(0), ID, 1);
              tc::mma_tf32(di, A(2), B(1), ID, 1);
              tc::mma_tf32(di, A(3), B(0), ID, 1);
            } else if constexpr (A_CPLX) {
              // real B (planes 0 hi, 1 lo)
              tc::mma_tf32(dr, A(0), B(0), ID, acc0);
              tc::mma_tf32(dr, A(0), B(1), ID, 1);
              tc::mma_tf32(dr, A(1), B(0), ID, 1);
              tc::mma_tf32(di, A(2), B(0), ID, acc0);
              tc::mma_tf32(di, A(2), B(1), ID, 1);
              tc::mma_tf32(di, A(3), B(0), ID, 1);
            } else {
              // real A, complex B
              tc::mma_tf32(dr, A(0), B(0), ID, acc0);
              tc::mma_tf32(dr, A(0), B(1), ID, 1);
              tc::mma_tf32(dr, A(1), B(0), ID, 1);
              tc::mma_tf32(di, A(0), B(2), ID, acc0);
              tc::mma_tf32(di, A(0), B(3), ID, 1);
              tc::mma_tf32(di, A(1), B(2), ID, 1);
            }
          }
          tc::mma_commit(&empty[s]);  // stage reusable once these MMAs have read it
        }
        if (!ok) break;
        tc::mma_commit(&acc_full[buf]);
      }
    }
  } else {
    // epilogue warps 2..5: TMEM lane quarter = warp % 4
    const int q = warp & 3;
    long ti = 0;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x, ++ti) {
      int mt, nt, z;
      tc_tile(t, MT, NT, p.order, mt, nt, z);
      const int buf = int(ti & 1);
      const bool ok = tc::mbar_wait(&acc_full[buf], unsigned(ti / 2) & 1u, p.err, abort_flag);
      tc::tc_fence_after();
      if (!ok) break;
      const int row = mt * 128 + q * 32 + lane;
      const int n0 = nt * BN;
      const uint32_t trow = taddr + (uint32_t(q * 32) << 16) + uint32_t(buf * 2 * BN);
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 16) {
        float vr[16], vi[16];
        tc::tmem_ld16(trow + c0, vr);
        tc::tmem_ld16(trow + BN + c0, vi);
        tc::tmem_ld_wait();
        if (c0 + 16 >= BN) {
          tc::tc_fence_before();
          tc::mbar_arrive(&acc_empty[buf]);  // accumulator free for tile ti+2
        }
        if (row >= p.m) continue;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          if (col >= p.n) break;
          const float ar = float(p.alpha.x), ai = float(p.alpha.y);
          const float xr = ar * vr[j] - ai * vi[j];
          const float xi = ar * vi[j] + ai * vr[j];
          if constexpr (EPI == EPI_C128 || EPI == EPI_S64) {
            const double dr = p.alpha.x * double(vr[j]) - p.alpha.y * double(vi[j]);
            const double di = p.alpha.x * double(vi[j]) + p.alpha.y * double(vr[j]);
            p.out_c[long(z) * p.outc_bs + long(row) * p.outc_ld + col] = cmk(dr, di);
          } else if constexpr (EPI == EPI_PLANES) {
            const long idx = long(z) * p.out_bs + long(row) * p.out_ld + col;
            split_store(xr, p.out[0], p.out[1], idx);
            split_store(xi, p.out[2], p.out[3], idx);
          } else if constexpr (EPI == EPI_VHS) {
            const int i = col / p.vhs_M, kq = col - i * p.vhs_M;
            const long idx = long(row) * p.out_bs + long(i) * p.out_ld + kq;
            split_store(xr, p.out[0], p.out[1], idx);
            split_store(xi, p.out[2], p.out[3], idx);
          } else if constexpr (EPI == EPI_TAYLOR) {
            // transposed store: [z][col][row]
            const long idx = long(z) * p.out_bs + long(col) * p.out_ld + row;
            split_store(xr, p.out[0], p.out[1], idx);
            split_store(xi, p.out[2], p.out[3], idx);
            float sr = xr, si = xi;
            if (!p.acc_init) {
              sr += p.acc[0][idx];
              si += p.acc[1][idx];
            }
            p.acc[0][idx] = sr;
            p.acc[1][idx] = si;
            if (p.acc_split[0]) {
              split_store(sr, p.acc_split[0], p.acc_split[1], idx);
              split_store(si, p.acc_split[2], p.acc_split[3], idx);
            }
          }
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(taddr, K::TMEM_COLS);
}

// ---------------------------------------------------------------------------------------------
// host: tensor maps
// ---------------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

// 3D map over an FP32 plane: element (x, y, z) at base + z*batch_stride + y*row_stride + x for
// x < k, y < rows, z < batch; box {32, box_rows, box_batch}, 128-byte swizzle, zero fill outside.
int make_plane_map_3d(CUtensorMap* map, const float* base, long k, long rows, long row_stride,
                      long batch, long batch_stride, int box_rows, int box_batch) {
  auto fn = encode_fn();
  if (!fn) {
    set_error_detail("cuTensorMapEncodeTiled is not available");
    return AFQMC_ERR_CUDA;
  }
  if (batch == 1) batch_stride = rows * row_stride;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_stride * 4) % 16 ||
      (batch_stride * 4) % 16) {
    set_error_detail("make_plane_map_3d: plane not 16-byte aligned (row stride=%ld, batch "
                     "stride=%ld)", row_stride, batch_stride);
    return AFQMC_ERR_SHAPE;
  }
  cuuint64_t dims[3] = {cuuint64_t(k), cuuint64_t(rows), cuuint64_t(batch)};
  cuuint64_t strides[2] = {cuuint64_t(row_stride * 4), cuuint64_t(batch_stride * 4)};
  cuuint32_t box[3] = {cuuint32_t(BK), cuuint32_t(box_rows), cuuint32_t(box_batch)};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides,
                  box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error_detail("cuTensorMapEncodeTiled failed (%d): k=%ld rows=%ld batch=%ld box=%dx%d",
                     int(r), k, rows, batch, box_rows, box_batch);
    return AFQMC_ERR_CUDA;
  }
  return AFQMC_OK;
}

namespace {

int make_map(CUtensorMap* map, const float* base, long k, long rows, long ld, long batch,
             long batch_stride, int box_rows) {
  return make_plane_map_3d(map, base, k, rows, ld, batch, batch_stride, box_rows, 1);
}

// FP32 planes of one operand: 4 (complex) or 2 (real) arrays [batch][rows][ld]
struct Planes {
  float* p[4] = {nullptr, nullptr, nullptr, nullptr};
  int nplanes = 0;
  long rows = 0, ld = 0, batch = 0, k = 0;
  long bstride() const { return rows * ld; }
  size_t elems() const { return size_t(batch) * rows * ld; }
};

int alloc_planes(Planes& P, int nplanes, long batch, long rows, long k) {
  P.nplanes = nplanes;
  P.batch = batch;
  P.rows = rows;
  P.k = k;
  P.ld = (k + 3) / 4 * 4;
  for (int q = 0; q < nplanes; ++q) {
    cudaError_t e = cudaMalloc(&P.p[q], sizeof(float) * P.elems());
    if (e != cudaSuccess) {
      set_error_detail("alloc_planes: %s", cudaGetErrorString(e));
      return AFQMC_ERR_ALLOC;
    }
    AFQMC_CUDA_TRY(cudaMemset(P.p[q], 0, sizeof(float) * P.elems()));
  }
  return AFQMC_OK;
}

void free_planes(Planes& P) {
  for (auto& q : P.p)
    if (q) {
      cudaFree(q);
      q = nullptr;
    }
}

int maps_for(const Planes& P, CUtensorMap* maps, int box_rows, long batch_override = -1) {
  const long batch = batch_override > 0 ? batch_override : P.batch;
  for (int q = 0; q < P.nplanes; ++q)
    AFQMC_TRY(make_map(&maps[q], P.p[q], P.k, P.rows, P.ld, batch, P.bstride(), box_rows));
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// conversions FP64 -> split FP32 planes
// ---------------------------------------------------------------------------------------------
// complex src [b][r][c] (ld_src, bstride_src) -> planes [b][r][c] or transposed [b][c][r]
template <bool TRANSPOSE>
__global__ void split_complex_kernel(const c128* __restrict__ src, long ld_src, long bs_src,
                                     int rows, int cols, float* __restrict__ rh,
                                     float* __restrict__ rl, float* __restrict__ ih,
                                     float* __restrict__ il, long ld_dst, long bs_dst) {
  const long b = blockIdx.z;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows || c >= cols) return;
  const c128 v = src[b * bs_src + long(r) * ld_src + c];
  const long d = TRANSPOSE ? b * bs_dst + long(c) * ld_dst + r : b * bs_dst + long(r) * ld_dst + c;
  split_store(float(v.x), rh, rl, d);
  split_store(float(v.y), ih, il, d);
}

__global__ void split_real_kernel(const double* __restrict__ src, long n_rows, long cols,
                                  long ld_src, float* __restrict__ h, float* __restrict__ l,
                                  long ld_dst) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= n_rows * cols) return;
  const long r = e / cols, c = e % cols;
  split_store(float(src[r * ld_src + c]), h, l, r * ld_dst + c);
}

int split_complex(cudaStream_t s, const c128* src, long ld_src, long bs_src, int batch, int rows,
                  int cols, Planes& P, bool transpose) {
  dim3 blk(32, 8);
  if (transpose) {
    // coalesce the writes along the destination's contiguous (row) index
    dim3 grid(ceil_div(cols, 32), ceil_div(rows, 8), batch);
    split_complex_kernel<true><<<grid, blk, 0, s>>>(src, ld_src, bs_src, rows, cols, P.p[0],
                                                    P.p[1], P.p[2], P.p[3], P.ld, P.bstride());
  } else {
    dim3 grid(ceil_div(cols, 32), ceil_div(rows, 8), batch);
    split_complex_kernel<false><<<grid, blk, 0, s>>>(src, ld_src, bs_src, rows, cols, P.p[0],
                                                     P.p[1], P.p[2], P.p[3], P.ld, P.bstride());
  }
  return launch_status("split_complex_kernel");
}

int split_real_host(const double* src_dev, long rows, long cols, long ld_src, Planes& P) {
  const long n = rows * cols;
  split_real_kernel<<<ceil_div(n, 256), 256>>>(src_dev, rows, cols, ld_src, P.p[0], P.p[1], P.ld);
  AFQMC_TRY(launch_status("split_real_kernel"));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// launcher
// ---------------------------------------------------------------------------------------------
template <bool A_CPLX, bool B_CPLX, int BN, int STAGES, int EPI>
int launch_tc(cudaStream_t s, TcParams& p, int batch) {
  using K = TcCfg<A_CPLX, B_CPLX, BN, STAGES>;
  auto kern = tc_cgemm_kernel<A_CPLX, B_CPLX, BN, STAGES, EPI>;
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(K::SMEM)));
  p.batch = batch;
  static int nsm = 0;
  if (nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  const long ntiles = long(ceil_div(p.m, 128)) * ceil_div(p.n, BN) * batch;
  const int grid = int(ntiles < nsm ? ntiles : nsm);
  kern<<<grid, TC_THREADS, K::SMEM, s>>>(p);
  return launch_status("tc_cgemm_kernel");
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// Mixed Hamiltonian: split-TF32 copies of the static tensors
// ---------------------------------------------------------------------------------------------
struct MixedHam {
  int M, Nc, nspin, nel[2], el_off[2], nel_tot;
  bool lnak_cplx;
  Planes Likn[2];   // [1][M*M][Nc]  (B of vHS, K = Nc)
  Planes Lnak[2];   // [1][Nc][nel*M] (B of vbias, K = nel*M); same memory viewed [Nc*nel][M] for exchange
  // dynamic operands, sized on demand
  int capW = 0;
  int exchange_split = 3;  // TF32 products per real product in the exchange contraction
  int taylor_mode = 1;    // 0: one GEMM launch per Taylor product; 1: fused, slots chosen by W;
  int taylor_slots = 0;   // 2 / 3: fused with one / two walkers in flight per CTA
  Planes G;         // [W][1][nel_tot*M]  (A of vbias);  exchange view [W*nel][M]
  Planes X;         // [1][W][Nc] (A of vHS)
  c128* vpart = nullptr;  // split-K partial sums of vbias [S][W][Nc]
  long vpart_elems = 0;
  unsigned* err = nullptr;
  // propagation buffers
  int capP = 0;
  Planes P1;        // [1][M][M] real (A of the P1 products)
  const void* P1_src = nullptr;
  Planes V;         // [W][M][M] complex (A of the Taylor products)
  Planes T0, T1, Tacc_split, Sst;  // [W][N][M] complex (B operands)
  float* acc[2] = {nullptr, nullptr};  // running Taylor sum [W][N][M]
  ~MixedHam() {
    for (int s = 0; s < 2; ++s) {
      free_planes(Likn[s]);
      free_planes(Lnak[s]);
    }
    free_planes(G);
    free_planes(X);
    free_planes(P1);
    free_planes(V);
    free_planes(T0);
    free_planes(T1);
    free_planes(Tacc_split);
    free_planes(Sst);
    for (auto& a : acc)
      if (a) cudaFree(a);
    if (vpart) cudaFree(vpart);
    if (err) cudaFree(err);
  }
};

void mixed_ham_destroy(MixedHam* m) { delete m; }

int mixed_ham_create(MixedHam** out, const EnergyArgs& a, cudaStream_t s) {
  *out = nullptr;
  if (a.M % 4 || a.Nc % 4) {
    set_error_detail("mixed precision needs M and Nc multiples of 4 (M=%d, Nc=%d)", a.M, a.Nc);
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (!a.Likn) {
    set_error_detail("mixed_ham_create: missing Likn");
    return AFQMC_ERR_ARG;
  }
  std::unique_ptr<MixedHam> m(new MixedHam());
  m->M = a.M;
  m->Nc = a.Nc;
  m->nspin = a.nspin;
  m->nel_tot = 0;
  for (int s2 = 0; s2 < 2; ++s2) {
    m->nel[s2] = a.nel[s2];
    m->el_off[s2] = a.el_off[s2];
    m->nel_tot += (s2 < a.nspin) ? a.nel[s2] : 0;
  }
  m->lnak_cplx = (a.Lnak_real[0] == nullptr);
  const long MM = long(a.M) * a.M;
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  for (int sp = 0; sp < a.nspin_H2; ++sp) {
    AFQMC_TRY(alloc_planes(m->Likn[sp], 2, 1, MM, a.Nc));
    AFQMC_TRY(split_real_host(a.Likn + size_t(sp) * MM * a.Nc, MM, a.Nc, a.Nc, m->Likn[sp]));
  }
  for (int sp = 0; sp < a.nspin; ++sp) {
    const int Ns = a.nel[sp];
    if (Ns == 0) continue;
    const long K = long(Ns) * a.M;
    if (m->lnak_cplx) {
      AFQMC_TRY(alloc_planes(m->Lnak[sp], 4, 1, a.Nc, K));
      AFQMC_TRY(split_complex(nullptr, a.Lnak[sp], K, 0, 1, a.Nc, int(K), m->Lnak[sp], false));
    } else {
      AFQMC_TRY(alloc_planes(m->Lnak[sp], 2, 1, a.Nc, K));
      AFQMC_TRY(split_real_host(a.Lnak_real[sp], a.Nc, K, K, m->Lnak[sp]));
    }
  }
  AFQMC_CUDA_TRY(cudaMalloc(&m->err, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaMemset(m->err, 0, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = m.release();
  return AFQMC_OK;
}

namespace {

int ensure_walker_buffers(MixedHam* m, int W) {
  if (m->capW >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->G);
  free_planes(m->X);
  AFQMC_TRY(alloc_planes(m->G, 4, 1, W, long(m->nel_tot) * m->M));
  AFQMC_TRY(alloc_planes(m->X, 4, 1, W, m->Nc));
  m->capW = W;
  return AFQMC_OK;
}

}  // namespace

namespace {
// v[i] (+)= sum_s part[s][i] in FP64
__global__ void sum_partials_kernel(const c128* __restrict__ part, int S, long n,
                                    c128* __restrict__ v, int accumulate) {
  const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  c128 acc = accumulate ? v[i] : cmk(0, 0);
  for (int z = 0; z < S; ++z) acc = cadd(acc, part[long(z) * n + i]);
  v[i] = acc;
}
}  // namespace

// vbias = a * G Lnak^T (Real3IndexFactorization.hpp:384): A = G planes [W][nel*M], B = Lnak
// [Nc][nel*M] (per spin block: the K range of the spin's rows of G).
int vbias_mixed(cudaStream_t s, MixedHam* m, const c128* G, long ldG, c128* v, int W, double a) {
  if (m->nspin > 1) {
    set_error_detail("vbias_mixed: COLLINEAR walkers are not supported in mixed precision");
    return AFQMC_ERR_UNSUPPORTED;
  }
  AFQMC_TRY(ensure_walker_buffers(m, W));
  const long Kt = long(m->nel_tot) * m->M;
  AFQMC_TRY(split_complex(s, G, ldG, 0, 1, W, int(Kt), m->G, false));
  bool first = true;
  for (int sp = 0; sp < m->nspin; ++sp) {
    const int Ns = m->nel[sp];
    if (Ns == 0) continue;
    const long K = long(Ns) * m->M;
    const long off = long(m->el_off[sp]) * m->M;
    // Split K = N M into S equal ranges (a multiple of 4 floats each): every range is one batch
    // of the GEMM, accumulated in FP32 on the tensor cores over K / S only, and the S partial
    // sums are added in FP64.  The shorter FP32 sums cut the accumulation error, and S times as
    // many output tiles fill the SMs (W / 128 x Nc / 128 tiles alone are fewer than 148).
    int S = 1;
    for (int c = 16; c >= 2; --c)
      if (K % c == 0 && (K / c) % 4 == 0 && K / c >= 512) {
        S = c;
        break;
      }
    const int bn_rows = m->lnak_cplx ? 64 : 128;
    TcParams p{};
    bool split = false;
    if (S > 1 && !m->lnak_cplx) {
      const long Kc = K / S;
      const long need = long(S) * W * m->Nc;
      if (m->vpart_elems < need) {
        if (m->vpart) cudaFree(m->vpart);
        m->vpart = nullptr;
        m->vpart_elems = 0;
        AFQMC_CUDA_TRY(cudaMalloc(&m->vpart, sizeof(c128) * need));
        m->vpart_elems = need;
      }
      // 3-D maps whose third coordinate steps through the K ranges (stride Kc floats)
      split = true;
      for (int q = 0; q < 4 && split; ++q)
        split = make_map(&p.a[q], m->G.p[q] + off, Kc, W, m->G.ld, S, Kc, 128) == AFQMC_OK;
      for (int q = 0; q < 2 && split; ++q)
        split = make_map(&p.b[q], m->Lnak[sp].p[q], Kc, m->Nc, m->Lnak[sp].ld, S, Kc,
                         bn_rows) == AFQMC_OK;
      if (split) {
        p.m = W; p.n = m->Nc; p.k = int(Kc);
        p.a_batched = 1; p.b_batched = 1;
        p.order = 1;
        p.alpha = cmk(a, 0);
        p.out_c = m->vpart; p.outc_ld = m->Nc; p.outc_bs = long(W) * m->Nc;
        p.err = m->err;
        AFQMC_TRY((launch_tc<true, false, 128, 2, EPI_C128>(s, p, S)));
        const long n = long(W) * m->Nc;
        sum_partials_kernel<<<ceil_div(n, 256), 256, 0, s>>>(m->vpart, S, n, v, first ? 0 : 1);
        AFQMC_TRY(launch_status("sum_partials_kernel"));
      }
    }
    if (!split) {
      p = TcParams{};
      for (int q = 0; q < 4; ++q)
        AFQMC_TRY(make_map(&p.a[q], m->G.p[q] + off, K, W, m->G.ld, 1, long(W) * m->G.ld, 128));
      AFQMC_TRY(maps_for(m->Lnak[sp], p.b, bn_rows));
      p.m = W; p.n = m->Nc; p.k = int(K);
      p.order = 1;  // a G tile (128 walkers x K) stays in L2 while the Lnak tiles stream past it
      p.alpha = cmk(a, 0);
      p.out_c = v; p.outc_ld = m->Nc; p.outc_bs = 0;
      p.err = m->err;
      if (m->lnak_cplx)
        AFQMC_TRY((launch_tc<true, true, 64, 2, EPI_C128>(s, p, 1)));
      else
        AFQMC_TRY((launch_tc<true, false, 128, 2, EPI_C128>(s, p, 1)));
    }
    first = false;
  }
  return AFQMC_OK;
}

// vHS = a * X L^T (Real3IndexFactorization.hpp:321) written as split planes V[w][i][k]; the
// propagation reads them as its A operand.  When V is a complex128 output (the C-ABI call
// afqmc_ham_vhs) the planes are re-assembled into V afterwards.
namespace {
__global__ void planes_to_c128_kernel(const float* __restrict__ rh, const float* __restrict__ rl,
                                      const float* __restrict__ ih, const float* __restrict__ il,
                                      long n, c128* __restrict__ out) {
  long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e < n) out[e] = cmk(double(rh[e]) + double(rl[e]), double(ih[e]) + double(il[e]));
}

int ensure_v_buffers(MixedHam* m, int W) {
  if (m->V.batch >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->V);
  return alloc_planes(m->V, 4, W, m->M, m->M);
}

int ensure_prop_buffers(MixedHam* m, int W, int N) {
  if (m->capP >= W && m->T0.rows == N) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->T0);
  free_planes(m->T1);
  free_planes(m->Tacc_split);
  free_planes(m->Sst);
  for (auto& a : m->acc)
    if (a) {
      cudaFree(a);
      a = nullptr;
    }
  const int M = m->M;
  AFQMC_TRY(alloc_planes(m->T0, 4, W, N, M));
  AFQMC_TRY(alloc_planes(m->T1, 4, W, N, M));
  AFQMC_TRY(alloc_planes(m->Tacc_split, 4, W, N, M));
  AFQMC_TRY(alloc_planes(m->Sst, 4, W, N, M));
  for (auto& a : m->acc) {
    AFQMC_CUDA_TRY(cudaMalloc(&a, sizeof(float) * m->T0.elems()));
    AFQMC_CUDA_TRY(cudaMemset(a, 0, sizeof(float) * m->T0.elems()));
  }
  m->capP = W;
  return AFQMC_OK;
}
}  // namespace

int vhs_planes(cudaStream_t s, MixedHam* m, const c128* X, int W, double a) {
  AFQMC_TRY(ensure_walker_buffers(m, W));
  AFQMC_TRY(ensure_v_buffers(m, W));
  AFQMC_TRY(split_complex(s, X, m->Nc, 0, 1, W, m->Nc, m->X, false));
  TcParams p{};
  AFQMC_TRY(maps_for(m->X, p.a, 128));
  AFQMC_TRY(maps_for(m->Likn[0], p.b, 128));
  const long MM = long(m->M) * m->M;
  p.m = W; p.n = int(MM); p.k = m->Nc;
  p.alpha = cmk(a, 0);
  for (int q = 0; q < 4; ++q) p.out[q] = m->V.p[q];
  p.out_ld = m->V.ld;
  p.out_bs = m->V.bstride();
  p.vhs_M = m->M;
  p.err = m->err;
  return launch_tc<true, false, 128, 2, EPI_VHS>(s, p, 1);
}

int vhs_mixed(cudaStream_t s, MixedHam* m, const c128* X, c128* V, int W, double a) {
  if (m->nspin > 1 && m->Likn[1].p[0]) {
    set_error_detail("vhs_mixed: spin-dependent Cholesky vectors are not supported");
    return AFQMC_ERR_UNSUPPORTED;
  }
  AFQMC_TRY(vhs_planes(s, m, X, W, a));
  if (V) {
    const long n = long(W) * m->M * m->M;
    if (m->V.ld != m->M) {
      set_error_detail("vhs_mixed: padded V planes cannot be copied out");
      return AFQMC_ERR_UNSUPPORTED;
    }
    planes_to_c128_kernel<<<ceil_div(n, 256), 256, 0, s>>>(m->V.p[0], m->V.p[1], m->V.p[2],
                                                           m->V.p[3], n, V);
    AFQMC_TRY(launch_status("planes_to_c128_kernel"));
  }
  return AFQMC_OK;
}

int taylor_fused_tc(cudaStream_t s, const float* const P1p[2], const float* const Vp[4], long ldV,
                    const float* const Sp[4], float* const Tp0[4], float* const Tp1[4],
                    float* const Rp[4], float* const sum[2], long pl_ld, c128* S, long ldS,
                    int W, int M, int N, int order, int nslots, unsigned* err);

// Taylor propagation S <- P1 sum_n (iV)^n/n! P1 S (propagate.hpp:238-298) on the split planes.
// V must have been produced by vhs_mixed (planes kept in MixedHam) for the same walkers.
int propagate_mixed(cudaStream_t s, MixedHam* m, const void* P1, bool p1_real, c128* S, long ldS,
                    int W, int M, int N, int order) {
  if (!p1_real) {
    set_error_detail("propagate_mixed: a complex one-body propagator is not supported");
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (m->V.batch < W) {
    set_error_detail("propagate_mixed: no vHS planes for %d walkers (call vhs_mixed first)", W);
    return AFQMC_ERR_ARG;
  }
  AFQMC_TRY(ensure_prop_buffers(m, W, N));
  if (m->P1_src != P1) {
    free_planes(m->P1);
    AFQMC_TRY(alloc_planes(m->P1, 2, 1, M, M));
    AFQMC_TRY(split_real_host(static_cast<const double*>(P1), M, M, M, m->P1));
    m->P1_src = P1;
  }
  // S^T planes [W][N][M] from the walkers' Slater matrices [W][M][N]
  AFQMC_TRY(split_complex(s, S, N, ldS, W, M, N, m->Sst, true));
  if (M <= 256 && N <= 64 && m->taylor_mode != 0 && m->P1.ld == m->T0.ld) {
    // one persistent kernel runs all order + 2 products of each walker
    const float* p1p[2] = {m->P1.p[0], m->P1.p[1]};
    const float* vp[4] = {m->V.p[0], m->V.p[1], m->V.p[2], m->V.p[3]};
    const float* sp[4] = {m->Sst.p[0], m->Sst.p[1], m->Sst.p[2], m->Sst.p[3]};
    return taylor_fused_tc(s, p1p, vp, m->V.ld, sp, m->T0.p, m->T1.p, m->Tacc_split.p, m->acc,
                           m->T0.ld, S, ldS, W, M, N, order, m->taylor_slots, m->err);
  }
  Planes* Tin = &m->T0;
  Planes* Tout = &m->T1;
  // T0 = P1 S  (acc = T0)
  {
    TcParams p{};
    AFQMC_TRY(maps_for(m->P1, p.a, 128));
    AFQMC_TRY(maps_for(m->Sst, p.b, 64, W));
    p.m = M; p.n = N; p.k = M; p.a_batched = 0; p.b_batched = 1;
    p.alpha = cmk(1, 0);
    for (int q = 0; q < 4; ++q) p.out[q] = Tin->p[q];
    p.out_ld = Tin->ld; p.out_bs = Tin->bstride();
    p.acc[0] = m->acc[0]; p.acc[1] = m->acc[1]; p.acc_init = 1;
    if (order == 0)
      for (int q = 0; q < 4; ++q) p.acc_split[q] = m->Tacc_split.p[q];
    p.err = m->err;
    AFQMC_TRY((launch_tc<false, true, 64, 3, EPI_TAYLOR>(s, p, W)));
  }
  for (int n = 1; n <= order; ++n) {
    TcParams p{};
    AFQMC_TRY(maps_for(m->V, p.a, 128, W));
    AFQMC_TRY(maps_for(*Tin, p.b, 64, W));
    p.m = M; p.n = N; p.k = M; p.a_batched = 1; p.b_batched = 1;
    p.alpha = cmk(0.0, 1.0 / double(n));
    for (int q = 0; q < 4; ++q) p.out[q] = Tout->p[q];
    p.out_ld = Tout->ld; p.out_bs = Tout->bstride();
    p.acc[0] = m->acc[0]; p.acc[1] = m->acc[1]; p.acc_init = 0;
    if (n == order)
      for (int q = 0; q < 4; ++q) p.acc_split[q] = m->Tacc_split.p[q];
    p.err = m->err;
    AFQMC_TRY((launch_tc<true, true, 64, 2, EPI_TAYLOR>(s, p, W)));
    std::swap(Tin, Tout);
  }
  // S = P1 * TMN
  {
    TcParams p{};
    AFQMC_TRY(maps_for(m->P1, p.a, 128));
    AFQMC_TRY(maps_for(m->Tacc_split, p.b, 64, W));
    p.m = M; p.n = N; p.k = M; p.a_batched = 0; p.b_batched = 1;
    p.alpha = cmk(1, 0);
    p.out_c = S; p.outc_ld = N; p.outc_bs = ldS;
    p.err = m->err;
    AFQMC_TRY((launch_tc<false, true, 64, 3, EPI_S64>(s, p, W)));
  }
  return AFQMC_OK;
}

int mixed_set_taylor_mode(MixedHam* m, int mode) {
  m->taylor_mode = mode;
  m->taylor_slots = mode >= 2 ? mode - 1 : 0;
  return AFQMC_OK;
}

int mixed_prepare_G(cudaStream_t s, MixedHam* m, const c128* G, long ldG, int W) {
  AFQMC_TRY(ensure_walker_buffers(m, W));
  const long Kt = long(m->nel_tot) * m->M;
  return split_complex(s, G, ldG, 0, 1, W, int(Kt), m->G, false);
}

// T chunk GEMM for the exchange energy (called from energy.cu's chunk loop through energy_tc)
int exchange_T_tc(cudaStream_t s, MixedHam* m, int sp, int w0, int wc, c128* workT) {
  const int Ns = m->nel[sp];
  const long off = long(m->el_off[sp]) * m->M;
  TcParams p{};
  // A: rows (w, b) of G for walkers [w0, w0+wc): plane rows of nel_tot*M, spin block at off
  for (int q = 0; q < 4; ++q)
    AFQMC_TRY(make_map(&p.a[q], m->G.p[q] + long(w0) * m->G.ld + off, m->M, Ns, m->M, wc,
                       m->G.ld, 128));
  // B: Lnak viewed as [Nc*Ns][M]
  for (int q = 0; q < m->Lnak[sp].nplanes; ++q)
    AFQMC_TRY(make_map(&p.b[q], m->Lnak[sp].p[q], m->M, long(m->Nc) * Ns, m->M, 1, 0,
                       m->lnak_cplx ? 64 : 128));
  p.m = Ns; p.n = m->Nc * Ns; p.k = m->M; p.a_batched = 1; p.b_batched = 0;
  p.alpha = cmk(1, 0);
  p.out_c = workT; p.outc_ld = long(m->Nc) * Ns; p.outc_bs = long(Ns) * m->Nc * Ns;
  p.err = m->err;
  if (m->lnak_cplx) return launch_tc<true, true, 64, 2, EPI_C128>(s, p, wc);
  return launch_tc<true, false, 128, 2, EPI_C128>(s, p, wc);
}

int exchange_fused_tc(cudaStream_t s, const float* const Gp[4], long ldG, long off,
                      const float* const Lp[2], int W, int N, int Nc, int M, int nsplit,
                      c128* exx, c128* kl, unsigned* err);

bool exchange_fused_ok(MixedHam* m, int sp) {
  return !m->lnak_cplx && m->nel[sp] >= 1 && m->nel[sp] <= 50;
}

int exchange_fused(cudaStream_t s, MixedHam* m, int sp, int W, c128* exx, c128* kl) {
  const float* Gp[4] = {m->G.p[0], m->G.p[1], m->G.p[2], m->G.p[3]};
  const float* Lp[2] = {m->Lnak[sp].p[0], m->Lnak[sp].p[1]};
  return exchange_fused_tc(s, Gp, m->G.ld, long(m->el_off[sp]) * m->M, Lp, W, m->nel[sp], m->Nc,
                           m->M, m->exchange_split, exx, kl, m->err);
}

int mixed_set_exchange_split(MixedHam* m, int nsplit) {
  if (nsplit != 1 && nsplit != 3) {
    set_error_detail("exchange split must be 1 or 3");
    return AFQMC_ERR_ARG;
  }
  m->exchange_split = nsplit;
  return AFQMC_OK;
}

int mixed_error_flag(MixedHam* m, unsigned* flag) {
  AFQMC_CUDA_TRY(cudaMemcpy(flag, m->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return AFQMC_OK;
}

}  // namespace afqmc
