// Fused Taylor propagation of the walkers on the tensor cores (mixed precision).
//
// Reference: det_ops::detail::propagate_impl / apply_expM (src/AFQMC/SlaterDeterminantOperations/
// propagate.hpp:41-70, 238-298):  S <- P1 * sum_{n=0..order} (i V)^n / n! * P1 * S, with the Taylor
// terms built iteratively T_n = (i/n) V T_{n-1}.
//
// One persistent CTA takes one walker at a time through all order+2 products ("phases"):
//   phase 0          T_0 = P1 S                    (A = P1, real;   B = S^T planes)
//   phase 1..order   T_n = (i/n) V_w T_{n-1}       (A = V_w planes; B = T_{n-1}^T planes)
//   phase order+1    S   = P1 R                    (A = P1;         B = R^T planes)
// Each phase is up to two 128-row tiles (M <= 256 orbitals) x 64 columns (N <= 64 electrons),
// FP32 accumulators in TMEM, 3xTF32 split products.  The running sum R = sum_n T_n stays in TMEM
// (columns 256..511); each T_n goes through global memory (one walker's worth, L2-resident) as the
// K-major B operand of the next phase, handed from the epilogue warps to the TMA warp by an
// mbarrier after an async-proxy fence.  V_w is re-read per term from L2 instead of HBM.
#include "mixed.cuh"
#include "tc.cuh"

namespace afqmc {
namespace {

constexpr int TY_THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int TBK = 32;
constexpr int TBN = 64;           // electrons per tile (N <= 64)
constexpr int T_STAGES = 2;
constexpr int T_A_TILE = 128 * TBK * 4;
constexpr int T_B_TILE = TBN * TBK * 4;
constexpr int T_STAGE = 4 * T_A_TILE + 4 * T_B_TILE;  // 96 KB
constexpr size_t T_SMEM = size_t(T_STAGES) * T_STAGE + 1024 + 256;

struct TyParams {
  CUtensorMap p1[2];     // P1 planes hi, lo: {M, M, 1}
  CUtensorMap v[4];      // V planes: {M, M, W}
  CUtensorMap s[4];      // S^T planes: {M, N, W}
  CUtensorMap t[2][4];   // T ping-pong planes: {M, N, W}
  CUtensorMap r[4];      // R^T planes: {M, N, W}
  float* tp[2][4];       // T ping-pong planes (epilogue writes) [W][N][M]
  float* rp[4];          // R planes [W][N][M]
  c128* S;               // walker Slater matrices (output), [W] x ldS, [M][N] each
  long ldS;
  long pl_ld, pl_bs;     // ld / batch stride of the [W][N][M] planes
  int W, M, N, order;
  unsigned* err;
};

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void split_store(float v, float* hi, float* lo, long idx) {
  const float h = tc::tf32_hi(v);
  hi[idx] = h;
  lo[idx] = v - h;
}

__global__ void __launch_bounds__(TY_THREADS, 1) taylor_tc_kernel(const __grid_constant__ TyParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + T_STAGES * T_STAGE);
  uint64_t* empty = full + T_STAGES;
  uint64_t* acc_full = empty + T_STAGES;  // [2] per m tile
  uint64_t* acc_empty = acc_full + 2;     // [2]
  uint64_t* phase_done = acc_empty + 2;   // epilogue -> TMA: T_n written
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(phase_done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nph = p.order + 2;
  const int nk = (p.M + TBK - 1) / TBK;
  const int MT = (p.M + 127) / 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < T_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], 128);
    }
    tc::mbar_init(phase_done, 128);
    *abort_flag = 0;
    tc::fence_mbar_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t taddr = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      long it = 0, wi = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < p.W && ok; w += gridDim.x, ++wi) {
        for (int ph = 0; ph < nph && ok; ++ph) {
          const bool p1 = (ph == 0 || ph == nph - 1);
          const CUtensorMap* amap = p1 ? p.p1 : p.v;
          const CUtensorMap* bmap = ph == 0 ? p.s : (ph == nph - 1 ? p.r : p.t[(ph - 1) & 1]);
          const int na = p1 ? 2 : 4;
          const unsigned bytes = unsigned(na * T_A_TILE + 4 * T_B_TILE);
          bool b_ready = (ph == 0);
          for (int mt = 0; mt < MT && ok; ++mt)
            for (int kc = 0; kc < nk; ++kc, ++it) {
              const int s = int(it % T_STAGES);
              if (it >= T_STAGES) {
                if (!tc::mbar_wait(&empty[s], unsigned((it / T_STAGES) - 1) & 1u, p.err,
                                   abort_flag)) {
                  ok = false;
                  break;
                }
              }
              unsigned char* st = base + size_t(s) * T_STAGE;
              tc::mbar_arrive_expect_tx(&full[s], bytes);
              // A (P1 or V_w) does not depend on the previous phase: issue it first
              for (int q = 0; q < na; ++q)
                tc::tma_load_3d(st + q * T_A_TILE, &amap[q], &full[s], kc * TBK, mt * 128,
                                p1 ? 0 : w);
              if (!b_ready) {
                // B of this phase is the previous phase's output, written by the epilogue warps
                const long done = wi * (nph - 1) + (ph - 1);
                if (!tc::mbar_wait(phase_done, unsigned(done) & 1u, p.err, abort_flag)) {
                  ok = false;
                  break;
                }
                b_ready = true;
              }
              for (int q = 0; q < 4; ++q)
                tc::tma_load_3d(st + 4 * T_A_TILE + q * T_B_TILE, &bmap[q], &full[s], kc * TBK, 0,
                                w);
            }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_tf32(128, TBN, false);
      constexpr uint32_t IDN = tc::idesc_tf32(128, TBN, true);
      long it = 0, use = 0;  // use: accumulator uses (per m tile, same count for both)
      bool ok = true;
      for (int w = blockIdx.x; w < p.W && ok; w += gridDim.x) {
        for (int ph = 0; ph < nph && ok; ++ph, ++use) {
          const bool p1 = (ph == 0 || ph == nph - 1);
          for (int mt = 0; mt < MT && ok; ++mt) {
            if (use >= 1) {
              if (!tc::mbar_wait(&acc_empty[mt], unsigned(use - 1) & 1u, p.err, abort_flag)) {
                ok = false;
                break;
              }
            }
            tc::tc_fence_after();
            const uint32_t dr = taddr + uint32_t(mt * 2 * TBN), di = dr + TBN;
            for (int kc = 0; kc < nk; ++kc, ++it) {
              const int s = int(it % T_STAGES);
              if (!tc::mbar_wait(&full[s], unsigned(it / T_STAGES) & 1u, p.err, abort_flag)) {
                ok = false;
                break;
              }
              tc::tc_fence_after();
              unsigned char* st = base + size_t(s) * T_STAGE;
              const uint32_t sa = tc::smem_u32(st);
              const uint32_t sb = tc::smem_u32(st + 4 * T_A_TILE);
#pragma unroll
              for (int kk = 0; kk < TBK / 8; ++kk) {
                auto A = [&](int q) { return tc::sdesc_sw128(sa + q * T_A_TILE) + uint64_t(2 * kk); };
                auto B = [&](int q) { return tc::sdesc_sw128(sb + q * T_B_TILE) + uint64_t(2 * kk); };
                const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
                if (p1) {
                  // real A (P1 hi, lo) x complex B
                  tc::mma_tf32(dr, A(0), B(0), ID, acc0);
                  tc::mma_tf32(dr, A(0), B(1), ID, 1);
                  tc::mma_tf32(dr, A(1), B(0), ID, 1);
                  tc::mma_tf32(di, A(0), B(2), ID, acc0);
                  tc::mma_tf32(di, A(0), B(3), ID, 1);
                  tc::mma_tf32(di, A(1), B(2), ID, 1);
                } else {
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
                }
              }
              tc::mma_commit(&empty[s]);
            }
            if (!ok) break;
            tc::mma_commit(&acc_full[mt]);
          }
        }
      }
    }
  } else {
    // epilogue warps: TMEM lane quarter q = warp % 4, one accumulator row per thread
    const int q = warp & 3;
    long use = 0;
    bool ok = true;
    for (int w = blockIdx.x; w < p.W && ok; w += gridDim.x) {
      for (int ph = 0; ph < nph && ok; ++ph, ++use) {
        // alpha = 1 (P1 phases) or i/ph (Taylor term ph)
        const bool taylor = (ph > 0 && ph < nph - 1);
        const float ai = taylor ? 1.0f / float(ph) : 0.0f;
        for (int mt = 0; mt < MT; ++mt) {
          if (!tc::mbar_wait(&acc_full[mt], unsigned(use) & 1u, p.err, abort_flag)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          const int row = mt * 128 + q * 32 + lane;  // orbital index i
          const bool rok = row < p.M;
          const uint32_t lane_off = uint32_t(q * 32) << 16;
          const uint32_t tacc = taddr + lane_off + uint32_t(mt * 2 * TBN);
          const uint32_t tsum = taddr + lane_off + 256u + uint32_t(mt * 2 * TBN);
          const long wb = long(w) * p.pl_bs;
#pragma unroll 1
          for (int c0 = 0; c0 < TBN; c0 += 16) {
            float vr[16], vi[16], sr[16], si[16];
            tc::tmem_ld16(tacc + c0, vr);
            tc::tmem_ld16(tacc + TBN + c0, vi);
            if (taylor) {
              tc::tmem_ld16(tsum + c0, sr);
              tc::tmem_ld16(tsum + TBN + c0, si);
            }
            tc::tmem_ld_wait();
            if (taylor) {
              // x = (i/ph) * acc
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const float xr = -ai * vi[j];
                const float xi = ai * vr[j];
                vr[j] = xr;
                vi[j] = xi;
              }
            }
            if (ph == nph - 1) {
              // S = P1 R  (complex128 walker matrix [M][N])
              if (rok)
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  const int n = c0 + j;
                  if (n < p.N) p.S[long(w) * p.ldS + long(row) * p.N + n] = cmk(vr[j], vi[j]);
                }
            } else {
              if (ph == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  sr[j] = vr[j];
                  si[j] = vi[j];
                }
              } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  sr[j] += vr[j];
                  si[j] += vi[j];
                }
              }
              tmem_st16(tsum + c0, sr);
              tmem_st16(tsum + TBN + c0, si);
              if (rok) {
                const bool last = (ph == nph - 2);
                float* const* dst = last ? p.rp : p.tp[ph & 1];
                const float* yr = last ? sr : vr;
                const float* yi = last ? si : vi;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  const int n = c0 + j;
                  if (n < p.N) {
                    // transposed store [w][n][i]: consecutive threads, consecutive i
                    const long idx = wb + long(n) * p.pl_ld + row;
                    split_store(yr[j], dst[0], dst[1], idx);
                    split_store(yi[j], dst[2], dst[3], idx);
                  }
                }
              }
            }
          }
          tmem_st_wait();
          tc::tc_fence_before();
          tc::mbar_arrive(&acc_empty[mt]);
        }
        if (!ok) break;
        if (ph < nph - 1) {
          // make this phase's planes visible to the TMA loads of the next phase
          fence_proxy_async_global();
          tc::mbar_arrive(phase_done);
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(taddr, 512);
}

int g_nsm = 0;

}  // namespace

int make_plane_map_3d(CUtensorMap* map, const float* base, long k, long rows, long row_stride,
                      long batch, long batch_stride, int box_rows, int box_batch);

int taylor_fused_tc(cudaStream_t s, const float* const P1p[2], const float* const Vp[4],
                    long ldV, const float* const Sp[4], float* const Tp0[4], float* const Tp1[4],
                    float* const Rp[4], long pl_ld, c128* S, long ldS, int W, int M, int N,
                    int order, unsigned* err) {
  if (M > 256 || N > TBN || order < 0) {
    set_error_detail("taylor_fused_tc: M = %d (<= 256), N = %d (<= 64), order = %d", M, N, order);
    return AFQMC_ERR_UNSUPPORTED;
  }
  TyParams p{};
  for (int q = 0; q < 2; ++q)
    AFQMC_TRY(make_plane_map_3d(&p.p1[q], P1p[q], M, M, pl_ld, 1, long(M) * pl_ld, 128, 1));
  for (int q = 0; q < 4; ++q) {
    AFQMC_TRY(make_plane_map_3d(&p.v[q], Vp[q], M, M, ldV, W, long(M) * ldV, 128, 1));
    AFQMC_TRY(make_plane_map_3d(&p.s[q], Sp[q], M, N, pl_ld, W, long(N) * pl_ld, TBN, 1));
    AFQMC_TRY(make_plane_map_3d(&p.t[0][q], Tp0[q], M, N, pl_ld, W, long(N) * pl_ld, TBN, 1));
    AFQMC_TRY(make_plane_map_3d(&p.t[1][q], Tp1[q], M, N, pl_ld, W, long(N) * pl_ld, TBN, 1));
    AFQMC_TRY(make_plane_map_3d(&p.r[q], Rp[q], M, N, pl_ld, W, long(N) * pl_ld, TBN, 1));
    p.tp[0][q] = Tp0[q];
    p.tp[1][q] = Tp1[q];
    p.rp[q] = Rp[q];
  }
  p.S = S;
  p.ldS = ldS;
  p.pl_ld = pl_ld;
  p.pl_bs = long(N) * pl_ld;
  p.W = W;
  p.M = M;
  p.N = N;
  p.order = order;
  p.err = err;
  if (g_nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(taylor_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(T_SMEM)));
  const int grid = W < g_nsm ? W : g_nsm;
  taylor_tc_kernel<<<grid, TY_THREADS, T_SMEM, s>>>(p);
  return launch_status("taylor_tc_kernel");
}

}  // namespace afqmc
