// Fused exchange / Coulomb contraction of the local energy on the tensor cores.
//
// Reference: Real3IndexFactorization::energy_impl (src/AFQMC/HamiltonianOperations/
// Real3IndexFactorization.hpp:476-590) forms T[w,b,n,a] = sum_k G[w,b,k] Lnak[n,a,k] in chunks of
// Cholesky vectors (71 GB at M=200, N=50, Nc=1600, W=1024 if materialised) and reduces
// EXX[w] += -scl/2 sum_{n,a,b} T[w,a,n,b] T[w,b,n,a] and Kl[w,n] = sum_a T[w,a,n,a].
// Here T never leaves the SM: a persistent kernel walks tiles of (2 walkers) x (2 Cholesky
// vectors); each tile is one 128 x 112 tcgen05 accumulator (TF32 split products, FP32 in TMEM):
//   rows   = 2 walker slots of 64 (b = 0..N-1, rows N..63 zero)   <- TMA box {32, 64, 2} of G
//   cols   = 2 vector slots of 56 (a = 0..N-1, cols N..55 zero)   <- TMA box {32, 56, 2} of Lnak
// The epilogue warps copy each walker's N x N block of T_n to shared memory, compute
// sum_{a,b} T[b][a] T[a][b] and the trace per (walker, n) in FP64, and store them; the next tile's
// MMAs run meanwhile into the second TMEM accumulator.
#include <cudaTypedefs.h>

#include "energy.cuh"
#include "mixed.cuh"
#include "tc.cuh"

namespace afqmc {
namespace {

constexpr int XT_THREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2-5 epilogue
constexpr int XBK = 32;
constexpr int XSLOT_A = 64;      // rows per walker slot
constexpr int XSLOT_B = 56;      // cols per Cholesky-vector slot (N <= 56)
constexpr int XBN = 2 * XSLOT_B; // 112
constexpr int NBLK_DEFAULT = 64; // n-pairs per L2 block of the tile order (autotuned: 16..128)

struct XParams {
  CUtensorMap a[4];  // G planes as {M, N, W}: re_hi, re_lo, im_hi, im_lo
  CUtensorMap b[2];  // Lnak planes as {M, N, Nc}: hi, lo (real trial)
  int W, N, Nc, M;
  c128* exx;         // [W][Nc] += sum_{a,b} T[b][a] T[a][b]
  c128* kl;          // [W][Nc] += trace T
  const float* ginv; // FP16 operands: per-walker inverse scale of G (null for TF32)
  float linv;        // FP16 operands: inverse scale of Lnak
  int nblk;          // vector pairs per L2 block of the tile order
  unsigned* err;
};

template <int NSPLIT>
struct XCfg {
  static constexpr int NA = NSPLIT == 3 ? 4 : 2;  // A planes used
  static constexpr int NB = NSPLIT == 3 ? 2 : 1;
  static constexpr int A_TILE = 128 * XBK * 4;
  static constexpr int B_TILE = XBN * XBK * 4;
  static constexpr int STAGE = NA * A_TILE + NB * B_TILE;
  static constexpr int STAGES = NSPLIT == 3 ? 2 : 4;
  static constexpr int STG_BYTES = 2 * 50 * 51 * 8;  // staging of 2 walkers' N x N block (N<=50)
  static constexpr size_t SMEM = size_t(STAGES) * STAGE + STG_BYTES + 1024 + 512;  // +barriers, sums
  static_assert(SMEM <= 232448, "shared memory");
};

__device__ __forceinline__ void named_bar(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// tile t -> (walker pair, vector pair): blocks of nblk vector pairs, inside a block all walker
// pairs for each vector pair in turn, so that a block's Lnak planes stay in L2 while every
// walker pair passes
__device__ __forceinline__ void tile_coords(long t, int WP, int NP, int nblk, int& wp, int& np) {
  const long per_blk = long(WP) * nblk;
  const int nb = int(t / per_blk);
  const long within = t % per_blk;
  const int width = min(nblk, NP - nb * nblk);
  wp = int(within / width);
  np = nb * nblk + int(within % width);
}

template <int NSPLIT, bool F16>
__global__ void __launch_bounds__(XT_THREADS, 1) exchange_tc_kernel(const __grid_constant__ XParams p) {
  using K = XCfg<NSPLIT>;
  // 128 bytes of K per stage and operand row: 32 TF32 or 64 FP16 elements; 32 bytes per MMA
  constexpr int XBKE = F16 ? 2 * XBK : XBK;
  constexpr int KSTEP = F16 ? 16 : 8;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  float* stg = reinterpret_cast<float*>(base + K::STAGES * K::STAGE);  // [2][N][PITCH] re, im
  uint64_t* full = reinterpret_cast<uint64_t*>(base + K::STAGES * K::STAGE + K::STG_BYTES);
  uint64_t* empty = full + K::STAGES;
  uint64_t* acc_full = empty + K::STAGES;  // [2]
  uint64_t* acc_empty = acc_full + 2;      // [2]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc_empty + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  double* red = reinterpret_cast<double*>(tmem_slot + 4);  // [4 lane quarters][4] partial sums

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int WP = (p.W + 1) / 2, NP = (p.Nc + 1) / 2;
  const long ntiles = long(WP) * NP;
  const int N = p.N;
  const int PITCH = N | 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < K::STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], 128);
    }
    *abort_flag = 0;
    tc::fence_mbar_init();
    for (int q = 0; q < K::NA; ++q) tc::prefetch_tmap(&p.a[q]);
    for (int q = 0; q < K::NB; ++q) tc::prefetch_tmap(&p.b[q]);
  }
  if (warp == 1) {
    tc::tmem_alloc(tmem_slot, 512);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t taddr = *tmem_slot;
  const int nk = (p.M + XBKE - 1) / XBKE;

  if (warp == 0) {
    if (lane == 0) {
      long it = 0;  // global k-chunk counter (stage ring position)
      for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int wp, np;
        tile_coords(t, WP, NP, p.nblk, wp, np);
        bool ok = true;
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = int(it % K::STAGES);
          if (it >= K::STAGES) {
            if (!tc::mbar_wait(&empty[s], unsigned((it / K::STAGES) - 1) & 1u, p.err, abort_flag)) {
              ok = false;
              break;
            }
          }
          unsigned char* st = base + size_t(s) * K::STAGE;
          tc::mbar_arrive_expect_tx(&full[s], K::STAGE);
          // A planes: re_hi, (re_lo), im_hi, (im_lo) -> plane order in smem 0..NA-1
#pragma unroll
          for (int q = 0; q < K::NA; ++q)
            tc::tma_load_3d(st + q * K::A_TILE, &p.a[q], &full[s], kc * XBKE, 0, 2 * wp);
#pragma unroll
          for (int q = 0; q < K::NB; ++q)
            tc::tma_load_3d(st + K::NA * K::A_TILE + q * K::B_TILE, &p.b[q], &full[s], kc * XBKE,
                            0, 2 * np);
        }
        if (!ok) break;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_split<F16>(128, XBN, false);
      long it = 0;
      long ti = 0;
      bool ok = true;
      for (long t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++ti) {
        const int buf = int(ti & 1);
        // wait for the epilogue to have drained this accumulator (tile ti-2)
        if (ti >= 2) {
          if (!tc::mbar_wait(&acc_empty[buf], unsigned((ti / 2) - 1) & 1u, p.err, abort_flag)) {
            ok = false;
            break;
          }
        }
        tc::tc_fence_after();
        const uint32_t dr = taddr + uint32_t(buf * 2 * XBN);
        const uint32_t di = dr + XBN;
        for (int kc = 0; kc < nk; ++kc, ++it) {
          const int s = int(it % K::STAGES);
          if (!tc::mbar_wait(&full[s], unsigned(it / K::STAGES) & 1u, p.err, abort_flag)) {
            ok = false;
            break;
          }
          tc::tc_fence_after();
          unsigned char* st = base + size_t(s) * K::STAGE;
          const uint32_t sa = tc::smem_u32(st);
          const uint32_t sb = tc::smem_u32(st + K::NA * K::A_TILE);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            if (kc * XBKE + kk * KSTEP >= p.M) break;  // zero fill past K
            auto A = [&](int q) { return tc::sdesc_sw128(sa + q * K::A_TILE) + uint64_t(2 * kk); };
            auto B = [&](int q) { return tc::sdesc_sw128(sb + q * K::B_TILE) + uint64_t(2 * kk); };
            const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
            if constexpr (NSPLIT == 3) {
              // Dr = Gr L, Di = Gi L (real trial): hi*hi + hi*lo + lo*hi
              tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<F16>(dr, A(0), B(1), ID, 1);
              tc::mma_split<F16>(dr, A(1), B(0), ID, 1);
              tc::mma_split<F16>(di, A(2), B(0), ID, acc0);
              tc::mma_split<F16>(di, A(2), B(1), ID, 1);
              tc::mma_split<F16>(di, A(3), B(0), ID, 1);
            } else {
              tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<F16>(di, A(1), B(0), ID, acc0);
            }
          }
          tc::mma_commit(&empty[s]);
        }
        if (!ok) break;
        tc::mma_commit(&acc_full[buf]);
      }
    }
  } else {
    // epilogue: TMEM lane quarter q = warp % 4; lane L = row of the accumulator
    const int q = warp & 3;
    const int L = q * 32 + lane;
    const int wl = L / XSLOT_A, b = L % XSLOT_A;
    const int et = threadIdx.x - 64;  // 0..127
    float2* st2 = reinterpret_cast<float2*>(stg);  // [2 walkers][N][PITCH] (re, im)
    long ti = 0;
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x, ++ti) {
      int wp, np;
      tile_coords(t, WP, NP, p.nblk, wp, np);
      const int buf = int(ti & 1);
      // the four epilogue warps meet at named barriers below: they leave the loop together, on
      // the outcome of all four waits (a wait that gave up on one warp ends every warp's loop)
      bool ok = tc::mbar_wait_warp(&acc_full[buf], unsigned(ti / 2) & 1u, p.err, abort_flag);
      int* const agree = reinterpret_cast<int*>(red + 16);
      if (lane == 0) agree[q] = ok ? 0 : 1;
      named_bar(1, 128);
      ok = (agree[0] | agree[1] | agree[2] | agree[3]) == 0;
      named_bar(1, 128);
      tc::tc_fence_after();
      if (!ok) break;
      const int w = 2 * wp + wl;
      const bool valid = (b < N) && (w < p.W);
      const uint32_t trow = taddr + (uint32_t(q * 32) << 16) + uint32_t(buf * 2 * XBN);
#pragma unroll 1
      for (int nl = 0; nl < 2; ++nl) {
        // row b of T_n (columns a) into registers (fourteen TMEM loads, one wait) and into the
        // staging block, from which the other rows read it as their column
        const int r = (wl * N + b) * PITCH;
        float vr[XSLOT_B], vi[XSLOT_B];
        {
          const uint32_t cr = trow + nl * XSLOT_B, ci = trow + XBN + nl * XSLOT_B;
#pragma unroll
          for (int c = 0; c < XSLOT_B; c += 8) {
            tmem_ld8(cr + c, vr + c);
            tmem_ld8(ci + c, vi + c);
          }
          tc::tmem_ld_wait();
        }
        if (nl == 1) {
          tc::tc_fence_before();
          tc::mbar_arrive(&acc_empty[buf]);  // accumulator free for tile ti+2
        }
        if (F16 && valid) {  // undo the power-of-two operand scales (exact)
          const float f = p.ginv[w] * p.linv;
#pragma unroll
          for (int a = 0; a < XSLOT_B; ++a) {
            vr[a] *= f;
            vi[a] *= f;
          }
        }
        if (valid) {
#pragma unroll
          for (int a = 0; a < XSLOT_B; ++a)
            if (a < N) st2[r + a] = make_float2(vr[a], vi[a]);
        }
        const int n = 2 * np + nl;
        // the running sums this tile adds to, fetched now so their latency hides behind the loop
        const int ww = 2 * wp + et;
        const bool upd = et < 2 && n < p.Nc && ww < p.W;
        const long o = long(ww) * p.Nc + n;
        c128 exx0 = cmk(0.0, 0.0), kl0 = cmk(0.0, 0.0);
        if (upd) {
          exx0 = p.exx[o];
          kl0 = p.kl[o];
        }
        named_bar(1, 128);
        // x = sum_a T[b][a] T[a][b];  tr = T[b][b]   (rows of one warp all belong to walker wl)
        // The sum over a runs in FP32 with four independent accumulator pairs (50 terms of
        // products of FP32 inputs); the partial sums are widened to FP64 for every later sum.
        double v4[4] = {0.0, 0.0, 0.0, 0.0};
        if (valid && n < p.Nc) {
          const int col0 = wl * N * PITCH + b;
          float xr[4] = {0.f, 0.f, 0.f, 0.f}, xi[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int a = 0; a < XSLOT_B; ++a)
            if (a < N) {
              const float2 u = st2[col0 + a * PITCH];  // T[a][b]
              xr[a & 3] = fmaf(vr[a], u.x, fmaf(-vi[a], u.y, xr[a & 3]));
              xi[a & 3] = fmaf(vr[a], u.y, fmaf(vi[a], u.x, xi[a & 3]));
            }
          v4[0] = (double(xr[0]) + double(xr[1])) + (double(xr[2]) + double(xr[3]));
          v4[1] = (double(xi[0]) + double(xi[1])) + (double(xi[2]) + double(xi[3]));
          const float2 d = st2[r + b];
          v4[2] = d.x;
          v4[3] = d.y;
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
          for (int off = 16; off > 0; off >>= 1)
            v4[c] += __shfl_xor_sync(0xffffffffu, v4[c], off);
        if (lane == 0)
#pragma unroll
          for (int c = 0; c < 4; ++c) red[q * 4 + c] = v4[c];
        named_bar(1, 128);
        // red is rewritten only after the next barrier, which these threads reach after their
        // reads; the staging block is rewritten only after every thread passed the one above
        if (upd) {
          // walker slot et = lane quarters {2et, 2et+1}
          const double* r0 = red + (2 * et) * 4;
          const double* r1 = red + (2 * et + 1) * 4;
          p.exx[o] = cadd(exx0, cmk(r0[0] + r1[0], r0[1] + r1[1]));
          p.kl[o] = cadd(kl0, cmk(r0[2] + r1[2], r0[3] + r1[3]));
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(taddr, 512);
}

int g_num_sms = 0;

}  // namespace

int make_plane_map_3d_es(CUtensorMap* map, const void* base, int esize, long k, long rows,
                         long row_stride, long batch, long batch_stride, int box_rows,
                         int box_batch);

namespace {
template <int NSPLIT, bool F16>
int launch_exchange(cudaStream_t s, const XParams& p, int grid) {
  using K = XCfg<NSPLIT>;
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(exchange_tc_kernel<NSPLIT, F16>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, int(K::SMEM)));
  exchange_tc_kernel<NSPLIT, F16><<<grid, XT_THREADS, K::SMEM, s>>>(p);
  return launch_status("exchange_tc_kernel");
}
}  // namespace

// T-free exchange: exx[w][n] += sum_{a,b} T[b][a]T[a][b], kl[w][n] += trace T for spin block sp.
// G planes: [W][ldG] with the spin block at element offset `off` (rows of M); Lnak planes
// [Nc][N][M]; FP32 (esize 4, TF32 split) or FP16 (esize 2, FP16 split: G rows scaled per walker,
// g_inv[w] and l_inv the inverse scales).
int exchange_fused_tc(cudaStream_t s, const void* const Gp[4], int esize, long ldG, long off,
                      const void* const Lp[2], int W, int N, int Nc, int M, int nsplit,
                      const float* g_inv, float l_inv, c128* exx, c128* kl, unsigned* err,
                      int nblk) {
  if (N > 50 || N < 1) {
    set_error_detail("exchange_fused_tc: N = %d outside 1..50", N);
    return AFQMC_ERR_UNSUPPORTED;
  }
  XParams p{};
  // A planes in the order the kernel expects: 3-split {re_hi, re_lo, im_hi, im_lo},
  // 1-split {re_hi, im_hi}
  const int amap3[4] = {0, 1, 2, 3}, amap1[2] = {0, 2};
  const int na = nsplit == 3 ? 4 : 2;
  for (int q = 0; q < na; ++q) {
    const int src = nsplit == 3 ? amap3[q] : amap1[q];
    AFQMC_TRY(make_plane_map_3d_es(&p.a[q], static_cast<const char*>(Gp[src]) + off * esize,
                                   esize, M, N, M, W, ldG, XSLOT_A, 2));
  }
  const int nb = nsplit == 3 ? 2 : 1;
  for (int q = 0; q < nb; ++q)
    AFQMC_TRY(make_plane_map_3d_es(&p.b[q], Lp[q], esize, M, N, M, Nc, long(N) * M, XSLOT_B, 2));
  p.W = W;
  p.N = N;
  p.Nc = Nc;
  p.M = M;
  p.exx = exx;
  p.kl = kl;
  p.ginv = g_inv;
  p.linv = l_inv;
  p.nblk = nblk > 0 ? nblk : NBLK_DEFAULT;
  p.err = err;
  if (g_num_sms == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev);
  }
  const long ntiles = long((W + 1) / 2) * ((Nc + 1) / 2);
  const int grid = int(ntiles < g_num_sms ? ntiles : g_num_sms);
  const bool f16 = esize == 2;
  if (f16 && !g_inv) {
    set_error_detail("exchange_fused_tc: FP16 planes without their scales");
    return AFQMC_ERR_ARG;
  }
  if (nsplit == 3) return f16 ? launch_exchange<3, true>(s, p, grid) : launch_exchange<3, false>(s, p, grid);
  return f16 ? launch_exchange<1, true>(s, p, grid) : launch_exchange<1, false>(s, p, grid);
}

}  // namespace afqmc
