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

#include <cstring>
#include <memory>
#include <new>
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
  EPI_VHS_SYM = 5,   // symmetric L: tile nt = (i block, k block) of the upper triangle; out
                     // planes [row][i][k] and [row][k][i] = split(alpha * acc), alpha real
  EPI_C64T = 6,      // out_c as complex64 [z][col][row] = alpha * col_inv[col] * acc
};

// Symmetric vHS tiles: the BN = 128 columns of a tile are the (i, k) pairs of an 8 x 16 block,
// column j = 8-row offset * 16 + 16-column offset; only blocks holding some i <= k are computed.
constexpr int SYM_IB = 8, SYM_KB = 16, SYM_MAXIB = 32;

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
  const float* col_inv;  // EPI_C64T: per-column scale (the B operand's row scale)
  int vhs_M;            // EPI_VHS: columns are (i, k) pairs of an M x M matrix
  // FP16 operands: the accumulator row r is multiplied by row_inv[r] (the A operand's row scale;
  // the B operand's scale is folded into alpha) before the epilogue uses it
  const float* row_inv;
  // EPI_VHS / EPI_VHS_SYM with out_f16: the output planes are FP16 holding value * out_sc[row]
  int out_f16;
  const float* out_sc;
  // EPI_VHS_SYM: sym_pre[a] = tiles of the i blocks before block a (a = 0..sym_nib), sym_nkb =
  // number of k blocks; block a covers the top sym_pre[a+1] - sym_pre[a] k blocks
  int sym_nib, sym_nkb;
  int sym_pre[SYM_MAXIB + 1];
  unsigned* err;
};

// tile nt of the symmetric vHS -> (i block a, k block c)
__device__ __forceinline__ void sym_tile(const TcParams& p, int nt, int& a, int& c) {
  a = 0;
  while (a + 1 < p.sym_nib && p.sym_pre[a + 1] <= nt) ++a;
  const int cnt = p.sym_pre[a + 1] - p.sym_pre[a];
  c = p.sym_nkb - cnt + (nt - p.sym_pre[a]);
}

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
  float h, l;
  tc::tf32_split(v, h, l);
  hi[idx] = h;
  lo[idx] = l;
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

// Epilogue of a symmetric vHS tile (BN = 128 columns = 8 x 16 (i, k) pairs) for one walker row:
// each value goes to V[w][i][k] (i <= k) and V[w][k][i] (i < k), the real then the imaginary
// part, so that a thread holds a whole 8 x 16 block (128 registers) and writes rows of 16 (direct)
// and 8 (mirrored) consecutive floats.
template <int NRUN>
__device__ __forceinline__ void store_run(float* hi, float* lo, long idx, const float* v,
                                          int first, int last, float alpha) {
  // v[0..NRUN): consecutive values of one row at idx; only offsets [first, last) are written
  // (fully unrolled: v stays in registers)
  if (first == 0 && last == NRUN) {
#pragma unroll
    for (int j = 0; j < NRUN; j += 4) {
      float4 h, l;
      tc::tf32_split(alpha * v[j + 0], h.x, l.x);
      tc::tf32_split(alpha * v[j + 1], h.y, l.y);
      tc::tf32_split(alpha * v[j + 2], h.z, l.z);
      tc::tf32_split(alpha * v[j + 3], h.w, l.w);
      *reinterpret_cast<float4*>(hi + idx + j) = h;
      *reinterpret_cast<float4*>(lo + idx + j) = l;
    }
  } else {
#pragma unroll
    for (int j = 0; j < NRUN; ++j)
      if (j >= first && j < last) split_store(alpha * v[j], hi, lo, idx + j);
  }
}

// the same run stored as FP16 split planes (value * alpha already in the FP16 range)
template <int NRUN>
__device__ __forceinline__ void store_run16(__half* hi, __half* lo, long idx, const float* v,
                                            int first, int last, float alpha) {
  if (first == 0 && last == NRUN) {
#pragma unroll
    for (int j = 0; j < NRUN; j += 8) {
      __align__(16) __half h[8], l[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) tc::f16_split(alpha * v[j + t], h[t], l[t]);
      *reinterpret_cast<uint4*>(hi + idx + j) = *reinterpret_cast<const uint4*>(h);
      *reinterpret_cast<uint4*>(lo + idx + j) = *reinterpret_cast<const uint4*>(l);
    }
  } else {
#pragma unroll
    for (int j = 0; j < NRUN; ++j)
      if (j >= first && j < last) {
        __half h, l;
        tc::f16_split(alpha * v[j], h, l);
        hi[idx + j] = h;
        lo[idx + j] = l;
      }
  }
}

__device__ __forceinline__ void vhs_sym_epilogue(const TcParams& p, uint32_t trow, int row, int nt,
                                                 uint64_t* acc_free) {
  int ab, cb;
  sym_tile(p, nt, ab, cb);
  const int M = p.vhs_M, i0 = ab * SYM_IB, k0 = cb * SYM_KB;
  float alpha = float(p.alpha.x) * ((p.row_inv && row < p.m) ? p.row_inv[row] : 1.f);
  if (p.out_f16 && row < p.m) alpha *= p.out_sc[row];
  const long wb = long(row) * p.out_bs;
#pragma unroll 1
  for (int part = 0; part < 2; ++part) {  // 0: real part, 1: imaginary part
    float v[SYM_IB][SYM_KB];
#pragma unroll
    for (int a = 0; a < SYM_IB; ++a)
      tc::tmem_ld16(trow + uint32_t(part * 128 + a * SYM_KB), v[a]);
    tc::tmem_ld_wait();
    if (part == 1) {
      tc::tc_fence_before();
      tc::mbar_arrive(acc_free);  // accumulator free for the tile after next
    }
    if (row >= p.m) continue;
    float* hi = p.out[2 * part];
    float* lo = p.out[2 * part + 1];
    __half* hi16 = reinterpret_cast<__half*>(hi);
    __half* lo16 = reinterpret_cast<__half*>(lo);
    // direct rows V[w][i][k0 .. k0+15], k >= i
#pragma unroll
    for (int a = 0; a < SYM_IB; ++a) {
      const int i = i0 + a;
      if (i >= M) break;
      const int first = i > k0 ? i - k0 : 0;
      const int last = M - k0 < SYM_KB ? M - k0 : SYM_KB;
      if (first >= last) continue;
      if (p.out_f16)
        store_run16<SYM_KB>(hi16, lo16, wb + long(i) * p.out_ld + k0, v[a], first, last, alpha);
      else
        store_run<SYM_KB>(hi, lo, wb + long(i) * p.out_ld + k0, v[a], first, last, alpha);
    }
    // mirrored rows V[w][k][i0 .. i0+7], i < k
#pragma unroll
    for (int b = 0; b < SYM_KB; ++b) {
      const int k = k0 + b;
      if (k >= M) break;
      if (k <= i0) continue;
      float col[SYM_IB];
#pragma unroll
      for (int a = 0; a < SYM_IB; ++a) col[a] = v[a][b];
      const int last = min(min(k - i0, SYM_IB), M - i0);
      if (p.out_f16)
        store_run16<SYM_IB>(hi16, lo16, wb + long(k) * p.out_ld + i0, col, 0, last, alpha);
      else
        store_run<SYM_IB>(hi, lo, wb + long(k) * p.out_ld + i0, col, 0, last, alpha);
    }
  }
}

// Persistent tensor-core GEMM: one CTA per SM walks the tiles; the TMA ring runs ahead across
// tiles and the epilogue of tile i overlaps the MMAs of tile i+1 (two TMEM accumulators).
template <bool A_CPLX, bool B_CPLX, int BN, int STAGES, int EPI, bool F16>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_cgemm_kernel(const __grid_constant__ TcParams p) {
  // a stage holds 128 bytes of K per operand row: 32 TF32 or 64 FP16 elements; one MMA takes
  // 32 bytes of it (K = 8 TF32 or 16 FP16)
  constexpr int BKE = F16 ? 2 * BK : BK;
  constexpr int KSTEP = F16 ? 16 : 8;
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
  const int nk = (p.k + BKE - 1) / BKE;

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
            tc::tma_load_3d(st + q * K::A_TILE, &p.a[q], &full[s], kc * BKE, mt * 128, za);
          if constexpr (EPI == EPI_VHS_SYM) {
            // B rows of the (i block, k block) pairs: box {32, 16 k, 8 i} of L viewed [i][k][n]
            int ab, cb;
            sym_tile(p, nt, ab, cb);
#pragma unroll
            for (int q = 0; q < K::NB; ++q)
              tc::tma_load_3d(st + K::NA * K::A_TILE + q * K::B_TILE, &p.b[q], &full[s],
                              kc * BKE, cb * SYM_KB, ab * SYM_IB);
          } else {
#pragma unroll
            for (int q = 0; q < K::NB; ++q)
              tc::tma_load_3d(st + K::NA * K::A_TILE + q * K::B_TILE, &p.b[q], &full[s],
                              kc * BKE, nt * BN, zb);
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_split<F16>(128, BN, false);
      constexpr uint32_t IDN = tc::idesc_split<F16>(128, BN, true);
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
          for (int kk = 0; kk < 4; ++kk) {
            if (kc * BKE + kk * KSTEP >= p.k) break;  // zero fill past K
            // +32 bytes per K step inside the 128-byte swizzle row (descriptor units of 16 B)
            auto A = [&](int q) { return tc::sdesc_sw128(sa + q * K::A_TILE) + uint64_t(2 * kk); };
            auto B = [&](int q) { return tc::sdesc_sw128(sb + q * K::B_TILE) + uint64_t(2 * kk); };
            const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
            if constexpr (A_CPLX && B_CPLX) {
              // Dr = Ar Br - Ai Bi ; Di = Ar Bi + Ai Br  (planes 0 re_hi, 1 re_lo, 2 im_hi, 3 im_lo)
              tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<F16>(dr, A(0), B(1), ID, 1);
              tc::mma_split<F16>(dr, A(1), B(0), ID, 1);
              tc::mma_split<F16>(dr, A(2), B(2), IDN, 1);
              tc::mma_split<F16>(dr, A(2), B(3), IDN, 1);
              tc::mma_split<F16>(dr, A(3), B(2), IDN, 1);
              tc::mma_split<F16>(di, A(0), B(2), ID, acc0);
              tc::mma_split<F16>(di, A(0), B(3), ID, 1);
              tc::mma_split<F16>(di, A(1), B(2), ID, 1);
              tc::mma_split<F16>(di, A(2), B(0), ID, 1);
              tc::mma_split<F16>(di, A(2), B(1), ID, 1);
              tc::mma_split<F16>(di, A(3), B(0), ID, 1);
            } else if constexpr (A_CPLX) {
              // real B (planes 0 hi, 1 lo)
              tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<F16>(dr, A(0), B(1), ID, 1);
              tc::mma_split<F16>(dr, A(1), B(0), ID, 1);
              tc::mma_split<F16>(di, A(2), B(0), ID, acc0);
              tc::mma_split<F16>(di, A(2), B(1), ID, 1);
              tc::mma_split<F16>(di, A(3), B(0), ID, 1);
            } else {
              // real A, complex B
              tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<F16>(dr, A(0), B(1), ID, 1);
              tc::mma_split<F16>(dr, A(1), B(0), ID, 1);
              tc::mma_split<F16>(di, A(0), B(2), ID, acc0);
              tc::mma_split<F16>(di, A(0), B(3), ID, 1);
              tc::mma_split<F16>(di, A(1), B(2), ID, 1);
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
      const bool ok =
          tc::mbar_wait_warp(&acc_full[buf], unsigned(ti / 2) & 1u, p.err, abort_flag);
      tc::tc_fence_after();
      if (!ok) break;
      const int row = mt * 128 + q * 32 + lane;
      const int n0 = nt * BN;
      const uint32_t trow = taddr + (uint32_t(q * 32) << 16) + uint32_t(buf * 2 * BN);
      if constexpr (EPI == EPI_VHS_SYM) {
        vhs_sym_epilogue(p, trow, row, nt, &acc_empty[buf]);
        continue;
      }
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
        if (p.row_inv) {
          const float f = p.row_inv[row];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            vr[j] *= f;
            vi[j] *= f;
          }
        }
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
          } else if constexpr (EPI == EPI_C64T) {
            // lanes hold consecutive rows: consecutive addresses of the transposed output
            const float f = p.col_inv ? p.col_inv[col] : 1.f;
            reinterpret_cast<float2*>(p.out_c)[long(z) * p.outc_bs + long(col) * p.outc_ld + row] =
                make_float2(xr * f, xi * f);
          } else if constexpr (EPI == EPI_PLANES) {
            const long idx = long(z) * p.out_bs + long(row) * p.out_ld + col;
            split_store(xr, p.out[0], p.out[1], idx);
            split_store(xi, p.out[2], p.out[3], idx);
          } else if constexpr (EPI == EPI_VHS) {
            const int i = col / p.vhs_M, kq = col - i * p.vhs_M;
            const long idx = long(row) * p.out_bs + long(i) * p.out_ld + kq;
            if (p.out_f16) {
              const float sc = p.out_sc[row];
              __half h, l;
              tc::f16_split(xr * sc, h, l);
              reinterpret_cast<__half*>(p.out[0])[idx] = h;
              reinterpret_cast<__half*>(p.out[1])[idx] = l;
              tc::f16_split(xi * sc, h, l);
              reinterpret_cast<__half*>(p.out[2])[idx] = h;
              reinterpret_cast<__half*>(p.out[3])[idx] = l;
            } else {
              split_store(xr, p.out[0], p.out[1], idx);
              split_store(xi, p.out[2], p.out[3], idx);
            }
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

// 3D map over an FP32 (esize 4) or FP16 (esize 2) plane: element (x, y, z) at base +
// (z*batch_stride + y*row_stride + x) * esize for x < k, y < rows, z < batch; box {128 bytes of
// x, box_rows, box_batch}, 128-byte swizzle, zero fill outside.
int make_plane_map_3d_es(CUtensorMap* map, const void* base, int esize, long k, long rows,
                         long row_stride, long batch, long batch_stride, int box_rows,
                         int box_batch) {
  auto fn = encode_fn();
  if (!fn) {
    set_error_detail("cuTensorMapEncodeTiled is not available");
    return AFQMC_ERR_CUDA;
  }
  if (batch == 1) batch_stride = rows * row_stride;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (row_stride * esize) % 16 ||
      (batch_stride * esize) % 16) {
    set_error_detail("make_plane_map_3d: plane not 16-byte aligned (row stride=%ld, batch "
                     "stride=%ld, element size %d)", row_stride, batch_stride, esize);
    return AFQMC_ERR_SHAPE;
  }
  cuuint64_t dims[3] = {cuuint64_t(k), cuuint64_t(rows), cuuint64_t(batch)};
  cuuint64_t strides[2] = {cuuint64_t(row_stride * esize), cuuint64_t(batch_stride * esize)};
  cuuint32_t box[3] = {cuuint32_t(128 / esize), cuuint32_t(box_rows), cuuint32_t(box_batch)};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, esize == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                  3, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error_detail("cuTensorMapEncodeTiled failed (%d): k=%ld rows=%ld batch=%ld box=%dx%d "
                     "esize=%d", int(r), k, rows, batch, box_rows, box_batch, esize);
    return AFQMC_ERR_CUDA;
  }
  return AFQMC_OK;
}

int make_plane_map_3d(CUtensorMap* map, const float* base, long k, long rows, long row_stride,
                      long batch, long batch_stride, int box_rows, int box_batch) {
  return make_plane_map_3d_es(map, base, 4, k, rows, row_stride, batch, batch_stride, box_rows,
                              box_batch);
}

namespace {

int make_map(CUtensorMap* map, const float* base, long k, long rows, long ld, long batch,
             long batch_stride, int box_rows) {
  return make_plane_map_3d(map, base, k, rows, ld, batch, batch_stride, box_rows, 1);
}

// Split planes of one operand: 4 (complex) or 2 (real) arrays [batch][rows][ld] of FP32 (TF32
// split, esize 4) or FP16 (FP16 split, esize 2) elements; p[] holds the base addresses.
struct Planes {
  float* p[4] = {nullptr, nullptr, nullptr, nullptr};
  int nplanes = 0;
  int esize = 4;
  long rows = 0, ld = 0, batch = 0, k = 0;
  long bstride() const { return rows * ld; }
  size_t elems() const { return size_t(batch) * rows * ld; }
  __half* h(int q) const { return reinterpret_cast<__half*>(p[q]); }
  // address of element `off` of plane q
  const void* at(int q, long off) const {
    return reinterpret_cast<const char*>(p[q]) + off * esize;
  }
};

int alloc_planes(Planes& P, int nplanes, long batch, long rows, long k, int esize = 4) {
  P.nplanes = nplanes;
  P.esize = esize;
  P.batch = batch;
  P.rows = rows;
  P.k = k;
  const long align = 16 / esize;  // rows start on 16 bytes (TMA strides)
  P.ld = (k + align - 1) / align * align;
  for (int q = 0; q < nplanes; ++q) {
    cudaError_t e = cudaMalloc(&P.p[q], size_t(esize) * P.elems());
    if (e != cudaSuccess) {
      set_error_detail("alloc_planes: %s", cudaGetErrorString(e));
      return AFQMC_ERR_ALLOC;
    }
    AFQMC_CUDA_TRY(cudaMemset(P.p[q], 0, size_t(esize) * P.elems()));
  }
  return AFQMC_OK;
}

int make_map_es(CUtensorMap* map, const Planes& P, int q, long off, long k, long rows, long ld,
                long batch, long batch_stride, int box_rows) {
  return make_plane_map_3d_es(map, P.at(q, off), P.esize, k, rows, ld, batch, batch_stride,
                              box_rows, 1);
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
    AFQMC_TRY(make_map_es(&maps[q], P, q, 0, P.k, P.rows, P.ld, batch, P.bstride(), box_rows));
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// conversions FP64 -> split FP32 planes
// ---------------------------------------------------------------------------------------------
// complex src [b][r][c] (ld_src, bstride_src) -> planes [b][r][c] or transposed [b][c][r]
// rev (non-transposed only): column c goes to column cols-1-c (the K order reversed)
template <bool TRANSPOSE>
__global__ void split_complex_kernel(const c128* __restrict__ src, long ld_src, long bs_src,
                                     int rows, int cols, float* __restrict__ rh,
                                     float* __restrict__ rl, float* __restrict__ ih,
                                     float* __restrict__ il, long ld_dst, long bs_dst, int rev) {
  const long b = blockIdx.z;
  const int r = blockIdx.y * blockDim.y + threadIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows || c >= cols) return;
  const c128 v = src[b * bs_src + long(r) * ld_src + c];
  const int cd = rev ? cols - 1 - c : c;
  const long d = TRANSPOSE ? b * bs_dst + long(c) * ld_dst + r : b * bs_dst + long(r) * ld_dst + cd;
  split_store(float(v.x), rh, rl, d);
  split_store(float(v.y), ih, il, d);
}

__global__ void split_real_kernel(const double* __restrict__ src, long n_rows, long cols,
                                  long ld_src, float* __restrict__ h, float* __restrict__ l,
                                  long ld_dst, int rev) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= n_rows * cols) return;
  const long r = e / cols, c = e % cols;
  split_store(float(src[r * ld_src + c]), h, l, r * ld_dst + (rev ? cols - 1 - c : c));
}

int split_complex(cudaStream_t s, const c128* src, long ld_src, long bs_src, int batch, int rows,
                  int cols, Planes& P, bool transpose, bool rev = false) {
  dim3 blk(32, 8);
  if (transpose) {
    // coalesce the writes along the destination's contiguous (row) index
    dim3 grid(ceil_div(cols, 32), ceil_div(rows, 8), batch);
    split_complex_kernel<true><<<grid, blk, 0, s>>>(src, ld_src, bs_src, rows, cols, P.p[0],
                                                    P.p[1], P.p[2], P.p[3], P.ld, P.bstride(), 0);
  } else {
    dim3 grid(ceil_div(cols, 32), ceil_div(rows, 8), batch);
    split_complex_kernel<false><<<grid, blk, 0, s>>>(src, ld_src, bs_src, rows, cols, P.p[0],
                                                     P.p[1], P.p[2], P.p[3], P.ld, P.bstride(),
                                                     rev ? 1 : 0);
  }
  return launch_status("split_complex_kernel");
}

int split_real_host(const double* src_dev, long rows, long cols, long ld_src, Planes& P,
                    bool rev = false) {
  const long n = rows * cols;
  split_real_kernel<<<ceil_div(n, 256), 256>>>(src_dev, rows, cols, ld_src, P.p[0], P.p[1], P.ld,
                                               rev ? 1 : 0);
  AFQMC_TRY(launch_status("split_real_kernel"));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// conversions FP64 -> FP16 split planes with power-of-two scales
// ---------------------------------------------------------------------------------------------
// One CTA per row r of a complex source [rows][ld_src]: the largest |re|, |im| of the row gives
// the exponent e_r (tc::f16_scale_exponent), inv[r] = 2^-e_r, and the planes receive the FP16
// split of x * 2^e_r.  The scale is exact, so a product of two scaled operands is the product of
// the originals times 2^(e_a + e_b), undone in the epilogue.
constexpr int SPLIT_ROW_THREADS = 256;

__global__ void __launch_bounds__(SPLIT_ROW_THREADS) split_rows_f16_kernel(
    const c128* __restrict__ src, long ld_src, int cols, __half* __restrict__ rh,
    __half* __restrict__ rl, __half* __restrict__ ih, __half* __restrict__ il, long ld_dst,
    float* __restrict__ inv, int rev, float vbound, float* __restrict__ v_inv,
    float* __restrict__ v_sc) {
  __shared__ float wmax[SPLIT_ROW_THREADS / 32], wsum[SPLIT_ROW_THREADS / 32];
  const long r = blockIdx.x;
  const c128* row = src + r * ld_src;
  float m = 0.f, l1 = 0.f;
  for (int c = threadIdx.x; c < cols; c += SPLIT_ROW_THREADS) {
    const c128 v = row[c];
    const float ar = fabsf(float(v.x)), ai = fabsf(float(v.y));
    m = fmaxf(m, fmaxf(ar, ai));
    l1 += ar + ai;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    l1 += __shfl_xor_sync(0xffffffffu, l1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    wmax[threadIdx.x >> 5] = m;
    wsum[threadIdx.x >> 5] = l1;
  }
  __syncthreads();
  m = 0.f;
  l1 = 0.f;
#pragma unroll
  for (int w = 0; w < SPLIT_ROW_THREADS / 32; ++w) {
    m = fmaxf(m, wmax[w]);
    l1 += wsum[w];
  }
  if (v_inv && threadIdx.x == 0) {
    // |sum_n X_n L_n| <= vbound * sum_n |X_n| (vbound = a max |L|): the scale of this row's V
    const int ev = tc::f16_scale_exponent(vbound * l1);
    v_inv[r] = ldexpf(1.f, -ev);
    v_sc[r] = ldexpf(1.f, ev);
  }
  const int e = tc::f16_scale_exponent(m);
  const float sc = ldexpf(1.f, e);
  if (threadIdx.x == 0) inv[r] = ldexpf(1.f, -e);
  const long d0 = r * ld_dst;
  for (int c = threadIdx.x; c < cols; c += SPLIT_ROW_THREADS) {
    const c128 v = row[c];
    const long d = d0 + (rev ? cols - 1 - c : c);
    __half h, l;
    tc::f16_split(float(v.x) * sc, h, l);
    rh[d] = h;
    rl[d] = l;
    tc::f16_split(float(v.y) * sc, h, l);
    ih[d] = h;
    il[d] = l;
  }
}

// One CTA per walker: S_w [M][N] (walker stride ldS) -> planes [w][n][m] (the K-major B operand
// of the Taylor kernel's first product) of S_w * 2^e_w, e_w from the walker's largest |re|, |im|;
// inv[w] = 2^-e_w.  Thread t handles orbitals m = t, t + 256, ...: the plane writes of a warp are
// consecutive in m.
__global__ void __launch_bounds__(SPLIT_ROW_THREADS) split_walkers_T_f16_kernel(
    const c128* __restrict__ S, long ldS, int M, int N, __half* __restrict__ rh,
    __half* __restrict__ rl, __half* __restrict__ ih, __half* __restrict__ il, long ld_dst,
    long bs_dst, float* __restrict__ inv) {
  __shared__ float wmax[SPLIT_ROW_THREADS / 32];
  const long w = blockIdx.x;
  const c128* Sw = S + w * ldS;
  float m = 0.f;
  for (long e = threadIdx.x; e < long(M) * N; e += SPLIT_ROW_THREADS) {
    const c128 v = Sw[e];
    m = fmaxf(m, fmaxf(fabsf(float(v.x)), fabsf(float(v.y))));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
  __syncthreads();
  m = 0.f;
#pragma unroll
  for (int k = 0; k < SPLIT_ROW_THREADS / 32; ++k) m = fmaxf(m, wmax[k]);
  const int ex = tc::f16_scale_exponent(m);
  const float sc = ldexpf(1.f, ex);
  if (threadIdx.x == 0) inv[w] = ldexpf(1.f, -ex);
  for (int i = threadIdx.x; i < M; i += SPLIT_ROW_THREADS) {
    const c128* r = Sw + long(i) * N;
    for (int n = 0; n < N; ++n) {
      const c128 v = r[n];
      const long d = w * bs_dst + long(n) * ld_dst + i;
      __half h, l;
      tc::f16_split(float(v.x) * sc, h, l);
      rh[d] = h;
      rl[d] = l;
      tc::f16_split(float(v.y) * sc, h, l);
      ih[d] = h;
      il[d] = l;
    }
  }
}

// largest |x| of a float64 array (non-negative floats order like their bit patterns)
__global__ void amax_kernel(const double* __restrict__ x, long n, unsigned* __restrict__ out) {
  float m = 0.f;
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
       i += long(gridDim.x) * blockDim.x)
    m = fmaxf(m, fabsf(float(x[i])));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void split_real_f16_kernel(const double* __restrict__ src, long n_rows, long cols,
                                      long ld_src, __half* __restrict__ h, __half* __restrict__ l,
                                      long ld_dst, float sc, int rev) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= n_rows * cols) return;
  const long r = e / cols, c = e % cols;
  const long d = r * ld_dst + (rev ? cols - 1 - c : c);
  __half hi, lo;
  tc::f16_split(float(src[r * ld_src + c]) * sc, hi, lo);
  h[d] = hi;
  l[d] = lo;
}

int split_rows_f16(cudaStream_t s, const c128* src, long ld_src, int rows, int cols, Planes& P,
                   float* inv, bool rev = false, float vbound = 0.f, float* v_inv = nullptr,
                   float* v_sc = nullptr) {
  split_rows_f16_kernel<<<rows, SPLIT_ROW_THREADS, 0, s>>>(src, ld_src, cols, P.h(0), P.h(1),
                                                           P.h(2), P.h(3), P.ld, inv,
                                                           rev ? 1 : 0, vbound, v_inv, v_sc);
  return launch_status("split_rows_f16_kernel");
}

// static real tensor [rows][cols] (device, synchronous set-up): one scale for the whole tensor;
// *inv receives 2^-e
int split_real_f16_host(const double* src_dev, long rows, long cols, long ld_src, Planes& P,
                        float* inv, bool rev = false, float* amax_out = nullptr) {
  unsigned* d = nullptr;
  AFQMC_CUDA_TRY(cudaMalloc(&d, sizeof(unsigned)));
  cudaMemset(d, 0, sizeof(unsigned));
  const long n = rows * ld_src;
  amax_kernel<<<1184, 256>>>(src_dev, n, d);
  unsigned bits = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&bits, d, sizeof(unsigned), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    set_error_detail("amax_kernel: %s", cudaGetErrorString(e));
    return AFQMC_ERR_CUDA;
  }
  float amax;
  memcpy(&amax, &bits, 4);
  if (amax_out) *amax_out = amax;
  const int ex = tc::f16_scale_exponent(amax);
  *inv = ldexpf(1.f, -ex);
  const long tot = rows * cols;
  split_real_f16_kernel<<<ceil_div(tot, 256), 256>>>(src_dev, rows, cols, ld_src, P.h(0),
                                                      P.h(1), P.ld, ldexpf(1.f, ex), rev ? 1 : 0);
  AFQMC_TRY(launch_status("split_real_f16_kernel"));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// launcher
// ---------------------------------------------------------------------------------------------
template <bool A_CPLX, bool B_CPLX, int BN, int STAGES, int EPI, bool F16 = false>
int launch_tc(cudaStream_t s, TcParams& p, int batch) {
  using K = TcCfg<A_CPLX, B_CPLX, BN, STAGES>;
  auto kern = tc_cgemm_kernel<A_CPLX, B_CPLX, BN, STAGES, EPI, F16>;
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
  // [1][M*M][Nc] (B of vHS, K = Nc).  The vHS planes of L and X hold the Cholesky index in
  // reverse order: the FP32 accumulation then adds the smallest vectors (decaying L_n) first and
  // the large ones last, which keeps the rounding of the long partial sums small.
  Planes Likn[2];
  Planes Lnak[2];   // [1][Nc][nel*M] (B of vbias, K = nel*M); same memory viewed [Nc*nel][M] for exchange
  // dynamic operands, sized on demand
  int capW = 0;
  int exchange_split = 3;  // TF32 products per real product in the exchange contraction
  // tile shapes / orders with bit-identical results, chosen by afqmc_prop_autotune_tiles
  int vbias_bn = 128;      // columns (Cholesky vectors) per vbias CTA tile: 128 or 64
  int exch_nblk = 64;      // vector pairs per L2 block of the exchange tile order
  bool likn_sym = false;   // every L_n symmetric (to 1e-10 of max |L|): vHS computes i <= k only
  bool vhs_sym = true;     // use the symmetric vHS when likn_sym
  // Operand format of vbias, vHS and the exchange: FP16 split with power-of-two scales when the
  // shapes allow it (f16_ok) unless the caller asks for the TF32 split (split_format 1).
  bool f16_ok = false;
  int split_format = 0;    // 0 auto, 1 TF32, 2 FP16
  Planes Likn16, Lnak16;   // FP16 split planes of the static tensors (spin block 0 / real Lnak)
  float likn_inv = 1.f, lnak_inv = 1.f;  // their inverse scales
  Planes G16, X16;         // FP16 split planes of G and X, rows scaled per walker
  float* g_inv = nullptr;  // [W] inverse row scales of G16
  float* x_inv = nullptr;  // [W] inverse row scales of X16
  int capW16 = 0;
  float likn_amax = 0.f;   // largest |L| (bound of V's scale)
  // FP16 propagation: V planes [W][M][M] with per-walker scales (from a * sum_n |X_n| max |L|),
  // P1 planes, S^T / T / R planes [W][N][M]
  Planes V16, P1_16, Sst16, T0_16, T1_16, R16;
  float* v_inv = nullptr;  // [W]
  float* v_sc = nullptr;   // [W]
  float* s_inv = nullptr;  // [W]
  float p1_inv = 1.f;
  const void* P1_16_src = nullptr;
  int capP16 = 0;
  bool v_is_f16 = false;   // format of the V planes the last vHS wrote
  // Taylor propagation (mixed_set_taylor_mode): 0 one GEMM launch per product; 2 / 3 the fused
  // kernel in the TF32 split with one / two walkers in flight per CTA; 4 / 5 the same in the FP16
  // split; one walker in flight (2, 4) gives the small split products their own accumulator,
  // 6 / 7 (TF32 / FP16) use that room for the running sum instead
  int taylor_mode = 2;
  int taylor_slots = 1;
  bool taylor_f16 = false;
  int taylor_one_slot = 0;  // 0 second accumulator, 1 running sum in tensor memory
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
    free_planes(Likn16);
    free_planes(Lnak16);
    free_planes(G16);
    free_planes(X16);
    if (g_inv) cudaFree(g_inv);
    if (x_inv) cudaFree(x_inv);
    free_planes(V16);
    free_planes(P1_16);
    free_planes(Sst16);
    free_planes(T0_16);
    free_planes(T1_16);
    free_planes(R16);
    if (v_inv) cudaFree(v_inv);
    if (v_sc) cudaFree(v_sc);
    if (s_inv) cudaFree(s_inv);
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

namespace {
// max |L[i][k][n] - L[k][i][n]| and max |L| (as ordered bit patterns of non-negative doubles)
__global__ void symmetry_check_kernel(const double* __restrict__ L, int M, int Nc,
                                      unsigned long long* out) {
  const long pair = blockIdx.x;  // (i, k), i < k ... walked over all pairs, skipping i >= k
  const int i = int(pair / M), k = int(pair % M);
  double dmax = 0.0, vmax = 0.0;
  const double* a = L + (long(i) * M + k) * Nc;
  const double* b = L + (long(k) * M + i) * Nc;
  for (int n = threadIdx.x; n < Nc; n += blockDim.x) {
    vmax = fmax(vmax, fabs(a[n]));
    if (i < k) dmax = fmax(dmax, fabs(a[n] - b[n]));
  }
  atomicMax(&out[0], __double_as_longlong(dmax));
  atomicMax(&out[1], __double_as_longlong(vmax));
}

int likn_is_symmetric(const double* L, int M, int Nc, bool* sym) {
  unsigned long long* d = nullptr;
  AFQMC_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
  cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  symmetry_check_kernel<<<unsigned(long(M) * M), 128>>>(L, M, Nc, d);
  cudaError_t e = cudaGetLastError();
  unsigned long long h[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    set_error_detail("symmetry_check_kernel: %s", cudaGetErrorString(e));
    return AFQMC_ERR_CUDA;
  }
  double dmax, vmax;
  memcpy(&dmax, &h[0], 8);
  memcpy(&vmax, &h[1], 8);
  *sym = dmax <= 1e-10 * vmax;
  return AFQMC_OK;
}
}  // namespace

int mixed_ham_create(MixedHam** out, const EnergyArgs& a, cudaStream_t s) {
  *out = nullptr;
  if (a.M % 4 || a.Nc % 4) {
    set_error_detail("mixed precision needs M and Nc multiples of 4 (M=%d, Nc=%d)", a.M, a.Nc);
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (!a.Likn) {
    set_error_detail("mixed precision needs the Cholesky factorisation (a THC Hamiltonian runs "
                     "in complex128)");
    return AFQMC_ERR_UNSUPPORTED;
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
    AFQMC_TRY(split_real_host(a.Likn + size_t(sp) * MM * a.Nc, MM, a.Nc, a.Nc, m->Likn[sp],
                              true));
  }
  // real orbitals make every Cholesky vector symmetric (L_n[i][k] = L_n[k][i]); then V_w is
  // complex symmetric and vHS computes only the i <= k half
  if (a.nspin_H2 == 1 && a.M <= SYM_IB * SYM_MAXIB)
    AFQMC_TRY(likn_is_symmetric(a.Likn, a.M, a.Nc, &m->likn_sym));
  // FP16 split: 16-byte rows of FP16 planes (M, Nc multiples of 8), one spin block of L, a real
  // trial and at most 50 electrons per spin (the fused exchange)
  m->f16_ok = (a.M % 8 == 0) && (a.Nc % 8 == 0) && a.nspin_H2 == 1 && !m->lnak_cplx &&
              a.nspin == 1 && a.nel[0] >= 1 && a.nel[0] <= 50;
  if (m->f16_ok) {
    AFQMC_TRY(alloc_planes(m->Likn16, 2, 1, MM, a.Nc, 2));
    AFQMC_TRY(split_real_f16_host(a.Likn, MM, a.Nc, a.Nc, m->Likn16, &m->likn_inv, true,
                                  &m->likn_amax));
    const long K = long(a.nel[0]) * a.M;
    AFQMC_TRY(alloc_planes(m->Lnak16, 2, 1, a.Nc, K, 2));
    AFQMC_TRY(split_real_f16_host(a.Lnak_real[0], a.Nc, K, K, m->Lnak16, &m->lnak_inv));
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

bool use_f16(const MixedHam* m) { return m->f16_ok && m->split_format != 1; }

int ensure_walker_buffers16(MixedHam* m, int W) {
  if (m->capW16 >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->G16);
  free_planes(m->X16);
  if (m->g_inv) cudaFree(m->g_inv);
  if (m->x_inv) cudaFree(m->x_inv);
  m->g_inv = m->x_inv = nullptr;
  AFQMC_TRY(alloc_planes(m->G16, 4, 1, W, long(m->nel_tot) * m->M, 2));
  AFQMC_TRY(alloc_planes(m->X16, 4, 1, W, m->Nc, 2));
  AFQMC_CUDA_TRY(cudaMalloc(&m->g_inv, sizeof(float) * W));
  AFQMC_CUDA_TRY(cudaMalloc(&m->x_inv, sizeof(float) * W));
  m->capW16 = W;
  return AFQMC_OK;
}

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
namespace {
// FP16 split: G planes with per-walker scales (row_inv), Lnak planes with one scale (alpha)
int vbias_mixed_f16(cudaStream_t s, MixedHam* m, const c128* G, long ldG, c128* v, int W,
                    double a) {
  AFQMC_TRY(ensure_walker_buffers16(m, W));
  const long K = long(m->nel[0]) * m->M;
  AFQMC_TRY(split_rows_f16(s, G, ldG, W, int(K), m->G16, m->g_inv));
  // K = N M in S ranges (multiples of 8 FP16 elements) summed in FP64, as in the TF32 split
  int S = 1;
  for (int c = 16; c >= 2; --c)
    if (K % c == 0 && (K / c) % 8 == 0 && K / c >= 512) {
      S = c;
      break;
    }
  TcParams p{};
  const long Kc = K / S;
  c128* out = v;
  if (S > 1) {
    const long need = long(S) * W * m->Nc;
    if (m->vpart_elems < need) {
      if (m->vpart) cudaFree(m->vpart);
      m->vpart = nullptr;
      m->vpart_elems = 0;
      AFQMC_CUDA_TRY(cudaMalloc(&m->vpart, sizeof(c128) * need));
      m->vpart_elems = need;
    }
    out = m->vpart;
  }
  for (int q = 0; q < 4; ++q)
    AFQMC_TRY(make_map_es(&p.a[q], m->G16, q, 0, Kc, W, m->G16.ld, S, Kc, 128));
  const int bn = m->vbias_bn == 64 ? 64 : 128;
  for (int q = 0; q < 2; ++q)
    AFQMC_TRY(make_map_es(&p.b[q], m->Lnak16, q, 0, Kc, m->Nc, m->Lnak16.ld, S, Kc, bn));
  p.m = W; p.n = m->Nc; p.k = int(Kc);
  p.a_batched = 1; p.b_batched = 1;
  p.order = 1;
  p.alpha = cmk(a * double(m->lnak_inv), 0);
  p.row_inv = m->g_inv;
  p.out_c = out; p.outc_ld = m->Nc; p.outc_bs = long(W) * m->Nc;
  p.err = m->err;
  if (bn == 64)
    AFQMC_TRY((launch_tc<true, false, 64, 2, EPI_C128, true>(s, p, S)));
  else
    AFQMC_TRY((launch_tc<true, false, 128, 2, EPI_C128, true>(s, p, S)));
  if (S > 1) {
    const long n = long(W) * m->Nc;
    sum_partials_kernel<<<ceil_div(n, 256), 256, 0, s>>>(m->vpart, S, n, v, 0);
    AFQMC_TRY(launch_status("sum_partials_kernel"));
  }
  return AFQMC_OK;
}
}  // namespace

int vbias_mixed(cudaStream_t s, MixedHam* m, const c128* G, long ldG, c128* v, int W, double a) {
  if (m->nspin > 1) {
    set_error_detail("vbias_mixed: COLLINEAR walkers are not supported in mixed precision");
    return AFQMC_ERR_UNSUPPORTED;
  }
  if (use_f16(m)) return vbias_mixed_f16(s, m, G, ldG, v, W, a);
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

// FP16 V planes -> complex128 [W][M*M]: (hi + lo) * v_inv[w]
__global__ void planes16_to_c128_kernel(const __half* __restrict__ rh,
                                        const __half* __restrict__ rl,
                                        const __half* __restrict__ ih,
                                        const __half* __restrict__ il, long n, long per_walker,
                                        const float* __restrict__ v_inv, c128* __restrict__ out) {
  long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= n) return;
  const double f = v_inv[e / per_walker];
  out[e] = cmk((double(__half2float(rh[e])) + double(__half2float(rl[e]))) * f,
               (double(__half2float(ih[e])) + double(__half2float(il[e]))) * f);
}

int ensure_v_buffers(MixedHam* m, int W) {
  if (m->V.batch >= W) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->V);
  return alloc_planes(m->V, 4, W, m->M, m->M);
}

int ensure_v_buffers16(MixedHam* m, int W) {
  if (m->V16.batch >= W && m->v_sc) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->V16);
  if (m->v_inv) cudaFree(m->v_inv);
  if (m->v_sc) cudaFree(m->v_sc);
  m->v_inv = m->v_sc = nullptr;
  AFQMC_TRY(alloc_planes(m->V16, 4, W, m->M, m->M, 2));
  AFQMC_CUDA_TRY(cudaMalloc(&m->v_inv, sizeof(float) * W));
  AFQMC_CUDA_TRY(cudaMalloc(&m->v_sc, sizeof(float) * W));
  return AFQMC_OK;
}

int ensure_prop_buffers16(MixedHam* m, int W, int N) {
  if (m->capP16 >= W && m->T0_16.rows == N) return AFQMC_OK;
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  free_planes(m->Sst16);
  free_planes(m->T0_16);
  free_planes(m->T1_16);
  free_planes(m->R16);
  if (m->s_inv) cudaFree(m->s_inv);
  m->s_inv = nullptr;
  AFQMC_TRY(alloc_planes(m->Sst16, 4, W, N, m->M, 2));
  AFQMC_TRY(alloc_planes(m->T0_16, 4, W, N, m->M, 2));
  AFQMC_TRY(alloc_planes(m->T1_16, 4, W, N, m->M, 2));
  AFQMC_TRY(alloc_planes(m->R16, 4, W, N, m->M, 2));
  AFQMC_CUDA_TRY(cudaMalloc(&m->s_inv, sizeof(float) * W));
  m->capP16 = W;
  return AFQMC_OK;
}

// FP16 V planes and the FP16 Taylor kernel go together: the FP16 split, the fused Taylor
// kernel, and shapes it takes (M <= 256, N <= 64)
bool v16_ok(const MixedHam* m) {
  return use_f16(m) && m->taylor_f16 && m->taylor_mode != 0 && m->M <= 256 && m->nel[0] <= 64;
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
  const bool f16 = use_f16(m);
  AFQMC_TRY(ensure_v_buffers(m, W));
  TcParams p{};
  const Planes& Lp = f16 ? m->Likn16 : m->Likn[0];
  const bool v16 = v16_ok(m);
  if (f16) {
    AFQMC_TRY(ensure_walker_buffers16(m, W));
    if (v16) AFQMC_TRY(ensure_v_buffers16(m, W));
    AFQMC_TRY(split_rows_f16(s, X, m->Nc, W, m->Nc, m->X16, m->x_inv, true,
                             float(a) * m->likn_amax, v16 ? m->v_inv : nullptr,
                             v16 ? m->v_sc : nullptr));
    AFQMC_TRY(maps_for(m->X16, p.a, 128));
    p.row_inv = m->x_inv;
    a *= double(m->likn_inv);
  } else {
    AFQMC_TRY(ensure_walker_buffers(m, W));
    AFQMC_TRY(split_complex(s, X, m->Nc, 0, 1, W, m->Nc, m->X, false, true));
    AFQMC_TRY(maps_for(m->X, p.a, 128));
  }
  if (m->likn_sym && m->vhs_sym) {
    // L planes viewed [i][k][n]: box {128 bytes of n, 16 k, 8 i} = the 128 (i, k) pairs of a tile
    const int M = m->M;
    for (int q = 0; q < 2; ++q)
      AFQMC_TRY(make_plane_map_3d_es(&p.b[q], Lp.p[q], Lp.esize, m->Nc, M, Lp.ld, M,
                                     long(M) * Lp.ld, SYM_KB, SYM_IB));
    p.sym_nib = ceil_div(M, SYM_IB);
    p.sym_nkb = ceil_div(M, SYM_KB);
    p.sym_pre[0] = 0;
    for (int ab = 0; ab < p.sym_nib; ++ab) {
      int cnt = 0;
      for (int cb = 0; cb < p.sym_nkb; ++cb)
        if (cb * SYM_KB + SYM_KB - 1 >= ab * SYM_IB) ++cnt;
      p.sym_pre[ab + 1] = p.sym_pre[ab] + cnt;
    }
    p.m = W; p.n = p.sym_pre[p.sym_nib] * 128; p.k = m->Nc;
    p.alpha = cmk(a, 0);
    const Planes& Vo = v16 ? m->V16 : m->V;
    for (int q = 0; q < 4; ++q) p.out[q] = Vo.p[q];
    p.out_ld = Vo.ld;
    p.out_bs = Vo.bstride();
    p.out_f16 = v16 ? 1 : 0;
    p.out_sc = v16 ? m->v_sc : nullptr;
    m->v_is_f16 = v16;
    p.vhs_M = M;
    p.err = m->err;
    if (f16) return launch_tc<true, false, 128, 2, EPI_VHS_SYM, true>(s, p, 1);
    return launch_tc<true, false, 128, 2, EPI_VHS_SYM>(s, p, 1);
  }
  AFQMC_TRY(maps_for(Lp, p.b, 128));
  const long MM = long(m->M) * m->M;
  p.m = W; p.n = int(MM); p.k = m->Nc;
  p.alpha = cmk(a, 0);
  const Planes& Vo = v16 ? m->V16 : m->V;
  for (int q = 0; q < 4; ++q) p.out[q] = Vo.p[q];
  p.out_ld = Vo.ld;
  p.out_bs = Vo.bstride();
  p.out_f16 = v16 ? 1 : 0;
  p.out_sc = v16 ? m->v_sc : nullptr;
  m->v_is_f16 = v16;
  p.vhs_M = m->M;
  p.err = m->err;
  if (f16) return launch_tc<true, false, 128, 2, EPI_VHS, true>(s, p, 1);
  return launch_tc<true, false, 128, 2, EPI_VHS>(s, p, 1);
}

int vhs_mixed(cudaStream_t s, MixedHam* m, const c128* X, c128* V, int W, double a) {
  if (m->nspin > 1 && m->Likn[1].p[0]) {
    set_error_detail("vhs_mixed: spin-dependent Cholesky vectors are not supported");
    return AFQMC_ERR_UNSUPPORTED;
  }
  AFQMC_TRY(vhs_planes(s, m, X, W, a));
  if (V && m->v_is_f16) {
    const long n = long(W) * m->M * m->M;
    if (m->V16.ld != m->M) {
      set_error_detail("vhs_mixed: padded V planes cannot be copied out");
      return AFQMC_ERR_UNSUPPORTED;
    }
    planes16_to_c128_kernel<<<ceil_div(n, 256), 256, 0, s>>>(
        m->V16.h(0), m->V16.h(1), m->V16.h(2), m->V16.h(3), n, long(m->M) * m->M, m->v_inv, V);
    return launch_status("planes16_to_c128_kernel");
  }
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

int taylor_fused_tc(cudaStream_t s, int esize, const void* const P1p[2], const void* const Vp[4],
                    long ldV, const void* const Sp[4], void* const Tp0[4], void* const Tp1[4],
                    void* const Rp[4], float* const sum[2], long pl_ld, c128* S, long ldS, int W,
                    int M, int N, int order, int nslots, int one_slot_use, const float* v_inv,
                    const float* s_inv, float p1_inv, unsigned* err);

// Taylor propagation S <- P1 sum_n (iV)^n/n! P1 S (propagate.hpp:238-298) on the split planes.
// V must have been produced by vhs_mixed (planes kept in MixedHam) for the same walkers.
int propagate_mixed(cudaStream_t s, MixedHam* m, const void* P1, bool p1_real, c128* S, long ldS,
                    int W, int M, int N, int order) {
  if (!p1_real) {
    set_error_detail("propagate_mixed: a complex one-body propagator is not supported");
    return AFQMC_ERR_UNSUPPORTED;
  }
  if ((m->v_is_f16 ? m->V16.batch : m->V.batch) < W) {
    set_error_detail("propagate_mixed: no vHS planes for %d walkers (call vhs_mixed first)", W);
    return AFQMC_ERR_ARG;
  }
  AFQMC_TRY(ensure_prop_buffers(m, W, N));
  if (m->v_is_f16) {
    if (M > 256 || N > 64) {
      set_error_detail("propagate_mixed: FP16 V planes need M <= 256 and N <= 64");
      return AFQMC_ERR_UNSUPPORTED;
    }
    AFQMC_TRY(ensure_prop_buffers16(m, W, N));
    if (m->P1_16_src != P1) {
      free_planes(m->P1_16);
      AFQMC_TRY(alloc_planes(m->P1_16, 2, 1, M, M, 2));
      AFQMC_TRY(split_real_f16_host(static_cast<const double*>(P1), M, M, M, m->P1_16,
                                    &m->p1_inv));
      m->P1_16_src = P1;
    }
    split_walkers_T_f16_kernel<<<W, SPLIT_ROW_THREADS, 0, s>>>(
        S, ldS, M, N, m->Sst16.h(0), m->Sst16.h(1), m->Sst16.h(2), m->Sst16.h(3), m->Sst16.ld,
        m->Sst16.bstride(), m->s_inv);
    AFQMC_TRY(launch_status("split_walkers_T_f16_kernel"));
    const void* p1p[2] = {m->P1_16.p[0], m->P1_16.p[1]};
    const void* vp[4] = {m->V16.p[0], m->V16.p[1], m->V16.p[2], m->V16.p[3]};
    const void* sp[4] = {m->Sst16.p[0], m->Sst16.p[1], m->Sst16.p[2], m->Sst16.p[3]};
    void* t0[4] = {m->T0_16.p[0], m->T0_16.p[1], m->T0_16.p[2], m->T0_16.p[3]};
    void* t1[4] = {m->T1_16.p[0], m->T1_16.p[1], m->T1_16.p[2], m->T1_16.p[3]};
    void* rp[4] = {m->R16.p[0], m->R16.p[1], m->R16.p[2], m->R16.p[3]};
    if (m->P1_16.ld != m->T0_16.ld || m->T0.ld != m->T0_16.ld) {
      set_error_detail("propagate_mixed: FP16 plane strides differ (M = %d)", M);
      return AFQMC_ERR_UNSUPPORTED;
    }
    return taylor_fused_tc(s, 2, p1p, vp, m->V16.ld, sp, t0, t1, rp, m->acc, m->T0_16.ld, S, ldS,
                           W, M, N, order, m->taylor_slots, m->taylor_one_slot, m->v_inv,
                           m->s_inv, m->p1_inv, m->err);
  }
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
    const void* p1p[2] = {m->P1.p[0], m->P1.p[1]};
    const void* vp[4] = {m->V.p[0], m->V.p[1], m->V.p[2], m->V.p[3]};
    const void* sp[4] = {m->Sst.p[0], m->Sst.p[1], m->Sst.p[2], m->Sst.p[3]};
    void* t0[4] = {m->T0.p[0], m->T0.p[1], m->T0.p[2], m->T0.p[3]};
    void* t1[4] = {m->T1.p[0], m->T1.p[1], m->T1.p[2], m->T1.p[3]};
    void* rp[4] = {m->Tacc_split.p[0], m->Tacc_split.p[1], m->Tacc_split.p[2],
                   m->Tacc_split.p[3]};
    return taylor_fused_tc(s, 4, p1p, vp, m->V.ld, sp, t0, t1, rp, m->acc, m->T0.ld, S, ldS, W,
                           M, N, order, m->taylor_slots, m->taylor_one_slot, nullptr, nullptr, 1.f,
                           m->err);
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
  if (mode < 0 || mode > 7) {
    set_error_detail("Taylor mode must be 0..7");
    return AFQMC_ERR_ARG;
  }
  if (mode == 1) mode = 2;  // the default: one walker in flight, two accumulators, TF32
  m->taylor_mode = mode;
  m->taylor_slots = (mode == 3 || mode == 5) ? 2 : (mode == 0 ? 0 : 1);
  m->taylor_f16 = (mode == 4 || mode == 5 || mode == 7);
  m->taylor_one_slot = mode >= 6 ? 1 : 0;
  return AFQMC_OK;
}

bool mixed_taylor_f16_ok(MixedHam* m) { return use_f16(m) && m->M <= 256 && m->nel[0] <= 64; }

int mixed_prepare_G(cudaStream_t s, MixedHam* m, const c128* G, long ldG, int W) {
  if (use_f16(m)) {
    AFQMC_TRY(ensure_walker_buffers16(m, W));
    return split_rows_f16(s, G, ldG, W, int(long(m->nel[0]) * m->M), m->G16, m->g_inv);
  }
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

int exchange_fused_tc(cudaStream_t s, const void* const Gp[4], int esize, long ldG, long off,
                      const void* const Lp[2], int W, int N, int Nc, int M, int nsplit,
                      const float* g_inv, float l_inv, c128* exx, c128* kl, unsigned* err,
                      int nblk);

bool exchange_fused_ok(MixedHam* m, int sp) {
  return !m->lnak_cplx && m->nel[sp] >= 1 && m->nel[sp] <= 50;
}

int exchange_fused(cudaStream_t s, MixedHam* m, int sp, int W, c128* exx, c128* kl) {
  if (use_f16(m)) {
    const void* Gp[4] = {m->G16.p[0], m->G16.p[1], m->G16.p[2], m->G16.p[3]};
    const void* Lp[2] = {m->Lnak16.p[0], m->Lnak16.p[1]};
    return exchange_fused_tc(s, Gp, 2, m->G16.ld, 0, Lp, W, m->nel[0], m->Nc, m->M,
                             m->exchange_split, m->g_inv, m->lnak_inv, exx, kl, m->err,
                             m->exch_nblk);
  }
  const void* Gp[4] = {m->G.p[0], m->G.p[1], m->G.p[2], m->G.p[3]};
  const void* Lp[2] = {m->Lnak[sp].p[0], m->Lnak[sp].p[1]};
  return exchange_fused_tc(s, Gp, 4, m->G.ld, long(m->el_off[sp]) * m->M, Lp, W, m->nel[sp],
                           m->Nc, m->M, m->exchange_split, nullptr, 1.f, exx, kl, m->err,
                           m->exch_nblk);
}

int mixed_set_split_format(MixedHam* m, int format, int* active_f16) {
  if (format < 0 || format > 2) {
    set_error_detail("split format must be 0 (auto), 1 (TF32) or 2 (FP16)");
    return AFQMC_ERR_ARG;
  }
  if (format == 2 && !m->f16_ok) {
    set_error_detail("the FP16 split needs M and N_chol multiples of 8, one spin block of "
                     "Cholesky vectors, a real trial, CLOSED walkers and 1..50 electrons");
    return AFQMC_ERR_UNSUPPORTED;
  }
  m->split_format = format;
  if (active_f16) *active_f16 = use_f16(m) ? 1 : 0;
  return AFQMC_OK;
}

int mixed_set_vhs_symmetry(MixedHam* m, int enable, int* active) {
  m->vhs_sym = enable != 0;
  if (active) *active = (m->likn_sym && m->vhs_sym) ? 1 : 0;
  return AFQMC_OK;
}

int mixed_set_exchange_split(MixedHam* m, int nsplit) {
  if (nsplit != 1 && nsplit != 3) {
    set_error_detail("exchange split must be 1 or 3");
    return AFQMC_ERR_ARG;
  }
  m->exchange_split = nsplit;
  return AFQMC_OK;
}

namespace {
// One bounded wait on an mbarrier that expects one arrival and never gets it: the wait the
// tensor-core kernels use, with a short budget, so that its timeout path can be exercised.
__global__ void wait_selftest_kernel(unsigned* err, long long budget) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&bar, 1);
    tc::fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) tc::mbar_wait(&bar, 0, err, nullptr, budget);
}
}  // namespace

int mixed_wait_selftest(cudaStream_t s, MixedHam* m, long long budget) {
  if (budget <= 0 || budget > tc::kWaitCycles) budget = tc::kWaitCycles;
  wait_selftest_kernel<<<1, 32, 0, s>>>(m->err, budget);
  AFQMC_TRY(launch_status("wait_selftest_kernel"));
  AFQMC_CUDA_TRY(cudaStreamSynchronize(s));
  unsigned flag = 0;
  AFQMC_CUDA_TRY(cudaMemcpy(&flag, m->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (flag & tc::kTimeoutFlag) {
    set_error_detail("wait_selftest_kernel: the bounded wait gave up after %lld cycles", budget);
    return AFQMC_ERR_TIMEOUT;
  }
  return AFQMC_OK;
}

int mixed_clear_error(MixedHam* m) {
  AFQMC_CUDA_TRY(cudaMemset(m->err, 0, sizeof(unsigned)));
  return AFQMC_OK;
}

int mixed_error_flag(MixedHam* m, unsigned* flag) {
  AFQMC_CUDA_TRY(cudaMemcpy(flag, m->err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  return AFQMC_OK;
}

int mixed_set_tiles(MixedHam* m, int vbias_bn, int exch_nblk) {
  if (vbias_bn != 64 && vbias_bn != 128) {
    set_error_detail("vbias tile width must be 64 or 128 (got %d)", vbias_bn);
    return AFQMC_ERR_ARG;
  }
  if (exch_nblk < 1 || exch_nblk > 1024) {
    set_error_detail("exchange block must be 1..1024 vector pairs (got %d)", exch_nblk);
    return AFQMC_ERR_ARG;
  }
  m->vbias_bn = vbias_bn;
  m->exch_nblk = exch_nblk;
  return AFQMC_OK;
}

int mixed_get_tiles(MixedHam* m, int* vbias_bn, int* exch_nblk) {
  *vbias_bn = m->vbias_bn;
  *exch_nblk = m->exch_nblk;
  return AFQMC_OK;
}

// ---------------------------------------------------------------------------------------------
// C = A B^T for a complex A and a real B held as complex128 with zero imaginary parts, in the
// FP16 split on the tensor cores (the PHMSD energy's half rotation G Lnak^T in mixed precision)
// ---------------------------------------------------------------------------------------------
namespace {
// largest |re| and |im| of a complex128 array (non-negative floats order like their bits)
__global__ void amax_c128_kernel(const c128* __restrict__ x, long n, unsigned* __restrict__ out) {
  float mr = 0.f, mi = 0.f;
  for (long i = blockIdx.x * long(blockDim.x) + threadIdx.x; i < n;
       i += long(gridDim.x) * blockDim.x) {
    mr = fmaxf(mr, fabsf(float(x[i].x)));
    mi = fmaxf(mi, fabsf(float(x[i].y)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
    mi = fmaxf(mi, __shfl_xor_sync(0xffffffffu, mi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, __float_as_uint(mr));
    atomicMax(out + 1, __float_as_uint(mi));
  }
}

__global__ void split_real_part_f16_kernel(const c128* __restrict__ src, long rows, long cols,
                                           long ld_src, __half* __restrict__ h,
                                           __half* __restrict__ l, long ld_dst, float sc) {
  const long e = blockIdx.x * long(blockDim.x) + threadIdx.x;
  if (e >= rows * cols) return;
  const long r = e / cols, c = e % cols;
  __half hi, lo;
  tc::f16_split(float(src[r * ld_src + c].x) * sc, hi, lo);
  h[r * ld_dst + c] = hi;
  l[r * ld_dst + c] = lo;
}
}  // namespace

struct TcGemmRB {
  Planes B;          // FP16 split of B (2 planes), one power-of-two scale
  float b_inv = 1.f;
  Planes A;          // FP16 split of A (4 planes), per-row scales a_inv
  float* a_inv = nullptr;
  long a_cap = 0;
  unsigned* err = nullptr;
  ~TcGemmRB() {
    free_planes(B);
    free_planes(A);
    if (a_inv) cudaFree(a_inv);
    if (err) cudaFree(err);
  }
};

int tcgemm_rb_create(TcGemmRB** out, const c128* B, long rows_b, long K, long ldb) {
  *out = nullptr;
  if (K % 8 != 0 || rows_b < 1) {
    set_error_detail("tcgemm_rb_create: K = %ld (a multiple of 8), rows = %ld", K, rows_b);
    return AFQMC_ERR_UNSUPPORTED;
  }
  unsigned* d = nullptr;
  AFQMC_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(unsigned)));
  cudaMemset(d, 0, 2 * sizeof(unsigned));
  long n = rows_b * ldb;
  amax_c128_kernel<<<1184, 256>>>(B, n, d);
  unsigned bits[2] = {0, 0};
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(bits, d, sizeof(bits), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    set_error_detail("amax_c128_kernel: %s", cudaGetErrorString(e));
    return AFQMC_ERR_CUDA;
  }
  float amax, imax;
  memcpy(&amax, &bits[0], 4);
  memcpy(&imax, &bits[1], 4);
  if (imax != 0.f) {
    set_error_detail("tcgemm_rb_create: B is not real (max |imag| %g)", double(imax));
    return AFQMC_ERR_UNSUPPORTED;
  }
  std::unique_ptr<TcGemmRB> g(new (std::nothrow) TcGemmRB());
  if (!g) return AFQMC_ERR_ALLOC;
  AFQMC_TRY(alloc_planes(g->B, 2, 1, rows_b, K, 2));
  const int ex = tc::f16_scale_exponent(amax);
  g->b_inv = ldexpf(1.f, -ex);
  const long tot = rows_b * K;
  split_real_part_f16_kernel<<<ceil_div(tot, 256), 256>>>(B, rows_b, K, ldb, g->B.h(0), g->B.h(1),
                                                         g->B.ld, ldexpf(1.f, ex));
  AFQMC_TRY(launch_status("split_real_part_f16_kernel"));
  AFQMC_CUDA_TRY(cudaMalloc(&g->err, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaMemset(g->err, 0, sizeof(unsigned)));
  AFQMC_CUDA_TRY(cudaDeviceSynchronize());
  *out = g.release();
  return AFQMC_OK;
}

void tcgemm_rb_destroy(TcGemmRB* g) { delete g; }

int tcgemm_rb_run(cudaStream_t s, TcGemmRB* g, const c128* A, long lda, int rows_a, c128* C,
                  long ldc, bool c64_out) {
  if (rows_a <= 0) return AFQMC_OK;
  const long K = g->B.k;
  if (g->a_cap < rows_a) {
    AFQMC_CUDA_TRY(cudaDeviceSynchronize());
    free_planes(g->A);
    if (g->a_inv) cudaFree(g->a_inv);
    g->a_inv = nullptr;
    g->a_cap = 0;
    AFQMC_TRY(alloc_planes(g->A, 4, 1, rows_a, K, 2));
    AFQMC_CUDA_TRY(cudaMalloc(&g->a_inv, sizeof(float) * rows_a));
    g->a_cap = rows_a;
  }
  AFQMC_TRY(split_rows_f16(s, A, lda, rows_a, int(K), g->A, g->a_inv));
  if (c64_out) {
    // C^T = B A^T with B (real) as the MMA's A operand: the accumulator rows are C's columns,
    // so the epilogue's lanes write consecutive complex64 elements of C
    TcParams p{};
    for (int q = 0; q < 2; ++q)
      AFQMC_TRY(make_map_es(&p.a[q], g->B, q, 0, K, g->B.rows, g->B.ld, 1, g->B.bstride(), 128));
    for (int q = 0; q < 4; ++q)
      AFQMC_TRY(make_map_es(&p.b[q], g->A, q, 0, K, rows_a, g->A.ld, 1, long(rows_a) * g->A.ld,
                            128));
    p.m = int(g->B.rows);
    p.n = rows_a;
    p.k = int(K);
    p.order = 1;  // a tile of B's rows stays in L2 while the tiles of A's rows stream past it
    p.alpha = cmk(double(g->b_inv), 0);
    p.col_inv = g->a_inv;
    p.out_c = C;
    p.outc_ld = ldc;
    p.outc_bs = 0;
    p.err = g->err;
    return launch_tc<false, true, 128, 2, EPI_C64T, true>(s, p, 1);
  }
  TcParams p{};
  for (int q = 0; q < 4; ++q)
    AFQMC_TRY(make_map_es(&p.a[q], g->A, q, 0, K, rows_a, g->A.ld, 1, long(rows_a) * g->A.ld,
                          128));
  for (int q = 0; q < 2; ++q)
    AFQMC_TRY(make_map_es(&p.b[q], g->B, q, 0, K, g->B.rows, g->B.ld, 1, g->B.bstride(), 128));
  p.m = rows_a;
  p.n = int(g->B.rows);
  p.k = int(K);
  p.order = 1;  // an A tile stays in L2 while the B tiles stream past it
  p.alpha = cmk(double(g->b_inv), 0);
  p.row_inv = g->a_inv;
  p.out_c = C;
  p.outc_ld = ldc;
  p.outc_bs = 0;
  p.err = g->err;
  return launch_tc<true, false, 128, 2, EPI_C128, true>(s, p, 1);
}

}  // namespace afqmc
