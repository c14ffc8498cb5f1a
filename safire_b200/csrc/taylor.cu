// Fused Taylor propagation of the walkers on the tensor cores (mixed precision).
//
// Reference: det_ops::detail::propagate_impl / apply_expM (src/AFQMC/SlaterDeterminantOperations/
// propagate.hpp:41-70, 238-298):  S <- P1 * sum_{n=0..order} (i V)^n / n! * P1 * S, with the Taylor
// terms built iteratively T_n = (i/n) V T_{n-1}.
//
// A persistent CTA runs each of its walkers through order+2 products ("phases"):
//   phase 0          T_0 = P1 S                    (A = P1, real;   B = S^T planes)
//   phase 1..order   T_n = (i/n) V_w T_{n-1}       (A = V_w planes; B = T_{n-1}^T planes)
//   phase order+1    S   = P1 R                    (A = P1;         B = R^T planes)
// Each phase is up to two 128-row tiles (M <= 256 orbitals) x 64 columns (N <= 64 electrons),
// FP32 accumulators in TMEM, 3xTF32 split products.  A phase needs the whole previous term, so
// the CTA keeps two walkers in flight ("slots", 256 TMEM columns each) and alternates their
// phases: the tensor core runs one walker's products while the epilogue warps finish the other's
// term.  Each T_n goes through global memory (one walker's worth, L2-resident) as the K-major B
// operand of the next phase, handed from the epilogue warps to the TMA warp by an mbarrier after
// an async-proxy fence; the running sum R = sum_n T_n is kept in FP32 in global memory (the
// epilogue adds each term, in the order of the per-term GEMM path) and split once for the last
// product.  K steps past M (zero fill of the last 32-wide chunk) are not issued.
//
// FP16 form (F16 = true): the operands are FP16 split planes of power-of-two-scaled values (P1
// one scale; V and S one scale per walker), twice the tensor rate and half the bytes of TF32.
// The epilogue turns each accumulator into the term's true values with the operands' inverse
// scales, and stores each term T_n (and R) in planes of its own scale: a first pass over the
// walker's accumulators (both 128-row tiles) finds the largest |value|, the epilogue warps
// agree on it through shared memory, and a second pass scales, splits and stores.  The running
// sum stays FP32 in true values.
#include "mixed.cuh"
#include "tc.cuh"

namespace afqmc {
namespace {

// warp 0 TMA, warp 1 MMA, then EPW epilogue warps: EPW / 4 per TMEM lane quarter, which split
// the accumulator columns between them in chunks of 16 * 4 / EPW
constexpr int TY_EPW = 8;
__host__ __device__ constexpr int ty_threads(int epw) { return 64 + 32 * epw; }
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
  void* tp[2][4];        // T ping-pong planes (epilogue writes) [W][N][M]
  void* rp[4];           // R planes [W][N][M]
  float* sum[2];         // running sum re, im (FP32) [W][N][M]
  c128* S;               // walker Slater matrices (output), [W] x ldS, [M][N] each
  long ldS;
  long pl_ld, pl_bs;     // ld / batch stride of the [W][N][M] planes
  int W, M, N, order;
  int nslots;            // walkers in flight per CTA (1 or 2)
  int sum_tmem;          // 1: the running sum lives in tensor memory (columns 256..511, one
                         // walker in flight), not in `sum`
  int dual;              // 1: the small split products (hi*lo, lo*hi) go to a second accumulator
                         // (columns 256..511, one walker in flight), added to the main one
                         // (hi*hi) in the epilogue: a third of the updates of the main
                         // accumulator, whose FP32 accumulation truncates toward zero
  // FP16 form: inverse power-of-two scales of the operands (V and S per walker, P1 one)
  const float* v_inv;
  const float* s_inv;
  float p1_inv;
  unsigned* err;
};

__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void split_store(float v, float* hi, float* lo, long idx) {
  float h, l;
  tc::tf32_split(v, h, l);
  hi[idx] = h;
  lo[idx] = l;
}

__device__ __forceinline__ void split_store16(float v, void* hi, void* lo, long idx) {
  __half h, l;
  tc::f16_split(v, h, l);
  static_cast<__half*>(hi)[idx] = h;
  static_cast<__half*>(lo)[idx] = l;
}

__device__ __forceinline__ void named_bar_sync(int id, int n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// The order in which a CTA runs (slot, walker, phase): the two slots alternate; a slot whose
// walker finished its last phase takes the CTA's next walker.  Every warp role walks the same
// sequence.
struct Schedule {
  int w0, w1, ph0, ph1, wi0, wi1;  // per slot: current walker, its phase, walkers finished
  int next, cur, W, nph, step;
  __device__ Schedule(int W_, int nph_, int first, int stride, int nslots)
      : w0(first), w1(nslots > 1 ? first + stride : W_), ph0(0), ph1(0), wi0(0), wi1(0),
        next(first + nslots * stride), cur(0), W(W_), nph(nph_), step(stride) {}
  __device__ int w(int s) const { return s ? w1 : w0; }
  __device__ int ph(int s) const { return s ? ph1 : ph0; }
  __device__ int wi(int s) const { return s ? wi1 : wi0; }
  __device__ bool get(int& s) {
    for (int k = 0; k < 2; ++k) {
      const int c = cur;
      cur ^= 1;
      if (w(c) < W) {
        s = c;
        return true;
      }
    }
    return false;
  }
  __device__ void advance(int s) {
    int& ph_ = s ? ph1 : ph0;
    if (++ph_ == nph) {
      ph_ = 0;
      ++(s ? wi1 : wi0);
      (s ? w1 : w0) = next;
      next += step;
    }
  }
};

// Epilogue of the FP16 form (the EPW warps from warp 2).  Per (slot, walker, phase): pass 1 reads
// the walker's accumulators (both 128-row tiles) and finds the largest |value| of what the phase
// stores (the new term, or R = sum + T_order for the last term); the warps exchange their maxima and
// failure flags through shared memory between two named barriers, so that they agree on the
// scale and on whether to go on (a bounded wait that gave up ends every warp's loop at the same
// point); pass 2 reads the accumulators again, frees them, and stores.  Values are true values
// (the accumulator times the operands' inverse scales); the planes hold them times 2^e.
template <int EPW>
__device__ __forceinline__ void taylor_epilogue_f16(const TyParams& p, uint32_t taddr,
                                                    uint64_t* acc_full, uint64_t* acc_empty,
                                                    uint64_t* phase_done,
                                                    volatile int* abort_flag, float* red,
                                                    int warp, int lane) {
  constexpr int NH = EPW / 4, CW = 16 / NH, NT = 32 * EPW;
  const int q = warp & 3;
  const int h = (warp - 2) >> 2;  // which of the quarter's warps: columns c0 = CW * h + CW * NH * k
  const int N = p.N, M = p.M, nph = p.order + 2, MT = (M + 127) / 128;
  const long pl_ld = p.pl_ld;
  float* __restrict__ const sum_r = p.sum[0];
  float* __restrict__ const sum_i = p.sum[1];
  int* const redf = reinterpret_cast<int*>(red + EPW);
  Schedule sc(p.W, nph, blockIdx.x, gridDim.x, p.nslots);
  long use0 = 0, use1 = 0;
  float pinv0 = 1.f, pinv1 = 1.f;  // inverse scale of the planes each slot stored last
  int sl;
  while (sc.get(sl)) {
    const int w = sc.w(sl), ph = sc.ph(sl);
    const bool taylor = (ph > 0 && ph < nph - 1);
    const bool last_phase = (ph == nph - 1);
    const bool last_term = (ph == nph - 2);
    const float ai = taylor ? 1.0f / float(ph) : 0.0f;
    const float pin = sl ? pinv1 : pinv0;
    // accumulator -> true values: inverse scales of the A (P1 or V_w) and B (S_w, T or R) planes
    const float f_in = ph == 0 ? p.p1_inv * p.s_inv[w]
                               : (last_phase ? p.p1_inv * pin : p.v_inv[w] * pin);
    const unsigned par = unsigned(sl ? use1 : use0) & 1u;
    const long wb = long(w) * p.pl_bs;
    bool ok = true;

    // the true values of accumulator chunk (mt, c0), with the running sum when `with_sum`
    auto values = [&](uint32_t tacc, int c0, float* xr, float* xi) {
      float vr[CW], vi[CW];
      tc::tmem_ld<CW>(tacc + c0, vr);
      tc::tmem_ld<CW>(tacc + TBN + c0, vi);
      if (p.dual) {  // + the small products' accumulator (FP32 add, rounded to nearest)
        float wr[CW], wi[CW];
        tc::tmem_ld<CW>(tacc + 256 + c0, wr);
        tc::tmem_ld<CW>(tacc + 256 + TBN + c0, wi);
        tc::tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < CW; ++j) {
          vr[j] += wr[j];
          vi[j] += wi[j];
        }
      }
      tc::tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        if (taylor) {
          xr[j] = -ai * (vi[j] * f_in);
          xi[j] = ai * (vr[j] * f_in);
        } else {
          xr[j] = vr[j] * f_in;
          xi[j] = vi[j] * f_in;
        }
      }
    };

    float mx = 0.f;
    if (!last_phase) {
      for (int mt = 0; mt < MT; ++mt) {
        if (ok && !tc::mbar_wait_warp(&acc_full[sl * 2 + mt], par, p.err, abort_flag))
          ok = false;
        if (!ok) continue;
        tc::tc_fence_after();
        const int row = mt * 128 + q * 32 + lane;
        const uint32_t tacc =
            taddr + (uint32_t(q * 32) << 16) + uint32_t(sl * 256 + mt * 2 * TBN);
        const uint32_t tsum = taddr + (uint32_t(q * 32) << 16) + uint32_t(256 + mt * 2 * TBN);
        const long off = wb + row;
#pragma unroll 1
        for (int c0 = CW * h; c0 < TBN; c0 += CW * NH) {
          if (c0 >= N) continue;
          const bool add_sum = last_term && taylor;
          float sr[CW], si[CW];
          if (add_sum && !p.sum_tmem && row < M) {
            // the running sum from global memory, in flight while the accumulator is read
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (c0 + j < N) {
                const long idx = off + long(c0 + j) * pl_ld;
                sr[j] = sum_r[idx];
                si[j] = sum_i[idx];
              }
          }
          float xr[CW], xi[CW];
          values(tacc, c0, xr, xi);
          if (add_sum && p.sum_tmem) {  // warp-collective: before any per-row branch
            tc::tmem_ld<CW>(tsum + c0, sr);
            tc::tmem_ld<CW>(tsum + TBN + c0, si);
            tc::tmem_ld_wait();
          }
          if (row >= M) continue;
#pragma unroll
          for (int j = 0; j < CW; ++j)
            if (c0 + j < N) {
              float ur = xr[j], ui = xi[j];
              if (add_sum) {
                ur += sr[j];
                ui += si[j];
              }
              mx = fmaxf(mx, fmaxf(fabsf(ur), fabsf(ui)));
            }
        }
      }
    }
    // agree on the scale and on going on
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      red[warp - 2] = mx;
      redf[warp - 2] = ok ? 0 : 1;
    }
    named_bar_sync(1, NT);
    float m4 = 0.f;
    int fail = 0;
#pragma unroll
    for (int k = 0; k < EPW; ++k) {
      m4 = fmaxf(m4, red[k]);
      fail |= redf[k];
    }
    named_bar_sync(1, NT);  // red is rewritten only after every warp has read it
    if (fail) break;
    const int e = tc::f16_scale_exponent(m4);
    const float osc = ldexpf(1.f, e);
    void* const* dst = last_term ? p.rp : p.tp[ph & 1];

    for (int mt = 0; mt < MT; ++mt) {
      if (last_phase) {
        if (ok && !tc::mbar_wait_warp(&acc_full[sl * 2 + mt], par, p.err, abort_flag))
          ok = false;
        if (!ok) continue;
        tc::tc_fence_after();
      }
      const int row = mt * 128 + q * 32 + lane;
      const bool rok = row < M;
      const uint32_t tacc = taddr + (uint32_t(q * 32) << 16) + uint32_t(sl * 256 + mt * 2 * TBN);
      const uint32_t tsum = taddr + (uint32_t(q * 32) << 16) + uint32_t(256 + mt * 2 * TBN);
      const long off = wb + row;
      c128* Sw = p.S + long(w) * p.ldS + long(row) * N;
#pragma unroll 1
      for (int c0 = CW * h; c0 < TBN; c0 += CW * NH) {
        // this warp's last chunk of the accumulator frees it for the slot's next phase
        const bool last_chunk = c0 + CW * NH >= TBN;
        if (c0 >= N) {
          // no electron column in this chunk: only free the accumulator
          if (last_chunk) {
            tc::tc_fence_before();
            tc::mbar_arrive(&acc_empty[sl * 2 + mt]);
          }
          continue;
        }
        float sr[CW], si[CW];
        if (!p.sum_tmem && taylor && rok) {
          // the running sum from global memory, in flight while the accumulator is read
#pragma unroll
          for (int j = 0; j < CW; ++j)
            if (c0 + j < N) {
              const long idx = off + long(c0 + j) * pl_ld;
              sr[j] = sum_r[idx];
              si[j] = sum_i[idx];
            }
        }
        float xr[CW], xi[CW];
        values(tacc, c0, xr, xi);
        // the running sum of this chunk (taylor phases), warp-collective in tensor memory
        if (taylor && p.sum_tmem) {
          tc::tmem_ld<CW>(tsum + c0, sr);
          tc::tmem_ld<CW>(tsum + TBN + c0, si);
          tc::tmem_ld_wait();
        }
        if (last_chunk) {
          tc::tc_fence_before();
          tc::mbar_arrive(&acc_empty[sl * 2 + mt]);
        }
        if (last_phase) {
          // S = P1 R  (complex128 walker matrix [M][N])
          if (!rok) continue;
#pragma unroll
          for (int j = 0; j < CW; ++j)
            if (c0 + j < N) Sw[c0 + j] = cmk(xr[j], xi[j]);
          continue;
        }
        float ur[CW], ui[CW];
#pragma unroll
        for (int j = 0; j < CW; ++j) {
          ur[j] = taylor ? xr[j] + sr[j] : xr[j];
          ui[j] = taylor ? xi[j] + si[j] : xi[j];
        }
        if (p.sum_tmem && !last_term) {  // the new running sum, warp-collective
          tc::tmem_st<CW>(tsum + c0, ur);
          tc::tmem_st<CW>(tsum + TBN + c0, ui);
          tc::tmem_st_wait();
        }
        if (!rok) continue;
#pragma unroll
        for (int j = 0; j < CW; ++j)
          if (c0 + j < N) {
            const long idx = off + long(c0 + j) * pl_ld;
            if (last_term) {
              split_store16(ur[j] * osc, dst[0], dst[1], idx);
              split_store16(ui[j] * osc, dst[2], dst[3], idx);
            } else {
              if (!p.sum_tmem) {
                sum_r[idx] = ur[j];
                sum_i[idx] = ui[j];
              }
              split_store16(xr[j] * osc, dst[0], dst[1], idx);
              split_store16(xi[j] * osc, dst[2], dst[3], idx);
            }
          }
      }
    }
    if (last_phase) {
      // the last phase has no pass 1: agree here on going on
      if (lane == 0) redf[warp - 2] = ok ? 0 : 1;
      named_bar_sync(1, NT);
      int fail2 = 0;
#pragma unroll
      for (int k = 0; k < EPW; ++k) fail2 |= redf[k];
      named_bar_sync(1, NT);
      if (fail2) break;
    } else {
      // make this phase's planes visible to the TMA loads of the next phase
      fence_proxy_async_global();
      tc::mbar_arrive(&phase_done[sl]);
      (sl ? pinv1 : pinv0) = ldexpf(1.f, -e);
    }
    ++(sl ? use1 : use0);
    sc.advance(sl);
  }
}

template <bool F16, int EPW>
__global__ void __launch_bounds__(ty_threads(EPW), 1)
    taylor_tc_kernel(const __grid_constant__ TyParams p) {
  static_assert(EPW == 4 || EPW == 8, "four or eight epilogue warps");
  // 128 bytes of K per stage and operand row: 32 TF32 or 64 FP16 elements; 32 bytes per MMA
  constexpr int TBKE = F16 ? 2 * TBK : TBK;
  constexpr int KSTEP = F16 ? 16 : 8;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + T_STAGES * T_STAGE);
  uint64_t* empty = full + T_STAGES;
  uint64_t* acc_full = empty + T_STAGES;  // [slot][m tile]
  uint64_t* acc_empty = acc_full + 4;     // [slot][m tile]
  uint64_t* phase_done = acc_empty + 4;   // [slot] epilogue -> TMA: the phase's term is written
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(phase_done + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  float* red = reinterpret_cast<float*>(tmem_slot + 2);  // [EPW] per-warp maxima, [EPW] flags

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nph = p.order + 2;
  const int M = p.M;
  const int nk = (M + TBKE - 1) / TBKE;
  const int MT = (M + 127) / 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < T_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 4; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], 32 * EPW);
    }
    tc::mbar_init(&phase_done[0], 32 * EPW);
    tc::mbar_init(&phase_done[1], 32 * EPW);
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
      Schedule sc(p.W, nph, blockIdx.x, gridDim.x, p.nslots);
      const uint64_t pol_last = tc::make_policy_evict_last();
      const uint64_t pol_first = tc::make_policy_evict_first();
      long it = 0;
      bool ok = true;
      int sl;
      while (ok && sc.get(sl)) {
        const int w = sc.w(sl), ph = sc.ph(sl);
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
            // A (P1 or V_w) does not depend on the previous phase: issue it first.  V_w is read
            // once per Taylor term: kept in L2 until its last term.
            const uint64_t pol = (ph == nph - 2) ? pol_first : pol_last;
            for (int q = 0; q < na; ++q)
              tc::tma_load_3d_hint(st + q * T_A_TILE, &amap[q], &full[s], kc * TBKE, mt * 128,
                                   p1 ? 0 : w, pol);
            if (!b_ready) {
              // B is the previous phase's term of this walker, written by the epilogue warps
              const long done = long(sc.wi(sl)) * (nph - 1) + (ph - 1);
              if (!tc::mbar_wait(&phase_done[sl], unsigned(done) & 1u, p.err, abort_flag)) {
                ok = false;
                break;
              }
              b_ready = true;
            }
            for (int q = 0; q < 4; ++q)
              tc::tma_load_3d(st + 4 * T_A_TILE + q * T_B_TILE, &bmap[q], &full[s], kc * TBKE, 0,
                              w);
          }
        sc.advance(sl);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_split<F16>(128, TBN, false);
      constexpr uint32_t IDN = tc::idesc_split<F16>(128, TBN, true);
      Schedule sc(p.W, nph, blockIdx.x, gridDim.x, p.nslots);
      long it = 0;
      long use0 = 0, use1 = 0;  // accumulator uses of each slot
      bool ok = true;
      int sl;
      while (ok && sc.get(sl)) {
        const int ph = sc.ph(sl);
        const bool p1 = (ph == 0 || ph == nph - 1);
        for (int mt = 0; mt < MT && ok; ++mt) {
          const long use = sl ? use1 : use0;
          if (use >= 1) {
            if (!tc::mbar_wait(&acc_empty[sl * 2 + mt], unsigned(use - 1) & 1u, p.err,
                               abort_flag)) {
              ok = false;
              break;
            }
          }
          tc::tc_fence_after();
          const uint32_t dr = taddr + uint32_t(sl * 256 + mt * 2 * TBN), di = dr + TBN;
          // the small products' accumulators (dual), else the main ones
          const uint32_t er = p.dual ? dr + 256u : dr, ei = er + TBN;
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
            for (int kk = 0; kk < 4; ++kk) {
              if (kc * TBKE + kk * KSTEP >= M) break;  // zero fill past M
              auto A = [&](int q) { return tc::sdesc_sw128(sa + q * T_A_TILE) + uint64_t(2 * kk); };
              auto B = [&](int q) { return tc::sdesc_sw128(sb + q * T_B_TILE) + uint64_t(2 * kk); };
              const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
              // hi*hi products into (dr, di); hi*lo and lo*hi into (er, ei), which are (dr, di)
              // themselves unless dual (the first product into each accumulator starts it)
              const uint32_t accs = p.dual ? acc0 : 1u;
              if (p1) {
                // real A (P1 hi, lo) x complex B
                tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
                tc::mma_split<F16>(er, A(0), B(1), ID, accs);
                tc::mma_split<F16>(er, A(1), B(0), ID, 1);
                tc::mma_split<F16>(di, A(0), B(2), ID, acc0);
                tc::mma_split<F16>(ei, A(0), B(3), ID, accs);
                tc::mma_split<F16>(ei, A(1), B(2), ID, 1);
              } else {
                tc::mma_split<F16>(dr, A(0), B(0), ID, acc0);
                tc::mma_split<F16>(dr, A(2), B(2), IDN, 1);
                tc::mma_split<F16>(er, A(0), B(1), ID, accs);
                tc::mma_split<F16>(er, A(1), B(0), ID, 1);
                tc::mma_split<F16>(er, A(2), B(3), IDN, 1);
                tc::mma_split<F16>(er, A(3), B(2), IDN, 1);
                tc::mma_split<F16>(di, A(0), B(2), ID, acc0);
                tc::mma_split<F16>(di, A(2), B(0), ID, 1);
                tc::mma_split<F16>(ei, A(0), B(3), ID, accs);
                tc::mma_split<F16>(ei, A(1), B(2), ID, 1);
                tc::mma_split<F16>(ei, A(2), B(1), ID, 1);
                tc::mma_split<F16>(ei, A(3), B(0), ID, 1);
              }
            }
            tc::mma_commit(&empty[s]);
          }
          if (!ok) break;
          tc::mma_commit(&acc_full[sl * 2 + mt]);
        }
        ++(sl ? use1 : use0);
        sc.advance(sl);
      }
    }
  } else if constexpr (F16) {
    taylor_epilogue_f16<EPW>(p, taddr, acc_full, acc_empty, phase_done, abort_flag, red, warp,
                             lane);
  } else {
    // epilogue warps: TMEM lane quarter q = warp % 4, one accumulator row per thread; the
    // quarter's NH warps take the column chunks c0 = CW * h + CW * NH * k
    constexpr int NH = EPW / 4, CW = 16 / NH;
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const int N = p.N;
    const long pl_ld = p.pl_ld;
    float* __restrict__ const sum_r = p.sum[0];
    float* __restrict__ const sum_i = p.sum[1];
    Schedule sc(p.W, nph, blockIdx.x, gridDim.x, p.nslots);
    long use0 = 0, use1 = 0;
    bool ok = true;
    int sl;
    while (ok && sc.get(sl)) {
      const int w = sc.w(sl), ph = sc.ph(sl);
      const bool taylor = (ph > 0 && ph < nph - 1);
      const bool last_phase = (ph == nph - 1);
      const bool last_term = (ph == nph - 2);
      const float ai = taylor ? 1.0f / float(ph) : 0.0f;
      // destination planes of this phase: the next B operand (T_ph, or R after the last term)
      void* const* dst = last_term ? p.rp : p.tp[ph & 1];
      float* __restrict__ const d0 = static_cast<float*>(dst[0]);
      float* __restrict__ const d1 = static_cast<float*>(dst[1]);
      float* __restrict__ const d2 = static_cast<float*>(dst[2]);
      float* __restrict__ const d3 = static_cast<float*>(dst[3]);
      const long wb = long(w) * p.pl_bs;
      for (int mt = 0; mt < MT; ++mt) {
        if (!tc::mbar_wait_warp(&acc_full[sl * 2 + mt], unsigned(sl ? use1 : use0) & 1u, p.err,
                                abort_flag)) {
          ok = false;
          break;
        }
        tc::tc_fence_after();
        const int row = mt * 128 + q * 32 + lane;  // orbital index i
        const bool rok = row < M;
        const uint32_t tacc =
            taddr + (uint32_t(q * 32) << 16) + uint32_t(sl * 256 + mt * 2 * TBN);
        // element (n, i) of the [w][n][i] planes: off + n * pl_ld
        const long off = wb + row;
        c128* Sw = p.S + long(w) * p.ldS + long(row) * N;
        // the running sum's columns in tensor memory (sum_tmem): this lane quarter's rows
        const uint32_t tsum = taddr + (uint32_t(q * 32) << 16) + uint32_t(256 + mt * 2 * TBN);
#pragma unroll 1
        for (int c0 = CW * h; c0 < TBN; c0 += CW * NH) {
          const bool last_chunk = c0 + CW * NH >= TBN;
          if (c0 >= N) {
            // no electron column in this chunk: only free the accumulator
            if (last_chunk) {
              tc::tc_fence_before();
              tc::mbar_arrive(&acc_empty[sl * 2 + mt]);
            }
            continue;
          }
          // running-sum loads of this chunk first, then the accumulator columns
          float sr[CW], si[CW];
          if (p.sum_tmem) {
            if (taylor) {  // tensor-memory loads are warp-collective: every lane takes part
              tc::tmem_ld<CW>(tsum + c0, sr);
              tc::tmem_ld<CW>(tsum + TBN + c0, si);
            }
          } else if (rok && taylor) {
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (c0 + j < N) {
                sr[j] = sum_r[off + long(c0 + j) * pl_ld];
                si[j] = sum_i[off + long(c0 + j) * pl_ld];
              }
          }
          float vr[CW], vi[CW];
          tc::tmem_ld<CW>(tacc + c0, vr);
          tc::tmem_ld<CW>(tacc + TBN + c0, vi);
          if (p.dual) {  // + the small products' accumulator (FP32 add, rounded to nearest)
            float wr[CW], wi[CW];
            tc::tmem_ld<CW>(tacc + 256 + c0, wr);
            tc::tmem_ld<CW>(tacc + 256 + TBN + c0, wi);
            tc::tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < CW; ++j) {
              vr[j] += wr[j];
              vi[j] += wi[j];
            }
          }
          tc::tmem_ld_wait();
          if (last_chunk) {
            // the accumulator is free for this slot's next phase
            tc::tc_fence_before();
            tc::mbar_arrive(&acc_empty[sl * 2 + mt]);
          }
          if (taylor) {
            // x = (i/ph) * acc
#pragma unroll
            for (int j = 0; j < CW; ++j) {
              const float xr = -ai * vi[j];
              const float xi = ai * vr[j];
              vr[j] = xr;
              vi[j] = xi;
            }
          }
          if (last_phase) {
            // S = P1 R  (complex128 walker matrix [M][N])
            if (!rok) continue;
#pragma unroll
            for (int j = 0; j < CW; ++j)
              if (c0 + j < N) Sw[c0 + j] = cmk(vr[j], vi[j]);
            continue;
          }
          if (!taylor) {  // phase 0: the sum starts at T_0
#pragma unroll
            for (int j = 0; j < CW; ++j) {
              sr[j] = 0.f;
              si[j] = 0.f;
            }
          }
          float ur[CW], ui[CW];
#pragma unroll
          for (int j = 0; j < CW; ++j) {
            ur[j] = sr[j] + vr[j];
            ui[j] = si[j] + vi[j];
          }
          if (p.sum_tmem && !last_term) {
            tc::tmem_st<CW>(tsum + c0, ur);
            tc::tmem_st<CW>(tsum + TBN + c0, ui);
            tc::tmem_st_wait();
          }
          if (!rok) continue;
#pragma unroll
          for (int j = 0; j < CW; ++j)
            if (c0 + j < N) {
              const long idx = off + long(c0 + j) * pl_ld;
              if (last_term) {
                split_store(ur[j], d0, d1, idx);
                split_store(ui[j], d2, d3, idx);
              } else {
                if (!p.sum_tmem) {
                  sum_r[idx] = ur[j];
                  sum_i[idx] = ui[j];
                }
                split_store(vr[j], d0, d1, idx);
                split_store(vi[j], d2, d3, idx);
              }
            }
        }
      }
      if (!ok) break;
      if (!last_phase) {
        // make this phase's planes visible to the TMA loads of the next phase
        fence_proxy_async_global();
        tc::mbar_arrive(&phase_done[sl]);
      }
      ++(sl ? use1 : use0);
      sc.advance(sl);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(taddr, 512);
}

// ---------------------------------------------------------------------------------------------
// Interleaved form (FP16 split, second accumulator).  Two walkers in flight per CTA, interleaved
// at row-tile granularity: a slot owns 256 TMEM columns that hold ONE 128-row tile of its
// walker's phase (hi*hi products in (dr, di), the small split products in (er, ei)), and the
// tensor core alternates between the slots' tiles, so that one slot's epilogue (and its
// phase-to-phase hand-off through global memory) overlaps the other slot's MMAs.
// The epilogue makes one pass: the power-of-two scale of the planes it stores comes from a
// bound known before the phase,
//   T_0 = P1 S:            |T_0| <= M |P1|max |S|max
//   T_n = (i/n) V T_{n-1}: |T_n| <= M |V|max |T_{n-1}|max / n   (|T_{n-1}|max measured)
//   R = sum_n T_n:         |R|   <= sum_{n<order} |T_n|max + the bound of T_order
// with |P1|max, |S|max, |V|max < 2^14 times their inverse scales.  A loose bound costs nothing:
// FP16 keeps the 22-bit split for every element within 17 binades of the scaled maximum, and an
// element further down has an absolute error (FP16 subnormal spacing) far below the largest
// products'.
constexpr int TI_EPW = 8;                  // epilogue warps: two per TMEM lane quarter
constexpr int TI_NT = 32 * TI_EPW;
constexpr int TI_THREADS = 64 + TI_NT;
constexpr int TI_CW = 8;                   // accumulator columns per epilogue chunk

// (slot, walker, phase, row tile) units in the order every warp role walks them: the slots take
// turns tile by tile; a slot whose walker finished its last phase takes the CTA's next walker
struct TileSchedule {
  int w0, w1, ph0, ph1, mt0, mt1, wi0, wi1;
  int next, cur, W, nph, MT, step;
  __device__ TileSchedule(int W_, int nph_, int MT_, int first, int stride, int nslots)
      : w0(first), w1(nslots > 1 ? first + stride : W_), ph0(0), ph1(0), mt0(0), mt1(0), wi0(0),
        wi1(0), next(first + nslots * stride), cur(0), W(W_), nph(nph_), MT(MT_), step(stride) {}
  __device__ int w(int s) const { return s ? w1 : w0; }
  __device__ int ph(int s) const { return s ? ph1 : ph0; }
  __device__ int mt(int s) const { return s ? mt1 : mt0; }
  __device__ int wi(int s) const { return s ? wi1 : wi0; }
  __device__ bool get(int& s) {
    for (int k = 0; k < 2; ++k) {
      const int c = cur;
      cur ^= 1;
      if (w(c) < W) {
        s = c;
        return true;
      }
    }
    return false;
  }
  __device__ void advance(int s) {
    int& mt_ = s ? mt1 : mt0;
    if (++mt_ < MT) return;
    mt_ = 0;
    int& ph_ = s ? ph1 : ph0;
    if (++ph_ < nph) return;
    ph_ = 0;
    ++(s ? wi1 : wi0);
    (s ? w1 : w0) = next;
    next += step;
  }
};

__global__ void __launch_bounds__(TI_THREADS, 1)
    taylor_il_kernel(const __grid_constant__ TyParams p) {
  constexpr int TBKE = 2 * TBK;  // 64 FP16 elements per 128-byte stage row
  constexpr int KSTEP = 16;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + T_STAGES * T_STAGE);
  uint64_t* empty = full + T_STAGES;
  uint64_t* acc_full = empty + T_STAGES;  // [slot]
  uint64_t* acc_empty = acc_full + 2;     // [slot]
  uint64_t* phase_done = acc_empty + 2;   // [slot] epilogue -> TMA: the phase's planes are written
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(phase_done + 2);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  // [slot][phase parity] maximum |stored value| of the phase (float bits, atomicMax)
  unsigned* maxbits = reinterpret_cast<unsigned*>(tmem_slot + 2);
  int* agree = reinterpret_cast<int*>(tmem_slot + 6);  // [TI_EPW]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nph = p.order + 2;
  const int M = p.M;
  const int nk = (M + TBKE - 1) / TBKE;
  const int MT = (M + 127) / 128;

  if (threadIdx.x == 0) {
    for (int s = 0; s < T_STAGES; ++s) {
      tc::mbar_init(&full[s], 1);
      tc::mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&acc_full[b], 1);
      tc::mbar_init(&acc_empty[b], TI_NT);
      tc::mbar_init(&phase_done[b], TI_NT);
      maxbits[2 * b] = maxbits[2 * b + 1] = 0u;
    }
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
      TileSchedule sc(p.W, nph, MT, blockIdx.x, gridDim.x, p.nslots);
      const uint64_t pol_last = tc::make_policy_evict_last();
      const uint64_t pol_first = tc::make_policy_evict_first();
      long it = 0;
      bool ok = true;
      int sl;
      while (ok && sc.get(sl)) {
        const int w = sc.w(sl), ph = sc.ph(sl), mt = sc.mt(sl);
        const bool p1 = (ph == 0 || ph == nph - 1);
        const CUtensorMap* amap = p1 ? p.p1 : p.v;
        const CUtensorMap* bmap = ph == 0 ? p.s : (ph == nph - 1 ? p.r : p.t[(ph - 1) & 1]);
        const int na = p1 ? 2 : 4;
        const unsigned bytes = unsigned(na * T_A_TILE + 4 * T_B_TILE);
        // B is the previous phase's planes of this walker: ready once its hand-off arrived (the
        // first row tile of the phase waits for it)
        bool b_ready = (ph == 0) || (mt > 0);
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
          // V_w is read once per Taylor term: kept in L2 until its last term
          const uint64_t pol = (ph == nph - 2) ? pol_first : pol_last;
          for (int q = 0; q < na; ++q)
            tc::tma_load_3d_hint(st + q * T_A_TILE, &amap[q], &full[s], kc * TBKE, mt * 128,
                                 p1 ? 0 : w, pol);
          if (!b_ready) {
            const long done = long(sc.wi(sl)) * (nph - 1) + (ph - 1);
            if (!tc::mbar_wait(&phase_done[sl], unsigned(done) & 1u, p.err, abort_flag)) {
              ok = false;
              break;
            }
            b_ready = true;
          }
          for (int q = 0; q < 4; ++q)
            tc::tma_load_3d(st + 4 * T_A_TILE + q * T_B_TILE, &bmap[q], &full[s], kc * TBKE, 0,
                            w);
        }
        sc.advance(sl);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr uint32_t ID = tc::idesc_split<true>(128, TBN, false);
      constexpr uint32_t IDN = tc::idesc_split<true>(128, TBN, true);
      TileSchedule sc(p.W, nph, MT, blockIdx.x, gridDim.x, p.nslots);
      long it = 0;
      long use0 = 0, use1 = 0;  // accumulator uses of each slot
      bool ok = true;
      int sl;
      while (ok && sc.get(sl)) {
        const int ph = sc.ph(sl);
        const bool p1 = (ph == 0 || ph == nph - 1);
        const long use = sl ? use1 : use0;
        if (use >= 1) {
          if (!tc::mbar_wait(&acc_empty[sl], unsigned(use - 1) & 1u, p.err, abort_flag)) break;
        }
        tc::tc_fence_after();
        const uint32_t dr = taddr + uint32_t(sl * 256), di = dr + TBN;
        const uint32_t er = dr + 2 * TBN, ei = dr + 3 * TBN;
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
          for (int kk = 0; kk < 4; ++kk) {
            if (kc * TBKE + kk * KSTEP >= M) break;  // zero fill past M
            auto A = [&](int q) { return tc::sdesc_sw128(sa + q * T_A_TILE) + uint64_t(2 * kk); };
            auto B = [&](int q) { return tc::sdesc_sw128(sb + q * T_B_TILE) + uint64_t(2 * kk); };
            const uint32_t acc0 = (kc > 0 || kk > 0) ? 1u : 0u;
            // hi*hi into (dr, di); hi*lo and lo*hi into (er, ei)
            if (p1) {
              tc::mma_split<true>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<true>(er, A(0), B(1), ID, acc0);
              tc::mma_split<true>(er, A(1), B(0), ID, 1);
              tc::mma_split<true>(di, A(0), B(2), ID, acc0);
              tc::mma_split<true>(ei, A(0), B(3), ID, acc0);
              tc::mma_split<true>(ei, A(1), B(2), ID, 1);
            } else {
              tc::mma_split<true>(dr, A(0), B(0), ID, acc0);
              tc::mma_split<true>(dr, A(2), B(2), IDN, 1);
              tc::mma_split<true>(er, A(0), B(1), ID, acc0);
              tc::mma_split<true>(er, A(1), B(0), ID, 1);
              tc::mma_split<true>(er, A(2), B(3), IDN, 1);
              tc::mma_split<true>(er, A(3), B(2), IDN, 1);
              tc::mma_split<true>(di, A(0), B(2), ID, acc0);
              tc::mma_split<true>(di, A(2), B(0), ID, 1);
              tc::mma_split<true>(ei, A(0), B(3), ID, acc0);
              tc::mma_split<true>(ei, A(1), B(2), ID, 1);
              tc::mma_split<true>(ei, A(2), B(1), ID, 1);
              tc::mma_split<true>(ei, A(3), B(0), ID, 1);
            }
          }
          tc::mma_commit(&empty[s]);
        }
        if (!ok) break;
        tc::mma_commit(&acc_full[sl]);
        ++(sl ? use1 : use0);
        sc.advance(sl);
      }
    }
  } else {
    // epilogue: TMEM lane quarter q = warp % 4 (one accumulator row per thread), the quarter's two
    // warps (h = 0, 1) take alternate 8-column chunks
    const int q = warp & 3;
    const int h = (warp - 2) >> 2;
    const int N = p.N;
    const long pl_ld = p.pl_ld;
    float* __restrict__ const sum_r = p.sum[0];
    float* __restrict__ const sum_i = p.sum[1];
    const float two14 = 16384.f;
    TileSchedule sc(p.W, nph, MT, blockIdx.x, gridDim.x, p.nslots);
    long use0 = 0, use1 = 0;
    // per slot: inverse scale of the planes it stored last, the output scale of its current
    // phase, the measured maximum of its previous term and the sum of its terms' maxima
    float pinv0 = 1.f, pinv1 = 1.f, osc0 = 1.f, osc1 = 1.f;
    float mprev0 = 0.f, mprev1 = 0.f, msum0 = 0.f, msum1 = 0.f;
    int eo0 = 0, eo1 = 0;
    bool wok = true;  // this warp's waits (agreed on at every phase end)
    int sl;
    while (sc.get(sl)) {
      const int w = sc.w(sl), ph = sc.ph(sl), mt = sc.mt(sl);
      const bool taylor = (ph > 0 && ph < nph - 1);
      const bool last_phase = (ph == nph - 1);
      const bool last_term = (ph == nph - 2);
      const float ai = taylor ? 1.0f / float(ph) : 0.0f;
      const float pin = sl ? pinv1 : pinv0;
      const float f_in = ph == 0 ? p.p1_inv * p.s_inv[w]
                                 : (last_phase ? p.p1_inv * pin : p.v_inv[w] * pin);
      if (mt == 0 && !last_phase) {
        // the bound of what this phase stores, and its scale
        const float mp = sl ? mprev1 : mprev0;
        float b;
        if (ph == 0) {
          b = float(M) * (two14 * p.p1_inv) * (two14 * p.s_inv[w]);
        } else {
          b = float(M) * (two14 * p.v_inv[w]) * mp * ai;
          if (last_term) b += sl ? msum1 : msum0;
        }
        const int e = tc::f16_scale_exponent(b);
        (sl ? eo1 : eo0) = e;
        (sl ? osc1 : osc0) = ldexpf(1.f, e);
      }
      const float osc = sl ? osc1 : osc0;
      const unsigned par = unsigned(sl ? use1 : use0) & 1u;
      if (wok) {
        wok = tc::mbar_wait_warp(&acc_full[sl], par, p.err, abort_flag);
        if (wok) tc::tc_fence_after();
      }
      const int row = mt * 128 + q * 32 + lane;
      const bool rok = row < M;
      const uint32_t tacc = taddr + (uint32_t(q * 32) << 16) + uint32_t(sl * 256);
      const long off = long(w) * p.pl_bs + row;
      void* const* dst = last_term ? p.rp : p.tp[ph & 1];
      c128* Sw = p.S + long(w) * p.ldS + long(row) * N;
      float lmax = 0.f;
#pragma unroll 1
      for (int c0 = TI_CW * h; c0 < TBN && wok; c0 += 2 * TI_CW) {
        const bool last_chunk = c0 + 2 * TI_CW >= TBN;
        if (c0 >= N) {
          if (last_chunk) {  // no electron column here: only free the accumulator
            tc::tc_fence_before();
            tc::mbar_arrive(&acc_empty[sl]);
          }
          continue;
        }
        float sr[TI_CW], si[TI_CW];
        if (taylor && rok) {
          // the running sum from global memory, in flight while the accumulators are read
#pragma unroll
          for (int j = 0; j < TI_CW; ++j)
            if (c0 + j < N) {
              const long idx = off + long(c0 + j) * pl_ld;
              sr[j] = sum_r[idx];
              si[j] = sum_i[idx];
            }
        }
        float vr[TI_CW], vi[TI_CW], wr[TI_CW], wi[TI_CW];
        tc::tmem_ld<TI_CW>(tacc + c0, vr);
        tc::tmem_ld<TI_CW>(tacc + TBN + c0, vi);
        tc::tmem_ld<TI_CW>(tacc + 2 * TBN + c0, wr);
        tc::tmem_ld<TI_CW>(tacc + 3 * TBN + c0, wi);
        tc::tmem_ld_wait();
        if (last_chunk) {  // the slot's accumulators are free for its next tile
          tc::tc_fence_before();
          tc::mbar_arrive(&acc_empty[sl]);
        }
        if (!rok) continue;
        float xr[TI_CW], xi[TI_CW];
#pragma unroll
        for (int j = 0; j < TI_CW; ++j) {
          // hi*hi plus the small products (FP32 add, rounded to nearest), in true values
          const float ar = (vr[j] + wr[j]) * f_in, aim = (vi[j] + wi[j]) * f_in;
          xr[j] = taylor ? -ai * aim : ar;
          xi[j] = taylor ? ai * ar : aim;
        }
        if (last_phase) {
          // S = P1 R  (complex128 walker matrix [M][N])
#pragma unroll
          for (int j = 0; j < TI_CW; ++j)
            if (c0 + j < N) Sw[c0 + j] = cmk(xr[j], xi[j]);
          continue;
        }
#pragma unroll
        for (int j = 0; j < TI_CW; ++j)
          if (c0 + j < N) {
            const long idx = off + long(c0 + j) * pl_ld;
            const float ur = taylor ? xr[j] + sr[j] : xr[j];
            const float ui = taylor ? xi[j] + si[j] : xi[j];
            // stored: T_ph (and the running sum), or R = sum + T_order after the last term
            const float tr = last_term ? ur : xr[j];
            const float ti = last_term ? ui : xi[j];
            if (!last_term) {
              sum_r[idx] = ur;
              sum_i[idx] = ui;
            }
            lmax = fmaxf(lmax, fmaxf(fabsf(tr), fabsf(ti)));
            split_store16(tr * osc, dst[0], dst[1], idx);
            split_store16(ti * osc, dst[2], dst[3], idx);
          }
      }
      // this warp's maximum of the tile, into the phase's maximum (non-negative floats order
      // like their bits)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
      if (lane == 0 && !last_phase) atomicMax(&maxbits[2 * sl + (ph & 1)], __float_as_uint(lmax));
      if (mt == MT - 1) {
        // the phase is complete: agree on going on, and on the maximum of what it stored
        if (lane == 0) agree[warp - 2] = wok ? 0 : 1;
        named_bar_sync(1, TI_NT);
        int fail = 0;
#pragma unroll
        for (int k = 0; k < TI_EPW; ++k) fail |= agree[k];
        const float m = __uint_as_float(maxbits[2 * sl + (ph & 1)]);
        // the slot's next phase accumulates into the other parity: cleared here, before the
        // barrier that every warp passes before it works on that phase
        if (threadIdx.x == 64) maxbits[2 * sl + (((ph + 1) % nph) & 1)] = 0u;
        named_bar_sync(1, TI_NT);  // agree and maxbits are rewritten only after everyone read them
        if (fail) break;
        if (!last_phase) {
          (sl ? mprev1 : mprev0) = m;
          if (ph == 0)
            (sl ? msum1 : msum0) = m;
          else if (!last_term)
            (sl ? msum1 : msum0) += m;
          (sl ? pinv1 : pinv0) = ldexpf(1.f, -(sl ? eo1 : eo0));
          // make this phase's planes visible to the TMA loads of the next phase
          fence_proxy_async_global();
          tc::mbar_arrive(&phase_done[sl]);
        }
      }
      ++(sl ? use1 : use0);
      sc.advance(sl);
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 1) tc::tmem_dealloc(taddr, 512);
}

int g_nsm = 0;

}  // namespace

int make_plane_map_3d_es(CUtensorMap* map, const void* base, int esize, long k, long rows,
                         long row_stride, long batch, long batch_stride, int box_rows,
                         int box_batch);

// Planes: FP32 (esize 4, TF32 split) or FP16 (esize 2, FP16 split; then v_inv, s_inv [W] and
// p1_inv give the operands' inverse scales).
int taylor_fused_tc(cudaStream_t s, int esize, const void* const P1p[2], const void* const Vp[4],
                    long ldV, const void* const Sp[4], void* const Tp0[4], void* const Tp1[4],
                    void* const Rp[4], float* const sum[2], long pl_ld, c128* S, long ldS, int W,
                    int M, int N, int order, int nslots, int one_slot_use,
                    const float* v_inv, const float* s_inv, float p1_inv, unsigned* err) {
  if (M > 256 || N > TBN || order < 0) {
    set_error_detail("taylor_fused_tc: M = %d (<= 256), N = %d (<= 64), order = %d", M, N, order);
    return AFQMC_ERR_UNSUPPORTED;
  }
  const bool f16 = esize == 2;
  if (f16 && (!v_inv || !s_inv)) {
    set_error_detail("taylor_fused_tc: FP16 planes without their scales");
    return AFQMC_ERR_ARG;
  }
  if (g_nsm == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_nsm, cudaDevAttrMultiProcessorCount, dev);
  }
  TyParams p{};
  for (int q = 0; q < 2; ++q)
    AFQMC_TRY(make_plane_map_3d_es(&p.p1[q], P1p[q], esize, M, M, pl_ld, 1, long(M) * pl_ld, 128,
                                   1));
  for (int q = 0; q < 4; ++q) {
    AFQMC_TRY(make_plane_map_3d_es(&p.v[q], Vp[q], esize, M, M, ldV, W, long(M) * ldV, 128, 1));
    AFQMC_TRY(make_plane_map_3d_es(&p.s[q], Sp[q], esize, M, N, pl_ld, W, long(N) * pl_ld, TBN,
                                   1));
    AFQMC_TRY(make_plane_map_3d_es(&p.t[0][q], Tp0[q], esize, M, N, pl_ld, W, long(N) * pl_ld,
                                   TBN, 1));
    AFQMC_TRY(make_plane_map_3d_es(&p.t[1][q], Tp1[q], esize, M, N, pl_ld, W, long(N) * pl_ld,
                                   TBN, 1));
    AFQMC_TRY(make_plane_map_3d_es(&p.r[q], Rp[q], esize, M, N, pl_ld, W, long(N) * pl_ld, TBN,
                                   1));
    p.tp[0][q] = Tp0[q];
    p.tp[1][q] = Tp1[q];
    p.rp[q] = Rp[q];
  }
  p.sum[0] = sum[0];
  p.sum[1] = sum[1];
  p.S = S;
  p.ldS = ldS;
  p.pl_ld = pl_ld;
  p.pl_bs = long(N) * pl_ld;
  p.W = W;
  p.M = M;
  p.N = N;
  p.order = order;
  p.v_inv = v_inv;
  p.s_inv = s_inv;
  p.p1_inv = p1_inv;
  p.err = err;
  auto kern = f16 ? taylor_tc_kernel<true, TY_EPW> : taylor_tc_kernel<false, TY_EPW>;
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(T_SMEM)));
  // nslots = 0: two walkers in flight per CTA once every CTA has two, else one
  if (nslots <= 0) nslots = (W >= 2 * g_nsm) ? 2 : 1;
  p.nslots = nslots > 1 ? 2 : 1;
  // with one walker in flight, columns 256..511 are free: for the small products' accumulator
  // (one_slot_use 0) or for the running sum (1)
  p.dual = (p.nslots == 1 && one_slot_use == 0) ? 1 : 0;
  p.sum_tmem = (p.nslots == 1 && one_slot_use == 1) ? 1 : 0;
  const int grid = W < g_nsm ? W : g_nsm;
  if (f16 && p.dual) {
    // the FP16 split with the second accumulator runs interleaved: two walkers per CTA once
    // every CTA has two, their row tiles taking turns on the tensor core
    p.nslots = (W >= 2 * g_nsm) ? 2 : 1;
    AFQMC_CUDA_TRY(cudaFuncSetAttribute(taylor_il_kernel,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, int(T_SMEM)));
    taylor_il_kernel<<<grid, TI_THREADS, T_SMEM, s>>>(p);
    return launch_status("taylor_il_kernel");
  }
  kern<<<grid, ty_threads(TY_EPW), T_SMEM, s>>>(p);
  return launch_status("taylor_tc_kernel");
}

}  // namespace afqmc
