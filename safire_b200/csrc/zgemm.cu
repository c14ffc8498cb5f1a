// Batched complex128 GEMM on the FP64 DMMA path (mma.sync.m8n8k4.f64), see zgemm.cuh.
//
// Tile: BM x BN complex outputs per CTA, BK-deep k tiles staged through shared memory with a
// register prefetch of the next tile (double-buffered shared memory, one barrier per k tile).
// Shared-memory row pitches are padded so that the 8x4 / 4x8 DMMA fragment loads are free of
// bank conflicts for both 16-byte (complex) and 8-byte (real) elements.
#include "zgemm.cuh"

namespace afqmc {
namespace {

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <bool REAL>
struct Elem;
template <>
struct Elem<true> {
  using T = double;
};
template <>
struct Elem<false> {
  using T = c128;
};

// pad (in elements) of the contiguous dimension of a shared tile
template <bool TRANSPOSED_STORAGE, bool REAL>
struct Pad {
  static constexpr int value = (TRANSPOSED_STORAGE && !REAL) ? 2 : 4;
};

template <int BM, int BN, int BK, int WM_WARPS, int WN_WARPS, bool AT, bool AC, bool AR, bool BT,
          bool BC, bool BR>
struct Cfg {
  static constexpr int NT = WM_WARPS * WN_WARPS * 32;
  static constexpr int WM = BM / WM_WARPS;  // warp tile rows
  static constexpr int WN = BN / WN_WARPS;  // warp tile cols
  static constexpr int TM = WM / 8;
  static constexpr int TN = WN / 8;
  using TA = typename Elem<AR>::T;
  using TB = typename Elem<BR>::T;
  // A tile: AT ? [BK][BM+pa] : [BM][BK+pa]
  static constexpr int PA = Pad<AT, AR>::value;
  static constexpr int A_ROWS = AT ? BK : BM;
  static constexpr int A_PITCH = (AT ? BM : BK) + PA;
  static constexpr int A_ELEMS = A_ROWS * A_PITCH;
  // B tile: BT ? [BN][BK+pb] : [BK][BN+pb]
  static constexpr int PB = Pad<!BT, BR>::value;
  static constexpr int B_ROWS = BT ? BN : BK;
  static constexpr int B_PITCH = (BT ? BK : BN) + PB;
  static constexpr int B_ELEMS = B_ROWS * B_PITCH;
  static constexpr int A_PER_T = BM * BK / NT;
  static constexpr int B_PER_T = BN * BK / NT;
  static constexpr size_t SMEM =
      2 * (size_t(A_ELEMS) * sizeof(TA) + size_t(B_ELEMS) * sizeof(TB));
  static_assert(BM * BK % NT == 0 && BN * BK % NT == 0, "tile/threads mismatch");
  static_assert(WM % 8 == 0 && WN % 8 == 0 && BK % 4 == 0, "tile granularity");
};

template <bool CONJ>
__device__ __forceinline__ c128 ld_c(const c128* p) {
  c128 v = __ldg(p);
  if (CONJ) v.y = -v.y;
  return v;
}

template <int BM, int BN, int BK, int WM_WARPS, int WN_WARPS, bool AT, bool AC, bool AR, bool BT,
          bool BC, bool BR>
__global__ void __launch_bounds__(WM_WARPS* WN_WARPS * 32)
    zgemm_kernel(GemmParams p) {
  using K = Cfg<BM, BN, BK, WM_WARPS, WN_WARPS, AT, AC, AR, BT, BC, BR>;
  using TA = typename K::TA;
  using TB = typename K::TB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TA* As = reinterpret_cast<TA*>(smem_raw);
  TB* Bs = reinterpret_cast<TB*>(smem_raw + 2 * size_t(K::A_ELEMS) * sizeof(TA));

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp / WN_WARPS) * K::WM;
  const int wn0 = (warp % WN_WARPS) * K::WN;
  const long b = blockIdx.z;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;

  const TA* Ag = reinterpret_cast<const TA*>(p.A) + b * p.strideA;
  const TB* Bg = reinterpret_cast<const TB*>(p.B) + b * p.strideB;

  TA ra[K::A_PER_T];
  TB rb[K::B_PER_T];

  auto load_regs = [&](int k0) {
#pragma unroll
    for (int i = 0; i < K::A_PER_T; ++i) {
      int e = tid + i * K::NT;
      int row = AT ? e / BM : e / BK;
      int col = AT ? e % BM : e % BK;
      int mm = AT ? col : row, kk = AT ? row : col;
      bool in = (m0 + mm < p.m) && (k0 + kk < p.k);
      long off = AT ? long(k0 + kk) * p.lda + (m0 + mm) : long(m0 + mm) * p.lda + (k0 + kk);
      if constexpr (AR) {
        ra[i] = in ? __ldg(Ag + off) : 0.0;
      } else {
        ra[i] = in ? ld_c<AC>(Ag + off) : cmk(0.0, 0.0);
      }
    }
#pragma unroll
    for (int i = 0; i < K::B_PER_T; ++i) {
      int e = tid + i * K::NT;
      int row = BT ? e / BK : e / BN;
      int col = BT ? e % BK : e % BN;
      int nn = BT ? row : col, kk = BT ? col : row;
      bool in = (n0 + nn < p.n) && (k0 + kk < p.k);
      long off = BT ? long(n0 + nn) * p.ldb + (k0 + kk) : long(k0 + kk) * p.ldb + (n0 + nn);
      if constexpr (BR) {
        rb[i] = in ? __ldg(Bg + off) : 0.0;
      } else {
        rb[i] = in ? ld_c<BC>(Bg + off) : cmk(0.0, 0.0);
      }
    }
  };
  auto store_regs = [&](int buf) {
    TA* as = As + buf * K::A_ELEMS;
    TB* bs = Bs + buf * K::B_ELEMS;
#pragma unroll
    for (int i = 0; i < K::A_PER_T; ++i) {
      int e = tid + i * K::NT;
      int row = AT ? e / BM : e / BK;
      int col = AT ? e % BM : e % BK;
      as[row * K::A_PITCH + col] = ra[i];
    }
#pragma unroll
    for (int i = 0; i < K::B_PER_T; ++i) {
      int e = tid + i * K::NT;
      int row = BT ? e / BK : e / BN;
      int col = BT ? e % BK : e % BN;
      bs[row * K::B_PITCH + col] = rb[i];
    }
  };

  double accr[K::TM][K::TN][2], acci[K::TM][K::TN][2];
#pragma unroll
  for (int i = 0; i < K::TM; ++i)
#pragma unroll
    for (int j = 0; j < K::TN; ++j) accr[i][j][0] = accr[i][j][1] = acci[i][j][0] = acci[i][j][1] = 0.0;

  const int ktiles = (p.k + BK - 1) / BK;
  load_regs(0);
  store_regs(0);
  __syncthreads();

  for (int kt = 0; kt < ktiles; ++kt) {
    const int buf = kt & 1;
    if (kt + 1 < ktiles) load_regs((kt + 1) * BK);
    const TA* as = As + buf * K::A_ELEMS;
    const TB* bs = Bs + buf * K::B_ELEMS;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      TA fa[K::TM];
      TB fb[K::TN];
#pragma unroll
      for (int i = 0; i < K::TM; ++i) {
        int r = wm0 + i * 8 + g, c = kk + t;
        fa[i] = AT ? as[c * K::A_PITCH + r] : as[r * K::A_PITCH + c];
      }
#pragma unroll
      for (int j = 0; j < K::TN; ++j) {
        int cn = wn0 + j * 8 + g, r = kk + t;
        fb[j] = BT ? bs[cn * K::B_PITCH + r] : bs[r * K::B_PITCH + cn];
      }
#pragma unroll
      for (int i = 0; i < K::TM; ++i) {
#pragma unroll
        for (int j = 0; j < K::TN; ++j) {
          if constexpr (AR && BR) {
            dmma(accr[i][j][0], accr[i][j][1], fa[i], fb[j]);
          } else if constexpr (AR) {
            dmma(accr[i][j][0], accr[i][j][1], fa[i], fb[j].x);
            dmma(acci[i][j][0], acci[i][j][1], fa[i], fb[j].y);
          } else if constexpr (BR) {
            dmma(accr[i][j][0], accr[i][j][1], fa[i].x, fb[j]);
            dmma(acci[i][j][0], acci[i][j][1], fa[i].y, fb[j]);
          } else {
            dmma(accr[i][j][0], accr[i][j][1], fa[i].x, fb[j].x);
            dmma(accr[i][j][0], accr[i][j][1], -fa[i].y, fb[j].y);
            dmma(acci[i][j][0], acci[i][j][1], fa[i].x, fb[j].y);
            dmma(acci[i][j][0], acci[i][j][1], fa[i].y, fb[j].x);
          }
        }
      }
    }
    if (kt + 1 < ktiles) store_regs(buf ^ 1);
    __syncthreads();
  }

  // epilogue
  c128* Cg = p.C + b * p.strideC;
  c128* Dg = p.D ? p.D + b * p.strideD : nullptr;
  const bool use_beta = (p.beta.x != 0.0 || p.beta.y != 0.0);
#pragma unroll
  for (int i = 0; i < K::TM; ++i) {
    int row = m0 + wm0 + i * 8 + g;
    if (row >= p.m) continue;
#pragma unroll
    for (int j = 0; j < K::TN; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int col = n0 + wn0 + j * 8 + 2 * t + h;
        if (col >= p.n) continue;
        c128 v = cmul(p.alpha, cmk(accr[i][j][h], acci[i][j][h]));
        long oc = long(row) * p.ldc + col;
        if (use_beta) v = cadd(v, cmul(p.beta, Cg[oc]));
        Cg[oc] = v;
        if (Dg) {
          long od = long(row) * p.ldd + col;
          Dg[od] = p.d_store ? v : cadd(Dg[od], v);
        }
      }
    }
  }
}

template <int BM, int BN, int BK, int WMW, int WNW, bool AT, bool AC, bool AR, bool BT, bool BC,
          bool BR>
int launch(cudaStream_t s, int batch, const GemmParams& p) {
  using K = Cfg<BM, BN, BK, WMW, WNW, AT, AC, AR, BT, BC, BR>;
  auto kern = zgemm_kernel<BM, BN, BK, WMW, WNW, AT, AC, AR, BT, BC, BR>;
  AFQMC_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(K::SMEM)));
  dim3 grid(ceil_div(p.n, BN), ceil_div(p.m, BM), batch);
  kern<<<grid, K::NT, K::SMEM, s>>>(p);
  return launch_status("zgemm_kernel");
}

template <bool AT, bool AC, bool AR, bool BT, bool BC, bool BR>
int launch_cfg(cudaStream_t s, int batch, const GemmParams& p) {
  // small problems (per-walker products with N ~ 50) use a 32-row tile to cut padding waste
  if (p.m <= 32) return launch<32, 64, 16, 1, 4, AT, AC, AR, BT, BC, BR>(s, batch, p);
  return launch<64, 64, 16, 2, 4, AT, AC, AR, BT, BC, BR>(s, batch, p);
}

}  // namespace

int zgemm(cudaStream_t s, int batch, GemmTrans ta, bool a_real, GemmTrans tb, bool b_real,
          const GemmParams& p) {
  if (p.m <= 0 || p.n <= 0 || batch <= 0) return AFQMC_OK;
  if (p.k <= 0) {
    set_error_detail("zgemm: k = 0 is not supported by the kernel launcher");
    return AFQMC_ERR_SHAPE;
  }
  if (batch > 65535) {
    set_error_detail("zgemm: batch %d exceeds the grid limit", batch);
    return AFQMC_ERR_SHAPE;
  }
  const bool AT = (ta == GT || ta == GH), AC = (ta == GC || ta == GH);
  const bool BT = (tb == GT || tb == GH), BC = (tb == GC || tb == GH);
  if ((a_real && AC) || (b_real && BC)) {
    // conjugating a real operand is the identity
    return zgemm(s, batch, AT ? GT : GN, a_real, BT ? GT : GN, b_real, p);
  }
  // Instantiated combinations (the products the walker step and its setup use).
#define AFQMC_GEMM_CASE(at, ac, ar, bt, bc, br)                                    \
  if (AT == at && AC == ac && a_real == ar && BT == bt && BC == bc && b_real == br) \
    return launch_cfg<at, ac, ar, bt, bc, br>(s, batch, p);
  AFQMC_GEMM_CASE(false, false, false, false, false, false)  // A*B
  AFQMC_GEMM_CASE(false, false, true, false, false, false)   // real A * B
  AFQMC_GEMM_CASE(false, false, false, false, false, true)   // A * real B
  AFQMC_GEMM_CASE(false, false, false, true, false, false)   // A * B^T
  AFQMC_GEMM_CASE(false, false, false, true, false, true)    // A * real B^T
  AFQMC_GEMM_CASE(true, false, false, true, false, false)    // A^T * B^T
  AFQMC_GEMM_CASE(true, false, false, false, false, false)   // A^T * B
  AFQMC_GEMM_CASE(true, true, false, false, false, false)    // A^H * B
  AFQMC_GEMM_CASE(false, false, true, true, false, true)     // real A * real B^T
  AFQMC_GEMM_CASE(false, false, false, false, true, false)   // A * conj(B)
  AFQMC_GEMM_CASE(false, false, false, true, true, false)    // A * B^H
#undef AFQMC_GEMM_CASE
  set_error_detail("zgemm: operand combination (ta=%d a_real=%d tb=%d b_real=%d) not instantiated",
                   int(ta), int(a_real), int(tb), int(b_real));
  return AFQMC_ERR_UNSUPPORTED;
}

}  // namespace afqmc
