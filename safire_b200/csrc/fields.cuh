// Force-bias field construction and the counter-based field generator (see fields.cu).
#pragma once

#include "common.cuh"

namespace afqmc {

// Philox4x32-10 (Salmon et al., SC'11): 4x32-bit counter, 2x32-bit key, 10 rounds.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = uint64_t(M0) * c[0];
    uint64_t p1 = uint64_t(M1) * c[2];
    uint32_t hi0 = uint32_t(p0 >> 32), lo0 = uint32_t(p0);
    uint32_t hi1 = uint32_t(p1 >> 32), lo1 = uint32_t(p1);
    uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += W0;
    k1 += W1;
  }
}

// Two uniforms in (0, 1) with 53 random bits each for field pair (walker w, index pair n2) of step
// `step` under `seed`.
__host__ __device__ __forceinline__ void philox_uniform2(unsigned long long seed,
                                                        unsigned long long step, uint32_t w,
                                                        uint32_t n2, double out[2]) {
  uint32_t c[4] = {n2, w, uint32_t(step), uint32_t(step >> 32)};
  philox4x32_10(c, uint32_t(seed), uint32_t(seed >> 32));
  const double scale = 1.1102230246251565e-16;  // 2^-53
  uint64_t a = ((uint64_t(c[0]) << 32) | c[1]) >> 11;
  uint64_t b = ((uint64_t(c[2]) << 32) | c[3]) >> 11;
  out[0] = (double(a) + 0.5) * scale;
  out[1] = (double(b) + 0.5) * scale;
}

// X, HW, mf from vbias (X may alias vbias).  mf0 = -Re(vMF.vMF)/2.
// u != nullptr: caller uniforms [W][ldu]; else Philox(seed, *counter) and ++*counter on device.
int construct_x(cudaStream_t s, const c128* vbias, long ldv, const double* u, long ldu,
                const c128* vMF, c128* X, long ldx, c128* HW, c128* mf, int W, int Nc,
                double vbias_bound, double mf0, unsigned long long seed,
                unsigned long long* counter);

}  // namespace afqmc
