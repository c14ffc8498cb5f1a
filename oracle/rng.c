/*
 * ORACLE (test infrastructure only; never linked into the product library).
 *
 * Plain-C restatement of the random-number plumbing of the reference AFQMC driver:
 *
 *  - split_seed: the splitmix64 finalizer that turns (seed, rank, stream) into a generator seed
 *    (reference: src/utilities/Random.cpp:7-20).
 *  - HostRandomGenerator: std::mt19937 seeded with the low 32 bits of that seed, sampled through
 *    std::uniform_real_distribution<double>(0,1) (reference: src/utilities/Random.hpp:37-51).
 *    libstdc++ implements that distribution with std::generate_canonical<double,53>, which draws
 *    two 32-bit words x0, x1 and returns (x0 + x1*2^32) / 2^64, clamped below 1.  The Mersenne
 *    Twister itself follows the published MT19937 algorithm (Matsumoto & Nishimura, 1998).
 *  - comb: the comb branching of population control
 *    (reference: src/AFQMC/Walkers/population_control.hpp:34-65).
 *
 * Built by oracle/Makefile into oracle/_build/liboracle.so and loaded with ctypes by the tests.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define MT_N 624
#define MT_M 397

typedef struct {
  uint32_t mt[MT_N];
  int mti;
} oracle_mt19937;

uint64_t oracle_split_seed(int seed, int rank, unsigned stream) {
  uint64_t x = ((uint64_t)(unsigned)seed << 32) | ((uint64_t)stream << 24) | (unsigned)rank;
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

int oracle_mt_state_size(void) { return (int)sizeof(oracle_mt19937); }

void oracle_mt_seed(oracle_mt19937* s, uint32_t seed) {
  s->mt[0] = seed;
  for (int i = 1; i < MT_N; ++i)
    s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
  s->mti = MT_N;
}

static void mt_twist(oracle_mt19937* s) {
  for (int i = 0; i < MT_N; ++i) {
    uint32_t y = (s->mt[i] & 0x80000000u) | (s->mt[(i + 1) % MT_N] & 0x7fffffffu);
    uint32_t v = s->mt[(i + MT_M) % MT_N] ^ (y >> 1);
    if (y & 1u) v ^= 0x9908b0dfu;
    s->mt[i] = v;
  }
  s->mti = 0;
}

uint32_t oracle_mt_next(oracle_mt19937* s) {
  if (s->mti >= MT_N) mt_twist(s);
  uint32_t y = s->mt[s->mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

double oracle_mt_canonical(oracle_mt19937* s) {
  /* generate_canonical<double,53> on a 32-bit engine: k = 2 draws. */
  double sum = (double)oracle_mt_next(s);
  sum += (double)oracle_mt_next(s) * 4294967296.0;
  double r = sum / 18446744073709551616.0;
  if (r >= 1.0) r = nextafter(1.0, 0.0);
  return r;
}

void oracle_mt_fill_uniform(oracle_mt19937* s, double* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = oracle_mt_canonical(s);
}

/*
 * comb(rng, weights, num_target): one uniform r; tooth ic sits at (ic + r) * total / num_target
 * on the running (sequential) sum of the weights.  Returns 0, or -1 when the total weight
 * collapsed (the reference aborts there).
 */
int oracle_comb(oracle_mt19937* s, const double* weights, int n, int num_target, int* offspring) {
  double total = 0.0;
  for (int i = 0; i < n; ++i) total += weights[i];
  if (!(total > 1e-6)) return -1;
  double r = oracle_mt_canonical(s);
  int last = n - 1;
  while (weights[last] <= 0.0) --last;
  memset(offspring, 0, sizeof(int) * (size_t)n);
  int iw = 0, ic = 0;
  double cum = weights[0];
  while (ic < num_target) {
    double tooth = (ic + r) * total / num_target;
    if (tooth < cum || iw == last) {
      offspring[iw] += 1;
      ++ic;
    } else {
      ++iw;
      cum += weights[iw];
    }
  }
  return 0;
}
