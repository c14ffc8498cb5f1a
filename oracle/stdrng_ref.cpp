// ORACLE pin (test infrastructure only).  Prints uniforms drawn exactly the way the reference's
// HostRandomGenerator draws them (src/utilities/Random.hpp:37-51): std::mt19937 constructed from
// the 32-bit truncation of the seed, sampled through std::uniform_real_distribution<double>(0,1)
// of the same libstdc++ the reference builds against.  Used to pin oracle/rng.c.
//   usage: stdrng_ref <seed64> <count>
#include <cstdio>
#include <cstdlib>
#include <random>

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  unsigned long long seed = std::strtoull(argv[1], nullptr, 10);
  long n = std::strtol(argv[2], nullptr, 10);
  std::mt19937 rng{std::mt19937::result_type(seed)};
  std::uniform_real_distribution<double> dist(0.0, 1.0);
  for (long i = 0; i < n; ++i) std::printf("%.17g\n", dist(rng));
  return 0;
}
