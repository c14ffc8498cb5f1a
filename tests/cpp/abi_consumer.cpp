// A C++ program that uses the library only through include/afqmc_c.h, as a SAFIRE build would:
// the host-side parts of the walker step (seed split, walker generator, comb, exchange plan, the
// particle-hole structure of a determinant list).  Prints one line per result for the test that
// compiles and runs it.
#include <cstdio>
#include <vector>

#include "afqmc_c.h"

int main() {
  std::printf("version %d\n", afqmc_version());
  std::printf("seed %llu\n", afqmc_split_seed(7, 1, 0));
  afqmc_host_rng rng = nullptr;
  if (afqmc_host_rng_create(afqmc_split_seed(3, 0, 0), &rng) != AFQMC_OK) return 1;
  std::vector<double> w = {0.5, 1.5, 0.25, 2.0, 0.75, 1.0};
  std::vector<int> off(w.size());
  if (afqmc_comb(rng, w.data(), int(w.size()), int(w.size()), off.data()) != AFQMC_OK) return 2;
  std::printf("offspring");
  for (int o : off) std::printf(" %d", o);
  std::printf("\n");
  const int counts[2] = {3, 3};
  std::vector<int> plan(4 * 8);
  int nplan = 0;
  if (afqmc_plan_walker_exchange(off.data(), counts, 2, plan.data(), 8, &nplan) != AFQMC_OK)
    return 3;
  std::printf("plan %d", nplan);
  for (int i = 0; i < 4 * nplan; ++i) std::printf(" %d", plan[i]);
  std::printf("\n");
  // reference 0 1 2 in 6 active orbitals; determinants in arbitrary column order
  const int refc[3] = {0, 1, 2};
  const int occ[4 * 3] = {0, 1, 2, 3, 1, 2, 0, 2, 4, 5, 4, 1};
  int det[4], nuniq = 0, nex[4], exc[4 * 2 * 3];
  double sign[4];
  if (afqmc_phmsd_excitations(6, 3, refc, 4, occ, det, sign, &nuniq, nex, exc) != AFQMC_OK)
    return 4;
  std::printf("excitations %d", nuniq);
  for (int k = 0; k < 4; ++k) std::printf(" %d:%+.0f", det[k], sign[k]);
  std::printf("\n");
  std::printf("status %s\n", afqmc_status_string(AFQMC_ERR_ARG));
  afqmc_host_rng_destroy(rng);
  return 0;
}
