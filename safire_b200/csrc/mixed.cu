// Mixed-precision contractions: not built yet in this revision; every entry reports
// AFQMC_ERR_UNSUPPORTED so that a mixed request never silently runs another path.
#include "mixed.cuh"

namespace afqmc {

struct MixedHam {
  int dummy;
};

int mixed_ham_create(MixedHam** out, const EnergyArgs&, cudaStream_t) {
  *out = nullptr;
  set_error_detail("mixed precision path is not available in this build");
  return AFQMC_ERR_UNSUPPORTED;
}
void mixed_ham_destroy(MixedHam* m) { delete m; }
int vbias_mixed(cudaStream_t, MixedHam*, const c128*, long, c128*, int, double) {
  return AFQMC_ERR_UNSUPPORTED;
}
int vhs_mixed(cudaStream_t, MixedHam*, const c128*, c128*, int, double) { return AFQMC_ERR_UNSUPPORTED; }
int propagate_mixed(cudaStream_t, MixedHam*, const void*, bool, const c128*, long, c128*, long, int,
                    int, int, int, c128*, c128*, c128*) {
  return AFQMC_ERR_UNSUPPORTED;
}
int energy_mixed(cudaStream_t, MixedHam*, const EnergyArgs&, c128*, int, bool, bool, bool) {
  return AFQMC_ERR_UNSUPPORTED;
}

}  // namespace afqmc
