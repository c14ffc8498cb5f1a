// Local-energy kernels (see energy.cu).
#pragma once

#include "common.cuh"

namespace afqmc {

struct EnergyArgs {
  const c128* G;  // [W][ldG], spin blocks of nel[s] rows x M starting at row el_off[s]
  long ldG;
  int M, Nc, nspin;
  int nel[2], el_off[2];
  const c128* haj;            // [nel_tot][M]
  const c128* Lnak[2];        // [Nc][nel[s]][M]
  const double* Lnak_real[2]; // real copies (real trial) or nullptr
  double E0, scl, sclj;
  const double* Likn;  // [nspin_H2][M*M][Nc] (mixed-precision set-up)
  int nspin_H2;
  // mixed precision: take the Coulomb vector Kl = sum_{a,k} G Lnak of EJ from a complex128 GEMM
  // instead of the traces of the tensor-core exchange tiles
  bool coulomb_fp64 = false;
};

struct MixedHam;

// complex128 path (and mixed-precision exchange GEMM when tc is given).  workT: chunk workspace of workT_elems complex elements; exx_part, Kl: [W][Nc].
// tc != nullptr: the exchange tensor chunks come from the tensor-core GEMM (mixed precision).
int energy_fp64(cudaStream_t s, const EnergyArgs& a, c128* E, int W, bool addH1, bool addEJ,
                bool addEXX, c128* workT, long workT_elems, c128* exx_part, c128* Kl,
                MixedHam* tc = nullptr);

}  // namespace afqmc
