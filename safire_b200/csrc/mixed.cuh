// Mixed-precision (tensor-core) contractions of the walker step (see mixed.cu).
#pragma once

#include "common.cuh"
#include "energy.cuh"

namespace afqmc {

struct MixedHam;  // tensor-core copies of the Hamiltonian tensors

int mixed_ham_create(MixedHam** out, const EnergyArgs& a, cudaStream_t s);
void mixed_ham_destroy(MixedHam* m);
int vbias_mixed(cudaStream_t s, MixedHam* m, const c128* G, long ldG, c128* v, int W, double a);
int vhs_mixed(cudaStream_t s, MixedHam* m, const c128* X, c128* V, int W, double a);
int propagate_mixed(cudaStream_t s, MixedHam* m, const void* P1, bool p1_real, const c128* V,
                    long strideV, c128* S, long ldS, int W, int M, int N, int order, c128* w1,
                    c128* w2, c128* w3);
int energy_mixed(cudaStream_t s, MixedHam* m, const EnergyArgs& a, c128* E, int W, bool addH1,
                 bool addEJ, bool addEXX);

}  // namespace afqmc
