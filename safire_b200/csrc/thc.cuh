// Tensor-hypercontraction Hamiltonian operations (see thc.cu).
#pragma once

#include "common.cuh"

namespace afqmc {

struct ThcData;  // THC factors on the device and their workspace

// X [M][nu] (real), Luv [nu][nv] (real), Z [nu][nu] (real; nullptr: Luv Luv^T), host arrays;
// PsiT_dev [nup + ndn (COLLINEAR) or nup][M] on the device (the conjugate-transposed trial)
int thc_create(ThcData** out, int walker_type, int M, int nup, int ndn, int nu, int nv,
               const double* X, const double* L, const double* Z, const c128* PsiT_dev);
void thc_destroy(ThcData* t);
// v [W][nv] = sqrt(dt) sum_u Luv[u][n] Guu[w][u], Guu scaled by a_occ (2 for CLOSED walkers)
int thc_vbias(cudaStream_t s, ThcData* t, const c128* G, long ldG, c128* v, int W, double dt,
              double a_occ);
// V [W][M][M] = sqrt(dt) X diag(Luv x_w) X^T
int thc_vhs(cudaStream_t s, ThcData* t, const c128* X, c128* V, int W, double dt);
// E [W][3] = (E1, EXX, EJ)
int thc_energy(cudaStream_t s, ThcData* t, const c128* G, long ldG, const c128* haj, double E0,
               double scl, double sclj, c128* E, int W, bool addH1, bool addEJ, bool addEXX);
int thc_sizes(const ThcData* t, int* nu, int* nv);

}  // namespace afqmc
