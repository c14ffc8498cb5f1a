// Walker-property kernels (see update.cu).
#pragma once

#include "common.cuh"

namespace afqmc {

// stats[5]: eloc {total, upper, lower}, weight {total, upper}
int walker_update(cudaStream_t s, c128* buf, long walker_size, long prop0, int W,
                  const c128* new_ovlp, const c128* mf, const c128* hw, double dt, double Eshift,
                  const double* Eshift_dev, double E0, double lower_cut, double upper_cut,
                  double max_weight, unsigned long long* stats);
int copy_rows(cudaStream_t s, c128* buf, long walker_size, const int* dst, const int* src, int n);
int pack_rows(cudaStream_t s, const c128* buf, long walker_size, const int* idx, int n, c128* out);
int unpack_rows(cudaStream_t s, c128* buf, long walker_size, const int* idx, int n, const c128* in);
int normalize_weights(cudaStream_t s, c128* buf, long walker_size, long prop0, int W);
int gather_property(cudaStream_t s, const c128* buf, long walker_size, long off, int W, c128* out);
int scatter_property(cudaStream_t s, c128* buf, long walker_size, long off, int W, const c128* in);
int energy_sums(cudaStream_t s, const c128* buf, long walker_size, long prop0, int W,
                const c128* E, c128* out4);
int pseudo_energy_sums(cudaStream_t s, const c128* buf, long walker_size, long prop0, int W,
                       double dt, c128* out2);

}  // namespace afqmc
