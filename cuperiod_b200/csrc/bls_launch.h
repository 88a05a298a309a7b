// Host-side launchers of the BLS kernels (defined in bls_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "bls_device.h"

namespace blsb200 {

// Opt the search kernels in to `smem` bytes of dynamic shared memory (called
// outside any stream capture).
cudaError_t configure_search(size_t smem);

// Persistent search over every work item of the batch in `args`.
cudaError_t launch_search(const BatchArgs& args, int mode, int n_ctas, size_t smem,
                          cudaStream_t stream);

// Phase bins of n points at one period through the fast fold and its fallback.
cudaError_t launch_fold_bins(const double* tau, int n, double P, double f, uint32_t S, double bin,
                             int width, int fb, uint32_t mu, uint32_t mphi, int fast,
                             int32_t* out, int32_t* used_fast, cudaStream_t stream);

// Per-curve largest power, its index, and the power's mean and standard deviation.
cudaError_t launch_best(const double* power, int n_curves, int64_t n_periods, int64_t* best_index,
                        double* best_power, double* mean, double* sd, cudaStream_t stream);

// Bytes of one period's histogram in the kernel's layout.
size_t period_hist_bytes(int mode, int hl);

int search_threads();
int max_resident_ctas(int mode, size_t smem);

}  // namespace blsb200
