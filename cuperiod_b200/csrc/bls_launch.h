// Host-side launchers of the BLS kernels (defined in bls_kernels.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "bls_device.h"

namespace blsb200 {

// Opt the search kernels of one accumulation mode in to `smem` bytes of dynamic
// shared memory (called outside any stream capture).
cudaError_t configure_search(int mode, size_t smem);

// Raise kernel fn's dynamic shared-memory limit on the current device to at
// least smem bytes.  The limit is process-wide per kernel and device, so it only
// ever grows (under a lock): a launch from one thread cannot lower it under a
// concurrent launch from another that needs more.
cudaError_t raise_smem_limit(const void* fn, size_t smem);

// Persistent search over every work item of the batch in `args`.
cudaError_t launch_search(const BatchArgs& args, int mode, int n_ctas, size_t smem,
                          cudaStream_t stream);

// Phase bins of n points at one period through the fast fold and its fallback.
cudaError_t launch_fold_bins(const double* tau, int n, double P, double f, uint32_t S, double bin,
                             int width, int fb, uint32_t mu, uint32_t mphi, int fast,
                             int32_t* out, int32_t* used_fast, cudaStream_t stream);

// Per-curve largest power, its index, and the power's mean and standard deviation.
// Curve c's spectrum is power[spec_off[c] .. spec_off[c + 1]).
cudaError_t launch_best(const double* power, int n_curves, const int64_t* spec_off,
                        int64_t* best_index, double* best_power, double* mean, double* sd,
                        cudaStream_t stream);

// Scratch of the allocation-free search (bls_launch_best_noalloc): one
// file-scope device array per device.  Bytes [0, 64): the work counters of the
// two accumulation modes (words 0 and 1) and the error flag (word 8), which
// must all be zero when a search starts.  From byte 256: per curve the best
// index (int64), then best power, power mean and power standard deviation
// (double), kStaticMaxCurves entries each, written in full by best_kernel.
constexpr int kStaticMaxCurves = 65536;
constexpr size_t kStaticResultsOffset = 256;
constexpr size_t kStaticScratchBytes = kStaticResultsOffset + (size_t)kStaticMaxCurves * 32;

// Device address of that array on `device`, which must be the current device.
// Looked up once per device (cudaGetSymbolAddress) and cached.
cudaError_t static_scratch_address(int device, void** ptr);

// Per-curve result rows: the up to n_best alias-diverse peaks of each curve's
// spectrum (grid index and 8 fields each: period, frequency, power, depth,
// depth_snr, duration, t0, sde) and their count.  Curve c's spectrum is
// [spec_off[c], spec_off[c + 1]) of each field; its grid's frequencies start at
// freq[grid_base[c]]; max_periods bounds every curve's spectrum length.
cudaError_t launch_rows(const double* out, int64_t out_stride, int n_curves,
                        const int64_t* spec_off, const int64_t* grid_base, int64_t max_periods,
                        const double* freq, const double* sep, const double* tol, int n_best,
                        int harmonic_max, int32_t* n_peaks, int64_t* index, double* fields,
                        cudaStream_t stream);

// Bytes of one period's histogram in the kernel's layout.
size_t period_hist_bytes(int mode, int hl);

// Joint-ephemeris multi-band search (bls_joint.cu): static shared memory of one
// CTA, CTAs resident per SM (histograms in `smem` bytes of dynamic shared memory,
// or in global scratch), and the persistent launch over every trial period.
size_t joint_static_smem();
cudaError_t configure_joint(size_t smem);
int joint_resident_ctas(bool in_smem, size_t smem);
cudaError_t launch_joint(const JointArgs& args, bool in_smem, size_t smem, int n_ctas,
                         cudaStream_t stream);

// Transit least squares (tls_kernels.cu): shared memory of one work item, the
// opt-in, CTAs resident per SM and the persistent launch over every item.
size_t tls_smem_bytes(int n_bins, int max_width, int tile, int n_tmpl);
cudaError_t configure_tls(size_t smem);
int tls_resident_ctas(size_t smem);
cudaError_t launch_tls(const TlsArgs& args, int n_ctas, size_t smem, cudaStream_t stream);

int search_threads();
int max_resident_ctas(int mode, size_t smem);
// Static shared memory of the search kernel of one accumulation mode (bytes).
size_t search_static_smem(int mode);

}  // namespace blsb200
