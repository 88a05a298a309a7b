// Transit least squares matched-filter kernel (sm_100a): the limb-darkened
// template search of cuPeriod src/cuperiod/methods/tls.py:516-593 (its CUDA
// tls_block, 323-414, searches one period per block).
//
// A persistent grid of 256-thread CTAs pulls work items (curve, tile of up to
// kTlsMaxTile consecutive trial periods).  Per item a CTA
//   1. folds every point of the curve into one phase histogram per period of
//      the tile: the reference's bin, q = tau/P, ph = q - floor(q),
//      bin = int(ph * n_bins) clipped -- from a fixed-point fast path where its
//      host-derived margins prove the result, else from those IEEE operations;
//      a thread holds 8 time-consecutive points (the BLS engine's chunked
//      layout) and merges runs of equal bins in registers.  yw and w are 64-bit
//      fixed point (a power-of-two scale per curve, magnitudes summing below
//      2^61); a run's sum is added to a bin's int64 as two native 32-bit shared
//      atomics, the low word first and then the high word plus the carry the
//      low word's old value shows (64-bit shared atomics are emulated on
//      sm_100), so every bin holds the exact integer sum; the words lie in
//      four planes (low and high of yw, of w), so different bins use
//      different banks;
//   2. turns every bin into FP64 (one rounding of the exact sum) and pads the
//      histogram circularly by max_width - 1 bins (the reference's pad);
//   3. per period, one thread per start phase slides every template over the
//      bins: num = sum g a, cwg = sum g b, den = sum g^2 b, accumulated in k
//      order with the reference's FP64 operations; a start counts when
//      num < 0, den > w_eps and de = den - cwg^2 / w_total > den_rel * den, and
//      the largest sr = num^2 / de wins, the first in (width, start) order among
//      equals (the reference's strict '>' sweep);
//   4. writes sr, depth = -num/de, duration = width / n_bins * P and the
//      mid-transit phase time (centre - floor(centre)) * P.
#include <cuda_runtime.h>
#include <stdint.h>

#include "bls_device.h"
#include "bls_fold.cuh"
#include "bls_launch.h"

namespace blsb200 {
namespace {

constexpr int kTThreads = kChunkThreads;
constexpr int kTWarps = kTThreads / 32;
constexpr int kTPts = kChunkPts;
constexpr unsigned kTAll = 0xffffffffu;

enum : int { TERR_DESC = 1 };

struct TlsShared {
    double red_sr[kTWarps];
    double red_depth[kTWarps];
    long long red_key[kTWarps];
    int next;
};

// The reference's phase bin (tls.py:535-542).
__device__ __forceinline__ int tls_bin(double x, double P, int n_bins) {
    const double q = __ddiv_rn(x, P);
    const double ph = __dsub_rn(q, floor(q));
    int b = (int)__dmul_rn(ph, (double)n_bins);
    b = b > n_bins - 1 ? n_bins - 1 : b;
    return b < 0 ? 0 : b;
}

// Fast TLS bin: the phase frac(x * RN(1/P)) on a 2^-32 grid (one FMA, as the
// BLS fast fold), times n_bins as a 64-bit integer product whose high word is
// the bin and low word the position inside it.  Returns the reference's bin
// when the phase is further than the combined rounding error from a cycle edge
// (margin mphi) and from a bin edge (margin mu), else -1.
__device__ __forceinline__ int tls_bin_fast(double x, double f, int n_bins, uint32_t mu,
                                            uint32_t mphi) {
    const double qm = __fma_rn(x, f, 1572864.0);
    const uint32_t phi = (uint32_t)__double2loint(qm);
    const unsigned long long prod = (unsigned long long)phi * (unsigned)n_bins;
    const uint32_t fr = (uint32_t)prod;
    const bool ok = ((phi - mphi) < (0u - 2u * mphi)) & ((fr - mu) < (0u - 2u * mu));
    return ok ? (int)(prod >> 32) : -1;
}

// Of two candidates (sr, key = width index << 32 | start, depth), the one the
// reference keeps: the larger sr, then the earlier (width, start); key < 0 is
// no candidate.
__device__ __forceinline__ void tls_keep(double& sr, long long& key, double& depth, double osr,
                                         long long okey, double odepth) {
    if (okey >= 0 && (key < 0 || osr > sr || (osr == sr && okey < key))) {
        sr = osr;
        key = okey;
        depth = odepth;
    }
}

// Add a run's sums to bin b of one period's four word planes (the low and high
// words of Y, then of W, each plane `stride` words): plane-major, so that the
// words of different bins fall on different banks.
__device__ __forceinline__ void flush_run(unsigned* planes, int stride, int b, long long ay,
                                          long long aw) {
    add_i64_split(planes + b, planes + stride + b, ay);
    add_i64_split(planes + 2 * stride + b, planes + 3 * stride + b, aw);
}

__device__ __forceinline__ long long plane_value(const unsigned* lo, const unsigned* hi, int b) {
    return (long long)(((unsigned long long)hi[b] << 32) | lo[b]);
}

__global__ void __launch_bounds__(kTThreads, 3) tls_kernel(TlsArgs a) {
    extern __shared__ __align__(16) unsigned char tls_dyn[];
    __shared__ TlsShared s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nb = a.n_bins, ext = a.n_bins + a.max_width - 1;
    // dynamic shared memory: the FP64 bins {a, b} (padded) of every period of
    // the tile, the four word planes of every period's exact sums, the templates
    double2* ab = reinterpret_cast<double2*>(tls_dyn);
    unsigned* words = reinterpret_cast<unsigned*>(ab + (size_t)a.tile * ext);
    double* g = reinterpret_cast<double*>(words + (size_t)a.tile * 4 * nb);
    for (int i = tid; i < a.n_tmpl; i += kTThreads) g[i] = a.tmpl[i];
    for (;;) {
        if (tid == 0) s.next = atomicAdd(a.work_counter, 1);
        __syncthreads();
        const int item = s.next;
        if (item >= a.n_items) break;
        const int c = item / a.tiles_per_curve;
        const int64_t p0 = (int64_t)(item % a.tiles_per_curve) * a.tile;
        const int np = (int)min((int64_t)a.tile, a.n_periods - p0);
        const TlsCurveDesc cv = a.curves[c];
        for (int i = tid; i < np * 4 * nb; i += kTThreads) words[i] = 0u;
        __syncthreads();

        // 1. fold: full chunks lane-interleaved, the tail in time order
        const int n = cv.n_points;
        const int full = (n / kChunk) * kChunk;
        for (int base = 0; base < full; base += kChunk) {
            double x[kTPts];
            long long yq[kTPts], wq[kTPts];
#pragma unroll
            for (int r = 0; r < kTPts; ++r) {
                const int64_t slot = cv.point_off + base + r * kTThreads + tid;
                x[r] = a.tau[slot];
                yq[r] = a.qy[slot];
                wq[r] = a.qw[slot];
            }
            for (int p = 0; p < np; ++p) {
                const double P = a.period[p0 + p], f = a.freq[p0 + p];
                unsigned* h = words + (size_t)p * 4 * nb;
                const bool fast = a.fast_fold != 0;
                const uint32_t mu = a.margin_u, mphi = a.margin_phi;
                int prev = fast ? tls_bin_fast(x[0], f, nb, mu, mphi) : -1;
                if (prev < 0) prev = tls_bin(x[0], P, nb);
                long long ay = yq[0], aw = wq[0];
#pragma unroll
                for (int r = 1; r < kTPts; ++r) {
                    int b = fast ? tls_bin_fast(x[r], f, nb, mu, mphi) : -1;
                    if (b < 0) b = tls_bin(x[r], P, nb);
                    if (b != prev) {
                        flush_run(h, nb, prev, ay, aw);
                        prev = b;
                        ay = yq[r];
                        aw = wq[r];
                    } else {
                        ay += yq[r];
                        aw += wq[r];
                    }
                }
                flush_run(h, nb, prev, ay, aw);
            }
        }
        for (int j = full + tid; j < n; j += kTThreads) {
            const int64_t slot = cv.point_off + j;
            const double xj = a.tau[slot];
            const long long yj = a.qy[slot], wj = a.qw[slot];
            for (int p = 0; p < np; ++p)
                flush_run(words + (size_t)p * 4 * nb, nb, tls_bin(xj, a.period[p0 + p], nb), yj,
                          wj);
        }
        __syncthreads();

        // 2. FP64 bins (a = sum yw, b = sum w), then the circular pad (544-546)
        for (int i = tid; i < np * nb; i += kTThreads) {
            const int p = i / nb, bin = i - p * nb;
            const unsigned* h = words + (size_t)p * 4 * nb;
            const long long y = plane_value(h, h + nb, bin);
            const long long w = plane_value(h + 2 * nb, h + 3 * nb, bin);
            ab[p * ext + bin] = make_double2(__dmul_rn(__ll2double_rn(y), cv.y_unit),
                                             __dmul_rn(__ll2double_rn(w), cv.w_unit));
        }
        __syncthreads();
        if (a.max_width > 1)
            for (int i = tid; i < np * (a.max_width - 1); i += kTThreads) {
                const int p = i / (a.max_width - 1), j = i - p * (a.max_width - 1);
                ab[p * ext + nb + j] = ab[p * ext + j];
            }
        __syncthreads();

        // 3-4. the template sweep and the winner of each period
        for (int p = 0; p < np; ++p) {
            const double2* v = ab + p * ext;
            double best = 0.0, best_depth = 0.0;
            long long best_key = -1;
            for (int st = tid; st < nb; st += kTThreads) {
                for (int di = 0; di < a.n_dur; ++di) {
                    const int W = a.dur_bins[di];
                    const double* gg = g + a.tmpl_off[di];
                    const double g0 = gg[0], g00 = __dmul_rn(g0, g0);
                    const double2 e0 = v[st];
                    double num = __dmul_rn(g0, e0.x);
                    double cwg = __dmul_rn(g0, e0.y);
                    double den = __dmul_rn(g00, e0.y);
                    for (int k = 1; k < W; ++k) {
                        const double gk = gg[k], gkk = __dmul_rn(gk, gk);
                        const double2 e = v[st + k];
                        num = __dadd_rn(num, __dmul_rn(gk, e.x));
                        cwg = __dadd_rn(cwg, __dmul_rn(gk, e.y));
                        den = __dadd_rn(den, __dmul_rn(gkk, e.y));
                    }
                    if (num < 0.0 && den > a.w_eps) {
                        const double de =
                            __dsub_rn(den, __ddiv_rn(__dmul_rn(cwg, cwg), cv.w_total));
                        if (de > __dmul_rn(a.den_rel, den)) {
                            const double sr = __ddiv_rn(__dmul_rn(num, num), de);
                            if (sr > 0.0)
                                tls_keep(best, best_key, best_depth, sr,
                                         ((long long)di << 32) | (long long)st,
                                         __ddiv_rn(-num, de));
                        }
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double osr = __shfl_down_sync(kTAll, best, o);
                const long long okey = __shfl_down_sync(kTAll, best_key, o);
                const double odep = __shfl_down_sync(kTAll, best_depth, o);
                tls_keep(best, best_key, best_depth, osr, okey, odep);
            }
            if (lane == 0) {
                s.red_sr[warp] = best;
                s.red_key[warp] = best_key;
                s.red_depth[warp] = best_depth;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < kTWarps; ++w)
                    tls_keep(best, best_key, best_depth, s.red_sr[w], s.red_key[w],
                             s.red_depth[w]);
                const double P = a.period[p0 + p];
                double o_sr = 0.0, o_depth = 0.0, o_dur = 0.0, o_t0 = 0.0;
                if (best_key >= 0) {
                    const int di = (int)(best_key >> 32);
                    const int st = (int)(best_key & 0xffffffffll);
                    if (di < a.n_dur) {
                        const double W = (double)a.dur_bins[di];
                        o_sr = best;
                        o_depth = best_depth;
                        o_dur = __dmul_rn(__ddiv_rn(W, (double)nb), P);
                        const double centre =
                            __ddiv_rn(__dadd_rn((double)st, __ddiv_rn(W, 2.0)), (double)nb);
                        o_t0 = __dmul_rn(__dsub_rn(centre, floor(centre)), P);
                    } else {
                        atomicOr(a.error_flag, TERR_DESC);
                    }
                }
                double* o = a.out + (int64_t)c * a.n_periods + p0 + p;
                o[0] = o_sr;
                o[a.out_stride] = o_depth;
                o[2 * a.out_stride] = o_dur;
                o[3 * a.out_stride] = o_t0;
            }
            __syncthreads();
        }
    }
}

}  // namespace

size_t tls_smem_bytes(int n_bins, int max_width, int tile, int n_tmpl) {
    return (size_t)tile * (size_t)(n_bins + max_width - 1) * sizeof(double2) +
           (size_t)tile * 4 * n_bins * sizeof(unsigned) + (size_t)n_tmpl * sizeof(double);
}

cudaError_t configure_tls(size_t smem) {
    return raise_smem_limit((const void*)tls_kernel, smem);
}

int tls_resident_ctas(size_t smem) {
    int n = 0;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tls_kernel, kTThreads, smem) ==
                   cudaSuccess
               ? n
               : 0;
}

cudaError_t launch_tls(const TlsArgs& args, int n_ctas, size_t smem, cudaStream_t stream) {
    tls_kernel<<<n_ctas, kTThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

}  // namespace blsb200
