// Joint-ephemeris multi-band BLS search kernel (sm_100a): one box, one duration
// and one phase, shared by every band of a star (cuPeriod
// src/cuperiod/multiband/_bls_joint.py:412-507 for the sweep, 359-404 for the
// reported fields).
//
// A persistent grid of CTAs claims trial periods from a global counter.  Per
// period a CTA
//   1. folds every band's points into that band's two histograms (centred
//      flux*weight and weight, exact 64-bit fixed point, atomics in shared
//      memory -- or in a per-CTA global slice when the bands do not fit) with
//      the reference's IEEE bin chain;
//   2. applies the reference's wrap pad per band and turns each histogram into
//      prefix sums in place, one warp per array;
//   3. sweeps every (duration, start) box: per band the reference's admissibility
//      floor and dip test, and the band-ordered FP64 sum of depth^2 /
//      (1/iv_in + 1/iv_out) (or 0.5 iv_in depth^2); the box with the largest
//      total that any band supports wins, the first in (duration index, start)
//      order among equals;
//   4. writes power (the sum of the bands' squared depth SNRs at that box), the
//      depth of the band with the largest SNR, depth_snr, duration, the
//      mid-transit time and that band's index.
// Box sums are exact differences of integer prefix sums, converted to FP64 with
// one rounding and scaled by a power of two; from there every operation is the
// reference's, each rounded on its own.
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "bls_device.h"
#include "bls_fold.cuh"
#include "bls_launch.h"

namespace blsb200 {
namespace {

constexpr int kJThreads = 256;
constexpr int kJWarps = kJThreads / 32;
constexpr unsigned kAll = 0xffffffffu;

enum : int { JERR_BIN = 1, JERR_DESC = 2 };

struct JointShared {
    JointBand band[kMaxJointBands];
    int32_t dur[kMaxDur];
    double red_v[kJWarps];
    long long red_key[kJWarps];
    int red_hit[kJWarps];
    int next;
};

// The box (its total and (duration index << 32 | start) key) that the reference's
// first-wins sweep keeps of two: the larger total, then the earlier box.
__device__ __forceinline__ void keep_better(double& v, long long& key, int& hit, double ov,
                                            long long okey, int ohit) {
    if (ohit && (!hit || ov > v || (ov == v && okey < key))) {
        v = ov;
        key = okey;
        hit = 1;
    }
}

// Inclusive prefix sum of one int64 array of L entries by one warp: each lane
// owns a run of R (odd, so the lanes' 8-byte words spread over the banks)
// consecutive entries.
__device__ __forceinline__ void warp_prefix(long long* v, int L, int lane) {
    int R = (L + 31) / 32;
    R |= 1;
    const int r0 = min(lane * R, L), r1 = min(r0 + R, L);
    long long s = 0;
    for (int i = r0; i < r1; ++i) s += v[i];
    long long inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(kAll, inc, o);
        if (lane >= o) inc += t;
    }
    long long run = inc - s;
    for (int i = r0; i < r1; ++i) {
        run += v[i];
        v[i] = run;
    }
}

template <bool SMEM>
__global__ void __launch_bounds__(kJThreads) joint_kernel(JointArgs a) {
    extern __shared__ __align__(16) unsigned char joint_dyn[];
    __shared__ JointShared s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int K = a.n_bands;
    for (int k = tid; k < K; k += kJThreads) s.band[k] = a.bands[k];
    long long* hist = SMEM ? reinterpret_cast<long long*>(joint_dyn)
                           : a.scratch + (size_t)blockIdx.x * 2 * K * a.hist_stride;
    for (;;) {
        if (tid == 0) s.next = atomicAdd(a.work_counter, 1);
        __syncthreads();
        const int64_t p = s.next;
        if (p >= a.n_periods) break;
        // the period's segment (segments are in grid order)
        int lo = 0, hi = a.n_segments - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.segments[mid].period_off <= p) lo = mid;
            else hi = mid - 1;
        }
        const JointSegment seg = a.segments[lo];
        const double P = a.period[p];
        const int nb = a.nbins[p];
        const int L = nb + 1;
        const bool bad = nb < seg.oversample + 1 || L > seg.hist_len || L > a.hist_stride ||
                         seg.n_dur > kMaxDur || nb > seg.width - 1;
        if (bad) {
            if (tid == 0) {
                atomicOr(a.error_flag, JERR_DESC);
                for (int f = 0; f < kJointFields; ++f) a.out[f * a.n_periods + p] = 0.0;
            }
            __syncthreads();
            continue;
        }
        for (int i = tid; i < seg.n_dur; i += kJThreads) s.dur[i] = a.dur_bins[seg.dur_off + i];
        for (int i = tid; i < 2 * K * L; i += kJThreads) hist[i] = 0;
        __syncthreads();

        // 1. fold (_bls_joint.py:436-451)
        const double bin = seg.bin_duration;
        for (int k = 0; k < K; ++k) {
            unsigned long long* Y = reinterpret_cast<unsigned long long*>(hist + 2 * k * L);
            unsigned long long* I = Y + L;
            const int64_t off = s.band[k].point_off;
            const int n = s.band[k].n_points;
            for (int j = tid; j < n; j += kJThreads) {
                const int ind = fold_exact(a.tau[off + j], P, bin, seg.width);
                if (ind > nb) {
                    atomicOr(a.error_flag, JERR_BIN);
                    continue;
                }
                atomicAdd(Y + ind, (unsigned long long)a.qy[off + j]);
                atomicAdd(I + ind, (unsigned long long)a.qi[off + j]);
            }
        }
        __syncthreads();

        // 2. wrap pad (452-459), in the reference's order, then prefix sums (460-465)
        const int os = seg.oversample;
        for (int k = tid; k < K; k += kJThreads) {
            long long* Y = hist + 2 * k * L;
            long long* I = Y + L;
            for (int o = 0; o < os; ++o) {
                int dst = nb - os + o;
                dst = dst < 0 ? 0 : (dst > seg.width - 1 ? seg.width - 1 : dst);
                Y[dst] = Y[1 + o];
                I[dst] = I[1 + o];
            }
        }
        __syncthreads();
        for (int arr = warp; arr < 2 * K; arr += kJWarps) warp_prefix(hist + arr * L, L, lane);
        __syncthreads();

        // 3. the sweep (466-496)
        double best = -CUDART_INF;
        long long best_key = 0;
        int hit_any = 0;
        for (int di = 0; di < seg.n_dur; ++di) {
            const int d = s.dur[di];
            if (d >= seg.width || d >= nb) continue;
            for (int n = tid; n <= nb - d; n += kJThreads) {
                double total = 0.0;
                int hit = 0;
                for (int k = 0; k < K; ++k) {
                    const long long* Y = hist + 2 * k * L;
                    const long long* I = Y + L;
                    const JointBand& b = s.band[k];
                    const double y_in = __dmul_rn(__ll2double_rn(Y[n + d] - Y[n]), b.y_unit);
                    const double iv_in = __dmul_rn(__ll2double_rn(I[n + d] - I[n]), b.i_unit);
                    const double iv_out = __dsub_rn(b.sum_ivar, iv_in);
                    if (iv_in < b.ivar_floor || iv_out < b.ivar_floor) continue;
                    const double yin = __ddiv_rn(y_in, iv_in);
                    const double yout = __ddiv_rn(__dsub_rn(b.sum_y, y_in), iv_out);
                    if (!(yout >= yin)) continue;
                    const double depth = __dsub_rn(yout, yin);
                    hit = 1;
                    const double term =
                        a.obj_flag == 0
                            ? __ddiv_rn(__dmul_rn(depth, depth),
                                        __dadd_rn(__ddiv_rn(1.0, iv_in), __ddiv_rn(1.0, iv_out)))
                            : __dmul_rn(__dmul_rn(__dmul_rn(0.5, iv_in), depth), depth);
                    total = __dadd_rn(total, term);
                }
                // a thread's boxes come in sweep order: strict '>' keeps the first
                if (hit && (!hit_any || total > best)) {
                    best = total;
                    best_key = ((long long)di << 32) | (long long)n;
                    hit_any = 1;
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_down_sync(kAll, best, o);
            const long long ok = __shfl_down_sync(kAll, best_key, o);
            const int oh = __shfl_down_sync(kAll, hit_any, o);
            keep_better(best, best_key, hit_any, ov, ok, oh);
        }
        if (lane == 0) {
            s.red_v[warp] = best;
            s.red_key[warp] = best_key;
            s.red_hit[warp] = hit_any;
        }
        __syncthreads();

        // 4. the reported fields (_finish, 359-404)
        if (tid == 0) {
            double v = s.red_v[0];
            long long key = s.red_key[0];
            int found = s.red_hit[0];
            for (int w = 1; w < kJWarps; ++w)
                keep_better(v, key, found, s.red_v[w], s.red_key[w], s.red_hit[w]);
            double f_power = 0.0, f_depth = 0.0, f_snr = 0.0, f_dur = 0.0, f_t0 = 0.0, f_band = 0.0;
            if (found) {
                const int bn = (int)(key & 0xffffffffll);
                const int bd = s.dur[(int)(key >> 32)];
                double power = 0.0, top_snr = 0.0, top_depth = 0.0;
                int top = -1;
                for (int k = 0; k < K; ++k) {
                    const long long* Y = hist + 2 * k * L;
                    const long long* I = Y + L;
                    const JointBand& b = s.band[k];
                    const double y_in = __dmul_rn(__ll2double_rn(Y[bn + bd] - Y[bn]), b.y_unit);
                    const double iv_in = __dmul_rn(__ll2double_rn(I[bn + bd] - I[bn]), b.i_unit);
                    const double iv_out = __dsub_rn(b.sum_ivar, iv_in);
                    const bool ok = iv_in >= b.ivar_floor && iv_out >= b.ivar_floor;
                    const double safe_in = ok ? iv_in : 1.0;
                    const double safe_out = ok ? iv_out : 1.0;
                    const double yin = __ddiv_rn(y_in, safe_in);
                    const double yout = __ddiv_rn(__dsub_rn(b.sum_y, y_in), safe_out);
                    const bool dip = ok && yout >= yin;
                    const double dd = __dsub_rn(yout, yin);
                    const double depth = dip ? dd : 0.0;
                    const double snr =
                        dip ? __ddiv_rn(dd, __dsqrt_rn(__dadd_rn(__ddiv_rn(1.0, safe_in),
                                                                 __ddiv_rn(1.0, safe_out))))
                            : 0.0;
                    power = __dadd_rn(power, __dmul_rn(snr, snr));
                    // np.argmax: the first largest
                    if (top < 0 || snr > top_snr) {
                        top = k;
                        top_snr = snr;
                        top_depth = depth;
                    }
                }
                const double duration = __dmul_rn((double)bd, bin);
                const double mid = __dadd_rn(__dmul_rn((double)bn, bin), __dmul_rn(0.5, duration));
                f_power = power;
                f_depth = top_depth;
                f_snr = __dsqrt_rn(power);
                f_dur = duration;
                f_t0 = __dadd_rn(fmod(mid, P), a.t_min);
                f_band = (double)top;
            }
            double* o = a.out + p;
            o[0] = f_power;
            o[a.n_periods] = f_depth;
            o[2 * a.n_periods] = f_snr;
            o[3 * a.n_periods] = f_dur;
            o[4 * a.n_periods] = f_t0;
            o[5 * a.n_periods] = f_band;
        }
        __syncthreads();
    }
}

}  // namespace

size_t joint_static_smem() { return sizeof(JointShared); }

cudaError_t configure_joint(size_t smem) {
    return cudaFuncSetAttribute(joint_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

int joint_resident_ctas(bool in_smem, size_t smem) {
    int n = 0;
    cudaError_t e = in_smem
        ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, joint_kernel<true>, kJThreads, smem)
        : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, joint_kernel<false>, kJThreads, 0);
    return e == cudaSuccess ? n : 0;
}

cudaError_t launch_joint(const JointArgs& args, bool in_smem, size_t smem, int n_ctas,
                         cudaStream_t stream) {
    if (in_smem)
        joint_kernel<true><<<n_ctas, kJThreads, smem, stream>>>(args);
    else
        joint_kernel<false><<<n_ctas, kJThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

}  // namespace blsb200
