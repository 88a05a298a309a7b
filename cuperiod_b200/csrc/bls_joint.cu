// Joint-ephemeris multi-band BLS search kernel (sm_100a): one box, one duration
// and one phase, shared by every band of a star (cuPeriod
// src/cuperiod/multiband/_bls_joint.py:412-507 for the sweep, 359-404 for the
// reported fields).
//
// A persistent grid of 1024-thread CTAs (one per SM: a six-band star's
// histograms take up to ~190 KB of shared memory) claims trial periods from a
// global counter.  Per period a CTA
//   1. folds every point of the star into its band's histogram (per bin a
//      16-byte record of the centred flux*weight and the weight, exact 64-bit
//      fixed point, added with native 32-bit shared atomics and carries -- or
//      in a per-CTA global slice when the bands do not fit); the bin is the
//      reference's, from the fast
//      fold where its margins prove it, else from the reference's IEEE chain;
//   2. applies the reference's wrap pad per band and turns each histogram into
//      prefix sums in place (every thread owns a run of bins of every band);
//   3. sweeps every (duration, start) box, boxes spread over all threads.
//      The threshold is a total some box certainly reaches (an FP32 lower
//      bound over a sample of boxes, raised by every FP64 total taken); an FP32
//      upper bound on each box's total (no FP64 division) discards every box
//      below it, and the few left are queued and evaluated as the reference
//      does: per band the admissibility floor and dip test, and the
//      band-ordered FP64 sum of depth^2 / (1/iv_in + 1/iv_out) (or
//      0.5 iv_in depth^2); the box with the largest total that any band
//      supports wins, the first in (duration index, start) order among equals;
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

constexpr int kJThreads = 1024;
constexpr int kJWarps = kJThreads / 32;
constexpr int kFlushRounds = 4;         // sweep rounds between evaluations of the queue
constexpr int kQueue = kFlushRounds * kJThreads;
constexpr unsigned kAll = 0xffffffffu;

enum : int { JERR_BIN = 1, JERR_DESC = 2 };

struct JointShared {
    JointBand band[kMaxJointBands];
    int32_t dur[kMaxDur];
    int32_t cum[kMaxDur + 1];           // boxes of the period before each duration
    longlong2 utot[kMaxJointBands];     // scan: totals of each warp's unit
    double red_v[kJWarps];
    long long red_key[kJWarps];
    int red_hit[kJWarps];
    double ep_snr[kMaxJointBands];
    double ep_depth[kMaxJointBands];
    int32_t queue[kQueue];              // boxes the screen kept, awaiting the FP64 total
    int qn;
    int next;
    uint32_t thr_bits;                  // a total some box of the period reaches, FP32 bits
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

__device__ __forceinline__ long long warp_inclusive(long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(kAll, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// In-place inclusive prefix sums of K histograms of L {Y, I} records (band k at
// rec + k*L) by the whole CTA.  Band k is cut into C chunks (C = 32 / K warps'
// worth when K <= 32, else 1), each chunk one warp's unit, a lane owning an odd
// run of R consecutive bins (so that the lanes' 16-byte records fall on
// distinct banks).  Pass 1 takes each unit's totals; pass 2 adds the band's
// earlier units, the lane's exclusive warp scan and the run itself.
__device__ void block_prefix(longlong2* rec, int K, int L, JointShared& s, int tid) {
    const int lane = tid & 31, warp = tid >> 5;
    const int C = K <= kJWarps ? kJWarps / K : 1;
    const int CL = (L + C - 1) / C;
    const int R = ((CL + 31) / 32) | 1;
    const int units = K * C;
    for (int u = warp; u < units; u += kJWarps) {
        const int k = u / C, c0 = (u % C) * CL, c1 = min(c0 + CL, L);
        const int r0 = min(c0 + lane * R, c1), r1 = min(r0 + R, c1);
        const longlong2* x = rec + (size_t)k * L;
        long long ry = 0, ri = 0;
        for (int j = r0; j < r1; ++j) {
            const longlong2 e = x[j];
            ry += e.x;
            ri += e.y;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ry += __shfl_xor_sync(kAll, ry, o);
            ri += __shfl_xor_sync(kAll, ri, o);
        }
        if (lane == 0) s.utot[u] = make_longlong2(ry, ri);
    }
    __syncthreads();
    for (int u = warp; u < units; u += kJWarps) {
        const int k = u / C, c0 = (u % C) * CL, c1 = min(c0 + CL, L);
        const int r0 = min(c0 + lane * R, c1), r1 = min(r0 + R, c1);
        longlong2* x = rec + (size_t)k * L;
        long long oy = 0, oi = 0;
        for (int q = k * C; q < u; ++q) {
            oy += s.utot[q].x;
            oi += s.utot[q].y;
        }
        long long ry = 0, ri = 0;
        for (int j = r0; j < r1; ++j) {
            const longlong2 e = x[j];
            ry += e.x;
            ri += e.y;
        }
        long long runy = oy + warp_inclusive(ry, lane) - ry;
        long long runi = oi + warp_inclusive(ri, lane) - ri;
        for (int j = r0; j < r1; ++j) {
            longlong2 e = x[j];
            runy += e.x;
            runi += e.y;
            e.x = runy;
            e.y = runi;
            x[j] = e;
        }
    }
    __syncthreads();
}

// The FP32 screen of box (n, d): an upper bound on the box's FP64 total (as
// exact_box computes it), -1 when no band can dip in the box, +inf when no
// bound can be formed.  Sums in units of 2^61 quanta: a = iv_in, y = y_in,
// t = y - ybar*a, whose sign is the dip's (depth = -S t / (a b), b = S - a), so
// the objective of a dipping band is at most (|t| + dt)^2 S / (a b)
// (likelihood: 0.5 (|t| + dt)^2 S^2 / (a b^2)) times c_n, dt covering the FP32
// conversions and products and the FP64 rounding that could flip a dip
// decision; the quotient's 2-ulp error and the sum's roundings are inside the
// final 2^-16.  A band whose box holds no weight (or all of it, when that fails
// the floor) is skipped as the FP64 test skips it.
//
// With LOWER, *lower receives a lower bound on the same total (0 when no band
// is certain to count): the bands that certainly pass both floor tests (a and
// b above twice the floor) and certainly dip (t < -dt) add at least
// (|t| - dt)^2 S / (a b) (likelihood: 0.5 (|t| - dt)^2 S^2 / (a b^2)), with a,
// b and S bounded on the unfavourable side; the other bands add >= 0.  The
// screen's threshold may be any such bound, since some box reaches it.
template <bool LOWER>
__device__ __forceinline__ float screen_bound(const longlong2* rec, const JointBand* band, int K,
                                              int L, int n, int d, int obj, float* lower) {
    float U = 0.0f, lo = 0.0f;
    bool maybe = false, unbounded = false;
    for (int k = 0; k < K; ++k) {
        const longlong2 e0 = rec[k * L + n], e1 = rec[k * L + n + d];
        const long long qi = e1.y - e0.y;
        const JointBand& b = band[k];
        if (qi == 0 || (qi == b.qi_total && b.full_skip)) continue;
        const float a = __ll2float_rn(qi) * 0x1p-61f;
        const float y = __ll2float_rn(e1.x - e0.x) * 0x1p-61f;
        const float t = fmaf(-b.ybar_n, a, y);
        const float dt =
            0x1p-20f * (fabsf(y) + fabsf(b.ybar_n) * (a + 0x1p-20f * b.s_n)) + 0x1p-100f;
        if (t > dt) continue;           // the box is certainly brighter: no dip
        maybe = true;
        const float a_lo = a * (1.0f - 0x1p-20f);
        const float b_lo = b.s_n - a - 0x1p-20f * b.s_n;
        if (LOWER && t < -dt && a_lo > 2.0f * b.floor_n && b_lo > 2.0f * b.floor_n) {
            const float tl = fabsf(t) - dt;
            const float s_lo = b.s_n * (1.0f - 0x1p-20f);
            const float a_hi = a * (1.0f + 0x1p-20f);
            const float b_hi = b.s_n - a + 0x1p-19f * b.s_n;
            const float dl = obj == 0 ? a_hi * b_hi : a_hi * b_hi * b_hi;
            if (dl > 0x1p-100f && dl < 0x1p100f) {
                const float nl = obj == 0 ? tl * tl * s_lo : 0.5f * tl * tl * s_lo * s_lo;
                lo = fmaf(__fdividef(nl, dl), b.c_n, lo);
            }
        }
        const float den = obj == 0 ? a_lo * b_lo : a_lo * b_lo * b_lo;
        // __fdividef needs a normal denominator below 2^126
        if (!(a_lo > 0.0f) || !(b_lo > 0.0f) || !(den > 0x1p-100f)) {
            unbounded = true;
            if (!LOWER) break;
            continue;
        }
        const float ta = fabsf(t) + dt;
        const float num = obj == 0 ? ta * ta * b.s_n : 0.5f * ta * ta * b.s_n * b.s_n;
        U = fmaf(__fdividef(num, den), b.c_n, U);
    }
    if (LOWER) {
        const float r = lo * (1.0f - 0x1p-16f);
        *lower = r < 0x1p126f ? r : 0.0f;
    }
    if (unbounded) return CUDART_INF_F;
    return maybe ? U * (1.0f + 0x1p-16f) : -1.0f;
}

// Duration index of box bx: the last di with cum[di] <= bx.
__device__ __forceinline__ int box_duration(const int32_t* cum, int bx) {
    int di = 0;
    while (bx >= cum[di + 1]) ++di;
    return di;
}

// The reference's box total (_bls_joint.py:474-493) on the exact sums.
__device__ __forceinline__ void exact_box(const longlong2* rec, const JointBand* band, int K,
                                          int L, int n, int d, int obj, double& total,
                                          int& hit) {
    total = 0.0;
    hit = 0;
    for (int k = 0; k < K; ++k) {
        const longlong2 e0 = rec[k * L + n], e1 = rec[k * L + n + d];
        const JointBand& b = band[k];
        const double y_in = __dmul_rn(__ll2double_rn(e1.x - e0.x), b.y_unit);
        const double iv_in = __dmul_rn(__ll2double_rn(e1.y - e0.y), b.i_unit);
        const double iv_out = __dsub_rn(b.sum_ivar, iv_in);
        if (iv_in < b.ivar_floor || iv_out < b.ivar_floor) continue;
        const double yin = __ddiv_rn(y_in, iv_in);
        const double yout = __ddiv_rn(__dsub_rn(b.sum_y, y_in), iv_out);
        if (!(yout >= yin)) continue;
        const double depth = __dsub_rn(yout, yin);
        hit = 1;
        const double term =
            obj == 0 ? __ddiv_rn(__dmul_rn(depth, depth),
                                 __dadd_rn(__ddiv_rn(1.0, iv_in), __ddiv_rn(1.0, iv_out)))
                     : __dmul_rn(__dmul_rn(__dmul_rn(0.5, iv_in), depth), depth);
        total = __dadd_rn(total, term);
    }
}

template <bool SMEM>
__global__ void __launch_bounds__(kJThreads, 1) joint_kernel(JointArgs a) {
    extern __shared__ __align__(16) unsigned char joint_dyn[];
    __shared__ JointShared s;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int K = a.n_bands;
    for (int k = tid; k < K; k += kJThreads) s.band[k] = a.bands[k];
    long long* hist = SMEM ? reinterpret_cast<long long*>(joint_dyn)
                           : a.scratch + (size_t)blockIdx.x * 2 * K * a.hist_stride;
    longlong2* rec = reinterpret_cast<longlong2*>(hist);
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
        if (tid < seg.n_dur) s.dur[tid] = a.dur_bins[seg.dur_off + tid];
        for (int i = tid; i < 2 * K * L; i += kJThreads) hist[i] = 0;
        __syncthreads();
        if (tid == 0) {
            // boxes per duration in sweep order (466-473: the widths the period admits)
            int c = 0;
            for (int di = 0; di < seg.n_dur; ++di) {
                s.cum[di] = c;
                const int d = s.dur[di];
                if (d < seg.width && d < nb) c += nb - d + 1;
            }
            s.cum[seg.n_dur] = c;
            s.thr_bits = 0u;
            s.qn = 0;
        }

        // 1. fold (_bls_joint.py:436-451): every point of the star into its band
        const double bin = seg.bin_duration;
        const bool fast = seg.fast_fold != 0;
        const double f = a.freq[p];
        const uint32_t S = a.scale[p];
        const int fb = seg.frac_bits;
        const uint32_t fmask = (1u << fb) - 1u, mu = seg.margin_u, mphi = seg.margin_phi;
        const uint32_t fr_span = (1u << fb) - 2u * mu, phi_span = 0u - 2u * mphi;
        for (int j = tid; j < a.n_points; j += kJThreads) {
            const int k = a.band_of[j];
            const double x = a.tau[j];
            int ind = fast ? fold_fast(x, f, S, fb, fmask, mu, fr_span, mphi, phi_span) : -1;
            if (ind < 0) ind = fold_exact(x, P, bin, seg.width);
            if (ind > nb) {
                atomicOr(a.error_flag, JERR_BIN);
                continue;
            }
            unsigned* r = reinterpret_cast<unsigned*>(hist + 2 * (k * L + ind));
            add_i64(r, a.qy[j]);
            add_i64(r + 2, a.qi[j]);
        }
        __syncthreads();

        // 2. wrap pad (452-459), in the reference's order, then prefix sums (460-465)
        const int os = seg.oversample;
        if (tid < K) {
            longlong2* r = rec + tid * L;
            for (int o = 0; o < os; ++o) {
                int dst = nb - os + o;
                dst = dst < 0 ? 0 : (dst > seg.width - 1 ? seg.width - 1 : dst);
                r[dst] = r[1 + o];
            }
        }
        __syncthreads();
        block_prefix(rec, K, L, s, tid);

        // 3. the sweep (466-496): box b of the period is start n of duration di,
        // boxes in (di, n) order; a thread's boxes come in that order, so strict
        // '>' keeps the first
        double best = -CUDART_INF;
        long long best_key = 0;
        int hit_any = 0;
        const int n_boxes = s.cum[seg.n_dur];
        if (a.screen != 0) {
            // every box through the FP32 screen; the boxes it keeps are queued
            // and their FP64 totals taken every kFlushRounds rounds with full
            // warps.  The threshold starts at the largest lower bound of the
            // first round's boxes and rises with every FP64 total taken.  Ties
            // go to the smaller (duration index, start) key, the reference's
            // first-wins order, whatever the order of evaluation.
            int di = 0, round = 0;
            for (int base = 0; base < n_boxes; base += kJThreads, ++round) {
                const int bx = base + tid;
                bool keep = false;
                if (round == 0) {
                    float u = -1.0f, lo = 0.0f;
                    if (bx < n_boxes) {
                        while (bx >= s.cum[di + 1]) ++di;
                        u = screen_bound<true>(rec, s.band, K, L, bx - s.cum[di], s.dur[di],
                                               a.obj_flag, &lo);
                        if (lo > 0.0f) atomicMax(&s.thr_bits, __float_as_uint(lo));
                    }
                    __syncthreads();
                    keep = bx < n_boxes && !(u < __uint_as_float(s.thr_bits));
                } else if (bx < n_boxes) {
                    while (bx >= s.cum[di + 1]) ++di;
                    const float thr =
                        __uint_as_float(*reinterpret_cast<volatile uint32_t*>(&s.thr_bits));
                    keep = !(screen_bound<false>(rec, s.band, K, L, bx - s.cum[di], s.dur[di],
                                                 a.obj_flag, nullptr) < thr);
                }
                const unsigned m = __ballot_sync(kAll, keep);
                if (m) {
                    const int leader = __ffs(m) - 1;
                    int pos = 0;
                    if (lane == leader) pos = atomicAdd(&s.qn, __popc(m));
                    pos = __shfl_sync(kAll, pos, leader);
                    if (keep) s.queue[pos + __popc(m & ((1u << lane) - 1u))] = bx;
                }
                if ((round + 1) % kFlushRounds == 0 || base + kJThreads >= n_boxes) {
                    __syncthreads();
                    const int q = s.qn;
                    for (int i = tid; i < q; i += kJThreads) {
                        const int qb = s.queue[i];
                        const int dq = box_duration(s.cum, qb);
                        const int n = qb - s.cum[dq];
                        double total;
                        int hit;
                        exact_box(rec, s.band, K, L, n, s.dur[dq], a.obj_flag, total, hit);
                        if (hit) {
                            keep_better(best, best_key, hit_any, total,
                                        ((long long)dq << 32) | (long long)n, 1);
                            // totals are >= 0: FP32 bit patterns order as the values
                            atomicMax(&s.thr_bits, __float_as_uint(__double2float_rd(total)));
                        }
                    }
                    __syncthreads();
                    if (tid == 0) s.qn = 0;
                    __syncthreads();
                }
            }
        } else {
            // every box in FP64, a thread's boxes in sweep order (strict '>'
            // keeps the first)
            int di = 0;
            for (int bx = tid; bx < n_boxes; bx += kJThreads) {
                while (bx >= s.cum[di + 1]) ++di;
                const int n = bx - s.cum[di];
                double total;
                int hit;
                exact_box(rec, s.band, K, L, n, s.dur[di], a.obj_flag, total, hit);
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

        // 4. the reported fields (_finish, 359-404), by warp 0: the winning box
        // over the warps' winners, band k's depth and SNR there by lane k (and
        // k + 32), then the band-ordered sum by lane 0
        if (warp == 0) {
            double v = s.red_v[lane];
            long long key = s.red_key[lane];
            int found = s.red_hit[lane];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(kAll, v, o);
                const long long ok = __shfl_xor_sync(kAll, key, o);
                const int oh = __shfl_xor_sync(kAll, found, o);
                keep_better(v, key, found, ov, ok, oh);
            }
            const int bn = (int)(key & 0xffffffffll);
            const int bd = found ? s.dur[(int)(key >> 32)] : 0;
            for (int k = lane; found && k < K; k += 32) {
                const longlong2 e0 = rec[k * L + bn], e1 = rec[k * L + bn + bd];
                const JointBand& b = s.band[k];
                const double y_in = __dmul_rn(__ll2double_rn(e1.x - e0.x), b.y_unit);
                const double iv_in = __dmul_rn(__ll2double_rn(e1.y - e0.y), b.i_unit);
                const double iv_out = __dsub_rn(b.sum_ivar, iv_in);
                const bool ok = iv_in >= b.ivar_floor && iv_out >= b.ivar_floor;
                const double safe_in = ok ? iv_in : 1.0;
                const double safe_out = ok ? iv_out : 1.0;
                const double yin = __ddiv_rn(y_in, safe_in);
                const double yout = __ddiv_rn(__dsub_rn(b.sum_y, y_in), safe_out);
                const bool dip = ok && yout >= yin;
                const double dd = __dsub_rn(yout, yin);
                s.ep_depth[k] = dip ? dd : 0.0;
                s.ep_snr[k] =
                    dip ? __ddiv_rn(dd, __dsqrt_rn(__dadd_rn(__ddiv_rn(1.0, safe_in),
                                                             __ddiv_rn(1.0, safe_out))))
                        : 0.0;
            }
            __syncwarp();
            if (lane == 0) {
                double f_power = 0.0, f_depth = 0.0, f_snr = 0.0, f_dur = 0.0, f_t0 = 0.0,
                       f_band = 0.0;
                if (found) {
                    double power = 0.0;
                    int top = 0;
                    for (int k = 0; k < K; ++k) {
                        const double snr = s.ep_snr[k];
                        power = __dadd_rn(power, __dmul_rn(snr, snr));
                        if (snr > s.ep_snr[top]) top = k;   // np.argmax: the first largest
                    }
                    const double duration = __dmul_rn((double)bd, bin);
                    const double mid =
                        __dadd_rn(__dmul_rn((double)bn, bin), __dmul_rn(0.5, duration));
                    f_power = power;
                    f_depth = s.ep_depth[top];
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
        }
        __syncthreads();
    }
}

}  // namespace

size_t joint_static_smem() { return sizeof(JointShared); }

cudaError_t configure_joint(size_t smem) {
    return raise_smem_limit((const void*)joint_kernel<true>, smem);
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
