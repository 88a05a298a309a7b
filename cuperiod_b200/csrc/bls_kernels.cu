// B200 box-least-squares search kernels (sm_100a).
//
// One persistent launch processes work items of (curve, segment, tile of up to
// kMaxTile consecutive trial periods).  Per item a CTA
//   1. folds every point of the curve into one shared-memory histogram per
//      period of the tile.  The phase bin is the reference's
//      w = x - P*floor(x/P); ind = int(w/bin) + 1   (cuPeriod
//      src/cuperiod/methods/_bls_core.py:369-376 / 536-538), computed by a fast
//      FP64 path -- q = x * RN(1/P) rounded onto a 2^-32 grid, then one 32-bit
//      multiply-high by P/bin -- whose result is used only when it is provably
//      the reference's (the scaled phase is further than the combined rounding
//      error from a cycle or bin edge); otherwise the reference's own IEEE chain
//      runs.  With one weight for every point the bin sums are exact integers
//      built with native 32-bit shared atomics only (64-bit and floating-point
//      shared atomics are emulated on sm_100): each point adds the unsigned low
//      13 bits and the signed high part of r_q (its centred flux*weight
//      quantised to 24-27 bits of the curve's largest, by its length) to two
//      words and 1 to the bin's count.  With per-point
//      weights the two sums stay FP64.  A lane holds 8 time-consecutive points
//      (the lanes of a warp 8 points apart, so their bins rarely collide);
//   2. per period: applies the reference's wrap pad (_bls_core.py:377-381),
//      turns the bins into prefix sums in place and writes an FP32 screen copy;
//   3. sweeps every (duration, start) box.  An FP32 bound on the box objective
//      -- maximising snr (or the log-likelihood) is maximising
//      t^2 / (iv_in iv_out) (or t^2 / (iv_in iv_out^2)) with t = y_in - ybar iv_in
//      -- discards every box that provably cannot be the period's best; the few
//      that remain are evaluated with the reference's FP64 formulas
//      (_bls_core.py:410-426) on the exact sums, and the winner is the first in
//      (duration index, start) order among equals, as in the reference;
//   4. writes the reference's seven per-period fields (_bls_core.py:443-460).
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include <algorithm>
#include <cfloat>
#include <map>
#include <mutex>
#include <utility>

#include "bls_device.h"
#include "bls_fold.cuh"
#include "bls_launch.h"

namespace blsb200 {
namespace {

constexpr int kThreads = kChunkThreads;
constexpr int kWarps = kThreads / 32;
constexpr int kPts = kChunkPts;
constexpr unsigned kFull = 0xffffffffu;
constexpr float kRel = 1.0f / 262144.0f;    // 2^-18: relative slack of FP32 key bounds
constexpr int kCasLimit = 1 << 16;          // retries of one FP64 shared add
constexpr int kNoBox = 1 << 29;             // duration slot past the last real duration
// WIDE: the FP32 screen holds weights scaled by 2^-13 (fixed-point weights are
// below 2^37 per point), the range of the FP64 mode's, so that the likelihood's
// iv_in * iv_out^2 stays finite in FP32
constexpr int kWideScreenShift = 13;

struct TileShared {
    WorkItem item;
    CurveDesc curve;
    SegmentDesc seg;
    double per[kMaxTile];
    double freq[kMaxTile];
    uint32_t scale[kMaxTile];
    int32_t nb[kMaxTile];
    alignas(16) int32_t dur[kMaxDur + 4];   // padded with kNoBox; read four at a time
    double win_v[kMaxTile];         // per period of the tile: the best box
    int32_t win_di[kMaxTile];
    int32_t win_n[kMaxTile];
    uint32_t tot_w[6][kWarps];      // integer prefix scan: per-warp totals of each word
    double tot_rd[kWarps];
    double tot_wd[kWarps];
    float red_f[kWarps];
    float red_t[kWarps];
    double red_v[kWarps];
    int red_di[kWarps];
    int red_n[kWarps];
    int red_ne[kWarps];             // GENERAL scan: last non-empty bin per warp
    int next;
    uint32_t thr_bits;              // the sweep's shared threshold (bits of a float >= 0)
};

// Shared-memory accesses by 32-bit shared-space address (the hot loops compute
// addresses in 32-bit arithmetic instead of converting generic pointers).
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
template <int OFF>
__device__ __forceinline__ void red_add_u32(uint32_t a, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0+%2], %1;" ::"r"(a), "r"(v), "n"(OFF) : "memory");
}
__device__ __forceinline__ uint32_t ld_u32(uint32_t a) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void st_u32(uint32_t a, uint32_t v) {
    asm volatile("st.shared.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ double ld_f64(uint32_t a) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void st_f64(uint32_t a, double v) {
    asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ float2 ld_f2(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
template <int OFF>
__device__ __forceinline__ float2 ld_f2_off(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2+%3];" : "=f"(v.x), "=f"(v.y) : "r"(a), "n"(OFF));
    return v;
}
__device__ __forceinline__ void st_f2(uint32_t a, float2 v) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}

// FP64 add to a shared-memory word by a bounded compare-and-swap loop in the
// shared state space.  The loop is lock-free (a failed swap means another thread
// succeeded); the bound only guards against the impossible and sets `flag`.
__device__ __forceinline__ void shared_add_f64(uint32_t addr, double v, int32_t* flag) {
    if (v == 0.0) return;
    unsigned long long old;
    asm volatile("ld.shared.u64 %0, [%1];" : "=l"(old) : "r"(addr) : "memory");
    for (int it = 0; it < kCasLimit; ++it) {
        const unsigned long long want = __double_as_longlong(__longlong_as_double(old) + v);
        unsigned long long seen;
        asm volatile("atom.shared.cas.b64 %0, [%1], %2, %3;"
                     : "=l"(seen) : "r"(addr), "l"(old), "l"(want) : "memory");
        if (seen == old) return;
        old = seen;
    }
    atomicExch(flag, 2);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// (v, di, n) is better than (w, dj, m): larger objective, then earlier
// (duration index, start) -- the reference's first-wins order.
__device__ __forceinline__ bool better(double v, int di, int n, double w, int dj, int m) {
    if (v > w) return true;
    if (v < w || !(v == w)) return false;
    return di < dj || (di == dj && n < m);
}

// Sums of one box inside and outside, in the reference's units: the reference
// forms the outside as sum_y - y_in and sum_ivar - iv_in; WIDE curves take them
// from the exact quantised totals instead (CurveDesc::rq_total).
struct BoxSums {
    double y_in, iv_in, y_out, iv_out;
};

// The reference's objective of one box (_bls_core.py:410-426); -inf when the box
// is not admissible.
__device__ __forceinline__ double box_objective(const BoxSums& s, const CurveDesc& c, int obj) {
    const double iv_out = s.iv_out;
    if (!(s.iv_in >= c.ivar_floor) || !(iv_out >= c.ivar_floor)) return -CUDART_INF;
    const double yin = s.y_in / s.iv_in;
    const double yout = s.y_out / iv_out;
    if (yout < yin) return -CUDART_INF;
    const double depth = yout - yin;
    if (obj == 0) return depth / sqrt(1.0 / s.iv_in + 1.0 / iv_out);
    return 0.5 * s.iv_in * depth * depth;
}

// Histogram layout of one period: one record per bin, prefix sums in place.
//  UNIFORM: {A, B, C}, 12 bytes -- sum of the low 13 bits of r_q, sum of its
//           signed high part, count (32-bit words);
//  GENERAL: {R, W}, 16 bytes -- FP64 sums of the scaled centred flux*weight and
//           of the scaled weight;
//  WIDE:    {R0, R1, R2, I0, I1, I2}, 24 bytes -- the three parts of the
//           fixed-point centred flux*weight and of the weight (32-bit words).
// A period's region is padded to 16 bytes.
template <int MODE>
__device__ __host__ constexpr int bin_bytes() {
    return MODE == MODE_UNIFORM ? 12 : (MODE == MODE_WIDE ? 24 : 16);
}
template <int MODE>
__device__ __host__ __forceinline__ size_t hist_period_bytes(int hl) {
    return ((size_t)hl * bin_bytes<MODE>() + 15) & ~size_t(15);
}

template <int MODE>
struct PointRegs {
    double x[kPts];
    uint32_t lo[MODE == MODE_UNIFORM ? kPts : 1], hi[MODE == MODE_UNIFORM ? kPts : 1];
    double rv[MODE == MODE_GENERAL ? kPts : 1], iv[MODE == MODE_GENERAL ? kPts : 1];
    long long rq[MODE == MODE_WIDE ? kPts : 1], iq[MODE == MODE_WIDE ? kPts : 1];
};

// WIDE: the three 32-bit parts of a fixed-point value (|v| < 2^37): low and
// middle 13 bits, and the signed high part.
__device__ __forceinline__ uint32_t wide_part(long long v, int k) {
    return k == 0 ? (uint32_t)(v & ((1ll << kWideBits) - 1))
                  : (k == 1 ? (uint32_t)((v >> kWideBits) & ((1ll << kWideBits) - 1))
                            : (uint32_t)(int32_t)(v >> (2 * kWideBits)));
}
// WIDE: the value of three prefix parts.
__device__ __forceinline__ long long wide_value(uint32_t p0, uint32_t p1, uint32_t p2) {
    return (long long)(int32_t)p2 * (1ll << (2 * kWideBits)) +
           (long long)p1 * (1ll << kWideBits) + (long long)p0;
}
template <int MODE>
__device__ __forceinline__ void add_point(uint32_t rec, const PointRegs<MODE>& p, int r,
                                          int32_t* flag);

template <int MODE, bool TAIL>
__device__ __forceinline__ void load_points(const BatchArgs& a, const CurveDesc& c, int base,
                                            PointRegs<MODE>& p) {
    const int tid = threadIdx.x;
    const double* __restrict__ tau = a.tau + c.point_off;
#pragma unroll
    for (int r = 0; r < kPts; ++r) {
        const int j = base + r * kThreads + tid;
        const bool ok = !TAIL || j < c.n_points;
        p.x[r] = ok ? __ldg(tau + j) : -1.0;
        if (MODE == MODE_UNIFORM) {
            const uint32_t w = ok ? __ldg(a.pay_r + c.point_off + j) : 0u;
            p.lo[r] = w & 0xffffu;
            p.hi[r] = (uint32_t)((int32_t)w >> 16);    // signed high part
        } else if (MODE == MODE_WIDE) {
            const long long* rq = reinterpret_cast<const long long*>(a.r64) + c.point_off;
            const long long* iq = reinterpret_cast<const long long*>(a.iv64) + c.point_off;
            p.rq[r] = ok ? __ldg(rq + j) : 0ll;
            p.iq[r] = ok ? __ldg(iq + j) : 0ll;
        } else {
            p.rv[r] = ok ? __ldg(a.r64 + c.point_off + j) : 0.0;
            p.iv[r] = ok ? __ldg(a.iv64 + c.point_off + j) : 0.0;
        }
    }
}

template <int MODE, bool TAIL>
__device__ __forceinline__ void fold_points(const TileShared& s, uint32_t hist_s,
                                            const PointRegs<MODE>& p, int pt, int hl,
                                            int32_t* flag) {
    const SegmentDesc& g = s.seg;
    const int fb = g.frac_bits;
    const uint32_t fmask = (1u << fb) - 1u;
    const uint32_t mu = g.margin_u;
    const uint32_t fr_span = (1u << fb) - 2u * mu;
    const uint32_t mphi = g.margin_phi;
    const uint32_t phi_span = 0u - 2u * mphi;
    const bool fast = g.fast_fold != 0;
    const double bin = g.bin_duration;
    const int width = g.width;
    const uint32_t pbytes = (uint32_t)hist_period_bytes<MODE>(hl);
    constexpr uint32_t kB = (uint32_t)bin_bytes<MODE>();
    for (int q = 0; q < pt; ++q) {
        const double f = s.freq[q];
        const uint32_t S = s.scale[q];
        const uint32_t hq = hist_s + (uint32_t)q * pbytes;
        if (!TAIL && fast) {
            // common case: every point's fast fold (fold_fast, inlined here) is
            // provably the reference's bin, and the records take their atomics
            // with no per-point test
            uint32_t rec[kPts];
            bool all_ok = true;
#pragma unroll
            for (int r = 0; r < kPts; ++r) {
                const double qm = __fma_rn(p.x[r], f, 1572864.0);
                const uint32_t phi = (uint32_t)__double2loint(qm);
                const uint32_t v = __umulhi(phi, S);
                all_ok &= ((phi - mphi) < phi_span) & (((v & fmask) - mu) < fr_span);
                rec[r] = hq + kB + (v >> fb) * kB;
            }
            if (all_ok) {
                if (MODE == MODE_UNIFORM) {
                    // a lane's points are consecutive in time, so dense curves in
                    // the wide-bin segments put several in one bin: each run of
                    // equal bins adds its exact sums once (low parts of at most 8
                    // points stay below 2^16), and lanes without a flush at a
                    // step sit out that step's atomics and their bank conflicts
                    uint32_t s_lo = p.lo[0], s_hi = p.hi[0], s_c = 1u;
#pragma unroll
                    for (int r = 1; r < kPts; ++r) {
                        if (rec[r] != rec[r - 1]) {
                            red_add_u32<0>(rec[r - 1], s_lo);
                            red_add_u32<4>(rec[r - 1], s_hi);
                            red_add_u32<8>(rec[r - 1], s_c);
                            s_lo = 0u;
                            s_hi = 0u;
                            s_c = 0u;
                        }
                        s_lo += p.lo[r];
                        s_hi += p.hi[r];
                        s_c += 1u;
                    }
                    red_add_u32<0>(rec[kPts - 1], s_lo);
                    red_add_u32<4>(rec[kPts - 1], s_hi);
                    red_add_u32<8>(rec[kPts - 1], s_c);
                } else {
#pragma unroll
                    for (int r = 0; r < kPts; ++r) add_point<MODE>(rec[r], p, r, flag);
                }
                continue;
            }
        }
        // 1. the fast fold of all points, straight-line (-1: near an edge, -2: skip)
        int ind[kPts];
        bool miss = false;
#pragma unroll
        for (int r = 0; r < kPts; ++r) {
            ind[r] = fast ? fold_fast(p.x[r], f, S, fb, fmask, mu, fr_span, mphi, phi_span) : -1;
            if (TAIL && p.x[r] < 0.0) ind[r] = -2;
            miss |= ind[r] == -1;
        }
        // 2. rare: the reference's IEEE chain for points near a cycle or bin edge
        if (miss) {
            const double P = s.per[q];
            const int nbq = s.nb[q];
#pragma unroll
            for (int r = 0; r < kPts; ++r) {
                if (ind[r] == -1) {
                    const int e = fold_exact(p.x[r], P, bin, width);
                    ind[r] = e > nbq ? -2 : e;        // a bin the reference never reads
                }
            }
        }
        // 3. accumulate: one record address per point feeds all its atomics
#pragma unroll
        for (int r = 0; r < kPts; ++r) {
            if (ind[r] < 0) continue;
            add_point<MODE>(hq + (uint32_t)ind[r] * (uint32_t)bin_bytes<MODE>(), p, r, flag);
        }
    }
}

// One point's contribution to its bin record.
template <int MODE>
__device__ __forceinline__ void add_point(uint32_t rec, const PointRegs<MODE>& p, int r,
                                          int32_t* flag) {
    if (MODE == MODE_UNIFORM) {
        red_add_u32<0>(rec, p.lo[r]);
        red_add_u32<4>(rec, p.hi[r]);
        red_add_u32<8>(rec, 1u);
    } else if (MODE == MODE_WIDE) {
        red_add_u32<0>(rec, wide_part(p.rq[r], 0));
        red_add_u32<4>(rec, wide_part(p.rq[r], 1));
        red_add_u32<8>(rec, wide_part(p.rq[r], 2));
        red_add_u32<12>(rec, wide_part(p.iq[r], 0));
        red_add_u32<16>(rec, wide_part(p.iq[r], 1));
        red_add_u32<20>(rec, wide_part(p.iq[r], 2));
    } else {
        shared_add_f64(rec, p.rv[r], flag);
        shared_add_f64(rec + 8, p.iv[r], flag);
    }
}

// WIDE: exact prefixes at bin i of the centred flux*weight and of the weight.
__device__ __forceinline__ long long wide_prefix_r(uint32_t hq, int i) {
    const uint32_t rec = hq + (uint32_t)i * 24u;
    return wide_value(ld_u32(rec), ld_u32(rec + 4), ld_u32(rec + 8));
}
__device__ __forceinline__ long long wide_prefix_i(uint32_t hq, int i) {
    const uint32_t rec = hq + (uint32_t)i * 24u + 12u;
    return wide_value(ld_u32(rec), ld_u32(rec + 4), ld_u32(rec + 8));
}

// Exact prefix of r_q at bin i from a UNIFORM record's two prefix words.
__device__ __forceinline__ long long prefix_r(uint32_t hq, int i) {
    const uint32_t rec = hq + (uint32_t)i * 12u;
    return (long long)(int32_t)ld_u32(rec + 4) * (1ll << kHalfBits) + (long long)ld_u32(rec);
}
__device__ __forceinline__ uint32_t prefix_c(uint32_t hq, int i) {
    return ld_u32(hq + (uint32_t)i * 12u + 8u);
}

// Exact sums of box (n, d) in the reference's units from one period's prefixes
// (hq: the period's region).
template <int MODE>
__device__ __forceinline__ BoxSums box_sums(uint32_t hq, const CurveDesc& cv, int n, int d);

// The reference's objective of box (n, d), out of line: the sweep reaches it
// rarely and keeps its own loop small.
template <int MODE>
__device__ __noinline__ double exact_objective(uint32_t hq, const CurveDesc* cv, int n, int d,
                                               int obj) {
    return box_objective(box_sums<MODE>(hq, *cv, n, d), *cv, obj);
}

template <int MODE>
__device__ __forceinline__ BoxSums box_sums(uint32_t hq, const CurveDesc& cv, int n, int d) {
    BoxSums b;
    if (MODE == MODE_UNIFORM) {
        const double cnt = (double)(prefix_c(hq, n + d) - prefix_c(hq, n));
        b.iv_in = cnt * cv.w_uniform;
        b.y_in = ldexp((double)(prefix_r(hq, n + d) - prefix_r(hq, n)), -cv.e_r) +
                 cv.center * cnt;
    } else if (MODE == MODE_WIDE) {
        const long long qi = wide_prefix_i(hq, n + d) - wide_prefix_i(hq, n);
        const long long qr = wide_prefix_r(hq, n + d) - wide_prefix_r(hq, n);
        b.iv_in = ldexp((double)qi, -cv.e_i);
        b.y_in = ldexp((double)qr, -cv.e_r) + cv.ybar * b.iv_in;
        b.iv_out = ldexp((double)(cv.iq_total - qi), -cv.e_i);
        b.y_out = ldexp((double)(cv.rq_total - qr), -cv.e_r) + cv.ybar * b.iv_out;
        return b;
    } else {
        const uint32_t r1 = hq + (uint32_t)(n + d) * 16u, r0 = hq + (uint32_t)n * 16u;
        b.iv_in = ldexp(ld_f64(r1 + 8) - ld_f64(r0 + 8), -cv.e_i);
        b.y_in = ldexp(ld_f64(r1) - ld_f64(r0), -cv.e_r) + cv.ybar * b.iv_in;
    }
    b.iv_out = cv.sum_ivar - b.iv_in;
    b.y_out = cv.sum_y - b.y_in;
    return b;
}

template <int MODE, int OBJ>
__global__ void __launch_bounds__(kThreads, MODE == MODE_UNIFORM ? 3 : 2)
    bls_search_kernel(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileShared s;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;

    for (;;) {
        __syncthreads();
        if (tid == 0) s.next = atomicAdd(a.work_counter, 1);
        __syncthreads();
        const int it = s.next;
        if (it >= a.n_items) break;
        if (tid == 0) {
            // one grid: the group is a launch parameter; several: a search
            WorkGroup gr = a.group0;
            if (a.n_groups > 1) {
                int glo = 0, ghi = a.n_groups;      // groups[glo].item_begin <= it
                while (ghi - glo > 1) {
                    const int mid = (glo + ghi) >> 1;
                    if (__ldg(&a.groups[mid].item_begin) <= it) glo = mid;
                    else ghi = mid;
                }
                gr = a.groups[glo];
            }
            const int local = it - gr.item_begin;
            const int r = local / gr.tiles_per_curve;
            const int j = local - r * gr.tiles_per_curve;
            const int32_t* tiles = a.seg_tiles + gr.tiles_begin;
            int lo = 0, hi = gr.n_segments;         // tiles[lo] <= j < tiles[hi]
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(tiles + mid) <= j) lo = mid;
                else hi = mid;
            }
            const int sg = gr.seg_begin + lo;
            const int cap = __ldg(a.seg_cap + sg);
            s.seg = a.segments[sg];
            WorkItem w;
            w.curve = __ldg(a.order + gr.order_begin + r);
            w.segment = sg;
            w.p_begin = (j - __ldg(tiles + lo)) * cap;
            w.p_count = min(cap, s.seg.n_periods - w.p_begin);
            s.item = w;
            s.curve = a.curves[w.curve];
        }
        __syncthreads();
        const int pt = s.item.p_count;
        const int hl = s.seg.hist_len;
        const int n_dur = s.seg.n_dur;
        if (pt < 1 || pt > kMaxTile || n_dur < 0 || n_dur > kMaxDur || hl < 2) {
            if (tid == 0) atomicExch(a.error_flag, 1);
            continue;
        }
        const int64_t g0 = s.seg.period_off + s.item.p_begin;
        if (tid < pt) {
            s.per[tid] = a.period[g0 + tid];
            s.freq[tid] = a.freq[g0 + tid];
            s.scale[tid] = a.scale[g0 + tid];
            s.nb[tid] = a.nbins[g0 + tid];
        }
        if (tid < kMaxDur + 4) s.dur[tid] = tid < n_dur ? a.dur_bins[s.seg.dur_off + tid] : kNoBox;
        __syncthreads();

        double* out = a.out + s.curve.out_off + g0;
        const int64_t ostride = a.out_stride;
        if (s.curve.skip || n_dur == 0) {       // nothing admissible anywhere
            if (tid < pt) {
                out[tid] = -CUDART_INF;
                for (int f = 1; f < kFields; ++f) out[f * ostride + tid] = 0.0;
            }
            continue;
        }

        // ---- 1. fold ---------------------------------------------------------
        const size_t pbytes = hist_period_bytes<MODE>(hl);
        const uint32_t smem_s = smem_addr(smem);
        {
            const int n16 = (int)((pt * pbytes) / 16);
            uint4* z = reinterpret_cast<uint4*>(smem);
            for (int i = tid; i < n16; i += kThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
        }
        __syncthreads();
        {
            const int n = s.curve.n_points;
            int base = 0;
            for (; base + kChunk <= n; base += kChunk) {
                PointRegs<MODE> p;
                load_points<MODE, false>(a, s.curve, base, p);
                fold_points<MODE, false>(s, smem_s, p, pt, hl, a.error_flag);
            }
            if (base < n) {
                PointRegs<MODE> p;
                load_points<MODE, true>(a, s.curve, base, p);
                fold_points<MODE, true>(s, smem_s, p, pt, hl, a.error_flag);
            }
        }
        __syncthreads();

        // ---- 2-3. per period: pad, prefix, sweep, reduce ------------------------
        const size_t hist_bytes = (size_t)pt * pbytes;               // multiple of 16
        const uint32_t scr_s = smem_s + (uint32_t)hist_bytes;        // FP32 screen copy
        const CurveDesc& cv = s.curve;
        constexpr int obj = OBJ;          // 0 snr, 1 log-likelihood
        const int e_r = cv.e_r, e_i = cv.e_i;
        const int o = s.seg.oversample;
        constexpr uint32_t kRec = (uint32_t)bin_bytes<MODE>();
        constexpr int kNW = MODE == MODE_UNIFORM ? 3 : (MODE == MODE_WIDE ? 6 : 1);   // words

        for (int q = 0; q < pt; ++q) {
            const int nb = s.nb[q];
            const int L = nb + 1;
            const uint32_t hq = smem_s + (uint32_t)(q * pbytes);
            auto copy_bin = [&](int dst, int src) {
                if (dst >= 0 && dst < s.seg.width && dst < hl && src < hl) {
                    const uint32_t rd = hq + (uint32_t)dst * kRec, rs = hq + (uint32_t)src * kRec;
                    if (MODE != MODE_GENERAL) {
#pragma unroll
                        for (int w = 0; w < kNW; ++w) st_u32(rd + 4 * w, ld_u32(rs + 4 * w));
                    } else {
                        st_f64(rd, ld_f64(rs));
                        st_f64(rd + 8, ld_f64(rs + 8));
                    }
                }
            };

            // wrap pad: bins 1..o copied to nb-o..nb-1 (_bls_core.py:377-381).  When
            // the two ranges overlap one thread copies in the reference's order;
            // otherwise the warp that owns each destination copies it in pass 1
            // (the source bins are not written before pass 2).
            const bool overlap = nb - o <= o;
            if (overlap) {
                if (tid == 0)
                    for (int k = 0; k < o; ++k) copy_bin(nb - o + k, 1 + k);
                __syncthreads();
            }

            // prefix scan.  Lane `lane` of warp `warp` owns K consecutive bins from
            // (warp * 32 + lane) * K, K odd so that the lanes' 12-byte records sit
            // in distinct banks.  Pass 1: each lane sums its bins, the warp scans
            // the 32 lane totals once and publishes its own total.
            const int K = ((L + kThreads - 1) / kThreads) | 1;
            const int lo_i = warp * 32 * K;
            const int hi_i = min(L, lo_i + 32 * K);
            const int l0 = min(L, lo_i + lane * K), l1 = min(L, l0 + K);
            if (tid == 0) s.thr_bits = 0u;      // every warp left the last sweep
            if (!overlap) {
                for (int k = lane; k < o; k += 32) {
                    const int dst = nb - o + k;
                    if (dst >= lo_i && dst < hi_i) copy_bin(dst, 1 + k);
                }
                __syncwarp();
            }
            uint32_t ex[kNW];                   // this lane's exclusive offsets in the warp
#pragma unroll
            for (int w = 0; w < kNW; ++w) ex[w] = 0u;
            double er = 0.0, ew = 0.0;
            // GENERAL: the lane's leading empty bins and its last non-empty bin
            // (the FP64 prefix of a run of empty bins is made exactly constant)
            int lead = 0, last_ne = -1;
            {
                uint32_t u[kNW];
#pragma unroll
                for (int w = 0; w < kNW; ++w) u[w] = 0u;
                double ur = 0.0, uw = 0.0;
                for (int i = l0; i < l1; ++i) {
                    const uint32_t rec = hq + (uint32_t)i * kRec;
                    if (MODE != MODE_GENERAL) {
#pragma unroll
                        for (int w = 0; w < kNW; ++w) u[w] += ld_u32(rec + 4 * w);
                    } else {
                        const double br = ld_f64(rec), bw = ld_f64(rec + 8);
                        ur += br;
                        uw += bw;
                        const bool empty = (br == 0.0) & (bw == 0.0);
                        if (!empty) last_ne = i;
                        else if (last_ne < 0) ++lead;
                    }
                }
                if (MODE != MODE_GENERAL) {
                    // 32-bit words added modulo 2^32; every prefix fits its word
                    uint32_t in[kNW];
#pragma unroll
                    for (int w = 0; w < kNW; ++w) in[w] = u[w];
#pragma unroll
                    for (int k = 1; k < 32; k <<= 1) {
#pragma unroll
                        for (int w = 0; w < kNW; ++w) {
                            const uint32_t x = __shfl_up_sync(kFull, in[w], k);
                            if (lane >= k) in[w] += x;
                        }
                    }
#pragma unroll
                    for (int w = 0; w < kNW; ++w) {
                        ex[w] = in[w] - u[w];
                        if (lane == 31) s.tot_w[w][warp] = in[w];
                    }
                } else {
                    double ir = ur, iw = uw;
#pragma unroll
                    for (int k = 1; k < 32; k <<= 1) {
                        const double xr = __shfl_up_sync(kFull, ir, k);
                        const double xw = __shfl_up_sync(kFull, iw, k);
                        if (lane >= k) { ir += xr; iw += xw; }
                    }
                    // the lane's offset as the sum of the lanes before it
                    er = __shfl_up_sync(kFull, ir, 1);
                    ew = __shfl_up_sync(kFull, iw, 1);
                    if (lane == 0) { er = 0.0; ew = 0.0; }
                    if (lane == 31) { s.tot_rd[warp] = ir; s.tot_wd[warp] = iw; }
                    // last non-empty bin before this lane: exclusive max-scan
                    int im = last_ne;
#pragma unroll
                    for (int k = 1; k < 32; k <<= 1) {
                        const int x = __shfl_up_sync(kFull, im, k);
                        if (lane >= k) im = max(im, x);
                    }
                    if (lane == 31) s.red_ne[warp] = im;
                    last_ne = __shfl_up_sync(kFull, im, 1);
                    if (lane == 0) last_ne = -1;
                }
            }
            __syncthreads();
            if (MODE == MODE_GENERAL)
                for (int w = 0; w < warp; ++w) last_ne = max(last_ne, s.red_ne[w]);
            // pass 2: the lane walks its bins again from its offset, writes the
            // prefix in place and the FP32 screen copy {t prefix, weight prefix}
            float tmax = 0.0f;
            {
                uint32_t run[kNW];
#pragma unroll
                for (int w = 0; w < kNW; ++w) run[w] = ex[w];
                double rr = er, rw = ew;
                for (int wp = 0; wp < warp; ++wp) {
                    if (MODE != MODE_GENERAL) {
#pragma unroll
                        for (int w = 0; w < kNW; ++w) run[w] += s.tot_w[w][wp];
                    } else {
                        rr += s.tot_rd[wp];
                        rw += s.tot_wd[wp];
                    }
                }
                const float cfrac = (float)cv.center_frac;
                for (int i = l0; i < l1; ++i) {
                    const uint32_t rec = hq + (uint32_t)i * kRec;
                    float tf, wf, tm = 0.0f;
                    if (MODE != MODE_GENERAL) {
#pragma unroll
                        for (int w = 0; w < kNW; ++w) {
                            run[w] += ld_u32(rec + 4 * w);
                            st_u32(rec + 4 * w, run[w]);
                        }
                        if (MODE == MODE_UNIFORM) {
                            // the screen's t is centred by ybar itself: the stored
                            // prefix minus center_frac per point, in FP32.  tf is
                            // within 2^-23 tm of the exact value (pf and tf round
                            // once each, cf <= 2^16 twice), so a box's t is within
                            // 1.5 * 2^-22 of the largest tm, inside Et
                            const float pf = (float)((long long)(int32_t)run[1] *
                                                         (1ll << kHalfBits) +
                                                     (long long)run[0]);
                            const float cf = cfrac * (float)run[2];
                            tf = pf - cf;
                            tm = fmaxf(fabsf(pf), fabsf(tf)) + fabsf(cf);
                            wf = (float)run[2];
                        } else {
                            tf = (float)wide_value(run[0], run[1], run[2]);
                            wf = (float)ldexp((double)wide_value(run[3], run[4], run[5]),
                                              -kWideScreenShift);
                        }
                    } else {
                        rr += ld_f64(rec);
                        rw += ld_f64(rec + 8);
                        st_f64(rec, rr);
                        st_f64(rec + 8, rw);
                        tf = (float)rr;
                        wf = (float)rw;
                    }
                    st_f2(scr_s + (uint32_t)i * 8u, make_float2(tf, wf));
                    tmax = fmaxf(tmax, MODE == MODE_UNIFORM ? tm : fabsf(tf));
                }
                tmax = warp_max(tmax);
                if (lane == 0) s.red_t[warp] = tmax;
            }
            // sentinel records past the last bin: t = NaN fails every screen
            for (int i = L + tid; i < L + kScreenPad; i += kThreads)
                st_f2(scr_s + (uint32_t)i * 8u, make_float2(CUDART_NAN_F, 0.0f));
            __syncthreads();
            if (MODE == MODE_GENERAL) {
                // The lanes' partial sums associate differently from one running
                // sum, so at a lane boundary an empty bin could move the FP64
                // prefix by a rounding.  The reference's running sum keeps it
                // exactly constant, which makes boxes that differ only by empty
                // end bins tie exactly (first wins); copy the prefix of the last
                // non-empty bin into this lane's leading empty bins.
                if (lead > 0 && last_ne >= 0) {
                    const uint32_t rs = hq + (uint32_t)last_ne * kRec;
                    const double pr = ld_f64(rs), pw = ld_f64(rs + 8);
                    for (int i = l0; i < l0 + lead; ++i) {
                        const uint32_t rec = hq + (uint32_t)i * kRec;
                        st_f64(rec, pr);
                        st_f64(rec + 8, pw);
                        st_f2(scr_s + (uint32_t)i * 8u, make_float2((float)pr, (float)pw));
                    }
                }
                __syncthreads();
            }
            tmax = 0.0f;
#pragma unroll
            for (int w = 0; w < kWarps; ++w) tmax = fmaxf(tmax, s.red_t[w]);

            auto iv_prefix = [&](int i) -> double {
                return MODE == MODE_UNIFORM ? (double)prefix_c(hq, i) * cv.w_uniform
                       : MODE == MODE_WIDE  ? ldexp((double)wide_prefix_i(hq, i), -e_i)
                                            : ldexp(ld_f64(hq + (uint32_t)i * 16u + 8u), -e_i);
            };
            auto exact = [&](int n, int d) -> double {
                return exact_objective<MODE>(hq, &cv, n, d, obj);
            };
            if (a.debug_prefix != nullptr && q == 0) {   // test hook: this period's prefixes
                for (int i = tid; i < L; i += kThreads) {
                    const double r_i =
                        MODE == MODE_UNIFORM ? ldexp((double)prefix_r(hq, i), -e_r)
                        : MODE == MODE_WIDE  ? ldexp((double)wide_prefix_r(hq, i), -e_r)
                                             : ldexp(ld_f64(hq + (uint32_t)i * 16u), -e_r);
                    a.debug_prefix[i] =
                        r_i + (MODE == MODE_UNIFORM ? cv.center * (double)prefix_c(hq, i)
                                                    : cv.ybar * iv_prefix(i));
                    a.debug_prefix[hl + i] = iv_prefix(i);
                }
            }

            // ---- sweep: durations outer (the reference's order), two starts per lane ----
            // bound on the FP32 error of a box's t: 2^-21 of the largest prefix
            // (one rounding per prefix, one per difference: 2^-22, 2x slack; one
            // weight: 1.5 * 2^-22 of the largest tm, 1.33x slack)
            const float Et = cv.exact_all ? CUDART_INF_F : tmax * (1.0f / 2097152.0f);
            const float Wt = MODE == MODE_UNIFORM ? (float)cv.n_points
                             : MODE == MODE_WIDE  ? (float)ldexp(cv.i_total, -kWideScreenShift)
                                                  : (float)cv.i_total;
            const float Ei = MODE == MODE_UNIFORM ? 0.0f : Wt * (1.0f / 2097152.0f);
            const float floor_q =
                MODE != MODE_UNIFORM
                    ? (float)ldexp(cv.ivar_floor,
                                   MODE == MODE_WIDE ? e_i - kWideScreenShift : e_i) * (1.0f + 1e-3f)
                    : 0.0f;

            bool has = false, ex_ok = false;
            int bn = 0, bdi = 0;
            float lb = -1.0f, hb = -1.0f;
            double ex_v = -CUDART_INF;
            float thr = 0.0f;
            const uint32_t thr_s = smem_addr(&s.thr_bits);

            // one box that passed the screen: keep it if it may be this lane's best
            auto consider = [&](int n, int di, int d, float t, float den_lo, float den_hi,
                                bool sure_valid) -> bool {
                const float th = fabsf(t) + Et;
                const float tl = fmaxf(fabsf(t) - Et, 0.0f);
                const float khi =
                    den_lo > 0.0f ? __fdividef(th * th, den_lo) * (1.0f + kRel) : CUDART_INF_F;
                const float klo = __fdividef(tl * tl, den_hi) * (1.0f - kRel);
                const bool sure = (t < -Et) & sure_valid & (klo > 0.0f);
                if (!has) {
                    if (sure) {
                        has = true; ex_ok = false; bn = n; bdi = di; lb = klo; hb = khi;
                        return true;
                    }
                    const double v = exact(n, d);
                    if (v > -CUDART_INF) {
                        has = true; ex_ok = true; ex_v = v; bn = n; bdi = di; lb = klo; hb = khi;
                        return true;
                    }
                    return false;
                }
                if (sure && klo > hb) {
                    ex_ok = false; bn = n; bdi = di; lb = klo; hb = khi;
                    return true;
                }
                if (khi >= lb) {
                    if (!ex_ok) { ex_v = exact(bn, s.dur[bdi]); ex_ok = true; }
                    const double v = exact(n, d);
                    if (v > -CUDART_INF && better(v, di, n, ex_v, bdi, bn)) {
                        ex_v = v; bn = n; bdi = di; lb = fmaxf(klo, lb); hb = khi;
                        return true;
                    }
                }
                return false;
            };
            // the screen of box (n, d) from its two screen records
            auto screen = [&](float2 av, float2 bv, int n, int d, float& t, float& den_lo,
                              float& den_hi, bool& sure_valid) -> bool {
                t = bv.x - av.x;
                const float iv = bv.y - av.y;              // count, or scaled weight
                const float ov = Wt - iv;
                bool ok;
                if (MODE == MODE_UNIFORM) {
                    den_lo = obj ? iv * ov * ov : iv * ov;  // exact counts: > 0 iff valid
                    den_hi = den_lo;
                    sure_valid = true;
                    ok = den_lo > 0.0f;
                } else {
                    const float il = fmaxf(iv - Ei, 0.0f), ol = fmaxf(ov - Ei, 0.0f);
                    const float ih = iv + Ei, oh = ov + Ei;
                    den_lo = obj ? il * ol * ol : il * ol;
                    den_hi = obj ? ih * oh * oh : ih * oh;
                    sure_valid = (il >= floor_q) & (ol >= floor_q);
                    ok = den_lo > 0.0f;
                    // an empty box is exactly 0 in the FP64 prefix; t <= Et also
                    // keeps sentinel boxes (t = NaN) away from these loads
                    if (!ok && t <= Et) {
                        ok = MODE == MODE_WIDE ? wide_prefix_i(hq, n + d) != wide_prefix_i(hq, n)
                                               : ld_f64(hq + (uint32_t)(n + d) * 16u + 8u) !=
                                                     ld_f64(hq + (uint32_t)n * 16u + 8u);
                    }
                }
                const float th = fabsf(t) + Et;
                return ok & (t <= Et) & !(th * th < thr * den_lo);
            };

            // Pilot: the lower key bounds of the warp's first chunk of the first
            // admissible duration set the screen's threshold before any box is
            // kept.  Each such box passes the screen again in the sweep below
            // (its upper bound is at least its lower bound), so its lane keeps it
            // or something better, and every box discarded against this
            // threshold is worse than a box that is kept.  Without it a warp's
            // first chunk of every period would pass the screen whole.
            {
                int dp = 0;
                while (dp < n_dur && s.dur[dp] >= nb) ++dp;
                if (dp < n_dur) {
                    const int d = s.dur[dp];
                    const int nmax = nb - d;
                    float kbest = -1.0f;
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int n = warp * 32 + lane + c * kThreads;
                        if (n <= nmax) {
                            const uint32_t sa = scr_s + (uint32_t)n * 8u;
                            float t, den_lo, den_hi;
                            bool sure_valid;
                            // thr is still -1 here: the screen checks admissibility only
                            const bool ok = screen(ld_f2(sa), ld_f2(sa + (uint32_t)d * 8u), n, d, t,
                                                   den_lo, den_hi, sure_valid);
                            const float tl = fmaxf(fabsf(t) - Et, 0.0f);
                            const float klo = __fdividef(tl * tl, den_hi) * (1.0f - kRel);
                            if (ok & (t < -Et) & sure_valid & (den_lo > 0.0f) & (klo > 0.0f) &
                                (klo < CUDART_INF_F))
                                kbest = fmaxf(kbest, klo);
                        }
                    }
                    kbest = warp_max(kbest);
                    if (kbest > 0.0f) {
                        thr = kbest * (1.0f - 2.0f * kRel);
                        if (lane == 0) atomicMax(&s.thr_bits, __float_as_uint(thr));
                    }
                }
            }

            // A cheaper screen in front of `screen`: th = Et - t bounds |t_exact|
            // for every dip (t_exact < 0 and |t - t_exact| <= Et), and den is a
            // lower bound of the box's exact denominator -- with one weight the
            // counts are exact in FP32 and den = c (N - c) (times N - c for the
            // likelihood); with per-point weights each side is lowered by the
            // weights' FP32 error Ei.  So a box failing th |th| >= thr den cannot
            // be the best; `screen` repeats its own test on the few that pass
            // (and decides, exactly, whether a box with den = 0 is empty).  The
            // threshold is shared by the CTA's warps through s.thr_bits
            // (non-negative floats order as their bits), each value a lower bound
            // of a box some lane keeps.
            {
                auto quick = [&](float2 av, float2 bv) -> bool {
                    const float t = bv.x - av.x;
                    const float th = Et - t;
                    const float c = bv.y - av.y;
                    if (MODE == MODE_UNIFORM) {
                        const float oc = Wt - c;
                        const float den = OBJ ? c * oc * oc : c * oc;
                        return (den > 0.0f) & (th * fabsf(th) >= thr * den);
                    } else {
                        const float il = fmaxf(c - Ei, 0.0f), ol = fmaxf(Wt - c - Ei, 0.0f);
                        const float den = OBJ ? il * ol * ol : il * ol;
                        return (th >= 0.0f) & ((den <= 0.0f) | (th * fabsf(th) >= thr * den));
                    }
                };
                // Starts outer: each lane's two start records (n, n + kThreads) load
                // once per chunk; widths inner in groups of four (one broadcast
                // load), so a lane screens eight independent boxes per step and
                // the warp votes once.  A width with no admissible start in the
                // chunk (too wide, past the chunk, or a kNoBox slot) reads the
                // sentinel record instead and fails.  Ties are ordered explicitly
                // by (duration index, start) in `consider` and the reductions.
                int dmin = nb;
                for (int k = 0; k < n_dur; ++k) dmin = min(dmin, s.dur[k]);
                const int nmax_all = nb - dmin;
                const int n_groups = (n_dur + 3) >> 2;
                const uint32_t sent = scr_s + (uint32_t)L * 8u;    // first sentinel record
                constexpr int kHalf = kThreads * 8;                 // bytes to the second start
                uint32_t sa = scr_s + (uint32_t)(warp * 32 + lane) * 8u;
                for (int n0 = warp * 32; n0 <= nmax_all; n0 += 2 * kThreads, sa += 2u * kHalf) {
                    thr = fmaxf(thr, __uint_as_float(ld_u32(thr_s)));
                    const float2 a1 = ld_f2(sa), a2 = ld_f2_off<kHalf>(sa);
                    for (int g = 0; g < n_groups; ++g) {
                        const int4 dg = *reinterpret_cast<const int4*>(&s.dur[4 * g]);
                        const int dk[4] = {dg.x, dg.y, dg.z, dg.w};
                        uint32_t m = 0u;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const int d = dk[k];
                            const bool fits = (d < nb) & (n0 <= nb - d);
                            const uint32_t sb = fits ? sa + (uint32_t)d * 8u : sent;
                            const float2 b1 = ld_f2(sb), b2 = ld_f2_off<kHalf>(sb);
                            m |= (quick(a1, b1) ? 1u : 0u) << (2 * k);
                            m |= (quick(a2, b2) ? 2u : 0u) << (2 * k);
                        }
                        if (__any_sync(kFull, m != 0u)) {
                            const int n1 = n0 + lane, n2 = n1 + kThreads;
                            bool upd = false;
#pragma unroll 1
                            for (int k = 0; k < 4; ++k) {
                                if ((m >> (2 * k) & 3u) == 0u) continue;
                                const int di = 4 * g + k;
                                const int d = s.dur[di];
                                const int nmax = nb - d;
                                float t, l, h;
                                bool v;
                                if ((m >> (2 * k) & 1u) && n1 <= nmax &&
                                    screen(a1, ld_f2(sa + (uint32_t)d * 8u), n1, d, t, l, h, v))
                                    upd |= consider(n1, di, d, t, l, h, v);
                                if ((m >> (2 * k) & 2u) && n2 <= nmax &&
                                    screen(a2, ld_f2_off<kHalf>(sa + (uint32_t)d * 8u), n2, d, t,
                                           l, h, v))
                                    upd |= consider(n2, di, d, t, l, h, v);
                            }
                            if (__any_sync(kFull, upd)) {
                                thr = fmaxf(thr,
                                            warp_max(has ? lb * (1.0f - 2.0f * kRel) : -1.0f));
                                if (lane == 0) atomicMax(&s.thr_bits, __float_as_uint(thr));
                            }
                        }
                    }
                }
            }

            // ---- reduce: lanes whose best may be the CTA's maximum --------------
            // After the barrier s.thr_bits is final: the largest published lower
            // bound (times 1 - 2 kRel), at most the CTA's best lower bound, so a
            // lane whose upper bound is below it cannot hold the best box.  The
            // lane holding that largest lower bound is always a candidate; when
            // it is the only one its box is the period's best and needs no FP64
            // comparison (the epilogue evaluates it).  Several candidates (near
            // ties, or every box in exact mode) are compared in FP64 with the
            // reference's first-wins order.
            __syncthreads();
            const float Lc = __uint_as_float(ld_u32(thr_s));
            const bool cand = has && hb >= Lc;
            const int n_cand = __syncthreads_count(cand);
            if (n_cand == 1) {
                if (cand) { s.win_v[q] = 0.0; s.win_di[q] = bdi; s.win_n[q] = bn; }
            } else {
                double v = -CUDART_INF;
                int vdi = 1 << 30, vn = 1 << 30;
                if (cand) {
                    if (!ex_ok) { ex_v = exact(bn, s.dur[bdi]); ex_ok = true; }
                    v = ex_v; vdi = bdi; vn = bn;
                }
                if (__any_sync(kFull, cand)) {
#pragma unroll
                    for (int k = 16; k > 0; k >>= 1) {
                        const double ov = __shfl_xor_sync(kFull, v, k);
                        const int odi = __shfl_xor_sync(kFull, vdi, k);
                        const int on = __shfl_xor_sync(kFull, vn, k);
                        if (better(ov, odi, on, v, vdi, vn)) { v = ov; vdi = odi; vn = on; }
                    }
                }
                if (lane == 0) { s.red_v[warp] = v; s.red_di[warp] = vdi; s.red_n[warp] = vn; }
                __syncthreads();
                if (tid == 0) {
                    for (int w = 1; w < kWarps; ++w)
                        if (better(s.red_v[w], s.red_di[w], s.red_n[w], v, vdi, vn)) {
                            v = s.red_v[w]; vdi = s.red_di[w]; vn = s.red_n[w];
                        }
                    s.win_v[q] = v;
                    s.win_di[q] = vdi;
                    s.win_n[q] = vn;
                }
            }
        }

        // ---- 4. the tile's seven output fields, one thread per period ----------
        __syncthreads();
        if (tid < pt) {
            const int q = tid;
            const uint32_t hq = smem_s + (uint32_t)(q * pbytes);
            double* op = out + q;
            if (!(s.win_v[q] > -CUDART_INF)) {
                op[0] = -CUDART_INF;
                for (int f = 1; f < kFields; ++f) op[f * ostride] = 0.0;
            } else {
                const int vn = s.win_n[q];
                const int d = s.dur[s.win_di[q]];
                const BoxSums b = box_sums<MODE>(hq, cv, vn, d);
                const double iv_out = b.iv_out;
                const double yin = b.y_in / b.iv_in;
                const double yout = b.y_out / iv_out;
                const double depth = yout - yin;
                const double derr = sqrt(1.0 / b.iv_in + 1.0 / iv_out);
                const double dsnr = depth / derr;
                const double ll = 0.5 * b.iv_in * depth * depth;
                const double bin = s.seg.bin_duration;
                const double dur = (double)d * bin;
                op[0] = obj == 0 ? dsnr : ll;
                op[1 * ostride] = depth;
                op[2 * ostride] = derr;
                op[3 * ostride] = dsnr;
                op[4 * ostride] = dur;
                op[5 * ostride] = fmod((double)vn * bin + 0.5 * dur, s.per[q]) + cv.t_min;
                op[6 * ostride] = ll;
            }
        }
    }
}

// ---- per-curve result rows: SDE normalisation and alias-diverse peaks -------
// The reference's row (src/cuperiod/batch/io.py:507-571) ranks the peaks of the
// assembled spectrum (methods/bls.py:274-301): power with non-finite values as
// 0, SDE = (power - mean) / std, candidates = interior local maxima in ascending
// frequency (strictly above the lower-frequency neighbour, >= the higher) plus
// the boundary points (core/result.py:369-406), then greedy highest-score
// candidates skipping any alias-related to one already chosen
// (core/peaks.py:128-231).  Greedy selection equals taking, n times, the best
// remaining candidate and dropping every candidate related to it, which is what
// one CTA per curve does here.  The grid is in ascending period, so frequency
// order is reversed grid order.

__device__ __forceinline__ double nan_to_zero(double v) { return isfinite(v) ? v : 0.0; }

// is_alias_related(f_new, f_chosen) with the reference's FP64 operations in its
// order (no contraction): duplicate within `sep`, harmonics and subharmonics up
// to `hmax`, sidereal/solar day offsets (x1, x2) and the yearly offset.
__device__ bool alias_related(double fn, double fc, double tol, int hmax, double sep,
                              const double* offs) {
    if (fabs(__dsub_rn(fn, fc)) < sep) return true;
    for (int m = 2; m <= hmax; ++m) {
        const double md = (double)m;
        if (fabs(__dsub_rn(fn, __dmul_rn(md, fc))) < __dmul_rn(md, tol)) return true;
        if (fabs(__dsub_rn(fn, __ddiv_rn(fc, md))) < tol) return true;
    }
    for (int k = 0; k < 5; ++k) {
        const double off = offs[k];
        if (fabs(__dsub_rn(fn, fabs(__dsub_rn(fc, off)))) < tol ||
            fabs(__dsub_rn(fn, __dadd_rn(fc, off))) < tol)
            return true;
    }
    return false;
}

// The alias test of candidates fn against one chosen peak fc, both directions,
// with fc's multiples, subharmonics and offsets computed once per round.  The
// only division per candidate, fn / m in the reverse subharmonic test, is taken
// as fn * (1/m) unless the comparison is within a few ulps of the tolerance,
// where the IEEE quotient decides as in the reference.
struct AliasRound {
    static constexpr int kMaxH = 32;
    double fc, tol, sep;
    int hmax;
    double mfc[kMaxH + 1], mtol[kMaxH + 1], fcm[kMaxH + 1];
    double lo[5], hi[5], off[5];

    __device__ void init(double f, double t, double s, int h, const double* offs) {
        fc = f; tol = t; sep = s; hmax = h;
        for (int m = 2; m <= h; ++m) {
            const double md = (double)m;
            mfc[m] = __dmul_rn(md, f);
            mtol[m] = __dmul_rn(md, t);
            fcm[m] = __ddiv_rn(f, md);
        }
        for (int k = 0; k < 5; ++k) {
            off[k] = offs[k];
            lo[k] = fabs(__dsub_rn(f, offs[k]));
            hi[k] = __dadd_rn(f, offs[k]);
        }
    }
    // is_alias_related(fn, fc) or is_alias_related(fc, fn)
    __device__ bool related(double fn) const {
        if (fabs(__dsub_rn(fn, fc)) < sep) return true;          // either way
        for (int m = 2; m <= hmax; ++m) {
            const double md = (double)m;
            if (fabs(__dsub_rn(fn, mfc[m])) < mtol[m]) return true;
            if (fabs(__dsub_rn(fn, fcm[m])) < tol) return true;
            if (fabs(__dsub_rn(fc, __dmul_rn(md, fn))) < mtol[m]) return true;
            double q = __dmul_rn(fn, __drcp_rn(md));
            const double gap = fabs(__dsub_rn(fc, q));
            if (fabs(gap - tol) <= 8.0 * DBL_EPSILON * fmax(fabs(fc), fmax(fabs(q), tol)))
                q = __ddiv_rn(fn, md);
            if (fabs(__dsub_rn(fc, q)) < tol) return true;
        }
        for (int k = 0; k < 5; ++k) {
            if (fabs(__dsub_rn(fn, lo[k])) < tol || fabs(__dsub_rn(fn, hi[k])) < tol) return true;
            if (fabs(__dsub_rn(fc, fabs(__dsub_rn(fn, off[k])))) < tol ||
                fabs(__dsub_rn(fc, __dadd_rn(fn, off[k]))) < tol)
                return true;
        }
        return false;
    }
};

// Position of grid index j among the reference's candidates: interior maxima in
// ascending frequency, then the lowest-frequency point, then the highest.  Among
// equal scores the later position ranks first (a stable ascending sort, reversed).
__device__ __forceinline__ long long cand_pos(long long j, long long P) {
    if (P == 1) return 0;
    if (j == P - 1) return P;
    if (j == 0) return P + 1;
    return P - 1 - j;
}

__global__ void __launch_bounds__(kThreads) rows_kernel(
    const double* __restrict__ out, int64_t out_stride, const int64_t* __restrict__ spec_off,
    const int64_t* __restrict__ grid_base, const double* __restrict__ freq_all,
    const double* __restrict__ sep_c,
    const double* __restrict__ tol_c, int n_best, int hmax, int32_t* n_peaks,
    int64_t* index, double* fields) {
    extern __shared__ uint32_t cand[];                   // ceil(P / 32) words
    __shared__ double red_d[kWarps];
    __shared__ double red_s[kWarps];
    __shared__ long long red_p[kWarps];
    __shared__ long long red_j[kWarps];
    __shared__ double s_mean, s_std;
    __shared__ long long s_win;
    __shared__ AliasRound s_alias;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int c = blockIdx.x;
    const int64_t so = spec_off[c];
    const int64_t P = spec_off[c + 1] - so;              // curve c's trial periods
    const double* pw = out + so;                         // field 0 (power) of curve c
    const double* freq = freq_all + grid_base[c];        // its grid's RN(1/P)
    const int64_t nw = (P + 31) / 32;
    if (P < 1) {
        if (tid == 0) n_peaks[c] = 0;
        return;
    }
    const double sep = sep_c[c], tol = tol_c[c];
    double offs[5];
    offs[0] = 1.0027379;                                 // sidereal day, cycles/day
    offs[1] = __dmul_rn(2.0, 1.0027379);
    offs[2] = 1.0;                                       // solar day
    offs[3] = 2.0;
    offs[4] = __ddiv_rn(1.0, 365.25);                    // year

    // mean and population standard deviation of the power (two passes)
    double sum = 0.0;
    for (int64_t j = tid; j < P; j += kThreads) sum += nan_to_zero(pw[j]);
    sum = warp_sum(sum);
    if (lane == 0) red_d[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kWarps; ++w) t += red_d[w];
        s_mean = t / (double)P;
    }
    __syncthreads();
    const double mean = s_mean;
    double ss = 0.0;
    for (int64_t j = tid; j < P; j += kThreads) {
        const double d = nan_to_zero(pw[j]) - mean;
        ss += d * d;
    }
    ss = warp_sum(ss);
    if (lane == 0) red_d[warp] = ss;
    // candidate words, each owned by one thread
    for (int64_t w = tid; w < nw; w += kThreads) {
        uint32_t bits = 0u;
        for (int b = 0; b < 32; ++b) {
            const int64_t j = w * 32 + b;
            if (j >= P) break;
            const double v = nan_to_zero(pw[j]);
            bool is;
            if (P == 1) {
                is = true;
            } else if (j == P - 1) {                     // lowest frequency
                is = v >= nan_to_zero(pw[j - 1]);
            } else if (j == 0) {                         // highest frequency
                is = v > nan_to_zero(pw[1]);
            } else {                                     // above the lower frequency, >= the higher
                is = (v > nan_to_zero(pw[j + 1])) & (v >= nan_to_zero(pw[j - 1]));
            }
            if (is) bits |= 1u << b;
        }
        cand[w] = bits;
    }
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int w = 0; w < kWarps; ++w) t += red_d[w];
        s_std = sqrt(t / (double)P);
    }

    int count = 0;
    for (int r = 0; r < n_best; ++r) {
        // the best remaining candidate: highest score, then later position
        double bs = -CUDART_INF;
        long long bp = -1, bj = -1;
        for (int64_t w = tid; w < nw; w += kThreads) {
            uint32_t bits = cand[w];
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const long long j = w * 32 + b;
                const double v = nan_to_zero(pw[j]);
                const long long pos = cand_pos(j, P);
                if (v > bs || (v == bs && pos > bp)) { bs = v; bp = pos; bj = j; }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double os = __shfl_xor_sync(kFull, bs, o);
            const long long op = __shfl_xor_sync(kFull, bp, o);
            const long long oj = __shfl_xor_sync(kFull, bj, o);
            if (oj >= 0 && (bj < 0 || os > bs || (os == bs && op > bp))) { bs = os; bp = op; bj = oj; }
        }
        if (lane == 0) { red_s[warp] = bs; red_p[warp] = bp; red_j[warp] = bj; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < kWarps; ++w)
                if (red_j[w] >= 0 && (bj < 0 || red_s[w] > bs || (red_s[w] == bs && red_p[w] > bp))) {
                    bs = red_s[w]; bp = red_p[w]; bj = red_j[w];
                }
            s_win = bj;
            if (bj >= 0) {
                const double f = freq[bj];
                const double v = nan_to_zero(pw[bj]);
                double* fo = fields + ((int64_t)c * n_best + r) * 8;
                fo[0] = __ddiv_rn(1.0, f);                          // period = 1 / frequency
                fo[1] = f;
                fo[2] = v;                                          // power
                fo[3] = out[1 * out_stride + so + bj];              // depth
                fo[4] = out[3 * out_stride + so + bj];              // depth_snr
                fo[5] = out[4 * out_stride + so + bj];              // duration
                fo[6] = out[5 * out_stride + so + bj];              // t0
                fo[7] = s_std > 0.0 ? (v - s_mean) / s_std : 0.0;  // sde
                index[(int64_t)c * n_best + r] = bj;
            }
        }
        __syncthreads();
        const long long win = s_win;
        if (win < 0) break;
        ++count;
        // drop the winner and every candidate alias-related to it, either way
        const double fc = freq[win];                  // RN(1/P), numpy's 1.0 / period
        const bool fast = hmax <= AliasRound::kMaxH;
        if (fast && tid == 0) s_alias.init(fc, tol, sep, hmax, offs);
        __syncthreads();
        for (int64_t w = tid; w < nw; w += kThreads) {
            uint32_t bits = cand[w], keep = bits;
            while (bits) {
                const int b = __ffs(bits) - 1;
                bits &= bits - 1u;
                const long long j = w * 32 + b;
                const double fn = freq[j];
                if (j == win ||
                    (fast ? s_alias.related(fn)
                          : alias_related(fn, fc, tol, hmax, sep, offs) ||
                                alias_related(fc, fn, tol, hmax, sep, offs)))
                    keep &= ~(1u << b);
            }
            cand[w] = keep;
        }
        __syncthreads();
    }
    if (tid == 0) n_peaks[c] = count;
}

// Phase bins of every point at one period through the fast path with its
// fallback (the tests compare them with the reference's fold bit for bit).
__global__ void fold_bins_kernel(const double* tau, int n, double P, double f, uint32_t S,
                                 double bin, int width, int fb, uint32_t mu, uint32_t mphi,
                                 int fast, int32_t* out, int32_t* used_fast) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t fmask = (1u << fb) - 1u;
    int ind = fast ? fold_fast(tau[j], f, S, fb, fmask, mu, (1u << fb) - 2u * mu, mphi,
                               0u - 2u * mphi)
                   : -1;
    used_fast[j] = ind >= 0;
    if (ind < 0) ind = fold_exact(tau[j], P, bin, width);
    out[j] = ind;
}

// Per curve: the largest power (non-finite values count as 0, as the
// reference's assembly does before its SDE and peak search) with its first
// index, and the mean and population standard deviation of that power.
__global__ void best_kernel(const double* power, const int64_t* spec_off, int64_t* best_index,
                            double* best_power, double* mean_out, double* std_out) {
    __shared__ double red_s[kWarps];
    __shared__ double red_v[kWarps];
    __shared__ long long red_i[kWarps];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double* p = power + spec_off[blockIdx.x];
    const int64_t n_periods = spec_off[blockIdx.x + 1] - spec_off[blockIdx.x];
    double sum = 0.0, bv = -CUDART_INF;
    long long bi = -1;
    for (int64_t i = tid; i < n_periods; i += kThreads) {
        const double v = p[i];
        const double z = isfinite(v) ? v : 0.0;
        sum += z;
        if (z > bv || (z == bv && i < bi)) { bv = z; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(kFull, sum, o);
        const double ov = __shfl_xor_sync(kFull, bv, o);
        const long long oi = __shfl_xor_sync(kFull, bi, o);
        if (ov > bv || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) { bv = ov; bi = oi; }
    }
    if (lane == 0) { red_s[warp] = sum; red_v[warp] = bv; red_i[warp] = bi; }
    __syncthreads();
    sum = 0.0;
    bv = -CUDART_INF;
    bi = -1;
    for (int w = 0; w < kWarps; ++w) {
        sum += red_s[w];
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] >= 0 && (bi < 0 || red_i[w] < bi))) {
            bv = red_v[w];
            bi = red_i[w];
        }
    }
    const double mean = n_periods > 0 ? sum / (double)n_periods : 0.0;
    __syncthreads();
    double ss = 0.0;
    for (int64_t i = tid; i < n_periods; i += kThreads) {
        const double v = p[i];
        const double z = (isfinite(v) ? v : 0.0) - mean;
        ss += z * z;
    }
    ss = warp_sum(ss);
    if (lane == 0) red_s[warp] = ss;
    __syncthreads();
    if (tid == 0) {
        ss = 0.0;
        for (int w = 0; w < kWarps; ++w) ss += red_s[w];
        best_index[blockIdx.x] = bi;
        best_power[blockIdx.x] = bv;
        mean_out[blockIdx.x] = mean;
        std_out[blockIdx.x] = n_periods > 0 ? sqrt(ss / (double)n_periods) : 0.0;
    }
}

}  // namespace

namespace {
template <int OBJ>
const void* search_fn(int mode) {
    return mode == MODE_UNIFORM ? (const void*)bls_search_kernel<MODE_UNIFORM, OBJ>
           : mode == MODE_WIDE  ? (const void*)bls_search_kernel<MODE_WIDE, OBJ>
                                : (const void*)bls_search_kernel<MODE_GENERAL, OBJ>;
}
}  // namespace

cudaError_t raise_smem_limit(const void* fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = limit[{dev, fn}];
    if (smem <= have) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) have = smem;
    return e;
}

cudaError_t configure_search(int mode, size_t smem) {
    for (const void* f : {search_fn<0>(mode), search_fn<1>(mode)}) {
        const cudaError_t e = raise_smem_limit(f, smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_search(const BatchArgs& args, int mode, int n_ctas, size_t smem,
                          cudaStream_t stream) {
    const bool ll = args.obj_flag != 0;
    if (mode == MODE_UNIFORM) {
        if (ll) bls_search_kernel<MODE_UNIFORM, 1><<<n_ctas, kThreads, smem, stream>>>(args);
        else bls_search_kernel<MODE_UNIFORM, 0><<<n_ctas, kThreads, smem, stream>>>(args);
    } else if (mode == MODE_WIDE) {
        if (ll) bls_search_kernel<MODE_WIDE, 1><<<n_ctas, kThreads, smem, stream>>>(args);
        else bls_search_kernel<MODE_WIDE, 0><<<n_ctas, kThreads, smem, stream>>>(args);
    } else {
        if (ll) bls_search_kernel<MODE_GENERAL, 1><<<n_ctas, kThreads, smem, stream>>>(args);
        else bls_search_kernel<MODE_GENERAL, 0><<<n_ctas, kThreads, smem, stream>>>(args);
    }
    return cudaGetLastError();
}

cudaError_t launch_best(const double* power, int n_curves, const int64_t* spec_off,
                        int64_t* best_index, double* best_power, double* mean, double* sd,
                        cudaStream_t stream) {
    if (n_curves <= 0) return cudaSuccess;
    best_kernel<<<n_curves, kThreads, 0, stream>>>(power, spec_off, best_index, best_power, mean,
                                                   sd);
    return cudaGetLastError();
}

cudaError_t launch_rows(const double* out, int64_t out_stride, int n_curves,
                        const int64_t* spec_off, const int64_t* grid_base, int64_t max_periods,
                        const double* freq, const double* sep, const double* tol, int n_best,
                        int harmonic_max, int32_t* n_peaks, int64_t* index, double* fields,
                        cudaStream_t stream) {
    if (n_curves <= 0) return cudaSuccess;
    const size_t smem = sizeof(uint32_t) * (size_t)((max_periods + 31) / 32);
    cudaError_t e = raise_smem_limit((const void*)rows_kernel, smem);
    if (e != cudaSuccess) return e;
    rows_kernel<<<n_curves, kThreads, smem, stream>>>(out, out_stride, spec_off, grid_base, freq,
                                                      sep, tol, n_best, harmonic_max, n_peaks,
                                                      index, fields);
    return cudaGetLastError();
}

cudaError_t launch_fold_bins(const double* tau, int n, double P, double f, uint32_t S, double bin,
                             int width, int fb, uint32_t mu, uint32_t mphi, int fast,
                             int32_t* out, int32_t* used_fast, cudaStream_t stream) {
    if (n <= 0) return cudaSuccess;
    fold_bins_kernel<<<(n + 255) / 256, 256, 0, stream>>>(tau, n, P, f, S, bin, width, fb, mu,
                                                          mphi, fast, out, used_fast);
    return cudaGetLastError();
}

// 2 MiB + 256 B per device, in the library's module (no allocation at run time).
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

cudaError_t static_scratch_address(int device, void** ptr) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        addr[device] = p;
    }
    *ptr = addr[device];
    return cudaSuccess;
}

int search_threads() { return kThreads; }

size_t period_hist_bytes(int mode, int hl) {
    return mode == MODE_UNIFORM ? hist_period_bytes<MODE_UNIFORM>(hl)
           : mode == MODE_WIDE  ? hist_period_bytes<MODE_WIDE>(hl)
                                : hist_period_bytes<MODE_GENERAL>(hl);
}

size_t search_static_smem(int mode) {
    size_t most = 0;
    for (const void* f : {search_fn<0>(mode), search_fn<1>(mode)}) {
        cudaFuncAttributes at{};
        if (cudaFuncGetAttributes(&at, f) == cudaSuccess) most = std::max(most, at.sharedSizeBytes);
    }
    return most;
}

int max_resident_ctas(int mode, size_t smem) {
    // the smaller of the two objectives' occupancies
    int b0 = 0, b1 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, search_fn<0>(mode), kThreads, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, search_fn<1>(mode), kThreads, smem);
    return b0 < b1 ? b0 : b1;
}

}  // namespace blsb200
