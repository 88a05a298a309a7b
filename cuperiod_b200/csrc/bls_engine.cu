// Host side of the B200 BLS engine: the C ABI of include/bls_b200.h.
//
// bls_prepare packs a batch on all host cores into pinned staging (the
// reference's host steps: time origin, median centring, inverse variances --
// cuPeriod src/cuperiod/methods/_bls_core.py:1043-1058, 709-738 -- then this
// engine's exact fixed-point encoding), derives each segment's binning exactly
// as _search_spec / _duration_bins do (_bls_core.py:134-149, 697-706), builds
// the work list and uploads everything in a few large copies.  bls_launch runs
// the persistent search kernels (replayed from a CUDA graph when enabled);
// bls_download / bls_download_best bring results back.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bls_b200.h"
#include "bls_device.h"
#include "bls_grid.h"
#include "bls_launch.h"

using namespace blsb200;

namespace {

thread_local std::string g_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? BLS_E_NOMEM : BLS_E_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
}

// Runs an entry's body; host allocation failures become BLS_E_NOMEM instead of
// an exception escaping the C ABI.
template <typename F>
int guarded(F&& body) {
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(BLS_E_NOMEM, "host allocation failed");
    }
}

#define CUDA_TRY(expr, what)                          \
    do {                                              \
        cudaError_t e_ = (expr);                      \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return BLS_OK;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) return cuda_fail(e, "device allocation");
        cap = want;
        return BLS_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Grow-only pinned host buffer.
struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    int ensure(size_t bytes) {
        if (bytes <= cap) return BLS_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e != cudaSuccess) return cuda_fail(e, "pinned host allocation");
        cap = want;
        return BLS_OK;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// numpy's pairwise summation of a contiguous float64 array (the algorithm of
// numpy's pairwise_sum: 8 partial sums over blocks of at most 128 elements,
// halves split on a multiple of 8), so sum_y and sum_ivar equal the reference's
// yw.sum() / ivar.sum() bit for bit.
double pairwise_sum(const double* a, int64_t n) {
    if (n < 8) {
        double res = 0.0;
        for (int64_t i = 0; i < n; ++i) res += a[i];
        return res;
    }
    if (n <= 128) {
        double r[8];
        for (int k = 0; k < 8; ++k) r[k] = a[k];
        int64_t i;
        for (i = 8; i < n - (n % 8); i += 8)
            for (int k = 0; k < 8; ++k) r[k] += a[i + k];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += a[i];
        return res;
    }
    int64_t n2 = n / 2;
    n2 -= n2 % 8;
    return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
}

// Fast-fold parameters of one segment (see the kernel's fold_fast): the
// fraction bits of the scaled phase and the margins that make its result
// provably the reference's.  q_max bounds tau * (1/P) over the batch, tau_max
// the largest time offset.
struct FoldParams {
    int fb = 0;
    uint32_t mu = 0, mphi = 0;
    bool fast = false;
};

FoldParams fold_params(int64_t width, double bin, double tau_max, double f_max, double s_max) {
    FoldParams fp;
    if (width < 2 || width > (1 << 20) || !(bin > 0.0)) return fp;
    const double q_max = tau_max * f_max;
    if (!(q_max < 262144.0)) return fp;                      // q must stay below 2^18
    int lw = 0;
    while ((int64_t(1) << (lw + 1)) <= width) ++lw;          // floor(log2(width))
    fp.fb = 31 - lw;                                         // width * 2^fb < 2^32
    const double two32 = 4294967296.0;
    // our phase error (cycles): RN(1/P) and the product x*RN(1/P) (the kernel
    // adds it to 1.5*2^20 in one FMA, so the product is not rounded on its own:
    // this bound is conservative) and the 2^-32 grid
    const double e_phi = q_max * std::ldexp(1.0, -52) * 1.01 + std::ldexp(1.0, -33);
    // the reference's floor(RN(x/P)) is exact unless the phase is this close to a cycle edge
    const double e_phi_ref = q_max * std::ldexp(1.0, -53);
    const double mphi = std::ceil((e_phi + e_phi_ref) * two32) + 2.0;
    // the reference's w/bin error (bins): x - P*floor rounds at ulp(x), the division at 2^-53
    int ex = 0;
    if (tau_max > 0.0) std::frexp(tau_max, &ex);            // tau_max < 2^ex
    const double e_ref = 2.0 * std::ldexp(1.0, ex - 52) / bin + (double)width * std::ldexp(1.0, -52);
    const double scale = std::ldexp(1.0, fp.fb);
    const double e_u = e_phi * s_max * scale + 2.0;          // + S rounding and the floor
    const double mu = std::ceil(e_u + e_ref * scale) + 2.0;
    if (!(mphi < 1e6) || !(mu * 4.0 < scale)) return fp;
    fp.mu = (uint32_t)mu;
    fp.mphi = (uint32_t)mphi;
    fp.fast = true;
    return fp;
}

struct PeriodConst {
    double f;
    uint32_t S;
    int32_t nb;
};

// The reference's n_bins of one period (_bls_core.py:358-360 / 525-526).
inline int64_t period_bins(double P, double bin, int oversample, int64_t width) {
    int64_t nb = (int64_t)std::ceil(P / bin) + oversample;
    return nb > width - 1 ? width - 1 : nb;
}

struct SegmentHost {
    SegmentDesc d;
    std::vector<int32_t> dur;
    bool empty_periods = false;
};

struct CurveHost {
    CurveDesc d;
    double tau_max = 0.0;
    int status = BLS_OK;
    std::string err;
};

}  // namespace

struct BlsEngine {
    int device = 0;
    int n_sm = 0;
    size_t smem_optin = 0;
    cudaStream_t stream = nullptr;
    BlsTune tune{};

    // device buffers
    DevBuf d_tau, d_pay_r, d_r64, d_iv64, d_period, d_freq, d_scale, d_nbins, d_dur, d_curves,
        d_segments, d_rows, d_out, d_ctl, d_best, d_joint, d_tls;
    // pinned staging
    HostBuf h_tau, h_pay_r, h_r64, h_iv64, h_grid, h_meta, h_ctl, h_best, h_rows, h_joint,
        h_tls;

    // the prepared batch
    bool prepared = false;
    int n_curves = 0;
    int n_grids = 0;
    int64_t spec_total = 0;             // spectrum entries per output field, all curves
    int64_t max_periods = 0;            // the longest curve spectrum
    std::vector<int64_t> grid_pbase;    // grid k's periods: [grid_pbase[k], grid_pbase[k + 1])
    std::vector<int64_t> spec_off;      // host: per-curve spectrum offsets (n_curves + 1)
    const int64_t* d_spec_off = nullptr;    // device: per-curve spectrum offsets (n_curves + 1)
    const int64_t* d_grid_base = nullptr;   // device: per-curve first period of its grid
    int n_items_mode[kModes] = {0, 0, 0};
    int ctas_mode[kModes] = {0, 0, 0};
    size_t smem_mode[kModes] = {0, 0, 0};
    BatchArgs args[kModes]{};
    BlsBatchInfo info{};

    // CUDA graph of one launch
    cudaGraphExec_t graph = nullptr;
    bool graph_valid = false;

    // the prepared TLS search
    bool tls_prepared = false;
    TlsArgs targs{};
    size_t tls_smem = 0;
    int tls_ctas = 0;
    size_t tls_out_bytes = 0;

    // the prepared joint (multi-band, shared box) search
    bool joint_prepared = false;
    JointArgs jargs{};
    bool joint_in_smem = false;
    size_t joint_smem = 0;
    int joint_ctas = 0;
    int64_t joint_periods = 0;

    ~BlsEngine() {
        if (graph) cudaGraphExecDestroy(graph);
        for (DevBuf* b : {&d_tau, &d_pay_r, &d_r64, &d_iv64, &d_period, &d_freq, &d_scale, &d_nbins,
                          &d_dur, &d_curves, &d_segments, &d_rows, &d_out, &d_ctl, &d_best,
                          &d_joint, &d_tls})
            b->release();
        for (HostBuf* b : {&h_tau, &h_pay_r, &h_r64, &h_iv64, &h_grid, &h_meta, &h_ctl, &h_best,
                           &h_rows, &h_joint, &h_tls})
            b->release();
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

cudaStream_t pick(BlsEngine* e, void* s) {
    return s ? static_cast<cudaStream_t>(s) : e->stream;
}

// One quantised value (|v| <= 2^27) as the kernel adds it: the unsigned low 13
// bits in the low half-word, the signed high part in the high half-word.
inline uint32_t split_word(long long v) {
    const uint32_t lo = (uint32_t)(v & ((1 << kHalfBits) - 1));
    const int32_t hi = (int32_t)(v >> kHalfBits);              // arithmetic shift
    return lo | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}

// Memory slot of the point with time index j in a curve of n points: every full
// chunk of kChunk points is stored lane-interleaved (see kChunk in bls_device.h),
// the tail in time order.
inline int64_t point_slot(int64_t j, int64_t n) {
    const int64_t full = (n / kChunk) * kChunk;
    if (j >= full) return j;
    const int64_t c = j / kChunk, w = j % kChunk;
    return c * kChunk + (w % kChunkPts) * kChunkThreads + w / kChunkPts;
}

// np.median of n >= 1 values: the mean of the two middle values for even n.
double median_of(const double* y, int64_t n, std::vector<double>& scratch) {
    scratch.assign(y, y + n);
    const int64_t mid = n / 2;
    std::nth_element(scratch.begin(), scratch.begin() + mid, scratch.end());
    double med = scratch[mid];
    if (n % 2 == 0) {
        const double lo = *std::max_element(scratch.begin(), scratch.begin() + mid);
        med = (lo + med) / 2.0;
    }
    return med;
}

// Pack one curve: the reference's host inputs, then the fixed-point words.
void pack_curve(const BlsCurves* cv, int c, int64_t off, double* tau, uint32_t* pay_r,
                double* r64, double* iv64, CurveHost& ch, std::vector<double>& scratch) {
    const int64_t b = cv->offsets[c], e = cv->offsets[c + 1];
    const int64_t n = e - b;
    CurveDesc& d = ch.d;
    std::memset(&d, 0, sizeof(d));
    d.point_off = off;
    d.n_points = (int32_t)n;
    if (n < 1) {
        ch.status = BLS_E_INVALID;
        ch.err = "light curve " + std::to_string(c) + " has no points";
        return;
    }
    if (n > kMaxPoints) {
        ch.status = BLS_E_INVALID;
        ch.err = "light curve " + std::to_string(c) + " has more than " +
                 std::to_string(kMaxPoints) + " points";
        return;
    }
    const double* t = cv->t + b;
    const double* y = cv->y + b;
    const double* dy = cv->dy ? cv->dy + b : nullptr;
    double t_min = t[0];
    for (int64_t j = 0; j < n; ++j) {
        if (!std::isfinite(t[j]) || !std::isfinite(y[j]) ||
            (dy && !(std::isfinite(dy[j]) && dy[j] > 0.0))) {
            ch.status = BLS_E_INVALID;
            ch.err = "light curve " + std::to_string(c) +
                     ": times, fluxes and errors must be finite (errors > 0)";
            return;
        }
        t_min = std::min(t_min, t[j]);
    }
    const double med = median_of(y, n, scratch);
    // yw, ivar (reference units); sums with numpy's pairwise order
    scratch.resize(3 * (size_t)n);
    double* yw = scratch.data();
    double* iv = yw + n;
    double* r = iv + n;
    double tau_max = 0.0;
    bool uniform = true;
    for (int64_t j = 0; j < n; ++j) {
        const double tj = t[j] - t_min;
        tau[point_slot(j, n)] = tj;
        tau_max = std::max(tau_max, tj);
        iv[j] = dy ? 1.0 / (dy[j] * dy[j]) : 1.0;
        yw[j] = (y[j] - med) * iv[j];
        uniform = uniform && iv[j] == iv[0];
    }
    // the exact integer sums hold up to kMaxExactPoints points; a longer curve
    // keeps FP64 sums (the reference's arithmetic, in atomic order)
    const bool exact_ok = n <= kMaxExactPoints;
    uniform = uniform && exact_ok;
    const double sum_y = pairwise_sum(yw, n);
    const double sum_ivar = pairwise_sum(iv, n);
    double sum_abs = 0.0;
    for (int64_t j = 0; j < n; ++j) sum_abs += std::fabs(yw[j]);
    const double ybar = sum_ivar > 0.0 ? sum_y / sum_ivar : 0.0;
    double max_r = 0.0, max_i = 0.0;
    for (int64_t j = 0; j < n; ++j) {
        r[j] = yw[j] - ybar * iv[j];
        max_r = std::max(max_r, std::fabs(r[j]));
        max_i = std::max(max_i, iv[j]);
    }
    // r_q = r * 2^e_r with |r_q| <= 2^bits: bits = min(27, 41 - ceil(log2 n)), so
    // the signed high part (r_q >> 13, 16 bits in the payload word) fits and the
    // high-part word's prefix sums, doubled at most by the wrap pad, stay below
    // 2^31 (n * 2^(bits - 12) <= 2^29); at least 24 bits up to 2^17 points
    int m = 0;
    while (m < 62 && ((int64_t)1 << m) < n) ++m;
    const int bits = std::min(27, 41 - m);
    int k = 0;
    int e_r = 0;
    if (max_r > 0.0 && std::isfinite(max_r)) {
        std::frexp(max_r, &k);             // max_r < 2^k
        e_r = bits - k;                    // |r_q| <= 2^bits
    }
    // one weight: every point is centred by the same whole number of quanta cq
    // (|stored| <= |r| * 2^e_r + 1: the median-centred mean is within max|r| of
    // 0, so nothing overflows); per-point weights keep r
    long long cq = 0;
    double c_frac = 0.0;
    if (uniform) {
        const double cw = std::ldexp(ybar * iv[0], e_r);
        cq = std::llrint(cw);
        c_frac = cw - (double)cq;
        for (int64_t j = 0; j < n; ++j)
            pay_r[point_slot(j, n)] = split_word(std::llrint(std::ldexp(yw[j], e_r)) - cq);
    } else {
        for (int64_t j = 0; j < n; ++j)
            pay_r[point_slot(j, n)] = split_word(std::llrint(std::ldexp(r[j], e_r)));
    }
    int e_i = 0;
    double i_total = 0.0;
    long long rq_total = 0, iq_total = 0;
    // per-point weights within a factor 2^8 of each other: 38-bit fixed point
    // (the smallest weight keeps >= 2^28 steps, a relative 2^-29)
    double min_i = max_i;
    for (int64_t j = 0; j < n && !uniform; ++j) min_i = std::min(min_i, iv[j]);
    const bool wide = exact_ok && !uniform && min_i > 0.0 && std::isfinite(max_i) &&
                      max_i <= 256.0 * min_i && max_r > 0.0 && std::isfinite(max_r);
    if (wide) {
        int kr = 0, ki = 0;
        std::frexp(max_r, &kr);            // max_r < 2^kr
        std::frexp(max_i, &ki);
        const int e_rw = 37 - kr, e_iw = 37 - ki;       // |v| < 2^37
        int64_t total = 0, rtotal = 0;
        for (int64_t j = 0; j < n; ++j) {
            const int64_t m = point_slot(j, n);
            const long long rq = std::llrint(std::ldexp(r[j], e_rw));
            const long long iq = std::llrint(std::ldexp(iv[j], e_iw));
            std::memcpy(&r64[m], &rq, sizeof(rq));
            std::memcpy(&iv64[m], &iq, sizeof(iq));
            total += iq;
            rtotal += rq;
        }
        e_r = e_rw;
        e_i = e_iw;
        i_total = (double)total;
        rq_total = rtotal;
        iq_total = total;
    } else if (!uniform) {
        // per-point weights: FP64 values scaled by powers of two (exact)
        if (max_i > 0.0 && std::isfinite(max_i)) {
            std::frexp(max_i, &k);
            e_i = 24 - k;
        }
        for (int64_t j = 0; j < n; ++j) {
            const int64_t m = point_slot(j, n);
            r64[m] = std::ldexp(r[j], e_r);
            iv64[m] = std::ldexp(iv[j], e_i);
            i_total += iv64[m];
        }
    }
    const double eps = DBL_EPSILON;
    double floor_v = 4.0 * (double)n * eps * sum_ivar;            // _ivar_floor, 75-94
    if (!(floor_v > 0.0)) floor_v = DBL_MIN;
    d.mode = uniform ? MODE_UNIFORM : (wide ? MODE_WIDE : MODE_GENERAL);
    d.exact_all = !(sum_abs >= 1e-150 && sum_abs <= 1e150 && sum_ivar >= 1e-150 &&
                    sum_ivar <= 1e150);
    d.skip = !(sum_ivar > 0.0 && std::isfinite(sum_ivar));
    d.t_min = t_min;
    d.sum_y = sum_y;
    d.sum_ivar = sum_ivar;
    d.ivar_floor = floor_v;
    d.ybar = ybar;
    d.w_uniform = iv[0];
    d.i_total = i_total;
    d.e_r = e_r;
    d.e_i = e_i;
    d.center = std::ldexp((double)cq, -e_r);
    d.center_frac = c_frac;
    d.rq_total = rq_total;
    d.iq_total = iq_total;
    ch.tau_max = tau_max;
}

template <typename F>
void parallel_for(int n, F&& fn) {
    int hw = (int)std::thread::hardware_concurrency();
    int nt = std::max(1, std::min(hw, n));
    if (nt <= 1) {
        for (int i = 0; i < n; ++i) fn(i, 0);
        return;
    }
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    th.reserve(nt);
    for (int w = 0; w < nt; ++w)
        th.emplace_back([&, w] {
            for (;;) {
                int i = next.fetch_add(1);
                if (i >= n) break;
                fn(i, w);
            }
        });
    for (auto& x : th) x.join();
}

// Dynamic shared memory per CTA: one weight per curve runs three CTAs per SM
// (the kernel is built for 80 registers), per-point weights (FP64 or wide
// fixed point) two.
constexpr size_t kDefaultSmem[kModes] = {72 * 1024, 108 * 1024, 108 * 1024};

size_t screen_bytes(int /*mode*/, int hl) { return ((size_t)hl + kScreenPad) * 8; }
size_t period_bytes(int mode, int hl) { return period_hist_bytes(mode, hl); }

int tile_cap(int mode, int hl, size_t smem, int max_tile) {
    const size_t scr = screen_bytes(mode, hl) + 16;
    if (smem <= scr) return 0;
    int cap = (int)((smem - scr) / period_bytes(mode, hl));
    cap = std::min(cap, kMaxTile);
    if (max_tile > 0) cap = std::min(cap, max_tile);
    return cap;
}

// Pack and upload one batch.  Curve c is searched over grids[grid_of_curve[c]]
// (over grids[0] for every curve when grid_of_curve is NULL); the grids'
// segments and periods are concatenated, grid k's from sbase[k] / pbase[k].
int do_prepare(BlsEngine* e, const BlsGrid* grids, int n_grids, const int32_t* grid_of_curve,
               const BlsCurves* cv, cudaStream_t st) {
    if (!grids || !cv || n_grids < 1) return fail(BLS_E_INVALID, "grid and curves are required");
    for (int k = 0; k < n_grids; ++k) {
        const BlsGrid* g = grids + k;
        if (g->n_segments < 0 || (g->n_segments > 0 && (!g->seg_offsets || !g->dur_offsets)))
            return fail(BLS_E_INVALID, "bad segment table");
        if (g->oversample < 1) return fail(BLS_E_INVALID, "oversample must be >= 1");
        if (g->objective != 0 && g->objective != 1)
            return fail(BLS_E_INVALID, "objective must be 'snr' or 'likelihood'");
        if (g->oversample != grids[0].oversample || g->objective != grids[0].objective)
            return fail(BLS_E_INVALID,
                        "the grids of one batch must share oversample and objective (grid %d)", k);
        if (g->n_segments > 0 && g->seg_offsets[0] != 0)
            return fail(BLS_E_INVALID, "seg_offsets[0] must be 0");
        if (g->n_segments > 0 && g->seg_offsets[g->n_segments] < 0)
            return fail(BLS_E_INVALID, "grid %d: bad period offsets", k);
    }
    if (cv->n_curves < 1 || !cv->offsets || !cv->t || !cv->y)
        return fail(BLS_E_INVALID, "at least one light curve is required");
    e->prepared = false;
    e->graph_valid = false;
    const int nc = cv->n_curves;
    const int o = grids[0].oversample;
    std::vector<int> sbase(n_grids + 1, 0);
    std::vector<int64_t> pbase(n_grids + 1, 0);
    for (int k = 0; k < n_grids; ++k) {
        const BlsGrid& g = grids[k];
        if ((int64_t)sbase[k] + g.n_segments > (1 << 24))
            return fail(BLS_E_INVALID, "too many segments in one batch");
        sbase[k + 1] = sbase[k] + g.n_segments;
        pbase[k + 1] = pbase[k] + (g.n_segments > 0 ? g.seg_offsets[g.n_segments] : 0);
    }
    const int ns = sbase[n_grids];
    const int64_t P_total = pbase[n_grids];
    std::vector<int32_t> gid(nc, 0);
    if (grid_of_curve)
        for (int c = 0; c < nc; ++c) {
            if (grid_of_curve[c] < 0 || grid_of_curve[c] >= n_grids)
                return fail(BLS_E_INVALID, "curve %d: grid index %d outside 0..%d", c,
                            grid_of_curve[c], n_grids - 1);
            gid[c] = grid_of_curve[c];
        }
    // curve c's spectrum: [spec_off[c], spec_off[c + 1]) of each output field
    std::vector<int64_t> spec_off(nc + 1, 0);
    for (int c = 0; c < nc; ++c)
        spec_off[c + 1] = spec_off[c] + (pbase[gid[c] + 1] - pbase[gid[c]]);
    const int64_t spec_total = spec_off[nc];
    const int64_t n_pts = cv->offsets[nc] - cv->offsets[0];
    if (cv->offsets[0] != 0 || n_pts < 0) return fail(BLS_E_INVALID, "offsets[0] must be 0");

    // ---- curves ---------------------------------------------------------------
    int rc;
    if ((rc = e->h_tau.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->h_pay_r.ensure(sizeof(uint32_t) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->h_r64.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->h_iv64.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    std::vector<CurveHost> curves(nc);
    int hw = std::max(1, (int)std::thread::hardware_concurrency());
    std::vector<std::vector<double>> scratch(hw);
    double* htau = e->h_tau.as<double>();
    uint32_t* hpr = e->h_pay_r.as<uint32_t>();
    double* hr64 = e->h_r64.as<double>();
    double* hiv64 = e->h_iv64.as<double>();
    parallel_for(nc, [&](int c, int w) {
        const int64_t off = cv->offsets[c];
        try {                       // a worker thread: nothing may escape it
            pack_curve(cv, c, off, htau + off, hpr + off, hr64 + off, hiv64 + off, curves[c],
                       scratch[w]);
        } catch (const std::bad_alloc&) {
            curves[c].status = BLS_E_NOMEM;
            curves[c].err = "host allocation failed while packing a light curve";
        }
        curves[c].d.out_off = spec_off[c] - pbase[gid[c]];
    });
    int n_uniform = 0;
    int n_mode[kModes] = {0, 0, 0};
    std::vector<double> tau_max(n_grids, 0.0);                  // per grid, over its curves
    std::vector<std::array<int, kModes>> grid_mode(n_grids, std::array<int, kModes>{0, 0, 0});
    for (int c = 0; c < nc; ++c) {
        if (curves[c].status) return fail(curves[c].status, "%s", curves[c].err.c_str());
        if (e->tune.exact_sweep) curves[c].d.exact_all = 1;
        tau_max[gid[c]] = std::max(tau_max[gid[c]], curves[c].tau_max);
        n_uniform += curves[c].d.mode == MODE_UNIFORM;
        n_mode[curves[c].d.mode]++;
        grid_mode[gid[c]][curves[c].d.mode]++;
    }

    // ---- segments and period constants (reference binning), grids in parallel ---
    std::vector<SegmentHost> segs(ns);
    std::vector<double> per(P_total);
    std::vector<PeriodConst> pc(P_total);
    std::vector<double> grid_boxes(n_grids, 0.0), grid_trials(n_grids, 0.0);
    std::vector<int> grid_err(n_grids, BLS_OK);
    std::vector<std::string> grid_msg(n_grids);
    parallel_for(n_grids, [&](int k, int /*w*/) {
      try {                         // a worker thread: nothing may escape it
        const BlsGrid& g = grids[k];
        auto bad = [&](int code, std::string msg) {
            grid_err[k] = code;
            grid_msg[k] = std::move(msg);
        };
        char buf[256];
        for (int sl = 0; sl < g.n_segments; ++sl) {
            const int s = sbase[k] + sl;
            const int64_t q0 = g.seg_offsets[sl], q1 = g.seg_offsets[sl + 1];   // this grid's
            const int64_t d0 = g.dur_offsets[sl], d1 = g.dur_offsets[sl + 1];
            if (q1 < q0 || d1 < d0) {
                std::snprintf(buf, sizeof buf, "segment %d: bad offsets", s);
                return bad(BLS_E_INVALID, buf);
            }
            const int64_t p0 = pbase[k] + q0, p1 = pbase[k] + q1;                // concatenated
            SegmentHost& sh = segs[s];
            SegmentDesc& sd = sh.d;
            std::memset(&sd, 0, sizeof(sd));
            sd.period_off = p0;
            sd.n_periods = (int32_t)(p1 - p0);
            sd.oversample = o;
            if (p1 == p0) {
                sh.empty_periods = true;
                continue;
            }
            if (d1 == d0) {
                std::snprintf(buf, sizeof buf, "segment %d has no durations", s);
                return bad(BLS_E_INVALID, buf);
            }
            double dmin = INFINITY, pmax = 0.0, fmax = 0.0;
            for (int64_t i = d0; i < d1; ++i) {
                const double d = g.durations[i];
                if (!(std::isfinite(d) && d > 0.0)) {
                    std::snprintf(buf, sizeof buf,
                                  "segment %d: durations must be finite and > 0", s);
                    return bad(BLS_E_INVALID, buf);
                }
                dmin = std::min(dmin, d);
            }
            for (int64_t i = q0; i < q1; ++i) {
                const double P = g.periods[i];
                if (!(std::isfinite(P) && P > 0.0)) {
                    std::snprintf(buf, sizeof buf,
                                  "BLS: trial periods must be finite and > 0 (segment %d)", s);
                    return bad(BLS_E_INVALID, buf);
                }
                pmax = std::max(pmax, P);
                per[pbase[k] + i] = P;
            }
            const double bin = dmin / (double)o;                              // _search_spec
            for (int64_t i = d0; i < d1; ++i) {                               // _duration_bins
                const double kd = std::floor(g.durations[i] / bin + 0.5);
                if (kd >= 1.0 && kd < 2147483647.0) {
                    const int32_t kk = (int32_t)kd;
                    if (std::find(sh.dur.begin(), sh.dur.end(), kk) == sh.dur.end())
                        sh.dur.push_back(kk);
                }
            }
            if ((int)sh.dur.size() > kMaxDur) {
                std::snprintf(buf, sizeof buf, "segment %d: more than %d distinct box widths", s,
                              kMaxDur);
                return bad(BLS_E_INVALID, buf);
            }
            const double wmax = std::ceil(pmax / bin) + (double)o + 1.0;
            if (!(wmax < 1073741824.0)) {
                std::snprintf(buf, sizeof buf, "segment %d: %.3g phase bins per period", s, wmax);
                return bad(BLS_E_RESOURCE, buf);
            }
            const int64_t width = (int64_t)wmax;
            int64_t hl = 2;
            double smax = 0.0;
            for (int64_t i = p0; i < p1; ++i) {
                const double P = per[i];
                const int64_t nb = period_bins(P, bin, o, width);
                hl = std::max(hl, nb + 1);
                fmax = std::max(fmax, 1.0 / P);
                smax = std::max(smax, P / bin);
            }
            sd.width = (int32_t)width;
            sd.bin_duration = bin;
            sd.n_dur = (int32_t)sh.dur.size();
            sd.hist_len = (int32_t)hl;
            FoldParams fp = fold_params(width, bin, tau_max[k], fmax, smax);
            const double scale = std::ldexp(1.0, fp.fb);
            for (int64_t i = p0; i < p1 && fp.fast; ++i) {
                const double P = per[i];
                const double sc = std::nearbyint((P / bin) * scale);
                const int64_t nb = period_bins(P, bin, o, width);
                if (!(sc >= 1.0 && sc < 4294967296.0)) { fp.fast = false; break; }
                const uint32_t S = (uint32_t)sc;
                // the fast fold's largest bin, ((S - 1) >> fb) + 1, must stay inside n_bins
                if ((int64_t)((S - 1u) >> fp.fb) + 1 > nb) { fp.fast = false; break; }
            }
            double boxes = 0.0;
            for (int64_t i = p0; i < p1; ++i) {
                const double P = per[i];
                pc[i].f = 1.0 / P;
                pc[i].nb = (int32_t)period_bins(P, bin, o, width);
                pc[i].S = fp.fast ? (uint32_t)std::nearbyint((P / bin) * scale) : 0u;
                for (int32_t kk : sh.dur)
                    if (kk < pc[i].nb) boxes += (double)(pc[i].nb - kk + 1);
            }
            sd.fast_fold = fp.fast;
            sd.frac_bits = fp.fast ? fp.fb : 0;
            sd.margin_u = fp.mu;
            sd.margin_phi = fp.mphi;
            grid_boxes[k] += boxes;                  // per curve of this grid
            grid_trials[k] += (double)sd.n_periods * sh.dur.size();
        }
      } catch (const std::bad_alloc&) {
        grid_err[k] = BLS_E_NOMEM;
        grid_msg[k] = "host allocation failed while preparing a grid";
      }
    });
    for (int k = 0; k < n_grids; ++k)
        if (grid_err[k]) return fail(grid_err[k], "%s", grid_msg[k].c_str());
    std::vector<int32_t> dur_all;
    int max_hl = 2;
    int fast_segments = 0;
    for (int s = 0; s < ns; ++s) {
        SegmentHost& sh = segs[s];
        sh.d.dur_off = (int32_t)dur_all.size();
        if (sh.empty_periods) continue;
        fast_segments += sh.d.fast_fold;
        max_hl = std::max<int>(max_hl, sh.d.hist_len);
        dur_all.insert(dur_all.end(), sh.dur.begin(), sh.dur.end());
    }
    (void)max_hl;
    std::vector<int> seg_grid(ns, 0);
    for (int k = 0; k < n_grids; ++k)
        for (int s = sbase[k]; s < sbase[k + 1]; ++s) seg_grid[s] = k;

    // ---- shared memory, tiles, work groups (costliest first) -------------------
    bool modes[kModes] = {n_mode[0] > 0, n_mode[1] > 0, n_mode[2] > 0};
    size_t smem_mode[kModes];
    for (int m = 0; m < kModes; ++m) {
        size_t sm = e->tune.smem_per_cta > 0 ? (size_t)e->tune.smem_per_cta : kDefaultSmem[m];
        for (int s = 0; s < ns && modes[m]; ++s) {
            if (segs[s].empty_periods || grid_mode[seg_grid[s]][m] == 0) continue;
            const size_t need = screen_bytes(m, segs[s].d.hist_len) + 16 +
                                period_bytes(m, segs[s].d.hist_len);
            if (need > sm) sm = need;
        }
        sm = (sm + 15) & ~size_t(15);
        // the opt-in limit covers the kernel's static shared state too
        const size_t limit = modes[m] ? e->smem_optin + 1024 - search_static_smem(m) : 0;
        if (modes[m] && sm > limit)
            return fail(BLS_E_RESOURCE,
                        "BLS: %zu bytes of shared memory per CTA exceed the device's %zu "
                        "(a period of the widest segment, or BlsTune.smem_per_cta); narrow "
                        "the period range (max_period_days)",
                        sm, limit);
        smem_mode[m] = sm;
    }
    // per mode: one group per grid with curves of that mode -- the grid's tile
    // prefix and its curves largest first -- groups in decreasing cost per curve
    // (so the last work items of a launch are the cheapest)
    std::vector<WorkGroup> plan_groups[kModes];
    std::vector<int32_t> plan_tiles[kModes], plan_cap[kModes], plan_order[kModes];
    int64_t n_items_mode[kModes] = {0, 0, 0};
    std::vector<std::vector<int32_t>> members(n_grids);
    for (int m = 0; m < kModes; ++m) {
        plan_cap[m].assign(std::max(ns, 1), 1);
        if (!modes[m]) continue;
        for (auto& v : members) v.clear();
        for (int c = 0; c < nc; ++c)
            if (curves[c].d.mode == m) members[gid[c]].push_back(c);
        struct Cand {
            int grid;
            int64_t tiles;
            double cost;
            std::vector<int32_t> prefix;
        };
        std::vector<Cand> cands;
        for (int k = 0; k < n_grids; ++k) {
            if (members[k].empty()) continue;
            Cand q{k, 0, 0.0, std::vector<int32_t>(grids[k].n_segments + 1, 0)};
            int64_t acc = 0;
            for (int sl = 0; sl < grids[k].n_segments; ++sl) {
                const int s = sbase[k] + sl;
                q.prefix[sl] = (int32_t)acc;
                if (segs[s].empty_periods) continue;
                const int cap = tile_cap(m, segs[s].d.hist_len, smem_mode[m], e->tune.max_tile);
                if (cap < 1) return fail(BLS_E_RESOURCE, "segment %d does not fit shared memory", s);
                plan_cap[m][s] = cap;
                acc += (segs[s].d.n_periods + cap - 1) / cap;
                if (acc > INT32_MAX) return fail(BLS_E_RESOURCE, "too many period tiles per curve");
            }
            q.prefix[grids[k].n_segments] = (int32_t)acc;
            q.tiles = acc;
            if (acc == 0) continue;                  // no trial period: nothing to search
            std::stable_sort(members[k].begin(), members[k].end(), [&](int x, int y) {
                return curves[x].d.n_points > curves[y].d.n_points;
            });
            q.cost = (double)curves[members[k][0]].d.n_points *
                     (double)(pbase[k + 1] - pbase[k]);
            cands.push_back(std::move(q));
        }
        std::stable_sort(cands.begin(), cands.end(),
                         [](const Cand& x, const Cand& y) { return x.cost > y.cost; });
        int64_t items = 0;
        for (const Cand& q : cands) {
            WorkGroup w;
            w.item_begin = (int32_t)items;
            w.tiles_per_curve = (int32_t)q.tiles;
            w.seg_begin = sbase[q.grid];
            w.n_segments = grids[q.grid].n_segments;
            w.order_begin = (int32_t)plan_order[m].size();
            w.tiles_begin = (int32_t)plan_tiles[m].size();
            plan_groups[m].push_back(w);
            plan_tiles[m].insert(plan_tiles[m].end(), q.prefix.begin(), q.prefix.end());
            plan_order[m].insert(plan_order[m].end(), members[q.grid].begin(),
                                 members[q.grid].end());
            items += q.tiles * (int64_t)members[q.grid].size();
            if (items > INT32_MAX)
                return fail(BLS_E_RESOURCE,
                            "%lld work items exceed one launch; split the batch into fewer curves",
                            (long long)items);
        }
        n_items_mode[m] = items;
    }
    double folds = 0.0, boxes = 0.0, trials = 0.0;
    for (int c = 0; c < nc; ++c) {
        const int k = gid[c];
        folds += (double)curves[c].d.n_points * (double)(pbase[k + 1] - pbase[k]);
        boxes += grid_boxes[k];
        trials += grid_trials[k];
    }

    // ---- stage metadata and upload ---------------------------------------------
    const int64_t n_items = n_items_mode[0] + n_items_mode[1] + n_items_mode[2];
    const size_t grid_bytes = (size_t)P_total * (8 + 8 + 4 + 4) + dur_all.size() * 4 + 64;
    // descriptors, per-curve spectrum offsets and grid bases (int64), then per
    // mode: groups, order, seg_tiles and seg_cap (int32 words)
    size_t plan_words = 0;
    for (int m = 0; m < kModes; ++m)
        plan_words += plan_groups[m].size() * (sizeof(WorkGroup) / 4) + plan_order[m].size() +
                      plan_tiles[m].size() + plan_cap[m].size();
    const size_t meta_bytes = sizeof(CurveDesc) * nc + sizeof(SegmentDesc) * std::max(ns, 1) +
                              sizeof(int64_t) * (2 * (size_t)nc + 1) +
                              sizeof(int32_t) * plan_words + 64;
    if ((rc = e->h_grid.ensure(grid_bytes))) return rc;
    if ((rc = e->h_meta.ensure(meta_bytes))) return rc;
    char* gp = e->h_grid.as<char>();
    double* hper = reinterpret_cast<double*>(gp);
    double* hfreq = hper + P_total;
    uint32_t* hscale = reinterpret_cast<uint32_t*>(hfreq + P_total);
    int32_t* hnb = reinterpret_cast<int32_t*>(hscale + P_total);
    int32_t* hdur = hnb + P_total;
    for (int64_t i = 0; i < P_total; ++i) {
        hper[i] = per[i];
        hfreq[i] = pc[i].f;
        hscale[i] = pc[i].S;
        hnb[i] = pc[i].nb;
    }
    std::copy(dur_all.begin(), dur_all.end(), hdur);
    char* mp = e->h_meta.as<char>();
    CurveDesc* hcur = reinterpret_cast<CurveDesc*>(mp);
    SegmentDesc* hseg = reinterpret_cast<SegmentDesc*>(hcur + nc);
    int64_t* hspec = reinterpret_cast<int64_t*>(hseg + std::max(ns, 1));
    int64_t* hgbase = hspec + nc + 1;
    int32_t* hplan = reinterpret_cast<int32_t*>(hgbase + nc);
    for (int c = 0; c < nc; ++c) hcur[c] = curves[c].d;
    for (int s = 0; s < ns; ++s) hseg[s] = segs[s].d;
    std::copy(spec_off.begin(), spec_off.end(), hspec);
    for (int c = 0; c < nc; ++c) hgbase[c] = pbase[gid[c]];
    size_t plan_off[kModes][4];     // per mode: groups, order, seg_tiles, seg_cap (in words)
    {
        size_t w = 0;
        for (int m = 0; m < kModes; ++m) {
            plan_off[m][0] = w;
            std::memcpy(hplan + w, plan_groups[m].data(), plan_groups[m].size() * sizeof(WorkGroup));
            w += plan_groups[m].size() * (sizeof(WorkGroup) / 4);
            plan_off[m][1] = w;
            std::copy(plan_order[m].begin(), plan_order[m].end(), hplan + w);
            w += plan_order[m].size();
            plan_off[m][2] = w;
            std::copy(plan_tiles[m].begin(), plan_tiles[m].end(), hplan + w);
            w += plan_tiles[m].size();
            plan_off[m][3] = w;
            std::copy(plan_cap[m].begin(), plan_cap[m].end(), hplan + w);
            w += plan_cap[m].size();
        }
    }
    for (int m = 0; m < kModes; ++m) e->n_items_mode[m] = (int32_t)n_items_mode[m];

    const size_t out_elems = (size_t)kFields * std::max<int64_t>(spec_total, 1);
    if ((rc = e->d_tau.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->d_pay_r.ensure(sizeof(uint32_t) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->d_r64.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->d_iv64.ensure(sizeof(double) * std::max<int64_t>(n_pts, 1)))) return rc;
    if ((rc = e->d_period.ensure(grid_bytes))) return rc;
    if ((rc = e->d_curves.ensure(meta_bytes))) return rc;
    if ((rc = e->d_out.ensure(sizeof(double) * out_elems))) return rc;
    if ((rc = e->d_ctl.ensure(64))) return rc;
    int64_t h2d = 0;
    CUDA_TRY(cudaMemcpyAsync(e->d_tau.p, htau, sizeof(double) * n_pts, cudaMemcpyHostToDevice, st),
             "upload times");
    CUDA_TRY(cudaMemcpyAsync(e->d_pay_r.p, hpr, sizeof(uint32_t) * n_pts, cudaMemcpyHostToDevice,
                             st),
             "upload flux words");
    h2d += (int64_t)n_pts * 12;
    if (n_uniform < nc) {               // FP64 or fixed-point per-point values
        CUDA_TRY(cudaMemcpyAsync(e->d_r64.p, hr64, sizeof(double) * n_pts, cudaMemcpyHostToDevice,
                                 st),
                 "upload flux*weight");
        CUDA_TRY(cudaMemcpyAsync(e->d_iv64.p, hiv64, sizeof(double) * n_pts,
                                 cudaMemcpyHostToDevice, st),
                 "upload weights");
        h2d += (int64_t)n_pts * 16;
    }
    CUDA_TRY(cudaMemcpyAsync(e->d_period.p, gp, grid_bytes, cudaMemcpyHostToDevice, st),
             "upload grid");
    CUDA_TRY(cudaMemcpyAsync(e->d_curves.p, mp, meta_bytes, cudaMemcpyHostToDevice, st),
             "upload descriptors");
    h2d += (int64_t)(grid_bytes + meta_bytes);
    CUDA_TRY(cudaMemsetAsync(e->d_ctl.p, 0, 64, st), "reset control words");
    for (int m = 0; m < kModes; ++m)
        if (modes[m]) CUDA_TRY(configure_search(m, smem_mode[m]), "shared-memory opt-in");

    const char* dgp = e->d_period.as<char>();
    const double* dper = reinterpret_cast<const double*>(dgp);
    const double* dfreq = dper + P_total;
    const uint32_t* dscale = reinterpret_cast<const uint32_t*>(dfreq + P_total);
    const int32_t* dnb = reinterpret_cast<const int32_t*>(dscale + P_total);
    const int32_t* ddur = dnb + P_total;
    const char* dmp = e->d_curves.as<char>();
    const CurveDesc* dcur = reinterpret_cast<const CurveDesc*>(dmp);
    const SegmentDesc* dseg = reinterpret_cast<const SegmentDesc*>(dcur + nc);
    const int64_t* dspec = reinterpret_cast<const int64_t*>(dseg + std::max(ns, 1));
    const int64_t* dgbase = dspec + nc + 1;
    const int32_t* dplan = reinterpret_cast<const int32_t*>(dgbase + nc);
    int32_t* ctl = e->d_ctl.as<int32_t>();
    int ctas_total = 0;
    for (int m = 0; m < kModes; ++m) {
        BatchArgs& a = e->args[m];
        a.curves = dcur;
        a.segments = dseg;
        a.groups = reinterpret_cast<const WorkGroup*>(dplan + plan_off[m][0]);
        a.n_groups = (int32_t)plan_groups[m].size();
        a.group0 = plan_groups[m].empty() ? WorkGroup{} : plan_groups[m][0];
        a.order = dplan + plan_off[m][1];
        a.seg_tiles = dplan + plan_off[m][2];
        a.seg_cap = dplan + plan_off[m][3];
        a.n_items = e->n_items_mode[m];
        a.tau = e->d_tau.as<double>();
        a.pay_r = e->d_pay_r.as<uint32_t>();
        a.r64 = e->d_r64.as<double>();
        a.iv64 = e->d_iv64.as<double>();
        a.period = dper;
        a.freq = dfreq;
        a.scale = dscale;
        a.nbins = dnb;
        a.dur_bins = ddur;
        a.out = e->d_out.as<double>();
        a.out_stride = spec_total;
        a.work_counter = ctl + m;
        a.error_flag = ctl + 8;
        a.debug_prefix = nullptr;
        a.obj_flag = grids[0].objective;
        const int per_sm = std::max(1, max_resident_ctas(m, smem_mode[m]));
        e->ctas_mode[m] = std::min(a.n_items, e->n_sm * per_sm);
        ctas_total = std::max(ctas_total, e->ctas_mode[m]);
    }
    int64_t max_periods = 0;
    for (int k = 0; k < n_grids; ++k) max_periods = std::max(max_periods, pbase[k + 1] - pbase[k]);
    for (int m = 0; m < kModes; ++m) e->smem_mode[m] = smem_mode[m];
    e->n_curves = nc;
    e->n_grids = n_grids;
    e->spec_total = spec_total;
    e->max_periods = max_periods;
    e->grid_pbase = pbase;
    e->spec_off = spec_off;
    e->d_spec_off = dspec;
    e->d_grid_base = dgbase;
    BlsBatchInfo& in = e->info;
    in.n_curves = nc;
    in.n_segments = ns;
    in.n_periods = max_periods;
    in.n_items = (int64_t)n_items;
    in.n_points = n_pts;
    in.folds = folds;
    in.boxes = boxes;
    in.trials = trials;
    in.h2d_bytes = h2d;
    in.ctas = ctas_total;
    in.smem_per_cta = (int32_t)(modes[0] ? smem_mode[0] : modes[2] ? smem_mode[2] : smem_mode[1]);
    in.uniform_curves = n_uniform;
    in.fast_fold_segments = fast_segments;
    in.spectrum = spec_total;
    in.n_grids = n_grids;
    in.reserved = 0;
    e->prepared = true;
    return BLS_OK;
}

// Enqueue one search (both accumulation modes) on `st`.
int enqueue_search(BlsEngine* e, cudaStream_t st) {
    // the work counters (words 0..kModes-1) and the error flag (word 8): every
    // search starts clean, so BLS_E_DEVICE reports this search's descriptors only
    CUDA_TRY(cudaMemsetAsync(e->d_ctl.p, 0, 64, st), "reset work counters and error flag");
    for (int m = 0; m < kModes; ++m) {
        if (e->args[m].n_items <= 0) continue;
        CUDA_TRY(launch_search(e->args[m], m, e->ctas_mode[m], e->smem_mode[m], st),
                 "search launch");
    }
    return BLS_OK;
}

int check_device_flag(BlsEngine* e, cudaStream_t st) {
    int rc;
    if ((rc = e->h_ctl.ensure(64))) return rc;
    int32_t* h = e->h_ctl.as<int32_t>();
    CUDA_TRY(cudaMemcpyAsync(h, e->d_ctl.as<int32_t>() + 8, sizeof(int32_t), cudaMemcpyDeviceToHost,
                             st),
             "read error flag");
    CUDA_TRY(cudaStreamSynchronize(st), "synchronize");
    if (h[0] != 0) return fail(BLS_E_DEVICE, "a kernel met an impossible work descriptor");
    return BLS_OK;
}

// ---- joint-ephemeris multi-band search ----------------------------------------

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// One star's bands, prepared as joint_bands does (_bls_joint.py:94-135): one time
// origin for every band, each band centred on its own median, y*ivar and ivar
// quantised to 64-bit fixed point with one power-of-two scale per band.
int pack_joint_bands(const BlsCurves* bv, double* tau, long long* qy, long long* qi,
                     uint8_t* band_of, JointBand* jb, double* t_min_out) {
    const int K = bv->n_curves;
    double t_min = INFINITY;
    for (int k = 0; k < K; ++k) {
        const int64_t b = bv->offsets[k], e = bv->offsets[k + 1];
        if (e - b < 1) return fail(BLS_E_INVALID, "band %d has no points", k);
        if (e - b > INT32_MAX) return fail(BLS_E_INVALID, "band %d has too many points", k);
        for (int64_t j = b; j < e; ++j) {
            if (!std::isfinite(bv->t[j]) || !std::isfinite(bv->y[j]) ||
                (bv->dy && !(std::isfinite(bv->dy[j]) && bv->dy[j] > 0.0)))
                return fail(BLS_E_INVALID,
                            "band %d: times, fluxes and errors must be finite (errors > 0)", k);
            t_min = std::min(t_min, bv->t[j]);
        }
    }
    std::vector<double> scratch, yw, iv;
    for (int k = 0; k < K; ++k) {
        const int64_t b = bv->offsets[k], n = bv->offsets[k + 1] - b;
        const double med = median_of(bv->y + b, n, scratch);
        yw.resize(n);
        iv.resize(n);
        double abs_y = 0.0, abs_i = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            tau[b + j] = bv->t[b + j] - t_min;
            iv[j] = bv->dy ? 1.0 / (bv->dy[b + j] * bv->dy[b + j]) : 1.0;
            yw[j] = (bv->y[b + j] - med) * iv[j];
            abs_y += std::fabs(yw[j]);
            abs_i += iv[j];
        }
        // scale so that the sum of magnitudes stays below 2^61: the wrap pad at
        // most doubles a prefix sum, so every prefix sum and box sum fits an int64
        auto exponent = [](double total) {
            if (!(total > 0.0) || !std::isfinite(total)) return 0;
            int x = 0;
            std::frexp(total * (1.0 + 1e-12), &x);          // total < 2^x
            return std::max(-1000, std::min(1000, 61 - x));
        };
        const int e_y = exponent(abs_y), e_i = exponent(abs_i);
        long long qi_total = 0;
        for (int64_t j = 0; j < n; ++j) {
            qy[b + j] = std::llrint(std::ldexp(yw[j], e_y));
            qi[b + j] = std::llrint(std::ldexp(iv[j], e_i));
            qi_total += qi[b + j];
            band_of[b + j] = (uint8_t)k;
        }
        JointBand& d = jb[k];
        std::memset(&d, 0, sizeof(d));
        d.point_off = b;
        d.n_points = (int32_t)n;
        d.sum_y = pairwise_sum(yw.data(), n);
        d.sum_ivar = pairwise_sum(iv.data(), n);
        double floor_v = 4.0 * (double)n * DBL_EPSILON * d.sum_ivar;   // _ivar_floor
        if (!(floor_v > 0.0)) floor_v = DBL_MIN;
        d.ivar_floor = floor_v;
        d.y_unit = std::ldexp(1.0, -e_y);
        d.i_unit = std::ldexp(1.0, -e_i);
        // a box holding every quantum of the band's weight: the kernel's FP64
        // floor test on it, operation for operation (the product is exact)
        d.qi_total = qi_total;
        const double iv_all = (double)qi_total * d.i_unit;
        const double out_all = d.sum_ivar - iv_all;
        d.full_skip = (iv_all < d.ivar_floor || out_all < d.ivar_floor) ? 1 : 0;
        // screen constants (the kernel's joint_screen); out of range or NaN
        // turns the screen off for the star
        const double ybar = d.sum_ivar > 0.0 ? d.sum_y / d.sum_ivar : NAN;
        d.ybar_n = (float)(ybar * d.i_unit / d.y_unit);
        d.s_n = (float)(d.sum_ivar / std::ldexp(d.i_unit, 61));
        d.c_n = (float)std::ldexp(d.y_unit * d.y_unit / d.i_unit, 61);
        d.floor_n = std::nextafter((float)(d.ivar_floor / std::ldexp(d.i_unit, 61)), INFINITY);
    }
    *t_min_out = t_min;
    return BLS_OK;
}

// The FP32 screen needs every band's constants well inside FP32's range.
bool joint_screen_ok(const JointBand* jb, int K) {
    for (int k = 0; k < K; ++k) {
        const double ybar = jb[k].ybar_n, sn = jb[k].s_n, cn = jb[k].c_n;
        if (!std::isfinite(ybar) || std::fabs(ybar) > 1e30) return false;
        if (!(sn > 1e-30 && sn <= 2.0)) return false;
        if (!(cn > 1e-30 && cn < 1e30)) return false;
    }
    return true;
}

int do_prepare_joint(BlsEngine* e, const BlsGrid* g, const BlsCurves* bv, cudaStream_t st) {
    if (!g || !bv) return fail(BLS_E_INVALID, "grid and bands are required");
    e->joint_prepared = false;
    if (g->n_segments < 0 || (g->n_segments > 0 && (!g->seg_offsets || !g->dur_offsets)))
        return fail(BLS_E_INVALID, "bad segment table");
    if (g->oversample < 1) return fail(BLS_E_INVALID, "oversample must be >= 1");
    if (g->objective != 0 && g->objective != 1)
        return fail(BLS_E_INVALID, "objective must be 'snr' or 'likelihood'");
    const int K = bv->n_curves;
    if (K < 1 || !bv->offsets || !bv->t || !bv->y)
        return fail(BLS_E_INVALID, "at least one band is required");
    if (K > kMaxJointBands)
        return fail(BLS_E_INVALID, "at most %d bands per star", kMaxJointBands);
    if (bv->offsets[0] != 0) return fail(BLS_E_INVALID, "offsets[0] must be 0");
    const int ns = g->n_segments;
    const int o = g->oversample;
    if (ns > 0 && g->seg_offsets[0] != 0) return fail(BLS_E_INVALID, "seg_offsets[0] must be 0");
    const int64_t P_total = ns > 0 ? g->seg_offsets[ns] : 0;
    const int64_t n_pts = bv->offsets[K];
    if (P_total > INT32_MAX - (1 << 22)) return fail(BLS_E_RESOURCE, "too many trial periods");
    if (n_pts > INT32_MAX - (1 << 22)) return fail(BLS_E_INVALID, "too many points in one star");

    // the star's largest time offset bounds the fast fold's error
    double t_lo = INFINITY, t_hi = -INFINITY;
    for (int64_t j = 0; j < n_pts; ++j) {
        t_lo = std::min(t_lo, bv->t[j]);
        t_hi = std::max(t_hi, bv->t[j]);
    }
    const double tau_max = n_pts > 0 && std::isfinite(t_hi - t_lo) ? t_hi - t_lo : 0.0;

    // ---- segments (_segment, _bls_joint.py:138-144; _duration_bins) -------------
    std::vector<JointSegment> segs(std::max(ns, 1));
    std::vector<int32_t> nbins(P_total), dur_all;
    std::vector<double> freq(P_total);
    std::vector<uint32_t> scale(P_total, 0u);
    int64_t hist_stride = 2;
    for (int s = 0; s < ns; ++s) {
        const int64_t p0 = g->seg_offsets[s], p1 = g->seg_offsets[s + 1];
        const int64_t d0 = g->dur_offsets[s], d1 = g->dur_offsets[s + 1];
        if (p1 < p0 || d1 < d0) return fail(BLS_E_INVALID, "segment %d: bad offsets", s);
        JointSegment& sd = segs[s];
        std::memset(&sd, 0, sizeof(sd));
        sd.period_off = p0;
        sd.n_periods = (int32_t)(p1 - p0);
        sd.oversample = o;
        sd.dur_off = (int32_t)dur_all.size();
        if (p1 == p0) continue;
        if (d1 == d0) return fail(BLS_E_INVALID, "segment %d has no durations", s);
        double dmin = INFINITY, pmax = 0.0;
        for (int64_t i = d0; i < d1; ++i) {
            const double d = g->durations[i];
            if (!(std::isfinite(d) && d > 0.0))
                return fail(BLS_E_INVALID, "segment %d: durations must be finite and > 0", s);
            dmin = std::min(dmin, d);
        }
        for (int64_t i = p0; i < p1; ++i) {
            const double P = g->periods[i];
            if (!(std::isfinite(P) && P > 0.0))
                return fail(BLS_E_INVALID,
                            "BLS: trial periods must be finite and > 0 (segment %d)", s);
            pmax = std::max(pmax, P);
        }
        const double bin = dmin / (double)o;
        std::vector<int32_t> dur;
        for (int64_t i = d0; i < d1; ++i) {
            const double kd = std::floor(g->durations[i] / bin + 0.5);
            if (kd >= 1.0 && kd < 2147483647.0) {
                const int32_t k = (int32_t)kd;
                if (std::find(dur.begin(), dur.end(), k) == dur.end()) dur.push_back(k);
            }
        }
        if ((int)dur.size() > kMaxDur)
            return fail(BLS_E_INVALID, "segment %d: more than %d distinct box widths", s, kMaxDur);
        const double wmax = std::ceil(pmax / bin) + (double)o + 1.0;
        if (!(wmax < 1073741824.0))
            return fail(BLS_E_RESOURCE, "segment %d: %.3g phase bins per period", s, wmax);
        const int64_t width = (int64_t)wmax;
        int64_t hl = 2;
        for (int64_t i = p0; i < p1; ++i) {
            const int64_t nb = period_bins(g->periods[i], bin, o, width);
            nbins[i] = (int32_t)nb;
            hl = std::max(hl, nb + 1);
        }
        sd.width = (int32_t)width;
        sd.bin_duration = bin;
        sd.n_dur = (int32_t)dur.size();
        sd.hist_len = (int32_t)hl;
        hist_stride = std::max(hist_stride, hl);
        dur_all.insert(dur_all.end(), dur.begin(), dur.end());
        // fast fold, with the single-band search's margins and checks
        double fmax = 0.0, smax = 0.0;
        for (int64_t i = p0; i < p1; ++i) {
            fmax = std::max(fmax, 1.0 / g->periods[i]);
            smax = std::max(smax, g->periods[i] / bin);
        }
        FoldParams fp = fold_params(width, bin, tau_max, fmax, smax);
        const double sc_unit = std::ldexp(1.0, fp.fb);
        for (int64_t i = p0; i < p1 && fp.fast; ++i) {
            const double sc = std::nearbyint((g->periods[i] / bin) * sc_unit);
            if (!(sc >= 1.0 && sc < 4294967296.0)) { fp.fast = false; break; }
            // the fast fold's largest bin, ((S - 1) >> fb) + 1, must stay inside n_bins
            if ((int64_t)(((uint32_t)sc - 1u) >> fp.fb) + 1 > nbins[i]) { fp.fast = false; break; }
        }
        for (int64_t i = p0; i < p1; ++i) {
            freq[i] = 1.0 / g->periods[i];
            scale[i] = fp.fast ? (uint32_t)std::nearbyint((g->periods[i] / bin) * sc_unit) : 0u;
        }
        sd.fast_fold = fp.fast ? 1 : 0;
        sd.frac_bits = fp.fast ? fp.fb : 0;
        sd.margin_u = fp.mu;
        sd.margin_phi = fp.mphi;
    }
    if (P_total == 0) {
        e->joint_periods = 0;
        e->joint_prepared = true;
        return BLS_OK;
    }

    // ---- where the histograms live ---------------------------------------------
    const size_t hist_bytes = (size_t)2 * K * hist_stride * sizeof(long long);
    const bool in_smem = hist_bytes + joint_static_smem() + 1024 <= e->smem_optin;
    if (in_smem) CUDA_TRY(configure_joint(hist_bytes), "shared-memory opt-in");
    const int per_sm = std::max(1, joint_resident_ctas(in_smem, in_smem ? hist_bytes : 0));
    int ctas = (int)std::min<int64_t>(P_total, (int64_t)e->n_sm * per_sm);

    // ---- stage and upload (one copy) -------------------------------------------
    const size_t o_tau = 0;
    const size_t o_qy = o_tau + align256(8 * (size_t)n_pts);
    const size_t o_qi = o_qy + align256(8 * (size_t)n_pts);
    const size_t o_bof = o_qi + align256(8 * (size_t)n_pts);
    const size_t o_band = o_bof + align256((size_t)n_pts);
    const size_t o_seg = o_band + align256(sizeof(JointBand) * K);
    const size_t o_per = o_seg + align256(sizeof(JointSegment) * segs.size());
    const size_t o_freq = o_per + align256(8 * (size_t)P_total);
    const size_t o_scale = o_freq + align256(8 * (size_t)P_total);
    const size_t o_nb = o_scale + align256(4 * (size_t)P_total);
    const size_t o_dur = o_nb + align256(4 * (size_t)P_total);
    const size_t staged = o_dur + align256(4 * std::max<size_t>(dur_all.size(), 1));
    const size_t o_out = staged;
    const size_t o_ctl = o_out + align256(8 * (size_t)kJointFields * P_total);
    const size_t o_scr = o_ctl + 256;
    const size_t total = o_scr + (in_smem ? 0 : (size_t)ctas * hist_bytes);
    int rc;
    if ((rc = e->h_joint.ensure(std::max(staged, (size_t)8 * kJointFields * P_total)))) return rc;
    char* h = e->h_joint.as<char>();
    double t_min = 0.0;
    if ((rc = pack_joint_bands(bv, reinterpret_cast<double*>(h + o_tau),
                               reinterpret_cast<long long*>(h + o_qy),
                               reinterpret_cast<long long*>(h + o_qi),
                               reinterpret_cast<uint8_t*>(h + o_bof),
                               reinterpret_cast<JointBand*>(h + o_band), &t_min)))
        return rc;
    std::memcpy(h + o_seg, segs.data(), sizeof(JointSegment) * segs.size());
    std::memcpy(h + o_per, g->periods, 8 * (size_t)P_total);
    std::memcpy(h + o_freq, freq.data(), 8 * (size_t)P_total);
    std::memcpy(h + o_scale, scale.data(), 4 * (size_t)P_total);
    std::memcpy(h + o_nb, nbins.data(), 4 * (size_t)P_total);
    if (!dur_all.empty()) std::memcpy(h + o_dur, dur_all.data(), 4 * dur_all.size());
    if ((rc = e->d_joint.ensure(total))) return rc;
    char* d = e->d_joint.as<char>();
    CUDA_TRY(cudaMemcpyAsync(d, h, staged, cudaMemcpyHostToDevice, st), "upload bands");
    CUDA_TRY(cudaMemsetAsync(d + o_ctl, 0, 256, st), "reset control words");

    JointArgs a{};
    a.tau = reinterpret_cast<const double*>(d + o_tau);
    a.qy = reinterpret_cast<const long long*>(d + o_qy);
    a.qi = reinterpret_cast<const long long*>(d + o_qi);
    a.band_of = reinterpret_cast<const uint8_t*>(d + o_bof);
    a.bands = reinterpret_cast<const JointBand*>(d + o_band);
    a.segments = reinterpret_cast<const JointSegment*>(d + o_seg);
    a.period = reinterpret_cast<const double*>(d + o_per);
    a.freq = reinterpret_cast<const double*>(d + o_freq);
    a.scale = reinterpret_cast<const uint32_t*>(d + o_scale);
    a.nbins = reinterpret_cast<const int32_t*>(d + o_nb);
    a.dur_bins = reinterpret_cast<const int32_t*>(d + o_dur);
    a.out = reinterpret_cast<double*>(d + o_out);
    a.n_periods = P_total;
    a.scratch = in_smem ? nullptr : reinterpret_cast<long long*>(d + o_scr);
    a.hist_stride = hist_stride;
    a.work_counter = reinterpret_cast<int32_t*>(d + o_ctl);
    a.error_flag = reinterpret_cast<int32_t*>(d + o_ctl) + 8;
    a.t_min = t_min;
    a.n_points = (int32_t)n_pts;
    a.screen = joint_screen_ok(reinterpret_cast<const JointBand*>(h + o_band), K) ? 1 : 0;
    a.n_bands = K;
    a.n_segments = ns;
    a.obj_flag = g->objective;
    e->jargs = a;
    e->joint_in_smem = in_smem;
    e->joint_smem = in_smem ? hist_bytes : 0;
    e->joint_ctas = ctas;
    e->joint_periods = P_total;
    e->joint_prepared = true;
    return BLS_OK;
}

int do_launch_joint(BlsEngine* e, cudaStream_t st) {
    if (!e->joint_prepared) return fail(BLS_E_STATE, "bls_joint_launch before bls_joint_prepare");
    if (e->joint_periods == 0) return BLS_OK;
    CUDA_TRY(cudaMemsetAsync(e->jargs.work_counter, 0, 64, st), "reset control words");
    CUDA_TRY(launch_joint(e->jargs, e->joint_in_smem, e->joint_smem, e->joint_ctas, st),
             "joint search launch");
    return BLS_OK;
}

int do_download_joint(BlsEngine* e, double* out, cudaStream_t st) {
    if (!e->joint_prepared) return fail(BLS_E_STATE, "bls_joint_download before bls_joint_prepare");
    const int64_t P = e->joint_periods;
    if (P == 0) return BLS_OK;
    int rc;
    if ((rc = e->h_ctl.ensure(64))) return rc;
    int32_t* hflag = e->h_ctl.as<int32_t>();
    const size_t bytes = 8 * (size_t)kJointFields * P;
    // the staging buffer holds at least this much (do_prepare_joint)
    char* h = e->h_joint.as<char>();
    CUDA_TRY(cudaMemcpyAsync(h, e->jargs.out, bytes, cudaMemcpyDeviceToHost, st),
             "download joint fields");
    CUDA_TRY(cudaMemcpyAsync(hflag, e->jargs.error_flag, sizeof(int32_t), cudaMemcpyDeviceToHost,
                             st),
             "read error flag");
    CUDA_TRY(cudaStreamSynchronize(st), "synchronize");
    if (hflag[0] != 0)
        return fail(BLS_E_DEVICE, "the joint search met an impossible descriptor (flag %d)",
                    hflag[0]);
    std::memcpy(out, h, bytes);
    return BLS_OK;
}

// ---- transit least squares ----------------------------------------------------

int do_prepare_tls(BlsEngine* e, const BlsTlsInputs* in, const double* periods, int64_t P,
                   cudaStream_t st) {
    e->tls_prepared = false;
    if (!in || (P > 0 && !periods)) return fail(BLS_E_INVALID, "inputs are required");
    const int nc = in->n_curves;
    if (nc < 1 || !in->offsets || !in->tau || !in->yw || !in->w || !in->w_total)
        return fail(BLS_E_INVALID, "at least one light curve is required");
    if (in->offsets[0] != 0) return fail(BLS_E_INVALID, "offsets[0] must be 0");
    const int nb = in->n_bins, nd = in->n_dur;
    if (nb < 2 || nb > (1 << 20)) return fail(BLS_E_INVALID, "n_bins must be in [2, 2^20]");
    if (nd < 1 || nd > kTlsMaxDur || !in->dur_bins || !in->templates)
        return fail(BLS_E_INVALID, "1 to %d template widths are required", kTlsMaxDur);
    int max_w = 1, n_tmpl = 0;
    for (int d = 0; d < nd; ++d) {
        const int w = in->dur_bins[d];
        if (w < 1 || w > nb - 1)
            return fail(BLS_E_INVALID, "template width %d outside [1, n_bins - 1]", w);
        max_w = std::max(max_w, w);
        n_tmpl += w;
    }
    for (int i = 0; i < n_tmpl; ++i)
        if (!std::isfinite(in->templates[i]))
            return fail(BLS_E_INVALID, "templates must be finite");
    if (!(in->den_rel >= 0.0) || !std::isfinite(in->den_rel))
        return fail(BLS_E_INVALID, "den_rel must be finite and >= 0");
    for (int64_t i = 0; i < P; ++i)
        if (!(std::isfinite(periods[i]) && periods[i] > 0.0))
            return fail(BLS_E_INVALID, "TLS: trial periods must be finite and > 0");
    if (P > INT32_MAX - (1 << 22)) return fail(BLS_E_RESOURCE, "too many trial periods");
    const int64_t n_pts = in->offsets[nc];
    for (int c = 0; c < nc; ++c) {
        const int64_t b = in->offsets[c], en = in->offsets[c + 1];
        if (en - b < 1 || en - b > kTlsMaxPoints)
            return fail(BLS_E_INVALID, "light curve %d: TLS needs 1 to %d points", c,
                        kTlsMaxPoints);
        if (!(std::isfinite(in->w_total[c]) && in->w_total[c] > 0.0))
            return fail(BLS_E_INVALID, "light curve %d: w_total must be finite and > 0", c);
        for (int64_t j = b; j < en; ++j)
            if (!std::isfinite(in->tau[j]) || !std::isfinite(in->yw[j]) ||
                !(std::isfinite(in->w[j]) && in->w[j] >= 0.0))
                return fail(BLS_E_INVALID,
                            "light curve %d: tau, yw and w must be finite (w >= 0)", c);
    }
    if (P == 0) {
        e->tls_out_bytes = 0;
        e->tls_prepared = true;
        return BLS_OK;
    }

    // one work item: a tile of periods, each one histogram of n_bins + max_w - 1 bins
    const int ext = nb + max_w - 1;
    const int64_t per_period = 16 * (int64_t)ext + 16 * (int64_t)nb;
    int tile = (int)std::max<int64_t>(1, (64 * 1024 - 8 * (int64_t)n_tmpl) / per_period);
    tile = std::min<int>(tile, kTlsMaxTile);
    const size_t smem = tls_smem_bytes(nb, max_w, tile, n_tmpl);
    if (smem + 1024 > e->smem_optin)
        return fail(BLS_E_RESOURCE,
                    "TLS: %zu bytes of shared memory per period exceed the device's %zu; "
                    "lower n_phase_bins", smem, e->smem_optin);
    const int64_t tiles = (P + tile - 1) / tile;
    if (tiles * nc > INT32_MAX - (1 << 22))
        return fail(BLS_E_RESOURCE, "too many work items; split the batch");

    // staging: descriptors, points (chunked layout), grid, templates
    const size_t o_cur = 0;
    const size_t o_tau = o_cur + align256(sizeof(TlsCurveDesc) * nc);
    const size_t o_qy = o_tau + align256(8 * (size_t)n_pts);
    const size_t o_qw = o_qy + align256(8 * (size_t)n_pts);
    const size_t o_per = o_qw + align256(8 * (size_t)n_pts);
    const size_t o_freq = o_per + align256(8 * (size_t)P);
    const size_t o_dur = o_freq + align256(8 * (size_t)P);
    const size_t o_off = o_dur + align256(4 * (size_t)nd);
    const size_t o_tmpl = o_off + align256(4 * (size_t)nd);
    const size_t staged = o_tmpl + align256(8 * (size_t)n_tmpl);
    const size_t out_bytes = 8 * (size_t)kTlsFields * nc * P;
    const size_t o_out = staged;
    const size_t o_ctl = o_out + align256(out_bytes);
    int rc;
    if ((rc = e->h_tls.ensure(std::max(staged, out_bytes)))) return rc;
    char* h = e->h_tls.as<char>();
    TlsCurveDesc* cd = reinterpret_cast<TlsCurveDesc*>(h + o_cur);
    double* htau = reinterpret_cast<double*>(h + o_tau);
    long long* hqy = reinterpret_cast<long long*>(h + o_qy);
    long long* hqw = reinterpret_cast<long long*>(h + o_qw);
    parallel_for(nc, [&](int c, int) {
        const int64_t b = in->offsets[c], n = in->offsets[c + 1] - b;
        // 64-bit fixed point: the magnitudes sum below 2^61
        double abs_y = 0.0, sum_w = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            abs_y += std::fabs(in->yw[b + j]);
            sum_w += in->w[b + j];
        }
        auto fixed_exp = [](double total) {
            if (!(total > 0.0) || !std::isfinite(total)) return 0;
            int x = 0;
            std::frexp(total * (1.0 + 1e-12), &x);               // total < 2^x
            return std::max(-1000, std::min(1000, 61 - x));
        };
        const int e_y = fixed_exp(abs_y), e_w = fixed_exp(sum_w);
        for (int64_t j = 0; j < n; ++j) {
            const int64_t m = b + point_slot(j, n);
            htau[m] = in->tau[b + j];
            hqy[m] = std::llrint(std::ldexp(in->yw[b + j], e_y));
            hqw[m] = std::llrint(std::ldexp(in->w[b + j], e_w));
        }
        TlsCurveDesc& d = cd[c];
        std::memset(&d, 0, sizeof(d));
        d.point_off = b;
        d.n_points = (int32_t)n;
        d.w_total = in->w_total[c];
        d.y_unit = std::ldexp(1.0, -e_y);
        d.w_unit = std::ldexp(1.0, -e_w);
    });
    std::memcpy(h + o_per, periods, 8 * (size_t)P);
    // fast fold: the phase frac(tau * RN(1/P)) on a 2^-32 grid is within e_phi
    // cycles of frac(tau / P) (RN(1/P) and the grid), the reference's
    // frac(RN(tau / P)) within e_ref, and its RN(ph * n_bins) within
    // n_bins * 2^-53 bins; the kernel takes the fast bin only further than the
    // sum from a cycle edge (mphi) and a bin edge (mu)
    double* hfreq = reinterpret_cast<double*>(h + o_freq);
    double f_max = 0.0, tau_max = 0.0;
    for (int64_t i = 0; i < P; ++i) {
        hfreq[i] = 1.0 / periods[i];
        f_max = std::max(f_max, hfreq[i]);
    }
    for (int64_t j = 0; j < n_pts; ++j) tau_max = std::max(tau_max, std::fabs(in->tau[j]));
    bool fast = false;
    uint32_t mu = 0, mphi = 0;
    {
        const double q_max = tau_max * f_max;
        bool tau_ok = true;
        for (int64_t j = 0; j < n_pts && tau_ok; ++j) tau_ok = in->tau[j] >= 0.0;
        if (tau_ok && q_max < 262144.0) {
            const double two32 = 4294967296.0;
            const double e_phi = q_max * std::ldexp(1.0, -52) * 1.01 + std::ldexp(1.0, -33);
            const double e_ref = q_max * std::ldexp(1.0, -53);
            const double m_phi = std::ceil((e_phi + e_ref) * two32) + 2.0;
            const double m_u =
                std::ceil(((double)nb * (e_phi + e_ref) + (double)nb * std::ldexp(1.0, -52)) *
                          two32) + 2.0;
            if (m_phi < 1e6 && m_u < 268435456.0) {
                fast = true;
                mu = (uint32_t)m_u;
                mphi = (uint32_t)m_phi;
            }
        }
    }
    int32_t* hoff = reinterpret_cast<int32_t*>(h + o_off);
    for (int d = 0, acc = 0; d < nd; ++d) {
        reinterpret_cast<int32_t*>(h + o_dur)[d] = in->dur_bins[d];
        hoff[d] = acc;
        acc += in->dur_bins[d];
    }
    std::memcpy(h + o_tmpl, in->templates, 8 * (size_t)n_tmpl);
    if ((rc = e->d_tls.ensure(o_ctl + 256))) return rc;
    char* d = e->d_tls.as<char>();
    CUDA_TRY(cudaMemcpyAsync(d, h, staged, cudaMemcpyHostToDevice, st), "upload TLS inputs");
    CUDA_TRY(cudaMemsetAsync(d + o_ctl, 0, 256, st), "reset control words");

    TlsArgs a{};
    a.curves = reinterpret_cast<const TlsCurveDesc*>(d + o_cur);
    a.tau = reinterpret_cast<const double*>(d + o_tau);
    a.qy = reinterpret_cast<const long long*>(d + o_qy);
    a.qw = reinterpret_cast<const long long*>(d + o_qw);
    a.period = reinterpret_cast<const double*>(d + o_per);
    a.freq = reinterpret_cast<const double*>(d + o_freq);
    a.margin_u = mu;
    a.margin_phi = mphi;
    a.fast_fold = fast ? 1 : 0;
    a.dur_bins = reinterpret_cast<const int32_t*>(d + o_dur);
    a.tmpl_off = reinterpret_cast<const int32_t*>(d + o_off);
    a.tmpl = reinterpret_cast<const double*>(d + o_tmpl);
    a.out = reinterpret_cast<double*>(d + o_out);
    a.out_stride = (int64_t)nc * P;
    a.n_periods = P;
    a.work_counter = reinterpret_cast<int32_t*>(d + o_ctl);
    a.error_flag = reinterpret_cast<int32_t*>(d + o_ctl) + 8;
    a.w_eps = 1e-300;
    a.den_rel = in->den_rel;
    a.n_curves = nc;
    a.n_bins = nb;
    a.n_dur = nd;
    a.n_tmpl = n_tmpl;
    a.max_width = max_w;
    a.tile = tile;
    a.tiles_per_curve = (int32_t)tiles;
    a.n_items = (int32_t)(tiles * nc);
    CUDA_TRY(configure_tls(smem), "shared-memory opt-in");
    const int per_sm = std::max(1, tls_resident_ctas(smem));
    e->targs = a;
    e->tls_smem = smem;
    e->tls_ctas = (int)std::min<int64_t>(a.n_items, (int64_t)e->n_sm * per_sm);
    e->tls_out_bytes = out_bytes;
    e->tls_prepared = true;
    return BLS_OK;
}

int do_launch_tls(BlsEngine* e, cudaStream_t st) {
    if (!e->tls_prepared) return fail(BLS_E_STATE, "bls_tls_launch before bls_tls_prepare");
    if (e->tls_out_bytes == 0) return BLS_OK;
    CUDA_TRY(cudaMemsetAsync(e->targs.work_counter, 0, 64, st), "reset control words");
    CUDA_TRY(launch_tls(e->targs, e->tls_ctas, e->tls_smem, st), "TLS launch");
    return BLS_OK;
}

int do_download_tls(BlsEngine* e, double* out, cudaStream_t st) {
    if (!e->tls_prepared) return fail(BLS_E_STATE, "bls_tls_download before bls_tls_prepare");
    if (e->tls_out_bytes == 0) return BLS_OK;
    int rc;
    if ((rc = e->h_ctl.ensure(64))) return rc;
    int32_t* hflag = e->h_ctl.as<int32_t>();
    // the staging buffer holds at least the output (do_prepare_tls)
    char* h = e->h_tls.as<char>();
    CUDA_TRY(cudaMemcpyAsync(h, e->targs.out, e->tls_out_bytes, cudaMemcpyDeviceToHost, st),
             "download TLS fields");
    CUDA_TRY(cudaMemcpyAsync(hflag, e->targs.error_flag, sizeof(int32_t),
                             cudaMemcpyDeviceToHost, st),
             "read error flag");
    CUDA_TRY(cudaStreamSynchronize(st), "synchronize");
    if (hflag[0] != 0) return fail(BLS_E_DEVICE, "the TLS kernel met an impossible descriptor");
    std::memcpy(out, h, e->tls_out_bytes);
    return BLS_OK;
}

// bls_prepare_default's body: one default grid per distinct baseline, built on
// the host cores, then one launch over all of them.
int prepare_default(BlsEngine* e, const BlsDefaultGrid* spec, const double* baselines,
                    const BlsCurves* cv, void* stream) {
    const int nc = cv->n_curves;
    // one grid per distinct baseline (bit pattern)
    std::unordered_map<uint64_t, int32_t> slot;
    std::vector<double> uniq;
    std::vector<int32_t> gid(nc);
    for (int c = 0; c < nc; ++c) {
        uint64_t bits;
        std::memcpy(&bits, baselines + c, sizeof bits);
        auto it = slot.emplace(bits, (int32_t)uniq.size());
        if (it.second) uniq.push_back(baselines[c]);
        gid[c] = it.first->second;
    }
    const int ng = (int)uniq.size();
    std::vector<DefaultGrid> built(ng);
    std::vector<int> codes(ng, BLS_OK);
    std::vector<std::string> msgs(ng);
    parallel_for(ng, [&](int k, int) { codes[k] = build_default_grid(*spec, uniq[k], built[k], msgs[k]); });
    std::vector<std::vector<int64_t>> dur_off(ng);
    std::vector<std::vector<double>> dur(ng);
    std::vector<BlsGrid> grids(ng);
    for (int k = 0; k < ng; ++k) {
        if (codes[k]) return fail(codes[k], "baseline %.9g: %s", uniq[k], msgs[k].c_str());
        const DefaultGrid& g = built[k];
        if (g.periods.empty())
            return fail(BLS_E_INVALID,
                        "BLS: the default grid of a %.6g-day baseline is empty (baseline too "
                        "short for the configured period range)", uniq[k]);
        dur_off[k].assign(1, 0);
        for (int32_t st : g.seg_start) {
            const int64_t d0 = spec->dur_offsets[st], d1 = spec->dur_offsets[st + 1];
            if (d1 < d0) return fail(BLS_E_INVALID, "bad duration table");
            dur[k].insert(dur[k].end(), spec->durations + d0, spec->durations + d1);
            dur_off[k].push_back((int64_t)dur[k].size());
        }
        BlsGrid& bg = grids[k];
        bg.n_segments = (int32_t)g.seg_start.size();
        bg.seg_offsets = g.seg_offsets.data();
        bg.periods = g.periods.data();
        bg.dur_offsets = dur_off[k].data();
        bg.durations = dur[k].data();
        bg.oversample = spec->oversample;
        bg.objective = spec->objective;
    }
    cudaSetDevice(e->device);
    return do_prepare(e, grids.data(), ng, gid.data(), cv, pick(e, stream));
}

}  // namespace

extern "C" {

const char* bls_last_error(void) { return g_error.c_str(); }

int bls_engine_create(const BlsTune* tune, BlsEngine** engine) {
    if (!engine) return fail(BLS_E_INVALID, "engine pointer is NULL");
    *engine = nullptr;
    BlsEngine* e = new BlsEngine();
    if (tune) e->tune = *tune;
    else {
        e->tune.device = -1;
        e->tune.use_graph = 1;
    }
    int dev = e->tune.device;
    if (dev < 0) {
        cudaError_t err = cudaGetDevice(&dev);
        if (err != cudaSuccess) { delete e; return cuda_fail(err, "no CUDA device"); }
    }
    e->device = dev;
    cudaError_t err = cudaSetDevice(dev);
    if (err != cudaSuccess) { delete e; return cuda_fail(err, "cudaSetDevice"); }
    cudaDeviceGetAttribute(&e->n_sm, cudaDevAttrMultiProcessorCount, dev);
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    e->smem_optin = (size_t)optin > 1024 ? (size_t)optin - 1024 : 0;   // static shared state
    err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess) { delete e; return cuda_fail(err, "cudaStreamCreate"); }
    *engine = e;
    return BLS_OK;
}

int bls_engine_destroy(BlsEngine* engine) {
    if (!engine) return BLS_OK;
    cudaSetDevice(engine->device);
    cudaStreamSynchronize(engine->stream);
    delete engine;
    return BLS_OK;
}

int bls_prepare(BlsEngine* e, const BlsGrid* grid, const BlsCurves* curves, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    cudaSetDevice(e->device);
    return guarded([&] { return do_prepare(e, grid, 1, nullptr, curves, pick(e, stream)); });
}

int bls_prepare_grids(BlsEngine* e, int32_t n_grids, const BlsGrid* grids,
                      const int32_t* grid_of_curve, const BlsCurves* curves, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (n_grids < 1 || !grids) return fail(BLS_E_INVALID, "at least one grid is required");
    if (n_grids > 1 && !grid_of_curve)
        return fail(BLS_E_INVALID, "grid_of_curve is required with more than one grid");
    cudaSetDevice(e->device);
    return guarded(
        [&] { return do_prepare(e, grids, n_grids, grid_of_curve, curves, pick(e, stream)); });
}

int bls_default_grid(const BlsDefaultGrid* spec, double baseline, int64_t capacity,
                     double* periods, int64_t* seg_offsets, int32_t* seg_start,
                     int32_t* n_segments, int64_t* n_periods) {
    if (!spec || !n_segments || !n_periods) return fail(BLS_E_INVALID, "bad arguments");
    DefaultGrid g;
    std::string err;
    const int rc = build_default_grid(*spec, baseline, g, err);
    if (rc) return fail(rc, "%s", err.c_str());
    *n_segments = (int32_t)g.seg_start.size();
    *n_periods = (int64_t)g.periods.size();
    if (!periods) return BLS_OK;
    if (!seg_offsets || !seg_start || capacity < *n_periods)
        return fail(BLS_E_INVALID, "the default grid needs %lld periods", (long long)*n_periods);
    std::copy(g.periods.begin(), g.periods.end(), periods);
    std::copy(g.seg_offsets.begin(), g.seg_offsets.end(), seg_offsets);
    std::copy(g.seg_start.begin(), g.seg_start.end(), seg_start);
    return BLS_OK;
}

int bls_default_grid_sizes(const BlsDefaultGrid* spec, int32_t n, const double* baselines,
                           int64_t* n_periods) {
    if (!spec || n < 0 || (n > 0 && (!baselines || !n_periods)))
        return fail(BLS_E_INVALID, "bad arguments");
    parallel_for(n, [&](int i, int) { n_periods[i] = default_grid_size(*spec, baselines[i]); });
    return BLS_OK;
}

int bls_prepare_default(BlsEngine* e, const BlsDefaultGrid* spec, const double* baselines,
                        const BlsCurves* cv, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (!spec || !baselines || !cv || cv->n_curves < 1)
        return fail(BLS_E_INVALID, "spec, baselines and curves are required");
    if (spec->n_starts < 0 || (spec->n_starts > 0 && (!spec->dur_offsets || !spec->durations)))
        return fail(BLS_E_INVALID, "bad duration table");
    return guarded([&] { return prepare_default(e, spec, baselines, cv, stream); });
}


int bls_launch(BlsEngine* e, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_launch before bls_prepare");
    cudaSetDevice(e->device);
    cudaStream_t st = pick(e, stream);
    if (!e->tune.use_graph) return enqueue_search(e, st);
    if (!e->graph_valid) {
        if (e->graph) {
            cudaGraphExecDestroy(e->graph);
            e->graph = nullptr;
        }
        // capture on the engine's own stream, ordered after the caller's stream
        cudaGraph_t g = nullptr;
        CUDA_TRY(cudaStreamSynchronize(st), "synchronize before capture");
        CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal),
                 "begin capture");
        int rc = enqueue_search(e, e->stream);
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "end capture");
        ce = cudaGraphInstantiate(&e->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(ce, "graph instantiate");
        e->graph_valid = true;
    }
    CUDA_TRY(cudaGraphLaunch(e->graph, st), "graph launch");
    return BLS_OK;
}

int bls_time_launches(BlsEngine* e, int32_t reps, double* ms_per_launch, void* stream) {
    if (!e || !ms_per_launch) return fail(BLS_E_INVALID, "engine and output are required");
    if (reps < 1) return fail(BLS_E_INVALID, "reps must be >= 1");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_time_launches before bls_prepare");
    cudaSetDevice(e->device);
    cudaStream_t st = pick(e, stream);
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (auto& x : ev)
        if (cudaEventCreate(&x) != cudaSuccess) {
            for (auto& y : ev)
                if (y) cudaEventDestroy(y);
            return cuda_fail(cudaGetLastError(), "event create");
        }
    int rc = BLS_OK;
    cudaError_t ce = cudaEventRecord(ev[0], st);
    for (int i = 0; i < reps && rc == BLS_OK && ce == cudaSuccess; ++i) rc = bls_launch(e, st);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[1], st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev[1]);
    float ms = 0.0f;
    if (rc == BLS_OK && ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (rc != BLS_OK) return rc;
    if (ce != cudaSuccess) return cuda_fail(ce, "timed launches");
    *ms_per_launch = (double)ms / reps;
    return check_device_flag(e, st);
}

int bls_download(BlsEngine* e, double* out, void* stream) {
    if (!e || !out) return fail(BLS_E_INVALID, "engine and output are required");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_download before bls_prepare");
    cudaSetDevice(e->device);
    cudaStream_t st = pick(e, stream);
    const size_t bytes = sizeof(double) * kFields * (size_t)e->spec_total;
    if (bytes) CUDA_TRY(cudaMemcpyAsync(out, e->d_out.p, bytes, cudaMemcpyDeviceToHost, st),
                        "download outputs");
    return check_device_flag(e, st);
}

int bls_download_curves(BlsEngine* e, const int32_t* curve_ids, int32_t n_ids, double* out,
                        void* stream) {
    if (!e || (n_ids > 0 && (!curve_ids || !out)) || n_ids < 0)
        return fail(BLS_E_INVALID, "engine, curve ids and output are required");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_download_curves before bls_prepare");
    for (int32_t k = 0; k < n_ids; ++k)
        if (curve_ids[k] < 0 || curve_ids[k] >= e->n_curves)
            return fail(BLS_E_INVALID, "curve id %d outside the prepared batch of %d curves",
                        (int)curve_ids[k], e->n_curves);
    cudaSetDevice(e->device);
    cudaStream_t st = pick(e, stream);
    const double* d = e->d_out.as<double>();
    size_t w = 0;
    for (int32_t k = 0; k < n_ids; ++k) {
        const int64_t b = e->spec_off[curve_ids[k]], len = e->spec_off[curve_ids[k] + 1] - b;
        for (int f = 0; f < kFields; ++f) {
            if (len > 0)
                CUDA_TRY(cudaMemcpyAsync(out + w, d + (size_t)f * e->spec_total + b,
                                         sizeof(double) * (size_t)len, cudaMemcpyDeviceToHost, st),
                         "download a curve's field");
            w += (size_t)len;
        }
    }
    return check_device_flag(e, st);
}

int bls_device_output(BlsEngine* e, const double** out) {
    if (!e || !out) return fail(BLS_E_INVALID, "engine and output are required");
    if (!e->prepared) return fail(BLS_E_STATE, "no prepared batch");
    *out = e->d_out.as<double>();
    return BLS_OK;
}

int bls_download_best(BlsEngine* e, int64_t* best_index, double* best_power, double* power_mean,
                      double* power_std, void* stream) {
    if (!e || !best_index || !best_power || !power_mean || !power_std)
        return fail(BLS_E_INVALID, "engine and outputs are required");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_download_best before bls_prepare");
    cudaSetDevice(e->device);
    cudaStream_t st = pick(e, stream);
    const int nc = e->n_curves;
    const size_t bytes = (size_t)nc * (8 * 4);
    int rc;
    if ((rc = e->d_best.ensure(bytes))) return rc;
    if ((rc = e->h_best.ensure(bytes))) return rc;
    int64_t* di = e->d_best.as<int64_t>();
    double* dv = reinterpret_cast<double*>(di + nc);
    CUDA_TRY(launch_best(e->d_out.as<double>(), nc, e->d_spec_off, di, dv, dv + nc, dv + 2 * nc,
                         st),
             "best-of-spectrum launch");
    CUDA_TRY(cudaMemcpyAsync(e->h_best.p, e->d_best.p, bytes, cudaMemcpyDeviceToHost, st),
             "download best");
    if ((rc = check_device_flag(e, st))) return rc;
    const int64_t* hi = e->h_best.as<int64_t>();
    const double* hv = reinterpret_cast<const double*>(hi + nc);
    std::memcpy(best_index, hi, sizeof(int64_t) * nc);
    std::memcpy(best_power, hv, sizeof(double) * nc);
    std::memcpy(power_mean, hv + nc, sizeof(double) * nc);
    std::memcpy(power_std, hv + 2 * nc, sizeof(double) * nc);
    return BLS_OK;
}

int bls_download_rows(BlsEngine* e, int32_t n_best, int32_t harmonic_max,
                      const double* min_separation, const double* alias_tolerance,
                      int32_t* n_peaks, int64_t* index, double* fields, void* stream) {
    if (!e || !min_separation || !alias_tolerance || !n_peaks || !index || !fields)
        return fail(BLS_E_INVALID, "engine, per-curve parameters and outputs are required");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_download_rows before bls_prepare");
    if (n_best < 1 || n_best > 1024) return fail(BLS_E_INVALID, "n_best must be in 1..1024");
    if (harmonic_max < 1 || harmonic_max > 4096)
        return fail(BLS_E_INVALID, "harmonic_max must be in 1..4096");
    const int nc = e->n_curves;
    const int64_t P = e->max_periods;
    if (P < 1) return fail(BLS_E_INVALID, "the prepared grid has no periods");
    // frequency order is reversed grid order only for strictly increasing periods
    const double* hper = e->h_grid.as<double>();
    for (int k = 0; k < e->n_grids; ++k)
        for (int64_t i = e->grid_pbase[k] + 1; i < e->grid_pbase[k + 1]; ++i)
            if (!(hper[i] > hper[i - 1]))
                return fail(BLS_E_INVALID, "rows need strictly increasing trial periods");
    const size_t mask_bytes = sizeof(uint32_t) * (size_t)((P + 31) / 32);
    if (mask_bytes + 4096 > e->smem_optin)
        return fail(BLS_E_RESOURCE, "%lld periods exceed the peak search's shared memory",
                    (long long)P);
    for (int c = 0; c < nc; ++c)
        if (!(min_separation[c] > 0.0) || !(alias_tolerance[c] > 0.0))
            return fail(BLS_E_INVALID, "separation and alias tolerance must be > 0 (curve %d)", c);
    CUDA_TRY(cudaSetDevice(e->device), "select device");
    cudaStream_t st = pick(e, stream);
    const size_t in_bytes = sizeof(double) * 2 * nc;
    const size_t idx_bytes = sizeof(int64_t) * (size_t)nc * n_best;
    const size_t fld_bytes = sizeof(double) * 8 * (size_t)nc * n_best;
    const size_t cnt_bytes = sizeof(int32_t) * (size_t)nc;
    const size_t out_bytes = idx_bytes + fld_bytes + ((cnt_bytes + 15) & ~size_t(15));
    int rc;
    if ((rc = e->d_rows.ensure(in_bytes + out_bytes))) return rc;
    if ((rc = e->h_rows.ensure(in_bytes + out_bytes))) return rc;
    char* hb = e->h_rows.as<char>();
    std::memcpy(hb, min_separation, sizeof(double) * nc);
    std::memcpy(hb + sizeof(double) * nc, alias_tolerance, sizeof(double) * nc);
    char* db = e->d_rows.as<char>();
    CUDA_TRY(cudaMemcpyAsync(db, hb, in_bytes, cudaMemcpyHostToDevice, st), "upload row parameters");
    const double* dsep = reinterpret_cast<const double*>(db);
    const double* dtol = dsep + nc;
    int64_t* didx = reinterpret_cast<int64_t*>(db + in_bytes);
    double* dfld = reinterpret_cast<double*>(db + in_bytes + idx_bytes);
    int32_t* dcnt = reinterpret_cast<int32_t*>(db + in_bytes + idx_bytes + fld_bytes);
    CUDA_TRY(launch_rows(e->d_out.as<double>(), e->spec_total, nc, e->d_spec_off, e->d_grid_base,
                         P, e->args[0].freq, dsep, dtol, n_best, harmonic_max, dcnt, didx, dfld,
                         st),
             "peak search launch");
    CUDA_TRY(cudaMemcpyAsync(hb + in_bytes, db + in_bytes, out_bytes, cudaMemcpyDeviceToHost, st),
             "download rows");
    if ((rc = check_device_flag(e, st))) return rc;
    std::memcpy(index, hb + in_bytes, idx_bytes);
    std::memcpy(fields, hb + in_bytes + idx_bytes, fld_bytes);
    std::memcpy(n_peaks, hb + in_bytes + idx_bytes + fld_bytes, cnt_bytes);
    return BLS_OK;
}

int bls_launch_best_noalloc(BlsEngine* e, int64_t* best_index, double* best_power,
                            double* power_mean, double* power_std, void* stream) {
    if (!e || !best_index || !best_power || !power_mean || !power_std)
        return fail(BLS_E_INVALID, "engine and outputs are required");
    if (!e->prepared) return fail(BLS_E_STATE, "bls_launch_best_noalloc before bls_prepare");
    const int nc = e->n_curves;
    if (nc > kStaticMaxCurves)
        return fail(BLS_E_INVALID,
                    "bls_launch_best_noalloc: %d curves exceed its static scratch of %d curves; "
                    "split the batch, or use bls_launch and bls_download_best",
                    nc, kStaticMaxCurves);
    CUDA_TRY(cudaSetDevice(e->device), "select device");
    cudaStream_t st = pick(e, stream);
    void* scr = nullptr;
    CUDA_TRY(static_scratch_address(e->device, &scr), "static scratch address");
    int32_t* ctl = static_cast<int32_t*>(scr);
    CUDA_TRY(cudaMemsetAsync(ctl, 0, 64, st), "reset work counters and error flag");
    for (int m = 0; m < kModes; ++m) {
        if (e->args[m].n_items <= 0) continue;
        BatchArgs a = e->args[m];
        a.work_counter = ctl + m;
        a.error_flag = ctl + 8;
        CUDA_TRY(launch_search(a, m, e->ctas_mode[m], e->smem_mode[m], st), "search launch");
    }
    int64_t* di = reinterpret_cast<int64_t*>(static_cast<char*>(scr) + kStaticResultsOffset);
    double* dv = reinterpret_cast<double*>(di + kStaticMaxCurves);
    double* dmean = dv + kStaticMaxCurves;
    double* dstd = dmean + kStaticMaxCurves;
    CUDA_TRY(launch_best(e->d_out.as<double>(), nc, e->d_spec_off, di, dv, dmean, dstd, st),
             "best-of-spectrum launch");
    // copies into the caller's (pageable) arrays complete before they return
    int32_t flag = 0;
    CUDA_TRY(cudaMemcpyAsync(best_index, di, sizeof(int64_t) * nc, cudaMemcpyDeviceToHost, st),
             "download best index");
    CUDA_TRY(cudaMemcpyAsync(best_power, dv, sizeof(double) * nc, cudaMemcpyDeviceToHost, st),
             "download best power");
    CUDA_TRY(cudaMemcpyAsync(power_mean, dmean, sizeof(double) * nc, cudaMemcpyDeviceToHost, st),
             "download power mean");
    CUDA_TRY(cudaMemcpyAsync(power_std, dstd, sizeof(double) * nc, cudaMemcpyDeviceToHost, st),
             "download power std");
    CUDA_TRY(cudaMemcpyAsync(&flag, ctl + 8, sizeof(int32_t), cudaMemcpyDeviceToHost, st),
             "read error flag");
    CUDA_TRY(cudaStreamSynchronize(st), "synchronize");
    if (flag != 0) return fail(BLS_E_DEVICE, "a kernel met an impossible work descriptor");
    return BLS_OK;
}

int bls_search(BlsEngine* e, const BlsGrid* grid, const BlsCurves* curves, double* out,
               void* stream) {
    int rc;
    if ((rc = bls_prepare(e, grid, curves, stream))) return rc;
    if ((rc = bls_launch(e, stream))) return rc;
    return bls_download(e, out, stream);
}

int bls_joint_prepare(BlsEngine* e, const BlsGrid* grid, const BlsCurves* bands, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    return do_prepare_joint(e, grid, bands, pick(e, stream));
}

int bls_joint_launch(BlsEngine* e, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    return do_launch_joint(e, pick(e, stream));
}

int bls_joint_download(BlsEngine* e, double* out, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (!out) return fail(BLS_E_INVALID, "output pointer is NULL");
    return do_download_joint(e, out, pick(e, stream));
}

int bls_search_joint(BlsEngine* e, const BlsGrid* grid, const BlsCurves* bands, double* out,
                     void* stream) {
    int rc;
    if ((rc = bls_joint_prepare(e, grid, bands, stream))) return rc;
    if ((rc = bls_joint_launch(e, stream))) return rc;
    return bls_joint_download(e, out, stream);
}

int bls_tls_prepare(BlsEngine* e, const BlsTlsInputs* inputs, const double* periods,
                    int64_t n_periods, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (n_periods < 0) return fail(BLS_E_INVALID, "n_periods must be >= 0");
    return do_prepare_tls(e, inputs, periods, n_periods, pick(e, stream));
}

int bls_tls_launch(BlsEngine* e, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    return do_launch_tls(e, pick(e, stream));
}

int bls_tls_download(BlsEngine* e, double* out, void* stream) {
    if (!e) return fail(BLS_E_INVALID, "engine is NULL");
    if (!out) return fail(BLS_E_INVALID, "output pointer is NULL");
    return do_download_tls(e, out, pick(e, stream));
}

int bls_tls_search(BlsEngine* e, const BlsTlsInputs* inputs, const double* periods,
                   int64_t n_periods, double* out, void* stream) {
    int rc;
    if (!out) return fail(BLS_E_INVALID, "output pointer is NULL");
    if ((rc = bls_tls_prepare(e, inputs, periods, n_periods, stream))) return rc;
    if ((rc = bls_tls_launch(e, stream))) return rc;
    return bls_tls_download(e, out, stream);
}

int bls_batch_info(BlsEngine* e, BlsBatchInfo* info) {
    if (!e || !info) return fail(BLS_E_INVALID, "engine and info are required");
    if (!e->prepared) return fail(BLS_E_STATE, "no prepared batch");
    *info = e->info;
    return BLS_OK;
}

int bls_debug_prefix(BlsEngine* e, const double* t, const double* y, const double* dy, int64_t n,
                     double period, const double* durations, int32_t n_durations,
                     int32_t oversample, double* yw_prefix, double* ivar_prefix,
                     int32_t* n_bins) {
    if (!e || !t || !y || !durations || !yw_prefix || !ivar_prefix || !n_bins || n < 1 ||
        n_durations < 1)
        return fail(BLS_E_INVALID, "bad arguments");
    cudaSetDevice(e->device);
    const int64_t seg_off[2] = {0, 1};
    const int64_t dur_off[2] = {0, n_durations};
    BlsGrid g{1, seg_off, &period, dur_off, durations, oversample, 0};
    const int64_t offs[2] = {0, n};
    BlsCurves c{1, offs, t, y, dy};
    int rc;
    if ((rc = do_prepare(e, &g, 1, nullptr, &c, e->stream))) return rc;
    int mode = 0;
    while (mode < kModes - 1 && e->args[mode].n_items <= 0) ++mode;
    int32_t hl = 0;
    CUDA_TRY(cudaStreamSynchronize(e->stream), "synchronize");
    {
        const char* dmp = e->d_curves.as<char>();
        const SegmentDesc* dseg =
            reinterpret_cast<const SegmentDesc*>(reinterpret_cast<const CurveDesc*>(dmp) + 1);
        SegmentDesc sd;
        CUDA_TRY(cudaMemcpy(&sd, dseg, sizeof(sd), cudaMemcpyDeviceToHost), "read segment");
        hl = sd.hist_len;
    }
    DevBuf dbg;
    if ((rc = dbg.ensure(sizeof(double) * 2 * (size_t)hl))) return rc;
    int32_t nb = 0;
    CUDA_TRY(cudaMemcpy(&nb, e->args[0].nbins, sizeof(int32_t), cudaMemcpyDeviceToHost),
             "read n_bins");
    e->args[mode].debug_prefix = dbg.as<double>();
    rc = enqueue_search(e, e->stream);
    e->args[mode].debug_prefix = nullptr;
    e->graph_valid = false;
    if (rc) { dbg.release(); return rc; }
    cudaError_t ce = cudaMemcpyAsync(yw_prefix, dbg.p, sizeof(double) * (nb + 1),
                                     cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(ivar_prefix, dbg.as<double>() + hl, sizeof(double) * (nb + 1),
                             cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    dbg.release();
    if (ce != cudaSuccess) return cuda_fail(ce, "debug prefix");
    *n_bins = nb;
    return check_device_flag(e, e->stream);
}

int bls_debug_fold_bins(BlsEngine* e, const double* t, int64_t n, double period,
                        double bin_duration, int32_t width, int32_t* bins, int32_t* used_fast) {
    if (!e || !t || !bins || !used_fast || n < 1 || n > (1 << 30))
        return fail(BLS_E_INVALID, "bad arguments");
    if (!(period > 0.0) || !(bin_duration > 0.0) || width < 2)
        return fail(BLS_E_INVALID, "period, bin width and width must be positive");
    cudaSetDevice(e->device);
    std::vector<double> tau(n);
    double t_min = t[0], tau_max = 0.0;
    for (int64_t j = 0; j < n; ++j) t_min = std::min(t_min, t[j]);
    for (int64_t j = 0; j < n; ++j) {
        tau[j] = t[j] - t_min;
        tau_max = std::max(tau_max, tau[j]);
    }
    FoldParams fp = fold_params(width, bin_duration, tau_max, 1.0 / period, period / bin_duration);
    uint32_t S = 0;
    if (fp.fast) {
        const double sc = std::nearbyint((period / bin_duration) * std::ldexp(1.0, fp.fb));
        if (sc >= 1.0 && sc < 4294967296.0) S = (uint32_t)sc;
        else fp.fast = false;
    }
    DevBuf d_t, d_b, d_u;
    int rc;
    if ((rc = d_t.ensure(sizeof(double) * n)) || (rc = d_b.ensure(sizeof(int32_t) * n)) ||
        (rc = d_u.ensure(sizeof(int32_t) * n))) {
        d_t.release(); d_b.release(); d_u.release();
        return rc;
    }
    cudaStream_t st = e->stream;
    cudaError_t ce = cudaMemcpyAsync(d_t.p, tau.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess)
        ce = launch_fold_bins(d_t.as<double>(), (int)n, period, 1.0 / period, S, bin_duration, width,
                              fp.fb, fp.mu, fp.mphi, fp.fast ? 1 : 0, d_b.as<int32_t>(),
                              d_u.as<int32_t>(), st);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(bins, d_b.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(used_fast, d_u.p, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    d_t.release(); d_b.release(); d_u.release();
    if (ce != cudaSuccess) return cuda_fail(ce, "fold bins");
    return BLS_OK;
}

}  // extern "C"
