/*
 * TEST INFRASTRUCTURE ONLY -- the CPU oracle of the BLS parity tests.
 *
 * A plain-C restatement of cuPeriod's numba box-least-squares kernel
 * (src/cuperiod/methods/_bls_core.py:341-462): its exact, unscreened form
 * (_bls_search_numba(..., screen=False), _bls_core.py:468-500) is the parity
 * checker, and its screened form (screen=True, the reference's default CPU
 * path, _bls_core.py:315-329, 395-440), which chooses the same box bit for bit,
 * is the timed CPU baseline.  Every
 * operation keeps the reference's order and IEEE rounding: the translation unit
 * is built with -ffp-contract=off (no fused multiply-add) and without fast-math,
 * like numba's fastmath=False, so the phase fold, the bin sums, the cumulative
 * sums and the box objective round exactly as the reference's do.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg load
 * this library, and only as the reference results are compared with or as the
 * timed CPU baseline.  The
 * product path (cuperiod_b200) never calls it.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <stdatomic.h>

/* Output fields, field-major (7 x n_periods), in the reference's order
 * (_OUTPUT_NAMES, _bls_core.py:675-684). */
enum { O_POWER, O_DEPTH, O_DEPTH_ERR, O_DEPTH_SNR, O_DURATION, O_TT, O_LL, O_NFIELDS };

/* Phase bin of one point, as the numba kernel computes it
 * (_bls_core.py:369-376): w = x - P*floor(x/P); ind = int(w/bin) + 1, clipped. */
static inline int64_t fold_bin(double x, double period, double bin_duration, int64_t width)
{
    double w = x - period * floor(x / period);
    int64_t ind = (int64_t)(w / bin_duration) + 1;
    if (ind < 0) ind = 0;
    else if (ind > width - 1) ind = width - 1;
    return ind;
}

/* Per-period bin count, _bls_core.py:358-360. */
static inline int64_t period_bins(double period, double bin_duration, int64_t oversample,
                                  int64_t width)
{
    int64_t n_bins = (int64_t)ceil(period / bin_duration) + oversample;
    if (n_bins > width - 1) n_bins = width - 1;
    return n_bins;
}

/* The phase bins of every point at one period (debug view used by the tests to
 * check the device's bit-exact bin assignment). */
int bls_oracle_fold_bins(const double* tau, int64_t n_points, double period,
                         double bin_duration, int64_t width, int32_t* out)
{
    for (int64_t j = 0; j < n_points; ++j)
        out[j] = (int32_t)fold_bin(tau[j], period, bin_duration, width);
    return 0;
}

/* Arguments shared by the worker threads of one search. */
typedef struct {
    const double *tau, *yw, *wv, *periods;
    const int64_t* dur_bins;
    int64_t n_points, n_periods, n_dur, oversample, width;
    double bin_duration, sum_y, sum_ivar, t_min, ivar_floor;
    int obj_flag;
    int screened;           /* 1: the reference's two-pass screened sweep */
    double inv_a, inv_s, slack;     /* its normalisations and slack */
    double* out;
    atomic_long next;       /* next unclaimed period block */
    atomic_int failed;
} search_args;

#define PERIOD_BLOCK 16

/* One trial period: _bls_core.py:357-460 (num, den: the screen's per-start
 * bounds, used when a->screened).  Built twice, for AVX2 and for any x86-64,
 * and chosen at load time: the vector build runs the screen's elementwise first
 * pass several points at a time, as the reference's JIT-compiled loop does on
 * the host CPU; every operation still rounds on its own (no contraction), so
 * both builds give the same bits. */
#if defined(__x86_64__)
__attribute__((target_clones("avx2", "default")))
#endif
static void search_period(const search_args* a, int64_t pidx, double* my, double* mi,
                          double* num, double* den)
{
    const int64_t n_periods = a->n_periods, width = a->width, oversample = a->oversample;
    const double bin_duration = a->bin_duration, sum_y = a->sum_y, sum_ivar = a->sum_ivar;
    const double ivar_floor = a->ivar_floor;
    double* o_power = a->out + (size_t)O_POWER * n_periods;
    double* o_depth = a->out + (size_t)O_DEPTH * n_periods;
    double* o_derr = a->out + (size_t)O_DEPTH_ERR * n_periods;
    double* o_dsnr = a->out + (size_t)O_DEPTH_SNR * n_periods;
    double* o_dur = a->out + (size_t)O_DURATION * n_periods;
    double* o_tt = a->out + (size_t)O_TT * n_periods;
    double* o_ll = a->out + (size_t)O_LL * n_periods;

    const double period = a->periods[pidx];
    const int64_t n_bins = period_bins(period, bin_duration, oversample, width);
    for (int64_t i = 0; i <= n_bins; ++i) { my[i] = 0.0; mi[i] = 0.0; }
    for (int64_t j = 0; j < a->n_points; ++j) {          /* fold, 365-376 */
        const int64_t ind = fold_bin(a->tau[j], period, bin_duration, width);
        my[ind] += a->yw[j];
        mi[ind] += a->wv[j];
    }
    for (int64_t k = 0; k < oversample; ++k) {           /* wrap pad, 377-381 */
        const int64_t dst = n_bins - oversample + k;
        if (0 <= dst && dst < width) { my[dst] = my[1 + k]; mi[dst] = mi[1 + k]; }
    }
    double ay = 0.0, ai = 0.0;                            /* cumulative sums, 382-388 */
    for (int64_t i = 0; i <= n_bins; ++i) {
        ay += my[i]; my[i] = ay;
        ai += mi[i]; mi[i] = ai;
    }
    double loc = -INFINITY;
    int64_t ln = 0, ld = 0;
    if (a->screened) {                                    /* screened sweep, 389-440 */
        const double ybar = sum_ivar > 0.0 ? sum_y / sum_ivar : 0.0;
        const double inv_a = a->inv_a, inv_s = a->inv_s, slack = a->slack;
        double best_t2 = 0.0, best_den = 1.0;
        for (int64_t di = 0; di < a->n_dur; ++di) {
            const int64_t d = a->dur_bins[di];
            if (d < 1 || d >= n_bins) continue;
            const int64_t m = n_bins - d + 1;
            for (int64_t n = 0; n < m; ++n) {             /* pass 1: optimistic bounds */
                const double y_in = my[n + d] - my[n];
                const double iv_in = mi[n + d] - mi[n];
                const double iv_out = sum_ivar - iv_in;
                const double t = (y_in - ybar * iv_in) * inv_a;
                const double t_hi = fabs(t) + slack;
                double dn = (iv_in * inv_s) * (iv_out * inv_s);
                if (a->obj_flag != 0) dn = dn * (iv_out * inv_s);
                const int ok = (iv_in >= ivar_floor) & (iv_out >= ivar_floor) & (t <= slack);
                num[n] = ok ? t_hi * t_hi : -1.0;
                den[n] = ok ? dn : 1.0;
            }
            for (int64_t n = 0; n < m; ++n) {             /* pass 2: exact where it can win */
                if (num[n] * best_den < best_t2 * den[n]) continue;
                const double y_in = my[n + d] - my[n];
                const double iv_in = mi[n + d] - mi[n];
                const double iv_out = sum_ivar - iv_in;
                if (iv_in < ivar_floor || iv_out < ivar_floor) continue;
                const double yin = y_in / iv_in;
                const double yout = (sum_y - y_in) / iv_out;
                if (yout < yin) continue;
                const double depth = yout - yin;
                double obj;
                if (a->obj_flag == 0) obj = depth / sqrt(1.0 / iv_in + 1.0 / iv_out);
                else obj = 0.5 * iv_in * depth * depth;
                if (obj > loc) {
                    loc = obj; ln = n; ld = d;
                    double t_lo = fabs((y_in - ybar * iv_in) * inv_a) - slack;
                    if (!(t_lo > 0.0)) t_lo = 0.0;
                    best_t2 = t_lo * t_lo;
                    best_den = den[n];
                }
            }
        }
    } else
    for (int64_t di = 0; di < a->n_dur; ++di) {           /* exact sweep, 395-440 */
        const int64_t d = a->dur_bins[di];
        if (d < 1 || d >= n_bins) continue;
        const int64_t m = n_bins - d + 1;
        for (int64_t n = 0; n < m; ++n) {
            const double y_in = my[n + d] - my[n];
            const double iv_in = mi[n + d] - mi[n];
            const double iv_out = sum_ivar - iv_in;
            if (iv_in < ivar_floor || iv_out < ivar_floor) continue;
            const double yin = y_in / iv_in;
            const double yout = (sum_y - y_in) / iv_out;
            if (yout < yin) continue;
            const double depth = yout - yin;
            double obj;
            if (a->obj_flag == 0) obj = depth / sqrt(1.0 / iv_in + 1.0 / iv_out);
            else obj = 0.5 * iv_in * depth * depth;
            if (obj > loc) { loc = obj; ln = n; ld = d; }
        }
    }
    if (!(loc > -INFINITY)) {                             /* no admissible box, 441-442 */
        o_power[pidx] = -INFINITY;
        o_depth[pidx] = 0.0; o_derr[pidx] = 0.0; o_dsnr[pidx] = 0.0;
        o_dur[pidx] = 0.0; o_tt[pidx] = 0.0; o_ll[pidx] = 0.0;
        return;
    }
    const double y_in = my[ln + ld] - my[ln];             /* epilogue, 443-460 */
    const double iv_in = mi[ln + ld] - mi[ln];
    const double iv_out = sum_ivar - iv_in;
    const double yin = y_in / iv_in;
    const double yout = (sum_y - y_in) / iv_out;
    const double depth = yout - yin;
    const double derr = sqrt(1.0 / iv_in + 1.0 / iv_out);
    const double dsnr = depth / derr;
    const double ll = 0.5 * iv_in * depth * depth;
    const double dur = (double)ld * bin_duration;
    o_power[pidx] = a->obj_flag == 0 ? dsnr : ll;
    o_depth[pidx] = depth;
    o_derr[pidx] = derr;
    o_dsnr[pidx] = dsnr;
    o_dur[pidx] = dur;
    o_tt[pidx] = fmod((double)ln * bin_duration + 0.5 * dur, period) + a->t_min;
    o_ll[pidx] = ll;
}

static void* search_worker(void* arg)
{
    search_args* a = (search_args*)arg;
    double* my = (double*)malloc(sizeof(double) * (size_t)a->width);
    double* mi = (double*)malloc(sizeof(double) * (size_t)a->width);
    double* num = (double*)malloc(sizeof(double) * (size_t)a->width);
    double* den = (double*)malloc(sizeof(double) * (size_t)a->width);
    if (!my || !mi || !num || !den) {
        atomic_store(&a->failed, 1);
    } else {
        for (;;) {
            const int64_t p0 = atomic_fetch_add(&a->next, PERIOD_BLOCK);
            if (p0 >= a->n_periods) break;
            const int64_t p1 = p0 + PERIOD_BLOCK < a->n_periods ? p0 + PERIOD_BLOCK : a->n_periods;
            for (int64_t p = p0; p < p1; ++p) search_period(a, p, my, mi, num, den);
        }
    }
    free(my);
    free(mi);
    free(num);
    free(den);
    return NULL;
}

/* The box search over every period (the numba kernel's prange loop, 356). The
 * periods are independent, so n_threads workers share them; the result does
 * not depend on the thread count.  screened = 0 is screen=False; screened = 1
 * runs the reference's screen with its normalisations inv_a = 1/sum|y*ivar|,
 * inv_s = 1/sum_ivar and slack (_bls_core.py:484-491). */
int bls_oracle_search_screened(const double* tau, const double* yw, const double* wv,
                               int64_t n_points, const double* periods, int64_t n_periods,
                               const int64_t* dur_bins, int64_t n_dur,
                               double bin_duration, int64_t oversample, int64_t width,
                               double sum_y, double sum_ivar, double t_min, int obj_flag,
                               double ivar_floor, int screened, double inv_a, double inv_s,
                               double slack, double* out, int n_threads)
{
    if (width < 2 || n_periods < 0 || n_points < 0) return 1;
    search_args a = {
        .tau = tau, .yw = yw, .wv = wv, .periods = periods, .dur_bins = dur_bins,
        .n_points = n_points, .n_periods = n_periods, .n_dur = n_dur,
        .oversample = oversample, .width = width, .bin_duration = bin_duration,
        .sum_y = sum_y, .sum_ivar = sum_ivar, .t_min = t_min, .ivar_floor = ivar_floor,
        .obj_flag = obj_flag, .screened = screened != 0, .inv_a = inv_a, .inv_s = inv_s,
        .slack = slack, .out = out,
    };
    atomic_init(&a.next, 0);
    atomic_init(&a.failed, 0);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 512) n_threads = 512;
    pthread_t th[512];
    int started = 0;
    for (int i = 1; i < n_threads; ++i) {
        if (pthread_create(&th[started], NULL, search_worker, &a) != 0) break;
        ++started;
    }
    search_worker(&a);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
    return atomic_load(&a.failed) ? 2 : 0;
}

/* The unscreened search (_bls_search_numba(..., screen=False)): the parity checker. */
int bls_oracle_search(const double* tau, const double* yw, const double* wv, int64_t n_points,
                      const double* periods, int64_t n_periods,
                      const int64_t* dur_bins, int64_t n_dur,
                      double bin_duration, int64_t oversample, int64_t width,
                      double sum_y, double sum_ivar, double t_min, int obj_flag,
                      double ivar_floor, double* out, int n_threads)
{
    return bls_oracle_search_screened(tau, yw, wv, n_points, periods, n_periods, dur_bins, n_dur,
                                      bin_duration, oversample, width, sum_y, sum_ivar, t_min,
                                      obj_flag, ivar_floor, 0, 0.0, 0.0, INFINITY, out, n_threads);
}

/* ---- joint multi-band search ------------------------------------------------
 * The joint-ephemeris sweep of src/cuperiod/multiband/_bls_joint.py:412-507: the
 * bands of one star (points of band k in [starts[k], starts[k+1]), one time
 * origin) are folded and binned each on its own, padded and accumulated over the
 * full width, and one box (d, n) is scored by the sum over bands, in band order,
 * of depth^2 / (1/iv_in + 1/iv_out) (obj 0) or 0.5 * iv_in * depth^2 (obj 1) of
 * the bands that are admissible there and have yout >= yin; the first box in
 * (duration, start) order with the largest strictly-improving total wins.
 * Outputs per period: the box (start n, width d in bins), whether one was found,
 * and each band's y_in and iv_in at it (n_bands x n_periods, band-major). */
typedef struct {
    const double *tau, *yw, *wv, *sum_y, *sum_ivar, *floors, *periods;
    const int64_t *starts, *dur_bins;
    int64_t n_bands, n_periods, n_dur, oversample, width;
    double bin_duration;
    int obj_flag;
    int64_t *out_n, *out_d;
    uint8_t* out_found;
    double *out_yin, *out_ivin;
    atomic_long next;
    atomic_int failed;
} joint_args;

static void joint_period(const joint_args* a, int64_t pidx, double* my, double* mi)
{
    const int64_t K = a->n_bands, width = a->width;
    const double period = a->periods[pidx];
    const int64_t n_bins = period_bins(period, a->bin_duration, a->oversample, width);
    for (int64_t k = 0; k < K; ++k) {
        double* y = my + k * width;
        double* w = mi + k * width;
        memset(y, 0, sizeof(double) * (size_t)width);
        memset(w, 0, sizeof(double) * (size_t)width);
        for (int64_t j = a->starts[k]; j < a->starts[k + 1]; ++j) {
            const int64_t ind = fold_bin(a->tau[j], period, a->bin_duration, width);
            y[ind] += a->yw[j];
            w[ind] += a->wv[j];
        }
        for (int64_t o = 0; o < a->oversample; ++o) {
            int64_t dst = n_bins - a->oversample + o;
            if (dst < 0) dst = 0;
            else if (dst > width - 1) dst = width - 1;
            y[dst] = y[1 + o];
            w[dst] = w[1 + o];
        }
        double ay = 0.0, ai = 0.0;
        for (int64_t i = 0; i < width; ++i) {
            ay += y[i];
            y[i] = ay;
            ai += w[i];
            w[i] = ai;
        }
    }
    double best = -INFINITY;
    int64_t bn = 0, bd = 0;
    for (int64_t di = 0; di < a->n_dur; ++di) {
        const int64_t d = a->dur_bins[di];
        if (d >= width || d >= n_bins) continue;
        for (int64_t n = 0; n <= n_bins - d; ++n) {
            double total = 0.0;
            int hit = 0;
            for (int64_t k = 0; k < K; ++k) {
                const double* y = my + k * width;
                const double* w = mi + k * width;
                const double y_in = y[n + d] - y[n];
                const double iv_in = w[n + d] - w[n];
                const double iv_out = a->sum_ivar[k] - iv_in;
                if (iv_in < a->floors[k] || iv_out < a->floors[k]) continue;
                const double yin = y_in / iv_in;
                const double yout = (a->sum_y[k] - y_in) / iv_out;
                if (!(yout >= yin)) continue;
                const double depth = yout - yin;
                hit = 1;
                if (a->obj_flag == 0) total += depth * depth / (1.0 / iv_in + 1.0 / iv_out);
                else total += 0.5 * iv_in * depth * depth;
            }
            if (hit && total > best) {
                best = total;
                bn = n;
                bd = d;
            }
        }
    }
    const int found = best > -INFINITY;
    a->out_found[pidx] = (uint8_t)found;
    a->out_n[pidx] = found ? bn : 0;
    a->out_d[pidx] = found ? bd : 0;
    for (int64_t k = 0; k < K; ++k) {
        const double* y = my + k * width;
        const double* w = mi + k * width;
        a->out_yin[k * a->n_periods + pidx] = found ? y[bn + bd] - y[bn] : 0.0;
        a->out_ivin[k * a->n_periods + pidx] = found ? w[bn + bd] - w[bn] : 0.0;
    }
}

static void* joint_worker(void* arg)
{
    joint_args* a = (joint_args*)arg;
    const size_t cells = (size_t)a->n_bands * (size_t)a->width;
    double* my = (double*)malloc(sizeof(double) * cells);
    double* mi = (double*)malloc(sizeof(double) * cells);
    if (!my || !mi) {
        atomic_store(&a->failed, 1);
    } else {
        for (;;) {
            const int64_t p = atomic_fetch_add(&a->next, 1);
            if (p >= a->n_periods) break;
            joint_period(a, p, my, mi);
        }
    }
    free(my);
    free(mi);
    return NULL;
}

int bls_oracle_joint(const double* tau, const double* yw, const double* wv, const int64_t* starts,
                     int64_t n_bands, const double* sum_y, const double* sum_ivar,
                     const double* floors, const double* periods, int64_t n_periods,
                     const int64_t* dur_bins, int64_t n_dur, double bin_duration,
                     int64_t oversample, int64_t width, int obj_flag, int64_t* out_n,
                     int64_t* out_d, uint8_t* out_found, double* out_yin, double* out_ivin,
                     int n_threads)
{
    if (width < 2 || n_periods < 0 || n_bands < 1) return 1;
    joint_args a = {
        .tau = tau, .yw = yw, .wv = wv, .sum_y = sum_y, .sum_ivar = sum_ivar, .floors = floors,
        .periods = periods, .starts = starts, .dur_bins = dur_bins, .n_bands = n_bands,
        .n_periods = n_periods, .n_dur = n_dur, .oversample = oversample, .width = width,
        .bin_duration = bin_duration, .obj_flag = obj_flag, .out_n = out_n, .out_d = out_d,
        .out_found = out_found, .out_yin = out_yin, .out_ivin = out_ivin,
    };
    atomic_init(&a.next, 0);
    atomic_init(&a.failed, 0);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 512) n_threads = 512;
    pthread_t th[512];
    int started = 0;
    for (int i = 1; i < n_threads; ++i) {
        if (pthread_create(&th[started], NULL, joint_worker, &a) != 0) break;
        ++started;
    }
    joint_worker(&a);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
    return atomic_load(&a.failed) ? 2 : 0;
}

/* ---- transit least squares (limb-darkened matched filter) --------------------
 * The numba TLS kernel of src/cuperiod/methods/tls.py:516-593: per trial period
 * the points are folded into n_bins phase bins (q = tau/P, ph = q - floor(q),
 * bin = int(ph * n_bins) clipped), sums of yw and w in point order, the bins
 * circularly padded by max_width - 1; each template g (widths dur_bins, samples
 * at tmpl + tmpl_off) is slid over every start s with num = sum g a, cwg = sum
 * g b, den = sum g^2 b accumulated in k order; a start counts when num < 0 and
 * den > w_eps, and de = den - cwg^2 / w_total > den_rel * den; the first
 * largest sr = num^2 / de in (width, start) order wins.  Outputs per period:
 * sr, depth = -num/de, duration = width / n_bins * P, t0 = frac(centre) * P. */
typedef struct {
    const double *tau, *yw, *wv, *periods, *tmpl;
    const int64_t *dur_bins, *tmpl_off;
    int64_t n_points, n_periods, n_dur, n_bins, max_width;
    double w_eps, w_total, den_rel;
    double *o_sr, *o_depth, *o_duration, *o_t0;
    atomic_long next;
    atomic_int failed;
} tls_args;

static void tls_period(const tls_args* a, int64_t pidx, double* ab, double* acc)
{
    const int64_t nb = a->n_bins, n_ext = nb + a->max_width - 1;
    double* A = ab;
    double* B = ab + n_ext;
    double* num = acc;
    double* cwg = acc + nb;
    double* den = acc + 2 * nb;
    const double period = a->periods[pidx];
    memset(ab, 0, sizeof(double) * 2 * (size_t)n_ext);
    for (int64_t j = 0; j < a->n_points; ++j) {
        const double q = a->tau[j] / period;
        const double ph = q - floor(q);
        int64_t bb = (int64_t)(ph * (double)nb);
        if (bb > nb - 1) bb = nb - 1;
        else if (bb < 0) bb = 0;
        A[bb] += a->yw[j];
        B[bb] += a->wv[j];
    }
    for (int64_t j = 0; j < a->max_width - 1; ++j) {
        A[nb + j] = A[j];
        B[nb + j] = B[j];
    }
    double loc_sr = 0.0, loc_depth = 0.0;
    int64_t loc_start = 0, loc_width = 0;
    for (int64_t di = 0; di < a->n_dur; ++di) {
        const int64_t width = a->dur_bins[di];
        const double* g = a->tmpl + a->tmpl_off[di];
        const double g0 = g[0], g00 = g0 * g0;
        for (int64_t s = 0; s < nb; ++s) {
            num[s] = g0 * A[s];
            cwg[s] = g0 * B[s];
            den[s] = g00 * B[s];
        }
        for (int64_t k = 1; k < width; ++k) {
            const double gk = g[k], gkk = gk * gk;
            for (int64_t s = 0; s < nb; ++s) {
                num[s] += gk * A[k + s];
                cwg[s] += gk * B[k + s];
                den[s] += gkk * B[k + s];
            }
        }
        for (int64_t s = 0; s < nb; ++s) {
            const double nm = num[s], dn = den[s];
            if (nm < 0.0 && dn > a->w_eps) {
                const double de = dn - cwg[s] * cwg[s] / a->w_total;
                if (de > a->den_rel * dn) {
                    const double sr = nm * nm / de;
                    if (sr > loc_sr) {
                        loc_sr = sr;
                        loc_start = s;
                        loc_width = width;
                        loc_depth = -nm / de;
                    }
                }
            }
        }
    }
    a->o_sr[pidx] = loc_sr;
    a->o_depth[pidx] = loc_depth;
    a->o_duration[pidx] = (double)loc_width / (double)nb * period;
    const double centre = ((double)loc_start + (double)loc_width / 2.0) / (double)nb;
    a->o_t0[pidx] = (centre - floor(centre)) * period;
}

static void* tls_worker(void* arg)
{
    tls_args* a = (tls_args*)arg;
    const int64_t n_ext = a->n_bins + a->max_width - 1;
    double* ab = (double*)malloc(sizeof(double) * 2 * (size_t)n_ext);
    double* acc = (double*)malloc(sizeof(double) * 3 * (size_t)a->n_bins);
    if (!ab || !acc) {
        atomic_store(&a->failed, 1);
    } else {
        for (;;) {
            const int64_t p = atomic_fetch_add(&a->next, 1);
            if (p >= a->n_periods) break;
            tls_period(a, p, ab, acc);
        }
    }
    free(ab);
    free(acc);
    return NULL;
}

int tls_oracle_search(const double* tau, const double* yw, const double* wv, int64_t n_points,
                      const double* periods, int64_t n_periods, const int64_t* dur_bins,
                      const int64_t* tmpl_off, const double* tmpl, int64_t n_dur,
                      int64_t n_bins, double w_eps, double w_total, double den_rel,
                      double* o_sr, double* o_depth, double* o_duration, double* o_t0,
                      int n_threads)
{
    if (n_bins < 1 || n_dur < 1 || n_periods < 0) return 1;
    int64_t max_width = 1;
    for (int64_t di = 0; di < n_dur; ++di)
        if (dur_bins[di] > max_width) max_width = dur_bins[di];
    tls_args a = {
        .tau = tau, .yw = yw, .wv = wv, .periods = periods, .tmpl = tmpl,
        .dur_bins = dur_bins, .tmpl_off = tmpl_off, .n_points = n_points,
        .n_periods = n_periods, .n_dur = n_dur, .n_bins = n_bins, .max_width = max_width,
        .w_eps = w_eps, .w_total = w_total, .den_rel = den_rel, .o_sr = o_sr,
        .o_depth = o_depth, .o_duration = o_duration, .o_t0 = o_t0,
    };
    atomic_init(&a.next, 0);
    atomic_init(&a.failed, 0);
    if (n_threads < 1) n_threads = 1;
    if (n_threads > 512) n_threads = 512;
    pthread_t th[512];
    int started = 0;
    for (int i = 1; i < n_threads; ++i) {
        if (pthread_create(&th[started], NULL, tls_worker, &a) != 0) break;
        ++started;
    }
    tls_worker(&a);
    for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
    return atomic_load(&a.failed) ? 2 : 0;
}
