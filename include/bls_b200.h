/*
 * C ABI of the B200 box-least-squares (BLS) engine: libbls_b200.so (the BLS
 * search, the multi-band joint search and the transit least squares filter).
 *
 * Plain pointers and sizes only.  Host arrays in, host (or device) arrays out;
 * the engine owns its device buffers, pinned staging, CUDA stream and graphs.
 * Every function returns 0 on success or a BLS_E_* code; bls_last_error()
 * describes the last failure of the calling thread.
 *
 * The entry points replace, in cuPeriod 1.3.0:
 *   bls_engine_create / bls_engine_destroy
 *       -- the per-worker engine hook PeriodogramMethod.make_engine
 *          (src/cuperiod/methods/base.py:388-396), built once per batch worker
 *          (src/cuperiod/batch/runner.py:253-277);
 *   bls_search
 *       -- _bls_search_cuda_specs (src/cuperiod/methods/_bls_core.py:741-840):
 *          one upload, one launch per segment, one download.  With one curve it
 *          is bls_power_segments (1075-1130) / bls_power (882-1028); with many
 *          curves it is the batch runner's per-curve loop
 *          (src/cuperiod/batch/runner.py:214-250) done in one launch;
 *   bls_prepare / bls_launch / bls_download
 *       -- the three phases of _bls_search_cuda_specs taken apart: the uploads
 *          of _cuda_curve (709-738), the kernel launches (796-825) and the
 *          stacked (7, P) download (828);
 *   bls_download_best
 *       -- the per-curve reduction of the spectrum that Periodogram.best_period
 *          and the batch row need (src/cuperiod/core/result.py:369-438,
 *          src/cuperiod/methods/bls.py:274-301 for the SDE);
 *   bls_debug_fold_bins / bls_debug_prefix
 *       -- the phase-bin lines of the fold (_bls_core.py:369-376 / 536-538) and
 *          the padded cumulative sums (377-388), exported so tests can compare
 *          the device's intermediate results with the reference's;
 *   bls_download_rows
 *       -- the batch runner's per-curve rows with alias-diverse peaks
 *          (src/cuperiod/batch/io.py:507-571, core/peaks.py:128-231);
 *   bls_search_joint, bls_joint_prepare / _launch / _download
 *       -- joint_search with the cupy backend and its _finish, the shared-box
 *          multi-band statistic (src/cuperiod/multiband/_bls_joint.py:151-204,
 *          359-404, 703-796);
 *   bls_tls_search, bls_tls_prepare / _launch / _download
 *       -- _tls_cuda / _tls_numba, the transit least squares matched filter
 *          (src/cuperiod/methods/tls.py:428-621);
 *   bls_prepare_grids, bls_default_grid, bls_default_grid_sizes,
 *   bls_prepare_default
 *       -- the batch runner searching every curve over its own default grid
 *          (src/cuperiod/batch/runner.py:187-250 -> BLSMethod.default_grid,
 *          src/cuperiod/methods/bls.py:52-125, 327-359): the grids built on the
 *          host cores and all curves in one launch;
 *   bls_launch_best_noalloc, bls_time_launches
 *       -- no counterpart: an allocation-free launch for services, and the
 *          tile-shape autotuner's clock;
 *   bls_last_error
 *       -- the exceptions the reference raises before a launch (ValueError,
 *          BackendUnavailableError from core/backend.py:340-384).
 */
#ifndef BLS_B200_H
#define BLS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    BLS_OK = 0,
    BLS_E_INVALID = 1,      /* bad argument or input data (the reference's ValueError) */
    BLS_E_CUDA = 2,         /* CUDA runtime failure */
    BLS_E_RESOURCE = 3,     /* a segment too wide for shared memory (BackendUnavailableError) */
    BLS_E_NOMEM = 4,        /* device or pinned host allocation failed */
    BLS_E_DEVICE = 5,       /* a kernel of the latest search met an impossible work descriptor */
    BLS_E_STATE = 6         /* call out of order (e.g. launch before prepare) */
};

/* Output fields, in the reference's order (_OUTPUT_NAMES, _bls_core.py:675-684). */
enum {
    BLS_F_POWER = 0, BLS_F_DEPTH, BLS_F_DEPTH_ERR, BLS_F_DEPTH_SNR,
    BLS_F_DURATION, BLS_F_TRANSIT_TIME, BLS_F_LOG_LIKELIHOOD, BLS_N_FIELDS
};

typedef struct BlsEngine BlsEngine;

typedef struct {
    int32_t device;          /* CUDA device ordinal; -1 = the current device */
    int32_t smem_per_cta;    /* dynamic shared memory per CTA in bytes; 0 = automatic */
    int32_t max_tile;        /* periods per work item, 1..16; 0 = as many as fit */
    int32_t use_graph;       /* 1: replay bls_launch from a captured CUDA graph */
    int32_t exact_sweep;     /* 1: evaluate every box in FP64, no FP32 screen (the
                                reference's screen=False, _bls_core.py:468-500) */
} BlsTune;

/* One trial-period grid, split into duration-homogeneous segments (each is one
 * _SearchSpec of the reference, _bls_core.py:687-706).  All host pointers. */
typedef struct {
    int32_t n_segments;
    const int64_t* seg_offsets;   /* n_segments+1 offsets into periods */
    const double* periods;        /* every segment's periods, concatenated */
    const int64_t* dur_offsets;   /* n_segments+1 offsets into durations */
    const double* durations;      /* every segment's box durations, concatenated */
    int32_t oversample;           /* phase bins per shortest duration */
    int32_t objective;            /* 0 = depth SNR, 1 = log-likelihood */
} BlsGrid;

/* A batch of light curves, concatenated.  All host pointers.  Times, fluxes and
 * errors must be finite, errors > 0; dy may be NULL (unit errors). */
typedef struct {
    int32_t n_curves;
    const int64_t* offsets;       /* n_curves+1 offsets into t / y / dy */
    const double* t;
    const double* y;              /* flux, transits as dips */
    const double* dy;             /* 1-sigma errors, or NULL */
} BlsCurves;

/* What one prepared batch holds (sizes and the algorithmic work of one launch). */
typedef struct {
    int32_t n_curves;
    int32_t n_segments;
    int64_t n_periods;            /* periods per curve (the most, with several grids) */
    int64_t n_items;              /* work items of one launch */
    int64_t n_points;             /* points over all curves */
    double folds;                 /* point-period folds per launch */
    double boxes;                 /* (duration, start) boxes per launch */
    double trials;                /* (period, duration) trials per launch */
    int64_t h2d_bytes;            /* bytes uploaded by bls_prepare */
    int32_t ctas;                 /* persistent CTAs per launch */
    int32_t smem_per_cta;
    int32_t uniform_curves;       /* curves on the one-weight fast path */
    int32_t fast_fold_segments;   /* segments whose fold runs the fast path */
    int64_t spectrum;             /* output entries per field: the curves' periods summed */
    int32_t n_grids;              /* trial grids of the batch (bls_prepare_grids) */
    int32_t reserved;
} BlsBatchInfo;

int bls_engine_create(const BlsTune* tune, BlsEngine** engine);
int bls_engine_destroy(BlsEngine* engine);
const char* bls_last_error(void);

/* Pack and upload a batch (host preparation runs on all host cores).  `stream`
 * is a cudaStream_t; NULL selects the engine's own stream. */
int bls_prepare(BlsEngine* engine, const BlsGrid* grid, const BlsCurves* curves, void* stream);

/* No counterpart in the reference, whose batch runner searches each curve over
 * its own default grid in a launch of its own (batch/runner.py:187-250 ->
 * methods/bls.py:361-395).  bls_prepare for a batch whose curves have different
 * grids: curve c is searched over grids[grid_of_curve[c]], every curve of the
 * batch in one launch.  The grids share oversample and objective.  Outputs are
 * field-major with each curve's spectrum in turn: field f of curve c at grid
 * index p is out[f * S + spec(c) + p], S = BlsBatchInfo.spectrum and spec(c) the
 * summed period counts of the grids of curves 0..c-1; bls_download_best and
 * bls_download_rows index each curve's own grid. */
int bls_prepare_grids(BlsEngine* engine, int32_t n_grids, const BlsGrid* grids,
                      const int32_t* grid_of_curve, const BlsCurves* curves, void* stream);

/* The reference's default trial grid (BLSMethod.default_grid, methods/bls.py:
 * 52-125 and 327-359) of a baseline: log segments [p_lo, p_hi) from
 * min_period_days, segment_factor wide, capped at min(max_period_days,
 * baseline / min_transits); each uniform in frequency with step
 * grid_duration_frac / (grid_oversample * baseline) as numpy's
 * arange(1/p_hi, 1/p_lo, step) trimmed below 1/p_lo, periods = 1/frequency
 * ascending; empty segments dropped.  Segment starts are min_period_days *
 * segment_factor^k (k = 0, 1, ...); the segment starting at start k searches
 * durations[dur_offsets[k] .. dur_offsets[k + 1]) (the reference's
 * _segment_durations of that start, which the caller computes). */
typedef struct {
    double min_period_days;
    double max_period_days;
    double min_transits;
    double segment_factor;
    double grid_duration_frac;
    double grid_oversample;
    int32_t n_starts;             /* segment starts covered by the duration table */
    int32_t oversample;           /* phase bins per shortest duration */
    int32_t objective;            /* 0 = depth SNR, 1 = log-likelihood */
    int32_t reserved;
    const int64_t* dur_offsets;   /* n_starts + 1 */
    const double* durations;
} BlsDefaultGrid;

/* No counterpart in the reference's ABI.  The default grid of one baseline on
 * the host: with periods == NULL only *n_segments and *n_periods are set;
 * otherwise periods (capacity entries), the segment offsets (n_segments + 1)
 * and each segment's start index k are written.  BLS_E_INVALID when capacity
 * is too small or the baseline is not positive. */
int bls_default_grid(const BlsDefaultGrid* spec, double baseline, int64_t capacity,
                     double* periods, int64_t* seg_offsets, int32_t* seg_start,
                     int32_t* n_segments, int64_t* n_periods);

/* Periods of the default grid of each of n baselines (-1 where none can be
 * built), on all host cores. */
int bls_default_grid_sizes(const BlsDefaultGrid* spec, int32_t n, const double* baselines,
                           int64_t* n_periods);

/* bls_prepare_grids with every curve over the default grid of its baseline
 * (baselines[c], the span of its finite times): the grids are built on the host
 * cores, one per distinct baseline, and the batch searched in one launch.
 * A curve whose default grid is empty is refused (BLS_E_INVALID). */
int bls_prepare_default(BlsEngine* engine, const BlsDefaultGrid* spec, const double* baselines,
                        const BlsCurves* curves, void* stream);

/* Run the search of the prepared batch on the device (no host transfers). */
int bls_launch(BlsEngine* engine, void* stream);

/* No counterpart in the reference (its tile shape is fixed at 128 threads per
 * period).  Runs bls_launch `reps` times on `stream` between two CUDA events and
 * returns the mean device time of one launch in milliseconds; the autotuner's
 * clock for comparing tile shapes (BlsTune smem_per_cta / max_tile).  Waits
 * for the stream. */
int bls_time_launches(BlsEngine* engine, int32_t reps, double* ms_per_launch, void* stream);

/* Copy every field of every curve, field-major: out[f][c][p] with
 * f < BLS_N_FIELDS, c < n_curves, p < n_periods (grid order); after
 * bls_prepare_grids, out[f * spectrum + spec(c) + p].  Waits for the stream. */
int bls_download(BlsEngine* engine, double* out, void* stream);

/* No counterpart in the reference (its per-curve calls return whole spectra).
 * Copy every field of the listed curves of the prepared batch: for each id in
 * turn, its BLS_N_FIELDS fields of its own spectrum length, field after field
 * (one grid: out[(k * BLS_N_FIELDS + f) * n_periods + p]).  Ids outside the
 * batch are refused (BLS_E_INVALID).  Waits for the stream. */
int bls_download_curves(BlsEngine* engine, const int32_t* curve_ids, int32_t n_ids, double* out,
                        void* stream);

/* Device address of the output fields (layout as bls_download), valid until the
 * next bls_prepare. */
int bls_device_output(BlsEngine* engine, const double** out);

/* Per curve: index (grid order) and value of the largest finite power, and the
 * mean and standard deviation of the power with non-finite values as 0 (the
 * reference's SDE normalisation, methods/bls.py:274-301).  Waits for the stream. */
int bls_download_best(BlsEngine* engine, int64_t* best_index, double* best_power,
                      double* power_mean, double* power_std, void* stream);

/* Per curve, the result row's peaks, ranked on the device: the reference's
 * periodogram_to_row / Periodogram.best_periods(alias_diverse=True) /
 * select_diverse_peaks (batch/io.py:507-571, core/result.py:285-406,
 * core/peaks.py:128-231) over the assembled spectrum of methods/bls.py:274-301
 * (non-finite power as 0, SDE normalisation).  Inputs per curve: the minimum
 * frequency separation (the reference's max(rayleigh/baseline, 1e-12)) and the
 * alias tolerance (max(tol, 1e-12)); n_best peaks at most; harmonics up to
 * harmonic_max.  Outputs: n_peaks[c]; index[c*n_best + k] (grid order) and
 * fields[(c*n_best + k)*8 + f], f = period, frequency, power, depth, depth_snr,
 * duration, t0, sde.  Needs strictly increasing trial periods (frequency order
 * is then reversed grid order).  Among candidates of exactly equal power the
 * later in the reference's candidate order ranks first (its stable-sort
 * order).  Waits for the stream. */
int bls_download_rows(BlsEngine* engine, int32_t n_best, int32_t harmonic_max,
                      const double* min_separation, const double* alias_tolerance,
                      int32_t* n_peaks, int64_t* index, double* fields, void* stream);

/* No counterpart in the reference.  bls_launch followed by bls_download_best,
 * for callers that must not allocate once their batch is prepared: a service
 * whose device memory is committed to other work, or whose latency cannot absorb
 * the device synchronisation of cudaMalloc/cudaFree, and callers whose memory
 * is handed out by another framework's pool.  The call allocates nothing --
 * no device or pinned memory, no graph: the search's work counters and error
 * flag and the per-curve results live in a static device array of this library
 * (2 MiB + 256 B per device); the counters and flag are zeroed by the call
 * before the search starts.  Limits: at most 65,536 curves in the prepared
 * batch (larger batches are refused with BLS_E_INVALID); calls that overlap in
 * time on one device (from several threads, streams or engines) share that
 * array and race -- serialise them.  The first call on a device looks up the
 * array's address (cudaGetSymbolAddress, which may load the module), so make it
 * outside any stream capture.  Results as bls_download_best; waits for the
 * stream. */
int bls_launch_best_noalloc(BlsEngine* engine, int64_t* best_index, double* best_power,
                            double* power_mean, double* power_std, void* stream);

/* prepare + launch + download in one call. */
int bls_search(BlsEngine* engine, const BlsGrid* grid, const BlsCurves* curves, double* out,
               void* stream);

int bls_batch_info(BlsEngine* engine, BlsBatchInfo* info);

/* Joint-ephemeris fields (JOINT_FIELDS, src/cuperiod/multiband/_bls_joint.py:52-54). */
enum {
    BLS_J_POWER = 0, BLS_J_DEPTH, BLS_J_DEPTH_SNR, BLS_J_DURATION, BLS_J_TRANSIT_TIME,
    BLS_J_BAND_INDEX, BLS_J_N_FIELDS
};

/* The joint-ephemeris ("shared") multi-band search of one star: one box -- one
 * duration and one phase on a phase grid binned from one time origin -- placed
 * in every band at once, chosen per trial period by the summed per-band
 * objective of the bands that dip in it.  Replaces joint_search with the
 * 'cupy' backend (src/cuperiod/multiband/_bls_joint.py:151-204, the launch of
 * _joint_cuda, 703-796) together with joint_bands (94-135) and _finish
 * (359-404).  `bands` holds the star's bands as curves (1 to 64; each band's
 * fluxes are centred on its own median here; dy may be NULL for unit errors).
 * out receives BLS_J_N_FIELDS x n_periods values, field-major, in grid order: a
 * period where no band dips in any admissible box has every field 0.  Waits for
 * the stream. */
int bls_search_joint(BlsEngine* engine, const BlsGrid* grid, const BlsCurves* bands, double* out,
                     void* stream);

/* A batch of light curves for the TLS matched filter, as the reference's kernel
 * receives one (_tls_cuda / _tls_numba, src/cuperiod/methods/tls.py:428-491,
 * 596-621): per point the time offset tau = t - t_ref, the weighted
 * mean-subtracted flux yw = w (y - y_mean) and the weight w, per curve the
 * float sum of w; per batch the phase-bin count, the template widths and the
 * templates themselves (limb_darkened_template, concatenated in width order)
 * and the relative floor of the level-corrected template energy.  The host
 * steps of tls_power before the kernel (flux scale, weights, mean) stay with
 * the caller, as in the reference.  All host pointers. */
typedef struct {
    int32_t n_curves;
    const int64_t* offsets;       /* n_curves+1 offsets into tau / yw / w */
    const double* tau;
    const double* yw;
    const double* w;
    const double* w_total;        /* per curve */
    int32_t n_bins;               /* phase bins (TLSSettings.n_phase_bins) */
    int32_t n_dur;                /* template widths, 1 .. 64 */
    const int32_t* dur_bins;      /* widths in bins, each in [1, n_bins - 1] */
    const double* templates;      /* sum(dur_bins) samples */
    double den_rel;               /* 1e-9 in float64 (_DEN_REL_EPS) */
} BlsTlsInputs;

/* The TLS matched filter of every curve over one period grid: the reference's
 * per-period fold into n_bins phase bins, circular pad, sliding template
 * correlation and joint level + depth fit, keeping the first largest signal
 * residue (tls.py:516-593; the CUDA tls_block of tls.py:323-414).  out receives
 * 4 x n_curves x n_periods values, field-major (sr, depth, duration, t0; t0
 * measured from tau's origin, in [0, P)); the SDE normalisation and the unit
 * conversions of tls_power stay with the caller.  Waits for the stream. */
int bls_tls_search(BlsEngine* engine, const BlsTlsInputs* inputs, const double* periods,
                   int64_t n_periods, double* out, void* stream);

/* bls_tls_search in its three phases, as _tls_cuda runs them (uploads, launch,
 * download).  A prepared batch stays on the device: bls_tls_launch may run
 * again; the next bls_tls_prepare replaces it.  bls_tls_download waits for the
 * stream. */
int bls_tls_prepare(BlsEngine* engine, const BlsTlsInputs* inputs, const double* periods,
                    int64_t n_periods, void* stream);
int bls_tls_launch(BlsEngine* engine, void* stream);
int bls_tls_download(BlsEngine* engine, double* out, void* stream);

/* bls_search_joint in its three phases, as _joint_cuda runs them: the uploads
 * (joint_bands and the segment tables, 703-760), the launch (one persistent
 * launch for every segment) and the download of the fields (784-796).  A
 * prepared star stays on the device: bls_joint_launch may run again; the next
 * bls_joint_prepare replaces it.  bls_joint_download waits for the stream. */
int bls_joint_prepare(BlsEngine* engine, const BlsGrid* grid, const BlsCurves* bands,
                      void* stream);
int bls_joint_launch(BlsEngine* engine, void* stream);
int bls_joint_download(BlsEngine* engine, double* out, void* stream);

/* Phase bin of every point of one curve (times t, n points; t_min removed as the
 * reference does) at one period of a segment whose shortest duration and
 * oversample give the bin width, as the search kernel computes it.  used_fast[j]
 * is 1 where the fast fold decided the bin.  Host arrays. */
int bls_debug_fold_bins(BlsEngine* engine, const double* t, int64_t n, double period,
                        double bin_duration, int32_t width, int32_t* bins, int32_t* used_fast);

/* Prefix sums of y*ivar and ivar over the phase bins 0..n_bins of one period,
 * after the wrap pad, as the search kernel holds them (the cumulative sums of
 * _bls_core.py:377-388), for one curve (dy may be NULL).  yw_prefix and
 * ivar_prefix need room for n_bins + 1 values; *n_bins receives n_bins. */
int bls_debug_prefix(BlsEngine* engine, const double* t, const double* y, const double* dy,
                     int64_t n, double period, const double* durations, int32_t n_durations,
                     int32_t oversample, double* yw_prefix, double* ivar_prefix, int32_t* n_bins);

#ifdef __cplusplus
}
#endif

#endif /* BLS_B200_H */
