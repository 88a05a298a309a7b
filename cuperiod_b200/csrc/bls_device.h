// Device-side data layout of the B200 box-least-squares engine.
//
// One launch searches a batch of light curves over one segmented trial-period
// grid.  The host packs every curve once (time origin removed in FP64, flux
// centred and quantised to exact fixed point) and splits the work into items of
// (curve, segment, tile of consecutive periods); a persistent grid of CTAs pulls
// items from a global counter.
#pragma once
#include <stdint.h>

namespace blsb200 {

// Accumulation modes.  Every sum is an exact integer built from native 32-bit
// shared atomics: a point's quantised value v (|v| <= 2^bits, bits =
// min(27, 41 - ceil(log2 n)) for a curve of n points, at least 24) is added as
// its unsigned low 13 bits to one word and its signed high part to another, so a
// bin's sum is (signed) B * 2^13 + A with no carry lost for up to 2^17 points.
//  UNIFORM: every point has the same inverse variance w: r_q (the quantised
//           centred flux * weight) and a count per bin (three atomics).
//  GENERAL: per-point weights spanning more than 2^8: the two sums (centred
//           flux*weight and weight, both scaled by powers of two) stay FP64, like
//           the reference's, with FP64 shared atomics.
//  WIDE:    per-point weights within a factor 2^8 of each other: centred
//           flux*weight and weight each quantised to 38-bit fixed point
//           (|v| < 2^37 after a power-of-two scale) and added as three 32-bit
//           parts (13, 13 and a signed 12-bit high part): six native atomics,
//           exact integer sums for up to 2^17 points.
enum : int { MODE_UNIFORM = 0, MODE_GENERAL = 1, MODE_WIDE = 2 };
constexpr int kModes = 3;
constexpr int kWideBits = 13;       // WIDE: bits of the low and middle parts

constexpr int kFields = 7;          // power, depth, depth_err, depth_snr, duration, t0, loglike
constexpr int kMaxDur = 32;         // deduplicated box widths per segment
constexpr int kMaxTile = 16;        // periods per work item
constexpr int kHalfBits = 13;       // bits per atomic half-word
constexpr int kCountShift = 18;     // packed prefix: R * 2^18 + count
constexpr int kMaxExactPoints = (1 << 17) - 1;  // UNIFORM / WIDE: 32-bit prefix words
                                                // stay exact; longer curves take GENERAL
constexpr int kMaxPoints = 1 << 30;             // per curve (int32 indices)

// One CTA folds points in chunks of kChunkThreads x kChunkPts.  The host stores
// every full chunk lane-interleaved: memory slot chunk*2048 + r*256 + lane holds
// the point of time index chunk*2048 + lane*8 + r, so a lane's kChunkPts points
// are consecutive in time (equal bins merge in registers) and the lanes of a
// warp are 8 points apart (distinct bins, few atomic conflicts), while loads
// stay coalesced.
constexpr int kChunkThreads = 256;
constexpr int kChunkPts = 8;
constexpr int kChunk = kChunkThreads * kChunkPts;

// The box sweep reads the FP32 screen records of starts up to 2 x kChunkThreads
// + 31 past the last admissible start; that many records after a period's last
// bin hold a sentinel that fails every screen, so the sweep needs no bounds test.
constexpr int kScreenPad = 2 * kChunkThreads + 32;

struct SegmentDesc {
    int64_t period_off;     // first period of this segment in the grid arrays
    int32_t n_periods;
    int32_t width;          // the reference's width: ceil(max P / bin) + oversample + 1
    double bin_duration;
    int32_t dur_off;        // into dur_bins
    int32_t n_dur;
    int32_t oversample;
    int32_t frac_bits;      // fast fold: fraction bits of the scaled phase
    uint32_t margin_u;      // fast fold: bin-edge margin, units of 2^-frac_bits bins
    uint32_t margin_phi;    // fast fold: cycle-edge margin, units of 2^-32 cycles
    int32_t fast_fold;      // 1: the fast fold's error bound holds for the batch
    int32_t hist_len;       // bins held per period: max n_bins + 1 over the segment
};

struct CurveDesc {
    int64_t point_off;      // first point in the packed point arrays
    int64_t out_off;        // this curve's spectrum in each output field starts at
                            // out_off + (its grid's first period in the period arrays)
    int32_t n_points;
    int32_t mode;           // MODE_UNIFORM / MODE_GENERAL
    int32_t exact_all;      // 1: every admissible box is evaluated in FP64
    int32_t skip;           // 1: nothing admissible (e.g. zero total weight)
    double t_min;           // time origin removed from tau (added back to t0)
    double sum_y;           // sum of y*ivar (reference units)
    double sum_ivar;        // sum of ivar
    double ivar_floor;      // admissibility floor of either side of a box
    double ybar;            // sum_y / sum_ivar
    double w_uniform;       // UNIFORM: the common ivar
    double i_total;         // GENERAL: sum of the scaled weights
    int32_t e_r;            // r (reference units) = stored r * 2^-e_r
    int32_t e_i;            // GENERAL: ivar (reference units) = stored weight * 2^-e_i
    // UNIFORM: a point's stored value is round(y*ivar * 2^e_r) - round(ybar*ivar
    // * 2^e_r): centred by a whole number of quanta, so each point's rounding is
    // its own (centring by ybar itself gave every point the same rounding error,
    // which grew with the box instead of its square root).
    double center;          // the per-point centring, reference units
    double center_frac;     // ybar*ivar*2^e_r minus that whole number (|.| <= 1/2)
    // WIDE: the exact sums of every point's quantised centred flux*weight and
    // weight.  A box's outside sums are these minus its inside sums, so a box
    // holding every point has exactly zero weight outside and fails the floor
    // test as the reference's does (sum_ivar minus a quantised inside sum would
    // leave the quantisation residual, far above the floor).
    long long rq_total;
    long long iq_total;
};

struct WorkItem {
    int32_t curve;
    int32_t segment;
    int32_t p_begin;        // first period of the tile, within the segment
    int32_t p_count;        // periods in the tile (<= kMaxTile)
};

// One launch may search several trial grids (each curve has one).  The curves
// of one accumulation mode and one grid form a group whose work is regular:
// every curve of the group is cut into the same tiles (segment s of the grid:
// ceil(n_periods / seg_cap[s]) tiles), so the group's local work index i is
// curve order[order_begin + i / tiles_per_curve] and tile i % tiles_per_curve of
// that curve, located by a search of the group's per-segment tile prefix.
// Groups follow one another in the item space, costliest curves first.
struct WorkGroup {
    int32_t item_begin;         // first work item of the group
    int32_t tiles_per_curve;
    int32_t seg_begin;          // the grid's first segment in the segment table
    int32_t n_segments;         // the grid's segments
    int32_t order_begin;        // the group's first entry of order
    int32_t tiles_begin;        // the group's tile prefix: seg_tiles[tiles_begin ..
                                // tiles_begin + n_segments]
};

struct BatchArgs {
    const CurveDesc* curves;
    const SegmentDesc* segments;
    const WorkGroup* groups;    // n_groups, ascending item_begin (the first is 0)
    const int32_t* order;       // per group: its curves, most points first
    const int32_t* seg_tiles;   // per group: n_segments + 1 tile prefix per curve
    const int32_t* seg_cap;     // per segment of the table: periods per tile
    WorkGroup group0;           // groups[0], read from the launch parameters
    int32_t n_groups;
    const double* tau;          // per point: t - t_min (FP64)
    const uint32_t* pay_r;      // per point: r_q as low 13 bits | signed high part << 16
    const double* r64;          // GENERAL: (y*ivar - ybar*ivar) * 2^e_r per point;
                                // WIDE: the same rounded to an int64 (bit pattern)
    const double* iv64;         // GENERAL: ivar * 2^e_i per point; WIDE: int64 likewise
    const double* period;       // per grid period
    const double* freq;         // RN(1/P)
    const uint32_t* scale;      // round(P/bin * 2^frac_bits)
    const int32_t* nbins;       // n_bins of the reference
    const int32_t* dur_bins;    // per segment, box widths in bins (first-seen order)
    double* out;                // kFields x out_stride, field-major
    int64_t out_stride;
    int32_t* work_counter;      // persistent scheduler: next unclaimed item
    int32_t* error_flag;        // set by a CTA that met an impossible descriptor
    double* debug_prefix;       // test hook: prefix sums of one period (NULL in searches)
    int32_t n_items;
    int32_t obj_flag;           // 0 snr, 1 log-likelihood
};

// ---- joint-ephemeris multi-band search --------------------------------------
// One star's bands share one box per trial period (cuPeriod
// src/cuperiod/multiband/_bls_joint.py).  Each band's centred flux*weight and
// weight are quantised to 64-bit fixed point with a power-of-two scale per band
// (the band's magnitudes sum below 2^61, so even wrap-padded prefix sums fit
// an int64), so every bin and prefix sum is an exact integer and a box's sums
// are exact differences.  One bin of one band is a 16-byte record {Y, I}.

constexpr int kJointFields = 6;     // power, depth, depth_snr, duration, t0, band_index
constexpr int kMaxJointBands = 64;

struct JointBand {
    int64_t point_off;      // first point of the band in tau / qy / qi
    int32_t n_points;
    // FP32 screen, box sums in units of 2^61 quanta (|y'|, i' <= 1):
    float ybar_n;           // (sum_y / sum_ivar) * i_unit / y_unit
    float s_n;              // sum_ivar / (i_unit * 2^61)
    float c_n;              // 2^61 * y_unit^2 / i_unit: the objective per unit of
                            // the normalised one
    float floor_n;          // ivar_floor / (i_unit * 2^61), rounded up
    double sum_y;           // the reference's float sums of y*ivar and ivar
    double sum_ivar;
    double ivar_floor;      // admissibility floor of either side of a box
    double y_unit;          // reference units of one quantum of y*ivar (2^-e)
    double i_unit;          // reference units of one quantum of ivar
    long long qi_total;     // sum of the band's quantised weights
    int32_t full_skip;      // 1: a box holding qi_total fails the floor test
    int32_t pad;
};

struct JointSegment {
    int64_t period_off;     // first period of the segment
    int32_t n_periods;
    int32_t width;          // ceil(max P / bin) + oversample + 1
    double bin_duration;
    int32_t dur_off;        // into dur_bins
    int32_t n_dur;
    int32_t oversample;
    int32_t hist_len;       // max n_bins + 1 over the segment
    int32_t frac_bits;      // fast fold (fold_fast): fraction bits of the scaled phase
    uint32_t margin_u;      // fast fold: bin-edge margin, units of 2^-frac_bits bins
    uint32_t margin_phi;    // fast fold: cycle-edge margin, units of 2^-32 cycles
    int32_t fast_fold;      // 1: the fast fold's error bound holds for the star
};

struct JointArgs {
    const double* tau;          // per point: t - t_min over all bands
    const long long* qy;        // per point: quantised (y - median) * ivar
    const long long* qi;        // per point: quantised ivar
    const uint8_t* band_of;     // per point: its band
    const JointBand* bands;
    const JointSegment* segments;
    const double* period;       // per grid period
    const double* freq;         // RN(1/P)
    const uint32_t* scale;      // round(P/bin * 2^frac_bits) (fast-fold segments)
    const int32_t* nbins;       // the reference's n_bins per period
    const int32_t* dur_bins;    // per segment, box widths in bins (first-seen order)
    double* out;                // kJointFields x n_periods, field-major
    int64_t n_periods;
    long long* scratch;         // global histograms when they exceed shared memory
    int64_t hist_stride;        // int64 entries of one band array (max hist_len)
    int32_t* work_counter;      // next unclaimed period
    int32_t* error_flag;
    double t_min;
    int32_t n_points;           // points of the star (all bands)
    int32_t screen;             // 1: the FP32 screen's constants are in range
    int32_t n_bands;
    int32_t n_segments;
    int32_t obj_flag;           // 0 snr, 1 log-likelihood
};

// ---- transit least squares (limb-darkened matched filter) --------------------
// cuPeriod src/cuperiod/methods/tls.py.  Per curve the weighted residuals yw and
// the weights w are quantised to 64-bit fixed point (a power-of-two scale each,
// magnitudes summing below 2^61), stored in the same chunked point layout as
// the BLS curves (kChunk); a phase bin's sums are exact int64s.

constexpr int kTlsFields = 4;       // sr, depth, duration, t0 (from tau's origin)
constexpr int kTlsMaxTile = 8;      // periods per work item
constexpr int kTlsMaxDur = 64;
constexpr int kTlsMaxPoints = INT32_MAX;

struct TlsCurveDesc {
    int64_t point_off;      // first point slot
    int32_t n_points;
    int32_t pad;
    double w_total;         // the reference's float sum of w
    double y_unit;          // reference units of one quantum of yw (2^-e)
    double w_unit;          // reference units of one quantum of w
};

struct TlsArgs {
    const TlsCurveDesc* curves;
    const double* tau;          // per point slot: t - t_ref
    const long long* qy;        // per point slot: quantised yw
    const long long* qw;        // per point slot: quantised w
    const double* period;       // the shared trial periods
    const double* freq;         // RN(1/P) (fast fold)
    const int32_t* dur_bins;    // template widths in bins
    const int32_t* tmpl_off;    // offsets of the templates in tmpl
    const double* tmpl;         // the templates, concatenated
    double* out;                // kTlsFields x out_stride, field-major; curve c at c * P
    int64_t out_stride;         // n_curves * n_periods
    int64_t n_periods;
    int32_t* work_counter;
    int32_t* error_flag;
    uint32_t margin_u;          // fast fold: bin-edge margin, units of 2^-32 bins
    uint32_t margin_phi;        // fast fold: cycle-edge margin, units of 2^-32 cycles
    int32_t fast_fold;          // 1: the fast fold's error bound holds for the batch
    int32_t pad;
    double w_eps;               // smallest admissible template energy (1e-300)
    double den_rel;             // relative floor of the level-corrected energy
    int32_t n_curves;
    int32_t n_bins;
    int32_t n_dur;
    int32_t n_tmpl;             // samples of all templates
    int32_t max_width;
    int32_t tile;               // periods per work item (<= kTlsMaxTile)
    int32_t tiles_per_curve;
    int32_t n_items;
};

}  // namespace blsb200
