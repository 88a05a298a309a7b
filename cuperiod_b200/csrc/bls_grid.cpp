// The reference's default BLS trial grid of one baseline, built on the host
// cores (cuPeriod src/cuperiod/methods/bls.py:52-125, BLSMethod.default_grid
// 327-359).
//
// Segments [p_lo, p_hi) start at min_period_days and step by segment_factor
// (p_lo of segment k+1 is p_hi of segment k), capped at
// min(max_period_days, baseline / min_transits).  Each is uniform in frequency:
// numpy's arange(1/p_hi, 1/p_lo, df) with df = grid_duration_frac /
// (grid_oversample * baseline) -- length ceil((stop - start) / df), values
// start, start + df and then start + i * ((start + df) - start), each product
// and sum rounded once -- trimmed to the values below 1/p_lo, and the periods are
// 1/frequency in ascending order.  Empty segments are dropped.  Every operation
// is the IEEE double operation the reference's Python and numpy perform, in the
// same order, so the periods are bit-identical (this file is built with
// floating-point contraction off).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/bls_b200.h"
#include "bls_grid.h"

namespace blsb200 {

namespace {
// The reference's hard limit on a grid's trial samples (MAX_GRID_SIZE,
// core/grid.py:417-505): a baseline beyond it is refused, not allocated.
constexpr int64_t kMaxGridPeriods = 250000000;

int build(const BlsDefaultGrid& sp, double baseline, DefaultGrid& out, std::string& err);
}  // namespace

int build_default_grid(const BlsDefaultGrid& sp, double baseline, DefaultGrid& out,
                       std::string& err) {
    try {
        return build(sp, baseline, out, err);
    } catch (const std::bad_alloc&) {
        out = DefaultGrid();
        err = "host allocation failed while building the default grid";
        return BLS_E_NOMEM;
    }
}

namespace {
int build(const BlsDefaultGrid& sp, double baseline, DefaultGrid& out, std::string& err) {
    out.periods.clear();
    out.seg_offsets.assign(1, 0);
    out.seg_start.clear();
    if (!(std::isfinite(baseline) && baseline > 0.0)) {
        err = "the default grid needs a positive, finite baseline";
        return BLS_E_INVALID;
    }
    const double by_transits = baseline / sp.min_transits;
    const double max_p = by_transits < sp.max_period_days ? by_transits : sp.max_period_days;
    const double df = sp.grid_duration_frac / (sp.grid_oversample * baseline);
    if (!(df > 0.0) || !std::isfinite(df)) {
        err = "the default grid's frequency step is not positive";
        return BLS_E_INVALID;
    }
    double p_lo = sp.min_period_days;
    for (int k = 0; p_lo < max_p; ++k) {
        const double cand = p_lo * sp.segment_factor;
        const double p_hi = max_p < cand ? max_p : cand;       // min(p_lo * factor, max_p)
        const double start = 1.0 / p_hi, stop = 1.0 / p_lo;
        const double span = std::ceil((stop - start) / df);
        if (!(span < 4.0e9)) {
            err = "a default-grid segment has too many periods";
            return BLS_E_RESOURCE;
        }
        const int64_t len = span > 0.0 ? (int64_t)span : 0;
        if ((int64_t)out.periods.size() + len > kMaxGridPeriods) {
            err = "the default grid exceeds the limit of 250,000,000 trial periods";
            return BLS_E_RESOURCE;
        }
        if (len > 0) {
            const double v1 = start + df;
            const double delta = v1 - start;
            int64_t n = 0;                                  // the values below stop (a prefix)
            while (n < len) {
                const double f = n == 0 ? start
                                 : n == 1 ? v1
                                          : start + (double)n * delta;
                if (!(f < stop)) break;
                ++n;
            }
            if (n > 0) {
                if (k >= sp.n_starts) {
                    err = "the duration table holds fewer segment starts than the grid needs";
                    return BLS_E_INVALID;
                }
                const size_t base = out.periods.size();
                out.periods.resize(base + (size_t)n);
                for (int64_t i = 0; i < n; ++i) {
                    const double f = i == 0 ? start : i == 1 ? v1 : start + (double)i * delta;
                    out.periods[base + (size_t)(n - 1 - i)] = 1.0 / f;
                }
                out.seg_start.push_back(k);
                out.seg_offsets.push_back((int64_t)out.periods.size());
            }
        }
        p_lo = p_hi;
    }
    return BLS_OK;
}
}  // namespace

int64_t default_grid_size(const BlsDefaultGrid& sp, double baseline) {
    DefaultGrid g;
    std::string err;
    if (build_default_grid(sp, baseline, g, err) != BLS_OK) return -1;
    return (int64_t)g.periods.size();
}

}  // namespace blsb200
