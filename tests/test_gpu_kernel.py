"""Device parity: the engine's BLS search against the reference's numba outputs
(golden vectors) and the CPU oracle, through the C ABI."""

from __future__ import annotations

import numpy as np
import pytest

from _cases import FIELDS, compare, kernel_golden, transit_curve
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from cuperiod_b200 import _lib
    eng = _lib.Engine()
    yield eng
    eng.close()


def _run(engine, t, y, dy, periods, durations, oversample, objective):
    from cuperiod_b200.core import bls_power
    out = bls_power(t, y, dy, periods, durations, oversample, objective=objective, engine=engine)
    return {f: getattr(out, f) for f in FIELDS}


# Inputs whose best boxes tie, or nearly tie, in exact arithmetic (a handful of
# points, quantised or constant flux, weights spanning eight decades): the
# reference's choice among equally good boxes then follows its cumulative-sum
# round-off, so only the power (equal within tolerance) is compared.
_DEGENERATE = ("five points", "quantised ties", "constant", "wild errors")


@pytest.mark.parametrize("meta_arrays", kernel_golden(), ids=lambda c: c[0]["name"])
def test_golden_case(engine, meta_arrays):
    meta, a = meta_arrays
    ref = dict(zip(FIELDS, a["out"]))
    with np.errstate(over="ignore"):
        got = _run(engine, a["t"], a["y"], a["dy"], a["periods"], a["durations"],
                   meta["oversample"], meta["objective"])
    degenerate = any(k in meta["name"] for k in _DEGENERATE)
    diag = compare(ref, got, rtol=1e-6, box_agree=0.0 if degenerate else 0.98)
    if diag["finite"] and not degenerate:
        assert diag["same_argmax"], diag


@pytest.mark.parametrize("span,period", [(27.0, 3.1), (90.0, 3.7), (1461.0, 37.0)])
def test_fold_bins_are_the_references(engine, span, period):
    t, _, _ = transit_curve(20000, span=span, period=period, seed=3)
    for P in (0.3137, 1.0, 2.0 ** -3, 3.7, period, 13.0001, span / 2.1):
        bin_duration = 0.1 * max(0.01, 0.01 * P) / 1.0 * 0.1 * 10
        width = int(np.ceil(P / bin_duration)) + 10 + 1
        got, fast = engine.fold_bins(t, P, bin_duration, width)
        ref = oracle.fold_bins(t, P, bin_duration, width)
        assert np.array_equal(got, ref), (P, np.flatnonzero(got != ref)[:5])
        assert fast.mean() > 0.99


def test_fold_bins_at_exact_edges(engine):
    # times that sit exactly on cycle and bin edges take the exact path
    P, bin_duration = 0.5, 0.005
    t = np.concatenate([np.arange(0, 200) * P, np.arange(0, 200) * bin_duration,
                        np.arange(0, 200) * P + 3 * bin_duration])
    width = int(np.ceil(P / bin_duration)) + 10 + 1
    got, fast = engine.fold_bins(t, P, bin_duration, width)
    assert np.array_equal(got, oracle.fold_bins(t, P, bin_duration, width))


@pytest.mark.parametrize("weights", ["uniform", "hetero", "wild"])
@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_random_curves_match_oracle(engine, weights, objective):
    t, y, dy = transit_curve(3000, span=60.0, period=4.3, depth=2e-3, seed=7, weights=weights)
    periods = np.geomspace(0.5, 20.0, 3000)
    durations = np.array([0.04, 0.07, 0.1, 0.15, 0.2])
    ref = oracle.bls_power(t, y, dy, periods, durations, 10, objective=objective)
    got = _run(engine, t, y, dy, periods, durations, 10, objective)
    diag = compare(ref, got, rtol=1e-6, box_agree=0.99)
    assert diag["same_argmax"]


def test_segments_equal_single_calls(engine):
    from cuperiod_b200.core import bls_power, bls_power_segments
    t, y, dy = transit_curve(1500, span=40.0, seed=11)
    segs = [(np.linspace(0.5, 1.0, 700), np.geomspace(0.01, 0.06, 8)),
            (np.zeros(0), np.array([0.01])),
            (np.linspace(1.0, 2.0, 900), np.geomspace(0.012, 0.12, 8))]
    many = bls_power_segments(t, y, dy, segs, 10, engine=engine)
    assert many[1].power.size == 0
    for (p, d), got in zip(segs, many):
        if p.size == 0:
            continue
        one = bls_power(t, y, dy, p, d, 10, engine=engine)
        for f in FIELDS:
            np.testing.assert_array_equal(getattr(got, f), getattr(one, f))


def test_batch_equals_single_curves(engine):
    from cuperiod_b200.core import bls_power, bls_power_many
    curves = [transit_curve(n, span=27.0, seed=s, weights=w)
              for n, s, w in ((500, 1, "uniform"), (2500, 2, "hetero"), (1200, 3, "uniform"))]
    periods = np.geomspace(0.6, 9.0, 1500)
    durations = np.geomspace(0.02, 0.2, 6)
    out = bls_power_many(curves, [(periods, durations)], 10, engine=engine)
    for i, (t, y, dy) in enumerate(curves):
        one = bls_power(t, y, dy, periods, durations, 10, engine=engine)
        for k, f in enumerate(FIELDS):
            if np.all(dy == dy[0]):
                # one weight: exact integer bin sums, identical in any batch
                np.testing.assert_array_equal(out[k, i], getattr(one, f))
            else:
                # per-point weights: FP64 bin sums whose atomic order varies
                np.testing.assert_allclose(out[k, i], getattr(one, f), rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("weights", ["uniform", "hetero", "wild"])
@pytest.mark.parametrize("period", [0.5310625902833277, 0.5619773606969279, 3.3, 17.7])
def test_padded_prefix_sums_match_oracle(engine, weights, period):
    t, y, dy = transit_curve(3000, span=60.0, period=4.3, depth=2e-3, seed=7, weights=weights)
    durations = np.array([0.04, 0.07, 0.1, 0.15, 0.2])
    yw_d, iv_d = engine.prefix_sums(t, y, dy, period, durations, 10)
    yw_o, iv_o = oracle.padded_cumsums(t, y, dy, period, durations, 10)
    assert yw_d.shape == yw_o.shape
    med = np.median(y)
    ivar = 1.0 / dy**2
    r = (y - med) * ivar - ivar * (np.sum((y - med) * ivar) / ivar.sum())
    # one weight: r quantised to at most 2^-24 of max|r| per point (finer for
    # curves below 2^17 points); weights within 2^8 of
    # each other: r and ivar quantised to 2^-38 of their largest; wider: FP64
    uniform = np.all(dy == dy[0])
    wide = not uniform and ivar.max() <= 256.0 * ivar.min()
    quant = (t.size * np.abs(r).max() * 2.0**-24 if uniform
             else t.size * np.abs(r).max() * 2.0**-37 if wide else 0.0)
    quant_i = t.size * ivar.max() * 2.0**-37 if wide else 0.0
    scale = np.abs((y - med) * ivar).sum() + np.abs(yw_o).max()
    np.testing.assert_allclose(yw_d, yw_o, rtol=0,
                               atol=quant + np.abs(med) * quant_i + 1e-12 * scale)
    np.testing.assert_allclose(iv_d, iv_o, rtol=1e-12, atol=quant_i + 1e-12 * ivar.sum())


@pytest.mark.parametrize("weights", ["hetero", "wild"])
@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_gappy_weighted_curve_picks_the_references_box(engine, objective, weights):
    # Per-point weights and long gaps: many boxes differ only by empty bins at
    # their ends, hold the same points and tie exactly in the reference (first
    # wins).  Weights spanning four decades ("wild") take FP64 sums, whose prefix
    # must stay exactly constant over every empty run (without that, 4 periods in
    # 3000 chose another box); what remains are boxes whose wrap-padded copy
    # holds the same points, a tie the reference's own round-off decides.
    # Weights within 2^8 ("hetero") take exact fixed-point sums: equal-content
    # ties are exact by construction, and only near ties of different content
    # (power equal to 1e-9) may resolve otherwise.
    t, y, dy = transit_curve(2500, span=40.0, period=3.3, depth=3e-3, seed=21, weights=weights)
    keep = (np.mod(t - t[0], 5.0) < 2.0) | (t - t[0] > 30.0)
    t, y, dy = t[keep], y[keep], dy[keep]
    periods = np.geomspace(0.4, 12.0, 3000)
    durations = np.array([0.04, 0.07, 0.1, 0.15, 0.2])
    ref = oracle.bls_power(t, y, dy, periods, durations, 10, objective=objective)
    got = _run(engine, t, y, dy, periods, durations, 10, objective)
    np.testing.assert_allclose(got["power"], ref["power"], rtol=1e-9, atol=0.0)
    same = (got["duration"] == ref["duration"]) & \
        (np.abs(got["transit_time"] - ref["transit_time"]) <= 1e-9)
    assert same.mean() >= (0.999 if weights == "wild" else 0.99)


@pytest.mark.parametrize("weights", ["uniform", "hetero"])
def test_curve_beyond_the_exact_sums_matches_oracle(engine, weights):
    # 150,000 points, past the 2^17 - 1 that the exact 32-bit sums hold: the
    # curve keeps FP64 sums (the reference's arithmetic) and is searched, not
    # refused
    t, y, dy = transit_curve(150000, span=120.0, period=3.3, depth=2e-3, seed=21,
                             weights=weights)
    periods = np.geomspace(0.5, 12.0, 1500)
    durations = np.array([0.04, 0.08, 0.12, 0.16])
    ref = oracle.bls_power(t, y, dy, periods, durations, 10)
    got = _run(engine, t, y, dy, periods, durations, 10, "snr")
    diag = compare(ref, got, rtol=1e-6, box_agree=0.99)
    assert diag["same_argmax"]


@pytest.mark.parametrize("weights", ["uniform", "hetero", "wild"])
@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_box_holding_every_point_is_not_admissible(engine, objective, weights):
    # Two short runs of observations a year apart and periods far longer than a
    # run: at many periods every point folds into a few days of phase, and the
    # widest boxes hold every point.  Such a box leaves no weight outside and the
    # reference rejects it (its outside weight is a rounding residual, below the
    # floor); with per-point weights within 2^8 the engine sums quantised
    # weights, and an outside weight of sum_ivar minus a quantised inside sum
    # would leave the quantisation residual -- far above the floor -- and admit it.
    rng = np.random.default_rng(5)
    t = np.concatenate([np.sort(rng.uniform(0.0, 3.0, 150)),
                        np.sort(rng.uniform(365.0, 368.0, 150))]) + 2458000.0
    y = 1.0 + rng.normal(0.0, 4e-3, t.size)
    if weights == "uniform":
        dy = np.full(t.size, 4e-3)
    elif weights == "hetero":
        dy = 4e-3 * rng.uniform(0.75, 2.0, t.size)
    else:
        dy = 4e-3 * 10.0 ** rng.uniform(-1.5, 1.5, t.size)
    periods = np.geomspace(20.0, 90.0, 600)
    durations = np.geomspace(0.4, 4.8, 8)
    ref = oracle.bls_power(t, y, dy, periods, durations, 10, objective=objective)
    got = _run(engine, t, y, dy, periods, durations, 10, objective)
    diag = compare(ref, got, rtol=1e-6, box_agree=0.98)
    assert diag["same_argmax"]



@pytest.mark.parametrize("objective", ["snr", "likelihood"])
@pytest.mark.parametrize("cadence,p_lo,dur_lo", [(2.0 / 1440, 0.3, 0.01),    # ~1 point a bin a cycle
                                                 (0.5 / 1440, 0.36, 0.0139)])  # ~300 a bin
def test_regular_cadence_spectra_are_identical(engine, objective, cadence, p_lo, dur_lo):
    # One weight, a regular cadence with dropouts, FP32 fluxes: the reference's
    # FP64 sums are exact, and so are the engine's fixed-point sums, so every
    # field of every period is identical.  The second case puts ~300 points in
    # one phase bin (a 0.5-minute cadence folded over 75 cycles).
    t, y, dy = transit_curve(int(27.0 / cadence), span=27.0, period=3.3, depth=2e-3, seed=5,
                             cadence=cadence)
    keep = np.random.default_rng(1).uniform(size=t.size) < 0.9          # gaps
    t, y = t[keep], y[keep].astype(np.float32).astype(np.float64)
    dy = np.ones_like(y)            # unit weights: the reference's FP64 sums are exact
    periods = np.geomspace(p_lo, 2.0 * p_lo, 400)
    durations = np.geomspace(dur_lo, 4.0 * dur_lo, 6)
    ref = oracle.bls_power(t, y, dy, periods, durations, 10, objective=objective)
    got = _run(engine, t, y, dy, periods, durations, 10, objective)
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)


def test_four_year_regular_cadence_spectra_are_identical(engine):
    # four years at 1.5-hour cadence: a bin of a 0.5 d period gathers points
    # from ~2900 cycles
    t, y, dy = transit_curve(int(1461.0 * 48), span=1461.0, period=3.3, depth=2e-3, seed=6,
                             cadence=30.0 / 1440)
    t, y = t[::3], y[::3].astype(np.float32).astype(np.float64)
    dy = np.ones_like(y)
    periods = np.geomspace(0.5, 1.0, 300)
    durations = np.geomspace(0.04, 0.16, 6)
    ref = oracle.bls_power(t, y, dy, periods, durations, 10)
    got = _run(engine, t, y, dy, periods, durations, 10, "snr")
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f], err_msg=f)
