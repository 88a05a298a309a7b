"""The host pipeline and the oracle against the reference itself on real data.

When the environment variable CUPERIOD_REFERENCE names a cuPeriod source tree
(with numba installed), every star of its bundled validation corpus
(benchmarks/dataset/light_curves.parquet: ASAS-SN magnitudes, read in place)
is searched twice on the reference's BLS parity grid
(benchmarks/bls_numba_parity.py:36-40): by the reference's own
``periodogram(..., backend="cpu")`` (its numba kernel), and by this package's
host steps (``to_input``, magnitude-to-flux conversion, the default segmented
grid) feeding the oracle's restatement of that kernel.  Frequency, power and
every extra must be identical.  Without the variable the test is skipped.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from oracle import oracle

REF = os.environ.get("CUPERIOD_REFERENCE")

pytestmark = pytest.mark.skipif(not REF, reason="CUPERIOD_REFERENCE is not set")


def test_corpus_matches_reference_bit_for_bit():
    pytest.importorskip("numba")
    pd = pytest.importorskip("pandas")
    sys.path.insert(0, os.path.join(REF, "src"))
    import cuperiod as cup

    from cuperiod_b200.api import to_input
    from cuperiod_b200.bls import BLSMethod
    from cuperiod_b200.lightcurve import Domain
    from cuperiod_b200.settings import BLSSettings

    df = pd.read_parquet(os.path.join(REF, "benchmarks", "dataset", "light_curves.parquet"))
    assert len(df) > 0
    for r in df.itertuples():
        t = np.asarray(r.jd, np.float64)
        y = np.asarray(r.mag, np.float64)
        e = np.asarray(r.mag_err, np.float64)
        p_true = float(r.vsx_period)
        kw = dict(min_period_days=max(0.05, p_true / 2.0), max_period_days=p_true * 2.0,
                  grid_oversample=1)
        ref = cup.periodogram((t, y, e), "BLS", backend="cpu", settings=cup.BLSSettings(**kw))
        lc = to_input((t, y, e)).in_domain(Domain.FLUX).finite()
        grid = BLSMethod().default_grid(lc, BLSSettings(**kw))
        freq, power, extras = oracle.method_power(lc.time, lc.value, lc.error, grid.period,
                                                  dict(grid.meta), oracle.Settings(**kw),
                                                  n_threads=8)
        np.testing.assert_array_equal(freq, ref.frequency, err_msg=str(r.asas_sn_id))
        np.testing.assert_array_equal(power, ref.power, err_msg=str(r.asas_sn_id))
        for name in ("depth", "depth_snr", "duration", "t0", "sde"):
            np.testing.assert_array_equal(extras[name], ref.extras[name],
                                          err_msg=f"{r.asas_sn_id} {name}")


def test_native_default_grids_are_the_references_on_the_corpus():
    # the engine library's host-side default-grid builder against the
    # reference's own BLSMethod.default_grid (methods/bls.py:327-359) on the
    # baselines of every corpus star, under the default settings and the
    # parity grid's settings: the same periods bit for bit, the same segments
    pytest.importorskip("numba")
    pd = pytest.importorskip("pandas")
    sys.path.insert(0, os.path.join(REF, "src"))
    import cuperiod as cup
    from cuperiod.methods.bls import BLSMethod as RefBLS

    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import default_grid_spec
    from cuperiod_b200.settings import BLSSettings

    df = pd.read_parquet(os.path.join(REF, "benchmarks", "dataset", "light_curves.parquet"))
    compared = 0
    for r in df.itertuples():
        t = np.asarray(r.jd, np.float64)
        y = np.asarray(r.mag, np.float64)
        e = np.asarray(r.mag_err, np.float64)
        p_true = float(r.vsx_period)
        for kw in ({}, dict(min_period_days=max(0.05, p_true / 2.0),
                            max_period_days=p_true * 2.0, grid_oversample=1)):
            finite = cup.to_input((t, y, e)).finite()
            try:
                ref = RefBLS().default_grid(finite, cup.BLSSettings(**kw))
            except Exception:                       # no searchable grid for this baseline
                continue
            spec = default_grid_spec(BLSSettings(**kw), float(finite.baseline))
            periods, offs, _ = _lib.default_grid(spec, float(finite.baseline))
            np.testing.assert_array_equal(periods, np.asarray(ref.period),
                                          err_msg=str(r.asas_sn_id))
            assert list(np.diff(offs)) == list(ref.meta["segment_sizes"]), r.asas_sn_id
            compared += 1
    assert compared >= 2 * len(df) - 5, compared         # nearly every star, both settings
