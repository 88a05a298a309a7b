"""The all-FP64 GPU oracle (oracle/bls_oracle_gpu.cu) equals the reference's
numba outputs bit for bit on every golden kernel case, and the CPU oracle on a
long-baseline curve; it is then the checker of the engine on the 4-year
workload at sizes the CPU oracle cannot reach."""

from __future__ import annotations

import numpy as np
import pytest

from _cases import FIELDS, compare, kernel_golden
from oracle import oracle, oracle_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("meta_arrays", kernel_golden(), ids=lambda c: c[0]["name"])
def test_gpu_oracle_bit_exact_on_golden(meta_arrays):
    meta, a = meta_arrays
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        out = oracle_gpu.bls_power(a["t"], a["y"], a["dy"], a["periods"], a["durations"],
                                   meta["oversample"], objective=meta["objective"])
    got = np.stack([out[f] for f in FIELDS])
    assert np.array_equal(got, a["out"], equal_nan=True)


def test_gpu_oracle_equals_cpu_oracle_on_a_long_baseline():
    from cuperiod_b200.synthetic import long_baseline_curves
    c = long_baseline_curves(1, seed=3)[0]
    keep = slice(0, 8000)
    t, y = c.t[keep], c.y[keep]
    dy = np.ones_like(y)
    periods = np.geomspace(0.5, 1.0, 2500)            # one default segment of the grid
    durations = np.geomspace(0.01, 0.06, 12)
    got = oracle_gpu.bls_power(t, y, dy, periods, durations, 10)
    ref = oracle.bls_power(t, y, dy, periods, durations, 10)
    for f in FIELDS:
        np.testing.assert_array_equal(got[f], ref[f])


def test_engine_against_gpu_oracle_on_four_year_curves():
    # the precision stress workload's curves at their full length over a cut of
    # its grid: the engine within 1e-6 relative power, same argmax
    from cuperiod_b200.core import bls_power
    from cuperiod_b200.synthetic import long_baseline_curves
    periods = np.geomspace(0.5, 400.0, 200000)[::40]
    durations = np.geomspace(0.01, 0.06, 12)
    for c in long_baseline_curves(2, seed=11):
        dy = np.ones_like(c.y)
        ref = oracle_gpu.bls_power(c.t, c.y, dy, periods[periods < 1.0], durations, 10)
        got = bls_power(c.t, c.y, dy, periods[periods < 1.0], durations, 10)
        diag = compare(ref, {f: getattr(got, f) for f in FIELDS}, rtol=1e-6, box_agree=0.99)
        assert diag["same_argmax"]
