"""The reference's own GPU kernel (bls_block, compiled from the reference's
source into oracle/_ref by oracle/build_ref_gpu.py) driven by this repository's
launcher, against the oracle: the baseline the engine is timed against must
compute the reference's result.  Its FP64 bin sums are shared-memory atomics in
arrival order, so powers agree to rounding (1e-9 relative), not bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from _cases import transit_curve
from oracle import oracle, ref_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(),
                                 reason="the reference's kernel was not built (no reference tree)")]


@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_reference_kernel_matches_the_oracle(objective):
    t, y, dy = transit_curve(3000, span=27.0, period=3.1, depth=3e-3, seed=3)
    segments = [(np.geomspace(0.5, 1.0, 700), np.geomspace(0.01, 0.06, 8)),
                (np.geomspace(1.0, 2.0, 700), np.geomspace(0.01, 0.12, 8)),
                (np.geomspace(2.0, 9.0, 900), np.geomspace(0.02, 0.24, 8))]
    got, ms = ref_gpu.search_curve(t, y, dy, segments, 10, objective=objective)
    ref = np.concatenate([np.stack([oracle.bls_power(t, y, dy, p, d, 10, objective=objective)[f]
                                    for f in oracle.OUTPUT_NAMES]) for p, d in segments], axis=1)
    fin = np.isfinite(ref[0])
    np.testing.assert_array_equal(np.isneginf(got[0]), np.isneginf(ref[0]))
    np.testing.assert_allclose(got[0][fin], ref[0][fin], rtol=1e-9, atol=0.0)
    assert int(np.argmax(got[0])) == int(np.argmax(ref[0]))
    assert ms > 0.0


def test_reference_kernel_float32_opt_in_finds_the_same_best_period():
    # the reference's float32 opt-in (tests/test_bls_segments.py:89-107 asks >= 99%
    # of periods close and the same argmax)
    t, y, dy = transit_curve(2000, span=27.0, period=2.3, depth=5e-3, seed=4)
    segments = [(np.geomspace(0.6, 6.0, 1500), np.geomspace(0.02, 0.2, 6))]
    got, _ = ref_gpu.search_curve(t, y, dy, segments, 10, precision="float32")
    ref = oracle.bls_power(t, y, dy, *segments[0], 10)["power"]
    assert int(np.argmax(got[0])) == int(np.argmax(ref))
    close = np.isclose(got[0], ref, rtol=1e-3, atol=0.0)
    assert close.mean() >= 0.99
