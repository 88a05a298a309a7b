"""Tile shapes on the device: every autotuner candidate gives the default
engine's output (bit for bit with exact integer sums), and the autotuner picks a
shape that runs."""

from __future__ import annotations

import numpy as np
import pytest

from _cases import transit_curve

pytestmark = pytest.mark.gpu


def _batch(objective: int):
    from cuperiod_b200 import _lib
    from cuperiod_b200.bls import _grid_segments
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings
    from cuperiod_b200.synthetic import batched_curves
    # six segments of the batched workload's 0.3-13 d grid (histograms of ~600 to
    # ~2000 bins, so the shapes cut the segments into different tiles)
    segments = _grid_segments(GridSpec(kind="period", values=np.geomspace(0.3, 13.0, 3000)),
                              BLSSettings())
    grid = _lib.PackedGrid.from_segments(segments, 10, objective)
    curves = [(c.t, c.y, None) for c in batched_curves(8, seed=41, n_range=(500, 5000))]
    curves.append(transit_curve(1500, weights="hetero", seed=42))     # per-point, narrow
    curves.append(transit_curve(900, weights="wild", seed=43))        # per-point, FP64 sums
    return grid, _lib.PackedCurves.from_arrays(curves)


@pytest.mark.parametrize("objective", [0, 1])
def test_every_candidate_shape_gives_the_default_output(objective):
    from cuperiod_b200 import _lib
    from cuperiod_b200.autotune import CANDIDATES
    grid, packed = _batch(objective)
    base_eng = _lib.Engine()
    base = base_eng.search(grid, packed)
    base_eng.close()
    exact = slice(0, 9)           # one weight and narrow per-point weights: integer sums
    for shape in CANDIDATES[1:]:
        eng = _lib.Engine(**shape.engine_kwargs())
        try:
            out = eng.search(grid, packed)
            info = eng.info()
        finally:
            eng.close()
        assert info["smem_per_cta"] >= (shape.smem_per_cta or 0), shape
        np.testing.assert_array_equal(out[:, exact], base[:, exact], err_msg=shape.label())
        # FP64 sums in atomic order: equal to rounding, same best period
        p_out, p_base = out[0, 9], base[0, 9]
        fin = np.isfinite(p_base)
        np.testing.assert_array_equal(np.isfinite(p_out), fin)
        np.testing.assert_allclose(p_out[fin], p_base[fin], rtol=1e-9)
        assert np.argmax(np.where(fin, p_out, -np.inf)) == np.argmax(np.where(fin, p_base,
                                                                             -np.inf))


def test_autotune_picks_a_runnable_shape_and_its_engine_matches(tmp_path):
    from cuperiod_b200 import _lib
    from cuperiod_b200.autotune import CANDIDATES, tuned_engine
    grid, packed = _batch(0)
    eng, res = tuned_engine(grid, packed, sample=6, refresh=True,
                            cache=tmp_path / "tune.json")
    try:
        assert res.shape in CANDIDATES and not res.cached
        assert set(res.ms) | set(res.errors) == {s.label() for s in CANDIDATES}
        assert all(ms > 0.0 for ms in res.ms.values())
        assert res.ms[res.shape.label()] == min(res.ms.values())
        out = eng.search(grid, packed)
    finally:
        eng.close()
    ref = _lib.Engine()
    try:
        base = ref.search(grid, packed)
        ms = ref.time_launches(2)
    finally:
        ref.close()
    assert ms > 0.0
    np.testing.assert_array_equal(out[:, :9], base[:, :9])
