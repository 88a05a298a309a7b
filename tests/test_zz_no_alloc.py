"""The allocation-free search (bls_launch_best_noalloc) against the allocating one.

Collected last (file name), so it runs both alone and after every other GPU test
has used the library's engines.
"""

from __future__ import annotations

import numpy as np
import pytest

from tests._cases import transit_curve

pytestmark = pytest.mark.gpu

# Per-point-weight curves keep FP64 bin sums added in atomic order, so two runs
# of the same search may differ in the last bits of their powers; one-weight
# curves are exact integers and agree bit for bit.
RTOL = 1e-12


@pytest.fixture(scope="module")
def lib():
    from cuperiod_b200 import _lib
    return _lib


def _batch(lib):
    from cuperiod_b200.bls import _grid_segments
    from cuperiod_b200.grid import GridSpec
    from cuperiod_b200.settings import BLSSettings

    curves = [transit_curve(n, span=27.0, period=p, depth=4e-3, seed=s, weights=w)
              for n, p, s, w in ((900, 2.3, 11, "uniform"), (2500, 4.1, 12, "hetero"),
                                 (1700, 1.7, 13, "uniform"), (600, 6.2, 14, "wild"),
                                 (3000, 3.3, 15, "uniform"))]
    settings = BLSSettings()
    segments = _grid_segments(GridSpec(kind="period", values=np.geomspace(0.5, 9.0, 4000)),
                              settings)
    grid = lib.PackedGrid.from_segments(segments, settings.bins_per_duration, 0)
    return grid, lib.PackedCurves.from_arrays(curves)


def test_no_alloc_matches_the_allocating_path_twice(lib):
    import torch

    grid, curves = _batch(lib)
    torch.cuda.init()
    torch.cuda.mem_get_info()
    eng = lib.Engine(use_graph=False)
    try:
        eng.prepare(grid, curves)
        eng.launch()
        ref = eng.download_best()
        torch.cuda.synchronize()
        # every buffer of the allocating path exists now; from here on neither the
        # device's free memory nor torch's allocator may move, the first call (which
        # looks up the static array's address) included
        free0 = torch.cuda.mem_get_info()[0]
        torch0 = torch.cuda.memory_allocated()
        for _ in range(2):                      # the counters must be zeroed again
            got = eng.launch_best_noalloc()
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0
            assert torch.cuda.memory_allocated() == torch0
            np.testing.assert_array_equal(got[0], ref[0])
            for g, r in zip(got[1:], ref[1:]):
                np.testing.assert_allclose(g, r, rtol=RTOL, atol=0.0)
    finally:
        eng.close()


def test_no_alloc_refuses_more_curves_than_its_scratch(lib):
    n = 65537
    t = np.linspace(0.0, 5.0, 8)
    y = 1.0 + 1e-3 * np.sin(np.arange(8.0))
    dy = np.full(8, 1e-3)
    curves = lib.PackedCurves.from_arrays([(t, y, dy)] * n)
    grid = lib.PackedGrid.from_segments([(np.array([1.3]), np.array([0.2]))], 10, 0)
    eng = lib.Engine(use_graph=False)
    try:
        eng.prepare(grid, curves)
        with pytest.raises(ValueError, match="65536"):
            eng.launch_best_noalloc()
    finally:
        eng.close()


def test_no_alloc_needs_a_prepared_batch(lib):
    eng = lib.Engine()
    z = np.zeros(1)
    i = np.zeros(1, dtype=np.int64)
    try:
        rc = eng._lib.bls_launch_best_noalloc(eng._h, i.ctypes.data, z.ctypes.data,
                                              z.ctypes.data, z.ctypes.data, None)
        assert rc == lib.BLS_E_STATE
        assert b"before bls_prepare" in eng._lib.bls_last_error()
    finally:
        eng.close()
