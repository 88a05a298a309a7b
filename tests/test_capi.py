"""The C ABI library loads without a GPU and exports every function the public
header declares."""

from __future__ import annotations

import ctypes
import os
import re

from conftest import ROOT


def _declared():
    inc = os.path.join(ROOT, "include")
    text = "\n".join(open(os.path.join(inc, f)).read() for f in sorted(os.listdir(inc))
                     if f.endswith(".h"))
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+((?:bls|pn)_\w+)\(", text, re.M)))


def test_header_declares_the_entry_points():
    names = _declared()
    for must in ("bls_engine_create", "bls_engine_destroy", "bls_last_error", "bls_prepare",
                 "bls_launch", "bls_download", "bls_download_best", "bls_search",
                 "bls_batch_info", "bls_debug_fold_bins", "bls_debug_prefix",
                 "bls_download_curves", "pn_gemm", "pn_bin_curves", "pn_topk"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from cuperiod_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_the_header():
    from cuperiod_b200 import _lib
    # BlsTune: 5 int32; BlsGrid: int32 + 4 pointers + 2 int32 (padded); BlsCurves: int32 + 4 ptrs
    assert ctypes.sizeof(_lib.BlsTune) == 20
    assert ctypes.sizeof(_lib.BlsGrid) == 8 + 4 * 8 + 8
    assert ctypes.sizeof(_lib.BlsCurves) == 8 + 4 * 8
    assert ctypes.sizeof(_lib.BlsBatchInfo) == 4 + 4 + 8 * 3 + 8 * 3 + 8 + 4 * 4 + 8 + 4 + 4


def test_engine_creation_without_a_device_raises():
    import pytest
    import torch
    from cuperiod_b200 import _lib
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises((_lib.EngineError, RuntimeError)):
        _lib.Engine()


def test_packed_curves_concatenate_in_order():
    # large batches are copied by several host threads; the layout is the plain
    # concatenation, missing errors filled with ones, and no error array at all
    # when no curve has one
    import numpy as np

    from cuperiod_b200 import _lib
    rng = np.random.default_rng(4)
    sizes = rng.integers(1, 40000, 120)
    curves = [(rng.uniform(size=n), rng.normal(size=n), None if i % 4 else rng.uniform(size=n))
              for i, n in enumerate(sizes)]
    pc = _lib.PackedCurves.from_arrays(curves)
    assert pc.t.size == sizes.sum() > (1 << 21)
    np.testing.assert_array_equal(pc.offsets, np.concatenate([[0], np.cumsum(sizes)]))
    np.testing.assert_array_equal(pc.t, np.concatenate([c[0] for c in curves]))
    np.testing.assert_array_equal(pc.y, np.concatenate([c[1] for c in curves]))
    np.testing.assert_array_equal(
        pc.dy, np.concatenate([np.ones(c[0].size) if c[2] is None else c[2] for c in curves]))
    assert _lib.PackedCurves.from_arrays([(c[0], c[1], None) for c in curves]).dy is None
    empty = _lib.PackedCurves.from_arrays([(np.zeros(0), np.zeros(0), None)])
    assert empty.t.size == 0 and empty.n_curves == 1
