"""TEST AND MEASUREMENT INFRASTRUCTURE ONLY -- the reference's own GPU kernel.

cuPeriod's ``bls_block`` (``src/cuperiod/methods/_bls_core.py:505-656``),
compiled from the reference's source for sm_100a by ``build_ref_gpu.py`` into
``oracle/_ref/libref_bls_block.so``, driven as ``_bls_search_cuda_specs``
(``:741-840``) drives it for one light curve: the host steps of ``bls_power``
(median-centred flux, ``ivar = 1/dy^2``, numpy's sums, ``_ivar_floor``), one
upload, one launch per segment, one download.  It is the "reference GPU kernel
on the same box" baseline and is never part of the engine.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import oracle

_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libref_bls_block.so")
_lib = None
F32_EPS = float(np.finfo(np.float32).eps)


def available() -> bool:
    return os.path.exists(_PATH)


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(_PATH)
        p, i32, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.ref_bls_search_curve.argtypes = [p, p, p, i32, p, p, p, p, p, p, i32, i32, i32, d, d,
                                             d, d, i32, p, p]
        lib.ref_bls_search_curve.restype = i32
        _lib = lib
    return _lib


def search_curve(t, y, dy, segments, oversample: int = 10, *, objective: str = "snr",
                 precision: str = "float64") -> tuple[np.ndarray, float]:
    """All segments of one curve through the reference's kernel: ``(out, kernel_ms)``
    with ``out`` the (7, n_periods) fields in the reference's order."""
    lib = _load()
    th, yh, ih = oracle.host_inputs(t, y, dy)
    t_min = float(th.min())
    tau = np.ascontiguousarray(th - t_min)
    yw = np.ascontiguousarray(yh * ih)
    sum_y, sum_ivar = float(yw.sum()), float(ih.sum())
    f32 = precision == "float32"
    floor = oracle.ivar_floor(tau.size, sum_ivar)
    if f32:             # _ivar_floor(..., float32=True), _bls_core.py:75-94
        floor = max(floor, 8.0 * F32_EPS * sum_ivar)
    floor = max(floor, float(np.finfo(np.float32 if f32 else np.float64).tiny))
    specs = [oracle.search_spec(p, d, oversample) for p, d in segments]
    periods = np.ascontiguousarray(np.concatenate([s.periods for s in specs]), dtype=np.float64)
    seg_sizes = np.array([s.periods.size for s in specs], dtype=np.int32)
    dur = np.ascontiguousarray(np.concatenate([np.asarray(s.dur_bins, dtype=np.int32)
                                               for s in specs]), dtype=np.int32)
    dur_sizes = np.array([len(s.dur_bins) for s in specs], dtype=np.int32)
    bins = np.array([s.bin_duration for s in specs], dtype=np.float64)
    widths = np.array([s.width for s in specs], dtype=np.int32)
    out = np.empty((7, periods.size), dtype=np.float64)
    ms = ctypes.c_float(0.0)
    rc = lib.ref_bls_search_curve(
        tau.ctypes.data, yw.ctypes.data, ih.ctypes.data, tau.size, periods.ctypes.data,
        seg_sizes.ctypes.data, dur.ctypes.data, dur_sizes.ctypes.data, bins.ctypes.data,
        widths.ctypes.data, len(specs), int(oversample), oracle.objective_flag(objective),
        sum_y, sum_ivar, t_min, floor, 1 if f32 else 0, out.ctypes.data, ctypes.byref(ms))
    if rc != 0:
        raise RuntimeError(f"reference GPU kernel failed ({rc})")
    return out, float(ms.value)
