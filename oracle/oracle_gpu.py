"""TEST INFRASTRUCTURE ONLY -- the all-FP64 GPU oracle.

``bls_oracle_gpu.cu`` restates cuPeriod's unscreened numba box search
(``src/cuperiod/methods/_bls_core.py:341-462``) on the GPU, bit for bit: every
bin sum and prefix in the reference's sequential order, every FP64 operation
rounded on its own.  It checks the engine where the CPU oracle is too slow (the
4-year workload: 60,000 points x 200,000 periods per curve).  Host steps are
the CPU oracle's (``oracle.py``).  Only ``tests/`` and ``bench.py``'s precision
checks use it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from . import oracle

_HERE = os.path.dirname(os.path.abspath(__file__))
_PATH = os.path.join(_HERE, "liboracle_gpu.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_PATH):
            subprocess.run(["make", "-s", "-C", _HERE, "liboracle_gpu.so"], check=True)
        lib = ctypes.CDLL(_PATH)
        p, i32, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.oracle_gpu_search.argtypes = [p, p, p, i32, p, i32, p, i32, d, i32, i32, d, d, d, i32,
                                          d, p, p]
        lib.oracle_gpu_search.restype = i32
        _lib = lib
    return _lib


def bls_power_segments(t, y, dy, segments, oversample: int = 10, *,
                       objective: str = "snr") -> np.ndarray:
    """The unscreened search of one curve over every ``(periods, durations)``
    segment: (7, total periods) FP64 in the reference's field order."""
    import torch
    lib = _load()
    th, yh, ih = oracle.host_inputs(t, y, dy)
    yw = np.ascontiguousarray(yh * ih)
    t_min = float(th.min())
    tau = np.ascontiguousarray(th - t_min)
    sum_y, sum_ivar = float(yw.sum()), float(ih.sum())
    floor = oracle.ivar_floor(tau.size, sum_ivar)
    flag = oracle.objective_flag(objective)
    dev = [torch.from_numpy(a).cuda() for a in (tau, yw, np.ascontiguousarray(ih))]
    outs = []
    for periods, durations in segments:
        spec = oracle.search_spec(periods, durations, oversample)
        per = torch.from_numpy(np.ascontiguousarray(spec.periods)).cuda()
        db = torch.from_numpy(np.asarray(spec.dur_bins, dtype=np.int64)).cuda()
        out = torch.empty((7, per.numel()), dtype=torch.float64, device="cuda")
        rc = lib.oracle_gpu_search(dev[0].data_ptr(), dev[1].data_ptr(), dev[2].data_ptr(),
                                   tau.size, per.data_ptr(), per.numel(), db.data_ptr(),
                                   db.numel(), spec.bin_duration, int(oversample), spec.width,
                                   sum_y, sum_ivar, t_min, flag, floor, out.data_ptr(), None)
        if rc != 0:
            raise RuntimeError(f"GPU oracle failed ({rc})")
        outs.append(out)
    return torch.cat(outs, dim=1).cpu().numpy()


def bls_power(t, y, dy, periods, durations, oversample: int, *, objective: str = "snr") -> dict:
    """``oracle.bls_power`` on the GPU (one segment)."""
    out = bls_power_segments(t, y, dy, [(periods, durations)], oversample, objective=objective)
    res = dict(zip(oracle.OUTPUT_NAMES, out))
    res["period"] = np.ascontiguousarray(periods, dtype=np.float64)
    return res
