"""ctypes binding of the engine library ``libbls_b200.so`` (``include/bls_b200.h``).

The library is built in-tree by ``csrc/Makefile``.  There is no fallback: if it
is missing, or no CUDA device is usable, every entry point raises
:class:`~cuperiod_b200.errors.BackendUnavailableError`.
"""

from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from .errors import BackendUnavailableError, EngineError  # noqa: F401  (re-exported)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbls_b200.so")

BLS_OK, BLS_E_INVALID, BLS_E_CUDA, BLS_E_RESOURCE, BLS_E_NOMEM, BLS_E_DEVICE, BLS_E_STATE = range(7)
N_FIELDS = 7
FIELD_NAMES = ("power", "depth", "depth_err", "depth_snr", "duration", "transit_time",
               "log_likelihood")
#: Fields of the joint-ephemeris search (``JOINT_FIELDS``, multiband/_bls_joint.py:52-54).
JOINT_FIELD_NAMES = ("power", "depth", "depth_snr", "duration", "transit_time", "band_index")

_i32, _i64, _dbl, _vp = ctypes.c_int32, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p


class BlsTune(ctypes.Structure):
    _fields_ = [("device", _i32), ("smem_per_cta", _i32), ("max_tile", _i32), ("use_graph", _i32),
                ("exact_sweep", _i32)]


class BlsGrid(ctypes.Structure):
    _fields_ = [("n_segments", _i32), ("seg_offsets", _vp), ("periods", _vp),
                ("dur_offsets", _vp), ("durations", _vp), ("oversample", _i32),
                ("objective", _i32)]


class BlsCurves(ctypes.Structure):
    _fields_ = [("n_curves", _i32), ("offsets", _vp), ("t", _vp), ("y", _vp), ("dy", _vp)]


class BlsTlsInputs(ctypes.Structure):
    _fields_ = [("n_curves", _i32), ("offsets", _vp), ("tau", _vp), ("yw", _vp), ("w", _vp),
                ("w_total", _vp), ("n_bins", _i32), ("n_dur", _i32), ("dur_bins", _vp),
                ("templates", _vp), ("den_rel", _dbl)]


#: Per-period outputs of the TLS kernel, in the C ABI's order.
TLS_FIELD_NAMES = ("sr", "depth", "duration", "t0")


class BlsDefaultGrid(ctypes.Structure):
    _fields_ = [("min_period_days", _dbl), ("max_period_days", _dbl), ("min_transits", _dbl),
                ("segment_factor", _dbl), ("grid_duration_frac", _dbl),
                ("grid_oversample", _dbl), ("n_starts", _i32), ("oversample", _i32),
                ("objective", _i32), ("reserved", _i32), ("dur_offsets", _vp),
                ("durations", _vp)]


class BlsBatchInfo(ctypes.Structure):
    _fields_ = [("n_curves", _i32), ("n_segments", _i32), ("n_periods", _i64),
                ("n_items", _i64), ("n_points", _i64), ("folds", _dbl), ("boxes", _dbl),
                ("trials", _dbl), ("h2d_bytes", _i64), ("ctas", _i32), ("smem_per_cta", _i32),
                ("uniform_curves", _i32), ("fast_fold_segments", _i32), ("spectrum", _i64),
                ("n_grids", _i32), ("reserved", _i32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib: ctypes.CDLL | None = None
_lib_lock = threading.Lock()


def load() -> ctypes.CDLL:
    """The engine library, loaded once; raises if it was not built."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise BackendUnavailableError(
                f"BLS engine library {LIB_PATH} is not built (run `make -C "
                f"{os.path.join(_HERE, 'csrc')}` or __graft_entry__.build())")
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        lib.bls_last_error.restype = ctypes.c_char_p
        lib.bls_last_error.argtypes = []
        lib.bls_engine_create.argtypes = [P(BlsTune), P(_vp)]
        lib.bls_engine_destroy.argtypes = [_vp]
        lib.bls_prepare.argtypes = [_vp, P(BlsGrid), P(BlsCurves), _vp]
        lib.bls_launch.argtypes = [_vp, _vp]
        lib.bls_download.argtypes = [_vp, _vp, _vp]
        lib.bls_download_curves.argtypes = [_vp, _vp, _i32, _vp, _vp]
        lib.bls_device_output.argtypes = [_vp, P(_vp)]
        lib.bls_download_best.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
        lib.bls_launch_best_noalloc.argtypes = [_vp, _vp, _vp, _vp, _vp, _vp]
        lib.bls_download_rows.argtypes = [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp]
        lib.bls_search.argtypes = [_vp, P(BlsGrid), P(BlsCurves), _vp, _vp]
        lib.bls_batch_info.argtypes = [_vp, P(BlsBatchInfo)]
        lib.bls_time_launches.argtypes = [_vp, _i32, P(_dbl), _vp]
        lib.bls_prepare_grids.argtypes = [_vp, _i32, P(BlsGrid), _vp, P(BlsCurves), _vp]
        lib.bls_default_grid.argtypes = [P(BlsDefaultGrid), _dbl, _i64, _vp, _vp, _vp,
                                         P(_i32), P(_i64)]
        lib.bls_default_grid_sizes.argtypes = [P(BlsDefaultGrid), _i32, _vp, _vp]
        lib.bls_prepare_default.argtypes = [_vp, P(BlsDefaultGrid), _vp, P(BlsCurves), _vp]
        lib.bls_search_joint.argtypes = [_vp, P(BlsGrid), P(BlsCurves), _vp, _vp]
        lib.bls_tls_search.argtypes = [_vp, P(BlsTlsInputs), _vp, _i64, _vp, _vp]
        lib.bls_tls_prepare.argtypes = [_vp, P(BlsTlsInputs), _vp, _i64, _vp]
        lib.bls_tls_launch.argtypes = [_vp, _vp]
        lib.bls_tls_download.argtypes = [_vp, _vp, _vp]
        lib.bls_joint_prepare.argtypes = [_vp, P(BlsGrid), P(BlsCurves), _vp]
        lib.bls_joint_launch.argtypes = [_vp, _vp]
        lib.bls_joint_download.argtypes = [_vp, _vp, _vp]
        lib.bls_debug_fold_bins.argtypes = [_vp, _vp, _i64, _dbl, _dbl, _i32, _vp, _vp]
        lib.bls_debug_prefix.argtypes = [_vp, _vp, _vp, _vp, _i64, _dbl, _vp, _i32, _i32, _vp, _vp,
                                         _vp]
        for name in ("bls_engine_create", "bls_engine_destroy", "bls_prepare", "bls_launch",
                     "bls_download", "bls_download_curves", "bls_device_output", "bls_download_best", "bls_search",
                     "bls_batch_info", "bls_debug_fold_bins", "bls_debug_prefix",
                     "bls_launch_best_noalloc", "bls_download_rows", "bls_search_joint",
                     "bls_joint_prepare", "bls_joint_launch", "bls_joint_download",
                     "bls_tls_search", "bls_tls_prepare", "bls_tls_launch",
                     "bls_tls_download", "bls_time_launches", "bls_prepare_grids",
                     "bls_default_grid", "bls_default_grid_sizes", "bls_prepare_default"):
            getattr(lib, name).restype = ctypes.c_int
        _lib = lib
        return lib


def _check(rc: int) -> None:
    if rc == BLS_OK:
        return
    msg = (load().bls_last_error() or b"").decode(errors="replace")
    if rc == BLS_E_INVALID:
        raise ValueError(msg)
    if rc == BLS_E_RESOURCE:
        raise BackendUnavailableError(msg)
    raise EngineError(f"BLS engine error {rc}: {msg}")


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _addr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


@dataclass
class PackedGrid:
    """A segmented period grid in the C ABI's layout (keeps its arrays alive)."""
    seg_offsets: np.ndarray
    periods: np.ndarray
    dur_offsets: np.ndarray
    durations: np.ndarray
    oversample: int
    objective: int

    @classmethod
    def from_segments(cls, segments, oversample: int, objective: int) -> "PackedGrid":
        per = [_f64(p).ravel() for p, _ in segments]
        dur = [_f64(d).ravel() for _, d in segments]
        seg_off = np.zeros(len(segments) + 1, dtype=np.int64)
        dur_off = np.zeros(len(segments) + 1, dtype=np.int64)
        seg_off[1:] = np.cumsum([p.size for p in per]) if per else []
        dur_off[1:] = np.cumsum([d.size for d in dur]) if dur else []
        return cls(seg_off, _f64(np.concatenate(per)) if per else np.empty(0),
                   dur_off, _f64(np.concatenate(dur)) if dur else np.empty(0),
                   int(oversample), int(objective))

    @property
    def n_periods(self) -> int:
        return int(self.seg_offsets[-1])

    def struct(self) -> BlsGrid:
        return BlsGrid(len(self.seg_offsets) - 1, _addr(self.seg_offsets), _addr(self.periods),
                       _addr(self.dur_offsets), _addr(self.durations), self.oversample,
                       self.objective)


@dataclass
class DefaultGridSpec:
    """The default-grid parameters in the C ABI's layout (``BlsDefaultGrid``),
    with the box durations of each segment start (keeps its arrays alive)."""
    min_period_days: float
    max_period_days: float
    min_transits: float
    segment_factor: float
    grid_duration_frac: float
    grid_oversample: float
    dur_offsets: np.ndarray         # n_starts + 1
    durations: np.ndarray
    oversample: int
    objective: int

    def struct(self) -> BlsDefaultGrid:
        return BlsDefaultGrid(float(self.min_period_days), float(self.max_period_days),
                              float(self.min_transits), float(self.segment_factor),
                              float(self.grid_duration_frac), float(self.grid_oversample),
                              len(self.dur_offsets) - 1, int(self.oversample),
                              int(self.objective), 0, _addr(self.dur_offsets),
                              _addr(self.durations))


def default_grid(spec: DefaultGridSpec, baseline: float):
    """The default grid of one baseline built by the engine library on the host:
    ``(periods, seg_offsets, seg_start)`` (``bls_default_grid``)."""
    lib = load()
    st = spec.struct()
    ns, npd = _i32(0), _i64(0)
    _check(lib.bls_default_grid(ctypes.byref(st), float(baseline), 0, None, None, None,
                                ctypes.byref(ns), ctypes.byref(npd)))
    periods = np.empty(npd.value, dtype=np.float64)
    offs = np.empty(ns.value + 1, dtype=np.int64)
    starts = np.empty(ns.value, dtype=np.int32)
    _check(lib.bls_default_grid(ctypes.byref(st), float(baseline), periods.size,
                                periods.ctypes.data, offs.ctypes.data, starts.ctypes.data,
                                ctypes.byref(ns), ctypes.byref(npd)))
    return periods, offs, starts


def default_grid_sizes(spec: DefaultGridSpec, baselines) -> np.ndarray:
    """Periods of the default grid of each baseline (-1: none can be built)."""
    lib = load()
    b = _f64(baselines).ravel()
    out = np.empty(b.size, dtype=np.int64)
    st = spec.struct()
    _check(lib.bls_default_grid_sizes(ctypes.byref(st), b.size, b.ctypes.data,
                                      out.ctypes.data))
    return out


_PACK_THREADS = max(1, min(16, os.cpu_count() or 1))
_pack_pool = None
_pack_pool_lock = threading.Lock()


def _concat(parts, off: np.ndarray, fill: float | None = None) -> np.ndarray:
    """The arrays of ``parts`` (``None``: ``fill``) end to end at ``off``; large
    batches are copied by several host threads (numpy's copies release the GIL),
    each writing, and so first touching, its own share of the output."""
    global _pack_pool
    total = int(off[-1])
    out = np.empty(total, dtype=np.float64)
    if total == 0:
        return out

    def copy(lo: int, hi: int) -> None:
        for i in range(lo, hi):
            dst = out[off[i]:off[i + 1]]
            if parts[i] is None:
                dst.fill(fill)
            else:
                dst[...] = parts[i]

    n = len(parts)
    k = min(_PACK_THREADS, n, max(1, total // (1 << 20)))      # >= 1M points a thread
    if k <= 1:
        copy(0, n)
        return out
    with _pack_pool_lock:
        if _pack_pool is None:
            from concurrent.futures import ThreadPoolExecutor
            _pack_pool = ThreadPoolExecutor(max_workers=_PACK_THREADS,
                                            thread_name_prefix="bls-pack")
        pool = _pack_pool
    # split by points, not curves, so the threads' shares are even
    cuts = np.searchsorted(off, np.linspace(0, total, k + 1)).tolist()
    cuts[0], cuts[-1] = 0, n
    for f in [pool.submit(copy, a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]:
        f.result()
    return out


@dataclass
class PackedCurves:
    """Light curves concatenated in the C ABI's layout (keeps its arrays alive)."""
    offsets: np.ndarray
    t: np.ndarray
    y: np.ndarray
    dy: np.ndarray | None

    @classmethod
    def from_arrays(cls, curves) -> "PackedCurves":
        ts, ys, dys = [], [], []
        any_dy = any(c[2] is not None for c in curves)
        for t, y, dy in curves:
            t, y = _f64(t).ravel(), _f64(y).ravel()
            if t.shape != y.shape:
                raise ValueError("t and y must have the same length")
            ts.append(t)
            ys.append(y)
            if any_dy:
                dys.append(None if dy is None else _f64(dy).ravel())
        off = np.zeros(len(curves) + 1, dtype=np.int64)
        off[1:] = np.cumsum([t.size for t in ts])
        return cls(off, _concat(ts, off), _concat(ys, off),
                   _concat(dys, off, fill=1.0) if any_dy else None)

    @property
    def n_curves(self) -> int:
        return len(self.offsets) - 1

    def struct(self) -> BlsCurves:
        return BlsCurves(self.n_curves, _addr(self.offsets), _addr(self.t), _addr(self.y),
                         _addr(self.dy))


class Engine:
    """One engine = one device context, stream, buffer set and graph cache.

    Not thread-safe (like the reference's per-worker engines,
    src/cuperiod/methods/base.py:388-396): use one per thread.
    """

    def __init__(self, device: int = -1, *, smem_per_cta: int = 0, max_tile: int = 0,
                 use_graph: bool = True, exact_sweep: bool = False) -> None:
        self._lib = load()
        tune = BlsTune(int(device), int(smem_per_cta), int(max_tile), int(bool(use_graph)),
                       int(bool(exact_sweep)))
        handle = _vp()
        _check(self._lib.bls_engine_create(ctypes.byref(tune), ctypes.byref(handle)))
        self._h = handle
        self._grid: PackedGrid | None = None
        self._curves: PackedCurves | None = None
        self._spec_off = np.zeros(1, dtype=np.int64)
        self._joint_periods = 0
        self._tls_shape = (0, 0)

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.bls_engine_destroy(self._h)
            self._h = None

    def __del__(self) -> None:  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def prepare(self, grid: PackedGrid, curves: PackedCurves, stream: int | None = None) -> None:
        self._grid, self._curves = grid, curves
        self._spec_off = np.arange(curves.n_curves + 1, dtype=np.int64) * grid.n_periods
        g, c = grid.struct(), curves.struct()
        _check(self._lib.bls_prepare(self._h, ctypes.byref(g), ctypes.byref(c), stream))

    def prepare_grids(self, grids: Sequence[PackedGrid], grid_of_curve, curves: PackedCurves,
                      stream: int | None = None) -> None:
        """A batch whose curves have their own grids, searched in one launch:
        curve ``c`` over ``grids[grid_of_curve[c]]`` (``bls_prepare_grids``)."""
        gids = np.ascontiguousarray(grid_of_curve, dtype=np.int32).reshape(-1)
        if gids.size != curves.n_curves:
            raise ValueError("grid_of_curve needs one grid index per curve")
        if not grids:
            raise ValueError("at least one grid is required")
        structs = (BlsGrid * len(grids))(*[g.struct() for g in grids])
        c = curves.struct()
        # one grid: the layout of ``prepare``, so ``download`` keeps its shape
        self._grid, self._curves = (grids[0] if len(grids) == 1 else None), curves
        counts = np.array([g.n_periods for g in grids], dtype=np.int64)
        if gids.size and (gids.min() < 0 or gids.max() >= len(grids)):
            raise ValueError("grid_of_curve holds an index outside the grids")
        self._spec_off = np.concatenate([[0], np.cumsum(counts[gids])]).astype(np.int64)
        _check(self._lib.bls_prepare_grids(self._h, len(grids), structs, gids.ctypes.data,
                                           ctypes.byref(c), stream))

    def prepare_default(self, spec: DefaultGridSpec, baselines, curves: PackedCurves,
                        stream: int | None = None) -> None:
        """Every curve over the default grid of its baseline, the grids built by
        the library on the host cores, in one launch (``bls_prepare_default``)."""
        b = _f64(baselines).ravel()
        if b.size != curves.n_curves:
            raise ValueError("one baseline per curve is required")
        sizes = default_grid_sizes(spec, b)
        st, c = spec.struct(), curves.struct()
        self._grid, self._curves = None, curves
        self._spec_off = np.concatenate([[0], np.cumsum(np.maximum(sizes, 0))]).astype(np.int64)
        _check(self._lib.bls_prepare_default(self._h, ctypes.byref(st), b.ctypes.data,
                                             ctypes.byref(c), stream))

    @property
    def spectrum_offsets(self) -> np.ndarray:
        """Curve ``c``'s periods in the prepared batch's flat spectra:
        ``[offsets[c], offsets[c + 1])``."""
        return self._spec_off

    def download_flat(self, stream: int | None = None) -> np.ndarray:
        """All fields of every curve, ``(7, spectrum)``: curve ``c`` at
        ``[:, spectrum_offsets[c]:spectrum_offsets[c + 1]]`` (its grid's order)."""
        assert self._curves is not None
        out = np.empty((N_FIELDS, int(self._spec_off[-1])), dtype=np.float64)
        _check(self._lib.bls_download(self._h, out.ctypes.data, stream))
        return out

    def download_curves(self, curve_ids, stream: int | None = None) -> list[np.ndarray]:
        """Every field of the listed curves only: one ``(7, spectrum)`` array
        per id (``bls_download_curves``)."""
        ids = np.ascontiguousarray(curve_ids, dtype=np.int32).reshape(-1)
        if ids.size and (ids.min() < 0 or ids.max() >= len(self._spec_off) - 1):
            raise ValueError("curve id outside the prepared batch")
        lens = self._spec_off[ids + 1] - self._spec_off[ids]
        flat = np.empty(int(N_FIELDS * lens.sum()), dtype=np.float64)
        _check(self._lib.bls_download_curves(self._h, ids.ctypes.data, int(ids.size),
                                             flat.ctypes.data, stream))
        out, w = [], 0
        for n in lens.tolist():
            out.append(flat[w:w + N_FIELDS * n].reshape(N_FIELDS, n))
            w += N_FIELDS * n
        return out

    def launch(self, stream: int | None = None) -> None:
        _check(self._lib.bls_launch(self._h, stream))

    def time_launches(self, reps: int = 1, stream: int | None = None) -> float:
        """Mean device milliseconds of one launch of the prepared batch over
        ``reps`` launches (CUDA events on the launching stream)."""
        ms = _dbl(0.0)
        _check(self._lib.bls_time_launches(self._h, int(reps), ctypes.byref(ms), stream))
        return float(ms.value)

    def download(self, stream: int | None = None) -> np.ndarray:
        """All fields: array of shape (7, n_curves, n_periods) (one grid; after
        ``prepare_grids`` use ``download_flat``)."""
        if self._grid is None:
            raise ValueError("the prepared batch has one grid per curve: use download_flat")
        assert self._curves is not None
        out = np.empty((N_FIELDS, self._curves.n_curves, self._grid.n_periods), dtype=np.float64)
        _check(self._lib.bls_download(self._h, out.ctypes.data, stream))
        return out

    def download_best(self, stream: int | None = None):
        assert self._curves is not None
        n = self._curves.n_curves
        idx = np.empty(n, dtype=np.int64)
        val, mean, std = (np.empty(n, dtype=np.float64) for _ in range(3))
        _check(self._lib.bls_download_best(self._h, idx.ctypes.data, val.ctypes.data,
                                           mean.ctypes.data, std.ctypes.data, stream))
        return idx, val, mean, std

    def rows(self, n_best: int, harmonic_max: int, min_separation, alias_tolerance,
             stream: int | None = None):
        """The prepared batch's result-row peaks ranked on the device:
        ``(n_peaks (C,), index (C, n_best), fields (C, n_best, 8))`` with fields
        period, frequency, power, depth, depth_snr, duration, t0, sde."""
        assert self._curves is not None
        n = self._curves.n_curves
        sep = np.ascontiguousarray(min_separation, dtype=np.float64).reshape(n)
        tol = np.ascontiguousarray(alias_tolerance, dtype=np.float64).reshape(n)
        counts = np.empty(n, dtype=np.int32)
        index = np.empty((n, n_best), dtype=np.int64)
        fields = np.empty((n, n_best, 8), dtype=np.float64)
        _check(self._lib.bls_download_rows(self._h, int(n_best), int(harmonic_max),
                                           sep.ctypes.data, tol.ctypes.data, counts.ctypes.data,
                                           index.ctypes.data, fields.ctypes.data, stream))
        return counts, index, fields

    def launch_best_noalloc(self, stream: int | None = None):
        """Search the prepared batch and return its per-curve best, allocating
        nothing (scratch in the library's static device array; at most 65,536
        curves; overlapping calls on one device race)."""
        assert self._curves is not None
        n = self._curves.n_curves
        idx = np.empty(n, dtype=np.int64)
        val, mean, std = (np.empty(n, dtype=np.float64) for _ in range(3))
        _check(self._lib.bls_launch_best_noalloc(self._h, idx.ctypes.data, val.ctypes.data,
                                                 mean.ctypes.data, std.ctypes.data, stream))
        return idx, val, mean, std

    def device_output(self) -> int:
        ptr = _vp()
        _check(self._lib.bls_device_output(self._h, ctypes.byref(ptr)))
        return int(ptr.value or 0)

    def info(self) -> dict:
        info = BlsBatchInfo()
        _check(self._lib.bls_batch_info(self._h, ctypes.byref(info)))
        return info.as_dict()

    def search(self, grid: PackedGrid, curves: PackedCurves, stream: int | None = None) -> np.ndarray:
        self.prepare(grid, curves, stream)
        self.launch(stream)
        return self.download(stream)

    def search_joint(self, grid: PackedGrid, bands: PackedCurves,
                     stream: int | None = None) -> np.ndarray:
        """The joint-ephemeris search of one star whose bands are ``bands``:
        ``(len(JOINT_FIELD_NAMES), n_periods)`` in grid order."""
        out = np.empty((len(JOINT_FIELD_NAMES), grid.n_periods), dtype=np.float64)
        g, c = grid.struct(), bands.struct()
        _check(self._lib.bls_search_joint(self._h, ctypes.byref(g), ctypes.byref(c),
                                          out.ctypes.data, stream))
        return out

    def tls_prepare(self, curves, periods, *, n_bins: int, dur_bins, templates,
                    den_rel: float, stream: int | None = None) -> None:
        """Upload curves ``[(tau, yw, w, w_total), ...]`` and ``periods`` for the
        TLS matched filter (``bls_tls_prepare``)."""
        taus = [_f64(c[0]).ravel() for c in curves]
        off = np.zeros(len(curves) + 1, dtype=np.int64)
        off[1:] = np.cumsum([x.size for x in taus])
        cat = lambda xs: _f64(np.concatenate(xs)) if xs else np.empty(0)
        tau = cat(taus)
        yw = cat([_f64(c[1]).ravel() for c in curves])
        w = cat([_f64(c[2]).ravel() for c in curves])
        if yw.size != tau.size or w.size != tau.size:
            raise ValueError("tau, yw and w must have the same length")
        w_total = _f64([float(c[3]) for c in curves])
        db = np.ascontiguousarray(dur_bins, dtype=np.int32)
        tmpl = _f64(np.concatenate([np.asarray(templates[int(d)], dtype=np.float64)
                                    for d in db])) if db.size else np.empty(0)
        per = _f64(periods).ravel()
        inp = BlsTlsInputs(len(curves), _addr(off), _addr(tau), _addr(yw), _addr(w),
                           _addr(w_total), int(n_bins), int(db.size), _addr(db), _addr(tmpl),
                           float(den_rel))
        _check(self._lib.bls_tls_prepare(self._h, ctypes.byref(inp), _addr(per), per.size,
                                         stream))
        self._tls_shape = (len(curves), per.size)

    def tls_launch(self, stream: int | None = None) -> None:
        _check(self._lib.bls_tls_launch(self._h, stream))

    def tls_download(self, stream: int | None = None) -> np.ndarray:
        """``(4, n_curves, n_periods)`` (``TLS_FIELD_NAMES``)."""
        out = np.empty((len(TLS_FIELD_NAMES),) + self._tls_shape, dtype=np.float64)
        _check(self._lib.bls_tls_download(self._h, out.ctypes.data, stream))
        return out

    def tls_search(self, curves, periods, *, n_bins: int, dur_bins, templates,
                   den_rel: float, stream: int | None = None) -> np.ndarray:
        """The TLS matched filter of curves ``[(tau, yw, w, w_total), ...]`` over
        ``periods``: ``(4, n_curves, n_periods)`` (``TLS_FIELD_NAMES``)."""
        self.tls_prepare(curves, periods, n_bins=n_bins, dur_bins=dur_bins,
                         templates=templates, den_rel=den_rel, stream=stream)
        self.tls_launch(stream)
        return self.tls_download(stream)

    def joint_prepare(self, grid: PackedGrid, bands: PackedCurves,
                      stream: int | None = None) -> None:
        g, c = grid.struct(), bands.struct()
        _check(self._lib.bls_joint_prepare(self._h, ctypes.byref(g), ctypes.byref(c), stream))
        self._joint_periods = grid.n_periods

    def joint_launch(self, stream: int | None = None) -> None:
        _check(self._lib.bls_joint_launch(self._h, stream))

    def joint_download(self, stream: int | None = None) -> np.ndarray:
        out = np.empty((len(JOINT_FIELD_NAMES), self._joint_periods), dtype=np.float64)
        _check(self._lib.bls_joint_download(self._h, out.ctypes.data, stream))
        return out

    def prefix_sums(self, t, y, dy, period: float, durations, oversample: int):
        """Debug view: the device's padded cumulative sums of y*ivar and ivar over
        the phase bins of one period (reference units)."""
        t, y = _f64(t).ravel(), _f64(y).ravel()
        dy = None if dy is None else _f64(dy).ravel()
        durations = _f64(durations).ravel()
        width = int(np.ceil(period / (durations.min() / oversample))) + oversample + 1
        yw = np.empty(width + 1, dtype=np.float64)
        iv = np.empty(width + 1, dtype=np.float64)
        nb = ctypes.c_int32()
        _check(self._lib.bls_debug_prefix(self._h, t.ctypes.data, y.ctypes.data, _addr(dy),
                                          t.size, float(period), durations.ctypes.data,
                                          durations.size, int(oversample), yw.ctypes.data,
                                          iv.ctypes.data, ctypes.byref(nb)))
        return yw[:nb.value + 1], iv[:nb.value + 1]

    def fold_bins(self, t, period: float, bin_duration: float, width: int):
        """Debug view: the device's phase bin of every point at one period."""
        t = _f64(t).ravel()
        bins = np.empty(t.size, dtype=np.int32)
        fast = np.empty(t.size, dtype=np.int32)
        _check(self._lib.bls_debug_fold_bins(self._h, t.ctypes.data, t.size, float(period),
                                             float(bin_duration), int(width), bins.ctypes.data,
                                             fast.ctypes.data))
        return bins, fast.astype(bool)


_local = threading.local()


def default_engine() -> Engine:
    """This thread's engine on the current CUDA device (created on first use)."""
    eng = getattr(_local, "engine", None)
    if eng is None:
        eng = Engine()
        _local.engine = eng
    return eng
