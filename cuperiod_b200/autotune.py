"""Tile-shape autotuner of the BLS search (no counterpart in the reference, whose
CUDA kernel runs one 128-thread block per trial period, cuPeriod
src/cuperiod/methods/_bls_core.py:505-656).

The persistent search kernel has two shape knobs (``BlsTune``): the dynamic
shared memory per CTA, which sets how many CTAs stay resident on an SM and how
many consecutive trial periods of a segment one work item folds at once (each
period needs its own histogram), and a cap on those periods per work item.
Larger items re-read a curve's points fewer times; more resident CTAs hide more
latency and balance the tail of a launch better.  Which wins depends on the
curves' lengths, the segments' histogram widths and the device, so ``autotune``
times every candidate shape on a sample of the batch -- curves picked evenly
across the batch's point-count order, the full grid -- with CUDA events on the
launching stream (``bls_time_launches``) and keeps the fastest.  A choice is
cached per device and workload shape (``workload_key``), in memory and, when
``cache`` names a file, in that JSON file.

Every shape gives the same results: the one-weight and narrow-weight sums are
exact integers and the winner of a period is chosen in the reference's
first-wins order whatever the tile, so a tuned engine's output equals the
default engine's bit for bit (per-point FP64 sums round in atomic order and may
differ in the last bits, as they may between any two launches).
"""

from __future__ import annotations

import json
import os
import threading
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import _lib
from .errors import BackendUnavailableError

KIB = 1024


@dataclass(frozen=True)
class TileShape:
    """``BlsTune`` shape knobs: 0 means the engine's default."""
    smem_per_cta: int = 0       # dynamic shared memory per CTA (bytes)
    max_tile: int = 0           # trial periods per work item (1..16)

    def engine_kwargs(self) -> dict:
        return {"smem_per_cta": self.smem_per_cta, "max_tile": self.max_tile}

    def label(self) -> str:
        smem = "default" if self.smem_per_cta == 0 else f"{self.smem_per_cta // KIB}K"
        tile = "fit" if self.max_tile == 0 else str(self.max_tile)
        return f"smem={smem},tile={tile}"


# The engine's defaults first (72 KB and three CTAs per SM for one weight per
# curve, 108 KB and two for per-point weights), then capped tiles at the default
# occupancy, then fewer resident CTAs with larger tiles.
CANDIDATES: tuple[TileShape, ...] = (
    TileShape(0, 0), TileShape(0, 8), TileShape(0, 4), TileShape(0, 2),
    TileShape(108 * KIB, 0), TileShape(152 * KIB, 0), TileShape(200 * KIB, 0),
)


@dataclass
class TuneResult:
    """The fastest shape and what every candidate measured."""
    shape: TileShape
    key: str
    sample_curves: int
    ms: dict[str, float] = field(default_factory=dict)      # label -> ms per sample launch
    errors: dict[str, str] = field(default_factory=dict)    # label -> why it could not run
    cached: bool = False

    def speedup_over_default(self) -> float | None:
        base = self.ms.get(TileShape().label())
        best = self.ms.get(self.shape.label())
        return base / best if base and best else None

    def as_dict(self) -> dict:
        return {"shape": self.shape.label(), "smem_per_cta": self.shape.smem_per_cta,
                "max_tile": self.shape.max_tile, "key": self.key,
                "sample_curves": self.sample_curves, "ms": dict(self.ms),
                "errors": dict(self.errors), "cached": self.cached}


def sample_indices(n_points: np.ndarray, n: int) -> np.ndarray:
    """``n`` curve indices spread evenly over the batch's point-count order
    (smallest, ..., largest), so the sample has the batch's length mix."""
    n_points = np.asarray(n_points)
    if n >= n_points.size:
        return np.arange(n_points.size)
    order = np.argsort(n_points, kind="stable")
    picks = np.round(np.linspace(0, n_points.size - 1, n)).astype(np.int64)
    return np.sort(order[np.unique(picks)])


def subset(curves: _lib.PackedCurves, idx: Sequence[int]) -> _lib.PackedCurves:
    """The curves ``idx`` of a packed batch, packed on their own."""
    off = curves.offsets
    parts = []
    for i in idx:
        a, b = int(off[i]), int(off[i + 1])
        parts.append((curves.t[a:b], curves.y[a:b],
                      None if curves.dy is None else curves.dy[a:b]))
    return _lib.PackedCurves.from_arrays(parts)


def _bucket(x: float) -> int:
    """Power-of-two bucket of a positive size (0 for 0)."""
    return 0 if x <= 0 else int(round(np.log2(x)))


def workload_key(grid: _lib.PackedGrid, curves: _lib.PackedCurves, device: str) -> str:
    """What a tuned shape depends on: the device, the grid's size, segments,
    widest duration and objective, the weighting (one weight or per-point) and
    the curves' typical length and count, bucketed by powers of two."""
    n_pts = np.diff(curves.offsets)
    seg_p = np.diff(grid.seg_offsets)
    med = float(np.median(n_pts)) if n_pts.size else 0.0
    per_point = curves.dy is not None and curves.dy.size > 0 and \
        bool(np.any(curves.dy != curves.dy[0]))
    return (f"{device}|P{_bucket(grid.n_periods)}|S{seg_p.size}"
            f"|Pmax{float(grid.periods.max()) if grid.periods.size else 0.0:.3g}"
            f"|o{grid.oversample}|obj{grid.objective}|N{_bucket(med)}"
            f"|C{_bucket(curves.n_curves)}|{'dy' if per_point else 'w1'}")


_memory: dict[str, TuneResult] = {}
_lock = threading.Lock()


def _device_name(device: int) -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(device if device >= 0 else None)
    except Exception:  # pragma: no cover - torch is plumbing only
        pass
    return "cuda"


def _load_cache(path: str | os.PathLike | None) -> dict:
    if path is None or not os.path.exists(path):
        return {}
    try:
        with open(path, encoding="utf-8") as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def _store_cache(path: str | os.PathLike, key: str, res: TuneResult) -> None:
    data = _load_cache(path)
    data[key] = res.as_dict()
    tmp = f"{path}.{os.getpid()}.{threading.get_ident()}.tmp"
    with open(tmp, "w", encoding="utf-8") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _timer_for(device: int, reps: int) -> Callable[[TileShape, _lib.PackedGrid,
                                                     _lib.PackedCurves], float]:
    def time_shape(shape, grid, sample):
        eng = _lib.Engine(device, use_graph=False, **shape.engine_kwargs())
        try:
            eng.prepare(grid, sample)
            eng.time_launches(1)                  # warm-up: module load, caches
            return eng.time_launches(reps)
        finally:
            eng.close()
    return time_shape


def autotune(grid: _lib.PackedGrid, curves: _lib.PackedCurves, *,
             candidates: Sequence[TileShape] = CANDIDATES, sample: int = 128, reps: int = 1,
             device: int = -1, cache: str | os.PathLike | None = None, refresh: bool = False,
             timer: Callable[[TileShape, _lib.PackedGrid, _lib.PackedCurves], float] | None = None
             ) -> TuneResult:
    """The fastest candidate shape for searching ``curves`` over ``grid``.

    ``sample`` curves (spread over the batch's length order) are searched once
    per candidate after a warm-up launch; ``reps`` timed launches each.  A shape
    the device cannot run (a segment too wide for its shared memory) is
    recorded in ``errors`` and skipped.  ``timer`` replaces the device clock
    (tests): ``timer(shape, grid, sample) -> ms``.
    """
    if not candidates:
        raise ValueError("autotune needs at least one candidate shape")
    key = workload_key(grid, curves, _device_name(device))
    if not refresh:
        with _lock:
            hit = _memory.get(key)
        if hit is None and cache is not None:
            row = _load_cache(cache).get(key)
            if isinstance(row, dict) and "smem_per_cta" in row and "max_tile" in row:
                hit = TuneResult(TileShape(int(row["smem_per_cta"]), int(row["max_tile"])), key,
                                 int(row.get("sample_curves", 0)),
                                 {str(k): float(v) for k, v in row.get("ms", {}).items()},
                                 {str(k): str(v) for k, v in row.get("errors", {}).items()})
        if hit is not None:
            return TuneResult(hit.shape, key, hit.sample_curves, dict(hit.ms), dict(hit.errors),
                              cached=True)
    idx = sample_indices(np.diff(curves.offsets), sample)
    sub = subset(curves, idx)
    time_shape = timer or _timer_for(device, reps)
    ms: dict[str, float] = {}
    errors: dict[str, str] = {}
    best: TileShape | None = None
    for shape in dict.fromkeys(candidates):        # in order, without repeats
        try:
            t = float(time_shape(shape, grid, sub))
        except (BackendUnavailableError, ValueError) as exc:
            errors[shape.label()] = f"{type(exc).__name__}: {exc}"
            continue
        ms[shape.label()] = t
        if best is None or t < ms[best.label()]:
            best = shape
    if best is None:
        raise BackendUnavailableError(
            "autotune: no candidate shape can run this grid: " + "; ".join(errors.values()))
    res = TuneResult(best, key, int(idx.size), ms, errors)
    with _lock:
        _memory[key] = res
    if cache is not None:
        _store_cache(cache, key, res)
    return res


def tuned_engine(grid: _lib.PackedGrid, curves: _lib.PackedCurves, *, device: int = -1,
                 use_graph: bool = True, **kwargs) -> tuple[_lib.Engine, TuneResult]:
    """An engine built with the autotuned shape for this batch, and the result."""
    res = autotune(grid, curves, device=device, **kwargs)
    return _lib.Engine(device, use_graph=use_graph, **res.shape.engine_kwargs()), res


__all__ = ["CANDIDATES", "TileShape", "TuneResult", "autotune", "sample_indices", "subset",
           "tuned_engine", "workload_key"]
