"""Kernel-level BLS entry points: ``bls_power`` and ``bls_power_segments``.

Drop-ins for cuPeriod's ``bls_power`` / ``bls_power_segments``
(src/cuperiod/methods/_bls_core.py:882-1028, 1075-1130) with the same arguments,
the same :class:`BLSPower` result and the same grid semantics (one
``_search_spec`` per segment: bin = shortest duration / oversample, durations
rounded half away from zero to bins and deduplicated in first-seen order, width
= ceil(max period / bin) + oversample + 1).  The search itself runs on the B200
engine (``libbls_b200.so``); there is no CPU path.
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Final

import numpy as np

from . import _lib

#: Accepted for signature compatibility with the reference (its array-API batch
#: size); the engine tiles the period grid itself.
DEFAULT_BATCH: Final = 2048

#: Backend names this engine answers to.  ``"b200"`` is its own name; the
#: reference's GPU backend name ``"cupy"`` and the generic ``"gpu"`` / ``"auto"``
#: resolve to it too, so callers written for the reference keep working.
BACKENDS: Final = ("b200", "cupy", "gpu", "auto", "cuda")

_F64_EPS: Final = float(np.finfo(np.float64).eps)


@dataclass(frozen=True, slots=True)
class BLSPower:
    """Per-period BLS maxima, aligned with the input ``periods`` order.

    The fields of the reference's ``BLSPower`` (``_bls_core.py:113-131``): ``power``
    is the objective (``depth_snr`` for ``"snr"``, ``log_likelihood`` for
    ``"likelihood"``); ``transit_time`` is in ``[t_min, t_min + period)``.  A period
    with no admissible box has ``power = -inf`` and zeros elsewhere.
    """

    period: np.ndarray
    power: np.ndarray
    depth: np.ndarray
    depth_err: np.ndarray
    depth_snr: np.ndarray
    duration: np.ndarray
    transit_time: np.ndarray
    log_likelihood: np.ndarray


def _ivar_floor(n_points: int, sum_ivar: float) -> float:
    """The relative admissibility floor of a box side (``_bls_core.py:75-94``)."""
    floor = 4.0 * n_points * _F64_EPS * sum_ivar
    if not floor > 0.0:
        return float(np.finfo(np.float64).tiny)
    return floor


def _duration_bins(durations, bin_duration: float) -> list[int]:
    """Box widths in bins, rounded half away from zero, deduplicated in order
    (``_bls_core.py:134-149``)."""
    seen: set[int] = set()
    out: list[int] = []
    for d in np.asarray(durations, dtype=np.float64).tolist():
        kd = math.floor(d / bin_duration + 0.5)
        if kd >= 1 and kd not in seen:
            seen.add(kd)
            out.append(kd)
    return out


def _objective_flag(objective: str) -> int:
    """0 = depth signal-to-noise, 1 = log-likelihood (``_bls_core.py:1031-1035``)."""
    if objective not in ("snr", "likelihood"):
        raise ValueError("objective must be 'snr' or 'likelihood'")
    return 0 if objective == "snr" else 1


def _check_backend(backend: str) -> None:
    if str(backend).lower() not in BACKENDS:
        raise ValueError(f"unknown backend {backend!r}; this engine runs {BACKENDS}")


def _empty_power() -> BLSPower:
    return BLSPower(*(np.empty(0, dtype=np.float64) for _ in range(8)))


def _to_power(periods: np.ndarray, fields: np.ndarray) -> BLSPower:
    """Rows of a (7, P) engine output as a :class:`BLSPower`."""
    return BLSPower(periods, *(np.ascontiguousarray(fields[i]) for i in range(_lib.N_FIELDS)))


def bls_power(
    t, y, dy, periods, durations, oversample: int, *,
    objective: str = "snr", backend: str = "b200", batch: int = DEFAULT_BATCH,
    precision: str = "auto", device_cache: dict[str, Any] | None = None,
    engine: _lib.Engine | None = None,
) -> BLSPower:
    """BLS box search of one light curve over ``periods`` on the B200 engine.

    Same contract as the reference's ``bls_power``: ``y`` in the dip convention,
    ``dy`` 1-sigma errors (``ivar = 1/dy**2``), ``durations`` absolute, ``oversample``
    phase bins per shortest duration.  ``batch``, ``precision`` and
    ``device_cache`` are accepted for compatibility and do not change the result
    (the engine's arithmetic is fixed: FP64 phase and bin index, exact integer
    bin sums, FP64 box statistics).
    """
    del batch, precision, device_cache
    obj_flag = _objective_flag(objective)
    _check_backend(backend)
    periods_host = np.ascontiguousarray(periods, dtype=np.float64)
    if periods_host.size == 0:
        return _empty_power()
    return bls_power_segments(t, y, dy, [(periods_host, durations)], oversample,
                              objective=objective, backend=backend, engine=engine,
                              _obj_flag=obj_flag)[0]


def bls_power_segments(
    t, y, dy, segments, oversample: int, *,
    objective: str = "snr", backend: str = "b200", batch: int = DEFAULT_BATCH,
    precision: str = "auto", device_cache: dict[str, Any] | None = None,
    engine: _lib.Engine | None = None, _obj_flag: int | None = None,
) -> list[BLSPower]:
    """:func:`bls_power` over the ``(periods, durations)`` segments of one curve in
    one upload, one launch and one download (``_bls_core.py:1075-1130``).

    Equal to calling :func:`bls_power` once per segment; an empty segment comes
    back empty, in its place.
    """
    del batch, precision, device_cache
    obj_flag = _objective_flag(objective) if _obj_flag is None else _obj_flag
    _check_backend(backend)
    segs = [(np.ascontiguousarray(p, dtype=np.float64).ravel(),
             np.ascontiguousarray(d, dtype=np.float64).ravel()) for p, d in segments]
    live = [(p, d) for p, d in segs if p.size]
    results: list[BLSPower] = []
    if live:
        grid = _lib.PackedGrid.from_segments(live, oversample, obj_flag)
        curves = _lib.PackedCurves.from_arrays([(t, y, dy)])
        eng = engine or _lib.default_engine()
        out = eng.search(grid, curves)[:, 0, :]
    off = 0
    for p, _ in segs:
        if p.size == 0:
            results.append(_empty_power())
            continue
        results.append(_to_power(p, out[:, off:off + p.size]))
        off += p.size
    return results


def bls_power_many(
    curves, segments, oversample: int, *, objective: str = "snr",
    engine: _lib.Engine | None = None,
) -> np.ndarray:
    """Many light curves over one segmented grid in one launch.

    ``curves`` is a sequence of ``(t, y, dy)`` (``dy`` may be ``None`` for unit
    errors); returns the (7, n_curves, n_periods) field array in grid order
    (segments concatenated), field order as :class:`BLSPower` without ``period``.
    """
    obj_flag = _objective_flag(objective)
    segs = [(np.ascontiguousarray(p, dtype=np.float64).ravel(),
             np.ascontiguousarray(d, dtype=np.float64).ravel()) for p, d in segments]
    grid = _lib.PackedGrid.from_segments(segs, oversample, obj_flag)
    packed = _lib.PackedCurves.from_arrays(list(curves))
    eng = engine or _lib.default_engine()
    return eng.search(grid, packed)


__all__ = ["BLSPower", "DEFAULT_BATCH", "bls_power", "bls_power_many", "bls_power_segments"]
