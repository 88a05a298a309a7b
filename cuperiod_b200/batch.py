"""Batch entry point: ``batch_periodograms`` (cuPeriod
src/cuperiod/batch/runner.py:764-1032) with the per-curve loop replaced by one
engine launch per chunk of light curves that share a grid, and the result row
of ``periodogram_to_row`` (src/cuperiod/batch/io.py:507-571)."""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Any, Iterable, Sequence

import numpy as np

from . import _lib
from .api import _settings, to_input
from .bls import get_method
from .errors import CuPeriodError
from .grid import GridSpec
from .lightcurve import Domain, MultiBandLightCurve
from .result import Periodogram

#: Per-peak extras of a BLS row (io.py:66-70).
PEAK_EXTRA_COLUMNS = ("depth", "depth_snr", "duration", "t0", "sde")


def periodogram_to_row(key: str, pg: Periodogram, *, n_best: int = 10,
                       extra_keys: Sequence[str] | None = None, alias_diverse: bool = True,
                       source: str | None = None) -> dict:
    """One result row: key, method, backend, n_samples, baseline, best_period and
    ``period_k``/``power_k`` for k = 1..n_best; each declared extra as
    ``{extra}_k`` for every rank (NaN past the last peak), other extras for the
    ranks that have them (io.py:507-571)."""
    row: dict[str, Any] = {"key": key, "method": pg.method}
    if source is not None:
        row["source"] = source
    row["backend"] = pg.backend
    row["n_samples"] = pg.n_samples
    row["baseline"] = pg.baseline
    peaks = pg.best_periods(max(int(n_best), 1), alias_diverse=alias_diverse)
    row["best_period"] = peaks[0].period if peaks else float("nan")
    for rank in range(1, n_best + 1):
        peak = peaks[rank - 1] if rank <= len(peaks) else None
        row[f"period_{rank}"] = peak.period if peak else float("nan")
        row[f"power_{rank}"] = peak.power if peak else float("nan")
        extra = peak.extra if peak is not None else {}
        declared = tuple(extra_keys) if extra_keys is not None else ()
        for ekey in declared:
            v = extra.get(ekey)
            row[f"{ekey}_{rank}"] = float("nan") if v is None else float(v)
        for ekey, v in extra.items():
            if ekey not in declared:
                row[f"{ekey}_{rank}"] = v
    return row


@dataclass
class BatchSummary:
    """What a batch did (runner.py:151-184): rows written and per-curve errors."""

    rows: list[dict] = field(default_factory=list)
    errors: dict[str, str] = field(default_factory=dict)
    launches: int = 0

    @property
    def n_ok(self) -> int:
        return len(self.rows)

    @property
    def n_failed(self) -> int:
        return len(self.errors)


def _grid_key(grid: GridSpec) -> str:
    h = hashlib.sha1(np.ascontiguousarray(grid.period).tobytes())
    h.update(repr(sorted(grid.meta.items())).encode())
    return h.hexdigest()


def batch_periodograms(inputs: Iterable[tuple[str, Any]], method: str = "BLS", *,
                       grid: GridSpec | None = None, settings: Any = None,
                       domain: Domain | str | None = None, n_best: int = 10,
                       chunk_size: int = 4096, sink: str | None = None,
                       engine: _lib.Engine | None = None) -> BatchSummary:
    """Search many light curves; one engine launch per chunk of curves that share
    a trial grid (the explicit ``grid``, or curves whose default grids coincide).

    ``inputs`` yields ``(key, data)`` with ``data`` a LightCurve or a
    ``(t, y[, dy])`` tuple.  A curve that cannot be searched (too few points,
    no baseline) is recorded in ``errors`` like the reference's per-curve
    failures (runner.py:248-249).  ``sink``: optional Parquet path for the rows.
    """
    m = get_method(method)
    s = _settings(settings)
    eng = engine or _lib.default_engine()
    summary = BatchSummary()
    groups: dict[str, tuple[GridSpec, list[tuple[str, Any]]]] = {}
    fixed_key = _grid_key(grid) if grid is not None else None     # one grid: hash it once
    for key, data in inputs:
        try:
            lc = to_input(data, domain=domain)
            if isinstance(lc, MultiBandLightCurve):
                # one star's bands: one launch of its own, peaks ranked on the host
                from .multiband import multiband_default_grid
                pg = m.multiband_power(grid or multiband_default_grid(m, lc, s), lc, s,
                                       engine=eng)
                summary.rows.append(periodogram_to_row(str(key), pg.with_peak_defaults(s),
                                                       n_best=n_best,
                                                       extra_keys=PEAK_EXTRA_COLUMNS,
                                                       alias_diverse=True))
                summary.launches += 1
                continue
            lc = lc.in_domain(m.natural_domain)
            g = grid or m.default_grid(lc, s)
        except (CuPeriodError, ValueError) as exc:
            summary.errors[str(key)] = f"{type(exc).__name__}: {exc}"
            continue
        gk = fixed_key if fixed_key is not None else _grid_key(g)
        groups.setdefault(gk, (g, []))[1].append((str(key), lc))
    for g, members in groups.values():
        for start in range(0, len(members), chunk_size):
            chunk = members[start:start + chunk_size]
            ok: list[tuple[str, Any]] = []
            for key, lc in chunk:
                finite = lc.finite()
                if finite.n < s.min_detections or finite.baseline <= 0.0:
                    summary.errors[key] = (f"InsufficientDataError: BLS: {finite.n} finite "
                                           f"points < min_detections {s.min_detections}"
                                           if finite.n < s.min_detections
                                           else "InsufficientDataError: BLS: no usable time baseline")
                    continue
                ok.append((key, lc))
            if not ok:
                continue
            # peaks ranked on the device: only the rows leave the GPU
            summary.rows.extend(m.rows_many(g, ok, s, n_best=n_best,
                                            extra_keys=PEAK_EXTRA_COLUMNS, engine=eng))
            summary.launches += 1
    if sink is not None and summary.rows:
        import pyarrow as pa
        import pyarrow.parquet as pq
        pq.write_table(pa.Table.from_pylist(summary.rows), sink)
    return summary


__all__ = ["BatchSummary", "PEAK_EXTRA_COLUMNS", "batch_periodograms", "periodogram_to_row"]
