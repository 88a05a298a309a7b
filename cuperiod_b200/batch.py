"""Batch entry point: ``batch_periodograms`` (cuPeriod
src/cuperiod/batch/runner.py:764-1032) with the per-curve loop replaced by one
engine launch per chunk of light curves that share a grid, and the result row
of ``periodogram_to_row`` (src/cuperiod/batch/io.py:507-571)."""

from __future__ import annotations

import hashlib
import os
import threading
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
#: Per-peak extras of each method's rows, in column order (batch/io.py:66-70).
METHOD_PEAK_EXTRAS = {"BLS": PEAK_EXTRA_COLUMNS, "TLS": ("sr", "depth", "duration", "t0")}


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


_pools: dict[int, Any] = {}
_pools_lock = threading.Lock()


def _worker_pool(n: int):
    """The process's pool of ``n`` batch worker threads, created once: each
    thread keeps its engine (``_lib.default_engine``: device buffers, pinned
    staging, graph cache) from one call to the next, so a batch does not pay
    for creating engines.  Jobs of concurrent calls share the threads; each job
    runs on one thread and its engine."""
    with _pools_lock:
        pool = _pools.get(n)
        if pool is None:
            from concurrent.futures import ThreadPoolExecutor
            pool = ThreadPoolExecutor(max_workers=n, thread_name_prefix=f"bls-batch-{n}")
            _pools[n] = pool
        return pool


def release_workers() -> None:
    """Shut the batch worker pools down: their threads exit, and with them each
    thread's engine (device buffers, pinned staging) is freed.  A later call
    with ``workers > 1`` starts a new pool."""
    with _pools_lock:
        pools = list(_pools.values())
        _pools.clear()
    for pool in pools:
        pool.shutdown(wait=True)


def _grid_key(grid: GridSpec) -> str:
    h = hashlib.sha1(np.ascontiguousarray(grid.period).tobytes())
    h.update(repr(sorted(grid.meta.items())).encode())
    return h.hexdigest()


_TABLE_SUFFIXES = (".csv", ".ecsv", ".tsv", ".tab", ".dat", ".txt", ".parquet", ".pq")


def _unique_keys(items: list[tuple[str, Any]]) -> list[tuple[str, Any]]:
    """Repeated keys keep the first and get #2, #3, ... (io.py:147-193)."""
    seen: dict[str, int] = {}
    out = []
    for key, src in items:
        k = str(key)
        n = seen.get(k, 0) + 1
        seen[k] = n
        out.append((k if n == 1 else f"{k}#{n}", src))
    return out


def resolve_inputs(inputs: Any, *, columns: Any = None, domain: Any = None,
                   band_column: str | None = None) -> list[tuple[str, Any]]:
    """``(key, source)`` pairs from ``(key, data)`` pairs, light curves, a
    ``(DataFrame, group_column)`` tuple, or files (a path, a directory or a glob),
    keyed by file stem (io.py:147-224)."""
    import glob
    import os
    from pathlib import Path

    from .lightcurve import LightCurve as _LC
    if isinstance(inputs, tuple) and len(inputs) == 2 and hasattr(inputs[0], "groupby"):
        df, group_col = inputs
        multiband = band_column is not None or (columns is not None and
                                                getattr(columns, "band", None) is not None)
        items = []
        for key, sub in df.groupby(group_col, sort=False):
            lc = (MultiBandLightCurve.from_dataframe(sub, band_column=band_column,
                                                     columns=columns, domain=domain)
                  if multiband else _LC.from_dataframe(sub, columns=columns, domain=domain))
            items.append((str(key), lc))
        return _unique_keys(items)
    if isinstance(inputs, (str, os.PathLike)):
        p = Path(inputs)
        if p.is_dir():
            paths = sorted(q for q in p.iterdir() if q.is_file() and any(
                str(q).lower().endswith(sfx) or str(q).lower().endswith(sfx + z)
                for sfx in _TABLE_SUFFIXES for z in ("", ".gz", ".bz2", ".xz")))
        elif p.exists():
            paths = [p]
        else:
            paths = sorted(Path(x) for x in glob.glob(str(inputs)))
            if not paths:
                raise FileNotFoundError(f"no light-curve files match {str(inputs)!r}")
        return _unique_keys([(q.name.split(".")[0], q) for q in paths])
    items = []
    for i, entry in enumerate(inputs):
        if isinstance(entry, tuple) and len(entry) == 2 and isinstance(entry[0], (str, int)):
            items.append((str(entry[0]), entry[1]))
        elif isinstance(entry, (str, os.PathLike)):
            items.append((Path(entry).name.split(".")[0], Path(entry)))
        else:
            meta = getattr(entry, "meta", {}) or {}
            items.append((str(meta.get("id", i)), entry))
    return _unique_keys(items)


def _load(src: Any, columns: Any, domain: Any, band_column: str | None) -> Any:
    """A path's light curve (split on a band column when one is named)."""
    import os

    from .lightcurve import LightCurve as _LC
    if isinstance(src, (str, os.PathLike)):
        if band_column is not None or (columns is not None and
                                       getattr(columns, "band", None) is not None):
            return MultiBandLightCurve.from_file(src, band_column=band_column, columns=columns,
                                                 domain=domain)
        return _LC.from_file(src, columns=columns, domain=domain)
    return src


def batch_periodograms(inputs: Any, method: str = "BLS", *,
                       grid: GridSpec | None = None, settings: Any = None,
                       columns: Any = None, domain: Domain | str | None = None,
                       band_column: str | None = None, n_best: int = 10,
                       chunk_size: int = 4096, sink: str | os.PathLike | None = None,
                       engine: _lib.Engine | None = None,
                       workers: int | None = None) -> BatchSummary:
    """Search many light curves: BLS searches each chunk of ``chunk_size`` curves
    in one engine launch, every curve over its own grid (the explicit ``grid``,
    else its default grid, which the engine library builds on the host cores);
    other methods launch once per chunk of curves that share a grid.  Multi-band stars are launches of their
    own; their rows come first, then the curves' rows in input order.

    ``inputs``: ``(key, data)`` pairs (``data`` a LightCurve, MultiBandLightCurve,
    ``(t, y[, dy])`` tuple or table), light curves, files (a path, a directory, a
    glob) or a ``(DataFrame, group_column)`` tuple (``resolve_inputs``).  A curve
    that cannot be searched (too few points, no baseline, unreadable) is recorded
    in ``errors`` like the reference's per-curve failures (runner.py:248-249).
    ``sink``: optional ``.parquet`` or ``.csv`` path for the rows (``write_rows``).
    ``workers``: host threads that run the launches (default 4; each thread its
    own engine and CUDA stream, so the small launches of curves with distinct
    default grids, and of multi-band stars, overlap each other and the host
    work; the threads and their engines persist from call to call); with an
    explicit ``engine`` every launch runs on that engine in this thread.  Rows
    keep the order of a single-threaded run.
    """
    m = get_method(method)
    s = _settings(settings, m.settings_cls)
    summary = BatchSummary()
    groups: dict[str, tuple[GridSpec, list[tuple[str, Any]]]] = {}
    entries: list[tuple[str, Any, str]] = []        # (key, curve, grid key) in input order
    star_jobs: list[tuple[str, Any, GridSpec]] = []
    fixed_key = _grid_key(grid) if grid is not None else None     # one grid: hash it once
    # BLS default grids are built by the engine library at launch time
    native_default = grid is None and hasattr(m, "rows_default")
    for key, data in resolve_inputs(inputs, columns=columns, domain=domain,
                                    band_column=band_column):
        try:
            data = _load(data, columns, domain, band_column)
            lc = to_input(data, columns=columns, domain=domain)
            if isinstance(lc, MultiBandLightCurve):
                if not m.supports_multiband:
                    raise ValueError(f"{m.name} does not support multi-band input")
                # one star's bands: a launch of its own, peaks ranked on the host
                from .multiband import multiband_default_grid
                star_jobs.append((str(key), lc, grid or multiband_default_grid(m, lc, s)))
                continue
            lc = lc.in_domain(m.natural_domain)
            if native_default:
                entries.append((str(key), lc, ""))
                continue
            g = grid or m.default_grid(lc, s)
        except (CuPeriodError, ValueError, OSError) as exc:
            summary.errors[str(key)] = f"{type(exc).__name__}: {exc}"
            continue
        gk = fixed_key if fixed_key is not None else _grid_key(g)
        groups.setdefault(gk, (g, []))[1].append((str(key), lc))
        entries.append((str(key), lc, gk))

    def searchable(key: str, lc: Any) -> Any:
        """The curve's finite points when they can be searched, else None (the
        failure recorded); the searches take these and do not filter again."""
        finite = lc.finite()
        if finite.n < s.min_detections or finite.baseline <= 0.0:
            summary.errors[key] = (f"InsufficientDataError: {m.name}: {finite.n} "
                                   f"finite points < min_detections {s.min_detections}"
                                   if finite.n < s.min_detections
                                   else f"InsufficientDataError: {m.name}: no usable "
                                        "time baseline")
            return None
        return finite

    jobs: list[Any] = [("star", job) for job in star_jobs]
    if native_default:
        # one launch per chunk of curves in input order, each over its default grid
        usable = ((key, searchable(key, lc)) for key, lc, _ in entries)
        ok_all, failed = m.split_default([(key, f) for key, f in usable if f is not None], s,
                                         prefiltered=True)
        summary.errors.update(failed)
        for start in range(0, len(ok_all), chunk_size):
            jobs.append(("default", ok_all[start:start + chunk_size]))
    elif hasattr(m, "rows_by_grid"):
        # one launch per chunk of curves in input order, each curve over its own
        # grid (equal grids shared)
        usable = ((key, searchable(key, lc), gk) for key, lc, gk in entries)
        ok_all = [(key, f, groups[gk][0]) for key, f, gk in usable if f is not None]
        for start in range(0, len(ok_all), chunk_size):
            jobs.append(("mixed", ok_all[start:start + chunk_size]))
    else:
        for g, members in groups.values():
            for start in range(0, len(members), chunk_size):
                usable = ((key, searchable(key, lc))
                          for key, lc in members[start:start + chunk_size])
                ok = [(key, f) for key, f in usable if f is not None]
                if ok:
                    jobs.append(("curves", (g, ok)))
    extras = METHOD_PEAK_EXTRAS.get(m.name, ())

    def run(job, job_engine):
        """``(rows, {key: error})`` of one job."""
        kind, body = job
        if kind == "star":
            key, star, g = body
            try:
                pg = m.multiband_power(g, star, s, engine=job_engine)
            except (CuPeriodError, ValueError) as exc:
                return [], {key: f"{type(exc).__name__}: {exc}"}
            return [periodogram_to_row(key, pg.with_peak_defaults(s), n_best=n_best,
                                       extra_keys=PEAK_EXTRA_COLUMNS, alias_diverse=True)], {}
        if kind == "default":
            return m.rows_default(body, s, n_best=n_best, extra_keys=extras,
                                  engine=job_engine, prefiltered=True), {}
        if kind == "mixed":
            # peaks ranked on the device: only the rows leave the GPU
            return m.rows_by_grid(body, s, n_best=n_best, extra_keys=extras,
                                  engine=job_engine, prefiltered=True), {}
        return run_curves(body, job_engine), {}

    def run_curves(body, job_engine):
        g, ok = body
        if hasattr(m, "rows_many"):
            # peaks ranked on the device: only the rows leave the GPU
            return m.rows_many(g, ok, s, n_best=n_best, extra_keys=extras, engine=job_engine)
        # one launch for the chunk, peaks ranked on the host
        pgs = m.power_many(g, [lc for _, lc in ok], s, engine=job_engine)
        return [periodogram_to_row(key, pg.with_peak_defaults(s), n_best=n_best,
                                   extra_keys=extras, alias_diverse=True)
                for (key, _), pg in zip(ok, pgs)]

    n_workers = 1 if engine is not None else max(1, int(workers if workers is not None else 4))
    # engine None: each launch runs on its thread's own engine (default_engine),
    # created at the thread's first launch and kept by the persistent pool
    if n_workers == 1 or len(jobs) <= 1:
        results = [run(job, engine) for job in jobs]
    else:
        results = list(_worker_pool(n_workers).map(lambda job: run(job, None), jobs))
    for rows, errors in results:
        summary.rows.extend(rows)
        summary.errors.update(errors)
        summary.launches += bool(rows)
    if sink is not None and summary.rows:
        from .sinks import write_rows
        write_rows(summary.rows, sink)
    return summary


__all__ = ["BatchSummary", "METHOD_PEAK_EXTRAS", "PEAK_EXTRA_COLUMNS", "batch_periodograms",
           "periodogram_to_row", "release_workers", "resolve_inputs"]
