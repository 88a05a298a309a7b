"""Streamed catalogue sweep: learned-pruned BLS over a catalogue held in pinned
host memory, chunk by chunk, with a full-grid audit.

No counterpart in the reference (its batch runner loops over curves,
src/cuperiod/batch/runner.py:214-250, in chunks of ``chunk_size``,
:326-331).  The catalogue is one packed pair of FP64 arrays (times, fluxes)
and offsets, pinned.  Two worker threads, each with its own engine, CUDA stream
and proposal network, take chunks in turn: while one packs and uploads its
chunk (host cores and the copy engine) the other's network and search run on
the GPU.  Per chunk: the network ranks each curve's log-period windows; curves
whose top-k probability mass reaches the calibrated threshold are searched
exactly over their windows, the others over the full grid (their full-grid
search is their audit); a seeded sample of ``audit_frac`` of the chunk's
confident curves is searched again over the full grid and compared.
"""

from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .proposal import Proposer, PrunedResult, Weights


@dataclass
class SweepResult:
    best_period: np.ndarray
    best_index: np.ndarray
    confident: np.ndarray
    audited: np.ndarray           # confident curves re-searched over the full grid
    audit_agree: np.ndarray       # for those: the same best period
    seconds: float
    chunks: list = field(default_factory=list)     # per chunk: timings and work

    @property
    def audit_agreement(self) -> float | None:
        n = int(self.audited.sum())
        return float(self.audit_agree[self.audited].mean()) if n else None


def pin(t: np.ndarray, y: np.ndarray):
    """The catalogue's arrays in pinned host memory (numpy views of pinned torch
    tensors), so chunk uploads are direct DMA."""
    import torch
    tp = torch.from_numpy(np.ascontiguousarray(t, dtype=np.float64)).pin_memory()
    yp = torch.from_numpy(np.ascontiguousarray(y, dtype=np.float64)).pin_memory()
    return tp.numpy(), yp.numpy(), (tp, yp)


def sweep(t: np.ndarray, y: np.ndarray, offsets: np.ndarray, weights: Weights, segments, *,
          chunk: int = 16384, workers: int = 2, audit_frac: float = 0.01, seed: int = 0,
          threshold: float | None = None, plain: bool = False) -> SweepResult:
    """Learned-pruned BLS of every curve of the packed catalogue (see the module
    docstring).  ``t``, ``y``: FP64 (ideally pinned, :func:`pin`); ``offsets``:
    int64, n_curves + 1.  ``plain=True`` searches every curve over the full grid
    (one launch per chunk, no network, no audit): the baseline of the sweep."""
    import torch
    n = int(offsets.size - 1)
    best_period = np.full(n, np.nan)
    best_index = np.full(n, -1, dtype=np.int64)
    confident = np.zeros(n, dtype=bool)
    audited = np.zeros(n, dtype=bool)
    audit_agree = np.zeros(n, dtype=bool)
    starts = list(range(0, n, chunk))
    lock = threading.Lock()
    next_chunk = [0]
    records: list = []
    errors: list = []

    def worker(wid: int) -> None:
        try:
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                engine = _lib.Engine()
                prop = Proposer(weights, segments, threshold=threshold, stream=stream)
                while True:
                    with lock:
                        if next_chunk[0] >= len(starts):
                            break
                        k = next_chunk[0]
                        next_chunk[0] += 1
                    a = starts[k]
                    b = min(a + chunk, n)
                    t0 = time.perf_counter()
                    o0, o1 = int(offsets[a]), int(offsets[b])
                    packed = _lib.PackedCurves(offsets[a:b + 1] - o0, t[o0:o1], y[o0:o1], None)
                    if plain:
                        engine.prepare(prop.full, packed)
                        engine.launch()
                        bi = engine.download_best()[0]
                        res = PrunedResult(prop.periods[bi], bi, None, np.zeros(b - a, bool),
                                           None, (b - a) * prop.full.n_periods)
                    else:
                        res = prop.search_packed(packed, engine)
                    t1 = time.perf_counter()
                    info = engine.info()
                    # the audit: a seeded sample of the confident curves, full grid
                    rng = np.random.default_rng((seed, k))
                    conf = np.flatnonzero(res.confident)
                    pick = conf[rng.random(conf.size) < audit_frac]
                    agree = np.zeros(pick.size, dtype=bool)
                    if pick.size:
                        engine.prepare(prop.full, _lib.PackedCurves.from_arrays(
                            [(t[offsets[a + i]:offsets[a + i + 1]],
                              y[offsets[a + i]:offsets[a + i + 1]], None) for i in pick]))
                        engine.launch()
                        full_best = engine.download_best()[0]
                        agree = full_best == res.best_index[pick]
                    t2 = time.perf_counter()
                    best_period[a:b] = res.best_period
                    best_index[a:b] = res.best_index
                    confident[a:b] = res.confident
                    audited[a + pick] = True
                    audit_agree[a + pick] = agree
                    with lock:
                        records.append({"chunk": k, "worker": wid, "curves": b - a,
                                        "search_s": t1 - t0, "audit_s": t2 - t1,
                                        "folds": info["folds"], "boxes": info["boxes"],
                                        "h2d_bytes": info["h2d_bytes"],
                                        "periods_searched": res.periods_searched})
                engine.close()
        except BaseException as exc:     # re-raised in the caller's thread
            errors.append(exc)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=worker, args=(w,)) for w in range(max(1, workers))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    seconds = time.perf_counter() - t0
    if errors:
        raise errors[0]
    records.sort(key=lambda r: r["chunk"])
    return SweepResult(best_period, best_index, confident, audited, audit_agree, seconds, records)


__all__ = ["SweepResult", "pin", "sweep"]
