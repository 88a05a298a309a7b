"""TEST INFRASTRUCTURE ONLY -- the CPU oracle of the BLS parity tests.

A restatement of cuPeriod's BLS path on the CPU: the host-side steps in numpy
(each function cites the reference file:line it follows) and the per-period box
search in plain C (``bls_oracle.c``, the numba kernel of
``src/cuperiod/methods/_bls_core.py:341-462``: without its screen as the parity
checker, with it as the timed CPU baseline).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
may import this module, and only as the reference results are compared with or as
the timed CPU baseline.  The
product package ``cuperiod_b200`` never imports it.

It is pinned against golden vectors produced by the reference's own numba
backend (``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_bls.so")
_lib: ctypes.CDLL | None = None

F64_EPS = float(np.finfo(np.float64).eps)
# The numba sweep's screen (_bls_core.py:67-72): slack in units of eps of
# sum|y*ivar|, and the range of sums inside which its normalisation is exact.
SCREEN_SLACK_EPS = 256.0
SCREEN_SCALE_RANGE = (1e-150, 1e150)
OUTPUT_NAMES = ("power", "depth", "depth_err", "depth_snr", "duration",
                "transit_time", "log_likelihood")
SEGMENT_FIELDS = ("period", "power", "depth", "depth_snr", "duration", "transit_time")


def build() -> str:
    """Compile the C oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        d, i64, i32 = ctypes.c_double, ctypes.c_int64, ctypes.c_int
        p = ctypes.c_void_p
        lib.bls_oracle_search.argtypes = [p, p, p, i64, p, i64, p, i64, d, i64, i64,
                                          d, d, d, i32, d, p, i32]
        lib.bls_oracle_search.restype = i32
        lib.bls_oracle_search_screened.argtypes = [p, p, p, i64, p, i64, p, i64, d, i64, i64,
                                                   d, d, d, i32, d, i32, d, d, d, p, i32]
        lib.bls_oracle_search_screened.restype = i32
        lib.bls_oracle_fold_bins.argtypes = [p, i64, d, d, i64, p]
        lib.bls_oracle_fold_bins.restype = i32
        lib.bls_oracle_joint.argtypes = [p, p, p, p, i64, p, p, p, p, i64, p, i64, d, i64,
                                         i64, i32, p, p, p, p, p, i32]
        lib.bls_oracle_joint.restype = i32
        lib.tls_oracle_search.argtypes = [p, p, p, i64, p, i64, p, p, p, i64, i64, d, d, d,
                                          p, p, p, p, i32]
        lib.tls_oracle_search.restype = i32
        _lib = lib
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


# --- kernel-level host steps ---------------------------------------------------

def ivar_floor(n_points: int, sum_ivar: float) -> float:
    """``_ivar_floor`` (float64 path), ``_bls_core.py:75-94``."""
    floor = 4.0 * n_points * F64_EPS * sum_ivar
    if not floor > 0.0:
        return float(np.finfo(np.float64).tiny)
    return floor


def duration_bins(durations, bin_duration: float) -> list[int]:
    """``_duration_bins``, ``_bls_core.py:134-149``: round half away, dedupe in order."""
    seen: set[int] = set()
    out: list[int] = []
    for d in np.asarray(durations, dtype=np.float64).tolist():
        kd = math.floor(d / bin_duration + 0.5)
        if kd >= 1 and kd not in seen:
            seen.add(kd)
            out.append(kd)
    return out


@dataclass
class Spec:
    periods: np.ndarray
    bin_duration: float
    dur_bins: list[int]
    width: int


def search_spec(periods, durations, oversample: int) -> Spec:
    """``_search_spec``, ``_bls_core.py:697-706``."""
    p = np.ascontiguousarray(periods, dtype=np.float64)
    d = np.ascontiguousarray(durations, dtype=np.float64)
    bin_duration = float(d.min()) / oversample
    dur = duration_bins(d, bin_duration)
    max_n_bins = int(np.ceil(float(p.max()) / bin_duration)) + oversample
    return Spec(p, bin_duration, dur, max_n_bins + 1)


def host_inputs(t, y, dy):
    """``_host_inputs``, ``_bls_core.py:1043-1058``."""
    t_host = np.ascontiguousarray(t, dtype=np.float64)
    y_host = np.ascontiguousarray(y, dtype=np.float64)
    if y_host.size:
        y_host = y_host - float(np.median(y_host))
    ivar_host = 1.0 / (np.ascontiguousarray(dy, dtype=np.float64) ** 2)
    return t_host, y_host, ivar_host


def objective_flag(objective: str) -> int:
    """``_objective_flag``, ``_bls_core.py:1031-1035``."""
    if objective not in ("snr", "likelihood"):
        raise ValueError("objective must be 'snr' or 'likelihood'")
    return 0 if objective == "snr" else 1


def search(t, y, ivar, periods, *, bin_duration, dur_bins, oversample, width,
           obj_flag, n_threads: int | None = None,
           screen: bool = False) -> dict[str, np.ndarray]:
    """``_bls_search_numba(..., screen=screen)``, ``_bls_core.py:468-500``:
    ``screen=False`` (the default here) evaluates every box, the parity
    checker; ``screen=True`` is the reference's default CPU path, which
    chooses the same boxes bit for bit and is the timed CPU baseline."""
    lib = _load()
    t = np.ascontiguousarray(t, dtype=np.float64)
    ivar = np.ascontiguousarray(ivar, dtype=np.float64)
    yw = np.ascontiguousarray(np.asarray(y, dtype=np.float64) * ivar, dtype=np.float64)
    t_min = float(t.min())
    tau = np.ascontiguousarray(t - t_min, dtype=np.float64)
    db = np.ascontiguousarray(dur_bins, dtype=np.int64)
    sum_y = float(yw.sum())
    sum_ivar = float(ivar.sum())
    per = np.ascontiguousarray(periods, dtype=np.float64)
    out = np.empty((7, per.size), dtype=np.float64)
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    sum_abs = float(np.abs(yw).sum())
    lo, hi = SCREEN_SCALE_RANGE
    if screen and lo <= sum_abs <= hi and lo <= sum_ivar <= hi:
        inv_a, inv_s, slack = 1.0 / sum_abs, 1.0 / sum_ivar, SCREEN_SLACK_EPS * F64_EPS
    else:
        inv_a, inv_s, slack = 0.0, 0.0, math.inf
    rc = lib.bls_oracle_search_screened(
        _ptr(tau), _ptr(yw), _ptr(ivar), tau.size, _ptr(per), per.size, _ptr(db), db.size,
        float(bin_duration), int(oversample), int(width), sum_y, sum_ivar, t_min,
        int(obj_flag), ivar_floor(int(tau.size), sum_ivar), int(bool(screen)), inv_a, inv_s,
        slack, _ptr(out), int(n_threads))
    if rc != 0:
        raise RuntimeError(f"oracle search failed ({rc})")
    return dict(zip(OUTPUT_NAMES, out))


def fold_bins(t, period: float, bin_duration: float, width: int) -> np.ndarray:
    """Phase bin of every point at one period (the numba fold, ``_bls_core.py:365-376``)."""
    lib = _load()
    t = np.ascontiguousarray(t, dtype=np.float64)
    tau = np.ascontiguousarray(t - float(t.min()), dtype=np.float64)
    out = np.empty(tau.size, dtype=np.int32)
    lib.bls_oracle_fold_bins(_ptr(tau), tau.size, float(period), float(bin_duration),
                             int(width), _ptr(out))
    return out


def padded_cumsums(t, y, dy, period: float, durations, oversample: int):
    """The cumulative sums of y*ivar and ivar over bins 0..n_bins of one period
    after the wrap pad (``_bls_core.py:357-388``), accumulated in point order."""
    spec = search_spec([period], durations, oversample)
    th, yh, ih = host_inputs(t, y, dy)
    yw = yh * ih
    bins = fold_bins(th, period, spec.bin_duration, spec.width)
    nb = min(int(np.ceil(period / spec.bin_duration)) + oversample, spec.width - 1)
    my = np.zeros(spec.width)
    mi = np.zeros(spec.width)
    np.add.at(my, bins, yw)
    np.add.at(mi, bins, ih)
    for k in range(oversample):
        dst = nb - oversample + k
        if 0 <= dst < spec.width:
            my[dst] = my[1 + k]
            mi[dst] = mi[1 + k]
    return np.cumsum(my[:nb + 1]), np.cumsum(mi[:nb + 1])


def bls_power(t, y, dy, periods, durations, oversample: int, *, objective: str = "snr",
              n_threads: int | None = None, screen: bool = False) -> dict[str, np.ndarray]:
    """``bls_power(..., backend="numba")``, ``_bls_core.py:882-1028`` (``screen``
    as in :func:`search`)."""
    obj_flag = objective_flag(objective)
    periods_host = np.ascontiguousarray(periods, dtype=np.float64)
    if periods_host.size == 0:
        out = {name: np.empty(0) for name in OUTPUT_NAMES}
        out["period"] = periods_host
        return out
    spec = search_spec(periods_host, durations, oversample)
    th, yh, ih = host_inputs(t, y, dy)
    out = search(th, yh, ih, periods_host, bin_duration=spec.bin_duration,
                 dur_bins=spec.dur_bins, oversample=oversample, width=spec.width,
                 obj_flag=obj_flag, n_threads=n_threads, screen=screen)
    out["period"] = periods_host
    return out


# --- grid and segments (methods/bls.py) ------------------------------------------

@dataclass
class Settings:
    """The ``BLSSettings`` fields the BLS path reads (``core/config.py:218-302``)."""
    min_period_days: float = 0.2
    max_period_days: float = 100.0
    min_transits: int = 2
    duration_min_frac: float = 0.01
    duration_max_frac: float = 0.12
    n_durations: int = 8
    min_duration_days: float = 0.01
    segment_factor: float = 2.0
    grid_duration_frac: float = 0.05
    grid_oversample: int = 2
    bins_per_duration: int = 10
    objective: str = "snr"
    min_detections: int = 20
    extra: dict = field(default_factory=dict)


def segment_durations(p_lo: float, s: Settings) -> np.ndarray:
    """``_segment_durations``, ``bls.py:39-49``."""
    d_hi = s.duration_max_frac * p_lo
    d_lo = max(s.duration_min_frac * p_lo, s.min_duration_days)
    if d_lo >= d_hi:
        return np.asarray([d_hi], dtype=np.float64)
    return np.asarray(np.geomspace(d_lo, d_hi, s.n_durations), dtype=np.float64)


def segment_periods(baseline: float, s: Settings) -> list[tuple[float, np.ndarray]]:
    """``_max_period`` + ``_segment_bounds`` + ``_segment_periods``, ``bls.py:52-105``
    (without the size guard)."""
    max_period = min(s.max_period_days, baseline / s.min_transits)
    bounds = []
    p_lo = s.min_period_days
    while p_lo < max_period:
        p_hi = min(p_lo * s.segment_factor, max_period)
        bounds.append((p_lo, p_hi))
        p_lo = p_hi
    if not bounds:
        return []
    df = s.grid_duration_frac / (s.grid_oversample * baseline)
    parts = []
    for p_lo, p_hi in bounds:
        freq = np.arange(1.0 / p_hi, 1.0 / p_lo, df)
        freq = freq[freq < 1.0 / p_lo]
        if freq.size:
            parts.append((p_lo, np.asarray(1.0 / freq[::-1], dtype=np.float64)))
    return parts


def default_grid(baseline: float, s: Settings):
    """``BLSMethod.default_grid``, ``bls.py:327-359``: ``(periods, meta)``."""
    parts = segment_periods(baseline, s)
    periods = np.concatenate([p for _, p in parts]) if parts else np.empty(0)
    meta = {"segmented": True,
            "segment_starts": tuple(float(p_lo) for p_lo, _ in parts),
            "segment_sizes": tuple(int(p.size) for _, p in parts)}
    return periods, meta


def log_segments(periods: np.ndarray, s: Settings):
    """``_log_segments``, ``bls.py:128-152``."""
    p0 = float(periods.min())
    with np.errstate(divide="ignore", invalid="ignore"):
        index = np.floor(np.log(periods / p0) / math.log(s.segment_factor) + 1e-9).astype(np.int64)
    return [(np.ascontiguousarray(periods[index == k]),
             segment_durations(p0 * s.segment_factor ** k, s))
            for k in np.unique(index).tolist()]


def grid_segments(periods: np.ndarray, meta: dict | None, s: Settings):
    """``_grid_segments``, ``bls.py:155-190``."""
    periods = np.asarray(periods, dtype=np.float64)
    if periods.size == 0:
        return []
    meta = meta or {}
    starts, sizes = meta.get("segment_starts"), meta.get("segment_sizes")
    if (starts is not None and sizes is not None and len(starts) == len(sizes)
            and sum(int(v) for v in sizes) == periods.size):
        segs, off = [], 0
        for p_lo, size in zip(starts, sizes):
            segs.append((periods[off:off + int(size)], segment_durations(float(p_lo), s)))
            off += int(size)
        return segs
    return log_segments(periods, s)


def method_power(t, flux, err, periods, meta, s: Settings, n_threads: int | None = None):
    """``BLSMethod.power`` + ``_assemble`` (``bls.py:274-301``, ``361-395``) on finite
    flux-domain input: ``(frequency, power, extras)`` sorted by ascending frequency."""
    t = np.asarray(t, dtype=np.float64)
    flux = np.asarray(flux, dtype=np.float64)
    err = np.ones_like(flux) if err is None else np.asarray(err, dtype=np.float64)
    chunks = {name: [] for name in SEGMENT_FIELDS}
    for per, dur in grid_segments(periods, meta, s):
        out = bls_power(t, flux, err, per, dur, s.bins_per_duration,
                        objective=s.objective, n_threads=n_threads)
        for name in SEGMENT_FIELDS:
            chunks[name].append(out[name])
    arrays = {k: np.concatenate(v) for k, v in chunks.items()}
    power = np.nan_to_num(arrays["power"], nan=0.0, posinf=0.0, neginf=0.0)
    mean, std = float(power.mean()), float(power.std())
    sde = (power - mean) / std if std > 0.0 else np.zeros_like(power)
    frequency = 1.0 / arrays["period"]
    order = np.argsort(frequency, kind="stable")
    extras = {"depth": arrays["depth"], "depth_snr": arrays["depth_snr"],
              "duration": arrays["duration"], "t0": arrays["transit_time"], "sde": sde}
    return frequency[order], power[order], {k: v[order] for k, v in extras.items()}


def robust_scatter(flux: np.ndarray) -> float:
    """``_robust_scatter``, ``multiband/bls_mb.py:63-76``: 1.4826 x MAD, else the
    standard deviation, else 1."""
    sigma = 1.4826 * float(np.median(np.abs(flux - np.median(flux))))
    if not (np.isfinite(sigma) and sigma > 0.0):
        sigma = float(np.std(flux))
    if not (np.isfinite(sigma) and sigma > 0.0):
        sigma = 1.0
    return sigma


def multiband_power(bands, periods, meta, s: Settings, n_threads: int | None = None,
                    ephemeris: str = "independent"):
    """``bls_multiband_power`` (``multiband/bls_mb.py:120-315``) on finite flux-domain
    bands ``[(name, t, flux, err or None), ...]``: bands with at least 3 points are
    searched over the common segments.  Independent: the per-period power is the
    sum of the squared clipped depth-SNRs and the box comes from the band with the
    largest.  Shared: one box for all bands (``joint_power``).  Returns
    ``(frequency, power, extras, used_band_names, n_samples, baseline)`` in
    ascending frequency."""
    used = [b for b in bands if len(b[1]) >= 3]
    n_total = sum(len(b[1]) for b in used)
    stacked = np.concatenate([np.asarray(b[1], dtype=np.float64) for b in used])
    baseline = float(stacked.max() - stacked.min())
    if all(b[3] is not None for b in used):
        errors = [np.asarray(b[3], dtype=np.float64) for b in used]
    else:
        errors = [np.full(len(b[1]), robust_scatter(np.asarray(b[2], dtype=np.float64)))
                  for b in used]
    parts = {k: [] for k in ("period", "power", "depth", "depth_snr", "duration", "t0",
                             "band_index")}
    segments = grid_segments(periods, meta, s)
    if ephemeris == "shared":
        jb = joint_bands([np.asarray(b[1], dtype=np.float64) for b in used],
                         [np.asarray(b[2], dtype=np.float64) for b in used], errors)
        for per, dur in segments:
            o = joint_power(jb, per, dur, s.bins_per_duration, objective_flag(s.objective),
                            n_threads)
            parts["period"].append(np.asarray(per, dtype=np.float64))
            parts["t0"].append(o.pop("transit_time"))
            for k, v in o.items():
                parts[k].append(v)
    else:
        for per, dur in segments:
            seg = [bls_power(np.asarray(b[1], dtype=np.float64),
                             np.asarray(b[2], dtype=np.float64), e, per, dur,
                             s.bins_per_duration, objective=s.objective, n_threads=n_threads)
                   for b, e in zip(used, errors)]
            dsnr = np.vstack([np.clip(o["depth_snr"], 0.0, None) for o in seg])
            combined = np.sum(dsnr ** 2, axis=0)
            best = np.argmax(dsnr, axis=0)
            cols = np.arange(dsnr.shape[1])
            parts["period"].append(per)
            parts["power"].append(combined)
            parts["depth_snr"].append(np.sqrt(combined))
            parts["depth"].append(np.vstack([o["depth"] for o in seg])[best, cols])
            parts["duration"].append(np.vstack([o["duration"] for o in seg])[best, cols])
            parts["t0"].append(np.vstack([o["transit_time"] for o in seg])[best, cols])
            parts["band_index"].append(best.astype(np.float64))
    joined = {k: np.concatenate(v) for k, v in parts.items()}
    period = joined.pop("period")
    power = np.nan_to_num(joined.pop("power"), nan=0.0, posinf=0.0)
    mean, std = float(power.mean()), float(power.std())
    sde = (power - mean) / std if std > 0.0 else np.zeros_like(power)
    frequency = 1.0 / period
    order = np.argsort(frequency, kind="stable")
    extras = {"depth": joined["depth"], "depth_snr": joined["depth_snr"],
              "duration": joined["duration"], "t0": joined["t0"], "sde": sde,
              "band_index": joined["band_index"]}
    return (frequency[order], power[order], {k: v[order] for k, v in extras.items()},
            [b[0] for b in used], n_total, baseline)


@dataclass
class JointBands:
    """``JointBands``, ``multiband/_bls_joint.py:65-91``: every band of one star with
    one time origin, concatenated; ``starts`` delimits the bands."""
    tau: np.ndarray
    yw: np.ndarray
    ivar: np.ndarray
    starts: np.ndarray
    sum_y: np.ndarray
    sum_ivar: np.ndarray
    floor: np.ndarray
    t_min: float


def joint_bands(times, values, errors) -> JointBands:
    """``joint_bands``, ``multiband/_bls_joint.py:94-135``: each band centred on its
    own median, ``yw = y_c / dy^2``, the times of all bands from the earliest."""
    t_min = float(min(float(np.min(t)) for t in times))
    taus, yws, ivars, sum_y, sum_ivar, floors = [], [], [], [], [], []
    for t, y, dy in zip(times, values, errors, strict=True):
        y_c = np.asarray(y, dtype=np.float64)
        y_c = y_c - float(np.median(y_c))
        ivar = 1.0 / (np.asarray(dy, dtype=np.float64) ** 2)
        yw = y_c * ivar
        taus.append(np.asarray(t, dtype=np.float64) - t_min)
        yws.append(yw)
        ivars.append(ivar)
        sum_y.append(float(yw.sum()))
        sum_ivar.append(float(ivar.sum()))
        floors.append(ivar_floor(int(yw.size), sum_ivar[-1]))
    starts = np.concatenate([[0], np.cumsum([t.size for t in taus])]).astype(np.int64)
    return JointBands(np.ascontiguousarray(np.concatenate(taus)),
                      np.ascontiguousarray(np.concatenate(yws)),
                      np.ascontiguousarray(np.concatenate(ivars)), starts,
                      np.asarray(sum_y, dtype=np.float64), np.asarray(sum_ivar, dtype=np.float64),
                      np.asarray(floors, dtype=np.float64), t_min)


JOINT_FIELDS = ("power", "depth", "depth_snr", "duration", "transit_time", "band_index")


def joint_sweep(jb: JointBands, periods, durations, oversample: int, obj_flag: int,
                n_threads: int | None = None):
    """The numba joint sweep, ``multiband/_bls_joint.py:412-507``, on one segment:
    ``(best_n, best_d, found, y_in[K, P], iv_in[K, P], spec)``."""
    lib = _load()
    spec = search_spec(periods, durations, oversample)
    per = np.ascontiguousarray(spec.periods, dtype=np.float64)
    db = np.ascontiguousarray(spec.dur_bins, dtype=np.int64)
    k = int(jb.starts.size - 1)
    out_n = np.zeros(per.size, dtype=np.int64)
    out_d = np.zeros(per.size, dtype=np.int64)
    found = np.zeros(per.size, dtype=np.uint8)
    yin = np.zeros((k, per.size), dtype=np.float64)
    ivin = np.zeros((k, per.size), dtype=np.float64)
    floors = np.ascontiguousarray(jb.floor, dtype=np.float64)
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    rc = lib.bls_oracle_joint(
        _ptr(jb.tau), _ptr(jb.yw), _ptr(jb.ivar), _ptr(jb.starts), k, _ptr(jb.sum_y),
        _ptr(jb.sum_ivar), _ptr(floors), _ptr(per), per.size, _ptr(db), db.size,
        float(spec.bin_duration), int(oversample), int(spec.width), int(obj_flag),
        _ptr(out_n), _ptr(out_d), _ptr(found), _ptr(yin), _ptr(ivin), int(n_threads))
    if rc != 0:
        raise RuntimeError(f"oracle joint search failed ({rc})")
    return out_n, out_d, found.astype(bool), yin, ivin, spec


def joint_finish(jb: JointBands, y_in, iv_in, best_n, best_d, found, periods,
                 bin_duration: float) -> dict[str, np.ndarray]:
    """``_finish``, ``multiband/_bls_joint.py:359-404``: each band's depth and SNR at
    the chosen box; power = sum of squared SNRs in band order, the depth of the
    band with the largest SNR, the box's duration and mid-transit time."""
    k_bands = int(jb.starts.size - 1)
    n_p = int(np.asarray(periods).size)
    snr = np.zeros((k_bands, n_p))
    depth = np.zeros((k_bands, n_p))
    with np.errstate(divide="ignore", invalid="ignore"):
        for k in range(k_bands):
            floor = float(jb.floor[k])
            iv_out = float(jb.sum_ivar[k]) - iv_in[k]
            ok = (iv_in[k] >= floor) & (iv_out >= floor)
            safe_in = np.where(ok, iv_in[k], 1.0)
            safe_out = np.where(ok, iv_out, 1.0)
            yin = y_in[k] / safe_in
            yout = (float(jb.sum_y[k]) - y_in[k]) / safe_out
            dip = ok & (yout >= yin)
            d = yout - yin
            depth[k] = np.where(dip, d, 0.0)
            snr[k] = np.where(dip, d / np.sqrt(1.0 / safe_in + 1.0 / safe_out), 0.0)
    power = np.zeros(n_p)
    for k in range(k_bands):
        power = power + snr[k] * snr[k]
    band = np.argmax(snr, axis=0)
    duration = best_d.astype(np.float64) * bin_duration
    t0 = np.remainder(best_n.astype(np.float64) * bin_duration + 0.5 * duration,
                      periods) + jb.t_min
    cols = np.arange(n_p)
    return {"power": np.where(found, power, 0.0),
            "depth": np.where(found, depth[band, cols], 0.0),
            "depth_snr": np.where(found, np.sqrt(power), 0.0),
            "duration": np.where(found, duration, 0.0),
            "transit_time": np.where(found, t0, 0.0),
            "band_index": np.where(found, band.astype(np.float64), 0.0)}


def joint_power(jb: JointBands, periods, durations, oversample: int, obj_flag: int,
                n_threads: int | None = None) -> dict[str, np.ndarray]:
    """One segment of ``joint_search`` (``multiband/_bls_joint.py:151-204``)."""
    bn, bd, found, yin, ivin, spec = joint_sweep(jb, periods, durations, oversample,
                                                 obj_flag, n_threads)
    return joint_finish(jb, yin, ivin, bn, bd, found, spec.periods, spec.bin_duration)


# --- transit least squares (methods/tls.py) -------------------------------------

TLS_W_EPS = 1e-300          # tls.py:57
TLS_DEN_REL = 1e-9          # tls.py:63
TLS_CONSTANT_ULPS = 64.0    # tls.py:68
TLS_OUTPUTS = ("sde", "sr", "depth", "duration", "t0")


def tls_template(n: int, u1: float, u2: float) -> np.ndarray:
    """``limb_darkened_template``, tls.py:84-111."""
    if n <= 1:
        return np.ones(max(n, 1), dtype=np.float64)
    x = (np.arange(n, dtype=np.float64) + 0.5) / n - 0.5
    z = np.clip(2.0 * np.abs(x), 0.0, 1.0)
    mu = np.sqrt(1.0 - z * z)
    g = 1.0 - u1 * (1.0 - mu) - u2 * (1.0 - mu) ** 2
    g = np.where(z < 1.0, g, 0.0)
    peak = float(g.max())
    return g / peak if peak > 0.0 else g


def tls_duration_bins(n_bins: int, dmin: float, dmax: float, n_dur: int) -> list[int]:
    """``_duration_bins``, tls.py:114-126."""
    fracs = np.geomspace(dmin, dmax, n_dur)
    return sorted({min(max(int(round(f * n_bins)), 1), n_bins - 1) for f in fracs})


def tls_period_grid(baseline: float, *, min_period: float, max_period: float, min_transits: int,
                    grid_duration_frac: float, duration_min_frac: float,
                    oversample: int) -> np.ndarray:
    """``_period_grid`` (tls.py:141-170) without its size check."""
    pmax = min(max_period, baseline / min_transits)
    if pmax <= min_period:
        return np.zeros(0, dtype=np.float64)
    step = min(grid_duration_frac, 2.0 * duration_min_frac)        # _grid_duration_frac
    df = step / (oversample * baseline)
    freq = np.arange(1.0 / pmax, 1.0 / min_period, df)
    if freq.size == 0:
        return np.zeros(0, dtype=np.float64)
    return np.ascontiguousarray(1.0 / freq[::-1], dtype=np.float64)


def tls_kernel(tau, yw, w, periods, *, n_bins: int, dur_bins, templates, w_total: float,
               den_rel: float = TLS_DEN_REL, n_threads: int | None = None):
    """The numba kernel (tls.py:516-593) through the C restatement: sr, depth,
    duration, t0 (t0 relative to tau's origin)."""
    lib = _load()
    tau = np.ascontiguousarray(tau, dtype=np.float64)
    yw = np.ascontiguousarray(yw, dtype=np.float64)
    w = np.ascontiguousarray(w, dtype=np.float64)
    per = np.ascontiguousarray(periods, dtype=np.float64)
    tmpl = np.ascontiguousarray(np.concatenate([templates[wd] for wd in dur_bins]),
                                dtype=np.float64)
    widths = [len(templates[wd]) for wd in dur_bins]
    off = np.zeros(len(dur_bins), dtype=np.int64)
    if len(widths) > 1:
        off[1:] = np.cumsum(widths[:-1])
    db = np.ascontiguousarray(dur_bins, dtype=np.int64)
    out = np.zeros((4, per.size), dtype=np.float64)
    if n_threads is None:
        n_threads = os.cpu_count() or 1
    rc = lib.tls_oracle_search(_ptr(tau), _ptr(yw), _ptr(w), tau.size, _ptr(per), per.size,
                               _ptr(db), _ptr(off), _ptr(tmpl), db.size, int(n_bins),
                               TLS_W_EPS, float(w_total), float(den_rel), _ptr(out[0]),
                               _ptr(out[1]), _ptr(out[2]), _ptr(out[3]), int(n_threads))
    if rc != 0:
        raise RuntimeError(f"oracle TLS search failed ({rc})")
    return dict(zip(("sr", "depth", "duration", "t0"), out))


def tls_host_inputs(t, y, dy):
    """``tls_power``'s host steps (tls.py:680-699): t_ref, flux scale, weights,
    weighted-mean-subtracted y*w; None when the flux is constant."""
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    t_ref = float(t.min())
    scale_y = float(np.max(np.abs(y))) if y.size else 0.0
    if y.size == 0 or float(np.ptp(y)) <= TLS_CONSTANT_ULPS * F64_EPS * scale_y:
        return None, t_ref, 1.0
    sc = float(np.std(y)) if dy is None else float(np.median(np.abs(dy)))
    scale = 1.0 if not (math.isfinite(sc) and sc > 0.0) else \
        2.0 ** min(max(round(math.log2(sc)), -1000), 1000)
    y = y / scale
    w = np.ones_like(y) if dy is None else \
        1.0 / (np.ascontiguousarray(dy, dtype=np.float64) / scale) ** 2
    w_total = float(w.sum())
    y_mean = float(np.dot(w, y) / w_total)
    yw = w * (y - y_mean)
    return (t - t_ref, yw, w, w_total), t_ref, scale


def tls_power(t, y, dy, periods, *, n_bins: int = 256, duration_min_frac: float = 0.01,
              duration_max_frac: float = 0.10, n_durations: int = 5, u1: float = 0.4,
              u2: float = 0.3, n_threads: int | None = None) -> dict[str, np.ndarray]:
    """``tls_power`` (tls.py:624-755) with the numba kernel: sde, sr, depth,
    duration and absolute t0 per period."""
    periods = np.ascontiguousarray(periods, dtype=np.float64)
    n_p = int(periods.size)
    if n_p == 0:
        return {k: np.zeros(0) for k in TLS_OUTPUTS}
    prep, t_ref, scale = tls_host_inputs(t, y, dy)
    dur = tls_duration_bins(n_bins, duration_min_frac, duration_max_frac, n_durations)
    if prep is None or not dur:
        out = {k: np.zeros(n_p) for k in TLS_OUTPUTS}
        out["t0"] = np.full(n_p, t_ref)
        return out
    tau, yw, w, w_total = prep
    templates = {wd: tls_template(wd, u1, u2) for wd in dur}
    res = tls_kernel(tau, yw, w, periods, n_bins=n_bins, dur_bins=dur, templates=templates,
                     w_total=w_total, n_threads=n_threads)
    sr = res["sr"]
    mean, std = float(sr.mean()), float(sr.std())
    res["sde"] = (sr - mean) / std if std > 0.0 else np.zeros_like(sr)
    res["depth"] = res["depth"] * scale
    if dy is None:
        res["sr"] = sr * (scale * scale)
    res["t0"] = res["t0"] + t_ref
    return res


def best_index(power: np.ndarray) -> int:
    """Index of ``Periodogram.best_period`` (``core/result.py:369-438``): the highest
    finite candidate among interior local maxima and boundary peaks."""
    safe = np.where(np.isfinite(power), power, -np.inf)
    n = safe.size
    cand = []
    if n >= 3:
        interior = (safe[1:-1] > safe[:-2]) & (safe[1:-1] >= safe[2:])
        cand = (np.flatnonzero(interior) + 1).tolist()
    if n == 1:
        cand.append(0)
    elif n >= 2:
        if safe[0] >= safe[1]:
            cand.append(0)
        if safe[-1] > safe[-2]:
            cand.append(n - 1)
    cand = [c for c in cand if np.isfinite(power[c])]
    if not cand:
        finite = np.flatnonzero(np.isfinite(power))
        return int(finite[np.argmax(power[finite])]) if finite.size else -1
    cand = np.asarray(cand)
    order = np.argsort(power[cand])[::-1]
    return int(cand[order[0]])
