"""Multi-band BLS (cuPeriod src/cuperiod/multiband/bls_mb.py:1-315).

Bands of one star share the trial period grid.  In the "independent" statistic
each band is box-searched on its own -- here all bands of the star are curves of
one engine launch -- and the per-period power is the quadrature stack of the
bands' clipped depth-SNRs, sum_k max(SNR_k, 0)^2, with the box (depth, duration,
mid-transit time) of the band detecting it most strongly.  In the "shared"
statistic (multiband/_bls_joint.py) one box -- one duration and one phase from
one time origin -- is placed in every band at once and chosen by the summed
per-band objective of the bands that dip in it (the engine's joint kernel); the
power is the same quadrature stack at that box.  A band's errors are used only
when every contributing band has them; otherwise every band is searched with a
constant error equal to its own robust scatter (1.4826 x MAD).
"""

from __future__ import annotations

from typing import Any, Final

import numpy as np

from . import _lib
from .errors import InsufficientDataError
from .grid import GridSpec
from .lightcurve import Domain, LightCurve, MultiBandLightCurve
from .result import Periodogram

#: A band needs at least this many finite points to contribute (bls_mb.py:52-53).
MIN_BAND_POINTS: Final = 3
#: Median absolute deviation to Gaussian sigma (bls_mb.py:55-56).
MAD_TO_SIGMA: Final = 1.4826
#: The multi-band box statistics (bls_mb.py:59-60).
EPHEMERIS_MODES: Final = ("independent", "shared")


def robust_scatter(flux: np.ndarray) -> float:
    """1.4826 x the median absolute deviation, else the standard deviation, else 1
    (bls_mb.py:63-76)."""
    sigma = MAD_TO_SIGMA * float(np.median(np.abs(flux - np.median(flux))))
    if not (np.isfinite(sigma) and sigma > 0.0):
        sigma = float(np.std(flux))
    if not (np.isfinite(sigma) and sigma > 0.0):
        sigma = 1.0
    return sigma


def band_errors(bands: list[LightCurve]) -> list[np.ndarray]:
    """Real errors when every band has them, else each band's robust scatter
    (bls_mb.py:79-92)."""
    if all(lc.error is not None for lc in bands):
        return [np.asarray(lc.error, dtype=np.float64) for lc in bands]
    return [np.full(lc.n, robust_scatter(lc.value)) for lc in bands]


def resolve_ephemeris(settings: Any, ephemeris: str | None = None) -> str:
    """The argument, else ``settings.mb_ephemeris``, else "independent"
    (bls_mb.py:95-117)."""
    mode = ephemeris if ephemeris is not None else getattr(settings, "mb_ephemeris",
                                                           "independent")
    mode = str(mode).strip().lower()
    if mode not in EPHEMERIS_MODES:
        raise ValueError(f"BLS multiband: unknown ephemeris {mode!r}; choose from "
                         f"{EPHEMERIS_MODES}")
    return mode


def multiband_default_grid(method: Any, mblc: MultiBandLightCurve, settings: Any) -> GridSpec:
    """The method's default grid over the stacked baseline (api.py:195-200)."""
    time, value, error, _ = mblc.finite().stacked()
    return method.default_grid(LightCurve(time, value, error, Domain.FLUX), settings)


def bls_multiband_power(grid: GridSpec, mblc: MultiBandLightCurve, settings: Any, *,
                        ephemeris: str | None = None,
                        engine: _lib.Engine | None = None) -> Periodogram:
    """The multi-band BLS periodogram on a shared period grid (bls_mb.py:120-315)."""
    from .bls import BACKEND_NAME, _grid_segments
    from .core import _objective_flag
    mode = resolve_ephemeris(settings, ephemeris)
    finite = mblc.finite()
    used = [(name, lc.in_domain(Domain.FLUX)) for name, lc in finite.bands.items()
            if lc.n >= MIN_BAND_POINTS]
    if not used:
        raise InsufficientDataError("BLS multiband: no band has enough finite points")
    bands = [lc for _, lc in used]
    n_total = sum(lc.n for lc in bands)
    if n_total < settings.min_detections:
        raise InsufficientDataError(
            f"BLS multiband: {n_total} finite points across usable bands "
            f"< min_detections {settings.min_detections}")
    stacked = np.concatenate([lc.time for lc in bands])
    baseline = float(stacked.max() - stacked.min())
    if baseline <= 0.0:
        raise InsufficientDataError("BLS multiband: no usable time baseline")
    segments = _grid_segments(grid, settings)
    if not segments:
        raise InsufficientDataError("BLS multiband: empty trial grid")
    errors = band_errors(bands)
    # every band of the star in one launch: out[field, band, period]
    packed_grid = _lib.PackedGrid.from_segments(segments, settings.bins_per_duration,
                                                _objective_flag(settings.objective))
    curves = _lib.PackedCurves.from_arrays([(lc.time, lc.value, e)
                                            for lc, e in zip(bands, errors)])
    eng = engine or _lib.default_engine()
    period = np.concatenate([np.asarray(p, dtype=np.float64) for p, _ in segments])
    if mode == "shared":
        # one box for every band (bls_mb.py:278-312): the joint kernel's fields
        joint = dict(zip(_lib.JOINT_FIELD_NAMES, eng.search_joint(packed_grid, curves)))
        combined = joint["power"]
        fields = {"depth": joint["depth"], "depth_snr": joint["depth_snr"],
                  "duration": joint["duration"], "t0": joint["transit_time"],
                  "band_index": joint["band_index"]}
    else:
        out = eng.search(packed_grid, curves)
        names = _lib.FIELD_NAMES
        dsnr = np.clip(out[names.index("depth_snr")], 0.0, None)
        combined = np.sum(dsnr ** 2, axis=0)
        best = np.argmax(dsnr, axis=0)
        cols = np.arange(dsnr.shape[1])
        fields = {"depth": out[names.index("depth")][best, cols],
                  "depth_snr": np.sqrt(combined),
                  "duration": out[names.index("duration")][best, cols],
                  "t0": out[names.index("transit_time")][best, cols],
                  "band_index": best.astype(np.float64)}
    power = np.nan_to_num(combined, nan=0.0, posinf=0.0)
    mean, std = float(power.mean()), float(power.std())
    sde = (power - mean) / std if std > 0.0 else np.zeros_like(power)
    extras = {"depth": fields["depth"], "depth_snr": fields["depth_snr"],
              "duration": fields["duration"], "t0": fields["t0"], "sde": sde,
              "band_index": fields["band_index"]}
    meta = {**dict(finite.meta), "bands": tuple(name for name, _ in used),
            "mb_ephemeris": mode}
    return Periodogram.from_spectrum(method="BLS", backend=BACKEND_NAME, frequency=1.0 / period,
                                     power=power, objective_sense="max", n_samples=n_total,
                                     baseline=baseline, extras=extras, meta=meta)


__all__ = ["EPHEMERIS_MODES", "band_errors", "bls_multiband_power", "multiband_default_grid",
           "resolve_ephemeris", "robust_scatter"]
