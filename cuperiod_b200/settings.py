"""``BLSSettings`` and ``TLSSettings``: the parameters of the BLS and TLS
searches, as cuPeriod defines them (src/cuperiod/core/config.py:218-302 and
605-702, with the device fields of 60-101).

A pydantic-settings model with the same field names, defaults, bounds and
``CUPERIOD_BLS_*`` environment overrides, so a settings object or a saved
configuration written for the reference is accepted unchanged.  ``backend``
additionally accepts ``"b200"``, this engine's own name.
"""

from __future__ import annotations

from typing import Any, Literal

from pydantic import Field, model_validator
from pydantic_settings import BaseSettings, SettingsConfigDict

_MAX_DURATION_FRAC = 1.0


class BLSSettings(BaseSettings):
    """Settings for the box least squares (BLS) search."""

    model_config = SettingsConfigDict(env_prefix="CUPERIOD_BLS_", extra="forbid")

    device: Literal["auto", "cpu", "cuda", "mps", "xpu"] = Field(default="auto")
    precision: Literal["auto", "float64", "float32"] = Field(default="auto")
    min_period_days: float = Field(default=0.2, gt=0.0)
    max_period_days: float = Field(default=100.0, gt=0.0)
    min_transits: int = Field(default=2, ge=1)
    duration_min_frac: float = Field(default=0.01, gt=0.0, lt=_MAX_DURATION_FRAC)
    duration_max_frac: float = Field(default=0.12, gt=0.0, lt=_MAX_DURATION_FRAC)
    n_durations: int = Field(default=8, ge=1)
    min_duration_days: float = Field(default=0.01, gt=0.0)
    segment_factor: float = Field(default=2.0, gt=1.0)
    grid_duration_frac: float = Field(default=0.05, gt=0.0)
    grid_oversample: int = Field(default=2, ge=1)
    bins_per_duration: int = Field(default=10, ge=1)
    objective: Literal["snr", "likelihood"] = Field(default="snr")
    mb_ephemeris: Literal["independent", "shared"] = Field(default="independent")
    n_peaks: int = Field(default=10, ge=1)
    peak_separation_rayleigh: float = Field(default=3.0, gt=0.0)
    alias_freq_tolerance: float = Field(default=0.0035, ge=0.0)
    harmonic_max: int = Field(default=8, ge=1)
    min_detections: int = Field(default=20, ge=3)
    backend: Literal["auto", "cpu", "gpu", "numba", "numpy", "astropy", "cupy", "torch",
                     "b200"] = Field(default="auto")
    batch_periods: int = Field(default=2048, ge=1)
    downsample_points: int = Field(default=2000, ge=2)

    @model_validator(mode="after")
    def _check_bounds(self) -> "BLSSettings":
        if not self.min_period_days < self.max_period_days:
            raise ValueError("min_period_days must be < max_period_days")
        if not self.duration_min_frac < self.duration_max_frac:
            raise ValueError("duration_min_frac must be < duration_max_frac")
        return self


class TLSSettings(BaseSettings):
    """Settings for the transit least squares (TLS) search (config.py:605-702):
    the same fields, defaults, bounds and ``CUPERIOD_TLS_*`` overrides."""

    model_config = SettingsConfigDict(env_prefix="CUPERIOD_TLS_", extra="forbid")

    device: Literal["auto", "cpu", "cuda", "mps", "xpu"] = Field(default="auto")
    precision: Literal["auto", "float64", "float32"] = Field(default="auto")
    min_period_days: float = Field(default=0.5, gt=0.0)
    max_period_days: float = Field(default=100.0, gt=0.0)
    min_transits: int = Field(default=2, ge=1)
    oversample: int = Field(default=2, ge=1)
    grid_duration_frac: float = Field(default=0.05, gt=0.0)
    n_phase_bins: int = Field(default=256, ge=16)
    duration_min_frac: float = Field(default=0.01, gt=0.0, lt=_MAX_DURATION_FRAC)
    duration_max_frac: float = Field(default=0.10, gt=0.0, lt=_MAX_DURATION_FRAC)
    n_durations: int = Field(default=5, ge=1)
    limb_dark_u1: float = Field(default=0.4, allow_inf_nan=False)
    limb_dark_u2: float = Field(default=0.3, allow_inf_nan=False)
    n_peaks: int = Field(default=10, ge=1)
    peak_separation_rayleigh: float = Field(default=3.0, gt=0.0)
    alias_freq_tolerance: float = Field(default=0.0035, ge=0.0)
    harmonic_max: int = Field(default=8, ge=1)
    min_detections: int = Field(default=20, ge=3)
    backend: Literal["auto", "cpu", "gpu", "numba", "numpy", "cupy", "torch",
                     "b200"] = Field(default="auto")
    period_batch: int = Field(default=256, ge=1)
    downsample_points: int = Field(default=2000, ge=2)

    @model_validator(mode="after")
    def _check_bounds(self) -> "TLSSettings":
        if not self.min_period_days < self.max_period_days:
            raise ValueError("min_period_days must be < max_period_days")
        if not self.duration_min_frac < self.duration_max_frac:
            raise ValueError("duration_min_frac must be < duration_max_frac")
        # the limb intensity 1 - u1 - u2 at mu = 0 must stay >= 0 (config.py:620-628)
        if self.limb_dark_u1 + self.limb_dark_u2 > 1.0:
            raise ValueError(f"limb_dark_u1 + limb_dark_u2 ({self.limb_dark_u1} + "
                             f"{self.limb_dark_u2}) must be <= 1 (non-negative limb intensity)")
        return self


def peak_defaults(settings: Any) -> dict[str, Any]:
    """The peak-selection defaults a settings object carries
    (``peak_defaults_from_settings``, src/cuperiod/core/result.py:53-80)."""
    out: dict[str, Any] = {}
    for src, dst in (("n_peaks", "n"), ("peak_separation_rayleigh", "min_separation_rayleigh"),
                     ("alias_freq_tolerance", "alias_tolerance"),
                     ("harmonic_max", "harmonic_max"), ("downsample_points", "n_points")):
        value = getattr(settings, src, None)
        if value is not None:
            out[dst] = value
    return out


__all__ = ["BLSSettings", "TLSSettings", "peak_defaults"]
