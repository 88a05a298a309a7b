"""Single-curve entry point: ``periodogram`` (cuPeriod src/cuperiod/api.py:204-307)
for the BLS method on the B200 engine."""

from __future__ import annotations

import warnings
from typing import Any, Mapping, Sequence

import numpy as np

from .bls import get_method
from .grid import GridSpec
from .lightcurve import Domain, LightCurve, MultiBandLightCurve, raise_if_unusable
from .result import Periodogram
from .settings import BLSSettings


def _looks_like_arrays(data: Any) -> bool:
    return isinstance(data, (tuple, list)) and len(data) in (2, 3) and all(
        np.ndim(x) == 1 for x in data)


def _check_bands(bands: Mapping[str, Any], domain: Domain | None) -> None:
    """Every band a LightCurve, all in one domain unless ``domain`` converts them
    (api.py:134-158)."""
    for name, lc in bands.items():
        if not isinstance(lc, LightCurve):
            raise TypeError(f"band {name!r} is a {type(lc).__name__}, not a LightCurve")
    if domain is None and len({lc.domain for lc in bands.values()}) > 1:
        raise ValueError("bands are in different brightness domains; pass domain='magnitude' "
                         "or domain='flux' to convert them all")


def to_input(data: Any, *, columns: Any = None,
             domain: Domain | str | None = None) -> LightCurve | MultiBandLightCurve:
    """A LightCurve or MultiBandLightCurve from a user input (api.py:47-131): a
    LightCurve/MultiBandLightCurve (converted when ``domain`` is given), a
    ``(t, y[, dy])`` tuple (magnitudes unless ``domain`` says otherwise), a
    ``{band: LightCurve}`` mapping, or a pandas/pyarrow/``{column: array}`` table
    read with column detection -- split into bands when ``columns`` names a band
    column."""
    dom = None if domain is None else Domain(domain)
    if isinstance(data, LightCurve):
        return data if dom is None else data.in_domain(dom)
    if isinstance(data, MultiBandLightCurve):
        _check_bands(data.bands, dom)
        if dom is None:
            return data
        return MultiBandLightCurve({k: lc.in_domain(dom) for k, lc in data.bands.items()},
                                   data.meta)
    if _looks_like_arrays(data):
        t, y = data[0], data[1]
        dy = data[2] if len(data) == 3 else None
        return LightCurve.from_arrays(np.asarray(t), np.asarray(y),
                                      None if dy is None else np.asarray(dy),
                                      domain=dom or Domain.MAGNITUDE)
    band_split = columns is not None and getattr(columns, "band", None) is not None
    if isinstance(data, Mapping):
        values = list(data.values())
        if values and all(isinstance(v, LightCurve) for v in values):
            _check_bands(data, dom)
            bands = data if dom is None else {k: lc.in_domain(dom) for k, lc in data.items()}
            return MultiBandLightCurve.from_light_curves({str(k): v for k, v in bands.items()})
    if band_split:
        return MultiBandLightCurve.from_dataframe(data, columns=columns, domain=dom)
    if isinstance(data, Mapping) or hasattr(data, "columns") or hasattr(data, "column_names"):
        return LightCurve.from_dataframe(data, columns=columns, domain=dom)
    raise TypeError("expected a LightCurve, a MultiBandLightCurve, a (t, y[, dy]) tuple, a "
                    "{band: LightCurve} mapping or a table")


def _settings(settings: Any, cls: type = BLSSettings) -> Any:
    """A settings object of the method's class: None gives the defaults, a mapping
    is read directly or under the method's name (``{"TLS": {...}}``)."""
    if settings is None:
        return cls()
    if isinstance(settings, cls):
        return settings
    if isinstance(settings, Mapping):
        name = cls.__name__[:-len("Settings")]
        for key in (name, name.lower()):
            if key in settings:
                return _settings(settings[key], cls)
        return cls(**settings)
    raise TypeError(f"settings must be {cls.__name__} or a mapping, "
                    f"got {type(settings).__name__}")


#: Median range of a bare tuple's values that looks like a normalised flux read as
#: magnitudes (api.py:36).
_NORMALISED_FLUX_RANGE = (0.5, 1.5)


def _warn_flux_tuple(data: Any, lc: Any, methods: Sequence[Any]) -> None:
    """Warn when a box or transit search is about to read a normalised flux as
    magnitudes (api.py:161-192): a bare ``(t, y[, dy])`` tuple is magnitudes by
    default, and the flux conversion turns every dip of a normalised flux into a
    brightening that a dip-only search cannot see.  Values centred in 0.5-1.5 are
    the tell-tale."""
    if not isinstance(lc, LightCurve) or not _looks_like_arrays(data):
        return
    flux_methods = [m.name for m in methods if m.natural_domain is Domain.FLUX]
    if not flux_methods or lc.value.size == 0:
        return
    with np.errstate(all="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        median = float(np.nanmedian(lc.value))
    lo, hi = _NORMALISED_FLUX_RANGE
    if lo < median < hi:
        warnings.warn(
            f"{', '.join(flux_methods)}: the (t, y, dy) tuple is read as magnitudes "
            f"(median {median:.3g}), but its values look like a normalised flux; pass "
            "domain='flux' if they are fluxes, or a LightCurve with an explicit domain "
            "to silence this.", UserWarning, stacklevel=3)


def _method_key(name: str) -> str:
    return "".join(ch for ch in str(name) if ch.isalnum()).upper()


class MultiResult(Mapping):
    """Several methods' periodograms of one light curve, keyed by method name
    (core/result.py:487-560): lookups ignore case and separators."""

    def __init__(self, results: Mapping[str, Periodogram]):
        self.results = dict(results)

    def _resolve(self, method: object) -> str | None:
        if not isinstance(method, str):
            return None
        if method in self.results:
            return method
        wanted = _method_key(method)
        for key in self.results:
            if _method_key(key) == wanted:
                return key
        return None

    def __getitem__(self, method: str) -> Periodogram:
        key = self._resolve(method)
        if key is None:
            raise KeyError(method)
        return self.results[key]

    def __contains__(self, method: object) -> bool:
        return self._resolve(method) is not None

    def __iter__(self):
        return iter(self.results)

    def __len__(self) -> int:
        return len(self.results)

    def best_periods(self, n: int | None = None, **kwargs: Any) -> dict:
        return {k: v.best_periods(n, **kwargs) for k, v in self.results.items()}


def _select_settings(methods: Sequence[Any], settings: Any) -> dict:
    """Each method's settings from one ``settings=`` argument
    (methods/base.py:459-540): None gives defaults; one settings object goes to
    the methods of its class (it must match one); a mapping is keyed like method
    names."""
    if settings is None:
        return {m.name: m.settings_cls() for m in methods}
    if not isinstance(settings, Mapping):
        if not any(isinstance(settings, m.settings_cls) for m in methods):
            expected = " or ".join(dict.fromkeys(m.settings_cls.__name__ for m in methods))
            raise TypeError(f"settings: expected {expected}, got {type(settings).__name__}")
        return {m.name: settings if isinstance(settings, m.settings_cls) else m.settings_cls()
                for m in methods}
    if any(_method_key(k) in {_method_key(m.name) for m in methods} for k in settings):
        keyed = {_method_key(k): v for k, v in settings.items()}
        return {m.name: _settings(keyed.get(_method_key(m.name)), m.settings_cls)
                for m in methods}
    return {m.name: _settings(settings, m.settings_cls) for m in methods}


def _run_one(m: Any, lc: Any, s: Any, backend: str | None, grid: GridSpec | None,
             engine: Any) -> Periodogram:
    """One method on one light curve (api.py:203-231): a placeholder error column
    is named before a grid is built, then the default grid unless one is given."""
    m.resolve_backend(backend if backend not in (None, "auto") else s.backend)
    if isinstance(lc, MultiBandLightCurve):
        if not m.supports_multiband:
            raise ValueError(f"{m.name} does not support multi-band input")
        raise_if_unusable(lc, f"{m.name} multiband")
        from .multiband import multiband_default_grid
        g = grid or multiband_default_grid(m, lc, s)
        return m.multiband_power(g, lc, s, engine=engine).with_peak_defaults(s)
    single = lc.in_domain(m.natural_domain)
    raise_if_unusable(single, m.name)
    g = grid or m.default_grid(single, s)
    return m.power(g, single, s, engine=engine).with_peak_defaults(s)


def periodogram(data: Any, method: str | Sequence[str] = "BLS", *,
                backend: str | None = "auto", grid: GridSpec | None = None,
                settings: Any = None, columns: Any = None,
                domain: Domain | str | None = None, engine=None) -> Periodogram | MultiResult:
    """The BLS or TLS periodogram of one light curve (api.py:233-307): flux domain
    (magnitudes converted), the default grid unless ``grid`` is given, peak
    defaults from the settings.  Several method names give a ``MultiResult``."""
    lc = to_input(data, columns=columns, domain=domain)
    names = [method] if isinstance(method, str) else list(method)
    methods = [get_method(name) for name in names]
    chosen = _select_settings(methods, settings)
    if domain is None:
        _warn_flux_tuple(data, lc, methods)
    results = {m.name: _run_one(m, lc, chosen[m.name], backend, grid, engine) for m in methods}
    if isinstance(method, str):
        return results[methods[0].name]
    return MultiResult(results)


__all__ = ["MultiResult", "periodogram", "to_input"]
