"""Light-curve table columns: which column is the time, the value, the error
and the band (cuPeriod src/cuperiod/core/columns.py:60-396).

The candidate name lists are the reference's, so a table cuPeriod reads resolves
to the same columns here; matching is case-insensitive and the first candidate
present wins.  The error column is resolved for the same measurement as the
value: names derived from the value column first (``PDCSAP_FLUX`` pairs with
``PDCSAP_FLUX_ERR``, ``uJy`` with ``duJy``), then the spellings of the value's
domain, then domain-neutral ones.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass
from typing import Final

from .errors import ColumnResolutionError
from .lightcurve import Domain

#: Time columns, most specific first (barycentric/heliocentric before plain JD).
TIME_NAMES: Final = ("bjd_tdb", "bjd", "hjd", "btjd", "bkjd", "mjd", "hmjd",
                     "midpointmjdtai", "midpointtai", "obstime", "jd", "time", "date", "t")
#: Magnitude value columns.
MAG_NAMES: Final = ("mag", "magnitude", "vmag", "gmag", "rmag", "bmag", "imag", "psfmag",
                    "phot_mag", "mag_0", "m")
#: Flux value columns (``ujy`` before the bare ``f``, ATLAS's filter column).
FLUX_NAMES: Final = ("pdcsap_flux", "kspsap_flux", "sap_flux", "psfflux", "psflux",
                     "psfdiffflux", "norm_flux", "rel_flux", "flux", "ujy", "mjy", "fnu", "f")
#: Magnitude errors.
MAG_ERR_NAMES: Final = ("mag_err", "magnitude_err", "mag_error", "magerr", "e_mag", "merr",
                        "dmag", "dm", "mer_0")
#: Flux errors.
FLUX_ERR_NAMES: Final = ("flux_err", "flux_error", "sap_flux_err", "pdcsap_flux_err",
                         "kspsap_flux_err", "psfflux_err", "psffluxerr", "psfluxerr",
                         "psfdiffflux_err", "psfdifffluxerr", "e_flux", "dujy")
#: Domain-neutral error spellings, tried last.
GENERIC_ERR_NAMES: Final = ("err", "error", "sigma")
ERR_NAMES: Final = MAG_ERR_NAMES + FLUX_ERR_NAMES + GENERIC_ERR_NAMES
#: Band/filter columns (multi-band tables only).
BAND_NAMES: Final = ("band", "filter", "filtercode", "filterid", "filtername", "phot_filter",
                     "passband", "fid")

_FLUX_TOKENS: Final = ("flux", "fnu", "ujy", "mjy", "njy", "nmgy", "jansky")


def coerce_domain(domain: Domain | str | None) -> Domain | None:
    return None if domain is None else Domain(domain)


def infer_domain(value_column: str) -> Domain | None:
    """Flux or magnitude from a value column's name, else None (columns.py:213-238)."""
    low = value_column.lower()
    if low in FLUX_NAMES:
        return Domain.FLUX
    if low in MAG_NAMES:
        return Domain.MAGNITUDE
    if any(tok in low for tok in _FLUX_TOKENS):
        return Domain.FLUX
    if "mag" in low:
        return Domain.MAGNITUDE
    return None


@dataclass(frozen=True)
class ResolvedColumns:
    time: str
    value: str
    error: str | None
    band: str | None
    domain: Domain


def _match(role: str, explicit: str | None, candidates, available: list[str],
           lower_to_actual: dict[str, str]) -> str | None:
    if explicit is not None:
        if explicit in available:
            return explicit
        if explicit.lower() in lower_to_actual:
            return lower_to_actual[explicit.lower()]
        raise ColumnResolutionError(
            f"{role} column {explicit!r} not found; available columns: {available}")
    for cand in candidates:
        if cand in lower_to_actual:
            return lower_to_actual[cand]
    return None


@dataclass(frozen=True)
class ColumnMap:
    """Explicit time/value/error/band column names; None fields are detected."""

    time: str | None = None
    value: str | None = None
    error: str | None = None
    band: str | None = None

    def __post_init__(self) -> None:
        for role in ("time", "value", "error", "band"):
            label = getattr(self, role)
            if label is not None and not isinstance(label, str):
                object.__setattr__(self, role, str(label))

    def resolve(self, columns, *, domain: Domain | str | None = None) -> ResolvedColumns:
        """The table's columns for each role (columns.py:280-375)."""
        explicit = coerce_domain(domain)
        available = [str(c) for c in columns]
        lower_to_actual: dict[str, str] = {}
        for col in available:
            lower_to_actual.setdefault(col.lower(), col)
        if self.value is not None:
            value_candidates: tuple[str, ...] = ()
        elif explicit is Domain.MAGNITUDE:
            value_candidates = MAG_NAMES + FLUX_NAMES
        else:
            value_candidates = FLUX_NAMES + MAG_NAMES
        time = _match("time", self.time, TIME_NAMES, available, lower_to_actual)
        value = _match("value", self.value, value_candidates, available, lower_to_actual)
        band = _match("band", self.band, BAND_NAMES, available, lower_to_actual)
        if time is None:
            raise ColumnResolutionError("could not resolve a time column; pass "
                                        f"ColumnMap(time=...). Available columns: {available}")
        if value is None:
            raise ColumnResolutionError("could not resolve a value (magnitude/flux) column; "
                                        f"pass ColumnMap(value=...). Available columns: {available}")
        inferred = infer_domain(value)
        if explicit is not None and self.value is None and inferred is not None \
                and inferred is not explicit:
            warnings.warn(f"domain={explicit.value!r} was given but no {explicit.value} column "
                          f"was found; {value!r} looks like a {inferred.value} column and is "
                          f"read as {explicit.value} as requested", UserWarning, stacklevel=2)
        resolved_domain = explicit or inferred or Domain.MAGNITUDE
        v = value.lower()
        derived = (f"{v}_err", f"{v}err", f"{v}_error", f"{v}error", f"e_{v}", f"d{v}")
        domain_err = FLUX_ERR_NAMES if resolved_domain is Domain.FLUX else MAG_ERR_NAMES
        error = _match("error", self.error, derived + domain_err + GENERIC_ERR_NAMES, available,
                       lower_to_actual)
        return ResolvedColumns(time=time, value=value, error=error, band=band,
                               domain=resolved_domain)


__all__ = ["BAND_NAMES", "ColumnMap", "ERR_NAMES", "FLUX_ERR_NAMES", "FLUX_NAMES",
           "GENERIC_ERR_NAMES", "MAG_ERR_NAMES", "MAG_NAMES", "ResolvedColumns", "TIME_NAMES",
           "coerce_domain", "infer_domain"]
