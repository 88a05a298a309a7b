"""cuperiod_b200 -- a B200-native Box Least Squares engine.

A drop-in for cuPeriod's BLS path (``method="bls"`` through ``periodogram`` and
``batch_periodograms``): the same trial grids, objective, result object and best
period, computed by hand-written sm_100a kernels behind a C ABI
(``include/bls_b200.h``, ``libbls_b200.so``).  Multi-band BLS (both
statistics) and the transit least squares search (``method="tls"``) run on the
same engine.  There is no CPU fallback: without
the built library or a CUDA device the entry points raise
``BackendUnavailableError``.
"""

from __future__ import annotations

from .api import periodogram, to_input
from .batch import BatchSummary, batch_periodograms, periodogram_to_row
from .bls import BLSMethod, get_method, register
from .columns import ColumnMap
from .core import BLSPower, bls_power, bls_power_many, bls_power_segments
from .errors import (BackendUnavailableError, ColumnResolutionError, CuPeriodError, EngineError,
                     GridTooLargeError, InsufficientDataError, UnknownMethodError)
from .grid import GridSpec, check_grid_size, log_period_grid
from .lightcurve import Domain, LightCurve, MultiBandLightCurve
from .multiband import bls_multiband_power
from .result import Peak, Periodogram
from .settings import BLSSettings, TLSSettings
from .tls import TLSMethod, tls_power

__version__ = "0.1.0"

__all__ = [
    "BLSMethod", "BLSPower", "BLSSettings", "BackendUnavailableError", "BatchSummary",
    "ColumnMap", "ColumnResolutionError",
    "CuPeriodError", "Domain", "EngineError", "GridSpec", "GridTooLargeError",
    "InsufficientDataError", "LightCurve", "MultiBandLightCurve", "Peak", "Periodogram", "UnknownMethodError",
    "batch_periodograms", "bls_multiband_power", "bls_power", "bls_power_many", "bls_power_segments",
    "check_grid_size", "get_method", "log_period_grid", "periodogram", "periodogram_to_row",
    "register", "to_input", "TLSMethod", "TLSSettings", "tls_power",
]
