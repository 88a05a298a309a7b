"""Exceptions of the BLS path, named as cuPeriod names them
(src/cuperiod/core/errors.py): callers that catch the reference's exception
types catch these the same way."""

from __future__ import annotations


class CuPeriodError(Exception):
    """Base class of this package's errors."""


class InsufficientDataError(CuPeriodError, ValueError):
    """Too few usable points, no baseline, or an empty trial grid."""


class GridTooLargeError(CuPeriodError, ValueError):
    """A trial grid above the hard size limit (checked before allocation)."""


class BackendUnavailableError(CuPeriodError, RuntimeError):
    """The CUDA engine cannot run here (no library, no device, shared memory)."""


class UnknownMethodError(CuPeriodError, KeyError):
    """A method name that is not registered."""


class ColumnResolutionError(CuPeriodError, ValueError):
    """A light-curve table's time, value or band column could not be resolved."""


class EngineError(CuPeriodError, RuntimeError):
    """The CUDA engine failed at run time (a CUDA error or a device-side check)."""


__all__ = [
    "BackendUnavailableError",
    "ColumnResolutionError",
    "CuPeriodError",
    "EngineError",
    "GridTooLargeError",
    "InsufficientDataError",
    "UnknownMethodError",
]
