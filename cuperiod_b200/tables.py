"""Reading light-curve tables (cuPeriod src/cuperiod/core/lightcurve.py:686-865):
pandas, pyarrow and ``{column: array}`` tables, and files by extension.

Parquet is read with pyarrow; CSV, TSV, ECSV and whitespace-separated text with
pandas (a ``.gz``/``.bz2``/``.xz`` suffix is looked through, a UTF-8 byte-order
mark is dropped from the first column name).  FITS needs astropy, which this
package does not depend on.
"""

from __future__ import annotations

from pathlib import Path
from typing import Any, Callable, Mapping

import numpy as np

COMPRESSION_SUFFIXES = frozenset({".gz", ".bz2", ".xz"})
FITS_SUFFIXES = frozenset({".fits", ".fit", ".fts", ".fz"})
_BOM_PREFIXES = ("\ufeff", "\xef\xbb\xbf")


def format_suffix(path: Path) -> str:
    """The extension naming the format: ``star.csv.gz`` -> ``.csv``."""
    suffixes = [s.lower() for s in Path(path).suffixes]
    if len(suffixes) >= 2 and suffixes[-1] in COMPRESSION_SUFFIXES:
        return suffixes[-2]
    return suffixes[-1] if suffixes else ""


def adapt_table(obj: Any) -> tuple[list[str], Callable[[str], Any]]:
    """``(column names, getter)`` of a pyarrow, pandas or mapping table; a
    non-string label is listed as its ``str()`` (first label wins)."""
    if hasattr(obj, "column_names") and hasattr(obj, "column"):
        return list(obj.column_names), lambda name: obj.column(name)
    if hasattr(obj, "iloc") and hasattr(obj, "columns"):
        keys: Any = obj.columns
    elif isinstance(obj, Mapping):
        keys = obj.keys()
    else:
        raise TypeError(f"unsupported table type: {type(obj)!r}")
    labels: dict[str, Any] = {}
    for key in keys:
        labels.setdefault(str(key), key)
    return list(labels), lambda name: obj[labels[name]]


def as_float(column: Any) -> np.ndarray:
    """A column as FP64, nulls as NaN."""
    mod = type(column).__module__
    if mod.startswith("pyarrow"):
        column = column.to_numpy(zero_copy_only=False)
    elif mod.startswith("pandas"):
        column = column.to_numpy(dtype=np.float64, na_value=np.nan)
    arr = np.ma.filled(np.ma.asarray(column, dtype=np.float64), np.nan)
    return np.ascontiguousarray(arr, dtype=np.float64).ravel()


def _strip_bom(df):
    cols = list(df.columns)
    if cols and isinstance(cols[0], str):
        for bom in _BOM_PREFIXES:
            if cols[0].startswith(bom):
                bare = cols[0][len(bom):]
                if bare and bare not in cols:
                    df = df.rename(columns={cols[0]: bare})
                break
    return df


def read_table_object(path: str | Path) -> Any:
    """A table object from a file, by extension."""
    path = Path(path)
    suffix = format_suffix(path)
    if suffix in {".parquet", ".pq"}:
        import pyarrow.parquet as pq
        return pq.read_table(path)
    if suffix in FITS_SUFFIXES:
        from .errors import BackendUnavailableError
        raise BackendUnavailableError(f"{path}: FITS tables need astropy, which is not installed")
    import pandas as pd
    if suffix == ".csv":
        return _strip_bom(pd.read_csv(path, comment=None))
    if suffix == ".ecsv":
        return pd.read_csv(path, comment="#")
    if suffix in {".tsv", ".tab"}:
        return _strip_bom(pd.read_csv(path, sep="\t"))
    return _strip_bom(pd.read_csv(path, sep=r"\s+", comment="#"))


def band_label(value: Any) -> str:
    """A band cell as a clean string, "" when missing (lightcurve.py:846-862)."""
    if value is None:
        return ""
    if isinstance(value, bytes):
        return value.decode("utf-8", errors="replace").strip()
    if isinstance(value, (float, np.floating)):
        if np.isnan(value):
            return ""
        if np.isfinite(value) and float(value).is_integer():
            return str(int(value))
    return str(value).strip()


def band_codes(column: Any) -> tuple[np.ndarray, list[str]]:
    """Per-row index into the distinct normalised labels (first-appearance
    order), -1 for a row without a label (lightcurve.py:786-843)."""
    mod = type(column).__module__
    if mod.startswith("pyarrow"):
        cells = np.asarray(column.to_pylist(), dtype=object)
    elif mod.startswith("pandas"):
        cells = np.asarray(column.astype(object).where(column.notna(), None), dtype=object)
    else:
        cells = np.asarray(column, dtype=object)
    names: dict[str, int] = {}
    codes = np.empty(cells.size, dtype=np.int64)
    for i, cell in enumerate(cells.ravel()):
        label = band_label(cell)
        codes[i] = -1 if not label else names.setdefault(label, len(names))
    return codes, list(names)


__all__ = ["adapt_table", "as_float", "band_codes", "band_label", "format_suffix",
           "read_table_object"]
