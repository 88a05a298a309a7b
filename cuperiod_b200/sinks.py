"""Writing batch result rows to disk (cuPeriod src/cuperiod/batch/io.py:574-674).

Parquet (``.parquet``, ``.pq``) or CSV (``.csv``) by the path's suffix.  The
columns are the union of the rows' keys in first-seen order (a row without a
column gets a null).  The table goes to a new temporary file next to the target
-- created exclusively, so an existing file or a symlink planted under that
name is never written through, and dot-prefixed so a dataset reader of the
directory skips a leftover -- and is then renamed over the target, so a reader
never sees half a file.  CSV text cells that a spreadsheet would evaluate as a
formula get a leading quote; CSV cannot hold array-valued columns.
"""

from __future__ import annotations

import csv
import os
import secrets
from pathlib import Path
from typing import Any, Mapping, Sequence

#: First characters that make a spreadsheet treat a text cell as a formula.
FORMULA_PREFIXES = ("=", "+", "-", "@", "\t", "\r")


def union_columns(rows: Sequence[Mapping[str, Any]]) -> list[str]:
    """Every key of every row, in the order first seen."""
    seen: dict[str, None] = {}
    for row in rows:
        for key in row:
            seen.setdefault(key, None)
    return list(seen)


def temp_path(path: Path) -> Path:
    """A fresh dot-prefixed sibling of ``path`` (process id and random tag)."""
    return path.with_name(f".{path.name}.{os.getpid()}.{secrets.token_hex(4)}.tmp")


def _replace(tmp: Path, path: Path) -> None:
    try:
        os.replace(tmp, path)
    except OSError as exc:
        raise type(exc)(f"could not replace {path} ({exc}); the complete result is kept "
                        f"in {tmp}") from exc


def csv_safe(value: Any) -> Any:
    """A text cell starting like a formula, prefixed with a quote; numbers such as
    ``-5`` and non-text values unchanged.  Applying it twice changes nothing more."""
    if isinstance(value, str) and value and value[0] in FORMULA_PREFIXES:
        try:
            float(value)
        except ValueError:
            return "'" + value
    return value


def _write_parquet(rows: Sequence[Mapping[str, Any]], path: Path) -> None:
    import pyarrow as pa
    import pyarrow.parquet as pq

    columns = union_columns(rows)
    table = pa.table({col: [row.get(col) for row in rows] for col in columns})
    tmp = temp_path(path)
    try:
        with tmp.open("xb") as fh:
            pq.write_table(table, fh)
    except BaseException:
        tmp.unlink(missing_ok=True)
        raise
    _replace(tmp, path)


def _write_csv(rows: Sequence[Mapping[str, Any]], path: Path) -> None:
    columns = union_columns(rows)
    arrays = [c for c in columns if any(isinstance(row.get(c), list) for row in rows)]
    if arrays:
        raise ValueError(f"CSV sink cannot store array-valued columns {arrays}; use a "
                         ".parquet sink")
    tmp = temp_path(path)
    try:
        with tmp.open("x", newline="", encoding="utf-8") as fh:
            out = csv.DictWriter(fh, fieldnames=columns, extrasaction="ignore")
            out.writeheader()
            out.writerows({c: csv_safe(v) for c, v in row.items()} for row in rows)
    except BaseException:
        tmp.unlink(missing_ok=True)
        raise
    _replace(tmp, path)


def write_rows(rows: Sequence[Mapping[str, Any]], path: str | os.PathLike) -> None:
    """Write result rows to ``path`` (Parquet or CSV by suffix), creating the
    parent directory; any other suffix is a ValueError."""
    path = Path(path)
    suffix = path.suffix.lower()
    if suffix not in {".parquet", ".pq", ".csv"}:
        raise ValueError(f"unsupported sink format {path.suffix!r}; use .parquet or .csv")
    path.parent.mkdir(parents=True, exist_ok=True)
    if suffix == ".csv":
        _write_csv(rows, path)
    else:
        _write_parquet(rows, path)


__all__ = ["FORMULA_PREFIXES", "csv_safe", "union_columns", "write_rows"]
