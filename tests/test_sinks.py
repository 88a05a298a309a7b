"""Result-row sinks (cuPeriod src/cuperiod/batch/io.py:574-674): Parquet and CSV by
suffix, the union of the rows' columns, write-then-rename through an exclusively
created temporary file, formula-safe CSV text, no array columns in CSV."""

from __future__ import annotations

import csv
import os

import pytest

from cuperiod_b200.sinks import csv_safe, union_columns, write_rows

ROWS = [{"key": "a", "best_period": 1.5, "power": 3.0},
        {"key": "=cmd()", "best_period": 2.5, "extra": -5.0},
        {"key": "-7", "power": None}]


def test_union_columns_first_seen_order():
    assert union_columns(ROWS) == ["key", "best_period", "power", "extra"]


@pytest.mark.parametrize("value,expected", [
    ("=SUM(A1)", "'=SUM(A1)"), ("+x", "'+x"), ("-x", "'-x"), ("@x", "'@x"),
    ("\tx", "'\tx"), ("\rx", "'\rx"), ("-5", "-5"), ("+7", "+7"), ("1e3", "1e3"),
    ("plain", "plain"), ("", ""), (-5.0, -5.0), (None, None)])
def test_csv_safe(value, expected):
    assert csv_safe(value) == expected
    assert csv_safe(csv_safe(value)) == expected


def test_parquet_round_trip(tmp_path):
    import pyarrow.parquet as pq
    path = tmp_path / "sub" / "rows.parquet"
    write_rows(ROWS, path)
    table = pq.read_table(path).to_pylist()
    assert [r["key"] for r in table] == ["a", "=cmd()", "-7"]
    assert table[0]["extra"] is None and table[2]["best_period"] is None
    assert table[1]["extra"] == -5.0
    assert sorted(os.listdir(path.parent)) == ["rows.parquet"]     # no temporary left


def test_csv_round_trip_and_formula_guard(tmp_path):
    path = tmp_path / "rows.csv"
    write_rows(ROWS, path)
    with open(path, newline="", encoding="utf-8") as fh:
        got = list(csv.DictReader(fh))
    assert list(got[0]) == ["key", "best_period", "power", "extra"]
    assert got[1]["key"] == "'=cmd()" and got[2]["key"] == "-7"
    assert got[0]["extra"] == "" and got[1]["extra"] == "-5.0"


def test_overwrites_atomically_and_never_through_a_symlink(tmp_path):
    path = tmp_path / "rows.parquet"
    write_rows(ROWS[:1], path)
    write_rows(ROWS, path)                         # replaced, not appended
    import pyarrow.parquet as pq
    assert pq.read_table(path).num_rows == 3
    victim = tmp_path / "victim.csv"
    victim.write_text("keep")
    link = tmp_path / "link.csv"
    link.symlink_to(victim)
    write_rows(ROWS, link)                         # the link is replaced, not followed
    assert victim.read_text() == "keep"
    assert not link.is_symlink()


def test_rejections(tmp_path):
    with pytest.raises(ValueError, match="unsupported sink format"):
        write_rows(ROWS, tmp_path / "rows.json")
    with pytest.raises(ValueError, match="array-valued"):
        write_rows([{"key": "a", "spectrum": [1.0, 2.0]}], tmp_path / "rows.csv")
    assert not any(p.name.endswith(".tmp") for p in tmp_path.iterdir())

