"""Light-curve tables: column detection, domain, error pairing and band split
against the reference's readers (tests/golden/make_golden_tables.py), for
DataFrames and for the same tables written as Parquet and CSV files."""

from __future__ import annotations

import json
import math
import os
import warnings

import numpy as np
import pytest

from _cases import GOLDEN

CASES = json.load(open(os.path.join(GOLDEN, "tables_cases.json")))


def _arr(x):
    return None if x is None else np.array([np.nan if v is None else v for v in x], dtype=float)


def _same(lc, want):
    np.testing.assert_array_equal(lc.time, _arr(want["time"]))
    np.testing.assert_array_equal(lc.value, _arr(want["value"]))
    if want["error"] is None:
        assert lc.error is None
    else:
        np.testing.assert_array_equal(lc.error, _arr(want["error"]))
    assert lc.domain.value == want["domain"]


def _read(case, source, tmp_path):
    import pandas as pd
    from cuperiod_b200.columns import ColumnMap
    from cuperiod_b200.lightcurve import LightCurve, MultiBandLightCurve
    df = pd.DataFrame(case["columns"])
    kw = dict(case["kwargs"])
    if "columns" in kw:
        kw["columns"] = ColumnMap(**kw["columns"])
    cls = MultiBandLightCurve if case["kind"] == "multi" else LightCurve
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        if source == "frame":
            return cls.from_dataframe(df, **kw)
        path = tmp_path / f"{case['name']}.{source}"
        if source == "parquet":
            if case["name"] == "band_labels":       # mixed-type labels: not a Parquet column
                pytest.skip("mixed-type band labels have no Parquet type")
            df.to_parquet(path)
        else:
            df.to_csv(path, index=False)
        return cls.from_file(path, **kw)


@pytest.mark.parametrize("source", ["frame", "parquet", "csv"])
@pytest.mark.parametrize("case", CASES, ids=lambda c: c["name"])
def test_tables_read_like_the_reference(case, source, tmp_path):
    got = _read(case, source, tmp_path)
    want = case["result"]
    if case["kind"] == "multi":
        assert list(got.bands) == list(want["bands"])
        for name, lc in got.bands.items():
            _same(lc, want["bands"][name])
    else:
        _same(got, want)
        if source != "frame":
            assert got.meta["source"].endswith(f"{case['name']}.{source}")


def test_compressed_csv_and_missing_columns(tmp_path):
    import pandas as pd
    from cuperiod_b200.errors import ColumnResolutionError
    from cuperiod_b200.lightcurve import LightCurve
    df = pd.DataFrame({"btjd": [1.0, 2.0], "sap_flux": [3.0, 4.0], "sap_flux_err": [0.1, 0.2]})
    df.to_csv(tmp_path / "x.csv.gz", index=False)
    lc = LightCurve.from_file(tmp_path / "x.csv.gz")
    assert lc.domain.value == "flux" and np.array_equal(lc.error, [0.1, 0.2])
    with pytest.raises(ColumnResolutionError):
        LightCurve.from_dataframe(pd.DataFrame({"a": [1.0], "b": [2.0]}))


def test_batch_inputs_resolve_like_the_reference(tmp_path):
    import pandas as pd
    from cuperiod_b200.batch import _load, resolve_inputs
    from cuperiod_b200.lightcurve import LightCurve, MultiBandLightCurve
    t = np.arange(30.0)
    df = pd.DataFrame({"obj": ["a"] * 10 + ["b"] * 20, "mjd": t, "flux": 1.0 + 0 * t,
                       "flux_err": 0.1 + 0 * t, "band": ["g", "r"] * 15})
    items = resolve_inputs((df, "obj"))
    assert [k for k, _ in items] == ["a", "b"] and isinstance(items[1][1], LightCurve)
    items = resolve_inputs((df, "obj"), band_column="band")
    assert isinstance(items[0][1], MultiBandLightCurve) and items[0][1].band_names == ("g", "r")
    (tmp_path / "f1").mkdir()
    (tmp_path / "f2").mkdir()
    for d in ("f1", "f2"):
        df.to_csv(tmp_path / d / "lc.csv", index=False)
    df.to_parquet(tmp_path / "f1" / "star.parquet")
    items = resolve_inputs(tmp_path / "f1")
    assert sorted(k for k, _ in items) == ["lc", "star"]
    items = resolve_inputs(str(tmp_path / "f*" / "lc.csv"))
    assert [k for k, _ in items] == ["lc", "lc#2"]
    lc = _load(items[1][1], None, None, None)
    assert isinstance(lc, LightCurve) and lc.n == 30 and lc.domain.value == "flux"
    mb = _load(items[0][1], None, None, "band")
    assert isinstance(mb, MultiBandLightCurve) and mb.bands["g"].n == 15
    with pytest.raises(FileNotFoundError):
        resolve_inputs(str(tmp_path / "nothing*.csv"))
