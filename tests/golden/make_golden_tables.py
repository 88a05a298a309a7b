"""Generate light-curve table golden cases from the reference's own readers.

Run once in a container that holds the reference source (the committed
``tables_cases.json`` is what the tests read)::

    PYTHONPATH=<reference>/src python tests/golden/make_golden_tables.py

Each case is a small table in a survey's column convention, read by
``LightCurve.from_dataframe`` or ``MultiBandLightCurve.from_dataframe``
(``src/cuperiod/core/lightcurve.py:143-158, 389-518``, column resolution
``src/cuperiod/core/columns.py:280-375``), with the resolved arrays, domain and
bands the reference produced.
"""

from __future__ import annotations

import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

T = [2459000.1, 2459000.3, 2459000.7, 2459001.2, 2459001.9, 2459002.4]


def cases():
    yield "tess", {"TIME": T, "PDCSAP_FLUX": [1.0, 0.99, 1.01, 1.0, 0.98, 1.0],
                   "PDCSAP_FLUX_ERR": [0.01] * 6, "SAP_FLUX": [2.0] * 6,
                   "SAP_FLUX_ERR": [0.5] * 6}, {}, None
    atlas = {"MJD": T, "m": [15.0, 15.1, 15.0, 14.9, 15.2, 15.0], "dm": [0.02] * 6,
             "uJy": [300.0, 290.0, 310.0, 305.0, 280.0, 300.0], "duJy": [5.0] * 6,
             "F": ["c", "o", "c", "o", "c", "o"]}
    yield "atlas", atlas, {}, None
    yield "atlas_magnitude", atlas, {"domain": "magnitude"}, None
    asassn = {"HJD": T, "mag": [12.0, 12.1, 12.0, 12.2, 12.0, 11.9], "mag_err": [0.03] * 6,
              "flux": [5.0, 4.9, 5.0, 4.8, 5.0, 5.1], "flux_err": [0.1] * 6}
    yield "asassn", asassn, {}, None
    yield "asassn_magnitude", asassn, {"domain": "magnitude"}, None
    yield "case_insensitive", {"Time": T, "Flux": [1.0] * 6, "Sigma": [0.2] * 6}, {}, None
    yield "no_error", {"jd": T, "vmag": [9.0, 9.1, 9.0, 9.2, 9.1, 9.0]}, {}, None
    yield "explicit_map", {"t0": T, "val": [3.0] * 6, "sig": [0.1] * 6, "flux": [1.0] * 6}, \
        {"columns": {"time": "t0", "value": "val", "error": "sig"}, "domain": "flux"}, None
    yield "ztf_multiband", {"mjd": T, "mag": [18.0, 18.2, 18.1, 18.3, 18.0, 18.4],
                            "magerr": [0.05] * 6,
                            "filtercode": ["zg", "zr", "zg", "zr", "zi", "zg"]}, {}, "multi"
    yield "gaia_multiband", {"time": T, "flux": [10.0, 9.0, 11.0, 10.5, 9.5, 10.0],
                             "flux_error": [0.1] * 6,
                             "band": ["G", "BP", "RP", "G", "BP", "RP"]}, {}, "multi"
    yield "band_labels", {"hjd": T, "mag": [10.0] * 6, "err": [0.1] * 6,
                          "filter": [1, 1.0, "1", " 2", None, float("nan")]}, {}, "multi"


def _enc(a):
    return None if a is None else [None if (isinstance(x, float) and math.isnan(x)) else x
                                   for x in a.tolist()]


def main() -> None:
    import warnings

    import pandas as pd
    from cuperiod.core.columns import ColumnMap
    from cuperiod.core.lightcurve import LightCurve, MultiBandLightCurve

    out = []
    for name, cols, kw, kind in cases():
        df = pd.DataFrame(cols)
        args = dict(kw)
        if "columns" in args:
            args["columns"] = ColumnMap(**args["columns"])
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            if kind == "multi":
                mb = MultiBandLightCurve.from_dataframe(df, **args)
                result = {"bands": {k: {"time": _enc(lc.time), "value": _enc(lc.value),
                                        "error": _enc(lc.error), "domain": lc.domain.value}
                                    for k, lc in mb.bands.items()}}
            else:
                lc = LightCurve.from_dataframe(df, **args)
                result = {"time": _enc(lc.time), "value": _enc(lc.value),
                          "error": _enc(lc.error), "domain": lc.domain.value}
        out.append({"name": name, "columns": cols, "kwargs": kw, "kind": kind or "single",
                    "result": result})
    with open(os.path.join(HERE, "tables_cases.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main()
