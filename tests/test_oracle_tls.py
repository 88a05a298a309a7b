"""The oracle's TLS restatement against the reference's own numba output
(tests/golden/make_golden_tls.py): every output bit for bit, the default
period grid and the template."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from _cases import GOLDEN
from oracle import oracle

DEFAULTS = {"n_phase_bins": 256, "duration_min_frac": 0.01, "duration_max_frac": 0.10,
            "n_durations": 5, "limb_dark_u1": 0.4, "limb_dark_u2": 0.3}


def tls_cases():
    index = json.load(open(os.path.join(GOLDEN, "tls_cases.json")))
    z = np.load(os.path.join(GOLDEN, "tls_cases.npz"))
    return [(m, z) for m in index]


def case_inputs(meta, z):
    k = meta["key"]
    s = {**DEFAULTS, **meta["settings"]}
    dy = z[f"{k}_dy"] if meta["with_error"] else None
    return z[f"{k}_t"], z[f"{k}_y"], dy, z[f"{k}_periods"], s


@pytest.mark.parametrize("case", tls_cases(), ids=lambda c: c[0]["key"])
def test_oracle_tls_on_golden(case):
    meta, z = case
    t, y, dy, periods, s = case_inputs(meta, z)
    out = oracle.tls_power(t, y, dy, periods, n_bins=s["n_phase_bins"],
                           duration_min_frac=s["duration_min_frac"],
                           duration_max_frac=s["duration_max_frac"],
                           n_durations=s["n_durations"], u1=s["limb_dark_u1"],
                           u2=s["limb_dark_u2"], n_threads=4)
    for name in meta["outputs"]:
        np.testing.assert_array_equal(out[name], z[f"{meta['key']}_{name}"], err_msg=name)


@pytest.mark.parametrize("case", [c for c in tls_cases() if c[0]["default_grid"]],
                         ids=lambda c: c[0]["key"])
def test_oracle_tls_default_grid(case):
    meta, z = case
    t, _, _, periods, s = case_inputs(meta, z)
    grid = oracle.tls_period_grid(float(t.max() - t.min()), min_period=0.5, max_period=100.0,
                                  min_transits=2, grid_duration_frac=0.05,
                                  duration_min_frac=s["duration_min_frac"], oversample=2)
    np.testing.assert_array_equal(grid, periods)


def test_template_and_duration_bins_known_answers():
    # _duration_bins of the defaults: round(256 * geomspace(0.01, 0.1, 5))
    assert oracle.tls_duration_bins(256, 0.01, 0.10, 5) == [3, 5, 8, 14, 26]
    # widths are clamped to [1, n_bins - 1], never empty
    assert oracle.tls_duration_bins(16, 1e-4, 2e-4, 3) == [1]
    g = oracle.tls_template(9, 0.4, 0.3)
    assert g.max() == 1.0 and g[4] == 1.0 and np.all(g[:4] == g[::-1][:4]) and g[0] > 0
    np.testing.assert_array_equal(oracle.tls_template(1, 0.4, 0.3), [1.0])
