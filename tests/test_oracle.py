"""The CPU oracle is pinned to the reference: bit-exact on every golden vector the
reference's numba backend produced (tests/golden/make_golden.py)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from _cases import FIELDS, GOLDEN, kernel_golden
from oracle import oracle


@pytest.mark.parametrize("meta_arrays", kernel_golden(), ids=lambda c: c[0]["name"])
def test_oracle_bit_exact_on_golden(meta_arrays):
    meta, a = meta_arrays
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        out = oracle.bls_power(a["t"], a["y"], a["dy"], a["periods"], a["durations"],
                               meta["oversample"], objective=meta["objective"], n_threads=4)
    got = np.stack([out[f] for f in FIELDS])
    assert np.array_equal(got, a["out"], equal_nan=True)


@pytest.mark.parametrize("meta_arrays", kernel_golden(), ids=lambda c: c[0]["name"])
def test_screened_oracle_bit_exact_on_golden(meta_arrays):
    """The screened sweep (the reference's default CPU path, timed as the CPU
    baseline) chooses the unscreened sweep's boxes bit for bit, as the
    reference's own test asserts of its numba kernel (tests/test_bls.py:397-424)."""
    meta, a = meta_arrays
    with np.errstate(over="ignore", divide="ignore", invalid="ignore"):
        out = oracle.bls_power(a["t"], a["y"], a["dy"], a["periods"], a["durations"],
                               meta["oversample"], objective=meta["objective"], n_threads=4,
                               screen=True)
    got = np.stack([out[f] for f in FIELDS])
    assert np.array_equal(got, a["out"], equal_nan=True)


def _method_cases():
    index = json.load(open(os.path.join(GOLDEN, "method_cases.json")))
    z = np.load(os.path.join(GOLDEN, "method_cases.npz"))
    return [(m, z) for m in index]


@pytest.mark.parametrize("case", _method_cases(), ids=lambda c: c[0]["name"])
def test_oracle_method_level_on_golden(case):
    meta, z = case
    k = meta["key"]
    s = oracle.Settings(**meta["settings"])
    periods = z[f"{k}_grid"]
    freq, power, extras = oracle.method_power(z[f"{k}_t"], z[f"{k}_flux"], z[f"{k}_err"],
                                              periods, meta["grid_meta"], s, n_threads=4)
    np.testing.assert_array_equal(freq, z[f"{k}_frequency"])
    np.testing.assert_array_equal(power, z[f"{k}_power"])
    for name in ("depth", "depth_snr", "duration", "t0", "sde"):
        np.testing.assert_array_equal(extras[name], z[f"{k}_x_{name}"])
    i = oracle.best_index(power)
    assert 1.0 / freq[i] == meta["best_period"]


def _multiband_cases():
    index = json.load(open(os.path.join(GOLDEN, "multiband_cases.json")))
    z = np.load(os.path.join(GOLDEN, "multiband_cases.npz"))
    return [(m, z) for m in index]


def multiband_inputs(meta, z):
    """The golden case's bands as ``(name, t, flux, err or None)``."""
    k = meta["key"]
    return [(b, z[f"{k}_{b}_t"], z[f"{k}_{b}_y"], z[f"{k}_{b}_dy"] if has else None)
            for b, has in zip(meta["bands"], meta["with_error"])]


@pytest.mark.parametrize("case", _multiband_cases(), ids=lambda c: c[0]["key"])
def test_oracle_multiband_on_golden(case):
    meta, z = case
    k = meta["key"]
    freq, power, extras, used, n, baseline = oracle.multiband_power(
        multiband_inputs(meta, z), z[f"{k}_periods"], meta["grid_meta"],
        oracle.Settings(objective=meta["objective"]), n_threads=4,
        ephemeris=meta["ephemeris"])
    assert used == meta["used_bands"] and n == meta["n_samples"] and baseline == meta["baseline"]
    np.testing.assert_array_equal(freq, z[f"{k}_frequency"])
    np.testing.assert_array_equal(power, z[f"{k}_power"])
    for name in meta["extras"]:
        np.testing.assert_array_equal(extras[name], z[f"{k}_x_{name}"])
    assert 1.0 / freq[oracle.best_index(power)] == meta["best_period"]
