"""Seeded synthetic light curves shared by the tests (no reference code)."""

from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ("power", "depth", "depth_err", "depth_snr", "duration", "transit_time",
          "log_likelihood")


def kernel_golden():
    """[(meta, arrays)] of the reference's bls_power outputs."""
    index = json.load(open(os.path.join(GOLDEN, "kernel_cases.json")))
    z = np.load(os.path.join(GOLDEN, "kernel_cases.npz"))
    out = []
    for meta in index:
        k = meta["key"]
        out.append((meta, {name: z[f"{k}_{name}"] for name in
                           ("t", "y", "dy", "periods", "durations", "out")}))
    return out


def transit_curve(n, *, span=27.0, period=3.1, depth=3e-3, duration=0.1, noise=1e-3,
                  seed=0, base=2458000.0, weights="uniform", cadence=None):
    """Sorted times over ``span`` days with box dips and Gaussian noise.

    ``weights``: "uniform" (dy = noise everywhere), "hetero" (dy varies by ~3x),
    "wild" (dy spans two decades).
    """
    rng = np.random.default_rng(seed)
    if cadence is None:
        t = np.sort(rng.uniform(0.0, span, n))
    else:
        t = np.arange(n) * cadence
        t = t[t < span] if t[-1] >= span else t
    t = t + base
    flux = 1.0 + rng.normal(0.0, noise, t.size)
    phase0 = rng.uniform(0.0, period)
    flux[np.mod(t - base - phase0, period) < duration] -= depth
    if weights == "uniform":
        dy = np.full(t.size, noise)
    elif weights == "hetero":
        dy = noise * rng.uniform(0.6, 1.8, t.size)
    else:
        dy = noise * 10.0 ** rng.uniform(-1.0, 1.0, t.size)
    return t, flux, dy


def compare(ref: dict, got: dict, *, rtol=1e-6, box_agree=0.99):
    """Parity of two per-period outputs: powers within ``rtol`` (plus an absolute
    floor of rtol * max|power| for near-zero powers), identical -inf pattern, the
    same chosen box on at least ``box_agree`` of the periods, depth within rtol
    where the box agrees.  Returns a dict of diagnostics."""
    rp, gp = np.asarray(ref["power"]), np.asarray(got["power"])
    assert rp.shape == gp.shape
    ninf_r, ninf_g = np.isneginf(rp), np.isneginf(gp)
    assert np.array_equal(ninf_r, ninf_g), "admissibility (-inf pattern) differs"
    fin = np.isfinite(rp)
    diag = {"n": int(rp.size), "finite": int(fin.sum())}
    if fin.any():
        scale = float(np.max(np.abs(rp[fin])))
        err = np.abs(gp[fin] - rp[fin])
        tol = rtol * np.abs(rp[fin]) + rtol * scale * 1e-3
        diag["max_rel_err"] = float(np.max(err / np.maximum(np.abs(rp[fin]), 1e-300)))
        assert np.all(err <= tol), f"power differs: max err {err.max()} (rel {diag['max_rel_err']})"
        same_box = (np.asarray(ref["duration"]) == np.asarray(got["duration"])) & np.isclose(
            np.asarray(ref["transit_time"]), np.asarray(got["transit_time"]), rtol=0.0, atol=1e-9)
        diag["box_agree"] = float(same_box[fin].mean())
        assert diag["box_agree"] >= box_agree, f"box agreement {diag['box_agree']}"
        rd, gd = np.asarray(ref["depth"]), np.asarray(got["depth"])
        m = fin & same_box
        if m.any():
            dscale = float(np.max(np.abs(rd[m]))) or 1.0
            assert np.all(np.abs(gd[m] - rd[m]) <= rtol * np.abs(rd[m]) + 1e-9 * dscale)
        diag["same_argmax"] = int(np.argmax(np.where(fin, gp, -np.inf))) == int(
            np.argmax(np.where(fin, rp, -np.inf)))
    return diag
