"""Train the period-proposal network (``python -m cuperiod_b200.proposal_train``).

No counterpart in the reference.  Steps, all on one GPU:

1. seeded training curves (:func:`cuperiod_b200.synthetic.proposal_curves`: the
   batched workload's cadence and noise, 60% box transits, 40% noise of which
   half carry a sinusoid), 4096 at a time;
2. labels: each curve's plain full-grid BLS best period (the engine's search
   over the 50,000-period grid of 0.3-13 d, default durations), as its class
   among 1024 log-period bins;
3. inputs: each curve binned to 4096 time bins (``pn_bin_curves``), kept on the
   device;
4. training: the network's tensor-core forward and backward passes, Adam with
   decoupled weight decay and a cosine learning-rate decay, cross-entropy with
   10% of the target on each neighbouring class, half of every batch reversed
   in time (a time-reversed curve has the same BLS spectrum, so the same label);
5. calibration on held-out curves: the confidence threshold (probability mass of
   the top-k classes) above which a curve's windows -- its top-k classes, each
   widened by one neighbour -- hold its best period for all but
   ``--miss-rate`` of all held-out curves; below it the pruned search falls back
   to the full grid.

The weights, the threshold and the training record go to ``--out`` (npz).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import _lib
from .bls import _grid_segments
from .grid import GridSpec
from .proposal import (IN_CHANNELS, N_BINS, ProposalNet, Weights, class_edges, device_curves,
                       labels_of, window_mask, windows_hold)
from .settings import BLSSettings
from .synthetic import batched_periods, proposal_curves

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "proposal_weights.npz")


def grid_segments():
    """The batched workload's grid: 50,000 log periods over 0.3-13 d in the
    default segments."""
    return _grid_segments(GridSpec(kind="period", values=batched_periods()), BLSSettings())


def build_dataset(n_curves: int, seed: int, engine, segments, chunk: int = 4096):
    """Binned inputs (device, bf16) and labels (host) of ``n_curves`` curves."""
    import torch
    grid = _lib.PackedGrid.from_segments(segments, 10, 0)
    n_periods = grid.n_periods
    x = torch.empty((n_curves, N_BINS, IN_CHANNELS), dtype=torch.bfloat16, device="cuda")
    labels = np.empty(n_curves, dtype=np.int32)
    best = np.empty(n_curves, dtype=np.int64)
    ops = None
    for a in range(0, n_curves, chunk):
        m = min(chunk, n_curves - a)
        curves = [(c.t, c.y, None) for c in proposal_curves(m, seed=seed + a)]
        engine.prepare(grid, _lib.PackedCurves.from_arrays(curves))
        engine.launch()
        bi = engine.download_best()[0]
        best[a:a + m] = bi
        labels[a:a + m] = labels_of(bi, n_periods)
        t, y, off = device_curves(curves)
        if ops is None:
            from .proposal import Ops
            ops = Ops()
        ops.bin_curves(t, y, off, m, x[a:a + m])
    ops.check()
    return x, labels, best


def window_hits(idx: np.ndarray, labels: np.ndarray, widen: int) -> np.ndarray:
    """Whether each label class lies inside the windows of its top-k classes."""
    d = np.abs(idx.astype(np.int64) - labels[:, None].astype(np.int64))
    return (d <= widen).any(axis=1)


def calibrate(mass: np.ndarray, hits: np.ndarray, miss_rate: float) -> float:
    """The smallest threshold whose confident curves (mass >= threshold) miss
    their label class in at most miss_rate of all curves."""
    order = np.argsort(-mass, kind="stable")
    misses = np.cumsum(~hits[order])
    ok = np.flatnonzero(misses <= miss_rate * mass.size)
    if ok.size == 0:
        return float("inf")
    return float(mass[order[int(ok[-1])]])


def train(args) -> dict:
    import torch
    torch.manual_seed(args.seed)
    segments = grid_segments()
    engine = _lib.Engine()
    t0 = time.perf_counter()
    x, labels, _ = build_dataset(args.curves + args.val, args.seed, engine, segments)
    t_data = time.perf_counter() - t0
    n_tr = args.curves
    net = ProposalNet(Weights.init(seed=args.seed), train=True)
    steps_per_epoch = n_tr // args.batch
    total = steps_per_epoch * args.epochs
    lab_dev = torch.from_numpy(labels).to("cuda")
    rng = np.random.default_rng(args.seed)
    history = []
    step = 0
    t1 = time.perf_counter()
    for epoch in range(args.epochs):
        perm = torch.from_numpy(rng.permutation(n_tr)).to("cuda")
        loss_sum = torch.zeros(1, device="cuda")
        for s in range(steps_per_epoch):
            sel = perm[s * args.batch:(s + 1) * args.batch]
            xb = x.index_select(0, sel)
            lb = lab_dev.index_select(0, sel)
            if args.flip:
                # time reversal leaves a curve's BLS spectrum, so its label, unchanged
                half = args.batch // 2
                xb[:half] = xb[:half].flip(1)
            lr = args.lr_min + 0.5 * (args.lr - args.lr_min) * (1 + math.cos(math.pi * step / total))
            logits = net.forward(xb)
            d, loss = net.loss_and_grad(logits, lb, side=args.side)
            net.zero_grad()
            net.backward(d)
            net.adam(lr, wd=args.wd)
            loss_sum += loss
            step += 1
        net.ops.check()
        history.append(float(loss_sum.item()) / (steps_per_epoch * args.batch))
        print(f"epoch {epoch + 1}/{args.epochs} loss {history[-1]:.4f}", flush=True)
    t_train = time.perf_counter() - t1
    # held-out curves: recall of the windows and the confidence threshold
    net.train = False
    idx, mass = [], []
    for a in range(n_tr, n_tr + args.val, 1024):
        logits = net.forward(x[a:min(a + 1024, n_tr + args.val)])
        i, m = net.topk(logits, args.k)
        idx.append(i.cpu().numpy())
        mass.append(m.cpu().numpy())
    idx = np.concatenate(idx)
    mass = np.concatenate(mass)
    val_labels = labels[n_tr:]
    hits = window_hits(idx, val_labels, args.widen)
    thr = calibrate(mass, hits, args.miss_rate)
    conf = mass >= thr
    top1 = float(np.mean(idx[:, 0] == val_labels))
    edges = class_edges(sum(p.size for p, _ in segments))
    frac_searched = float(np.mean([sum(hi - lo for lo, hi in window_mask(r, edges, args.widen))
                                   for r in idx[:256]]) / edges[-1])
    meta = {"k": args.k, "widen": args.widen, "threshold": thr,
            "train_curves": n_tr, "val_curves": args.val, "epochs": args.epochs,
            "batch": args.batch, "seed": args.seed, "wd": args.wd, "flip": args.flip,
            "loss_history": history,
            "val_top1": top1, "val_window_recall": float(hits.mean()),
            "val_confident_frac": float(conf.mean()),
            "val_confident_recall": float(hits[conf].mean()) if conf.any() else None,
            "val_agreement_bound": float(1.0 - np.sum(conf & ~hits) / conf.size),
            "window_period_fraction": frac_searched,
            "seconds": {"data": round(t_data, 1), "train": round(t_train, 1)},
            "grid": "50,000 log periods 0.3-13 d, default segments and durations"}
    net.weights(meta).save(args.out)
    engine.close()
    return meta


def calibrate_batch(weights_path: str, n_curves: int, seed: int, agreement: float) -> dict:
    """The confidence threshold for the batched workload: ``n_curves`` curves of
    its generator (``synthetic.batched_curves``, a seed apart from any benchmark
    batch) searched over the full grid, then ranked by the network; the
    threshold is the smallest at which the confident curves whose full-grid best
    period falls outside their windows stay within ``1 - agreement`` of all
    curves.  Written to the weights' meta as ``threshold_batch`` with a record;
    the training-distribution threshold (``threshold``) is kept."""
    from .proposal import Proposer
    from .synthetic import batched_curves
    segments = grid_segments()
    w = Weights.load(weights_path)
    engine = _lib.Engine()
    curves = [(c.t, c.y, c.dy) for c in batched_curves(n_curves, seed=seed)]
    packed = _lib.PackedCurves.from_arrays(curves)
    grid = _lib.PackedGrid.from_segments(segments, 10, 0)
    engine.prepare(grid, packed)
    engine.launch()
    best = np.asarray(engine.download_best()[0], dtype=np.int64)
    prop = Proposer(w, segments, threshold=0.0)
    idx, mass = prop.propose_packed(packed.t, packed.y, packed.offsets)
    hit = windows_hold(idx, best, prop.edges, prop.widen)
    window = float(np.mean([sum(hi - lo for lo, hi in window_mask(r, prop.edges, prop.widen))
                            for r in idx[:256]]) / prop.edges[-1])

    def at(thr: float) -> dict:
        conf = mass >= thr
        return {"threshold": float(thr), "confident_frac": float(conf.mean()),
                "agreement_bound": float(1.0 - np.mean(conf & ~hit)),
                "periods_searched_frac": float(1.0 - conf.mean() * (1.0 - window))}
    thr = calibrate(mass, hit, 1.0 - agreement)
    record = {"curves": n_curves, "seed": seed, "target_agreement": agreement, **at(thr),
              "window_hit_frac": float(hit.mean()),
              "table": [at(calibrate(mass, hit, 1.0 - a)) for a in (0.999, 0.998, 0.995, 0.99)]}
    w.meta["threshold_batch"] = float(thr)
    w.meta["batch_calibration"] = record
    w.save(weights_path, compact=True)
    engine.close()
    return record


def main(argv=None) -> None:
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--curves", type=int, default=65536, help="training curves")
    p.add_argument("--val", type=int, default=4096, help="held-out curves")
    p.add_argument("--epochs", type=int, default=24)
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--lr", type=float, default=2e-3)
    p.add_argument("--lr-min", type=float, default=2e-5)
    p.add_argument("--wd", type=float, default=0.05)
    p.add_argument("--side", type=float, default=0.1)
    p.add_argument("--k", type=int, default=16)
    p.add_argument("--widen", type=int, default=1)
    p.add_argument("--miss-rate", type=float, default=0.005)
    p.add_argument("--seed", type=int, default=1000003)
    p.add_argument("--flip", type=int, default=1, help="time-reversal augmentation (0: off)")
    p.add_argument("--out", default=DEFAULT_OUT)
    p.add_argument("--calibrate-batch", type=int, default=0, metavar="N",
                   help="instead of training: set the batched workload's threshold on N "
                        "curves of its generator (weights at --out)")
    p.add_argument("--calib-seed", type=int, default=424242)
    p.add_argument("--agreement", type=float, default=0.995)
    args = p.parse_args(argv)
    if args.calibrate_batch > 0:
        rec = calibrate_batch(args.out, args.calibrate_batch, args.calib_seed, args.agreement)
        print(json.dumps(rec), flush=True)
        return
    meta = train(args)
    print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}), flush=True)


if __name__ == "__main__":
    main()
