"""Learned period proposals: a small 1D convolutional network that ranks
log-period windows of the full BLS grid, so that the exact search runs only
there.

No counterpart in the reference (cuPeriod searches every trial period).  The
network reads each light curve binned into 4096 time bins over its own span
(bf16: the bin's standardised mean flux and an occupancy flag), applies six
convolutions (64 channels, width 7, stride 2, ReLU: 4096 -> 64 positions) and a
two-layer MLP (4096 -> 256 -> 1024, ReLU between) giving logits over 1024
log-period bins of the grid.  Every contraction runs on the tensor cores
through the library's tcgen05 GEMM (``pn_gemm``, bf16 operands, fp32
accumulation); training (cross-entropy against the full-grid BLS argmax bin,
Adam on fp32 master weights) uses the same kernels for the backward pass.
PyTorch only holds the device buffers.

:class:`Proposer` is the learned-pruned BLS: the top-k bins (each widened
by its neighbours) of every confident curve are searched exactly at the full
grid's resolution, with the full grid's segment durations, so a window that
holds the full grid's best period returns that period; curves whose top-k
probability mass is below the threshold are searched over the full grid.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib

N_BINS = 4096           # time bins of the network's input
CHANNELS = 64
N_CONV = 6
WIDTH = 7
HIDDEN = 256
N_CLASSES = 1024        # log-period bins of the grid
IN_CHANNELS = 2

_p, _i32, _i64, _f32 = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float
_bound = False


def _lib_pn() -> ctypes.CDLL:
    global _bound
    lib = _lib.load()
    if not _bound:
        lib.pn_gemm.argtypes = [_p, _i64, _p, _i64, _i32, _i32, _i32, _i32, _p, _i64, _i32, _i32,
                                _p, _i32, _p, _p, _p]
        lib.pn_bin_curves.argtypes = [_p, _p, _p, _i32, _i32, _p, _p]
        lib.pn_im2col.argtypes = [_p, _p, _i32, _i32, _i32, _i32, _p]
        lib.pn_col2im.argtypes = [_p, _p, _p, _i32, _i32, _i32, _i32, _p]
        lib.pn_transpose.argtypes = [_p, _i64, _p, _i64, _i64, _i64, _p]
        lib.pn_colsum.argtypes = [_p, _i64, _i64, _i32, _p, _p]
        lib.pn_softmax_xent.argtypes = [_p, _i32, _i32, _p, _f32, _f32, _p, _p, _p]
        lib.pn_adam.argtypes = [_p, _p, _p, _p, _p, _i64, _f32, _f32, _f32, _f32, _f32, _i32, _p]
        lib.pn_topk.argtypes = [_p, _i32, _i32, _i32, _p, _p, _p]
        for name in ("pn_gemm", "pn_bin_curves", "pn_im2col", "pn_col2im", "pn_transpose",
                     "pn_colsum", "pn_softmax_xent", "pn_adam", "pn_topk"):
            getattr(lib, name).restype = ctypes.c_int
        _bound = True
    return lib


def _ok(rc: int, what: str) -> None:
    if rc != 0:
        raise _lib.EngineError(f"{what} failed (code {rc})")


def _ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())


def _bf16_bits(a: np.ndarray) -> np.ndarray:
    """fp32 values rounded to bf16 (nearest, ties to even), as uint16 bits."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


class _null:
    def __enter__(self):
        return None

    def __exit__(self, *exc):
        return False


def kp(layer: int) -> int:
    """Patch width (GEMM K) of convolution ``layer``: 7 taps x input channels,
    padded to a multiple of 8."""
    c = IN_CHANNELS if layer == 0 else CHANNELS
    return (WIDTH * c + 7) // 8 * 8


class Ops:
    """The library's device steps on torch tensors (all on one stream)."""

    def __init__(self, stream=None):
        import torch
        self.torch = torch
        self.lib = _lib_pn()
        self.stream = stream
        with torch.cuda.stream(stream) if stream is not None else _null():
            self.err = torch.zeros(1, dtype=torch.int32, device="cuda")

    @property
    def _st(self):
        return None if self.stream is None else self.stream.cuda_stream

    def gemm(self, A, B, out, *, M, N, K, lda, ldb, ldo, mode=0, transpose=False, bias=None,
             relu=False, mask=None, splits=1):
        _ok(self.lib.pn_gemm(_ptr(A), lda, _ptr(B), ldb, M, N, K, splits, _ptr(out), ldo, mode,
                             int(transpose), _ptr(bias), int(relu), _ptr(mask), _ptr(self.err),
                             self._st), "pn_gemm")

    def im2col(self, X, A, B, L_in, C, k):
        _ok(self.lib.pn_im2col(_ptr(X), _ptr(A), B, L_in, C, k, self._st), "pn_im2col")

    def col2im(self, dcol, act, dX, B, L_in, C, k):
        _ok(self.lib.pn_col2im(_ptr(dcol), _ptr(act), _ptr(dX), B, L_in, C, k, self._st),
            "pn_col2im")

    def transpose(self, x, ld_in, out, ld_out, R, C):
        _ok(self.lib.pn_transpose(_ptr(x), ld_in, _ptr(out), ld_out, R, C, self._st),
            "pn_transpose")

    def colsum(self, g, ld, M, N, db):
        _ok(self.lib.pn_colsum(_ptr(g), ld, M, N, _ptr(db), self._st), "pn_colsum")

    def bin_curves(self, t, y, offsets, n_curves, out):
        _ok(self.lib.pn_bin_curves(_ptr(t), _ptr(y), _ptr(offsets), n_curves, N_BINS, _ptr(out),
                                   self._st), "pn_bin_curves")

    def check(self) -> None:
        if self.stream is None:
            self.torch.cuda.synchronize()
        else:
            self.stream.synchronize()
        if int(self.err.item()) != 0:
            raise _lib.EngineError("a tensor-core GEMM of the proposal network timed out")


@dataclass
class Weights:
    """fp32 master weights (numpy, host) of the network."""
    conv_w: list          # N_CONV arrays (CHANNELS, kp(l))
    conv_b: list          # N_CONV arrays (CHANNELS,)
    w1: np.ndarray        # (HIDDEN, CHANNELS * 64)
    b1: np.ndarray
    w2: np.ndarray        # (N_CLASSES, HIDDEN)
    b2: np.ndarray
    meta: dict = field(default_factory=dict)     # threshold, k, widen, training record

    @classmethod
    def init(cls, seed: int = 0) -> "Weights":
        rng = np.random.default_rng(seed)

        def he(shape, fan_in):
            return (rng.standard_normal(shape) * math.sqrt(2.0 / fan_in)).astype(np.float32)
        conv_w, conv_b = [], []
        for layer in range(N_CONV):
            k = kp(layer)
            real = WIDTH * (IN_CHANNELS if layer == 0 else CHANNELS)
            w = np.zeros((CHANNELS, k), np.float32)
            w[:, :real] = he((CHANNELS, real), real)
            conv_w.append(w)
            conv_b.append(np.zeros(CHANNELS, np.float32))
        flat = CHANNELS * (N_BINS >> N_CONV)
        return cls(conv_w, conv_b, he((HIDDEN, flat), flat), np.zeros(HIDDEN, np.float32),
                   (he((N_CLASSES, HIDDEN), HIDDEN) * 0.5).astype(np.float32),
                   np.zeros(N_CLASSES, np.float32))

    def arrays(self) -> list:
        return [*self.conv_w, *self.conv_b, self.w1, self.b1, self.w2, self.b2]

    def save(self, path: str, *, compact: bool = False) -> None:
        """npz of the arrays (fp32) and the meta record; ``compact`` stores the
        weight matrices as their bf16 bit patterns (what the GEMMs read; half
        the size, biases stay fp32)."""
        import json
        arrays = {}
        for i, a in enumerate(self.arrays()):
            if compact and a.ndim == 2:
                arrays[f"h{i}"] = _bf16_bits(a)
            else:
                arrays[f"p{i}"] = a
        np.savez_compressed(path, meta=np.array(json.dumps(self.meta)), **arrays)

    @classmethod
    def load(cls, path: str) -> "Weights":
        import json
        z = np.load(path)
        a = [z[f"p{i}"].astype(np.float32) if f"p{i}" in z else
             (z[f"h{i}"].astype(np.uint32) << 16).view(np.float32)
             for i in range(2 * N_CONV + 4)]
        meta = json.loads(str(z["meta"])) if "meta" in z else {}
        return cls(a[:N_CONV], a[N_CONV:2 * N_CONV], *a[2 * N_CONV:], meta=meta)


class ProposalNet:
    """The network on the device: bf16 copies of the weights for the GEMMs and,
    when trained, fp32 masters, Adam moments and gradients."""

    def __init__(self, weights: Weights, ops: Ops | None = None, *, train: bool = False):
        import torch
        self.torch = torch
        self.ops = ops or Ops()
        dev = "cuda"
        self.master = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in weights.arrays()]
        self.train = train
        # bf16 copies of the matrices (conv weights, W1, W2); biases stay fp32
        self.mats = list(range(N_CONV)) + [2 * N_CONV, 2 * N_CONV + 2]
        self.half = {i: self.master[i].to(torch.bfloat16) for i in self.mats}
        if train:
            self.m = [torch.zeros_like(p) for p in self.master]
            self.v = [torch.zeros_like(p) for p in self.master]
            self.g = [torch.zeros_like(p) for p in self.master]
            self.step = 0

    def weights(self, meta: dict | None = None) -> Weights:
        a = [p.detach().cpu().numpy().copy() for p in self.master]
        return Weights(a[:N_CONV], a[N_CONV:2 * N_CONV], *a[2 * N_CONV:], meta=dict(meta or {}))

    # ---- forward -------------------------------------------------------------------
    def forward(self, x):
        """x: (B, N_BINS, IN_CHANNELS) bf16 -> logits (B, N_CLASSES) fp32."""
        torch, ops = self.torch, self.ops
        B = int(x.shape[0])
        cache = {"x": x, "cols": [], "acts": []}
        act, L, C = x, N_BINS, IN_CHANNELS
        for layer in range(N_CONV):
            k = kp(layer)
            R = B * (L // 2)
            col = torch.empty((R, k), dtype=torch.bfloat16, device="cuda")
            ops.im2col(act, col, B, L, C, k)
            y = torch.empty((R, CHANNELS), dtype=torch.bfloat16, device="cuda")
            ops.gemm(col, self.half[layer], y, M=R, N=CHANNELS, K=k, lda=k, ldb=k,
                     ldo=CHANNELS, mode=0, bias=self.master[N_CONV + layer], relu=True)
            if self.train:
                cache["cols"].append(col)
                cache["acts"].append(y)
            act, L, C = y, L // 2, CHANNELS
        flat_n = CHANNELS * L
        h = torch.empty((B, HIDDEN), dtype=torch.bfloat16, device="cuda")
        ops.gemm(act, self.half[2 * N_CONV], h, M=B, N=HIDDEN, K=flat_n, lda=flat_n, ldb=flat_n,
                 ldo=HIDDEN, mode=0, bias=self.master[2 * N_CONV + 1], relu=True)
        logits = torch.empty((B, N_CLASSES), dtype=torch.float32, device="cuda")
        ops.gemm(h, self.half[2 * N_CONV + 2], logits, M=B, N=N_CLASSES, K=HIDDEN, lda=HIDDEN,
                 ldb=HIDDEN, ldo=N_CLASSES, mode=1, bias=self.master[2 * N_CONV + 3])
        cache["flat"], cache["h"] = act, h
        self._cache = cache
        return logits

    # ---- backward and update ------------------------------------------------------------
    def backward(self, dlogits):
        """dlogits: (B, N_CLASSES) bf16 -> gradients accumulated in self.g."""
        torch, ops = self.torch, self.ops
        c = self._cache
        B = int(dlogits.shape[0])
        h, flat = c["h"], c["flat"]
        flat_n = CHANNELS * (N_BINS >> N_CONV)
        iw1, ib1, iw2, ib2 = 2 * N_CONV, 2 * N_CONV + 1, 2 * N_CONV + 2, 2 * N_CONV + 3

        def T(x, R, C):
            out = torch.empty((C, R), dtype=torch.bfloat16, device="cuda")
            ops.transpose(x, C, out, R, R, C)
            return out

        def splits(K, tiles):
            return max(1, min(64, (148 * 2) // max(tiles, 1), (K + 63) // 64))

        # logits = h W2^T + b2
        dT = T(dlogits, B, N_CLASSES)                 # (N_CLASSES, B)
        hT = T(h, B, HIDDEN)                          # (HIDDEN, B)
        ops.gemm(dT, hT, self.g[iw2], M=N_CLASSES, N=HIDDEN, K=B, lda=B, ldb=B, ldo=HIDDEN,
                 mode=2, splits=splits(B, 8))
        ops.colsum(dlogits, N_CLASSES, B, N_CLASSES, self.g[ib2])
        w2T = T(self.half[iw2], N_CLASSES, HIDDEN)    # (HIDDEN, N_CLASSES)
        dh = torch.empty((B, HIDDEN), dtype=torch.bfloat16, device="cuda")
        ops.gemm(dlogits, w2T, dh, M=B, N=HIDDEN, K=N_CLASSES, lda=N_CLASSES, ldb=N_CLASSES,
                 ldo=HIDDEN, mode=0, mask=h)
        # h = relu(flat W1^T + b1)
        dhT = T(dh, B, HIDDEN)
        flatT = T(flat, B, flat_n)
        ops.gemm(dhT, flatT, self.g[iw1], M=HIDDEN, N=flat_n, K=B, lda=B, ldb=B, ldo=flat_n,
                 mode=2, splits=splits(B, 2 * (flat_n // 256)))
        ops.colsum(dh, HIDDEN, B, HIDDEN, self.g[ib1])
        w1T = T(self.half[iw1], HIDDEN, flat_n)
        dy = torch.empty((B, flat_n), dtype=torch.bfloat16, device="cuda")
        ops.gemm(dh, w1T, dy, M=B, N=flat_n, K=HIDDEN, lda=HIDDEN, ldb=HIDDEN, ldo=flat_n,
                 mode=0, mask=flat)
        # the convolutions, last to first; dy is the pre-activation gradient
        L = N_BINS >> (N_CONV - 1)
        for layer in reversed(range(N_CONV)):
            k = kp(layer)
            R = B * (L // 2)
            col = c["cols"][layer]
            colT = T(col, R, k)                       # (k, R)
            dyT = T(dy, R, CHANNELS)                  # (CHANNELS, R)
            ops.gemm(colT, dyT, self.g[layer], M=k, N=CHANNELS, K=R, lda=R, ldb=R, ldo=k,
                     mode=2, transpose=True, splits=splits(R, (k + 127) // 128))
            ops.colsum(dy, CHANNELS, R, CHANNELS, self.g[N_CONV + layer])
            if layer > 0:
                wT = T(self.half[layer], CHANNELS, k)     # (k, CHANNELS)
                dcol = torch.empty((R, k), dtype=torch.bfloat16, device="cuda")
                ops.gemm(dy, wT, dcol, M=R, N=k, K=CHANNELS, lda=CHANNELS, ldb=CHANNELS, ldo=k,
                         mode=0)
                prev = c["acts"][layer - 1]           # the ReLU output this layer read
                dx = torch.empty((B * L, CHANNELS), dtype=torch.bfloat16, device="cuda")
                ops.col2im(dcol, prev, dx, B, L, CHANNELS, k)
                dy = dx
            L *= 2

    def zero_grad(self):
        for g in self.g:
            g.zero_()

    def adam(self, lr: float, *, b1=0.9, b2=0.999, eps=1e-8, wd=1e-4):
        self.step += 1
        lib = self.ops.lib
        for i, p in enumerate(self.master):
            w16 = self.half.get(i)
            decay = wd if i in self.mats else 0.0
            _ok(lib.pn_adam(_ptr(p), _ptr(self.m[i]), _ptr(self.v[i]), _ptr(self.g[i]),
                            _ptr(w16), p.numel(), lr, b1, b2, eps, decay, self.step,
                            self.ops._st), "pn_adam")

    def loss_and_grad(self, logits, labels, side: float = 0.1):
        """Cross-entropy against the label bins (``side`` of the target on each
        neighbour); returns (dlogits bf16, loss tensor)."""
        torch = self.torch
        B = int(logits.shape[0])
        d = torch.empty((B, N_CLASSES), dtype=torch.bfloat16, device="cuda")
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        _ok(self.ops.lib.pn_softmax_xent(_ptr(logits), B, N_CLASSES, _ptr(labels), side,
                                         1.0 / B, _ptr(d), _ptr(loss), self.ops._st),
            "pn_softmax_xent")
        return d, loss

    def topk(self, logits, k: int):
        torch = self.torch
        B = int(logits.shape[0])
        idx = torch.empty((B, k), dtype=torch.int32, device="cuda")
        mass = torch.empty(B, dtype=torch.float32, device="cuda")
        _ok(self.ops.lib.pn_topk(_ptr(logits), B, N_CLASSES, k, _ptr(idx), _ptr(mass),
                                 self.ops._st), "pn_topk")
        return idx, mass


def class_edges(n_periods: int) -> np.ndarray:
    """Grid-index edges of the N_CLASSES log-period bins of a log-spaced grid of
    ``n_periods`` periods: class j holds indices [edges[j], edges[j + 1])."""
    return (np.arange(N_CLASSES + 1, dtype=np.int64) * n_periods) // N_CLASSES


def labels_of(best_index: np.ndarray, n_periods: int) -> np.ndarray:
    """The class of each curve's best grid index."""
    return np.minimum((np.asarray(best_index, np.int64) * N_CLASSES) // n_periods,
                      N_CLASSES - 1).astype(np.int32)


def window_mask(classes, edges: np.ndarray, widen: int) -> list[tuple[int, int]]:
    """Grid-index intervals [lo, hi) covered by the given classes, each widened
    by ``widen`` neighbouring classes on either side, merged and sorted."""
    n = edges.size - 1
    spans = sorted((int(edges[max(int(j) - widen, 0)]), int(edges[min(int(j) + widen + 1, n)]))
                   for j in classes if 0 <= int(j) < n)
    out: list[tuple[int, int]] = []
    for lo, hi in spans:
        if out and lo <= out[-1][1]:
            out[-1] = (out[-1][0], max(out[-1][1], hi))
        else:
            out.append((lo, hi))
    return out


def windows_hold(classes: np.ndarray, index: np.ndarray, edges: np.ndarray,
                 widen: int) -> np.ndarray:
    """Per row: whether the windows of ``classes[i]`` (``window_mask``) hold grid
    index ``index[i]`` -- a chosen class within ``widen`` of the index's class."""
    cls = np.searchsorted(edges, np.asarray(index, dtype=np.int64), side="right") - 1
    return (np.abs(np.asarray(classes, dtype=np.int64) - cls[:, None]) <= widen).any(axis=1)


def device_packed(t, y, offsets):
    """Packed FP64 times and fluxes and their int64 offsets (host arrays,
    offsets from 0) on the device, copied on the current stream (asynchronously
    when the host arrays are pinned)."""
    import torch
    return tuple(torch.from_numpy(np.ascontiguousarray(a)).to("cuda", non_blocking=True)
                 for a in (np.asarray(t, np.float64), np.asarray(y, np.float64),
                           np.asarray(offsets, np.int64)))


def device_curves(curves):
    """:func:`device_packed` of ``(t, y, ...)`` curves."""
    sizes = np.array([np.asarray(c[0]).size for c in curves], dtype=np.int64)
    off = np.zeros(sizes.size + 1, dtype=np.int64)
    off[1:] = np.cumsum(sizes)
    return device_packed(np.concatenate([np.asarray(c[0], np.float64) for c in curves]),
                         np.concatenate([np.asarray(c[1], np.float64) for c in curves]), off)


@dataclass
class PrunedResult:
    """Per curve: the best period found, its grid index in the full grid, the
    power there, whether the network's windows were searched (else the full
    grid), and the probability mass of the chosen classes."""
    best_period: np.ndarray
    best_index: np.ndarray
    best_power: np.ndarray
    confident: np.ndarray
    mass: np.ndarray
    periods_searched: int


class Proposer:
    """Learned-pruned BLS over one segmented trial grid (``segments``: the full
    grid's ``(periods, durations)`` pairs, periods ascending).  A curve whose
    top-``k`` classes hold at least ``threshold`` of the network's probability
    is searched exactly over those classes' periods (each widened by ``widen``
    classes), with the full grid's durations for each period's segment, so any
    period searched gets the full search's result; the others are searched over
    the full grid.  Ties in the best power resolve as the full search's do (the
    lowest grid index)."""

    def __init__(self, weights: Weights, segments, *, oversample: int = 10, objective: int = 0,
                 k: int | None = None, widen: int | None = None,
                 threshold: float | None = None, chunk: int = 1024, stream=None):
        meta = weights.meta
        self._init_grid(segments, oversample, objective,
                        int(widen if widen is not None else meta.get("widen", 1)))
        self.net = ProposalNet(weights, Ops(stream))
        self.stream = stream
        self.k = int(k if k is not None else meta.get("k", 16))
        self.threshold = float(threshold if threshold is not None else meta.get("threshold", 0.0))
        self.chunk = int(chunk)

    def _init_grid(self, segments, oversample: int, objective: int, widen: int) -> None:
        """The host-side grid state (no device work): the full grid, its class
        edges and segment bounds."""
        self.segments = [(np.ascontiguousarray(p, dtype=np.float64),
                          np.ascontiguousarray(d, dtype=np.float64)) for p, d in segments]
        self.periods = np.concatenate([p for p, _ in self.segments])
        if self.periods.size < N_CLASSES or not np.all(np.diff(self.periods) > 0.0):
            raise ValueError("the proposal network needs an ascending grid of at least "
                             f"{N_CLASSES} periods")
        self.seg_bounds = np.concatenate([[0], np.cumsum([p.size for p, _ in self.segments])])
        self.edges = class_edges(self.periods.size)
        self.oversample, self.objective, self.widen = int(oversample), int(objective), int(widen)
        self.full = _lib.PackedGrid.from_segments(self.segments, self.oversample, self.objective)

    def propose_packed(self, t, y, offsets):
        """Top-k classes (n, k) and their probability mass (n,) of every curve of
        a packed batch (host arrays; ``offsets`` from 0)."""
        import torch
        n = int(len(offsets) - 1)
        with torch.cuda.stream(self.stream) if self.stream is not None else _null():
            td, yd, od = device_packed(t, y, offsets)
            x = torch.empty((min(self.chunk, n), N_BINS, IN_CHANNELS), dtype=torch.bfloat16,
                            device="cuda")
            idx, mass = [], []
            for a in range(0, n, self.chunk):
                m = min(self.chunk, n - a)
                self.net.ops.bin_curves(td, yd, od[a:], m, x)
                logits = self.net.forward(x[:m])
                i, s = self.net.topk(logits, self.k)
                idx.append(i)
                mass.append(s)
            idx = torch.cat(idx).cpu().numpy()
            mass = torch.cat(mass).cpu().numpy()
        self.net.ops.check()
        return idx, mass

    def propose(self, curves):
        """:meth:`propose_packed` of ``(t, y, ...)`` curves."""
        pc = _lib.PackedCurves.from_arrays([(c[0], c[1], None) for c in curves])
        return self.propose_packed(pc.t, pc.y, pc.offsets)

    def window_segments(self, classes):
        """The full grid's segments cut down to the windows of ``classes``."""
        out = []
        spans = window_mask(classes, self.edges, self.widen)
        for s, (p, d) in enumerate(self.segments):
            s0, s1 = int(self.seg_bounds[s]), int(self.seg_bounds[s + 1])
            parts = [p[max(lo, s0) - s0:min(hi, s1) - s0] for lo, hi in spans
                     if lo < s1 and hi > s0]
            if parts:
                out.append((np.concatenate(parts), d))
        return out

    def search(self, curves, engine) -> PrunedResult:
        """``curves``: ``(t, y, dy or None)`` tuples; one engine launch for all."""
        pc = _lib.PackedCurves.from_arrays(curves)
        return self.search_packed(pc, engine)

    def window_grids(self, classes: np.ndarray):
        """Every row's window grid at once: ``(grids, index)`` with one
        ``_lib.PackedGrid`` per row of ``classes`` (its periods a view into one
        array, its segments the full grid's, empty where no window reaches) and
        the full-grid index of every period, concatenated row after row."""
        n = classes.shape[0]
        if n == 0:
            return [], np.empty(0, dtype=np.int64)
        if not hasattr(self, "_pieces"):
            # the grid's index runs cut at every class edge and segment bound:
            # piece p is [cut[p], cut[p + 1]), of one class and one segment
            cut = np.unique(np.concatenate([self.edges, self.seg_bounds]))
            lo = cut[:-1]
            self._pieces = (lo, np.diff(cut),
                            np.searchsorted(self.edges, lo, side="right") - 1,
                            np.searchsorted(self.seg_bounds, lo, side="right") - 1)
        lo, ln, pcls, pseg = self._pieces
        sel = np.zeros((n, N_CLASSES), dtype=bool)
        rows = np.arange(n)[:, None]
        for off in range(-self.widen, self.widen + 1):
            sel[rows, np.clip(classes.astype(np.int64) + off, 0, N_CLASSES - 1)] = True
        ci, pi = np.nonzero(sel[:, pcls])              # row-major: each row's pieces ascending
        lens = ln[pi]
        # the index runs as one cumulative sum: steps of 1, a jump at each piece
        ends = np.cumsum(lens)
        index = np.ones(int(ends[-1]), dtype=np.int64)
        index[0] = lo[pi[0]]
        index[ends[:-1]] = lo[pi[1:]] - (lo[pi[:-1]] + lens[:-1] - 1)
        np.cumsum(index, out=index)
        n_seg = len(self.segments)
        counts = np.zeros((n, n_seg), dtype=np.int64)
        np.add.at(counts, (ci, pseg[pi]), lens)
        seg_off = np.zeros((n, n_seg + 1), dtype=np.int64)
        seg_off[:, 1:] = np.cumsum(counts, axis=1)
        row_off = np.concatenate([[0], np.cumsum(seg_off[:, -1])])
        periods = self.periods[index]
        grids = [_lib.PackedGrid(seg_off[i], periods[row_off[i]:row_off[i + 1]],
                                 self.full.dur_offsets, self.full.durations, self.oversample,
                                 self.objective) for i in range(n)]
        return grids, index

    def search_packed(self, packed, engine) -> PrunedResult:
        """A packed batch (``_lib.PackedCurves``): the network, then one engine
        launch over every curve's windows or full grid."""
        idx, mass = self.propose_packed(packed.t, packed.y, packed.offsets)
        confident = mass >= self.threshold
        conf = np.flatnonzero(confident)
        wgrids, windex = self.window_grids(idx[conf])
        grids = [self.full] + wgrids
        gid = np.zeros(packed.n_curves, dtype=np.int32)
        gid[conf] = np.arange(1, conf.size + 1, dtype=np.int32)
        engine.prepare_grids(grids, gid, packed)
        engine.launch()
        bi, bp, _, _ = engine.download_best()
        bi = np.asarray(bi, dtype=np.int64)
        full_index = bi.copy()
        if conf.size:
            # a window grid's index k is the k-th period of its row in windex
            sizes = np.array([g.n_periods for g in wgrids], dtype=np.int64)
            base = np.concatenate([[0], np.cumsum(sizes)[:-1]])
            full_index[conf] = windex[base + bi[conf]]
        searched = int((packed.n_curves - conf.size) * self.full.n_periods + windex.size)
        return PrunedResult(self.periods[full_index], full_index, bp, confident, mass, searched)


__all__ = ["N_BINS", "N_CLASSES", "Ops", "PrunedResult", "ProposalNet", "Proposer", "Weights",
           "class_edges", "device_curves", "device_packed", "kp", "labels_of", "window_mask",
           "windows_hold"]
