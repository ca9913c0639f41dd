"""Learned wake proposal (pattern (4)): which bricks will wake within the next k ticks.

Traces come from the exact engine itself: at tick t the per-brick features are recorded (32 fp16
values per materialised brick: water sum and max level, partial/water/solid/active counts,
exposed surface, the six face neighbours' water sums and active counts, water-sum changes over
the last four ticks (own and the faces': the flux proxy), wake recency, height, bias); the label
is whether any cell of the brick is drained by the exact scheduler in ticks (t, t+k]. The network
(32 -> 64 -> 64 -> 1) trains on the GPU with the library's own fp16 forward/backward kernels.

At run time the proposal's positives are pre-staged (L2 prefetch of their atlas lines) before the
tick; the exact FIFO still decides what runs, so a miss costs time and never correctness.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import VfError, lib

NFEAT = 32
HORIZON = 8


def _current_stream() -> int:
    import torch

    return torch.cuda.current_stream().cuda_stream


def _sim_stream(sim, torch):
    """A torch stream context on the sim's own stream, so tensors made for the sim's kernels are
    ordered with them."""
    return torch.cuda.stream(torch.cuda.ExternalStream(sim.stream))


def _sig():
    L = lib()
    P = C.c_void_p
    for name, res, args in (
        ("vf_mlp_create", C.c_int, [C.c_int32, C.c_uint64, C.POINTER(P)]),
        ("vf_mlp_destroy", None, [P]),
        ("vf_mlp_nparams", C.c_int, []),
        ("vf_mlp_get_params", C.c_int, [P, C.POINTER(C.c_float)]),
        ("vf_mlp_set_params", C.c_int, [P, C.POINTER(C.c_float)]),
        ("vf_mlp_forward", C.c_int, [P, P, C.c_uint64, P, P]),
        ("vf_mlp_grads", C.c_int, [P, P, P, C.c_uint64, C.POINTER(C.c_float), P]),
        ("vf_mlp_train_step", C.c_int, [P, P, P, C.c_uint64, C.c_float, C.POINTER(C.c_float), P]),
        ("vf_fluid_proposal_features", C.c_int, [P, P, C.c_uint64, C.POINTER(C.c_uint64)]),
        ("vf_fluid_proposal_labels", C.c_int, [P, C.c_uint32, P, C.c_uint64]),
        ("vf_fluid_stage_bricks", C.c_int, [P, P, C.c_uint64, C.c_float, C.POINTER(C.c_uint64)]),
    ):
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    return L


class MLP:
    """The proposal network on the GPU (weights, Adam state and kernels in libvf_fluid.so)."""

    def __init__(self, device: int = 0, seed: int = 1):
        L = _sig()
        h = C.c_void_p()
        rc = L.vf_mlp_create(device, seed, C.byref(h))
        if rc:
            raise VfError(rc, "vf_mlp_create")
        self.h = h
        self.nparams = L.vf_mlp_nparams()

    def close(self):
        if getattr(self, "h", None):
            lib().vf_mlp_destroy(self.h)
            self.h = None

    __del__ = close

    def params(self) -> np.ndarray:
        out = np.zeros(self.nparams, np.float32)
        lib().vf_mlp_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        lib().vf_mlp_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)))

    def forward(self, x, torch, stream=None):
        """x: (n, 32) float16 CUDA tensor -> (n,) float32 probabilities (on torch's current stream
        unless a stream handle is given)."""
        stream = _current_stream() if stream is None else stream
        out = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        rc = lib().vf_mlp_forward(self.h, C.c_void_p(x.data_ptr()), x.shape[0], C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        if rc:
            raise VfError(rc, "vf_mlp_forward")
        return out

    def grads(self, x, y, stream=None) -> np.ndarray:
        stream = _current_stream() if stream is None else stream
        g = np.zeros(self.nparams, np.float32)
        rc = lib().vf_mlp_grads(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.shape[0], g.ctypes.data_as(C.POINTER(C.c_float)),
                                C.c_void_p(stream))
        if rc:
            raise VfError(rc, "vf_mlp_grads")
        return g

    def train_step(self, x, y, lr: float, stream=None, want_loss=False):
        stream = _current_stream() if stream is None else stream
        loss = C.c_float(0.0)
        rc = lib().vf_mlp_train_step(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), x.shape[0], lr,
                                     C.byref(loss) if want_loss else None, C.c_void_p(stream))
        if rc:
            raise VfError(rc, "vf_mlp_train_step")
        return loss.value


def reference_forward_backward(p: np.ndarray, x: np.ndarray, y: np.ndarray):
    """fp64 restatement of the network and of its mean-BCE gradient (the kernels' checker)."""
    W1 = p[0:2048].reshape(32, 64).astype(np.float64)
    b1 = p[2048:2112].astype(np.float64)
    W2 = p[2112:6208].reshape(64, 64).astype(np.float64)
    b2 = p[6208:6272].astype(np.float64)
    w3 = p[6272:6336].astype(np.float64)
    b3 = float(p[6336])
    X = x.astype(np.float64)
    Z1 = X @ W1 + b1
    H1 = np.maximum(Z1, 0)
    Z2 = H1 @ W2 + b2
    H2 = np.maximum(Z2, 0)
    z = H2 @ w3 + b3
    prob = 1 / (1 + np.exp(-z))
    n = len(y)
    dz = (prob - y) / n
    g = np.zeros_like(p, dtype=np.float64)
    g[6272:6336] = H2.T @ dz
    g[6336] = dz.sum()
    dZ2 = np.outer(dz, w3) * (Z2 > 0)
    g[2112:6208] = (H1.T @ dZ2).ravel()
    g[6208:6272] = dZ2.sum(0)
    dZ1 = (dZ2 @ W2.T) * (Z1 > 0)
    g[0:2048] = (X.T @ dZ1).ravel()
    g[2048:2112] = dZ1.sum(0)
    loss = np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))
    return prob, g, loss


def features(sim, torch):
    """(x (nslots, 32) float16 CUDA tensor, nslots) at the sim's current state."""
    L = _sig()
    n = C.c_uint64()
    rc = L.vf_fluid_proposal_features(sim.h, None, 0, C.byref(n))
    if rc:
        raise VfError(rc, "proposal_features")
    with _sim_stream(sim, torch):
        x = torch.zeros((max(n.value, 1), NFEAT), dtype=torch.float16, device="cuda")
    rc = L.vf_fluid_proposal_features(sim.h, C.c_void_p(x.data_ptr()), x.shape[0], C.byref(n))
    if rc:
        raise VfError(rc, "proposal_features")
    torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(sim.stream))
    x.record_stream(torch.cuda.current_stream())
    return x[: n.value], n.value


def labels(sim, since_tick: int, nslots: int, torch):
    L = _sig()
    with _sim_stream(sim, torch):
        y = torch.zeros(max(nslots, 1), dtype=torch.float32, device="cuda")
    rc = L.vf_fluid_proposal_labels(sim.h, since_tick, C.c_void_p(y.data_ptr()), nslots)
    if rc:
        raise VfError(rc, "proposal_labels")
    torch.cuda.current_stream().wait_stream(torch.cuda.ExternalStream(sim.stream))
    y.record_stream(torch.cuda.current_stream())
    return y[:nslots]


def stage(sim, prob, threshold: float = 0.5) -> int:
    """Pre-stage the bricks whose probability reaches the threshold (prob made on torch's current
    stream; the sim's stream waits for it)."""
    import torch

    torch.cuda.ExternalStream(sim.stream).wait_stream(torch.cuda.current_stream())
    L = _sig()
    n = C.c_uint64()
    rc = L.vf_fluid_stage_bricks(sim.h, C.c_void_p(prob.data_ptr()), prob.shape[0], threshold, C.byref(n))
    if rc:
        raise VfError(rc, "stage_bricks")
    return n.value


def collect(vf, torch, runs, every: int = 2, horizon: int = HORIZON):
    """Traces of the exact engine. runs: [(workload id, scale, seed, warm ticks, ticks, regions)].
    Returns (X float16 (N,32), Y float32 (N,), baseline persistence predictions (N,))."""
    xs, ys, base = [], [], []
    for wid, scale, seed, warm, ticks, nreg in runs:
        wl = vf.Workload(wid, scale, seed)
        for r in range(min(nreg, wl.regions)):
            sim = vf.FluidSim(wl.world(r))
            for b in wl.wakes(r):
                sim.wake(*map(int, b))
            em, amt = wl.emitters(r)
            pending = []
            for t in range(warm + ticks + horizon):
                if wl.emit_every and t % wl.emit_every == 0 and len(em):
                    sim.emit(em, amt)
                if wl.edit_every and t % wl.edit_every == wl.edit_every - 1:
                    ed = wl.edit(r, t)
                    if ed is not None:
                        sim.apply_brush(ed[0], ed[1])
                        sim.wake(*map(int, ed[2]))
                x, n = features(sim, torch)
                now = sim.stats().tick_no
                if t >= warm and t < warm + ticks and (t - warm) % every == 0 and n:
                    pending.append((now, x.clone(), n))
                while pending and pending[0][0] + horizon <= now:
                    t0, x0, n0 = pending.pop(0)
                    y0 = labels(sim, t0, n0, torch)
                    xs.append(x0)
                    ys.append(y0)
                    base.append((x0[:, 26] > 0.5).float())  # "woke in the last tick" persistence rule
                sim.tick(1)
            sim.close()
    X = torch.cat(xs) if xs else torch.zeros((0, NFEAT), dtype=torch.float16, device="cuda")
    Y = torch.cat(ys) if ys else torch.zeros(0, device="cuda")
    B = torch.cat(base) if base else torch.zeros(0, device="cuda")
    return X, Y, B


def train(mlp: MLP, X, Y, torch, epochs: int = 4, batch: int = 8192, lr: float = 2e-3, seed: int = 0):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    losses = []
    n = X.shape[0]
    for _ in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        for i in range(0, n, batch):
            idx = perm[i : i + batch]
            xb, yb = X[idx].contiguous(), Y[idx].contiguous()
            loss = mlp.train_step(xb, yb, lr, want_loss=(i == 0))
            if i == 0:
                losses.append(loss)  # loss of each epoch's first batch, before its step
    return losses


@dataclass
class Score:
    recall: float
    precision: float
    positives: int
    predicted: int
    n: int


def score(pred, Y) -> Score:
    p = pred > 0.5
    t = Y > 0.5
    tp = int((p & t).sum())
    npos, npred = int(t.sum()), int(p.sum())
    return Score(tp / npos if npos else 1.0, tp / npred if npred else 1.0, npos, npred, int(Y.numel()))


# Trace runs the default network trains on: (workload id, scale, seed, warm ticks, ticks, regions)
# - the basin, the dam break (x/z scaled to 1/4) and eight small batched regions.
DEFAULT_TRACES = [(1, 1.0, 1, 10, 60, 1), (2, 0.25, 3, 5, 40, 1), (3, 0.08, 2, 5, 40, 8)]


def train_default(vf, torch, seed: int = 5, traces=None, epochs: int = 8):
    """Collect traces of the exact engine, train a fresh network on 80% of them on the GPU and
    score it on the other 20% against the persistence rule. Returns (mlp, dict of results)."""
    import time

    t0 = time.perf_counter()
    X, Y, B = collect(vf, torch, traces or DEFAULT_TRACES, every=2)
    t1 = time.perf_counter()
    n = X.shape[0]
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    perm = torch.randperm(n, device="cuda", generator=g)
    tr, te = perm[: int(0.8 * n)], perm[int(0.8 * n):]
    mlp = MLP(seed=seed)
    losses = train(mlp, X[tr].contiguous(), Y[tr].contiguous(), torch, epochs=epochs, batch=4096, lr=2e-3)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    s = score(mlp.forward(X[te].contiguous(), torch), Y[te])
    base = score(B[te], Y[te])
    return mlp, {"samples": n, "collect_s": t1 - t0, "train_s": t2 - t1, "loss_first": losses[0], "loss_last": losses[-1],
                 "heldout": s.__dict__, "persistence": base.__dict__}
