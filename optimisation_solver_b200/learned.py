"""Learned warm start for a parameterised LP family (the min-cost flow family).

A 3-layer BF16 MLP of width 512 maps an instance's parameters (node supplies
and arc costs) to a starting point for PDLP: the arc flows (as a fraction of
capacity), the node potentials (row duals, PDLP sign) and the initial primal
weight. It is trained with the library's tensor-core kernels on instances
that plain PDLP solved; PDLP then runs from the prediction to the requested
tolerance, and the session keeps the cold start wherever that scores better
on KKT. Node potentials are determined only up to a common constant (every
incidence row sums to zero), so the training targets are centred per
instance.

torch provides the device memory of the training set; every computation on
it is a libpdlpgpu kernel (encode, GEMMs, backward, Adam, decode).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .mlp import Mlp


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _round_up(v, k):
    return (v + k - 1) // k * k


class FlowWarmStart:
    def __init__(self, graph, hidden: int = 512, batch: int = 256, seed: int = 0, device: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.n, self.m = graph.arcs, graph.nodes
        self.count = self.m + self.n                 # supplies, then costs
        self.padded = _round_up(self.count, 8)
        self.out = _round_up(self.n + self.m + 1, 64)
        self.batch = batch
        self.mlp = Mlp(self.padded, hidden, self.out, batch, seed=seed, device=device)
        self.cap = torch.as_tensor(graph.capacity, dtype=torch.float64, device=self.dev)
        w = np.zeros(self.out, dtype=np.float32)
        w[: self.n] = 1.0 / self.n
        w[self.n: self.n + self.m] = 1.0 / self.m
        w[self.n + self.m] = 1.0
        self.loss_weights = torch.as_tensor(w, device=self.dev)
        self.stats = None

    # -- normalisation ------------------------------------------------------
    def _fit_stats(self, supply, cost, y, w):
        feats = np.concatenate([supply, cost], axis=1)
        fmean = feats.mean(axis=0).astype(np.float32)
        fstd = feats.std(axis=0).astype(np.float32)
        fstd[fstd < 1e-12] = 1.0
        yc = y - y.mean(axis=1, keepdims=True)
        ymean = yc.mean(axis=0).astype(np.float32)
        ystd = yc.std(axis=0).astype(np.float32)
        ystd[ystd < 1e-12] = 1.0
        lw = np.log(np.maximum(w, 1e-12))
        t = self.torch
        self.stats = dict(
            fmean=t.as_tensor(fmean, device=self.dev), finv=t.as_tensor(1.0 / fstd, device=self.dev),
            ymean=t.as_tensor(ymean, device=self.dev), ystd=t.as_tensor(ystd, device=self.dev),
            yinv=t.as_tensor(1.0 / ystd, device=self.dev),
            wmean=float(lw.mean()), wstd=float(max(lw.std(), 1e-3)))

    def _features(self, supply_dev, cost_dev, out_bf16):
        params = self.torch.cat([supply_dev, cost_dev], dim=1).contiguous()
        rc = native.lib().pdlpgpu_encode_features(_p(params), params.shape[0], self.count,
                                                  self.padded, _p(self.stats["fmean"]),
                                                  _p(self.stats["finv"]), _p(out_bf16))
        if rc != 0:
            raise RuntimeError(native.last_error())

    # -- training -----------------------------------------------------------
    def fit(self, supply, cost, x, y, w, epochs: int = 30, lr: float = 1e-3,
            lr_final: float = 1e-4, seed: int = 0, log=None):
        """supply [N, m], cost [N, n], x [N, n], y [N, m] (PDLP sign), w [N]
        (final primal weights), host arrays. Returns the per-epoch mean loss."""
        t = self.torch
        self._fit_stats(supply, cost, y, w)
        N = supply.shape[0]
        yc = y - y.mean(axis=1, keepdims=True)
        sup_d = t.as_tensor(supply, dtype=t.float64, device=self.dev)
        cost_d = t.as_tensor(cost, dtype=t.float64, device=self.dev)
        X = t.empty((N, self.padded), dtype=t.bfloat16, device=self.dev)
        for b0 in range(0, N, 4096):
            b1 = min(N, b0 + 4096)
            self._features(sup_d[b0:b1], cost_d[b0:b1], X[b0:b1])
        Y = t.empty((N, self.out), dtype=t.float32, device=self.dev)
        xd = t.as_tensor(x, dtype=t.float64, device=self.dev)
        yd = t.as_tensor(yc, dtype=t.float64, device=self.dev)
        wd = t.as_tensor(w, dtype=t.float64, device=self.dev)
        rc = native.lib().pdlpgpu_encode_targets(
            _p(xd), _p(yd), _p(wd), N, self.n, self.m, self.out, _p(self.cap),
            _p(self.stats["ymean"]), _p(self.stats["yinv"]), self.stats["wmean"],
            1.0 / self.stats["wstd"], _p(Y))
        if rc != 0:
            raise RuntimeError(native.last_error())
        del sup_d, cost_d, xd, yd, wd
        rng = np.random.default_rng(seed)
        steps_per_epoch = N // self.batch
        total = epochs * steps_per_epoch
        history = []
        step = 0
        for ep in range(epochs):
            order = t.as_tensor(rng.permutation(N)[: steps_per_epoch * self.batch], device=self.dev)
            losses = []
            for s in range(steps_per_epoch):
                idx = order[s * self.batch:(s + 1) * self.batch]
                xb = X.index_select(0, idx)
                yb = Y.index_select(0, idx)
                frac = step / max(1, total - 1)
                rate = lr * (lr_final / lr) ** frac
                losses.append(self.mlp.train_step(xb, yb, self.loss_weights, rate))
                step += 1
            history.append(float(np.mean(losses)))
            if log:
                log(f"epoch {ep}: loss {history[-1]:.5f}")
        return history

    # -- prediction ---------------------------------------------------------
    def predict(self, supply_dev, cost_dev):
        """Device FP64 [batch, m] supplies and [batch, n] costs -> device FP64
        warm start (primal [batch, n], row duals [batch, m], weights [batch])."""
        t = self.torch
        B = supply_dev.shape[0]
        X = t.empty((B, self.padded), dtype=t.bfloat16, device=self.dev)
        self._features(supply_dev, cost_dev, X)
        out = t.empty((B, self.out), dtype=t.float32, device=self.dev)
        self.mlp.forward(X, out)
        wx = t.empty((B, self.n), dtype=t.float64, device=self.dev)
        wy = t.empty((B, self.m), dtype=t.float64, device=self.dev)
        ww = t.empty((B,), dtype=t.float64, device=self.dev)
        rc = native.lib().pdlpgpu_decode_warmstart(
            _p(out), B, self.n, self.m, self.out, _p(self.cap), _p(self.stats["ymean"]),
            _p(self.stats["ystd"]), self.stats["wmean"], self.stats["wstd"], _p(wx), _p(wy), _p(ww))
        if rc != 0:
            raise RuntimeError(native.last_error())
        return wx, wy, ww


def train_flow_model(graph, count: int, tol: float = 1e-4, precision: str = "mixed",
                     slots: int = 1024, seed: int = 7, device: int = 0, epochs: int = 30,
                     lr: float = 1e-3, lr_final: float = 1e-4, log=None):
    """Solves `count` seeded instances of the flow family with the batched
    engine (a stream through `slots` device slots, cold start, tolerance
    `tol`), then fits a FlowWarmStart on their solutions. Returns (model,
    info) with the timings and the final training loss."""
    import time

    from . import generators as g
    from .lp import PdlpOptions
    from .session import Session

    supply, cost = g.flow_parameters(graph, count, seed=seed)
    family = g.flow_lp(graph, supply[0], cost[0])
    t0 = time.perf_counter()
    S = Session(family, min(slots, count), PdlpOptions().with_tolerance(tol), precision=precision,
                device=device)
    out = S.stream(count, objective=cost, row_lower=supply, row_upper=supply)
    S.close()
    t1 = time.perf_counter()
    ok = np.array([st == 0 for st in out["status"]])
    model = FlowWarmStart(graph, device=device, seed=seed)
    hist = model.fit(supply[ok], cost[ok], out["primal"][ok], out["dual"][ok],
                     out["final_primal_weight"][ok], epochs=epochs, lr=lr, lr_final=lr_final,
                     log=log)
    t2 = time.perf_counter()
    base = baseline_loss(graph, out["primal"][ok], out["dual"][ok], out["final_primal_weight"][ok])
    info = dict(instances=int(count), solved=int(ok.sum()), label_tolerance=tol,
                label_precision=precision, label_seconds=round(t1 - t0, 2),
                label_mean_iterations=float(out["iterations"].mean()),
                train_seconds=round(t2 - t1, 2), epochs=epochs, final_loss=float(hist[-1]),
                baseline_loss=base, explained_fraction=1.0 - float(hist[-1]) / base)
    return model, info


def baseline_loss(graph, x, y, w) -> float:
    """The training loss of the best constant prediction (each target's mean):
    the loss weights each flow by 1/n and each potential by 1/m and the
    log-weight by 1, over flows as capacity fractions, potentials centred per
    instance and standardised per node, and the standardised log-weight
    (FlowWarmStart.fit's encoding), so this is the weighted sum of the
    targets' variances. `explained_fraction` = 1 - final_loss / this."""
    xf = x / graph.capacity[None, :]
    yc = y - y.mean(axis=1, keepdims=True)
    ys = yc.std(axis=0)
    ys[ys < 1e-12] = 1.0
    yz = (yc - yc.mean(axis=0)) / ys
    lw = np.log(np.maximum(w, 1e-12))
    lz = (lw - lw.mean()) / max(lw.std(), 1e-3)
    n, m = xf.shape[1], yz.shape[1]
    return float(xf.var(axis=0).sum() / n + yz.var(axis=0).sum() / m + lz.var())
