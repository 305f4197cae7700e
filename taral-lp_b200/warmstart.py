"""Learned warm start for a scenario family of refinery LPs (one B200).

A scenario is the family's base LP with its prices and capacities scaled by a 256-vector p of factors in
[0.8, 1.2] (lpgen.RefineryBase.instance). The network maps the normalised p to the normalised optimal (x, y) of
that scenario and to the logarithm of the primal weight that scenario's solve ended with; it is trained on
solutions the batched PDHG engine itself computes, with this library's own BF16 tensor-core kernels (pdhg.Mlp). At
solve time x is projected onto the column bounds, and (x, y, w) are handed to the solver as its start point and
initial primal weight.

Fallback: the unmodified cold start stays the default. For each scenario the warm and the cold start are both run
for one evaluation block (64 iterations); if the warm start's relative KKT error after that block is not better
than the cold start's, the scenario is solved cold. Every answer, warm or cold, is judged by the same FP64 KKT
test of the solver.
"""
from __future__ import annotations

import dataclasses
import time
from typing import List, Optional

import numpy as np

import lpgen
import pdhg

P_MEAN, P_STD = 1.0, 0.4 / np.sqrt(12.0)  # U(0.8, 1.2)


def features(P: np.ndarray) -> np.ndarray:
    return (np.atleast_2d(P) - P_MEAN) / P_STD


@dataclasses.dataclass
class Normalizer:
    mean: np.ndarray
    std: np.ndarray

    @classmethod
    def fit(cls, T: np.ndarray) -> "Normalizer":
        mean = T.mean(axis=0)
        std = T.std(axis=0)
        floor = 1e-3 * (np.abs(T).mean() + 1e-12)
        return cls(mean, np.maximum(std, floor))

    def encode(self, T):
        return (T - self.mean) / self.std

    def decode(self, Z):
        return Z * self.std + self.mean


def kkt(r: dict) -> float:
    return max(r["rel_primal"], r["rel_dual"], r["rel_gap"])


def solve_batch(lps, tol, precision=pdhg.FP32, x0=None, y0=None, max_iter=2_000_000_000, time_limit=3600.0,
                chunk=256, w0=None):
    """Solve many scenarios in batches of `chunk` (one context per chunk). Returns (outcomes, xs, ys, seconds)."""
    outs, xs, ys = [], [], []
    t = 0.0
    for c0 in range(0, len(lps), chunk):
        part = lps[c0:c0 + chunk]
        b = pdhg.Batch(part, tol=tol, precision=precision, max_iter=max_iter, time_limit=time_limit)
        px = None if x0 is None else x0[c0:c0 + chunk]
        py = None if y0 is None else y0[c0:c0 + chunk]
        pw = None if w0 is None else w0[c0:c0 + chunk]
        t0 = time.perf_counter()
        r, x, y = b.solve(x0=px, y0=py, w0=pw)
        t += time.perf_counter() - t0
        outs += r
        xs += x
        ys += y
        b.close()
    return outs, xs, ys, t


@dataclasses.dataclass
class WarmStart:
    net: pdhg.Mlp
    norm: Normalizer
    n: int
    m: int

    def predict(self, P: np.ndarray, lps: List[lpgen.LP]):
        """Predicted (x, y, w) per scenario: x projected onto the column bounds, w the initial primal weight."""
        Z = self.net.forward(features(P))
        T = self.norm.decode(Z.astype(np.float64))
        xs, ys, ws = [], [], []
        for t, lp in zip(T, lps):
            xs.append(np.clip(t[:self.n], lp.col_lo, lp.col_up))
            ys.append(t[self.n:self.n + self.m])
            ws.append(float(np.exp(np.clip(t[self.n + self.m], -30.0, 30.0))))
        return xs, ys, np.array(ws)


def train(P: np.ndarray, X: List[np.ndarray], Y: List[np.ndarray], W: np.ndarray, hidden=512, depth=3, epochs=400,
          batch=64, lr=3e-4, seed=0) -> WarmStart:
    """Fit the network to (x, y, log w) of solved scenarios (W: their final primal weights). The output layer
    starts at zero, so the untrained network predicts the training mean and training can only move away from it
    where the data supports that."""
    T = np.hstack([np.vstack(X), np.vstack(Y), np.log(np.asarray(W, np.float64))[:, None]])
    norm = Normalizer.fit(T)
    batch = min(batch, len(P))
    net = pdhg.Mlp(P.shape[1], hidden, depth, T.shape[1], max_batch=batch)
    net.init(seed, out_scale=0.0)
    net.set_dataset(features(P), norm.encode(T))
    net.last_loss = net.train(epochs=epochs, batch=batch, lr=lr, seed=seed)
    return WarmStart(net, norm, X[0].size, Y[0].size)


def evaluate(lps, P, ws: Optional[WarmStart], tol=1e-6, precision=pdhg.FP32, probe_iters=64):
    """Cold start against learned warm start (with the fallback rule) on the same scenarios."""
    cold, xc, yc, t_cold = solve_batch(lps, tol, precision)
    res = {"cold_iterations": [r["iterations"] for r in cold], "cold_status": [r["status"] for r in cold],
           "cold_s": t_cold, "cold_objective": [r["objective"] for r in cold]}
    if ws is None:
        return res
    t0 = time.perf_counter()
    x0, y0, w0 = ws.predict(P, lps)
    t_pred = time.perf_counter() - t0
    # fallback probe: one block from each start
    pw, _, _, t_pw = solve_batch(lps, tol, precision, x0=x0, y0=y0, w0=w0, max_iter=probe_iters)
    pc, _, _, t_pc = solve_batch(lps, tol, precision, max_iter=probe_iters)
    use = [kkt(a) < kkt(b) for a, b in zip(pw, pc)]
    wx = [x if u else None for x, u in zip(x0, use)]
    wy = [y if u else None for y, u in zip(y0, use)]
    ww = np.where(use, w0, 0.0)
    warm, _, _, t_warm = solve_batch(lps, tol, precision, x0=wx, y0=wy, w0=ww)
    res.update({"warm_iterations": [r["iterations"] for r in warm], "warm_status": [r["status"] for r in warm],
                "warm_s": t_warm, "predict_s": t_pred, "probe_s": t_pw + t_pc, "used_warm": use,
                "warm_objective": [r["objective"] for r in warm]})
    return res
