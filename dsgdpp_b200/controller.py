"""Learned step-size control: trace generation, training and evaluation.

The controller network (16 -> 64 -> 64 -> 1, GELU; kernels in
csrc/kernels_mlp.cu) replaces BoldDriver's multiplier; BoldDriver stays the
fallback whenever a proposed step raises the training loss
(csrc/controller.cc, ``Context.run_controlled``).

Traces are epochs of the method itself on matrices of the 100M-entry
workload's family (Zipf row/column weights) with varied rank, noise and
density.  At each recorded state the factors are saved on the device and
every candidate log multiplier is tried from the same state; the label is the
candidate with the lowest training loss after the epoch.  The run then moves
on by a behaviour policy: BoldDriver's rule or a random multiplier.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import Config, Context, Mlp, TEST, TRAIN, controller_features

CANDIDATES = np.array([-1.0, -0.5, -0.25, -0.1, 0.0, 0.05, 0.1, 0.25, 0.5, 1.0])


def family_problem(rng, device=0):
    """One matrix of the workload family, generated on the GPU."""
    from . import synth_gpu
    m = int(rng.integers(40_000, 160_000))
    n = int(rng.integers(15_000, 50_000))
    density = float(math.exp(rng.uniform(math.log(3e-4), math.log(2e-3))))
    nnz = int(min(6_000_000, density * m * n))
    r = int(rng.choice([8, 16, 32, 64, 128]))
    noise = float(rng.uniform(0.05, 0.5))
    data = synth_gpu.make(m, n, nnz, max(1000, nnz // 50), rank_true=r, r=r, noise=noise,
                          seed=int(rng.integers(1 << 30)), s_row=1.1, s_col=1.1,
                          device=f"cuda:{device}")
    return dict(m=m, n=n, r=r, noise=noise, nnz=nnz, data=data)


def _context(prob, precision="fp32", d=16, device=0):
    ctx = Context(Config(m=prob["m"], n=prob["n"], rank=prob["r"], d=d, precision=precision,
                         device=device))
    dd = prob["data"]
    ctx.set_matrix(TRAIN, dd["rows"], dd["cols"], dd["vals"])
    ctx.set_matrix(TEST, dd["trows"], dd["tcols"], dd["tvals"])
    ctx.set_factors(dd["W0"], dd["H0"])
    return ctx


def generate_traces(count=2000, epochs=25, seed=0, device=0, log=print):
    """(features [count, 16], labels [count]) from the method's own epochs."""
    rng = np.random.default_rng(seed)
    X, y = [], []
    t0 = time.time()
    while len(X) < count:
        prob = family_problem(rng, device)
        with _context(prob, device=device) as ctx:
            ctx.seed(int(rng.integers(1 << 31)))
            eps = float(math.exp(rng.uniform(math.log(3e-4), math.log(3e-3))))
            bold = rng.random() < 0.5  # behaviour policy of this run
            tr, te = [ctx.loss()], [ctx.nzsl(TEST)]
            upd, last_m = (0.0, 0.0), 0.0
            for e in range(epochs):
                f = controller_features(tr[::-1][:5], te[::-1][:5], eps, upd[0], upd[1],
                                        e / epochs, last_m)
                ctx.save_factors()
                losses = []
                for c in CANDIDATES:
                    ctx.restore_factors()
                    ctx.epoch(eps * math.exp(c))
                    losses.append(ctx.loss())
                losses = np.array(losses)
                if np.all(~np.isfinite(losses)) or not np.all(np.isfinite(f)):
                    break
                losses[~np.isfinite(losses)] = np.inf
                X.append(f)
                y.append(float(CANDIDATES[int(np.argmin(losses))]))
                # advance by the behaviour policy from the saved state
                ctx.restore_factors()
                if bold:
                    ctx.epoch(eps)
                    cur = ctx.loss()
                    used_m = 0.0
                    nxt = eps * (0.5 if tr[-1] <= cur else 1.05)
                else:
                    used_m = float(rng.choice(CANDIDATES))
                    ctx.epoch(eps * math.exp(used_m))
                    cur = ctx.loss()
                    nxt = eps * math.exp(used_m)
                upd = ctx.update_norms()
                tr.append(cur)
                te.append(ctx.nzsl(TEST))
                last_m = used_m
                eps = nxt
                if len(X) >= count:
                    break
                if not math.isfinite(cur) or cur > 4.0 * tr[0]:
                    break  # the behaviour policy diverged: later states are not useful
        log(f"traces {len(X)}/{count} (m={prob['m']} n={prob['n']} r={prob['r']} "
            f"nnz={prob['nnz']} noise={prob['noise']:.2f}) {time.time() - t0:.0f}s")
    return np.array(X, np.float32), np.array(y, np.float32)


def train(X, y, steps=3000, batch=256, lr=1e-3, seed=0, device=0, val_frac=0.1):
    """Trains a fresh network with the CUDA Adam kernels; returns (net, train, val loss)."""
    rng = np.random.default_rng(seed)
    keep = np.all(np.isfinite(X), axis=1) & np.isfinite(y)
    X, y = X[keep], y[keep]
    idx = rng.permutation(len(X))
    nval = max(1, int(val_frac * len(X)))
    val, tr = idx[:nval], idx[nval:]
    net = Mlp(device=device, seed=seed + 1)
    for s in range(steps):
        b = rng.choice(tr, size=min(batch, len(tr)), replace=False)
        net.train_step(X[b], y[b], lr=lr)
    tl, _ = net.gradient(X[tr], y[tr])
    vl, _ = net.gradient(X[val], y[val])
    return net, tl, vl


def time_to_target(trace, target_test_loss):
    """Epochs and seconds until the test loss first reaches the target."""
    elapsed = 0.0
    for row in trace:
        elapsed += (row["time_eps"] + row["time_epoch"] + row["time_loss"]
                    + row["time_test_loss"]) / 1e9
        if row["test_loss"] <= target_test_loss:
            return int(row["epoch"]), elapsed
    return None, elapsed
