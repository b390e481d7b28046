"""Learned step-size control: trace generation, training and evaluation.

The controller network (16 -> 64 -> 64 -> 1, GELU; kernels in
csrc/kernels_mlp.cu) replaces BoldDriver's multiplier; BoldDriver stays the
fallback whenever a proposed step raises the training loss
(csrc/controller.cc, ``Context.run_controlled``).

Traces are epochs of the method itself on matrices of the 100M-entry
workload's family (Zipf row/column weights) with varied rank, noise, density
and L2 regularisation.  At each recorded state the factors are saved on the
device and every candidate log multiplier is tried from the same state for
`horizon` epochs at that step; the label is the candidate with the lowest
training loss at the end.  The run then moves on by a behaviour policy:
BoldDriver's rule, a random multiplier, or a trained network with the
BoldDriver fallback (so later training rounds see the states the controller
itself visits, as in DAgger: Ross, Gordon, Bagnell, AISTATS 2011).
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
    l2 = float(rng.choice([0.0, 0.02, 0.05]))
    data = synth_gpu.make(m, n, nnz, max(1000, nnz // 50), rank_true=r, r=r, noise=noise,
                          seed=int(rng.integers(1 << 30)), s_row=1.1, s_col=1.1,
                          device=f"cuda:{device}")
    return dict(m=m, n=n, r=r, noise=noise, nnz=nnz, l2=l2, data=data)


def _context(prob, precision="fp32", d=16, device=0):
    l2 = prob.get("l2", 0.0)
    ctx = Context(Config(m=prob["m"], n=prob["n"], rank=prob["r"], d=d, precision=precision,
                         device=device, regularize="L2" if l2 else "None",
                         regularize_lambda=l2))
    dd = prob["data"]
    ctx.set_matrix(TRAIN, dd["rows"], dd["cols"], dd["vals"])
    ctx.set_matrix(TEST, dd["trows"], dd["tcols"], dd["tvals"])
    ctx.set_factors(dd["W0"], dd["H0"])
    return ctx


KEEP_RISE = 0.01  # as the constants of the same meaning in csrc/controller.cc
MAX_HALVINGS = 8
CAP_FRAC = 0.9
CAP_RELAX = 1.05
BOMB_RATIO = 40.0
BOMB_GROW = 4.0


def controlled_step(ctx, net, f, eps, prev_loss, fail_eps=0.0, decrease=0.5, decision=1,
                    kept_max=()):
    """One epoch under the controller with the BoldDriver fallback, exactly as
    dsgdpp_run_controlled takes it (`decision` = its index, 0 for the first;
    `kept_max` = the largest row movement of every kept epoch so far);
    returns (training loss, next step, the smallest step that raised the loss
    in this decision or 0)."""
    last3 = sorted(kept_max[-3:])
    recent = last3[len(last3) // 2] if last3 else 0.0

    def bomb():
        mean, largest = ctx.update_norms()
        return decision > 0 and largest > BOMB_RATIO * mean and largest > BOMB_GROW * recent

    m = float(net.forward(f[None, :])[0])
    proposed = eps * math.exp(m)
    if fail_eps > 0:
        proposed = min(proposed, CAP_FRAC * fail_eps)
    ctx.save_factors()
    ctx.epoch(proposed)
    cur = ctx.loss()
    bad = bomb()
    if cur <= prev_loss and not bad:
        return cur, proposed, 0.0
    if cur <= prev_loss * (1.0 + KEEP_RISE) and not bad:
        return cur, proposed * decrease, proposed
    step, failed = proposed, proposed
    for _ in range(MAX_HALVINGS):
        step *= decrease
        ctx.restore_factors()
        ctx.epoch(step)
        cur = ctx.loss()
        if cur <= prev_loss * (1.0 + KEEP_RISE) and not bomb():
            break
        failed = step
    return cur, (step if cur <= prev_loss else step * decrease), failed


def label_states(first, last, prev):
    """Labels from the candidates' lookahead losses: the candidate with the
    lowest loss after the lookahead among those whose first epoch did not raise
    the training loss (a proposal that raises it triggers the fallback); the
    smallest multiplier when every candidate raised it.  first, last:
    [states, candidates]; prev: [states]."""
    ok = np.isfinite(last) & (first <= prev[:, None])
    score = np.where(ok, last, np.inf)
    idx = np.argmin(score, axis=1)
    idx[~ok.any(axis=1)] = 0
    return CANDIDATES[idx].astype(np.float32)


def generate_traces(count=2000, epochs=25, seed=0, device=0, log=print, net=None, horizon=2,
                    policies=("bold", "random"), details=False):
    """(features [count, 16], labels [count]) from the method's own epochs;
    with details also the lookahead losses (first, last [count, candidates])
    and the state's training loss (prev [count]) that the labels come from.

    Each run follows one behaviour policy drawn from `policies`: "bold"
    (BoldDriver), "random" (a random candidate multiplier) or "net" (`net`
    proposing, with the fallback of dsgdpp_run_controlled)."""
    rng = np.random.default_rng(seed)
    X, F1, FL, PV = [], [], [], []
    t0 = time.time()
    while len(X) < count:
        prob = family_problem(rng, device)
        policy = str(rng.choice(list(policies)))
        with _context(prob, device=device) as ctx:
            ctx.seed(int(rng.integers(1 << 31)))
            eps = float(math.exp(rng.uniform(math.log(3e-4), math.log(3e-3))))
            tr, te = [ctx.loss()], [ctx.nzsl(TEST)]
            upd, last_m, fail_eps = (0.0, 0.0), 0.0, 0.0
            kept_max = []
            for e in range(epochs):
                f = controller_features(tr[::-1][:5], te[::-1][:5], eps, upd[0], upd[1],
                                        e / epochs, last_m, fail_eps)
                ctx.save_factors()
                first, last = [], []
                for c in CANDIDATES:
                    ctx.restore_factors()
                    ctx.epoch(eps * math.exp(c))
                    first.append(ctx.loss())
                    for _ in range(horizon - 1):
                        ctx.epoch(eps * math.exp(c))
                    last.append(ctx.loss())
                first, last = np.array(first), np.array(last)
                if np.all(~np.isfinite(last)) or not np.all(np.isfinite(f)):
                    break
                first[~np.isfinite(first)] = np.inf
                last[~np.isfinite(last)] = np.inf
                X.append(f)
                F1.append(first)
                FL.append(last)
                PV.append(tr[-1])
                # advance by the behaviour policy from the saved state
                ctx.restore_factors()
                failed = 0.0
                if policy == "bold":
                    ctx.epoch(eps)
                    cur = ctx.loss()
                    used_m = 0.0
                    nxt = eps * (0.5 if tr[-1] <= cur else 1.05)
                    failed = eps if not cur <= tr[-1] else 0.0
                elif policy == "net":
                    cur, nxt, failed = controlled_step(ctx, net, f, eps, tr[-1], fail_eps,
                                                       decision=e, kept_max=kept_max)
                    used_m = math.log(nxt / eps)
                else:
                    used_m = float(rng.choice(CANDIDATES))
                    ctx.epoch(eps * math.exp(used_m))
                    cur = ctx.loss()
                    nxt = eps * math.exp(used_m)
                    failed = eps * math.exp(used_m) if not cur <= tr[-1] else 0.0
                if failed > 0:
                    fail_eps = min(fail_eps, failed) if fail_eps > 0 else failed
                elif fail_eps > 0:
                    fail_eps *= CAP_RELAX
                upd = ctx.update_norms()
                kept_max.append(upd[1])
                tr.append(cur)
                te.append(ctx.nzsl(TEST))
                last_m = used_m
                eps = nxt
                if len(X) >= count:
                    break
                if not math.isfinite(cur) or cur > 4.0 * tr[0]:
                    break  # the behaviour policy diverged: later states are not useful
        log(f"traces {len(X)}/{count} ({policy}; m={prob['m']} n={prob['n']} r={prob['r']} "
            f"nnz={prob['nnz']} l2={prob['l2']} noise={prob['noise']:.2f}) "
            f"{time.time() - t0:.0f}s")
    X = np.array(X, np.float32)
    F1, FL, PV = np.array(F1), np.array(FL), np.array(PV)
    y = label_states(F1, FL, PV)
    if details:
        return X, y, F1, FL, PV
    return X, y


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


def train_dagger(rounds=2, first=2000, per_round=1500, epochs=25, horizon=2, device=0,
                 log=print):
    """Round 0: traces under BoldDriver / random multipliers; each later round
    adds traces under the current network (with the fallback) and retrains on
    everything gathered.  Returns (net, data dict with X, y and the lookahead
    losses, per-round (train, val) losses)."""
    quiet = lambda s: None
    X, y, F1, FL, PV = generate_traces(first, epochs=epochs, seed=0, device=device,
                                       horizon=horizon, policies=("bold", "random"), log=quiet,
                                       details=True)
    net, tl, vl = train(X, y, steps=4000, seed=0, device=device)
    hist = [(tl, vl)]
    log(f"round 0: {len(X)} states, labels {np.unique(y, return_counts=True)}, "
        f"train {tl:.4f} val {vl:.4f}")
    for rnd in range(1, rounds + 1):
        X1, y1, F11, FL1, PV1 = generate_traces(per_round, epochs=epochs, seed=100 + rnd,
                                                device=device, horizon=horizon, net=net,
                                                policies=("net", "net", "bold"), log=quiet,
                                                details=True)
        X, y = np.concatenate([X, X1]), np.concatenate([y, y1])
        F1, FL, PV = np.concatenate([F1, F11]), np.concatenate([FL, FL1]), np.concatenate([PV, PV1])
        net, tl, vl = train(X, y, steps=6000, seed=rnd, device=device)
        hist.append((tl, vl))
        log(f"round {rnd}: {len(X)} states, labels {np.unique(y1, return_counts=True)}, "
            f"train {tl:.4f} val {vl:.4f}")
    return net, dict(X=X, y=y, first=F1, last=FL, prev=PV), hist


def main():
    import argparse
    import os
    ap = argparse.ArgumentParser(description="train the step-size controller (DAgger rounds)")
    ap.add_argument("--rounds", type=int, default=2)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                  "controller_params.npy"))
    ap.add_argument("--traces", default=None, help="also save the (X, y) states here (.npz)")
    args = ap.parse_args()
    net, data, _ = train_dagger(rounds=args.rounds)
    np.save(args.out, net.params)
    if args.traces:
        np.savez(args.traces, **data)


if __name__ == "__main__":
    main()

