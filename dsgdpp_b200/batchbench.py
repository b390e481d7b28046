"""Batched form against looping single launches: many independent factorizations.

The workload: `count` problems (default 256) with rows log-uniform in
[1,000, 200,000], columns log-uniform in [1,000, 50,000], density log-uniform
in [1e-4, 1e-2] and rank drawn from {8, 16, 32, 64}; entries are uniform
positions with values from a rank-10 truth plus N(0, 0.1^2) noise (the 1M-entry
uniform workload's generator) with per-problem seeds and 1% held out as test
entries.  FP32 factors, Nzsl_L2(1) update, L2(0.02) regularize, BoldDriver per
problem from eps 0.001, `epochs` epochs each.

Both arms report aggregate updates/s = (sum of training entries) x epochs /
time.  The batched arm runs every problem's epoch as one graph of launches
(dsgdpp_batch_run) with d and CTAs per SM from the batched autotuner
(dsgdpp_batch_autotune, timed on every 8th problem); the looped arm runs each
problem in its own context (dsgdpp_run) one after another with the same d.
`speedup_wall` compares wall time of the whole runs (epochs, per-epoch
losses and step decisions).

    python -m dsgdpp_b200.batchbench --count 256 --epochs 30
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def draw_shapes(count, seed):
    rng = np.random.default_rng(seed)
    shapes = []
    for _ in range(count):
        m = int(round(math.exp(rng.uniform(math.log(1_000), math.log(200_000)))))
        n = int(round(math.exp(rng.uniform(math.log(1_000), math.log(50_000)))))
        dens = math.exp(rng.uniform(math.log(1e-4), math.log(1e-2)))
        r = int(rng.choice([8, 16, 32, 64]))
        nnz = max(16, int(round(dens * m * n)))
        shapes.append((m, n, nnz, r))
    return shapes


def generate(shapes, seed, device):
    from . import synth_gpu
    probs = []
    for k, (m, n, nnz, r) in enumerate(shapes):
        ntest = max(1, nnz // 100)
        d = synth_gpu.make(m, n, nnz, ntest, rank_true=10, r=r, noise=0.1, seed=seed + 7919 * k,
                           device=device)
        probs.append(dict(m=m, n=n, rank=r, rows=d["rows"], cols=d["cols"], vals=d["vals"],
                          trows=d["trows"], tcols=d["tcols"], tvals=d["tvals"], W=d["W0"],
                          H=d["H0"], seed=1000 + k, eps0=0.001))
    return probs


def main():
    sys.path.insert(0, ROOT)
    import torch
    import dsgdpp_b200 as P

    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--loop", type=int, default=-1,
                    help="problems timed in the looped arm (-1: all); the looped rate is "
                         "taken over those problems")
    ap.add_argument("--launch", default="graph")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the built-in d rule (cap 16) and the occupancy CTA count")
    args = ap.parse_args()

    dev = f"cuda:{torch.cuda.current_device()}"
    t0 = time.time()
    shapes = draw_shapes(args.count, args.seed)
    probs = generate(shapes, args.seed, dev)
    gen_s = time.time() - t0
    total = sum(len(p["vals"]) for p in probs)
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision="fp32", launch=args.launch,
                   update="Nzsl_L2", update_lambda=1.0, regularize="L2", regularize_lambda=0.02,
                   loss="Nzsl_L2", loss_lambda=1.0)
    out = {"workload": f"{args.count} problems, rows log-uniform [1e3, 2e5], columns "
                       f"log-uniform [1e3, 5e4], density log-uniform [1e-4, 1e-2], rank in "
                       f"{{8, 16, 32, 64}}, FP32, Nzsl_L2(1) update, L2(0.02), BoldDriver per "
                       f"problem, {args.epochs} epochs",
           "problems": args.count, "entries": int(total), "generate_s": gen_s}

    if not args.no_autotune:
        t0 = time.time()
        ds, ctas, ms = P.Batch.autotune(cfg, probs, sample_stride=8, epochs=2)
        for p, d in zip(probs, ds):
            p["d"] = d
        cfg.ctas_per_sm = ctas
        out["autotune"] = {"seconds": time.time() - t0, "ctas_per_sm": ctas,
                           "sample_epoch_ms": ms, "sample": "every 8th problem"}
    t0 = time.time()
    b = P.Batch(cfg, probs)
    out["batch_setup_s"] = time.time() - t0
    ds = [b.problem_d(k) for k in range(args.count)]
    t0 = time.perf_counter()
    train, test, ms = b.run(args.epochs)
    wall = time.perf_counter() - t0
    b.close()
    out["batched"] = {"updates_per_s": total * args.epochs / (ms / 1e3), "epoch_device_s": ms / 1e3,
                      "wall_s": wall, "wall_updates_per_s": total * args.epochs / wall,
                      "mean_test_rmse": float(np.mean([math.sqrt(test[k] / len(p["tvals"]))
                                                        for k, p in enumerate(probs)]))}
    out["d_histogram"] = {str(v): ds.count(v) for v in sorted(set(ds))}

    loop = range(args.count) if args.loop < 0 else range(min(args.loop, args.count))
    dev_s, wall_s, ent, rmses = 0.0, 0.0, 0, []
    for k in loop:
        p = probs[k]
        c = P.Config(m=p["m"], n=p["n"], rank=p["rank"], d=ds[k], precision="fp32",
                     launch=args.launch, update="Nzsl_L2", update_lambda=1.0, regularize="L2",
                     regularize_lambda=0.02, loss="Nzsl_L2", loss_lambda=1.0)
        with P.Context(c) as ctx:
            ctx.set_matrix(P.TRAIN, p["rows"], p["cols"], p["vals"])
            ctx.set_matrix(P.TEST, p["trows"], p["tcols"], p["tvals"])
            ctx.set_factors(p["W"], p["H"])
            ctx.seed(p["seed"])
            t0 = time.perf_counter()
            tr = ctx.run(args.epochs, "BoldDriver", p["eps0"])
            wall_s += time.perf_counter() - t0
            dev_s += sum(r["time_epoch"] for r in tr[1:]) / 1e9
            ent += len(p["vals"])
            rmses.append(math.sqrt(tr[-1]["test_loss"] / len(p["tvals"])))
    out["looped"] = {"problems": len(loop), "updates_per_s": ent * args.epochs / dev_s,
                     "epoch_host_s": dev_s, "wall_s": wall_s,
                     "wall_updates_per_s": ent * args.epochs / wall_s,
                     "mean_test_rmse": float(np.mean(rmses))}
    out["speedup_wall"] = out["batched"]["wall_updates_per_s"] / out["looped"]["wall_updates_per_s"]
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
