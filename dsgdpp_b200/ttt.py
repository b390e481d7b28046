"""Time to target test RMSE: plain FP32 BoldDriver against the tuned forms.

The plain run is FP32 DSGD++ with BoldDriver for a fixed number of epochs;
its final test RMSE is the target.  The tuned runs (BF16 factors, the learned
step controller with BoldDriver fallback, or both) stop once their test RMSE
is within +0.5% of that target.  Wall time counts every epoch, loss
evaluation and step decision of a run (device work is synchronous per epoch).

    python -m dsgdpp_b200.ttt --workload c2 --epochs 50 --controller params.npy
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
PARAMS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "controller_params.npy")


def evaluate(P, wl, data, d, epochs=50, eps0=0.001, net=None, seed=777, device=0,
             layout="runs", log_dump=None):
    """Plain FP32 BoldDriver for `epochs` epochs sets the target (its final test
    RMSE, +0.5%); then BF16 + BoldDriver and, with `net`, the controller at
    FP32 and BF16 run until they reach it.  Returns the summary dict."""
    from dsgdpp_b200.controller import time_to_target
    ntest = len(data["tvals"])

    def ctx_for(precision):
        l2 = wl["s"] is not None
        ctx = P.Context(P.Config(m=wl["m"], n=wl["n"], rank=wl["rank"], d=d, precision=precision,
                                 regularize="L2" if l2 else "None",
                                 regularize_lambda=0.05 if l2 else 0.0, device=device,
                                 layout=layout))
        ctx.set_matrix(P.TRAIN, data["rows"], data["cols"], data["vals"])
        ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
        ctx.set_factors(data["W0"], data["H0"])
        ctx.seed(seed)
        return ctx

    def rmse(loss):
        return math.sqrt(loss / ntest)

    out = {"workload": wl["text"], "d": d, "epochs": epochs, "eps0": eps0, "layout": layout}
    with ctx_for("fp32") as ctx:
        t0 = time.perf_counter()
        plain = ctx.run(epochs, "BoldDriver", eps0)
        out["plain_fp32_s"] = time.perf_counter() - t0
    target_rmse = rmse(plain[-1]["test_loss"])
    target_loss = (target_rmse * 1.005) ** 2 * ntest
    out["target_test_rmse"] = target_rmse
    _, out["plain_fp32_s_traced"] = time_to_target(plain, -1)

    dump = {"plain_fp32": plain}
    runs = [("bf16_bolddriver", "bf16", None)]
    if net is not None:
        runs += [("fp32_controller", "fp32", net), ("bf16_controller", "bf16", net)]
    for name, prec, ctl in runs:
        with ctx_for(prec) as ctx:
            t0 = time.perf_counter()
            if ctl is None:
                tr = ctx.run(epochs * 2, "BoldDriver", eps0)
                fb = None
            else:
                tr, fb = ctx.run_controlled(ctl, epochs * 2, eps0, target_test_loss=target_loss)
            wall = time.perf_counter() - t0
        dump[name] = tr
        ep, secs = time_to_target(tr, target_loss)
        out[name] = {"epochs_to_target": ep, "seconds_to_target": secs, "wall_s": wall,
                     "final_test_rmse": rmse(tr[-1]["test_loss"]), "fallbacks": fb,
                     "ratio_to_plain": (secs / out["plain_fp32_s_traced"]) if ep else None,
                     "precision": prec,
                     # the step sizes of the kept epochs, in order
                     "eps": [r["eps"] for r in tr[1:]]}
    out["plain_fp32"] = {"precision": "fp32", "eps": [r["eps"] for r in plain[1:]]}
    if log_dump:
        with open(log_dump, "w") as f:
            json.dump(dump, f)
    return out


def main():
    sys.path.insert(0, ROOT)
    import bench
    import dsgdpp_b200 as P

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--epochs", type=int, default=50)
    ap.add_argument("--eps", type=float, default=0.001)
    ap.add_argument("--controller", default=PARAMS)
    ap.add_argument("--seed", type=int, default=777)
    ap.add_argument("--d", type=int, default=0)
    ap.add_argument("--layout", default="runs")
    ap.add_argument("--dump", default=None, help="write every run's trace rows here (JSON)")
    args = ap.parse_args()

    wl = bench.WORKLOADS[args.workload]
    data, _ = bench.generate(wl, args.seed)
    net = None
    if args.controller and os.path.exists(args.controller):
        net = P.Mlp(seed=1)
        net.params = np.load(args.controller)
    out = evaluate(P, wl, data, args.d or wl["d"], args.epochs, args.eps, net, args.seed,
                   layout=args.layout, log_dump=args.dump)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
