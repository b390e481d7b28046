"""Precision form: BF16 factors (FP32 update math, stochastic rounding) against
FP32 and FP64 factors on the same data, losses accumulated in FP64.

    python -m dsgdpp_b200.precision --workload c3 --epochs 20

Prints, per precision, the test RMSE after each epoch, its difference from the
FP64 run, and the median epoch time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def main():
    sys.path.insert(0, ROOT)
    import bench
    import dsgdpp_b200 as P

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--eps", type=float, default=0.001)
    ap.add_argument("--decay", default="BoldDriver")
    ap.add_argument("--seed", type=int, default=11)
    args = ap.parse_args()
    wl = bench.WORKLOADS[args.workload]
    data, _ = bench.generate(wl, args.seed)
    ntest = len(data["tvals"])
    out = {"workload": wl["text"], "epochs": args.epochs, "decay": f"{args.decay}({args.eps})"}
    for prec in ("fp64", "fp32", "bf16"):
        cfg = P.Config(m=wl["m"], n=wl["n"], rank=wl["rank"], d=wl["d"], precision=prec)
        with P.Context(cfg) as ctx:
            ctx.set_matrix(P.TRAIN, data["rows"], data["cols"], data["vals"])
            ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
            ctx.set_factors(data["W0"], data["H0"])
            ctx.seed(args.seed)
            tr = ctx.run(args.epochs, args.decay, args.eps)
        out[prec] = {"test_rmse": [math.sqrt(r["test_loss"] / ntest) for r in tr],
                     "epoch_ms_median": float(np.median([r["time_epoch"] for r in tr[1:]]) / 1e6)}
    ref = out["fp64"]["test_rmse"]
    for prec in ("fp32", "bf16"):
        rm = out[prec]["test_rmse"]
        out[prec]["final_delta_vs_fp64"] = rm[-1] - ref[-1]
        out[prec]["final_rel_delta_vs_fp64"] = (rm[-1] - ref[-1]) / ref[-1]
        out[prec]["max_abs_delta_vs_fp64"] = float(np.max(np.abs(np.array(rm) - np.array(ref))))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
