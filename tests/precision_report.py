"""Precision report: test RMSE of FP64 / FP32 / BF16 factor storage on the GPU
against the sequential FP64 oracle, on the Netflix-shaped workload.

Same data, d, seed, step schedule (BoldDriver) and epochs for every run; the
oracle runs the reference's per-block sequential SGD on the host cores (one
thread per task, a barrier per sub-epoch).  Prints one JSON object: per run
the test RMSE after every epoch, its relative error against the oracle's, and
the median epoch time.  Not collected by pytest (it takes minutes on the CPU):

    python tests/precision_report.py --epochs 10 [--scale 0.25]
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
sys.path.insert(0, ROOT)


def main():
    import bench
    import dsgdpp_b200 as P
    from dsgdpp_b200 import synth_gpu
    from oracle import oracle as O

    ap = argparse.ArgumentParser()
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--eps", type=float, default=0.001)
    ap.add_argument("--scale", type=float, default=1.0, help="fraction of the rows and entries")
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()

    wl = dict(bench.WORKLOADS["c3"])
    m = max(1000, int(wl["m"] * args.scale))
    nnz = int(wl["nnz"] * args.scale)
    ntest = int(wl["nnz_test"] * args.scale)
    n, r, d = wl["n"], wl["rank"], wl["d"]
    t0 = time.time()
    data = synth_gpu.make_ratings(m, n, nnz, ntest, r, args.seed)
    out = {"workload": f"Netflix-shaped, {m:,} x {n:,}, {nnz:,} entries (+{ntest:,} test), "
                       f"rank {r}, d = {d}, Nzsl_L2(1) update, BoldDriver({args.eps})",
           "epochs": args.epochs, "generate_s": time.time() - t0}

    t0 = time.time()
    ref = O.Problem(m, n, r, d, data["rows"], data["cols"], data["vals"], data["trows"],
                    data["tcols"], data["tvals"])
    ref.configure()
    ref.set_factors(data["W0"], data["H0"])
    ref.seed(args.seed)
    tr = ref.run(args.epochs, "BoldDriver", args.eps, threads=args.threads)
    oracle_rmse = [math.sqrt(row[1] / ntest) for row in tr]
    out["oracle_fp64"] = {"test_rmse": oracle_rmse, "seconds": time.time() - t0,
                          "threads": args.threads}

    for prec in ("fp64", "fp32", "bf16"):
        cfg = P.Config(m=m, n=n, rank=r, d=d, precision=prec)
        with P.Context(cfg) as ctx:
            ctx.set_matrix(P.TRAIN, data["rows"], data["cols"], data["vals"])
            ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
            ctx.set_factors(data["W0"], data["H0"])
            ctx.seed(args.seed)
            rows = ctx.run(args.epochs, "BoldDriver", args.eps)
        rm = [math.sqrt(row["test_loss"] / ntest) for row in rows]
        rel = [(a - b) / b for a, b in zip(rm, oracle_rmse)]
        out[prec] = {"test_rmse": rm, "final_rel_error_vs_oracle": rel[-1],
                     "max_abs_rel_error_vs_oracle": float(np.max(np.abs(rel))),
                     "epoch_ms_median": float(np.median([row["time_epoch"]
                                                         for row in rows[1:]]) / 1e6)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
