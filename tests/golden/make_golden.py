"""Freezes golden vectors of the DSGD++ restatement into golden.json.

Run from the repository root:  python tests/golden/make_golden.py
The reference ships no golden vectors and cannot be built here, so these are
produced by the oracle (oracle/dsgdpp_oracle.cc) after it was pinned against
numpy's MT19937 and the pure-Python restatement (tests/test_oracle.py).  They
freeze the pinned random stream, the stratum schedules of every order, the
point orders and a three-epoch BoldDriver run, so later changes to either the
oracle or the CUDA path are caught.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from dsgdpp_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def problem():
    return synth.make(700, 500, 8000, 800, rank_true=6, r=8, noise=0.1, seed=2012)


def main():
    g = {"generator": "tests/golden/make_golden.py"}
    g["random32"] = {}
    for s in (0, 1, 1499881717):
        r = O.Random32(s)
        g["random32"][str(s)] = [r.next() for _ in range(10)]
    r = O.Random32(7)
    g["next_int"] = {"seed": 7, "n": [2, 3, 10, 1000, 2**31 + 1, 1],
                     "values": [[r.next_int(n) for n in [2, 3, 10, 1000, 2**31 + 1, 1]]
                                for _ in range(5)]}
    g["schedules"] = []
    for d in (1, 2, 4, 7):
        for order in ("SEQ", "RSEQ", "WR", "WOR", "COWOR"):
            s, t = O.dsgdpp_schedule(O.Random32(1000 + d), d, order)
            g["schedules"].append({"d": d, "order": order, "seed": 1000 + d,
                                   "schedule": s.tolist(), "task_seeds": t.tolist()})
    p = problem()
    d = 4
    ref = O.Problem(p.m, p.n, 8, d, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals)
    ref.configure()
    sched, seeds = O.dsgdpp_schedule(O.Random32(55), d, "COWOR")
    pos = ref.positions(sched, seeds)
    g["positions"] = {"problem": "synth.make(700, 500, 8000, 800, rank_true=6, r=8, noise=0.1, "
                                 "seed=2012), d=4, WOR, schedule seed 55",
                      "count": int(len(pos)), "sha256": sha(pos), "head": pos[:40].tolist(),
                      "block_nnz": ref.block_nnz().tolist()}
    ref.set_factors(p.W0, p.H0)
    ref.seed(1499881717)
    trace = ref.run(3, "BoldDriver", 0.01)
    W, H = ref.get_factors()
    g["run"] = {"problem": g["positions"]["problem"], "d": d, "seed": 1499881717,
                "update": "Nzsl_L2(1)", "loss": "Nzsl_L2(1)", "decay": "BoldDriver(0.01)",
                "trace": trace.tolist(), "W_sha256": sha(W), "H_sha256": sha(H),
                "W_sum": float(W.sum()), "H_sum": float(H.sum())}
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
