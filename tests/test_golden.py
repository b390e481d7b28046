"""Golden vectors (tests/golden/golden.json, frozen by tests/golden/make_golden.py)
checked against the oracle and the product: host side on CPU, replay on GPU."""
import hashlib
import json
import os

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth
from oracle import oracle as O

G = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def problem():
    return synth.make(700, 500, 8000, 800, rank_true=6, r=8, noise=0.1, seed=2012)


def test_random32_golden():
    for seed, draws in G["random32"].items():
        a, b = O.Random32(int(seed)), P.Random32(int(seed))
        assert [a.next() for _ in draws] == draws
        assert [b.next() for _ in draws] == draws
    # std::mt19937 seeded with 1 starts 1791095845 (the standard engine)
    assert G["random32"]["1"][0] == 1791095845


def test_next_int_golden():
    ng = G["next_int"]
    a, b = O.Random32(ng["seed"]), P.Random32(ng["seed"])
    for row in ng["values"]:
        assert [a.next_int(n) for n in ng["n"]] == row
        assert [b.next_int(n) for n in ng["n"]] == row


def test_schedules_golden():
    for e in G["schedules"]:
        s, t = O.dsgdpp_schedule(O.Random32(e["seed"]), e["d"], e["order"])
        assert s.tolist() == e["schedule"] and t.tolist() == e["task_seeds"]
        s, t = P.draw_schedule(P.Random32(e["seed"]), e["d"], e["order"])
        assert s.tolist() == e["schedule"] and t.tolist() == e["task_seeds"]


def test_positions_golden():
    gp = G["positions"]
    p = problem()
    ref = O.Problem(p.m, p.n, 8, 4, p.rows, p.cols, p.vals).configure()
    assert ref.block_nnz().tolist() == gp["block_nnz"]
    sched, seeds = O.dsgdpp_schedule(O.Random32(55), 4, "COWOR")
    pos = ref.positions(sched, seeds)
    assert sha(pos) == gp["sha256"] and pos[:40].tolist() == gp["head"]
    prod = P.point_orders(4, "WOR", np.array(gp["block_nnz"]), sched, seeds)
    assert sha(prod) == gp["sha256"]


def test_oracle_run_golden():
    gr = G["run"]
    p = problem()
    ref = O.Problem(p.m, p.n, 8, 4, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals)
    ref.configure()
    ref.set_factors(p.W0, p.H0)
    ref.seed(gr["seed"])
    tr = ref.run(3, "BoldDriver", 0.01)
    W, H = ref.get_factors()
    assert sha(W) == gr["W_sha256"] and sha(H) == gr["H_sha256"]
    np.testing.assert_array_equal(tr, np.array(gr["trace"]))


@pytest.mark.gpu
def test_gpu_replay_run_golden():
    gr = G["run"]
    p = problem()
    cfg = P.Config(m=p.m, n=p.n, rank=8, d=4, precision="fp64", exec="replay", launch="stream")
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        ctx.seed(gr["seed"])
        tr = ctx.run(3, "BoldDriver", 0.01)
        W, H = ctx.get_factors()
    assert sha(W) == gr["W_sha256"] and sha(H) == gr["H_sha256"]
    want = np.array(gr["trace"])
    for k, row in enumerate(tr):
        assert row["loss"] == pytest.approx(want[k, 0], rel=1e-12)
        assert row["test_loss"] == pytest.approx(want[k, 1], rel=1e-12)
