"""DSGD++ with its tasks spread over ranks (dsgdpp_b200/shard.py), emulated as
several contexts on one GPU that run one after another and hand H blocks to
each other between sub-epochs: the result must be the single-context epoch's
(bit for bit in the FP64 replay)."""
import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import shard, synth

pytestmark = pytest.mark.gpu


def _ranks_run(p, d, world, epochs, precision, exec_, regularize, seed=3, eps=0.02):
    kw = dict(m=p.m, n=p.n, rank=8, d=d, precision=precision, exec=exec_, launch="stream",
              regularize=regularize, regularize_lambda=0.05 if regularize == "L2" else 0.0)
    off1 = list(P.block_offsets(p.m, d)) + [p.m]
    ctxs = {}
    ref = P.Context(P.Config(**kw))
    try:
        ref.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ref.set_factors(p.W0, p.H0)
        for r in range(world):
            lo, hi = shard.rank_rows(off1, d, world, r)
            keep = (p.rows >= lo) & (p.rows < hi)
            c = P.Context(P.Config(**kw))
            c.set_matrix(P.TRAIN, p.rows[keep], p.cols[keep], p.vals[keep])
            ctxs[r] = c
        # the update weights are counts over the whole matrix, as the reference's
        n1, n2, _ = ref.nnz12()
        for c in ctxs.values():
            c.set_counts(n1, n2)
            c.set_factors(p.W0, p.H0)
        holder = shard.new_holders(2 * d)
        rng = P.Random32(seed)
        for _ in range(epochs):
            sched, seeds = P.draw_schedule(rng, d, "COWOR")
            ref.epoch_explicit(eps, sched, seeds)
            shard.run_epoch(eps, sched, seeds, d, world, holder, list(range(world)),
                            lambda r, s: ctxs[r].epoch_part(eps, sched, seeds, s, s + 1),
                            lambda moves: shard.local_exchange(ctxs, moves))
        W = np.empty_like(p.W0[:, :8])
        H = np.empty_like(p.H0[:, :8])
        off2 = list(P.block_offsets(p.n, 2 * d)) + [p.n]
        parts = {r: ctxs[r].get_factors() for r in range(world)}
        for r in range(world):
            lo, hi = shard.rank_rows(off1, d, world, r)
            W[lo:hi] = parts[r][0][lo:hi]
        for b in range(2 * d):
            src = holder[b] if holder[b] != shard.EVERYONE else 0
            H[off2[b]:off2[b + 1]] = parts[src][1][off2[b]:off2[b + 1]]
        Wr, Hr = ref.get_factors()
        # with every block shared, the ranks' losses over their entries add up
        # to the single context's
        shard.share_local(ctxs, holder)
        total = sum(ctxs[r].nzsl(P.TRAIN) for r in range(world))
        pred = np.einsum("kz,kz->k", W[p.rows], H[p.cols])
        assert total == pytest.approx(float(np.sum((p.vals - pred) ** 2)), rel=1e-9)
        if precision == "fp64":
            assert total == pytest.approx(ref.nzsl(P.TRAIN), rel=1e-12)
        return W, H, Wr, Hr
    finally:
        ref.close()
        for c in ctxs.values():
            c.close()


@pytest.mark.parametrize("regularize", ["None", "L2"])
@pytest.mark.parametrize("world", [2, 4])
def test_replay_over_ranks_equals_one_context(world, regularize):
    p = synth.make(900, 700, 20000, 100, rank_true=6, r=8, noise=0.1, seed=8)
    W, H, Wr, Hr = _ranks_run(p, 4, world, 3, "fp64", "replay", regularize)
    np.testing.assert_array_equal(W, Wr)
    np.testing.assert_array_equal(H, Hr)


@pytest.mark.parametrize("regularize", ["None", "L2"])
def test_hogwild_over_ranks_tracks_one_context(regularize):
    p = synth.make(4000, 3000, 200000, 100, rank_true=6, r=8, noise=0.1, seed=9)
    W, H, Wr, Hr = _ranks_run(p, 4, 2, 3, "fp32", "hogwild", regularize)
    # Hogwild runs differ run to run; the products on the training entries agree closely
    got = np.einsum("kz,kz->k", W[p.rows], H[p.cols])
    want = np.einsum("kz,kz->k", Wr[p.rows], Hr[p.cols])
    rmse_got = np.sqrt(np.mean((p.vals - got) ** 2))
    rmse_want = np.sqrt(np.mean((p.vals - want) ** 2))
    assert abs(rmse_got - rmse_want) <= 0.005 * rmse_want, (rmse_got, rmse_want)


def test_parts_must_follow_one_another():
    p = synth.make(300, 200, 3000, 100, rank_true=4, r=8, noise=0.1, seed=1)
    with P.Context(P.Config(m=p.m, n=p.n, rank=8, d=2, launch="stream")) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_factors(p.W0, p.H0)
        sched, seeds = P.draw_schedule(P.Random32(1), 2, "COWOR")
        with pytest.raises(P.DsgdppError):
            ctx.epoch_part(0.01, sched, seeds, 1, 2)      # must start at 0
        ctx.epoch_part(0.01, sched, seeds, 0, 1)
        with pytest.raises(P.DsgdppError):
            ctx.epoch(0.01)                              # the epoch in parts is unfinished
        with pytest.raises(P.DsgdppError):
            ctx.epoch_part(0.02, sched, seeds, 1, 4)      # another step size
        ctx.epoch_part(0.01, sched, seeds, 1, 4)
        ctx.epoch(0.01)                                   # whole epochs again


def _gloo_rank(rank, world, port, out):
    import datetime
    import os
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        d, eps = 4, 0.02
        p = synth.make(900, 700, 20000, 100, rank_true=6, r=8, noise=0.1, seed=8)
        kw = dict(m=p.m, n=p.n, rank=8, d=d, precision="fp64", exec="replay", launch="stream")
        off1 = list(P.block_offsets(p.m, d)) + [p.m]
        lo, hi = shard.rank_rows(off1, d, world, rank)
        keep = (p.rows >= lo) & (p.rows < hi)
        with P.Context(P.Config(**kw)) as full, P.Context(P.Config(**kw)) as ctx:
            full.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
            n1, n2, _ = full.nnz12()
            ctx.set_matrix(P.TRAIN, p.rows[keep], p.cols[keep], p.vals[keep])
            ctx.set_counts(n1, n2)
            ctx.set_factors(p.W0, p.H0)
            holder = shard.new_holders(2 * d)
            rng = P.Random32(5)  # every rank draws the same epochs here; a job would
            for _ in range(2):   # draw them on rank 0 and broadcast them
                sched, seeds = P.draw_schedule(rng, d, "COWOR")
                shard.run_epoch(eps, sched, seeds, d, world, holder, [rank],
                                lambda r, s: ctx.epoch_part(eps, sched, seeds, s, s + 1),
                                lambda moves: shard.torch_exchange(dist, rank, ctx, moves, "cpu"))
            W, H = ctx.get_factors()
            out[rank] = (W[lo:hi].copy(), H.copy(), list(holder))
            shard.share_torch(dist, rank, ctx, holder, "cpu")
            loss = torch.tensor([ctx.nzsl(P.TRAIN)], dtype=torch.float64)
            dist.all_reduce(loss)
            out[f"loss{rank}"] = float(loss.item())
            if rank == 0:
                full.set_factors(p.W0, p.H0)
                rng = P.Random32(5)
                for _ in range(2):
                    sched, seeds = P.draw_schedule(rng, d, "COWOR")
                    full.epoch_explicit(eps, sched, seeds)
                out["ref"] = full.get_factors()
                out["ref_loss"] = full.nzsl(P.TRAIN)
    finally:
        dist.destroy_process_group()


def test_two_processes_hand_blocks_over_with_torch_distributed():
    # two ranks as two processes sharing this GPU; they meet only on the host
    # (gloo), never inside a kernel
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    Wr, Hr = out["ref"]
    d = 4
    off1 = list(P.block_offsets(900, d)) + [900]
    off2 = list(P.block_offsets(700, 2 * d)) + [700]
    holder = out[0][2]
    for r in range(2):
        lo, hi = shard.rank_rows(off1, d, 2, r)
        np.testing.assert_array_equal(out[r][0], Wr[lo:hi])
    for b in range(2 * d):
        H = out[holder[b]][1]
        np.testing.assert_array_equal(H[off2[b]:off2[b + 1]], Hr[off2[b]:off2[b + 1]])
    for r in range(2):
        assert out[f"loss{r}"] == pytest.approx(out["ref_loss"], rel=1e-12)


def test_torchrun_job_matches_the_single_context_run(tmp_path):
    # the whole job (BoldDriver, losses over ranks) as two torchrun processes
    # sharing this GPU and meeting over gloo; FP64 replay, so the per-epoch
    # losses must be the single context's
    import json
    import os
    import socket
    import subprocess
    import sys
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    m, n, nnz, ntest, r, d, epochs, seed = 900, 700, 20000, 2000, 8, 4, 4, 6
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", "-m", "dsgdpp_b200.shard",
           f"--synthetic={m},{n},{nnz},{ntest},{r}", f"--tasks={d}", f"--epochs={epochs}",
           f"--seed={seed}", "--precision=fp64", "--exec=replay", "--backend=gloo"]
    env = dict(os.environ, PYTHONPATH=os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stderr[-3000:]
    rows = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert [x["epoch"] for x in rows] == list(range(epochs + 1))
    p = synth.make(m, n, nnz, ntest, rank_true=min(r, 8), r=r, noise=0.1, seed=seed)
    with P.Context(P.Config(m=m, n=n, rank=r, d=d, precision="fp64", exec="replay")) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        ctx.seed(seed)
        trace = ctx.run(epochs, "BoldDriver", 0.001)
    for got, want in zip(rows, trace):
        assert got["loss"] == pytest.approx(want["loss"], rel=1e-11)
        assert got["test_loss"] == pytest.approx(want["test_loss"], rel=1e-11)
        if got["epoch"] > 0:
            assert got["eps"] == pytest.approx(want["eps"], rel=1e-15)
