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


# ---- the library's hand-off (dsgdpp_shard_*): transfers on a stream of their own ----
def _shard_contexts(p, d, world, kw, seed):
    """Rank r's context: its tasks' rows of the training and test entries, the
    counts of the whole matrix, its own W rows (the others zero)."""
    off1 = list(P.block_offsets(p.m, d)) + [p.m]
    n1 = np.bincount(p.rows, minlength=p.m).astype(np.uint64)
    n2 = np.bincount(p.cols, minlength=p.n).astype(np.uint64)
    ctxs = []
    for r in range(world):
        lo, hi = shard.rank_rows(off1, d, world, r)
        keep = (p.rows >= lo) & (p.rows < hi)
        tkeep = (p.trows >= lo) & (p.trows < hi)
        c = P.Context(P.Config(**kw))
        c.set_tasks(r * (d // world), d // world)
        c.set_matrix(P.TRAIN, p.rows[keep], p.cols[keep], p.vals[keep])
        c.set_matrix(P.TEST, p.trows[tkeep], p.tcols[tkeep], p.tvals[tkeep])
        c.set_counts(n1, n2)
        Wz = np.zeros_like(p.W0)
        Wz[lo:hi] = p.W0[lo:hi]
        c.set_factors(Wz, p.H0)
        c.seed(seed)
        ctxs.append(c)
    return ctxs, off1


def _gather(ctxs, off1, d, world):
    W = ctxs[0].get_factors()[0].copy()
    for r, c in enumerate(ctxs):
        lo, hi = shard.rank_rows(off1, d, world, r)
        W[lo:hi] = c.get_factors()[0][lo:hi]
    return W, ctxs[0].get_factors()[1]


@pytest.mark.parametrize("method", ["dsgdpp", "dsgd"])
@pytest.mark.parametrize("regularize", ["None", "L2"])
@pytest.mark.parametrize("world", [2, 4])
def test_library_shard_replay_equals_one_context(world, regularize, method):
    p = synth.make(900, 700, 20000, 2000, rank_true=6, r=8, noise=0.1, seed=8)
    d, eps = 4, 0.02
    kw = dict(m=p.m, n=p.n, rank=8, d=d, precision="fp64", exec="replay", launch="stream",
              regularize=regularize, regularize_lambda=0.05 if regularize == "L2" else 0.0,
              loss="Nzsl_L2", loss_lambda=0.1, method=method)
    ctxs, off1 = _shard_contexts(p, d, world, kw, seed=3)
    ref = P.Context(P.Config(**kw))
    try:
        ref.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ref.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ref.set_factors(p.W0, p.H0)
        ref.seed(3)
        with P.Shard.local(ctxs) as sh:
            moved = 0
            for _ in range(3):
                ref.epoch(eps)  # both draw from a master generator seeded 3
                sh.epoch(eps)
                moved += sh.moved()[0]
                sh.share()
                loss, test = sh.losses()
                assert loss == pytest.approx(ref.loss(), rel=1e-12)
                assert test == pytest.approx(ref.nzsl(P.TEST), rel=1e-12)
            assert moved > 0
        W, H = _gather(ctxs, off1, d, world)
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)
        for c in ctxs[1:]:  # after share every rank holds all of H
            np.testing.assert_array_equal(c.get_factors()[1], Hr)
    finally:
        ref.close()
        for c in ctxs:
            c.close()


@pytest.mark.parametrize("precision,tol", [("fp32", 0.005), ("bf16", 0.01)])
def test_library_shard_hogwild_tracks_one_context(precision, tol):
    p = synth.make(40000, 20000, 800000, 20000, rank_true=8, r=16, noise=0.1, seed=9)
    d, world = 8, 4
    kw = dict(m=p.m, n=p.n, rank=16, d=d, precision=precision, exec="hogwild",
              launch="stream", regularize="L2", regularize_lambda=0.05)
    ctxs, off1 = _shard_contexts(p, d, world, kw, seed=5)
    ref = P.Context(P.Config(**dict(kw, launch="graph")))
    try:
        ref.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ref.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ref.set_factors(p.W0, p.H0)
        ref.seed(5)
        with P.Shard.local(ctxs) as sh:
            for _ in range(6):
                ref.epoch(0.01)
                sh.epoch(0.01)
                sh.share()
            _, test = sh.losses()
        got = np.sqrt(test / len(p.tvals))
        want = np.sqrt(ref.nzsl(P.TEST) / len(p.tvals))
        assert abs(got - want) <= tol * want, (got, want)
    finally:
        ref.close()
        for c in ctxs:
            c.close()


def test_library_shard_transfers_overlap_the_next_sub_epoch():
    # two emulated ranks: a block used at sub-epoch s travels on the transfer
    # stream while sub-epoch s + 1 (the other colour) computes, and sub-epoch
    # s + 1 does not wait for it.  Both ranks share one GPU here, so whether a
    # copy finds room beside the running sub-epochs varies from epoch to epoch:
    # the ordering holds in every epoch, the overlap in at least one of three.
    p = synth.make(200000, 400000, 2000000, 100, rank_true=8, r=32, noise=0.1, seed=4)
    d, world = 4, 2
    kw = dict(m=p.m, n=p.n, rank=32, d=d, precision="fp32", exec="hogwild", launch="stream")
    ctxs, _ = _shard_contexts(p, d, world, kw, seed=2)
    try:
        with P.Shard.local(ctxs) as sh:
            sh.epoch(0.01)
            sh.share()
            sh.set_timeline(True)
            seen = []
            for _ in range(3):
                sh.epoch(0.01)
                moves, nbytes = sh.moved()
                assert moves > 0 and nbytes > 0
                overlapped = total = 0
                for r in range(world):
                    comp, xfer = sh.timeline(r, 2 * d)
                    for g in range(1, 2 * d - 1):  # posted after sub-epoch g - 1
                        if np.isnan(xfer[g, 0]):
                            continue
                        total += 1
                        assert xfer[g, 0] >= comp[g - 1, 1] - 1e-3  # after the sub-epoch that used it
                        # it travels while sub-epoch g computes: it begins before g ends
                        if xfer[g, 0] < comp[g, 1] and xfer[g, 1] > comp[g, 0]:
                            overlapped += 1
                assert total > 0
                seen.append((overlapped, total))
            assert any(o >= t // 2 for o, t in seen), seen
    finally:
        for c in ctxs:
            c.close()


def test_library_shard_checks_its_contexts():
    p = synth.make(300, 200, 3000, 100, rank_true=4, r=8, noise=0.1, seed=1)
    kw = dict(m=p.m, n=p.n, rank=8, d=4, launch="stream")
    a, b = P.Context(P.Config(**kw)), P.Context(P.Config(**kw))
    try:
        with pytest.raises(P.DsgdppError):  # the task ranges were not set
            P.Shard.local([a, b])
        a.set_tasks(0, 2)
        b.set_tasks(2, 2)
        a.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)  # rows of rank 1 in rank 0's context
        a.set_factors(p.W0, p.H0)
        b.set_matrix(P.TRAIN, [], [], [])
        b.set_factors(p.W0, p.H0)
        with P.Shard.local([a, b]) as sh:
            with pytest.raises(P.DsgdppError, match="does not run here"):
                sh.epoch(0.01)
        with pytest.raises(P.DsgdppError):
            a.set_tasks(3, 2)
    finally:
        a.close()
        b.close()


def test_library_shard_over_nccl_with_one_rank_equals_one_context():
    # the NCCL transport's plumbing on one GPU (one rank: nothing moves)
    p = synth.make(900, 700, 20000, 2000, rank_true=6, r=8, noise=0.1, seed=8)
    kw = dict(m=p.m, n=p.n, rank=8, d=4, precision="fp64", exec="replay", launch="stream")
    ctxs, _ = _shard_contexts(p, 4, 1, kw, seed=3)
    ref = P.Context(P.Config(**kw))
    try:
        ref.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ref.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ref.set_factors(p.W0, p.H0)
        ref.seed(3)
        with P.Shard.nccl(ctxs[0], 0, 1, P.shard_unique_id()) as sh:
            for _ in range(2):
                ref.epoch(0.02)
                sh.epoch(0.02)
                sh.share()
                loss, test = sh.losses()
                assert loss == pytest.approx(ref.loss(), rel=1e-12)
                assert test == pytest.approx(ref.nzsl(P.TEST), rel=1e-12)
        np.testing.assert_array_equal(ctxs[0].get_factors()[1], ref.get_factors()[1])
    finally:
        ref.close()
        ctxs[0].close()
