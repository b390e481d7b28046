"""CPU tests of the multi-rank DSGD++ hand-off (dsgdpp_b200/shard.py): the
plan of H-block moves, and two gloo ranks moving blocks whose contents record
every task that updated them, against one process running all tasks."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dsgdpp_b200 import shard


def _schedules(d, epochs, seed):
    import dsgdpp_b200 as P
    rng = P.Random32(seed)
    return [P.draw_schedule(rng, d, "COWOR") for _ in range(epochs)]


def test_plan_puts_every_block_on_its_task_rank():
    d, world = 6, 3
    owner = shard.task_owner(d, world)
    holder = shard.new_holders(2 * d)
    where = [shard.EVERYONE] * (2 * d)  # replayed independently of the plan's own bookkeeping
    for sched, _ in _schedules(d, 3, 5):
        plan = shard.handoff_plan(sched, d, world, holder)
        assert len(plan) == 2 * d
        for s, moves in enumerate(plan):
            assert len({m[0] for m in moves}) == len(moves)  # a block moves at most once
            for b2, src, dst in moves:
                assert src == where[b2] and src != dst
                where[b2] = dst
            for task in range(d):
                b2 = int(sched[s, task])
                # the block is with its task's rank (or still with every rank)
                assert where[b2] in (owner[task], shard.EVERYONE)
                where[b2] = owner[task]
        assert where == holder


@pytest.mark.parametrize("world", [1, 2, 4])
@pytest.mark.parametrize("method", ["dsgdpp", "dsgd"])
def test_library_plan_matches_the_python_plan(world, method):
    # dsgdpp_shard_plan (the C++ hand-off) posts each move right after the
    # block's previous use; its moves are the Python plan's, block for block
    import dsgdpp_b200 as P
    d = 8
    nb2 = 2 * d if method == "dsgdpp" else d
    rng = P.Random32(11)
    holder_py = shard.new_holders(nb2)
    holder_c = np.full(nb2, -1, np.int32)
    for e in range(3):
        if method == "dsgdpp":
            sched, _ = P.draw_schedule(rng, d, "COWOR")
        else:
            sched = P.dsgd_schedule(rng, 1, d, "COWOR")
        before = holder_c.copy()
        plan = shard.handoff_plan(sched, d, world, holder_py)
        moves, holder_c = P.shard_plan(d, nb2, world, sched, holder_c)
        assert list(holder_c) == holder_py
        # the group of a move = one past the block's previous use in the epoch
        last = {}
        want = []
        for s in range(nb2):
            for b2, src, dst in plan[s]:
                want.append((last.get(b2, -1) + 1, b2, src, dst))
            for t in range(d):
                last[int(sched[s, t])] = s
        assert sorted(map(tuple, moves.tolist())) == sorted(want)
        if method == "dsgdpp":
            # red/blue: inside an epoch a block moves while the other colour computes
            inner = [m for m in moves.tolist() if m[0] > 0]
            for g, b2, _, _ in inner:
                nxt = min(s for s in range(g, nb2) if b2 in set(sched[s].tolist()))
                assert nxt >= g + 1  # used again no earlier than two sub-epochs later
        if (before == -1).all():  # every rank holds every block: nothing moves before the epoch
            assert all(m[0] > 0 for m in moves.tolist())
        if world == 1:
            assert len(moves) == 0


def test_task_ranges_need_a_multiple():
    with pytest.raises(ValueError):
        shard.task_owner(5, 2)
    assert list(shard.task_owner(4, 2)) == [0, 0, 1, 1]


class _FakeCtx:
    """Blocks of int64 whose contents fold in every (sub-epoch, task) visit."""

    def __init__(self, nb2, tasks, d, width=4):
        self.blocks = {b: np.zeros(width, np.int64) for b in range(nb2)}
        self.tasks, self.d = tasks, d

    def visit(self, sched, s, epoch):
        for task in self.tasks:
            b = int(sched[s, task])
            self.blocks[b] = (self.blocks[b] * 31 + (epoch * 1000 + s * self.d + task + 1)) % (1 << 40)

    def h_block_bytes(self, b2):
        return self.blocks[b2].nbytes

    def h_block_copy(self, b2, ptr, to_context):
        a = self.blocks[b2]
        if to_context:
            ctypes.memmove(a.ctypes.data, ptr, a.nbytes)
        else:
            ctypes.memmove(ptr, a.ctypes.data, a.nbytes)


def _rank(rank, world, port, d, epochs, out):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        owner = shard.task_owner(d, world)
        ctx = _FakeCtx(2 * d, [t for t in range(d) if owner[t] == rank], d)
        holder = shard.new_holders(2 * d)
        for e, (sched, _) in enumerate(_schedules(d, epochs, 9)):
            shard.run_epoch(0.0, sched, None, d, world, holder, [rank],
                            lambda r, s: ctx.visit(sched, s, e),
                            lambda moves: shard.torch_exchange(dist, rank, ctx, moves, "cpu"))
        shard.share_torch(dist, rank, ctx, holder, "cpu")  # every rank gets every block
        assert holder == shard.new_holders(2 * d)
        out[rank] = {b: ctx.blocks[b].tolist() for b in range(2 * d)}
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_hand_blocks_over_as_one_process_would():
    d, world, epochs = 4, 2, 3
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctxm = mp.get_context("spawn")
    out = ctxm.Manager().dict()
    procs = [ctxm.Process(target=_rank, args=(r, world, port, d, epochs, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    ref = _FakeCtx(2 * d, list(range(d)), d)
    for e, (sched, _) in enumerate(_schedules(d, epochs, 9)):
        for s in range(2 * d):
            ref.visit(sched, s, e)
    want = {b: ref.blocks[b].tolist() for b in range(2 * d)}
    assert out[0] == want and out[1] == want
