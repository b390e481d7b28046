"""DSGD++ with its tasks spread over several ranks (one GPU each).

The reference runs d tasks per epoch on the ranks of an MPI job: a task owns
one row block of V and W for the whole run, and the H column blocks move
between ranks between sub-epochs, each to the rank whose task needs it next
(mf/sgd/dsgdpp_impl.h:153-263).  Here each rank holds a context with the
entries of its own tasks' row blocks only (the other tasks' blocks are empty
in it), runs the epoch one sub-epoch at a time (``Context.epoch_part``) and
hands H blocks over in between (``Context.h_block_copy``).  Every rank draws
nothing itself: the schedule and task seeds of an epoch come from rank 0's
master generator, so all ranks follow one epoch, as in the reference.

Tasks are dealt to ranks in contiguous ranges (rank r owns tasks
r*d/world .. (r+1)*d/world - 1; d must be a multiple of world).  Before
sub-epoch s every block that a task uses at s is moved to that task's rank
from the rank that holds its latest version; ``handoff_plan`` lists these
moves for a whole epoch, identically on every rank.

After an epoch, ``share_local`` / ``share_torch`` give every rank every
block's latest version; the training loss is then the sum of the ranks'
losses over their own entries.

With NCCL, ``main`` runs the job through the library's own hand-off
(:class:`dsgdpp_b200.Shard`, ``dsgdpp_shard_*`` in C++): blocks move from H
to H on a transfer stream while the next sub-epoch computes.  The transports
here (``torch_exchange`` over gloo through pinned host buffers,
``local_exchange``) stay for CPU process groups and for tests.

Transports: ``torch_exchange`` moves blocks with torch.distributed
point-to-point operations (NCCL between GPUs; gloo works for host buffers),
``local_exchange`` moves them between contexts of one process (several
emulated ranks run one after another on one GPU -- no kernel waits for
another).
"""
from __future__ import annotations

from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

Move = Tuple[int, int, int]  # (column block, from rank, to rank)
EVERYONE = -1                # every rank holds the block (the starting factors)


def task_owner(d: int, world: int) -> np.ndarray:
    """rank of each task id"""
    if world < 1 or d % world:
        raise ValueError("d must be a multiple of the number of ranks")
    return np.arange(d) // (d // world)


def rank_rows(off1: Sequence[int], d: int, world: int, rank: int) -> Tuple[int, int]:
    """[first, last) row of the rows owned by `rank` (off1: d + 1 row offsets)"""
    per = d // world
    return int(off1[rank * per]), int(off1[(rank + 1) * per])


def new_holders(nb2: int) -> List[int]:
    return [EVERYONE] * nb2


def handoff_plan(schedule: np.ndarray, d: int, world: int, holder: List[int]) -> List[List[Move]]:
    """Moves to make before each sub-epoch of one epoch; updates `holder`
    (the rank holding each block's latest version) as the moves happen.
    schedule: nb2 x d (row = sub-epoch, column = task id, entry = block)."""
    owner = task_owner(d, world)
    sched = np.asarray(schedule, np.int64).reshape(-1, d)
    plan: List[List[Move]] = []
    for s in range(sched.shape[0]):
        moves = []
        for task in range(d):
            b2 = int(sched[s, task])
            dst = int(owner[task])
            if holder[b2] != EVERYONE and holder[b2] != dst:
                moves.append((b2, holder[b2], dst))
            holder[b2] = dst
        plan.append(moves)
    return plan


def local_exchange(ctxs: Dict[int, object], moves: List[Move], device: int = 0):
    """Moves between contexts of this process (emulated ranks)."""
    import torch
    for b2, src, dst in moves:
        nbytes = ctxs[src].h_block_bytes(b2)
        buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=f"cuda:{device}")
        ctxs[src].h_block_copy(b2, buf.data_ptr(), False)
        ctxs[dst].h_block_copy(b2, buf.data_ptr(), True)


def torch_exchange(pg, rank: int, ctx, moves: List[Move], device: str = "cuda"):
    """This rank's part of the moves, as one batch of torch.distributed
    point-to-point operations (every rank calls it with the same moves).
    With NCCL, torch wants every rank in the group's first communication, so
    a collective (the schedule broadcast of the job) must come first; ranks
    without a move in a sub-epoch then simply skip the batch."""
    import torch
    ops, recvs = [], []
    for b2, src, dst in moves:
        if rank not in (src, dst):
            continue
        nbytes = ctx.h_block_bytes(b2)
        pin = device == "cpu" and torch.cuda.is_available()  # host buffers the GPU copies into
        buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device, pin_memory=pin)
        if rank == src:
            ctx.h_block_copy(b2, buf.data_ptr(), False)
            ops.append(pg.P2POp(pg.isend, buf, dst))
        else:
            ops.append(pg.P2POp(pg.irecv, buf, src))
            recvs.append((b2, buf))
    if ops:
        for w in pg.batch_isend_irecv(ops):
            w.wait()
    if device != "cpu":
        torch.cuda.synchronize()
    for b2, buf in recvs:
        ctx.h_block_copy(b2, buf.data_ptr(), True)


def share_local(ctxs: Dict[int, object], holder: List[int], device: int = 0):
    """Every context gets every block's latest version (emulated ranks)."""
    import torch
    for b2, src in enumerate(holder):
        if src == EVERYONE:
            continue
        nbytes = ctxs[src].h_block_bytes(b2)
        buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=f"cuda:{device}")
        ctxs[src].h_block_copy(b2, buf.data_ptr(), False)
        for r, c in ctxs.items():
            if r != src:
                c.h_block_copy(b2, buf.data_ptr(), True)
        holder[b2] = EVERYONE


def share_torch(pg, rank: int, ctx, holder: List[int], device: str = "cuda"):
    """Every rank gets every block's latest version: one broadcast per block
    from its holder, in block order on every rank.  Needed before the training
    loss (a rank's entries touch every column block) and makes the next
    epoch's hand-off start from blocks that every rank holds."""
    import torch
    for b2, src in enumerate(holder):
        if src == EVERYONE:
            continue
        nbytes = ctx.h_block_bytes(b2)
        pin = device == "cpu" and torch.cuda.is_available()
        buf = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device, pin_memory=pin)
        if rank == src:
            ctx.h_block_copy(b2, buf.data_ptr(), False)
        pg.broadcast(buf, src=src)
        if device != "cpu":
            torch.cuda.synchronize()
        if rank != src:
            ctx.h_block_copy(b2, buf.data_ptr(), True)
        holder[b2] = EVERYONE


def run_epoch(eps: float, schedule: np.ndarray, seeds: np.ndarray, d: int, world: int,
              holder: List[int], ranks: Sequence[int],
              epoch_part: Callable[[int, int], None],
              exchange: Callable[[List[Move]], None]):
    """One epoch over the ranks this process drives: before each sub-epoch the
    plan's moves, then that sub-epoch on every driven rank."""
    plan = handoff_plan(schedule, d, world, holder)
    nb2 = len(plan)
    for s in range(nb2):
        exchange(plan[s])
        for r in ranks:
            epoch_part(r, s)


# ---- a whole job over torchrun ranks ---------------------------------------------------
def _bold_driver(eps: float, prev: float, cur: float, dec: float = 0.5, inc: float = 1.05) -> float:
    """BoldDriver (mf/sgd/decay/decay_bolddriver.h:59-67)"""
    return eps * (dec if prev <= cur else inc)


def _run_library_shard(args, ctx, rank, world, d, dist):
    """The job over NCCL through the library's hand-off (dsgdpp_shard_*): the
    transfers overlap the sub-epochs in between, the schedule comes from every
    rank's master generator seeded alike."""
    import json
    from . import Shard, shard_unique_id
    per = d // world
    ctx.set_tasks(rank * per, per)
    ctx.seed(args.seed)
    uid = [shard_unique_id() if rank == 0 else None]
    dist.broadcast_object_list(uid, src=0)
    with Shard.nccl(ctx, rank, world, uid[0]) as sh:
        sh.share()
        loss, test = sh.losses()
        if rank == 0:
            print(json.dumps({"epoch": 0, "loss": loss, "test_loss": test}), flush=True)
        eps, prev = args.eps0, None
        for e in range(1, args.epochs + 1):
            if prev is not None:
                eps = _bold_driver(eps, prev, loss)
            sh.epoch(eps)
            sh.share()
            prev = loss
            loss, test = sh.losses()
            if rank == 0:
                print(json.dumps({"epoch": e, "loss": loss, "test_loss": test, "eps": eps}),
                      flush=True)


def main(argv=None):
    """DSGD++ over torchrun ranks with BoldDriver, one GPU per rank:

        torchrun --nproc-per-node G -m dsgdpp_b200.shard --tasks D --epochs E \\
            --input-file V.mmc --input-test-file T.mmc --input-row-file W.mma --input-col-file H.mma

    or --synthetic M,N,NNZ,NTEST,RANK for seeded synthetic data.  Prints one
    JSON line per epoch on rank 0 (training and test loss, step)."""
    import argparse
    import datetime
    import json
    import os
    import torch
    import torch.distributed as dist
    from . import Config, Context, Random32, TEST, TRAIN, block_offsets, draw_schedule
    from . import read_mm_array, read_sparse, synth

    ap = argparse.ArgumentParser(prog="python -m dsgdpp_b200.shard")
    ap.add_argument("--input-file"); ap.add_argument("--input-test-file")
    ap.add_argument("--input-row-file"); ap.add_argument("--input-col-file")
    ap.add_argument("--synthetic", help="M,N,NNZ,NTEST,RANK")
    ap.add_argument("--tasks", type=int, required=True)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--eps0", type=float, default=0.001)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--exec", default="hogwild")
    ap.add_argument("--loss-lambda", type=float, default=1.0)
    ap.add_argument("--backend", default="nccl")
    args = ap.parse_args(argv)

    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    dev = local % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    dist.init_process_group(args.backend, timeout=datetime.timedelta(seconds=300))
    xdev = "cuda" if args.backend == "nccl" else "cpu"
    try:
        if args.synthetic:
            m, n, nnz, ntest, r = (int(x) for x in args.synthetic.split(","))
            p = synth.make(m, n, nnz, ntest, rank_true=min(r, 8), r=r, noise=0.1, seed=args.seed)
            rows, cols, vals = p.rows, p.cols, p.vals
            trows, tcols, tvals = p.trows, p.tcols, p.tvals
            W0, H0 = p.W0, p.H0
        else:
            m, n, rows, cols, vals = read_sparse(args.input_file)
            _, _, trows, tcols, tvals = read_sparse(args.input_test_file)
            W0 = read_mm_array(args.input_row_file)
            H0 = np.ascontiguousarray(read_mm_array(args.input_col_file).T)
            r = W0.shape[1]
        d = args.tasks
        off1 = list(block_offsets(m, d)) + [m]
        lo, hi = rank_rows(off1, d, world, rank)
        keep = (rows >= lo) & (rows < hi)
        tkeep = (trows >= lo) & (trows < hi)
        ctx = Context(Config(m=m, n=n, rank=r, d=d, precision=args.precision, exec=args.exec,
                             launch="stream", device=dev, loss_lambda=args.loss_lambda))
        ctx.set_matrix(TRAIN, rows[keep], cols[keep], vals[keep])
        ctx.set_matrix(TEST, trows[tkeep], tcols[tkeep], tvals[tkeep])
        ctx.set_counts(np.bincount(rows, minlength=m).astype(np.uint64),
                       np.bincount(cols, minlength=n).astype(np.uint64))
        Wz = np.zeros_like(W0)  # rows of other ranks stay zero: they add nothing to L2 here
        Wz[lo:hi] = W0[lo:hi]
        ctx.set_factors(Wz, H0)
        if args.backend == "nccl":
            _run_library_shard(args, ctx, rank, world, d, dist)
            ctx.close()
            return
        holder = new_holders(2 * d)

        def job_losses():
            share_torch(dist, rank, ctx, holder, xdev)
            w2, h2 = ctx.l2()
            t = torch.tensor([ctx.nzsl(TRAIN), w2, ctx.nzsl(TEST)], dtype=torch.float64,
                             device=xdev)
            dist.all_reduce(t)
            a = t.cpu().numpy()
            return a[0] + args.loss_lambda * (a[1] + h2), a[2]

        master = Random32(args.seed)
        loss, test = job_losses()
        if rank == 0:
            print(json.dumps({"epoch": 0, "loss": loss, "test_loss": test}), flush=True)
        eps, prev = args.eps0, None
        for e in range(1, args.epochs + 1):
            if prev is not None:
                eps = _bold_driver(eps, prev, loss)
            sched, seeds = draw_schedule(master, d)
            t = torch.from_numpy(np.concatenate([sched.ravel(), seeds]).astype(np.int64)).to(xdev)
            dist.broadcast(t, 0)  # rank 0's draws for every rank
            a = t.cpu().numpy().astype(np.uint32)
            sched, seeds = a[:2 * d * d].reshape(2 * d, d), a[2 * d * d:]
            run_epoch(eps, sched, seeds, d, world, holder, [rank],
                      lambda _r, s: ctx.epoch_part(eps, sched, seeds, s, s + 1),
                      lambda moves: torch_exchange(dist, rank, ctx, moves, xdev))
            prev = loss
            loss, test = job_losses()
            if rank == 0:
                print(json.dumps({"epoch": e, "loss": loss, "test_loss": test, "eps": eps}),
                      flush=True)
        ctx.close()
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
