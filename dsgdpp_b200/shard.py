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
    point-to-point operations (every rank calls it with the same moves)."""
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
