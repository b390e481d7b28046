"""Seeded synthetic matrices of the benchmark shapes, generated on the GPU.

Same distributions as :mod:`dsgdpp_b200.synth`, sized for 100M+ entries:
positions are drawn with replacement from the row and column weight
distributions (uniform, or Zipf(s) over randomly permuted ids) and duplicate
pairs are rejected until enough distinct pairs exist, then a uniformly random
subset of the distinct pairs is kept and split into training and test
entries.  With Zipf(1.1) on both sides the heaviest rows and columns saturate
(every column of a head row is filled), so several times more draws than
entries are needed.  torch is used here only to produce input data.
"""
from __future__ import annotations

import math

import numpy as np


def _weights(torch, g, size, s, device):
    if s is None:
        return None
    w = 1.0 / torch.arange(1, size + 1, device=device, dtype=torch.float64) ** s
    perm = torch.randperm(size, generator=g, device=device)
    out = torch.empty_like(w)
    out[perm] = w
    c = torch.cumsum(out, 0)
    return (c / c[-1]).to(torch.float64)


def _draw(torch, g, cdf, size, count, device):
    if cdf is None:
        return torch.randint(0, size, (count,), generator=g, device=device, dtype=torch.int64)
    u = torch.rand(count, generator=g, device=device, dtype=torch.float64)
    return torch.clamp(torch.searchsorted(cdf, u), max=size - 1)


def _cdf(torch, w):
    c = torch.cumsum(w.to(torch.float64), 0)
    return c / c[-1]


def distinct_pairs(m, n, total, seed, s_row=None, s_col=None, device="cuda", row_weights=None):
    """`total` distinct (row, col) keys; rows by Zipf(s_row) (or `row_weights`,
    a length-m tensor), columns by Zipf(s_col); None = uniform."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    cr = _cdf(torch, row_weights) if row_weights is not None else _weights(torch, g, m, s_row, device)
    cc = _weights(torch, g, n, s_col, device)
    keys = torch.empty(0, dtype=torch.int64, device=device)
    rounds = 0
    while keys.numel() < total:
        need = total - keys.numel()
        count = int(min(400_000_000, max(2 * need, 1_000_000)))
        i = _draw(torch, g, cr, m, count, device)
        j = _draw(torch, g, cc, n, count, device)
        k = i * n + j
        del i, j
        keys = torch.unique(torch.cat([keys, k]))
        del k
        rounds += 1
        if rounds > 40:
            raise RuntimeError("too few distinct pairs: distribution too skewed")
    sel = torch.randperm(keys.numel(), generator=g, device=device)[:total]
    return keys[sel], g


def make(m, n, nnz, nnz_test, rank_true, r, noise, seed, s_row=None, s_col=None,
         device="cuda", chunk=8_000_000):
    """Returns host arrays: rows, cols (uint32), vals (float64) of the training
    and test entries, and the initial factors W0 (m x r), H0 (n x r)."""
    import torch
    keys, g = distinct_pairs(m, n, nnz + nnz_test, seed, s_row, s_col, device)
    rows = (keys // n).to(torch.int32)
    cols = (keys % n).to(torch.int32)
    del keys
    Ws = torch.randn(m, rank_true, generator=g, device=device) / math.sqrt(rank_true)
    Hs = torch.randn(n, rank_true, generator=g, device=device) / math.sqrt(rank_true)
    vals = torch.empty(rows.numel(), dtype=torch.float64, device=device)
    for a in range(0, rows.numel(), chunk):
        b = min(a + chunk, rows.numel())
        ri, ci = rows[a:b].long(), cols[a:b].long()
        v = (Ws[ri] * Hs[ci]).sum(1).double()
        v += noise * torch.randn(b - a, generator=g, device=device, dtype=torch.float64)
        vals[a:b] = v
    del Ws, Hs
    W0 = torch.rand(m, r, generator=g, device=device, dtype=torch.float64) - 0.5
    H0 = torch.rand(n, r, generator=g, device=device, dtype=torch.float64) - 0.5
    out = dict(
        rows=rows[:nnz].cpu().numpy().view(np.uint32), cols=cols[:nnz].cpu().numpy().view(np.uint32),
        vals=vals[:nnz].cpu().numpy(),
        trows=rows[nnz:].cpu().numpy().view(np.uint32),
        tcols=cols[nnz:].cpu().numpy().view(np.uint32), tvals=vals[nnz:].cpu().numpy(),
        W0=W0.cpu().numpy(), H0=H0.cpu().numpy())
    del rows, cols, vals, W0, H0
    torch.cuda.empty_cache()
    return out


def make_ratings(m, n, nnz, nnz_test, r, seed, mu=4.2, sigma=1.3, s_col=0.9, rank_true=16,
                 mean=3.6, std=1.1, device="cuda", chunk=8_000_000):
    """Netflix-shaped stand-in: row degrees lognormal(mu, sigma) capped at n,
    column popularity Zipf(s_col), integer ratings 1..5 from rounding and
    clipping a rank-`rank_true` truth scaled to the given mean and std."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1)
    deg = torch.exp(mu + sigma * torch.randn(m, generator=g, device=device, dtype=torch.float64))
    deg = torch.clamp(deg, max=float(n))
    keys, g = distinct_pairs(m, n, nnz + nnz_test, seed, None, s_col, device, row_weights=deg)
    rows = (keys // n).to(torch.int32)
    cols = (keys % n).to(torch.int32)
    del keys
    U = torch.randn(m, rank_true, generator=g, device=device) / math.sqrt(rank_true)
    V = torch.randn(n, rank_true, generator=g, device=device) / math.sqrt(rank_true)
    vals = torch.empty(rows.numel(), dtype=torch.float64, device=device)
    for a in range(0, rows.numel(), chunk):
        b = min(a + chunk, rows.numel())
        z = (U[rows[a:b].long()] * V[cols[a:b].long()]).sum(1).double()
        vals[a:b] = torch.clamp(torch.round(mean + std * z), 1.0, 5.0)
    del U, V
    W0 = torch.rand(m, r, generator=g, device=device, dtype=torch.float64) - 0.5
    H0 = torch.rand(n, r, generator=g, device=device, dtype=torch.float64) - 0.5
    out = dict(
        rows=rows[:nnz].cpu().numpy().view(np.uint32), cols=cols[:nnz].cpu().numpy().view(np.uint32),
        vals=vals[:nnz].cpu().numpy(),
        trows=rows[nnz:].cpu().numpy().view(np.uint32),
        tcols=cols[nnz:].cpu().numpy().view(np.uint32), tvals=vals[nnz:].cpu().numpy(),
        W0=W0.cpu().numpy(), H0=H0.cpu().numpy())
    del rows, cols, vals, W0, H0
    torch.cuda.empty_cache()
    return out
