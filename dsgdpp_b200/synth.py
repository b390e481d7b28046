"""Seeded synthetic matrices of the DSGD++ benchmark shapes.

The reference benchmarks on Netflix / KDD-Cup data (not available here) and on
matrices from its own generator (mf/matrix/op/generate.h, tools/mfgenerate.cc).
These generators produce stand-ins of the stated shapes and distributions:

* uniform:  positions uniform over distinct (i, j) pairs;
* zipf:     row and column degrees Zipf(s), positions drawn by degree weight
            (ids randomly permuted so heavy rows spread over all blocks),
            duplicates rejected;
values are a rank-k ground truth W* H* (entries N(0,1)/sqrt(k)) plus
N(0, noise^2); initial factors are U[-0.5, 0.5].
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Problem:
    m: int
    n: int
    rows: np.ndarray      # uint32, 0-based
    cols: np.ndarray
    vals: np.ndarray      # float64
    trows: np.ndarray
    tcols: np.ndarray
    tvals: np.ndarray
    W0: np.ndarray        # m x r
    H0: np.ndarray        # n x r (column j of H contiguous)


def _distinct_uniform(rng, m, n, count):
    keys = np.empty(0, np.uint64)
    while len(keys) < count:
        need = int((count - len(keys)) * 1.1) + 16
        k = rng.integers(0, m * n, size=need, dtype=np.uint64)
        keys = np.unique(np.concatenate([keys, k]))
    keys = rng.permutation(keys)[:count]
    return keys


def _zipf_weights(rng, size, s):
    w = 1.0 / np.arange(1, size + 1, dtype=np.float64) ** s
    return rng.permutation(w / w.sum())


def _distinct_weighted(rng, m, n, count, s_row, s_col, max_rounds=60):
    pr = _zipf_weights(rng, m, s_row)
    pc = _zipf_weights(rng, n, s_col)
    cr, cc = np.cumsum(pr), np.cumsum(pc)
    keys = np.empty(0, np.uint64)
    for _ in range(max_rounds):
        if len(keys) >= count:
            break
        need = int((count - len(keys)) * 1.3) + 16
        i = np.minimum(np.searchsorted(cr, rng.random(need)), m - 1).astype(np.uint64)
        j = np.minimum(np.searchsorted(cc, rng.random(need)), n - 1).astype(np.uint64)
        keys = np.unique(np.concatenate([keys, i * np.uint64(n) + j]))
    if len(keys) < count:
        raise ValueError("degree distribution too skewed for this many distinct entries")
    return rng.permutation(keys)[:count]


def make(m, n, nnz, nnz_test, rank_true, r, noise, seed, kind="uniform", s_row=1.1,
         s_col=1.1):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        keys = _distinct_uniform(rng, m, n, nnz + nnz_test)
    else:
        keys = _distinct_weighted(rng, m, n, nnz + nnz_test, s_row, s_col)
    rows = (keys // np.uint64(n)).astype(np.uint32)
    cols = (keys % np.uint64(n)).astype(np.uint32)
    Ws = rng.standard_normal((m, rank_true)) / np.sqrt(rank_true)
    Hs = rng.standard_normal((n, rank_true)) / np.sqrt(rank_true)
    vals = np.einsum("ij,ij->i", Ws[rows], Hs[cols]) + noise * rng.standard_normal(len(keys))
    W0 = rng.uniform(-0.5, 0.5, (m, r))
    H0 = rng.uniform(-0.5, 0.5, (n, r))
    return Problem(m, n, rows[:nnz], cols[:nnz], vals[:nnz], rows[nnz:], cols[nnz:],
                   vals[nnz:], W0, H0)


def quickstart(out_dir="/tmp/", size1=100000, size2=100000, nnz=1000000, nnz_test=100000,
               r=10, seed=0):
    """The four files of the reference's quick start, as tools/generateSyntheticData.cc
    writes them (its sizes are the defaults here): truth factors W* (size1 x r)
    and H* (r x size2) with N(0, 10) entries; train.mmc with `nnz` distinct
    uniformly drawn cells, value w*_i . h*_j plus N(0, 1) noise; test.mmc with
    `nnz_test` cells drawn apart, without noise; W.mma (size1 x r) and H.mma
    (r x size2) with U[-0.5, 0.5] entries.  Cells are listed row by row, as
    the reference's sequential sampling emits them.  The draws are this
    module's own (seeded numpy), not the reference's generator: the same
    shapes and distributions, not the same numbers."""
    import os

    import dsgdpp_b200 as P

    if max(nnz, nnz_test) > size1 * size2:  # mf/matrix/op/generate.h:209-211
        raise ValueError("nnz must be less than matrix size")
    rng = np.random.default_rng(seed)
    sigma = np.sqrt(10.0)
    Ws = rng.normal(0.0, sigma, (size1, r))
    Hs = rng.normal(0.0, sigma, (size2, r))

    def cells(count):
        keys = np.sort(_distinct_uniform(rng, size1, size2, count))
        return (keys // np.uint64(size2)).astype(np.uint32), (keys % np.uint64(size2)).astype(np.uint32)

    rows, cols = cells(nnz)
    vals = np.einsum("ij,ij->i", Ws[rows], Hs[cols]) + rng.standard_normal(nnz)
    trows, tcols = cells(nnz_test)
    tvals = np.einsum("ij,ij->i", Ws[trows], Hs[tcols])
    W0 = rng.uniform(-0.5, 0.5, (size1, r))
    H0 = rng.uniform(-0.5, 0.5, (r, size2))
    P.write_mm_coord(os.path.join(out_dir, "train.mmc"), size1, size2, rows, cols, vals)
    P.write_mm_coord(os.path.join(out_dir, "test.mmc"), size1, size2, trows, tcols, tvals)
    P.write_mm_array(os.path.join(out_dir, "W.mma"), W0)
    P.write_mm_array(os.path.join(out_dir, "H.mma"), H0)


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser(
        description="write train.mmc, test.mmc, W.mma and H.mma as "
                    "tools/generateSyntheticData.cc does (own seeded draws)")
    ap.add_argument("--out-dir", default="/tmp/")
    ap.add_argument("--size1", type=int, default=100000)
    ap.add_argument("--size2", type=int, default=100000)
    ap.add_argument("--nnz", type=int, default=1000000)
    ap.add_argument("--nnz-test", type=int, default=100000)
    ap.add_argument("--rank", type=int, default=10)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args()
    quickstart(a.out_dir, a.size1, a.size2, a.nnz, a.nnz_test, a.rank, a.seed)
