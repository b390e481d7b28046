"""A second, pure-Python restatement of the DSGD++ epoch for tiny cases.

Written independently of oracle/dsgdpp_oracle.cc from the reference sources
(mf/sgd/dsgdpp_impl.h, mf/sgd/dsgd_impl.h, mf/matrix/op/shuffle.h,
mf/sgd/sgd_impl.h, mf/sgd/functions/update-*.h, mf/loss/*.h).  Its raw
random stream is numpy's legacy MT19937 (RandomState), an implementation
independent of both the oracle and the product; every float operation is a
Python double operation in the reference's source order.  Used only to pin the
C++ oracle on small problems.
"""
from __future__ import annotations

import numpy as np


class Rand:
    """rg::Random32 as pinned: MT19937 raw draws, Boost bucket nextInt."""

    def __init__(self, seed):
        self.rs = np.random.RandomState(seed & 0xFFFFFFFF)

    def raw(self):
        return int(self.rs.randint(0, 2**32, dtype=np.uint64))

    def next_int(self, n):
        if n == 1:
            return 0
        if n == 0:
            return self.raw()
        rng = n - 1
        bucket = 0xFFFFFFFF // n
        if 0xFFFFFFFF % n == rng:
            bucket += 1
        while True:
            v = self.raw() // bucket
            if v <= rng:
                return v


def shuffle(a, R):
    a = list(a)
    for i in range(1, len(a)):
        j = R.next_int(i + 1)
        a[i], a[j] = a[j], a[i]
    return a


def sample(R, k, n):
    out = []
    for t in range(n):
        if len(out) >= k:
            break
        if R.next_int(n - t) < k - len(out):
            out.append(t)
    return out


def dsgd_schedule(w, t, order, R):
    D = w * t
    S = [[(s + i) % D for i in range(D)] for s in range(D)]
    if order == "RSEQ":
        b = shuffle(range(D), R)
        S = [[b[v] for v in row] for row in S]
    elif order == "WR":
        S = [shuffle(row, R) for row in S]
    elif order == "WOR":
        v = shuffle(range(D), R)
        u = shuffle(range(D), R)
        # r: permutation matrix with r[i, v[i]] = 1 ; c[k, u[k]] = 1 ; S' = r S c
        RS = [S[v[i]] for i in range(D)]
        out = [[0] * D for _ in range(D)]
        for i in range(D):
            for k in range(D):
                out[i][u[k]] = RS[i][k]
        S = out
    elif order == "COWOR":
        blocks = shuffle(range(D), R)
        G = dsgd_schedule(w, 1, "WOR", R)
        for bi in range(w):
            for bj in range(w):
                go = G[bi][bj] * t
                L = dsgd_schedule(t, 1, "WOR", R)
                for ti in range(t):
                    for tj in range(t):
                        S[bi * t + ti][bj * t + tj] = blocks[go + L[ti][tj]]
    return S


def dsgdpp_schedule(R, d, order):
    if order == "SEQ":
        b0 = [2 * k for k in range(d)]
        b1 = [2 * k + 1 for k in range(d)]
    else:
        b0 = sample(R, d, 2 * d)
        b1 = [b for b in range(2 * d) if b not in set(b0)][:d]
    s0 = dsgd_schedule(1, d, order, R)
    s1 = dsgd_schedule(1, d, order, R)
    sched = [[0] * d for _ in range(2 * d)]
    for i in range(d):
        for k in range(d):
            sched[2 * i][k] = b0[s0[i][k]]
            sched[2 * i + 1][k] = b1[s1[i][k]]
    seeds = [R.raw() for _ in range(d)]
    return sched, seeds


def block_offsets(size, blocks):
    base, rem = divmod(size, blocks)
    off = [0]
    for b in range(1, blocks):
        off.append(off[-1] + base + (1 if b <= rem else 0))
    return off


class Task:
    def __init__(self, seed):
        self.R = Rand(seed)
        self.perm = []

    def order(self, kind, n):
        if kind == "SEQ":
            return list(range(n))
        if kind == "WR":
            a, b = self.R.next_int(n), self.R.next_int(n)
            out = []
            for _ in range(n):
                out.append(a)
                a, b = b, self.R.next_int(n)
            return out
        if n == 0:
            return []
        if len(self.perm) != n:
            self.perm = list(range(n))
        p = self.perm
        nxt = self.R.next_int(n)
        for step in range(1, n):
            cur = nxt
            nxt = step + self.R.next_int(n - step)
            p[step - 1], p[cur] = p[cur], p[step - 1]
        return list(p)


class Job:
    """Blocked problem with global factors as lists of rows."""

    def __init__(self, m, n, r, d, rows, cols, vals, nb2=None):
        self.m, self.n, self.r, self.d = m, n, r, d
        self.nb2 = 2 * d if nb2 is None else nb2  # d x 2d (DSGD++) or d x d (DSGD)
        self.o1 = block_offsets(m, d) + [m]
        self.o2 = block_offsets(n, self.nb2) + [n]
        self.blocks = {}
        for i, j, x in sorted(zip(rows.tolist(), cols.tolist(), vals.tolist()),
                              key=lambda e: (e[0], e[1])):
            b1 = max(b for b in range(d) if self.o1[b] <= i)
            b2 = max(b for b in range(self.nb2) if self.o2[b] <= j)
            self.blocks.setdefault((b1, b2), []).append((i, j, x))
        self.nnz1 = [0] * m
        self.nnz2 = [0] * n
        for i, j in zip(rows.tolist(), cols.tolist()):
            self.nnz1[i] += 1
            self.nnz2[j] += 1

    def set_factors(self, W, H):
        self.W = [list(map(float, row)) for row in W]
        self.H = [list(map(float, row)) for row in H]

    def update(self, kind, lam, i, j, x, eps):
        w, h, r = self.W[i], self.H[j], self.r
        wh = 0.0
        for z in range(r):
            wh += w[z] * h[z]
        if kind == "Nzsl":
            f = eps * -2. * (x - wh)
            for z in range(r):
                t = w[z]
                w[z] -= f * h[z]
                h[z] -= f * t
        elif kind == "Nzsl_L2":
            f1 = eps * -2. * (x - wh)
            f2 = eps * 2. * lam
            f3 = 1. / self.nnz1[i]
            f4 = 1. / self.nnz2[j]
            for z in range(r):
                t = w[z]
                w[z] -= f1 * h[z] + f2 * w[z] * f3
                h[z] -= f1 * t + f2 * h[z] * f4
        else:
            f1 = eps * -2. * (x - wh)
            f2 = eps * 2. * lam
            for z in range(r):
                t = w[z]
                w[z] -= f1 * h[z] + f2 * w[z]
                h[z] -= f1 * t + f2 * h[z]

    def epoch(self, eps, sched, seeds, update="Nzsl_L2", lam=1.0, sgd_order="WOR"):
        d = self.d
        tasks = [Task(s) for s in seeds]
        for s in range(self.nb2):
            for tid in range(d):
                recs = self.blocks.get((tid, sched[s][tid]), [])
                for p in tasks[tid].order(sgd_order, len(recs)):
                    i, j, x = recs[p]
                    self.update(update, lam, i, j, x, eps)

    def nzsl(self):
        total = 0.0
        for b1 in range(self.d):
            for b2 in range(self.nb2):
                res = 0.0
                for i, j, x in self.blocks.get((b1, b2), []):
                    ip = 0.0
                    for z in range(self.r):
                        ip += self.W[i][z] * self.H[j][z]
                    diff = x - ip
                    res += diff * diff
                total += res
        return total
