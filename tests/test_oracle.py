"""CPU tests of the oracle: pins and known answers.

The reference ships no tests or golden vectors (it cannot be built here), so
the oracle is pinned against (a) the one known answer the reference prints
(README.md:84-96: BoldDriver step sizes 0.001 -> 0.00105 -> 0.0011025), (b)
independent implementations of the pinned primitives (numpy's MT19937 stream),
(c) an independent pure-Python restatement of the epoch on tiny problems, and
(d) hand-derived cases of the blocking and schedule rules.
"""
import numpy as np
import pytest

from dsgdpp_b200 import synth
from oracle import oracle as O
from tests import pyref


def test_random32_raw_stream_is_mt19937():
    # numpy's legacy RandomState is an independent MT19937 with the same seeding
    for seed in (0, 1, 1234, 1499881717, 0xFFFFFFFF):
        ours = O.Random32(seed)
        rs = np.random.RandomState(seed)
        expect = rs.randint(0, 2**32, size=3000, dtype=np.uint64)
        got = np.array([ours.next() for _ in range(3000)], dtype=np.uint64)
        assert np.array_equal(got, expect)


def test_next_int_bucket_method():
    for seed in (3, 77):
        a, b = O.Random32(seed), pyref.Rand(seed)
        for n in [1, 2, 3, 5, 10, 97, 1000, 65537, 2**31 - 1, 2**31, 2**32 - 1, 0]:
            for _ in range(40):
                assert a.next_int(n) == b.next_int(n)


def test_next_int_in_range_and_one_consumes_nothing():
    r1, r2 = O.Random32(5), O.Random32(5)
    assert r1.next_int(1) == 0
    assert r1.next() == r2.next()  # nextInt(1) drew nothing
    for n in (2, 7, 1000):
        assert all(0 <= O.Random32(n).next_int(n) < n for _ in range(100))


def test_shuffle_and_sample():
    a = O.Random32(9).shuffle(np.arange(50))
    b = pyref.shuffle(range(50), pyref.Rand(9))
    assert a.tolist() == b
    assert sorted(a.tolist()) == list(range(50))
    s = O.Random32(4).sample(16, 32)
    assert s.tolist() == pyref.sample(pyref.Rand(4), 16, 32)
    assert list(s) == sorted(set(s.tolist())) and len(s) == 16


def test_block_offsets_known_values():
    # computeDefaultBlockOffsets: equal split, the first size % blocks blocks one larger
    assert O.block_offsets(10, 4).tolist() == [0, 3, 6, 8]
    assert O.block_offsets(100000, 8).tolist() == [12500 * k for k in range(8)]
    assert O.block_offsets(7, 7).tolist() == list(range(7))
    for size, blocks in [(100003, 8), (17, 5), (1, 1), (500000, 512)]:
        assert O.block_offsets(size, blocks).tolist() == pyref.block_offsets(size, blocks)


@pytest.mark.parametrize("order", ["SEQ", "RSEQ", "WR", "WOR", "COWOR"])
@pytest.mark.parametrize("d", [1, 2, 3, 4, 7])
def test_dsgdpp_schedule_matches_python_restatement(order, d):
    s, t = O.dsgdpp_schedule(O.Random32(100 + d), d, order)
    ps, pt = pyref.dsgdpp_schedule(pyref.Rand(100 + d), d, order)
    assert s.tolist() == ps and t.tolist() == pt


@pytest.mark.parametrize("order", ["SEQ", "RSEQ", "WOR", "COWOR"])
def test_schedule_is_a_stratification(order):
    d = 6
    s, _ = O.dsgdpp_schedule(O.Random32(1), d, order)
    for row in s:  # one sub-epoch: d distinct column blocks
        assert len(set(row.tolist())) == d
    for k in range(d):  # one task visits all 2d column blocks once per epoch
        assert sorted(s[:, k].tolist()) == list(range(2 * d))
    # even sub-epochs use one half of the column blocks, odd ones the other
    assert set(s[0::2].ravel().tolist()).isdisjoint(set(s[1::2].ravel().tolist()))


def test_seq_schedule_known_answer():
    s, _ = O.dsgdpp_schedule(O.Random32(0), 2, "SEQ")
    # blocks0 = {0, 2}, blocks1 = {1, 3}; base schedule (s + id) mod 2
    assert s.tolist() == [[0, 2], [1, 3], [2, 0], [3, 1]]


def test_bold_driver_readme_known_answer():
    # README.md:84-96: Step size 0.001, then 0.00105, then 0.0011025 after
    # train losses 1.00091e+09 -> 9.94144e+08 -> 9.84892e+08 (decreasing)
    e = O.bold_driver(0.001, None, 1.00091e9)
    assert e == 0.001
    e = O.bold_driver(e, 1.00091e9, 9.94144e8)
    assert e == pytest.approx(0.00105, rel=0, abs=1e-18)
    e = O.bold_driver(e, 9.94144e8, 9.84892e8)
    assert e == pytest.approx(0.0011025, rel=1e-15)
    assert O.bold_driver(0.002, 5.0, 5.0) == 0.001  # prev <= cur halves


def _tiny(seed=3, m=23, n=19, nnz=150, r=3):
    return synth.make(m, n, nnz, 20, rank_true=2, r=r, noise=0.1, seed=seed)


@pytest.mark.parametrize("update", ["Nzsl", "Nzsl_L2", "Nzsl_Nzl2"])
@pytest.mark.parametrize("sgd_order", ["SEQ", "WR", "WOR"])
def test_oracle_epoch_matches_python_restatement(update, sgd_order):
    p = _tiny()
    d = 2
    ref = O.Problem(p.m, p.n, 3, d, p.rows, p.cols, p.vals)
    ref.configure(update=update, update_lambda=0.7, loss="Nzsl", sgd_order=sgd_order)
    ref.set_factors(p.W0, p.H0)
    py = pyref.Job(p.m, p.n, 3, d, p.rows, p.cols, p.vals)
    py.set_factors(p.W0, p.H0)
    R = O.Random32(42)
    for e in range(2):
        sched, seeds = O.dsgdpp_schedule(R, d, "COWOR")
        ref.epoch_explicit(0.05, sched, seeds)
        py.epoch(0.05, sched.tolist(), seeds.tolist(), update=update, lam=0.7,
                 sgd_order=sgd_order)
    W, H = ref.get_factors()
    assert np.array_equal(W, np.array(py.W)) and np.array_equal(H, np.array(py.H))
    assert ref.nzsl() == py.nzsl()


@pytest.mark.parametrize("stratum_order", ["SEQ", "RSEQ", "WR", "WOR", "COWOR"])
@pytest.mark.parametrize("sgd_order", ["SEQ", "WR", "WOR"])
def test_oracle_dsgd_epoch_matches_python_restatement(stratum_order, sgd_order):
    # DsgdRunner::epoch (mf/sgd/dsgd_impl.h:328-350): the d x d schedule of
    # computeDsgdSchedule(1, d), then one raw draw per task seed; d x d blocks
    p = _tiny()
    d = 3
    ref = O.Problem(p.m, p.n, 3, d, p.rows, p.cols, p.vals, method="dsgd")
    ref.configure(update="Nzsl_L2", update_lambda=0.7, loss="Nzsl", sgd_order=sgd_order,
                  stratum_order=stratum_order)
    ref.set_factors(p.W0, p.H0)
    ref.seed(11)
    py = pyref.Job(p.m, p.n, 3, d, p.rows, p.cols, p.vals, nb2=d)
    py.set_factors(p.W0, p.H0)
    R = pyref.Rand(11)
    for e in range(3):
        S = pyref.dsgd_schedule(1, d, stratum_order, R)
        seeds = [R.raw() for _ in range(d)]
        ref.epoch(0.05)
        py.epoch(0.05, S, seeds, update="Nzsl_L2", lam=0.7, sgd_order=sgd_order)
    W, H = ref.get_factors()
    assert np.array_equal(W, np.array(py.W)) and np.array_equal(H, np.array(py.H))
    assert ref.nzsl() == py.nzsl()
    assert ref.block_nnz(0).shape == (d, d)


def test_positions_are_permutations_and_persist():
    p = _tiny(nnz=200)
    d = 2
    ref = O.Problem(p.m, p.n, 3, d, p.rows, p.cols, p.vals).configure(sgd_order="WOR")
    sched, seeds = O.dsgdpp_schedule(O.Random32(1), d, "COWOR")
    pos = ref.positions(sched, seeds)
    bn = ref.block_nnz()
    at = 0
    for s in range(2 * d):
        for tid in range(d):
            k = int(bn[tid, sched[s, tid]])
            assert sorted(pos[at:at + k].tolist()) == list(range(k))
            at += k
    assert at == len(pos) == 200


def test_blocking_sorted_and_duplicates_summed():
    rows = np.array([5, 0, 5, 3, 0], np.uint32)
    cols = np.array([1, 7, 1, 2, 0], np.uint32)
    vals = np.array([1.0, 2.0, 0.5, 3.0, 4.0])
    ref = O.Problem(6, 8, 2, 2, rows, cols, vals)
    # row blocks [0,3), [3,6); column blocks of 8 in 4: [0,2),[2,4),[4,6),[6,8)
    i, j, x = ref.block_records(0, 0)
    assert i.tolist() == [0] and j.tolist() == [0] and x.tolist() == [4.0]
    i, j, x = ref.block_records(0, 3)
    assert i.tolist() == [0] and j.tolist() == [1] and x.tolist() == [2.0]
    i, j, x = ref.block_records(1, 0)  # (5,1) twice -> one entry 1.5 (local (2,1))
    assert i.tolist() == [2] and j.tolist() == [1] and x.tolist() == [1.5]
    i, j, x = ref.block_records(1, 1)
    assert i.tolist() == [0] and j.tolist() == [0] and x.tolist() == [3.0]
    a, b, mx = ref.nnz12()
    assert a.tolist() == [2, 0, 0, 1, 0, 1] and mx == 2


def test_blocking_of_a_large_matrix_on_all_threads_matches_numpy():
    # above 2^20 entries the oracle routes and sorts blocks on all host threads;
    # each block must still hold its entries in (i, j) order with duplicates
    # summed in input order (mf/matrix/io/read_impl.h:162-164, 421)
    rng = np.random.default_rng(4)
    m, n, d, k = 5000, 3000, 4, 1_200_000
    rows = rng.integers(0, m, k).astype(np.uint32)
    cols = rng.integers(0, n, k).astype(np.uint32)
    vals = rng.standard_normal(k)
    ref = O.Problem(m, n, 2, d, rows, cols, vals)
    off1, off2 = O.block_offsets(m, d), O.block_offsets(n, 2 * d)
    key = rows.astype(np.int64) * n + cols
    order = np.argsort(key, kind="stable")
    skey = key[order]
    first = np.flatnonzero(np.r_[True, skey[1:] != skey[:-1]])
    ukey = skey[first]
    sv = vals[order]
    usum = sv[first].copy()
    ends = np.r_[first[1:], k]
    for g in np.flatnonzero(ends - first > 1):  # duplicates: summed one after another
        for q in range(first[g] + 1, ends[g]):
            usum[g] += sv[q]
    ur, uc = ukey // n, ukey % n
    b1 = np.searchsorted(off1, ur, side="right") - 1
    b2 = np.searchsorted(off2, uc, side="right") - 1
    total = 0
    for a in range(d):
        for b in range(2 * d):
            sel = (b1 == a) & (b2 == b)
            i, j, x = ref.block_records(a, b)
            np.testing.assert_array_equal(i, ur[sel] - off1[a])
            np.testing.assert_array_equal(j, uc[sel] - off2[b])
            np.testing.assert_array_equal(x, usum[sel])
            total += len(x)
    assert total == len(ukey) < k


def test_losses_against_numpy():
    p = _tiny(nnz=120, r=4)
    ref = O.Problem(p.m, p.n, 4, 2, p.rows, p.cols, p.vals)
    ref.configure(loss="Nzsl_L2", loss_lambda=0.3)
    ref.set_factors(p.W0, p.H0)
    pred = np.einsum("ij,ij->i", p.W0[p.rows], p.H0[p.cols])
    nz = float(np.sum((p.vals - pred) ** 2))
    assert ref.nzsl() == pytest.approx(nz, rel=1e-13)
    l2w, l2h = ref.l2()
    assert l2w == pytest.approx(float(np.sum(p.W0**2)), rel=1e-13)
    assert ref.loss() == pytest.approx(nz + 0.3 * (l2w + l2h), rel=1e-13)
    a, b, _ = ref.nnz12()
    nw, nh = ref.nzl2()
    assert nw == pytest.approx(float(np.sum(a * np.sum(p.W0**2, 1))), rel=1e-13)
    assert nh == pytest.approx(float(np.sum(b * np.sum(p.H0**2, 1))), rel=1e-13)


def test_threaded_epoch_equals_sequential():
    p = synth.make(400, 300, 5000, 0, rank_true=4, r=8, noise=0.1, seed=11)
    d = 4
    outs = []
    for threads in (1, 4):
        ref = O.Problem(p.m, p.n, 8, d, p.rows, p.cols, p.vals).configure()
        ref.set_factors(p.W0, p.H0)
        ref.seed(5)
        for _ in range(2):
            ref.epoch(0.01, threads=threads)
        outs.append(ref.get_factors())
    assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])


def test_regularize_l2_scales_blocks():
    p = _tiny(nnz=0 + 60)
    d = 2
    ref = O.Problem(p.m, p.n, 3, d, p.rows, p.cols, p.vals)
    ref.configure(update="Nzsl", regularize="L2", regularize_lambda=0.5, loss="Nzsl")
    ref.set_factors(p.W0, p.H0)
    # with eps = 0 the updates do nothing; L2 scales W by f per sub-epoch
    # (2d times) and each H column block once per visit (d times)
    eps = 0.0
    sched, seeds = O.dsgdpp_schedule(O.Random32(2), d, "COWOR")
    ref.epoch_explicit(eps, sched, seeds)
    W, H = ref.get_factors()
    assert np.array_equal(W, p.W0) and np.array_equal(H, p.H0)
    eps = 0.2
    ref.set_factors(p.W0, p.H0)
    py = pyref.Job(p.m, p.n, 3, d, p.rows, p.cols, p.vals)
    py.set_factors(p.W0, p.H0)
    ref.epoch_explicit(eps, sched, seeds)
    f = 1 - (eps / d) * 2 * 0.5
    W, H = ref.get_factors()
    # W after the epoch: every row scaled 2d times, interleaved with updates;
    # check the pure scaling part on rows without entries
    a, _, _ = ref.nnz12()
    empty = np.where(a == 0)[0]
    for i in empty:
        expect = p.W0[i].copy()
        for _ in range(2 * d):
            expect = expect * f
        assert np.array_equal(W[i], expect)
