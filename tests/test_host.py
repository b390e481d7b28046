"""CPU tests of the product library's host side and of its C ABI surface."""
import ctypes
import os
import re

import numpy as np
import pytest

import dsgdpp_b200 as P
from oracle import oracle as O
from tests.conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "dsgdpp.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set(re.findall(r"\b(dsgdpp_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(P.LIB_PATH)
    names = _header_symbols()
    assert len(names) >= 30
    for name in names:
        assert hasattr(lib, name), name
    assert names == set(P.SIGNATURES), names ^ set(P.SIGNATURES)
    assert lib.dsgdpp_abi_version() == 1


def test_status_strings():
    for s in (0, -1, -2, -3, -4, -5, -6):
        assert P.lib.dsgdpp_status_string(s).decode() != "unknown status"


@pytest.mark.skipif(HAS_GPU, reason="checks the behaviour without a GPU")
def test_create_fails_loudly_without_gpu():
    with pytest.raises(P.DsgdppError) as e:
        P.Context(P.Config(m=100, n=100, rank=8, d=2))
    assert e.value.status == P.E_CUDA


def test_invalid_config_rejected_before_device():
    bad = [dict(m=0, n=10, rank=4, d=1), dict(m=10, n=10, rank=4, d=6),
           dict(m=10, n=10, rank=4, d=2, precision="fp32", exec="replay"),
           dict(m=10, n=10, rank=300, d=1, precision="fp64", exec="replay")]
    for kw in bad:
        with pytest.raises(P.DsgdppError) as e:
            P.Context(P.Config(**kw))
        assert e.value.status in (P.E_INVALID, P.E_UNSUPPORTED)


def test_rng_matches_oracle():
    a, b = P.Random32(2024), O.Random32(2024)
    assert [a.next() for _ in range(1000)] == [b.next() for _ in range(1000)]
    for n in (1, 2, 3, 1000, 2**31 + 5, 0):
        assert [a.next_int(n) for _ in range(50)] == [b.next_int(n) for _ in range(50)]


@pytest.mark.parametrize("order", ["SEQ", "RSEQ", "WR", "WOR", "COWOR"])
@pytest.mark.parametrize("d", [1, 2, 4, 5, 16, 64])
def test_schedule_matches_oracle(order, d):
    ra, rb = P.Random32(7 * d), O.Random32(7 * d)
    for _ in range(3):  # consecutive epochs share the master stream
        sa, ta = P.draw_schedule(ra, d, order)
        sb, tb = O.dsgdpp_schedule(rb, d, order)
        assert np.array_equal(sa, sb) and np.array_equal(ta, tb)


@pytest.mark.parametrize("order", ["RSEQ", "WR", "WOR", "COWOR"])
def test_dsgd_schedule_matches_oracle(order):
    for w, t in [(1, 5), (2, 3), (3, 4)]:
        a = P.dsgd_schedule(P.Random32(3), w, t, order)
        b = O.dsgd_schedule(O.Random32(3), w, t, order)
        assert np.array_equal(a, b)


@pytest.mark.parametrize("sgd_order", ["SEQ", "WR", "WOR"])
def test_point_orders_match_oracle(sgd_order):
    from dsgdpp_b200 import synth
    p = synth.make(300, 200, 3000, 0, rank_true=3, r=4, noise=0.1, seed=1)
    d = 3
    ref = O.Problem(p.m, p.n, 4, d, p.rows, p.cols, p.vals).configure(sgd_order=sgd_order)
    sched, seeds = O.dsgdpp_schedule(O.Random32(8), d, "COWOR")
    got = P.point_orders(d, sgd_order, ref.block_nnz(), sched, seeds)
    assert np.array_equal(got, ref.positions(sched, seeds))


def test_point_orders_reuse_permutation_buffer():
    # SgdRunner::permute keeps the buffer when the block size repeats
    # (mf/sgd/sgd_impl.h:257-262): equal-size blocks continue the same array
    d = 2
    bn = np.full((d, 2 * d), 5, np.uint64)
    sched = np.array([[0, 1], [1, 0], [2, 3], [3, 2]], np.uint32)
    seeds = np.array([1, 2], np.uint32)
    out = P.point_orders(d, "WOR", bn, sched, seeds)
    # replay by hand for task 0 with the pinned generator
    R = O.Random32(1)
    perm = list(range(5))
    expect = []
    for _ in range(4):
        nxt = R.next_int(5)
        for step in range(1, 5):
            cur = nxt
            nxt = step + R.next_int(5 - step)
            perm[step - 1], perm[cur] = perm[cur], perm[step - 1]
        expect.append(list(perm))
    task0 = [out[(2 * s) * 5:(2 * s) * 5 + 5].tolist() for s in range(4)]
    assert task0 == expect


def test_block_offsets_match_oracle():
    for size, blocks in [(100000, 4), (100000, 8), (2_000_000, 128), (500_000, 1024), (13, 13)]:
        assert np.array_equal(P.block_offsets(size, blocks), O.block_offsets(size, blocks))


def test_philox_known_answers():
    # Random123 known-answer vectors for Philox4x32-10
    kat = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
           ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
           ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
            [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for ctr, key, out in kat:
        assert P.philox4x32_10(ctr, key).tolist() == out


def test_controller_features_shape_and_values():
    f = P.controller_features([90.0, 100.0, 110.0, 120.0, 130.0], [9.0, 10.0, 10.0, 11.0, 12.0],
                              0.001, 0.02, 0.5, 0.25, 0.1)
    assert f.shape == (16,) and f.dtype == np.float32
    assert f[0] == pytest.approx(10 * np.log(90 / 100), rel=1e-6)
    assert f[8] == pytest.approx(-1.0, rel=1e-6)  # log10(0.001) / 3
    assert f[11] == pytest.approx(0.25) and f[13] == pytest.approx(0.1)
    assert f[15] == 3.0  # no step has raised the loss
    g = P.controller_features([5.0], [], 0.01, 0.0, 0.0, 0.0, 0.0)  # short history
    assert np.all(g[0:8] == 0) and np.all(np.isfinite(g))
    h = P.controller_features([5.0], [], 0.01, 0.0, 0.0, 0.0, 0.0, fail_eps=0.02)
    assert h[15] == pytest.approx(np.log(2.0), rel=1e-6)
    assert P.controller_features([5.0], [], 0.01, 0, 0, 0, 0, fail_eps=1e9)[15] == 3.0


def test_mlp_oracle_gradient_matches_finite_differences():
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, 5313)
    X = rng.normal(0, 1, (7, 16))
    y = rng.uniform(-0.8, 0.8, 7)
    _, g = M.loss_and_grad(p, X, y)
    for k in [0, 100, 1024, 1100, 3000, 5200, 5312]:
        e = np.zeros_like(p)
        e[k] = 1e-6
        num = (M.loss_and_grad(p + e, X, y)[0] - M.loss_and_grad(p - e, X, y)[0]) / 2e-6
        assert g[k] == pytest.approx(num, rel=1e-5, abs=1e-9)
