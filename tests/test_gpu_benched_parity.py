"""GPU parity of the kernel instances the benchmark runs, against the CPU oracle.

The throughput path is checked here on the data and shapes it is measured on,
not only on small uniform problems:

* the deterministic FP64 replay on a 1M-entry sample of the benchmark's
  generator (2,000,000 x 500,000, Zipf(1.1) rows and columns, rank-32 truth,
  rank 32, Nzsl_L2(1) update, L2(0.05) regularize, BoldDriver(0.001)): factors
  bit-identical to the oracle, losses within 1e-12 relative (the reference
  loop is SgdRunner::updateWor, mf/sgd/sgd_impl.h:293-351, with
  UpdateNzslL2, mf/sgd/functions/update-nzsl-l2.h:34-57);
* the Hogwild kernel on a 2M-entry Zipf(1.1) problem with the default record
  layout (column runs), for ranks 32, 64 and 128 and every lane mapping the
  autotuner can return (the automatic one and the other of one vector per
  lane or two on half the lanes, at the occupancy limit and at 3 CTAs per
  SM): final test RMSE
  after 8 BoldDriver epochs within 0.5% (FP32 factors) or 1% (BF16 factors)
  of the FP64 oracle's;
* a Netflix-shaped problem (lognormal row degrees, Zipf(0.9) columns, integer
  ratings 1..5) at rank 128, FP32 and BF16 factors, same tolerances.

Updates inside a block run concurrently in the Hogwild kernel, so its factors
differ from the sequential oracle's; the test RMSE after several epochs is the
size-independent property compared.
"""
import os

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth_gpu
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOSS_RTOL = 1e-12
TOL = {"fp32": 0.005, "bf16": 0.01}
THREADS = os.cpu_count() or 1


class _Data:
    def __init__(self, m, n, out):
        self.m, self.n = m, n
        for k, v in out.items():
            setattr(self, k, v)


def _zipf(m, n, nnz, ntest, r, seed, rank_true=32):
    return _Data(m, n, synth_gpu.make(m, n, nnz, ntest, rank_true=rank_true, r=r, noise=0.2,
                                      seed=seed, s_row=1.1, s_col=1.1, device="cuda:0"))


def _oracle(p, r, d, l2=True):
    ref = O.Problem(p.m, p.n, r, d, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals)
    ref.configure(update="Nzsl_L2", update_lambda=1.0, regularize="L2" if l2 else "None",
                  regularize_lambda=0.05 if l2 else 0.0, loss="Nzsl_L2", loss_lambda=1.0)
    ref.set_factors(p.W0, p.H0)
    return ref


def _context(p, r, d, l2=True, **kw):
    cfg = P.Config(m=p.m, n=p.n, rank=r, d=d, update="Nzsl_L2", update_lambda=1.0,
                   regularize="L2" if l2 else "None", regularize_lambda=0.05 if l2 else 0.0,
                   loss="Nzsl_L2", loss_lambda=1.0, **kw)
    ctx = P.Context(cfg)
    ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
    ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
    ctx.set_factors(p.W0, p.H0)
    return ctx


def test_benchmark_generator_sample_fp64_replay_matches_oracle():
    # 1M entries of the 100M-entry workload's generator, at its shape and rank
    p = _zipf(2_000_000, 500_000, 1_000_000, 20_000, r=32, seed=11)
    d = 16
    ref = _oracle(p, 32, d)
    with _context(p, 32, d, precision="fp64", exec="replay", launch="graph") as ctx:
        ctx.seed(5)
        ref.seed(5)
        tr = ctx.run(2, "BoldDriver", 0.001)
        rt = ref.run(2, "BoldDriver", 0.001, threads=THREADS)
        for k, row in enumerate(tr):
            assert row["loss"] == pytest.approx(rt[k, 0], rel=LOSS_RTOL)
            assert row["test_loss"] == pytest.approx(rt[k, 1], rel=LOSS_RTOL)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)
        assert rt[-1, 1] < rt[0, 1]  # the run made progress


# ---- Hogwild on the benchmark's data, every lane mapping the autotuner returns ----
M, N, NNZ, NTEST, D, EPOCHS, EPS0 = 200_000, 50_000, 2_000_000, 50_000, 16, 8, 0.001
_cache = {}


def _zipf_case(r):
    """The 2M-entry Zipf(1.1) problem at factor rank r, and the FP64 oracle's
    BoldDriver run on it (computed once per rank)."""
    if r not in _cache:
        p = _zipf(M, N, NNZ, NTEST, r=r, seed=21)
        ref = _oracle(p, r, D)
        ref.seed(3)
        tr = ref.run(EPOCHS, "BoldDriver", EPS0, threads=THREADS)
        _cache.clear()  # one problem held at a time
        _cache[r] = (p, tr)
    return _cache[r]


def _threads(precision, lanes):
    """Threads per CTA of the sub-epoch kernel instance."""
    return 256 if precision == "bf16" and lanes > 4 else 128


def _auto_shape(precision, r):
    """The lane mapping the library picks by itself for this rank."""
    p = _Data(64, 64, {})
    cfg = P.Config(m=p.m, n=p.n, rank=r, d=4, precision=precision)
    with P.Context(cfg) as ctx:
        lanes, vecs, _ = ctx.launch_shape()
    return lanes, vecs


SHAPES = [(r, prec, half, ctas) for r in (32, 64, 128) for prec in ("fp32", "bf16")
          for half in (False, True) for ctas in (0, 3)]


@pytest.mark.parametrize("r,precision,half,ctas", SHAPES,
                         ids=[f"r{r}-{p}-{'other' if h else 'auto'}-ctas{c or 'occ'}"
                              for r, p, h, c in SHAPES])
def test_hogwild_benchmarked_shapes_track_fp64_oracle(r, precision, half, ctas):
    p, tr = _zipf_case(r)
    lanes, vecs = _auto_shape(precision, r)
    if half:  # the autotuner's alternative mapping (dsgdpp_autotune)
        if vecs == 2 and lanes <= 16:
            lanes, vecs = lanes * 2, 1
        else:
            assert lanes >= 4
            lanes, vecs = lanes // 2, vecs * 2
    with _context(p, r, D, precision=precision, exec="hogwild", launch="graph", layout="runs",
                  lanes_per_nnz=lanes, vecs_per_lane=vecs, ctas_per_sm=ctas) as ctx:
        got_lanes, got_vecs, grid = ctx.launch_shape()
        assert (got_lanes, got_vecs) == (lanes, vecs)
        if ctas:  # a cap counts CTAs of 256 threads (FP32 CTAs hold 128)
            assert grid * _threads(precision, lanes) <= ctas * 256 * 148
        ctx.seed(3)
        trace = ctx.run(EPOCHS, "BoldDriver", EPS0)
    got = float(np.sqrt(trace[-1]["test_loss"] / NTEST))
    want = float(np.sqrt(tr[-1, 1] / NTEST))
    start = float(np.sqrt(tr[0, 1] / NTEST))
    assert want < 0.8 * start  # the oracle run made progress
    assert abs(got - want) <= TOL[precision] * want, (got, want, [t["eps"] for t in trace])


def test_benchmark_autotuned_instance_tracks_fp64_oracle():
    # the instance the 100M-entry benchmark line runs: FP32, rank 32, 4 lanes x
    # 2 vectors per entry, 7 CTAs of 128 threads per SM (the register limit at
    # 72 registers; grid 1036 on 148 SMs)
    p, tr = _zipf_case(32)
    with _context(p, 32, D, precision="fp32", exec="hogwild", launch="graph", layout="runs",
                  lanes_per_nnz=4, vecs_per_lane=2) as ctx:
        assert ctx.launch_shape() == (4, 2, 7 * 148)
        ctx.seed(3)
        trace = ctx.run(EPOCHS, "BoldDriver", EPS0)
    got = float(np.sqrt(trace[-1]["test_loss"] / NTEST))
    want = float(np.sqrt(tr[-1, 1] / NTEST))
    assert abs(got - want) <= TOL["fp32"] * want, (got, want)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_netflix_shaped_rank128_tracks_fp64_oracle(precision):
    m, n, nnz, ntest, r, d = 40_000, 17_770, 2_000_000, 20_000, 128, 16
    p = _Data(m, n, synth_gpu.make_ratings(m, n, nnz, ntest, r, seed=31, device="cuda:0"))
    ref = _oracle(p, r, d, l2=False)
    ref.seed(7)
    rt = ref.run(EPOCHS, "BoldDriver", EPS0, threads=THREADS)
    with _context(p, r, d, l2=False, precision=precision, exec="hogwild", launch="graph",
                  layout="runs") as ctx:
        ctx.seed(7)
        trace = ctx.run(EPOCHS, "BoldDriver", EPS0)
    got = float(np.sqrt(trace[-1]["test_loss"] / ntest))
    want = float(np.sqrt(rt[-1, 1] / ntest))
    assert want < 0.8 * float(np.sqrt(rt[0, 1] / ntest))
    assert abs(got - want) <= TOL[precision] * want, (got, want)
