"""GPU parity tests: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances:
* FP64 replay factors: bit-identical to the oracle (the bar is 1e-10 relative
  per entry; the replay repeats every operation in the reference order);
* FP64 losses: 1e-12 relative (the terms are identical, only the summation
  order differs);
* blocking, counts, schedules: exact;
* FP32 / BF16 Hogwild runs: final test RMSE within a stated tolerance of the
  FP64 oracle's, since updates inside a block run concurrently.
"""
import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

LOSS_RTOL = 1e-12


def _problem(m=500, n=400, nnz=6000, ntest=600, r=10, seed=5, kind="uniform"):
    return synth.make(m, n, nnz, ntest, rank_true=min(r, 8), r=r, noise=0.1, seed=seed,
                      kind=kind)


def _pair(p, r, d, precision="fp64", exec="replay", launch="stream", **kw):
    okw = {k: v for k, v in kw.items() if k in ("update", "update_lambda", "regularize",
                                                 "regularize_lambda", "loss", "loss_lambda",
                                                 "truncate", "sgd_order", "stratum_order")}
    ref = O.Problem(p.m, p.n, r, d, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals)
    ref.configure(**okw)
    ref.set_factors(p.W0, p.H0)
    cfg = P.Config(m=p.m, n=p.n, rank=r, d=d, precision=precision, exec=exec, launch=launch,
                   **{k: v for k, v in kw.items()})
    ctx = P.Context(cfg)
    ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
    ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
    ctx.set_factors(p.W0, p.H0)
    return ref, ctx


@pytest.mark.parametrize("update", ["Nzsl", "Nzsl_L2", "Nzsl_Nzl2"])
@pytest.mark.parametrize("sgd_order", ["SEQ", "WR", "WOR"])
@pytest.mark.parametrize("truncate", [None, (-0.3, 0.3)])
def test_replay_bit_exact(update, sgd_order, truncate):
    p = _problem()
    d = 3
    ref, ctx = _pair(p, 10, d, update=update, update_lambda=0.5, sgd_order=sgd_order,
                     truncate=truncate, loss="Nzsl")
    with ctx:
        R = P.Random32(77)
        for _ in range(2):
            sched, seeds = P.draw_schedule(R, d, "COWOR")
            ctx.epoch_explicit(0.02, sched, seeds)
            ref.epoch_explicit(0.02, sched, seeds)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


@pytest.mark.parametrize("r", [1, 3, 32, 33, 64, 128])
def test_replay_ranks(r):
    p = _problem(m=300, n=200, nnz=3000, r=r)
    d = 2
    ref, ctx = _pair(p, r, d)
    with ctx:
        sched, seeds = P.draw_schedule(P.Random32(r), d, "WOR")
        ctx.epoch_explicit(0.01, sched, seeds)
        ref.epoch_explicit(0.01, sched, seeds)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


def test_replay_l2_regularize_exact():
    p = _problem()
    d = 4
    ref, ctx = _pair(p, 10, d, update="Nzsl", regularize="L2", regularize_lambda=0.05,
                     loss="Nzsl_L2", loss_lambda=0.05)
    with ctx:
        R = P.Random32(3)
        for _ in range(2):
            sched, seeds = P.draw_schedule(R, d, "COWOR")
            ctx.epoch_explicit(0.05, sched, seeds)
            ref.epoch_explicit(0.05, sched, seeds)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


@pytest.mark.parametrize("stratum_order", ["SEQ", "RSEQ", "WR", "WOR", "COWOR"])
def test_replay_master_rng_epochs(stratum_order):
    # dsgdpp_epoch draws the schedule itself, like DsgdPpRunner::epoch
    p = _problem()
    d = 2
    ref, ctx = _pair(p, 10, d, stratum_order=stratum_order)
    with ctx:
        ctx.seed(1499881717)
        ref.seed(1499881717)
        for _ in range(3):
            ctx.epoch(0.01)
            ref.epoch(0.01)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


@pytest.mark.parametrize("loss", ["Nzsl", "Nzsl_L2", "Nzsl_Nzl2"])
def test_loss_parity(loss):
    p = _problem(m=2000, n=1500, nnz=60000, ntest=5000, r=16)
    ref, ctx = _pair(p, 16, 4, loss=loss, loss_lambda=0.3)
    with ctx:
        assert ctx.loss() == pytest.approx(ref.loss(), rel=LOSS_RTOL)
        assert ctx.nzsl(P.TEST) == pytest.approx(ref.nzsl(1), rel=LOSS_RTOL)
        assert ctx.nzsl(P.TRAIN) == pytest.approx(ref.nzsl(0), rel=LOSS_RTOL)
        for a, b in zip(ctx.l2(), ref.l2()):
            assert a == pytest.approx(b, rel=LOSS_RTOL)
        for a, b in zip(ctx.nzl2(), ref.nzl2()):
            assert a == pytest.approx(b, rel=LOSS_RTOL)


def test_loss_parity_fp32_and_bf16_factors():
    # the FP64 loss of stored low-precision factors equals the oracle's loss of
    # the same factors read back as doubles
    p = _problem(m=2000, n=1500, nnz=40000, r=32)
    # FP32 / BF16 factor storage keeps the entry values in FP32 (12-byte records)
    p.vals = p.vals.astype(np.float32).astype(np.float64)
    p.tvals = p.tvals.astype(np.float32).astype(np.float64)
    for prec in ("fp32", "bf16"):
        ref, ctx = _pair(p, 32, 4, precision=prec, exec="hogwild")
        with ctx:
            W, H = ctx.get_factors()
            ref.set_factors(W, H)
            assert ctx.nzsl(P.TRAIN) == pytest.approx(ref.nzsl(0), rel=LOSS_RTOL)
            assert ctx.loss() == pytest.approx(ref.loss(), rel=LOSS_RTOL)


def _extreme(rng, shape):
    """Factor values over the whole float range: zeros, subnormals, tiny,
    ordinary and large magnitudes, both signs."""
    kind = rng.choice(5, size=shape, p=[0.2, 0.1, 0.1, 0.58, 0.02])
    mag = np.select([kind == 0, kind == 1, kind == 2, kind == 3, kind == 4],
                    [0.0, rng.uniform(1e-42, 1e-39, shape), rng.uniform(1e-22, 1e-18, shape),
                     rng.uniform(0.0, 2.0, shape), rng.uniform(1e3, 1e4, shape)])
    return mag * rng.choice([-1.0, 1.0], size=shape)


@pytest.mark.parametrize("r", [7, 32, 100])
def test_loss_parity_extreme_factor_values(r):
    # the FP32/BF16 loss kernels form exact FP64 products (H's values built
    # from their bits, scaled by a power of two and back): zeros, subnormal,
    # tiny and large factor values give the oracle's loss of the same stored
    # factors, at ranks with and without a partial last vector
    p = _problem(m=300, n=200, nnz=6000, ntest=500, r=r)
    p.vals = p.vals.astype(np.float32).astype(np.float64)
    p.tvals = p.tvals.astype(np.float32).astype(np.float64)
    rng = np.random.default_rng(r)
    p.W0 = _extreme(rng, p.W0.shape)
    p.H0 = _extreme(rng, p.H0.shape)
    for prec in ("fp32", "bf16"):
        ref, ctx = _pair(p, r, 4, precision=prec, exec="hogwild")
        with ctx:
            W, H = ctx.get_factors()
            assert np.count_nonzero((W != 0) & (np.abs(W) < 1.1754944e-38)) > 0  # subnormals stored
            ref.set_factors(W, H)
            assert ctx.nzsl(P.TRAIN) == pytest.approx(ref.nzsl(0), rel=LOSS_RTOL)
            assert ctx.nzsl(P.TEST) == pytest.approx(ref.nzsl(1), rel=LOSS_RTOL)
            assert ctx.loss() == pytest.approx(ref.loss(), rel=LOSS_RTOL)


def test_blocking_and_counts():
    p = _problem(m=1001, n=997, nnz=20000, kind="zipf")
    for d in (1, 3, 8):
        ref, ctx = _pair(p, 8, d)
        with ctx:
            np.testing.assert_array_equal(ctx.block_nnz(P.TRAIN), ref.block_nnz(0))
            np.testing.assert_array_equal(ctx.block_nnz(P.TEST), ref.block_nnz(1))
            a, b, mx = ctx.nnz12()
            ra, rb, rmx = ref.nnz12()
            np.testing.assert_array_equal(a, ra)
            np.testing.assert_array_equal(b, rb)
            assert mx == rmx


def test_duplicates_are_summed():
    rows = np.array([5, 0, 5, 3, 0, 5], np.uint32)
    cols = np.array([1, 7, 1, 2, 0, 1], np.uint32)
    vals = np.array([1.0, 2.0, 0.5, 3.0, 4.0, 0.25])
    W0 = np.random.default_rng(0).uniform(-0.5, 0.5, (6, 2))
    H0 = np.random.default_rng(1).uniform(-0.5, 0.5, (8, 2))
    ref = O.Problem(6, 8, 2, 2, rows, cols, vals).configure()
    ref.set_factors(W0, H0)
    with P.Context(P.Config(m=6, n=8, rank=2, d=2, precision="fp64", exec="replay")) as ctx:
        ctx.set_matrix(P.TRAIN, rows, cols, vals)
        ctx.set_factors(W0, H0)
        np.testing.assert_array_equal(ctx.block_nnz(), ref.block_nnz())
        assert ctx.nzsl() == pytest.approx(ref.nzsl(), rel=LOSS_RTOL)


@pytest.mark.parametrize("layout", ["shuffled", "col_runs", "row_runs"])
def test_hogwild_layouts_block_and_merge_like_the_oracle(layout):
    """Hogwild training records are blocked and laid out by one sort whose key
    permutes the positions inside a block.  On a matrix where nearly every
    position of every block holds one or more entries (uneven block extents,
    so the permuted ranges are not powers of two), two positions sharing a key
    would merge distinct entries: the block counts and the training loss must
    still equal the oracle's, which merges exact duplicates only
    (ReadMatrixBlocksMm's coordinate sort, mf/matrix/io/read_impl.h:162-164)."""
    rng = np.random.default_rng(3)
    m, n, d, r = 203, 181, 3, 5
    rows = rng.integers(0, m, 150000).astype(np.uint32)
    cols = rng.integers(0, n, 150000).astype(np.uint32)
    vals = rng.normal(0, 1, 150000)
    W0 = rng.uniform(-0.5, 0.5, (m, r))
    H0 = rng.uniform(-0.5, 0.5, (n, r))
    ref = O.Problem(m, n, r, d, rows, cols, vals).configure()
    ref.set_factors(W0, H0)
    assert len(set(zip(rows.tolist(), cols.tolist()))) > 0.98 * m * n
    cfg = P.Config(m=m, n=n, rank=r, d=d, precision="fp64", exec="hogwild", layout=layout)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, rows, cols, vals)
        ctx.set_factors(W0, H0)
        np.testing.assert_array_equal(ctx.block_nnz(), ref.block_nnz())
        assert ctx.nzsl() == pytest.approx(ref.nzsl(), rel=LOSS_RTOL)


def test_run_trace_matches_oracle():
    p = _problem(m=800, n=600, nnz=10000, ntest=1000)
    ref, ctx = _pair(p, 10, 2)
    with ctx:
        ctx.seed(42)
        ref.seed(42)
        tr = ctx.run(6, "BoldDriver", 0.01)
        rt = ref.run(6, "BoldDriver", 0.01)
        for k, row in enumerate(tr):
            assert row["loss"] == pytest.approx(rt[k, 0], rel=LOSS_RTOL)
            assert row["test_loss"] == pytest.approx(rt[k, 1], rel=LOSS_RTOL)
            if k:
                assert row["eps"] == rt[k, 2]


def test_empty_matrix_and_empty_blocks():
    p = _problem(m=50, n=40, nnz=30, ntest=0)
    ref, ctx = _pair(p, 4, 4)  # 4 x 8 blocks, most of them empty
    with ctx:
        sched, seeds = P.draw_schedule(P.Random32(1), 4, "COWOR")
        ctx.epoch_explicit(0.1, sched, seeds)
        ref.epoch_explicit(0.1, sched, seeds)
        np.testing.assert_array_equal(ctx.get_factors()[0], ref.get_factors()[0])
        assert ctx.nzsl(P.TEST) == 0.0
    with P.Context(P.Config(m=10, n=10, rank=2, d=1, precision="fp32")) as ctx:
        ctx.set_matrix(P.TRAIN, [], [], [])
        ctx.set_factors(np.ones((10, 2)), np.ones((10, 2)))
        ctx.epoch(0.1)
        assert ctx.nzsl() == 0.0
        np.testing.assert_array_equal(ctx.get_factors()[0], np.ones((10, 2)))


def test_errors_are_reported_not_crashed():
    with P.Context(P.Config(m=10, n=10, rank=2, d=2)) as ctx:
        with pytest.raises(P.DsgdppError) as e:
            ctx.epoch(0.1)
        assert e.value.status == P.E_STATE
        with pytest.raises(P.DsgdppError) as e:
            ctx.set_matrix(P.TRAIN, [1, 10], [0, 0], [1.0, 2.0])
        assert e.value.status == P.E_INVALID
        with pytest.raises(P.DsgdppError):
            ctx.epoch_explicit(0.1, np.full((4, 2), 9, np.uint32), np.zeros(2, np.uint32))


def _rmse(ctx, ntest):
    return float(np.sqrt(ctx.nzsl(P.TEST) / ntest))


# Test RMSE after 8 constant-step epochs against the sequential FP64 oracle.
# Atomic writes lose no concurrent update and track the oracle to 0.5% (BF16:
# 1%, it rounds every write stochastically); plain stores lose some updates of
# rows updated at the same time, and how many varies run to run (8%).
@pytest.mark.parametrize("precision,write_mode,tol", [
    ("fp64", "atomic", 0.005), ("fp32", "atomic", 0.005), ("bf16", "atomic", 0.01),
    ("fp64", "store", 0.08), ("fp32", "store", 0.08), ("bf16", "store", 0.08)])
@pytest.mark.parametrize("launch", ["stream", "graph"])
def test_hogwild_tracks_fp64_oracle(precision, write_mode, tol, launch):
    p = synth.make(20000, 20000, 400000, 40000, rank_true=10, r=10, noise=0.1, seed=3)
    d = 4
    ref, ctx = _pair(p, 10, d, precision=precision, exec="hogwild", launch=launch,
                     write_mode=write_mode, layout="shuffled")
    with ctx:
        ctx.seed(9)
        ref.seed(9)
        eps = 0.01
        for _ in range(8):
            ctx.epoch(eps)
            ref.epoch(eps)
        got = _rmse(ctx, len(p.tvals))
        want = float(np.sqrt(ref.nzsl(1) / len(p.tvals)))
        start = float(np.sqrt(np.sum((p.tvals - np.einsum("ij,ij->i", p.W0[p.trows],
                                                          p.H0[p.tcols])) ** 2) / len(p.tvals)))
        assert want < 0.9 * start  # the run made progress
        assert abs(got - want) <= tol * want, (got, want)


# Records in runs of one H row (or W row) per group: the run's updates of the
# shared row are sequential and written once; the same tolerances hold.
@pytest.mark.parametrize("layout", ["col_runs", "row_runs"])
@pytest.mark.parametrize("precision,write_mode,tol", [
    ("fp64", "atomic", 0.005), ("fp32", "atomic", 0.005), ("bf16", "atomic", 0.01),
    ("fp32", "store", 0.08)])
def test_hogwild_runs_layout_tracks_fp64_oracle(layout, precision, write_mode, tol):
    p = synth.make(20000, 20000, 400000, 40000, rank_true=10, r=10, noise=0.1, seed=3)
    ref, ctx = _pair(p, 10, 4, precision=precision, exec="hogwild", launch="graph",
                     write_mode=write_mode, layout=layout)
    with ctx:
        ctx.seed(9)
        ref.seed(9)
        for _ in range(8):
            ctx.epoch(0.01)
            ref.epoch(0.01)
        got = _rmse(ctx, len(p.tvals))
        want = float(np.sqrt(ref.nzsl(1) / len(p.tvals)))
        assert abs(got - want) <= tol * want, (got, want)


@pytest.mark.parametrize("layout", ["shuffled", "col_runs", "row_runs"])
def test_hogwild_truncation_bounds_every_factor(layout):
    p = _problem(m=3000, n=2000, nnz=60000, ntest=100, r=12)
    cfg = P.Config(m=p.m, n=p.n, rank=12, d=4, precision="fp32", write_mode="store",
                   truncate=(-0.2, 0.25), layout=layout)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_factors(np.clip(p.W0, -0.2, 0.25), np.clip(p.H0, -0.2, 0.25))
        for _ in range(3):
            ctx.epoch(0.05)
        W, H = ctx.get_factors()
    assert W.min() >= -0.2 and W.max() <= 0.25 and H.min() >= -0.2 and H.max() <= 0.25


def test_hogwild_lazy_l2_scaling_matches_exact():
    # with no training entries the epoch is pure RegularizeL2 scaling: W is
    # scaled 2d times, each H column block d times
    m, n, r, d = 64, 64, 8, 4
    rng = np.random.default_rng(0)
    W0, H0 = rng.uniform(-1, 1, (m, r)), rng.uniform(-1, 1, (n, r))
    outs = []
    for prec, ex in (("fp64", "replay"), ("fp32", "hogwild"), ("fp64", "hogwild")):
        cfg = P.Config(m=m, n=n, rank=r, d=d, precision=prec, exec=ex, update="Nzsl",
                       regularize="L2", regularize_lambda=0.5, loss="Nzsl")
        with P.Context(cfg) as ctx:
            ctx.set_matrix(P.TRAIN, [], [], [])
            ctx.set_factors(W0, H0)
            sched, seeds = P.draw_schedule(P.Random32(4), d, "COWOR")
            ctx.epoch_explicit(0.3, sched, seeds)
            outs.append(ctx.get_factors())
    for W, H in outs[1:]:
        np.testing.assert_allclose(W, outs[0][0], rtol=2e-6)
        np.testing.assert_allclose(H, outs[0][1], rtol=2e-6)


def test_epoch_time_is_reported():
    p = _problem()
    _, ctx = _pair(p, 10, 2, precision="fp32", exec="hogwild")
    with ctx:
        ctx.epoch(0.01)
        assert ctx.last_epoch_ms() > 0


# One persistent launch per epoch: a block starts when the blocks it depends on
# (its task's previous block, the previous block on its column block) are done.
@pytest.mark.parametrize("precision,tol", [("fp64", 0.005), ("fp32", 0.005), ("bf16", 0.01)])
@pytest.mark.parametrize("sgd_order", ["SEQ", "WOR"])
@pytest.mark.parametrize("layout", ["col_runs", "row_runs"])
def test_persistent_epoch_tracks_fp64_oracle(precision, tol, sgd_order, layout):
    p = synth.make(20000, 20000, 400000, 40000, rank_true=10, r=10, noise=0.1, seed=3)
    ref, ctx = _pair(p, 10, 4, precision=precision, exec="hogwild", launch="persistent",
                     layout=layout, sgd_order=sgd_order)
    with ctx:
        ctx.seed(9)
        ref.seed(9)
        for _ in range(8):
            ctx.epoch(0.01)
            ref.epoch(0.01)
        got = _rmse(ctx, len(p.tvals))
        want = float(np.sqrt(ref.nzsl(1) / len(p.tvals)))
        assert abs(got - want) <= tol * want, (got, want)


def test_persistent_epoch_kernel_timing_and_unsupported_forms():
    p = _problem(m=3000, n=2000, nnz=60000, ntest=100, r=12)
    cfg = P.Config(m=p.m, n=p.n, rank=12, d=8, launch="persistent", layout="col_runs")
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_factors(p.W0, p.H0)
        ctx.set_kernel_timing(True)
        for _ in range(3):
            ctx.epoch(0.01)
        ms, launches = ctx.kernel_timing()
        assert launches == 3 and ms > 0
    for bad in (dict(sgd_order="WR"), dict(write_mode="store"), dict(layout="shuffled"),
                dict(exec="replay", precision="fp64")):
        with pytest.raises(P.DsgdppError):
            P.Context(P.Config(m=p.m, n=p.n, rank=12, d=8, launch="persistent",
                               **dict(dict(layout="col_runs"), **bad)))


def test_persistent_epoch_wait_limit_gives_up_and_the_context_recovers():
    # the bounded dependency wait of the one-launch epoch (in place of the
    # reference's unbounded sub-epoch barrier, mf/sgd/dsgdpp_impl.h:259-263):
    # with a zero limit the first unmet dependency ends the epoch with an error
    # status, and the next epoch on the same context runs normally.  Every
    # sub-epoch here has ~120 chunks against thousands of resident warps, so
    # warps holding later sub-epochs' tickets meet unfinished dependencies.
    p = _problem(m=3000, n=2000, nnz=60000, ntest=600, r=12)
    cfg = P.Config(m=p.m, n=p.n, rank=12, d=8, launch="persistent", layout="col_runs")
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        ctx.seed(1)
        ctx.epoch(0.01)
        ctx.set_wait_limit(0.0)
        with pytest.raises(P.DsgdppError) as err:
            ctx.epoch(0.01)
        assert err.value.status == P.E_CUDA and "gave up" in str(err.value)
        ctx.set_wait_limit(1.0)
        before = ctx.nzsl(P.TEST)
        for _ in range(3):
            ctx.epoch(0.01)
        after = ctx.nzsl(P.TEST)
        W, H = ctx.get_factors()
        assert np.isfinite(W).all() and np.isfinite(H).all()
        assert after < before
    with pytest.raises(P.DsgdppError):
        with P.Context(cfg) as ctx:
            ctx.set_wait_limit(-1.0)


def test_small_cpu_workload_replay_run_matches_oracle():
    # the reference's CPU-runnable case at full size: 100,000 x 100,000, 1M
    # uniform entries (+100k test), rank 10, FP64, Nzsl_L2(1), d = 4 (4 x 8
    # blocks), BoldDriver(0.001); 3 epochs of the 50 (the oracle is sequential)
    p = synth.make(100_000, 100_000, 1_000_000, 100_000, rank_true=10, r=10, noise=0.1, seed=2024)
    ref, ctx = _pair(p, 10, 4, precision="fp64", exec="replay", launch="graph")
    with ctx:
        ctx.seed(1)
        ref.seed(1)
        tr = ctx.run(3, "BoldDriver", 0.001)
        rt = ref.run(3, "BoldDriver", 0.001)
        for k, row in enumerate(tr):
            assert row["loss"] == pytest.approx(rt[k, 0], rel=LOSS_RTOL)
            assert row["test_loss"] == pytest.approx(rt[k, 1], rel=LOSS_RTOL)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


# ---- DSGD (d x d blocking, d sub-epochs; mf/sgd/dsgd_impl.h) -------------------
@pytest.mark.parametrize("stratum_order", ["SEQ", "RSEQ", "WR", "WOR", "COWOR"])
@pytest.mark.parametrize("sgd_order", ["SEQ", "WOR"])
def test_dsgd_replay_master_rng_epochs_bit_exact(stratum_order, sgd_order):
    p = _problem()
    d = 3
    ref = O.Problem(p.m, p.n, 10, d, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals,
                    method="dsgd")
    ref.configure(sgd_order=sgd_order, stratum_order=stratum_order, update_lambda=0.5)
    ref.set_factors(p.W0, p.H0)
    cfg = P.Config(m=p.m, n=p.n, rank=10, d=d, precision="fp64", exec="replay", method="dsgd",
                   sgd_order=sgd_order, stratum_order=stratum_order, update_lambda=0.5)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        assert ctx.block_nnz(P.TRAIN).shape == (d, d)
        np.testing.assert_array_equal(ctx.block_nnz(P.TRAIN), ref.block_nnz(0))
        ctx.seed(5)
        ref.seed(5)
        for _ in range(3):
            ctx.epoch(0.02)
            ref.epoch(0.02)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)
        assert ctx.loss() == pytest.approx(ref.loss(), rel=LOSS_RTOL)


def test_dsgd_replay_l2_regularize_and_run_trace():
    p = _problem(m=800, n=600, nnz=10000, ntest=1000)
    ref = O.Problem(p.m, p.n, 10, 4, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals,
                    method="dsgd")
    ref.configure(regularize="L2", regularize_lambda=0.05)
    ref.set_factors(p.W0, p.H0)
    cfg = P.Config(m=p.m, n=p.n, rank=10, d=4, precision="fp64", exec="replay", method="dsgd",
                   regularize="L2", regularize_lambda=0.05)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        ctx.seed(42)
        ref.seed(42)
        tr = ctx.run(5, "BoldDriver", 0.01)
        rt = ref.run(5, "BoldDriver", 0.01)
        for k, row in enumerate(tr):
            assert row["loss"] == pytest.approx(rt[k, 0], rel=LOSS_RTOL)
            assert row["test_loss"] == pytest.approx(rt[k, 1], rel=LOSS_RTOL)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)


@pytest.mark.parametrize("precision,tol", [("fp32", 0.005), ("bf16", 0.01)])
@pytest.mark.parametrize("launch", ["graph", "persistent"])
def test_dsgd_hogwild_tracks_fp64_oracle(precision, tol, launch):
    p = synth.make(20000, 20000, 400000, 40000, rank_true=10, r=10, noise=0.1, seed=3)
    ref = O.Problem(p.m, p.n, 10, 4, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals,
                    method="dsgd")
    ref.configure(regularize="L2", regularize_lambda=0.02)
    ref.set_factors(p.W0, p.H0)
    cfg = P.Config(m=p.m, n=p.n, rank=10, d=4, precision=precision, launch=launch,
                   method="dsgd", regularize="L2", regularize_lambda=0.02)
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        ctx.seed(9)
        ref.seed(9)
        for _ in range(8):
            ctx.epoch(0.01)
            ref.epoch(0.01)
        got = _rmse(ctx, len(p.tvals))
        want = float(np.sqrt(ref.nzsl(1) / len(p.tvals)))
        assert abs(got - want) <= tol * want, (got, want)


def test_dsgd_blocking_limits_and_batch_rejection():
    p = _problem(m=50, n=5, nnz=100, ntest=10)
    P.Context(P.Config(m=p.m, n=p.n, rank=4, d=5, method="dsgd")).close()  # n >= d suffices
    with pytest.raises(P.DsgdppError):
        P.Context(P.Config(m=p.m, n=p.n, rank=4, d=5))  # DSGD++ needs n >= 2d
    prob = dict(m=p.m, n=p.n, rank=4, rows=p.rows, cols=p.cols, vals=p.vals, W=p.W0[:, :4],
                H=p.H0[:, :4])
    with pytest.raises(P.DsgdppError):
        P.Batch(P.Config(m=1, n=1, rank=1, d=1, method="dsgd"), [prob])


# ---- blocked input and caller-held counts (the runner's own data form) ---------------
def _oracle_blocks(ref, d, nb2, which=0):
    parts = [ref.block_records(b1, b2, which) for b1 in range(d) for b2 in range(nb2)]
    bn = np.array([len(x) for _, _, x in parts], np.uint64)
    cat = lambda k: np.concatenate([p[k] for p in parts]) if len(parts) else np.empty(0)
    return bn, cat(0), cat(1), cat(2)


@pytest.mark.parametrize("method", ["dsgdpp", "dsgd"])
def test_set_blocks_matches_set_matrix_and_oracle(method):
    p = _problem()
    d = 3
    nb2 = d if method == "dsgd" else 2 * d
    ref = O.Problem(p.m, p.n, 10, d, p.rows, p.cols, p.vals, p.trows, p.tcols, p.tvals,
                    method=method)
    ref.configure(update_lambda=0.5)
    ref.set_factors(p.W0, p.H0)
    cfg = P.Config(m=p.m, n=p.n, rank=10, d=d, precision="fp64", exec="replay", method=method,
                   update_lambda=0.5)
    bn, li, lj, lx = _oracle_blocks(ref, d, nb2)
    tbn, ti, tj, tx = _oracle_blocks(ref, d, nb2, which=1)
    with P.Context(cfg) as ctx:
        ctx.set_blocks(P.TRAIN, bn, li, lj, lx)
        ctx.set_blocks(P.TEST, tbn, ti, tj, tx)
        ctx.set_factors(p.W0, p.H0)
        np.testing.assert_array_equal(ctx.block_nnz(P.TRAIN).ravel(), bn)
        a1, a2, _ = ctx.nnz12()
        r1, r2, _ = ref.nnz12()
        np.testing.assert_array_equal(a1, r1)
        np.testing.assert_array_equal(a2, r2)
        ctx.seed(11)
        ref.seed(11)
        for _ in range(2):
            ctx.epoch(0.02)
            ref.epoch(0.02)
        W, H = ctx.get_factors()
        Wr, Hr = ref.get_factors()
        np.testing.assert_array_equal(W, Wr)
        np.testing.assert_array_equal(H, Hr)
        assert ctx.nzsl(P.TEST) == pytest.approx(ref.nzsl(1), rel=LOSS_RTOL)


def test_set_blocks_rejects_entries_outside_their_block():
    p = _problem(m=60, n=40, nnz=300, ntest=30)
    d = 2
    cfg = P.Config(m=p.m, n=p.n, rank=4, d=d)
    bn = np.zeros(d * 2 * d, np.uint64)
    bn[0] = 2
    with P.Context(cfg) as ctx:
        # block (0, 0) spans rows [0, 30) and columns [0, 10)
        with pytest.raises(P.DsgdppError, match="outside their block"):
            ctx.set_blocks(P.TRAIN, bn, [0, 30], [0, 1], [1.0, 2.0])
        with pytest.raises(P.DsgdppError, match="outside their block"):
            ctx.set_blocks(P.TRAIN, bn, [0, 1], [0, 10], [1.0, 2.0])
        ctx.set_blocks(P.TRAIN, bn, [0, 29], [0, 9], [1.0, 2.0])
        assert int(ctx.block_nnz(P.TRAIN).sum()) == 2


def test_set_counts_replaces_the_update_weights():
    p = _problem()
    cfg = dict(m=p.m, n=p.n, rank=10, d=3, precision="fp64", exec="replay")
    with P.Context(P.Config(**cfg)) as a, P.Context(P.Config(**cfg)) as b:
        for ctx in (a, b):
            ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
            ctx.set_factors(p.W0, p.H0)
            ctx.seed(4)
        n1, n2, _ = a.nnz12()
        b.set_counts(n1, n2)  # the same counts: the same run, bit for bit
        a.epoch(0.02)
        b.epoch(0.02)
        np.testing.assert_array_equal(a.get_factors()[0], b.get_factors()[0])
        b.set_counts(n1 * 2, n2 * 2)  # doubled counts halve the regularization weights
        a.epoch(0.02)
        b.epoch(0.02)
        assert not np.array_equal(a.get_factors()[0], b.get_factors()[0])
        m1, m2, _ = b.nnz12()
        np.testing.assert_array_equal(m1, n1 * 2)
        with pytest.raises(P.DsgdppError):
            b.set_counts(np.full(p.m, 1 << 33, np.uint64), n2)
