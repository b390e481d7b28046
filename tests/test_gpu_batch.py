"""GPU tests of the batched form (dsgdpp_batch_*): many problems per launch.

* Each problem of a batch tracks the sequential FP64 oracle run on that
  problem alone with the same d, seed and (constant) step, to the Hogwild
  tolerances of the single-problem path.
* The per-problem losses the batch reports equal the losses of the factors it
  returns, recomputed here in FP64 (segmented reductions, lazy-L2 scaling).
* Invalid or unsupported requests fail with a status, not a crash.
"""
import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# (m, n, nnz, rank): uneven sizes, ranks that share and do not share a padded width
SHAPES = [(6000, 5000, 120000, 8), (20000, 8000, 300000, 16), (3000, 2500, 40000, 10),
          (12000, 15000, 200000, 16), (9000, 4000, 150000, 32)]


def _problems(shapes, seed0=11, ntest_frac=0.1):
    out = []
    for k, (m, n, nnz, r) in enumerate(shapes):
        p = synth.make(m, n, nnz, int(nnz * ntest_frac), rank_true=min(r, 8), r=r, noise=0.1,
                       seed=seed0 + k)
        out.append(dict(m=m, n=n, rank=r, rows=p.rows, cols=p.cols, vals=p.vals,
                        trows=p.trows, tcols=p.tcols, tvals=p.tvals, W=p.W0, H=p.H0,
                        seed=100 + k, eps0=0.01, _p=p))
    return out


def _nzsl(W, H, rows, cols, vals):
    pred = np.einsum("ij,ij->i", W[rows], H[cols])
    return float(np.sum((vals - pred) ** 2))


@pytest.mark.parametrize("precision,tol", [("fp32", 0.01), ("bf16", 0.02)])
def test_batch_tracks_oracle_per_problem(precision, tol):
    probs = _problems(SHAPES)
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision=precision, regularize="L2",
                   regularize_lambda=0.02)
    epochs = 6
    with P.Batch(cfg, probs) as b:
        ds = [b.problem_d(k) for k in range(len(probs))]
        _, test, ms = b.run(epochs, decrease=1.0, increase=1.0)  # constant step
        assert ms > 0
    for k, q in enumerate(probs):
        p = q["_p"]
        ref = O.Problem(p.m, p.n, q["rank"], ds[k], p.rows, p.cols, p.vals, p.trows, p.tcols,
                        p.tvals)
        ref.configure(regularize="L2", regularize_lambda=0.02)
        ref.set_factors(p.W0, p.H0)
        ref.seed(q["seed"])
        for _ in range(epochs):
            ref.epoch(q["eps0"])
        want = float(np.sqrt(ref.nzsl(1) / len(p.tvals)))
        got = float(np.sqrt(test[k] / len(p.tvals)))
        start = float(np.sqrt(_nzsl(p.W0, p.H0, p.trows, p.tcols, p.tvals) / len(p.tvals)))
        assert abs(got - want) <= tol * want, (k, ds[k], got, want)
        assert want < 0.97 * start, (k, want, start)  # the run made progress


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_batch_losses_match_returned_factors(precision):
    probs = _problems(SHAPES[:4], seed0=21)
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision=precision, regularize="L2",
                   regularize_lambda=0.02, loss="Nzsl_L2", loss_lambda=0.5)
    with P.Batch(cfg, probs) as b:
        train, test, _ = b.run(3)  # BoldDriver per problem
        for k, q in enumerate(probs):
            W, H = b.get_factors(k)
            # with FP32 factors the entry values are held in FP32 on the device
            cast = (lambda v: v.astype(np.float32).astype(np.float64)) if precision == "fp32" \
                else (lambda v: v)
            want_tr = _nzsl(W, H, q["rows"], q["cols"], cast(q["vals"])) + 0.5 * (
                float(np.sum(W * W)) + float(np.sum(H * H)))
            want_te = _nzsl(W, H, q["trows"], q["tcols"], cast(q["tvals"]))
            np.testing.assert_allclose(train[k], want_tr, rtol=1e-9)
            np.testing.assert_allclose(test[k], want_te, rtol=1e-9)


def test_batch_zero_epochs_reports_initial_losses():
    probs = _problems(SHAPES[:3], seed0=31)
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision="fp64", loss="Nzsl")
    with P.Batch(cfg, probs) as b:
        train, test, ms = b.run(0)
        assert ms == 0
    for k, q in enumerate(probs):
        np.testing.assert_allclose(train[k], _nzsl(q["W"], q["H"], q["rows"], q["cols"],
                                                   q["vals"]), rtol=1e-12)
        np.testing.assert_allclose(test[k], _nzsl(q["W"], q["H"], q["trows"], q["tcols"],
                                                  q["tvals"]), rtol=1e-12)


def test_batch_stream_and_graph_launch_agree_on_progress():
    probs = _problems(SHAPES[:3], seed0=41)
    res = []
    for launch in ("stream", "graph"):
        cfg = P.Config(m=1, n=1, rank=1, d=1, precision="fp32", launch=launch)
        with P.Batch(cfg, probs) as b:
            res.append(b.run(5, decrease=1.0, increase=1.0)[1])
    np.testing.assert_allclose(res[0], res[1], rtol=0.01)


def test_batch_given_d_and_tiny_problems():
    # d = 1 problems with a handful of entries sit next to larger ones
    rng = np.random.default_rng(3)
    probs = _problems(SHAPES[:2], seed0=51)
    for k in range(3):
        m, n = 5 + k, 4 + k
        rows = rng.integers(0, m, 6).astype(np.uint32)
        cols = rng.integers(0, n, 6).astype(np.uint32)
        probs.append(dict(m=m, n=n, rank=8, d=1, rows=rows, cols=cols,
                          vals=rng.normal(size=6), W=rng.uniform(-0.5, 0.5, (m, 8)),
                          H=rng.uniform(-0.5, 0.5, (n, 8)), seed=k, eps0=0.01))
    probs[0]["d"] = 2
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision="fp32")
    with P.Batch(cfg, probs) as b:
        assert b.problem_d(0) == 2
        assert all(b.problem_d(k) == 1 for k in range(2, 5))
        train, _, _ = b.run(4)
        assert np.all(np.isfinite(train))


def test_batch_errors():
    probs = _problems(SHAPES[:1], seed0=61)
    with pytest.raises(P.DsgdppError):
        P.Batch(P.Config(m=1, n=1, rank=1, d=1, exec="replay", precision="fp64"), probs)
    with pytest.raises(P.DsgdppError):
        P.Batch(P.Config(m=1, n=1, rank=1, d=1, truncate=(-1.0, 1.0)), probs)
    bad = dict(probs[0], d=probs[0]["n"])  # 2d > n
    with pytest.raises(P.DsgdppError):
        P.Batch(P.Config(m=1, n=1, rank=1, d=1), [bad])
    with pytest.raises(P.DsgdppError):
        P.Batch(P.Config(m=1, n=1, rank=1, d=1), [])


def test_batch_autotune_picks_valid_shapes():
    probs = _problems(SHAPES, seed0=71)
    probs[1]["d"] = 3  # a problem's own d is kept
    cfg = P.Config(m=1, n=1, rank=1, d=1, precision="fp32")
    ds, ctas, ms = P.Batch.autotune(cfg, probs, sample_stride=2, epochs=1)
    assert ds[1] == 3 and ctas in (0, 2, 3) and ms > 0
    for d, q in zip(ds, probs):
        assert 1 <= d <= 32 and d <= q["m"] and 2 * d <= q["n"]
    for p, d in zip(probs, ds):
        p["d"] = d
    cfg.ctas_per_sm = ctas
    with P.Batch(cfg, probs) as b:
        assert [b.problem_d(k) for k in range(len(probs))] == ds
        train, _, _ = b.run(2)
        assert np.all(np.isfinite(train))
