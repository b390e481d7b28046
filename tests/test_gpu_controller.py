"""GPU tests of the learned step-size controller's runner (dsgdpp_run_controlled).

* The fallback: with a network that always proposes the largest increase, no
  kept epoch raises the training loss by more than 1%, and rises are counted.
* The gain: the committed trained network reaches BoldDriver's final test loss
  in less wall time than BoldDriver itself, on a matrix of the training
  family that the network was not trained on (time counts every epoch,
  rollback re-run, loss evaluation and step decision).
"""
import math
import os

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200.controller import time_to_target

pytestmark = pytest.mark.gpu

PARAMS = os.path.join(os.path.dirname(P.__file__), "controller_params.npy")


def _problem(seed=12345, m=100_000, n=30_000, nnz=3_000_000, r=32):
    from dsgdpp_b200 import synth_gpu
    return synth_gpu.make(m, n, nnz, nnz // 50, rank_true=r, r=r, noise=0.2, seed=seed,
                          s_row=1.1, s_col=1.1, device="cuda:0"), (m, n, r)


def _context(data, shape, seed=7, d=16):
    m, n, r = shape
    ctx = P.Context(P.Config(m=m, n=n, rank=r, d=d, regularize="L2", regularize_lambda=0.05))
    ctx.set_matrix(P.TRAIN, data["rows"], data["cols"], data["vals"])
    ctx.set_matrix(P.TEST, data["trows"], data["tcols"], data["tvals"])
    ctx.set_factors(data["W0"], data["H0"])
    ctx.seed(seed)
    return ctx


def test_fallback_keeps_loss_from_rising():
    data, shape = _problem()
    net = P.Mlp(seed=3)
    p = np.zeros(net.n_params, np.float32)
    p[-1] = 5.0  # output bias: raw output 5, proposal clipped to +1 (eps * e) every epoch
    net.params = p
    with _context(data, shape) as ctx:
        tr, fb = ctx.run_controlled(net, 14, eps0=0.002)
    losses = [r["loss"] for r in tr]
    assert fb > 0  # always increasing the step must overshoot
    for a, b in zip(losses, losses[1:]):
        assert math.isfinite(b) and b <= a * 1.01 * (1 + 1e-12), (a, b)


def test_trained_controller_beats_bolddriver():
    net = P.Mlp(seed=1)
    net.params = np.load(PARAMS)
    data, shape = _problem(seed=424242)
    ntest = len(data["tvals"])
    with _context(data, shape) as ctx:
        base = ctx.run(40, "BoldDriver", 0.001)
    target = base[-1]["test_loss"]
    _, t_base = time_to_target(base, target)
    with _context(data, shape) as ctx:
        tr, fb = ctx.run_controlled(net, 80, eps0=0.001, target_test_loss=target)
    ep, t_ctl = time_to_target(tr, target)
    assert ep is not None, ("controller never reached", math.sqrt(target / ntest))
    assert t_ctl <= 0.8 * t_base, (t_ctl, t_base, ep, fb)
