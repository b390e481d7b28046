"""The allocation-free loss entry point (dsgdpp_nzsl_fp32_noalloc).

Some callers cannot allocate device memory themselves -- code that runs inside
another framework's memory pool, or under an allocator it does not own -- so
this entry point takes caller-owned device buffers and keeps its scratch in a
fixed device array.  This test calls it through the C ABI and checks its
result against the existing entry point (dsgdpp_nzsl on a context holding the
same FP32 data), within the 1e-12 relative tolerance of the other loss tests,
on consecutive calls that share the scratch.  It lives in a file of its own
that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth

pytestmark = pytest.mark.gpu
LOSS_RTOL = 1e-12


def _device(torch, a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def _padded(torch, a, ld):
    out = np.zeros((a.shape[0], ld), np.float32)
    out[:, :a.shape[1]] = a.astype(np.float32)
    return _device(torch, out, torch.float32)


def _call(torch, rows, cols, vals, W, H, r, ld, partials=0):
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    rc = P.lib.dsgdpp_nzsl_fp32_noalloc(
        rows.data_ptr(), cols.data_ptr(), vals.data_ptr(), vals.numel(), W.data_ptr(),
        H.data_ptr(), r, ld, partials, out.data_ptr(), None)
    assert rc == P.OK
    torch.cuda.synchronize()
    return float(out.item())


def test_noalloc_nzsl_matches_context_loss():
    import torch
    r, ld = 30, 32
    p = synth.make(3000, 2000, 80000, 9000, rank_true=8, r=r, noise=0.1, seed=21, kind="zipf")
    with P.Context(P.Config(m=p.m, n=p.n, rank=r, d=4, precision="fp32")) as ctx:
        ctx.set_matrix(P.TRAIN, p.rows, p.cols, p.vals)
        ctx.set_matrix(P.TEST, p.trows, p.tcols, p.tvals)
        ctx.set_factors(p.W0, p.H0)
        want_train, want_test = ctx.nzsl(P.TRAIN), ctx.nzsl(P.TEST)
    W, H = _padded(torch, p.W0, ld), _padded(torch, p.H0, ld)
    # entry values are held in FP32, as in the context
    tr = [_device(torch, p.rows.view(np.int32), torch.int32),
          _device(torch, p.cols.view(np.int32), torch.int32),
          _device(torch, p.vals.astype(np.float32), torch.float32)]
    te = [_device(torch, p.trows.view(np.int32), torch.int32),
          _device(torch, p.tcols.view(np.int32), torch.int32),
          _device(torch, p.tvals.astype(np.float32), torch.float32)]
    # two calls in a row share the scratch: training entries, then test entries
    got_train = _call(torch, *tr, W, H, r, ld)
    got_test = _call(torch, *te, W, H, r, ld)
    assert got_train == pytest.approx(want_train, rel=LOSS_RTOL)
    assert got_test == pytest.approx(want_test, rel=LOSS_RTOL)
    # fewer partial sums than the previous call: stale slots are not read
    assert _call(torch, *te, W, H, r, ld, partials=7) == pytest.approx(want_test, rel=LOSS_RTOL)
    assert _call(torch, *tr, W, H, r, ld, partials=4096) == pytest.approx(
        want_train, rel=LOSS_RTOL)


def test_noalloc_rejects_requests_beyond_capacity():
    import torch
    W = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    idx = torch.zeros(1, dtype=torch.int32, device="cuda")
    v = torch.zeros(1, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    args = (idx.data_ptr(), idx.data_ptr(), v.data_ptr(), 1, W.data_ptr(), W.data_ptr(), 4, 4)
    assert P.lib.dsgdpp_nzsl_fp32_noalloc(*args, 4097, out.data_ptr(), None) == P.E_INVALID
    # a row stride that is not a whole number of 16-byte vectors is refused
    assert P.lib.dsgdpp_nzsl_fp32_noalloc(idx.data_ptr(), idx.data_ptr(), v.data_ptr(), 1,
                                          W.data_ptr(), W.data_ptr(), 3, 3, 0, out.data_ptr(),
                                          None) == P.E_INVALID
    # a row wider than the widest loss kernel (512 floats) is refused, not failed
    wide = torch.zeros((2, 516), dtype=torch.float32, device="cuda")
    assert P.lib.dsgdpp_nzsl_fp32_noalloc(idx.data_ptr(), idx.data_ptr(), v.data_ptr(), 1,
                                          wide.data_ptr(), wide.data_ptr(), 516, 516, 0,
                                          out.data_ptr(), None) == P.E_INVALID
    assert P.lib.dsgdpp_nzsl_fp32_noalloc(*args, 1, out.data_ptr(), None) == P.OK
    torch.cuda.synchronize()
