"""The mfdsgdpp drop-in tool end to end on the GPU against the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "dsgdpp_b200", "bin", "mfdsgdpp")


def _write(tmp_path, p):
    P.write_mm_coord(str(tmp_path / "train.mmc"), p.m, p.n, p.rows, p.cols, p.vals)
    P.write_mm_coord(str(tmp_path / "test.mmc"), p.m, p.n, p.trows, p.tcols, p.tvals)
    P.write_mm_array(str(tmp_path / "W.mma"), p.W0)
    P.write_mm_array(str(tmp_path / "H.mma"), p.H0.T)


@pytest.mark.parametrize("tool", ["mfdsgdpp", "mfdsgd"])
@pytest.mark.parametrize("blocked", [False, True])
def test_cli_replay_matches_oracle(tmp_path, blocked, tool):
    p = synth.make(400, 300, 6000, 600, rank_true=4, r=5, noise=0.1, seed=4)
    _write(tmp_path, p)
    d = 3
    dsgd = tool == "mfdsgd"  # d x d blocks, d sub-epochs (mf/sgd/dsgd_impl.h)
    train = str(tmp_path / "train.mmc")
    if blocked:
        train = str(tmp_path / "V.xml")
        P.write_blocked(train, str(tmp_path), "V", p.m, p.n, d, d if dsgd else 2 * d, p.rows,
                        p.cols, p.vals)
    extra = ["--map-reduce=1"] if dsgd else []
    r = subprocess.run([os.path.join(os.path.dirname(CLI), tool), *extra,
                        f"--input-file={train}", f"--input-test-file={tmp_path}/test.mmc",
                        f"--input-row-file={tmp_path}/W.mma", f"--input-col-file={tmp_path}/H.mma",
                        "--rank=5", f"--tasks-per-rank={d}", "--update=Nzsl_L2(1)",
                        "--regularize=None", "--loss=Nzsl_L2(1)", "--decay=BoldDriver(0.01)",
                        "--epochs=4", "--seed=1499881717", "--precision=fp64", "--exec=replay",
                        f"--trace={tmp_path}/trace.R", f"--output-row-file={tmp_path}/Wout.mma",
                        f"--output-col-file={tmp_path}/Hout.mma"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    # the same job on the oracle; the files hold 16 significant digits
    W0 = P.read_mm_array(str(tmp_path / "W.mma"))
    H0 = P.read_mm_array(str(tmp_path / "H.mma")).T
    _, _, tr, tc, tv = P.read_sparse(str(tmp_path / "train.mmc"))
    _, _, sr, sc, sv = P.read_sparse(str(tmp_path / "test.mmc"))
    ref = O.Problem(p.m, p.n, 5, d, tr, tc, tv, sr, sc, sv,
                    method="dsgd" if dsgd else "dsgdpp").configure()
    ref.set_factors(W0, H0)
    ref.seed(1499881717)
    trace = ref.run(4, "BoldDriver", 0.01)
    W, H = ref.get_factors()
    np.testing.assert_allclose(P.read_mm_array(str(tmp_path / "Wout.mma")), W, rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(P.read_mm_array(str(tmp_path / "Hout.mma")).T, H, rtol=1e-14, atol=1e-15)
    losses = [float(x) for x in re.findall(r"\| Loss: ([0-9.e+-]+)", r.stdout)]
    assert len(losses) == 5
    np.testing.assert_allclose(losses, trace[:, 0], rtol=1e-5)
    text = open(tmp_path / "trace.R").read()
    assert text.startswith("trace <- list(trace=list(")
    assert "eps=NA" in text and 'update = "Nzsl_L2(1)"' in text and "rank = 5" in text
    assert "Step size: 0.01 " in r.stdout and "Finished epoch 4" in r.stdout
    if dsgd:
        assert "Starting DSGD on" in r.stdout and "DSGD options" in r.stdout
        assert "Slow MapReduce implementation: 1" in r.stdout


def test_cli_runs_on_mfdblock_output(tmp_path):
    # the reference's pipeline: mfdblock blocks the data matrix d x 2d and the
    # factors d x 1 / 1 x 2d (.xml descriptors with an empty path, so both
    # tools run in the directory of the blocks); mfdsgdpp on those files gives
    # the run on the plain files, up to the values' 16-digit rewrite
    p = synth.make(400, 300, 6000, 600, rank_true=4, r=5, noise=0.1, seed=4)
    _write(tmp_path, p)
    d = 3
    block = os.path.join(os.path.dirname(CLI), "mfdblock")
    for args in (["--blocks1=3", "--blocks2=6", "train.mmc", "V"],
                 ["--blocks1=3", "W.mma", "Wb"], ["--blocks2=6", "H.mma", "Hb"]):
        r = subprocess.run([block] + args, cwd=str(tmp_path), capture_output=True, text=True,
                           timeout=120)
        assert r.returncode == 0, r.stdout + r.stderr
    outs = {}
    for tag, (v, w, h) in {"plain": ("train.mmc", "W.mma", "H.mma"),
                           "blocked": ("V.xml", "Wb.xml", "Hb.xml")}.items():
        r = subprocess.run([CLI, f"--input-file={v}", "--input-test-file=test.mmc",
                            f"--input-row-file={w}", f"--input-col-file={h}", "--rank=5",
                            f"--tasks-per-rank={d}", "--update=Nzsl_L2(1)", "--regularize=None",
                            "--loss=Nzsl_L2(1)", "--decay=BoldDriver(0.01)", "--epochs=3",
                            "--seed=7", "--precision=fp64", "--exec=replay",
                            f"--output-row-file=W-{tag}.mma", f"--output-col-file=H-{tag}.mma"],
                           cwd=str(tmp_path), capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stdout + r.stderr
        losses = [float(x) for x in re.findall(r"\| Loss: ([0-9.e+-]+)", r.stdout)]
        outs[tag] = (losses, P.read_mm_array(str(tmp_path / f"W-{tag}.mma")),
                     P.read_mm_array(str(tmp_path / f"H-{tag}.mma")))
        if tag == "blocked":
            for f in (v, w, h):
                assert f"File '{f}' is not blocked" not in r.stdout
    assert len(outs["plain"][0]) == 4
    for a, b in zip(outs["plain"], outs["blocked"]):
        np.testing.assert_allclose(np.asarray(b), np.asarray(a), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("tool", ["mfdsgdpp", "mfdsgd"])
def test_cli_multirank_path_with_one_rank_matches_oracle(tmp_path, tool):
    # the tool's path for several ranks (task range, counts of the whole
    # matrix, NCCL hand-off, losses summed over the ranks), run with one rank
    p = synth.make(400, 300, 6000, 600, rank_true=4, r=5, noise=0.1, seed=4)
    _write(tmp_path, p)
    d = 3
    dsgd = tool == "mfdsgd"
    env = dict(os.environ, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([os.path.join(os.path.dirname(CLI), tool),
                        f"--input-file={tmp_path}/train.mmc", f"--input-test-file={tmp_path}/test.mmc",
                        f"--input-row-file={tmp_path}/W.mma", f"--input-col-file={tmp_path}/H.mma",
                        "--rank=5", f"--tasks-per-rank={d}", "--update=Nzsl_L2(1)",
                        "--regularize=None", "--loss=Nzsl_L2(1)", "--decay=BoldDriver(0.01)",
                        "--epochs=4", "--seed=1499881717", "--precision=fp64", "--exec=replay",
                        f"--shard-id-file={tmp_path}/nccl.id",
                        f"--output-row-file={tmp_path}/Wout.mma",
                        f"--output-col-file={tmp_path}/Hout.mma"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "1 ranks, one GPU each" in r.stdout
    assert not os.path.exists(tmp_path / "nccl.id")  # removed once every rank joined
    W0 = P.read_mm_array(str(tmp_path / "W.mma"))
    H0 = P.read_mm_array(str(tmp_path / "H.mma")).T
    _, _, tr, tc, tv = P.read_sparse(str(tmp_path / "train.mmc"))
    _, _, sr, sc, sv = P.read_sparse(str(tmp_path / "test.mmc"))
    ref = O.Problem(p.m, p.n, 5, d, tr, tc, tv, sr, sc, sv,
                    method="dsgd" if dsgd else "dsgdpp").configure()
    ref.set_factors(W0, H0)
    ref.seed(1499881717)
    trace = ref.run(4, "BoldDriver", 0.01)
    W, H = ref.get_factors()
    np.testing.assert_allclose(P.read_mm_array(str(tmp_path / "Wout.mma")), W, rtol=1e-14, atol=1e-15)
    np.testing.assert_allclose(P.read_mm_array(str(tmp_path / "Hout.mma")).T, H, rtol=1e-14, atol=1e-15)
    losses = [float(x) for x in re.findall(r"\| Loss: ([0-9.e+-]+)", r.stdout)]
    np.testing.assert_allclose(losses, trace[:, 0], rtol=1e-5)
    tests = [float(x) for x in re.findall(r"\| Test loss: ([0-9.e+-]+)", r.stdout)]
    np.testing.assert_allclose(tests, trace[:, 1], rtol=1e-5)
