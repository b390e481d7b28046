"""CPU tests of the mfdblock tool (the drop-in for tools/mfdblock.cc).

The blocks it writes are pinned against the oracle's blocking, which restates
ReadMatrixBlocksMm (mf/matrix/io/read_impl.h:364-486): each block holds
block-local coordinates sorted by (i, j), values of equal coordinates summed
in file order.
"""
import os
import subprocess

import numpy as np
import pytest

import dsgdpp_b200 as P
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TOOL = os.path.join(ROOT, "dsgdpp_b200", "bin", "mfdblock")
# a value written with 16 significant digits and read back
FMT_RTOL = 1e-15


def _run(args, cwd):
    return subprocess.run([TOOL] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


def _matrix_with_duplicates(m, n, nnz, seed):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, m, nnz).astype(np.uint32)
    cols = rng.integers(0, n, nnz).astype(np.uint32)
    vals = rng.normal(0, 1, nnz)
    # repeat some entries so that blocks hold duplicates, out of order
    k = nnz // 5
    rows = np.concatenate([rows, rows[:k][::-1]])
    cols = np.concatenate([cols, cols[:k][::-1]])
    vals = np.concatenate([vals, rng.normal(0, 1, k)])
    return rows, cols, vals


@pytest.mark.parametrize("d,method", [(3, "dsgdpp"), (4, "dsgd"), (1, "dsgdpp")])
def test_sparse_blocks_equal_the_oracle_blocking(tmp_path, monkeypatch, d, method):
    m, n = 37, 29
    rows, cols, vals = _matrix_with_duplicates(m, n, 400, seed=d)
    src = str(tmp_path / "V.mmc")
    P.write_mm_coord(src, m, n, rows, cols, vals)
    out = tmp_path / "blocks"
    out.mkdir()
    _, _, rows, cols, vals = P.read_sparse(src)  # the values as the tool reads them
    nb2 = d if method == "dsgd" else 2 * d
    r = _run([f"--blocks1={d}", "--blocks2", str(nb2), "--threads", "3", src,
              str(out / "V")], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    assert "Blocks            : %dx%d" % (d, nb2) in r.stdout
    assert "Output file       : V.xml (+ blocks)" in r.stdout
    ref = O.Problem(m, n, 2, d, rows, cols, vals, method=method)
    for b1 in range(d):
        for b2 in range(nb2):
            bm, bn, i, j, x = P.read_sparse(str(out / f"V-{b1}-{b2}.mmc"))
            ri, rj, rx = ref.block_records(b1, b2)
            np.testing.assert_array_equal(i, ri)
            np.testing.assert_array_equal(j, rj)
            # summed in file order, as the oracle; written with 16 significant
            # digits, as the reference writes them (write_impl.h:98)
            np.testing.assert_allclose(x, rx, rtol=FMT_RTOL, atol=0)
    # the descriptor: reference fields, default offsets, an empty path
    xml = open(out / "V.xml").read()
    assert "<path></path>" in xml and "<format>mmc</format>" in xml
    assert f"<filename>V-{d - 1}-{nb2 - 1}.mmc</filename>" in xml
    for off in P.block_offsets(n, nb2).tolist():
        assert f"<offset>{off}</offset>" in xml
    # the block names resolve against the reader's working directory
    monkeypatch.chdir(out)
    m2, n2, gi, gj, gx = P.read_sparse("V.xml")
    assert (m2, n2) == (m, n)
    assert len(gx) == int(ref.block_nnz().sum())


def test_dense_matrix_round_trips_through_mma_blocks(tmp_path, monkeypatch):
    W = np.random.default_rng(4).uniform(-1, 1, (23, 5))
    src = str(tmp_path / "W.mma")
    P.write_mm_array(src, W)
    r = _run(["--blocks1", "4", src, "Wb"], cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr
    xml = open(tmp_path / "Wb.xml").read()
    assert "<format>mma</format>" in xml and "<filename>Wb-3-0.mma</filename>" in xml
    monkeypatch.chdir(tmp_path)
    W = P.read_mm_array(src)  # the values as the tool reads them
    np.testing.assert_allclose(P.read_mm_array("Wb.xml"), W, rtol=FMT_RTOL, atol=0)
    offs = P.block_offsets(23, 4).tolist() + [23]
    for b in range(4):
        blk = P.read_mm_array(f"Wb-{b}-0.mma")
        assert blk.shape == (offs[b + 1] - offs[b], 5)
        np.testing.assert_allclose(blk, W[offs[b]:offs[b + 1]], rtol=FMT_RTOL, atol=0)


def test_blocked_input_is_blocked_again(tmp_path, monkeypatch):
    m, n = 41, 30
    rows, cols, vals = _matrix_with_duplicates(m, n, 300, seed=9)
    P.write_mm_coord(str(tmp_path / "V.mmc"), m, n, rows, cols, vals)
    _, _, rows, cols, vals = P.read_sparse(str(tmp_path / "V.mmc"))
    monkeypatch.chdir(tmp_path)
    assert _run(["--blocks1=2", "--blocks2=4", "V.mmc", "A"], cwd=str(tmp_path)).returncode == 0
    assert _run(["--blocks1=3", "--blocks2=6", "A.xml", "B"], cwd=str(tmp_path)).returncode == 0
    ref = O.Problem(m, n, 2, 3, rows, cols, vals)
    for b1 in range(3):
        for b2 in range(6):
            _, _, i, j, x = P.read_sparse(f"B-{b1}-{b2}.mmc")
            ri, rj, rx = ref.block_records(b1, b2)
            np.testing.assert_array_equal(i, ri)
            np.testing.assert_array_equal(j, rj)
            np.testing.assert_allclose(x, rx, rtol=2 * FMT_RTOL, atol=0)  # written twice


@pytest.mark.parametrize("args,msg", [
    ([], "mfdblock [options] <input-file> <output-base-file>"),
    (["--help"], "--blocks1 arg (=1)"),
    (["--blocks1=0", "V.mmc", "o"], "invalid value for --blocks1"),
    (["--blocks2=x", "V.mmc", "o"], "invalid value for --blocks2"),
    (["--format=mma", "V.mmc", "o"], "unsupported block format mma"),
    (["--format=bsb", "V.mmc", "o"], "unsupported block format bsb"),
    (["V.txt", "o"], "unsupported input file"),
    (["--speed=1", "V.mmc", "o"], "unrecognised option '--speed'"),
    (["missing.mmc", "o"], "Cannot open file missing.mmc"),
])
def test_usage_and_errors(tmp_path, args, msg):
    P.write_mm_coord(str(tmp_path / "V.mmc"), 3, 3, np.array([0], np.uint32),
                     np.array([1], np.uint32), np.array([1.0]))
    (tmp_path / "V.txt").write_text("x\n")
    r = _run(args, cwd=str(tmp_path))
    assert r.returncode == 1
    assert msg in r.stdout + r.stderr


def test_dense_descriptor_with_a_wrong_block_is_rejected(tmp_path, monkeypatch):
    W = np.arange(40, dtype=np.float64).reshape(8, 5)
    P.write_mm_array(str(tmp_path / "W.mma"), W)
    assert _run(["--blocks1=2", "W.mma", "Wb"], cwd=str(tmp_path)).returncode == 0
    P.write_mm_array(str(tmp_path / "Wb-1-0.mma"), W[:3])  # the descriptor says 4 x 5
    monkeypatch.chdir(tmp_path)
    with pytest.raises(Exception, match="the descriptor says 4 x 5"):
        P.read_mm_array("Wb.xml")
