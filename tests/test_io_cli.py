"""CPU tests of the .mmc/.mma/.xml I/O and of the mfdsgdpp command line."""
import os
import subprocess

import numpy as np
import pytest

import dsgdpp_b200 as P
from dsgdpp_b200 import synth
from tests.conftest import HAS_GPU

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "dsgdpp_b200", "bin", "mfdsgdpp")


def test_mmc_roundtrip(tmp_path):
    p = synth.make(50, 40, 300, 0, rank_true=2, r=2, noise=0.1, seed=1)
    f = str(tmp_path / "v.mmc")
    P.write_mm_coord(f, 50, 40, p.rows, p.cols, p.vals)
    m, n, r, c, v = P.read_sparse(f)
    assert (m, n) == (50, 40)
    np.testing.assert_array_equal(r, p.rows)
    np.testing.assert_array_equal(c, p.cols)
    np.testing.assert_allclose(v, p.vals, rtol=1e-15)
    text = open(f).read().splitlines()
    assert text[0] == "%%MatrixMarket matrix coordinate real general"
    assert f"{p.rows[0] + 1} {p.cols[0] + 1} " in text[text.index("50 40 300") + 1]


def test_mma_roundtrip_column_major(tmp_path):
    a = np.arange(12, dtype=np.float64).reshape(3, 4) / 8.0
    f = str(tmp_path / "w.mma")
    P.write_mm_array(f, a)
    lines = open(f).read().splitlines()
    assert lines[0] == "%%MatrixMarket matrix array real general"
    assert lines[3] == "3 4"
    assert [float(x) for x in lines[4:7]] == a[:, 0].tolist()  # column by column
    np.testing.assert_array_equal(P.read_mm_array(f), a)


def test_mma_sixteen_significant_digits(tmp_path):
    f = str(tmp_path / "x.mma")
    P.write_mm_array(f, np.array([[1.0 / 3.0]]))
    assert open(f).read().splitlines()[-1] == "0.3333333333333333"


def test_xml_blocked_roundtrip(tmp_path):
    p = synth.make(37, 29, 200, 0, rank_true=2, r=2, noise=0.1, seed=2)
    xml = str(tmp_path / "V.xml")
    P.write_blocked(xml, str(tmp_path), "V", 37, 29, 3, 6, p.rows, p.cols, p.vals)
    m, n, r, c, v = P.read_sparse(xml)
    assert (m, n) == (37, 29)
    got = sorted(zip(r.tolist(), c.tolist(), v.tolist()))
    want = sorted(zip(p.rows.tolist(), p.cols.tolist(), p.vals.tolist()))
    assert [g[:2] for g in got] == [w[:2] for w in want]
    np.testing.assert_allclose([g[2] for g in got], [w[2] for w in want], rtol=1e-15)
    text = open(xml).read()
    assert "<blocks1>3</blocks1>" in text and "<filename>V-2-5.mmc</filename>" in text
    # block files hold block-local coordinates
    blk = P.read_sparse(str(tmp_path / "V-0-0.mmc"))
    assert blk[0] == 13 and blk[1] == 5  # 37 = 13+12+12, 29 = 5+5+5+5+5+4


@pytest.mark.parametrize("content,msg", [
    ("%%MatrixMarket matrix array real general\n1 1\n1\n", "Wrong matrix-market banner"),
    ("%%MatrixMarket matrix coordinate real general\n% c\n2 2 2\n1 1 1.0\n", "Unexpected EOF"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1.0\n", "Parse error at line 3"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 1 1.0\n2 2 2.0\n",
     "Unexpected input at at line 4"),
    ("%%MatrixMarket matrix coordinate real general\n2 2\n", "Invalid matrix dimensions"),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", "Parse error"),
])
def test_mmc_errors(tmp_path, content, msg):
    f = tmp_path / "bad.mmc"
    f.write_text(content)
    with pytest.raises(P.DsgdppError) as e:
        P.read_sparse(str(f))
    assert msg in str(e.value)
    assert e.value.status == P.E_IO


def test_missing_file():
    with pytest.raises(P.DsgdppError):
        P.read_sparse("/nonexistent/file.mmc")


def _cli(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=120)


def test_cli_requires_options():
    r = _cli("--input-file=x.mmc")
    assert r.returncode == 1
    assert "have to be present" in r.stderr
    assert "--stratum-order" in r.stdout


def _files(tmp_path):
    p = synth.make(60, 50, 500, 50, rank_true=3, r=3, noise=0.1, seed=3)
    P.write_mm_coord(str(tmp_path / "train.mmc"), 60, 50, p.rows, p.cols, p.vals)
    P.write_mm_coord(str(tmp_path / "test.mmc"), 60, 50, p.trows, p.tcols, p.tvals)
    P.write_mm_array(str(tmp_path / "W.mma"), p.W0)
    P.write_mm_array(str(tmp_path / "H.mma"), p.H0.T)
    return p


def _base(tmp_path):
    return [f"--input-file={tmp_path}/train.mmc", f"--input-test-file={tmp_path}/test.mmc",
            f"--input-row-file={tmp_path}/W.mma", f"--input-col-file={tmp_path}/H.mma",
            "--rank=3", "--tasks-per-rank=2"]


@pytest.mark.parametrize("upd,reg,loss", [("Nzsl_L2(1)", "L1(1)", "Nzsl_L2(1)"),
                                          ("Nzsl", "None", "Nzsl_L2(1)"),
                                          ("Sl", "None", "Sl")])
def test_cli_invalid_combination(tmp_path, upd, reg, loss):
    _files(tmp_path)
    r = _cli(*_base(tmp_path), f"--update={upd}", f"--regularize={reg}", f"--loss={loss}",
             "--decay=BoldDriver(0.01)")
    assert r.returncode == 1
    assert "Invalid combination of update, regularize, and loss arguments" in r.stderr


def test_cli_wrong_arity_and_abs(tmp_path):
    _files(tmp_path)
    r = _cli(*_base(tmp_path), "--update=Nzsl_L2", "--regularize=None", "--loss=Nzsl_L2(1)",
             "--decay=BoldDriver(0.01)")
    assert r.returncode == 1 and "Invalid number of arguments in Nzsl_L2" in r.stdout
    r = _cli(*_base(tmp_path), "--update=Nzsl", "--regularize=None", "--loss=Nzsl", "--abs",
             "--decay=BoldDriver(0.01)")
    assert r.returncode == 1 and "Invalid combination" in r.stderr


def test_cli_bad_orders_and_decay(tmp_path):
    _files(tmp_path)
    common = [*_base(tmp_path), "--update=Nzsl", "--regularize=None", "--loss=Nzsl"]
    r = _cli(*common, "--decay=BoldDriver(0.01)", "--sgd-order=XYZ")
    assert r.returncode == 1 and 'expected "SEQ", "WR" or "WOR"' in r.stderr
    r = _cli(*common, "--decay=BoldDriver(0.01)", "--stratum-order=XYZ")
    assert r.returncode == 1 and "Invalid arguments for stratumOrder" in r.stderr
    r = _cli(*common, "--decay=Foo(1)")
    assert r.returncode == 1 and "Unknown or invalid loss 'Foo(1)'" in r.stderr
    r = _cli(*common, "--decay=BoldDriver(0.01)", "--truncate=(1)")
    assert r.returncode == 1 and "(<min>,<max>)" in r.stderr


@pytest.mark.skipif(HAS_GPU, reason="checks the behaviour without a GPU")
def test_cli_fails_loudly_without_gpu(tmp_path):
    _files(tmp_path)
    r = _cli(*_base(tmp_path), "--update=Nzsl_L2(1)", "--regularize=None", "--loss=Nzsl_L2(1)",
             "--decay=BoldDriver(0.01)", "--epochs=1")
    assert r.returncode == 1
    assert "dsgdpp_create" in r.stderr
    assert "    Update function: Nzsl_L2(1)" in r.stdout


def test_dsgd_tool_name_and_map_reduce_option(tmp_path):
    _files(tmp_path)
    dsgd = os.path.join(os.path.dirname(CLI), "mfdsgd")
    r = subprocess.run([dsgd, "--input-file=x.mmc"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and r.stdout.startswith("mfdsgd [options]")
    common = [*_base(tmp_path), "--update=Nzsl", "--regularize=None", "--loss=Nzsl",
              "--decay=BoldDriver(0.01)"]
    r = _cli(*common, "--map-reduce=1")  # mfdsgdpp has no such option
    assert r.returncode == 1 and "unrecognised option '--map-reduce'" in r.stderr
    r = subprocess.run([dsgd, *common, "--map-reduce=maybe"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "'--map-reduce' is invalid" in r.stderr


def test_writers_format_like_printf_16g(tmp_path):
    # the reference writes with 16 significant digits (write_impl.h:51,98); the
    # multi-threaded writers must give printf's %.16g text for every value
    rng = np.random.default_rng(3)
    vals = np.concatenate([rng.standard_normal(200_000) * 10.0 ** rng.integers(-300, 300, 200_000),
                           [0.0, -0.0, 1e-310, 5e-324, 1.7976931348623157e308, np.inf, -np.inf,
                            np.nan, 1.0, 0.1, 1e16, 1e15, 9.999999999999999e15]])
    P.write_mm_array(str(tmp_path / "v.mma"), vals.reshape(-1, 1))
    lines = open(tmp_path / "v.mma").read().splitlines()
    assert lines[3] == f"{len(vals)} 1"
    assert lines[4:] == ["%.16g" % x for x in vals]
    rows = rng.integers(0, 1000, len(vals)).astype(np.uint32)
    cols = rng.integers(0, 50, len(vals)).astype(np.uint32)
    P.write_mm_coord(str(tmp_path / "v.mmc"), 1000, 50, rows, cols, vals)
    body = open(tmp_path / "v.mmc").read().splitlines()[7:]
    assert body == ["%d %d %s" % (i + 1, j + 1, "%.16g" % x) for i, j, x in zip(rows, cols, vals)]


def test_readers_take_what_strtod_takes(tmp_path):
    # values are parsed in place; anything unusual must still read as strtod reads it
    import ctypes
    libc = ctypes.CDLL(None)
    libc.strtod.restype = ctypes.c_double
    libc.strtod.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    vals = ["1", "+2.5", "-0", "1e-310", "1e400", "-1e400", "0x1p3", "inf", "-Infinity", "nan",
            "  7.25  ", "3.", ".5", "1E+5", "1.7976931348623157e308", "4.9e-324"]
    path = tmp_path / "s.mma"
    path.write_text("%%MatrixMarket matrix array real general\n%c\n"
                    + f"{len(vals)} 1\n" + "\n".join(vals) + "\n")
    got = P.read_mm_array(str(path)).ravel()
    want = np.array([libc.strtod(x.encode(), None) for x in vals])
    np.testing.assert_array_equal(got, want)
    assert np.array_equal(np.signbit(got), np.signbit(want))
    coo = tmp_path / "s.mmc"
    coo.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n+1 2 0x1p-2\n3\t3  -1e400\n")
    _, _, r, c, v = P.read_sparse(str(coo))
    assert list(r) == [0, 2] and list(c) == [1, 2] and v[0] == 0.25 and v[1] == -np.inf
    for bad in ("1.5x", "abc", ""):
        path.write_text("%%MatrixMarket matrix array real general\n1 1\n" + bad + "\n")
        with pytest.raises(P.DsgdppError, match="Parse error at line 3"):
            P.read_mm_array(str(path))


def test_cli_rm_input_errors(tmp_path):
    # .rm inputs are checked before any device work
    base = ["--rank=3", "--tasks-per-rank=2", "--update=Nzsl", "--regularize=None", "--loss=Nzsl",
            "--decay=BoldDriver(0.01)"]
    missing = str(tmp_path / "none.rm")
    r = _cli(f"--input-file={missing}", f"--input-row-file={missing}",
             f"--input-col-file={missing}", *base)
    assert r.returncode == 1 and "Cannot open file" in r.stderr
    factors_only = str(tmp_path / "f.rm")
    P.RandomMatrix.create(60, 40, 3, 4, 0, 0, 3, "Uniform(-1,1)").save(factors_only)
    r = _cli(f"--input-file={factors_only}", f"--input-row-file={factors_only}",
             f"--input-col-file={factors_only}", *base)
    assert r.returncode == 1 and "holds no data matrix" in r.stderr
    assert "generating data matrices on the fly" in r.stdout


def test_quickstart_files_like_generate_synthetic_data(tmp_path):
    # python -m dsgdpp_b200.synth writes the quick start's four files with the
    # shapes and distributions of tools/generateSyntheticData.cc
    import sys
    r = subprocess.run([sys.executable, "-m", "dsgdpp_b200.synth", "--out-dir", str(tmp_path),
                        "--size1", "300", "--size2", "200", "--nnz", "3000", "--nnz-test", "400",
                        "--rank", "4", "--seed", "3"], cwd=ROOT, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    m, n, rows, cols, vals = P.read_sparse(str(tmp_path / "train.mmc"))
    assert (m, n, len(vals)) == (300, 200, 3000)
    keys = rows.astype(np.int64) * n + cols
    assert np.all(np.diff(keys) > 0)  # distinct cells, row by row
    assert 250 < vals.var() < 600  # 4 products of N(0, 10) entries, plus N(0, 1)
    _, _, tr, tc, tv = P.read_sparse(str(tmp_path / "test.mmc"))
    assert len(tv) == 400 and np.all(np.diff(tr.astype(np.int64) * n + tc) > 0)
    W = P.read_mm_array(str(tmp_path / "W.mma"))
    H = P.read_mm_array(str(tmp_path / "H.mma"))
    assert W.shape == (300, 4) and H.shape == (4, 200)
    assert np.abs(W).max() <= 0.5 and np.abs(H).max() <= 0.5
    bad = subprocess.run([sys.executable, "-m", "dsgdpp_b200.synth", "--out-dir", str(tmp_path),
                          "--size1", "3", "--size2", "3", "--nnz", "10"], cwd=ROOT,
                         capture_output=True, text=True, timeout=300)
    assert bad.returncode != 0 and "nnz must be less than matrix size" in bad.stderr
