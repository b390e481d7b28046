"""CPU tests of the .rm random-matrix descriptors (RandomMatrixDescriptor,
mf/matrix/io/randomMatrixDescriptor.h and _impl.cc) and of the oracle's
restatement of the generator."""
import os

import numpy as np
import pytest

import dsgdpp_b200 as P
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
SMALL = os.path.join(HERE, "golden", "small.rm")


def test_fixture_loads_with_the_fields_python_reads():
    rm = P.RandomMatrix(SMALL)
    info = rm.info()
    d = O.read_rm(SMALL)
    assert (info["size1"], info["size2"], info["rank"]) == (d["size1"], d["size2"], d["rank"])
    assert (info["blocks1"], info["blocks2"]) == (d["blocks1"], d["blocks2"])
    assert info["data_nnz"] == sum(d["V.nnzs"]) == 46
    assert info["test_nnz"] == sum(d["Vtest.nnzs"]) == 8


def test_save_round_trip(tmp_path):
    rm = P.RandomMatrix(SMALL)
    out = str(tmp_path / "again.rm")
    rm.save(out)
    assert O.read_rm(out) == O.read_rm(SMALL)
    out2 = str(tmp_path / "again2.rm")
    P.RandomMatrix(out).save(out2)
    assert open(out).read() == open(out2).read()


def test_create_draws_seeds_in_the_reference_order(tmp_path):
    # RandomMatrixDescriptor::create (randomMatrixDescriptor.h:36-68): one
    # generator seeded 123; per row chunk the Worig seed, then per column chunk
    # (the Horig seed in the first row only) the V seed and the Vtest seed.
    c1, c2 = 3, 4
    rm = P.RandomMatrix.create(30, 40, c1, c2, 500, 60, 5, "Normal(0,1)", "Normal(0,0.1)")
    path = str(tmp_path / "c.rm")
    rm.save(path)
    d = O.read_rm(path)
    raw = iter(np.random.RandomState(123)._bit_generator.random_raw(64).astype(np.uint64))
    w, h, v, vt = [], [], [], []
    for b1 in range(c1):
        w.append(int(next(raw)) & 0xFFFFFFFF)
        for b2 in range(c2):
            if b1 == 0:
                h.append(int(next(raw)) & 0xFFFFFFFF)
            v.append(int(next(raw)) & 0xFFFFFFFF)
            vt.append(int(next(raw)) & 0xFFFFFFFF)
    assert d["Worig"] == w and d["Horig"] == h
    assert d["V.seeds"] == v and d["Vtest.seeds"] == vt
    assert sum(d["V.nnzs"]) == 500 and sum(d["Vtest.nnzs"]) == 60
    assert max(d["V.nnzs"]) <= 10 * 10
    # deterministic
    rm.save(str(tmp_path / "d.rm"))
    assert P.RandomMatrix.create(30, 40, c1, c2, 500, 60, 5, "Normal(0,1)",
                                 "Normal(0,0.1)").info() == rm.info()


def test_create_without_test_count_has_no_data_part(tmp_path):
    # nonzeros per chunk are only drawn when both counts are given
    # (randomMatrixDescriptor.h:71-74, _impl.cc:99)
    rm = P.RandomMatrix.create(30, 40, 3, 4, 500, 0, 5, "Uniform(-1,1)")
    path = str(tmp_path / "f.rm")
    rm.save(path)
    d = O.read_rm(path)
    assert "V.seeds" not in d and len(d["Worig"]) == 3
    assert rm.info()["data_nnz"] == 0


@pytest.mark.parametrize("body,msg", [
    ("<size1>4</size1>", "lacks"),
    (open(SMALL).read().replace("<nnz>20</nnz>", "<nnz>21</nnz>"), "nnz must be less"),
    (open(SMALL).read().replace("Uniform(-0.5,0.5)", "Gamma(1,2)"), "invalid distribution"),
    (open(SMALL).read().replace("<seed>13</seed>", ""), "Worig seed"),
])
def test_bad_descriptors_are_rejected(tmp_path, body, msg):
    path = str(tmp_path / "bad.rm")
    open(path, "w").write(body)
    with pytest.raises(P.DsgdppError) as e:
        P.RandomMatrix(path)
    assert msg in str(e.value)


def test_create_rejects_sizes_that_do_not_divide():
    with pytest.raises(P.DsgdppError):
        P.RandomMatrix.create(31, 40, 3, 4, 500, 60, 5, "Normal(0,1)")


def test_oracle_generator_properties():
    d = O.read_rm(SMALL)
    W, H = O.rm_factors(d)
    assert W.shape == (12, 2) and H.shape == (10, 2)
    assert np.all(np.abs(W) <= 0.5) and np.all(np.abs(H) <= 0.5)
    for which, part in ((0, "V"), (1, "Vtest")):
        r, c, v = O.rm_data(d, which, W, H)
        assert len(r) == sum(d[part + ".nnzs"])
        # chunk by chunk, each chunk's cells distinct and inside the chunk
        k = 0
        o1, o2 = [0, 4, 8, 12], [0, 5, 10]
        for b1 in range(3):
            for b2 in range(2):
                n = d[part + ".nnzs"][b1 * 2 + b2]
                rr, cc = r[k:k + n], c[k:k + n]
                assert np.all((rr >= o1[b1]) & (rr < o1[b1 + 1]))
                assert np.all((cc >= o2[b2]) & (cc < o2[b2 + 1]))
                assert len(set(zip(rr.tolist(), cc.tolist()))) == n
                k += n
        exact = np.array([sum(W[i, z] * H[j, z] for z in range(2)) for i, j in zip(r, c)])
        if which == 1:  # the test matrix has no noise
            np.testing.assert_array_equal(v, exact)
        else:
            noise = v - exact
            assert 0.01 < noise.std() < 0.3
    # the full chunk (20 of 20 cells) is every cell once
    r, c, _ = O.rm_data(d, 0, W, H)
    full = set(zip(r[26:46].tolist(), c[26:46].tolist()))
    assert full == {(i, j) for i in range(8, 12) for j in range(0, 5)}
