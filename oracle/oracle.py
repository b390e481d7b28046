"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  Only tests/,
the smoke check and bench.py's CPU-baseline leg import this module.
PARITY UNPINNED: see dsgdpp_oracle.cc for the pinned assumptions.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

_P = C.c_void_p
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)

_SIGS = {
    "orc_random_create": (_P, [C.c_uint32]),
    "orc_random_destroy": (None, [_P]),
    "orc_random_next": (C.c_uint32, [_P]),
    "orc_random_next_int": (C.c_uint32, [_P, C.c_uint32]),
    "orc_random_shuffle_u32": (None, [_P, _u32p, C.c_uint64]),
    "orc_random_sample": (None, [_P, C.c_uint32, C.c_uint32, _u32p]),
    "orc_block_offsets": (None, [C.c_uint64, C.c_uint32, _u64p]),
    "orc_compute_dsgd_schedule": (None, [_P, C.c_uint32, C.c_uint32, C.c_int, _u32p]),
    "orc_dsgdpp_schedule": (None, [_P, C.c_uint32, C.c_int, _u32p, _u32p]),
    "orc_create": (_P, [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _u32p,
                        _u32p, _f64p, C.c_uint64, _u32p, _u32p, _f64p, C.c_int]),
    "orc_destroy": (None, [_P]),
    "orc_configure": (C.c_int, [_P, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int,
                                C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int]),
    "orc_set_factors": (None, [_P, _f64p, _f64p]),
    "orc_get_factors": (None, [_P, _f64p, _f64p]),
    "orc_seed": (None, [_P, C.c_uint32]),
    "orc_nnz12": (None, [_P, _u64p, _u64p, _u64p]),
    "orc_block_nnz": (None, [_P, C.c_int, _u64p]),
    "orc_block_records": (C.c_uint64, [_P, C.c_int, C.c_uint32, C.c_uint32, _u32p, _u32p,
                                       _f64p]),
    "orc_epoch_explicit": (C.c_double, [_P, C.c_double, _u32p, _u32p, C.c_int]),
    "orc_epoch": (C.c_double, [_P, C.c_double, C.c_int]),
    "orc_positions": (C.c_uint64, [_P, _u32p, _u32p, _u32p]),
    "orc_nzsl": (C.c_double, [_P, C.c_int]),
    "orc_l2w": (C.c_double, [_P]),
    "orc_l2h": (C.c_double, [_P]),
    "orc_nzl2w": (C.c_double, [_P]),
    "orc_nzl2h": (C.c_double, [_P]),
    "orc_loss": (C.c_double, [_P]),
    "orc_run": (C.c_int, [_P, C.c_uint32, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                          _f64p]),
    "orc_bold_driver": (C.c_double, [C.c_double, _f64p, C.c_double, C.c_double, C.c_double]),
    "orc_rm_factor": (None, [C.c_int, C.c_double, C.c_double, _u32p, C.c_uint64, C.c_uint64,
                             C.c_uint32, C.c_uint32, _f64p]),
    "orc_rm_data": (C.c_uint64, [C.c_int, C.c_double, C.c_double, _u32p, _u64p, C.c_uint64,
                                 C.c_uint64, C.c_uint64, C.c_uint64, _f64p, _f64p, C.c_uint32,
                                 _u32p, _u32p, _f64p]),
}


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

UPDATE = {"Nzsl": 0, "Nzsl_L2": 1, "Nzsl_Nzl2": 2}
REGULARIZE = {"None": 0, "L2": 1}
LOSS = {"Nzsl": 0, "Nzsl_L2": 1, "Nzsl_Nzl2": 2}
SGD_ORDER = {"SEQ": 0, "WR": 1, "WOR": 2}
STRATUM_ORDER = {"SEQ": 0, "RSEQ": 1, "WR": 2, "WOR": 3, "COWOR": 4}


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


class Random32:
    def __init__(self, seed):
        self._h = lib.orc_random_create(seed & 0xFFFFFFFF)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.orc_random_destroy(self._h)

    def next(self):
        return lib.orc_random_next(self._h)

    def next_int(self, n):
        return lib.orc_random_next_int(self._h, n)

    def shuffle(self, a):
        a = np.ascontiguousarray(a, np.uint32).copy()
        lib.orc_random_shuffle_u32(self._h, _p(a, C.c_uint32), len(a))
        return a

    def sample(self, k, n):
        out = np.empty(k, np.uint32)
        lib.orc_random_sample(self._h, k, n, _p(out, C.c_uint32))
        return out


def block_offsets(size, blocks):
    out = np.empty(blocks, np.uint64)
    lib.orc_block_offsets(size, blocks, _p(out, C.c_uint64))
    return out


def dsgd_schedule(rng, w, t, order):
    out = np.empty((w * t, w * t), np.uint32)
    lib.orc_compute_dsgd_schedule(rng._h, w, t, STRATUM_ORDER[order], _p(out, C.c_uint32))
    return out


def dsgdpp_schedule(rng, d, order):
    s = np.empty((2 * d, d), np.uint32)
    t = np.empty(d, np.uint32)
    lib.orc_dsgdpp_schedule(rng._h, d, STRATUM_ORDER[order], _p(s, C.c_uint32), _p(t, C.c_uint32))
    return s, t


def bold_driver(eps, prev, cur, dec=0.5, inc=1.05):
    if prev is None:
        return lib.orc_bold_driver(eps, None, cur, dec, inc)
    pv = C.c_double(prev)
    return lib.orc_bold_driver(eps, C.byref(pv), cur, dec, inc)


METHOD = {"dsgdpp": 0, "dsgd": 1}


class Problem:
    """The CPU restatement of one DSGD++ job (d x 2d blocking), or of one DSGD
    job (d x d blocking, d sub-epochs; method="dsgd")."""

    def __init__(self, m, n, r, d, rows, cols, vals, trows=None, tcols=None, tvals=None,
                 method="dsgdpp"):
        self.m, self.n, self.r, self.d = m, n, r, d
        self.nb2 = d if method == "dsgd" else 2 * d
        rows = np.ascontiguousarray(rows, np.uint32)
        cols = np.ascontiguousarray(cols, np.uint32)
        vals = np.ascontiguousarray(vals, np.float64)
        if trows is None:
            trows = np.zeros(0, np.uint32)
            tcols = np.zeros(0, np.uint32)
            tvals = np.zeros(0, np.float64)
        trows = np.ascontiguousarray(trows, np.uint32)
        tcols = np.ascontiguousarray(tcols, np.uint32)
        tvals = np.ascontiguousarray(tvals, np.float64)
        self._h = lib.orc_create(m, n, r, d, len(vals), _p(rows, C.c_uint32),
                                 _p(cols, C.c_uint32), _p(vals, C.c_double), len(tvals),
                                 _p(trows, C.c_uint32), _p(tcols, C.c_uint32),
                                 _p(tvals, C.c_double), METHOD[method])
        if not self._h:
            raise ValueError("orc_create failed")

    def __del__(self):
        if getattr(self, "_h", None):
            lib.orc_destroy(self._h)

    def configure(self, update="Nzsl_L2", update_lambda=1.0, regularize="None",
                  regularize_lambda=0.0, loss="Nzsl_L2", loss_lambda=1.0, truncate=None,
                  sgd_order="WOR", stratum_order="COWOR"):
        t = truncate is not None
        rc = lib.orc_configure(self._h, UPDATE[update], update_lambda, REGULARIZE[regularize],
                               regularize_lambda, LOSS[loss], loss_lambda, int(t),
                               truncate[0] if t else float("nan"),
                               truncate[1] if t else float("nan"), SGD_ORDER[sgd_order],
                               STRATUM_ORDER[stratum_order])
        if rc != 0:
            raise ValueError("orc_configure failed")
        self.sgd_order = sgd_order
        return self

    def set_factors(self, W, H):
        w = np.ascontiguousarray(W, np.float64)
        h = np.ascontiguousarray(H, np.float64)
        lib.orc_set_factors(self._h, _p(w, C.c_double), _p(h, C.c_double))

    def get_factors(self):
        w = np.empty((self.m, self.r), np.float64)
        h = np.empty((self.n, self.r), np.float64)
        lib.orc_get_factors(self._h, _p(w, C.c_double), _p(h, C.c_double))
        return w, h

    def seed(self, s):
        lib.orc_seed(self._h, s & 0xFFFFFFFF)

    def nnz12(self):
        a = np.empty(self.m, np.uint64)
        b = np.empty(self.n, np.uint64)
        mx = C.c_uint64()
        lib.orc_nnz12(self._h, _p(a, C.c_uint64), _p(b, C.c_uint64), C.byref(mx))
        return a, b, mx.value

    def block_nnz(self, which=0):
        out = np.empty(self.nb2 * self.d, np.uint64)
        lib.orc_block_nnz(self._h, which, _p(out, C.c_uint64))
        return out.reshape(self.d, self.nb2)

    def block_records(self, b1, b2, which=0):
        n = lib.orc_block_records(self._h, which, b1, b2, None, None, None)
        i = np.empty(n, np.uint32)
        j = np.empty(n, np.uint32)
        x = np.empty(n, np.float64)
        lib.orc_block_records(self._h, which, b1, b2, _p(i, C.c_uint32), _p(j, C.c_uint32),
                              _p(x, C.c_double))
        return i, j, x

    def epoch_explicit(self, eps, schedule, seeds, threads=1):
        s = np.ascontiguousarray(schedule, np.uint32)
        t = np.ascontiguousarray(seeds, np.uint32)
        return lib.orc_epoch_explicit(self._h, eps, _p(s, C.c_uint32), _p(t, C.c_uint32), threads)

    def epoch(self, eps, threads=1):
        return lib.orc_epoch(self._h, eps, threads)

    def positions(self, schedule, seeds):
        s = np.ascontiguousarray(schedule, np.uint32)
        t = np.ascontiguousarray(seeds, np.uint32)
        n = lib.orc_positions(self._h, _p(s, C.c_uint32), _p(t, C.c_uint32), None)
        out = np.empty(n, np.uint32)
        lib.orc_positions(self._h, _p(s, C.c_uint32), _p(t, C.c_uint32), _p(out, C.c_uint32))
        return out

    def nzsl(self, which=0):
        return lib.orc_nzsl(self._h, which)

    def l2(self):
        return lib.orc_l2w(self._h), lib.orc_l2h(self._h)

    def nzl2(self):
        return lib.orc_nzl2w(self._h), lib.orc_nzl2h(self._h)

    def loss(self):
        return lib.orc_loss(self._h)

    def run(self, epochs, decay="BoldDriver", eps0=0.001, dec=0.5, inc=1.05, threads=1):
        tr = np.empty((epochs + 1, 3), np.float64)
        lib.orc_run(self._h, epochs, 1 if decay == "BoldDriver" else 0, eps0, dec, inc, threads,
                    _p(tr, C.c_double))
        return tr


# ---- .rm descriptors (rm_oracle.cc) ------------------------------------------------
def read_rm(path):
    """The property_tree XML of a .rm descriptor (randomMatrixDescriptor_impl.cc:21-91),
    read with Python's own XML parser: a dict of sizes, specs, seeds and counts."""
    import re
    import xml.etree.ElementTree as ET
    text = open(path).read()
    text = re.sub(r"<\?xml[^>]*\?>", "", text)
    root = ET.fromstring("<root>" + text + "</root>")
    num = lambda tag: int(root.find(tag).text.strip())
    d = dict(size1=num("size1"), size2=num("size2"), blocks1=num("blocks1"),
             blocks2=num("blocks2"), nnz=num("nnz"), nnzTest=num("nnzTest"), rank=num("rank"),
             values=(root.find("values").text or "").strip(),
             noise=(root.find("noise").text or "").strip())
    d["Worig"] = [int(e.text) for e in root.find("Worig")]
    d["Horig"] = [int(e.text) for e in root.find("Horig")]
    if d["nnz"] and d["nnzTest"]:
        for part in ("V", "Vtest"):
            d[part + ".seeds"] = [int(e.text) for e in root.find(part).find("seeds")]
            d[part + ".nnzs"] = [int(e.text) for e in root.find(part).find("nnzs")]
    return d


def parse_dist(spec):
    """(kind, a, b): Normal -> 0, Uniform -> 1, empty -> -1 (tools/parse.h:75-110)."""
    spec = (spec or "").strip()
    if not spec:
        return -1, 0.0, 0.0
    name, args = spec.split("(", 1)
    a, b = [float(x) for x in args.rstrip(")").split(",")]
    return {"Normal": 0, "Uniform": 1}[name.strip()], a, b


def rm_factors(d):
    """Worig (size1 x rank) and Horig (size2 x rank), row-major."""
    kind, a, b = parse_dist(d["values"])
    out = []
    for rows, key, tag, blocks in ((d["size1"], "Worig", 1, d["blocks1"]),
                                   (d["size2"], "Horig", 2, d["blocks2"])):
        seeds = np.ascontiguousarray(d[key], np.uint32)
        X = np.empty((rows, d["rank"]), np.float64)
        lib.orc_rm_factor(kind, a, b, _p(seeds, C.c_uint32), blocks, rows, d["rank"], tag,
                          _p(X, C.c_double))
        out.append(X)
    return out[0], out[1]


def rm_data(d, which, W, H):
    """The data (which=0, with noise) or test (which=1) matrix: rows, cols, vals."""
    part = "V" if which == 0 else "Vtest"
    seeds = np.ascontiguousarray(d[part + ".seeds"], np.uint32)
    counts = np.ascontiguousarray(d[part + ".nnzs"], np.uint64)
    total = int(counts.sum())
    kind, a, b = parse_dist(d["noise"]) if which == 0 else (-1, 0.0, 0.0)
    rows = np.empty(total, np.uint32)
    cols = np.empty(total, np.uint32)
    vals = np.empty(total, np.float64)
    W = np.ascontiguousarray(W, np.float64)
    H = np.ascontiguousarray(H, np.float64)
    n = lib.orc_rm_data(kind, a, b, _p(seeds, C.c_uint32), _p(counts, C.c_uint64), d["blocks1"],
                        d["blocks2"], d["size1"], d["size2"], _p(W, C.c_double),
                        _p(H, C.c_double), d["rank"], _p(rows, C.c_uint32), _p(cols, C.c_uint32),
                        _p(vals, C.c_double))
    assert n == total
    return rows, cols, vals
