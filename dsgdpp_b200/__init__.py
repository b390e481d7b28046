"""Python binding of the B200 DSGD++ library (C ABI in include/dsgdpp.h).

The compute path is the CUDA library ``dsgdpp_b200/lib/libdsgdpp_b200.so``;
this module only marshals arguments through ctypes.  There is no CPU
fallback: if the library is missing, importing the binding raises, and if no
GPU is present, :class:`Context` creation fails with ``DsgdppError``.

The classes mirror the reference's C++ entry points:

* :class:`Context` -- a ``DsgdPpJob`` plus ``DsgdPpRunner`` bound to one GPU
  (mf/sgd/dsgdpp.h:38-134): ``epoch`` is ``DsgdPpRunner::epoch``, ``run`` is
  ``detail::defaultRunner`` (mf/sgd/sgd_impl.h:34-145), ``loss``/``nzsl``/
  ``l2``/``nzl2`` are the losses of mf/loss.
* :class:`Random32`, :func:`draw_schedule`, :func:`dsgd_schedule`,
  :func:`point_orders`, :func:`block_offsets` -- host-side random draws and
  blocking (mf/sgd/dsgdpp_impl.h:282-349, mf/sgd/dsgd_impl.h:246-325,
  mf/sgd/sgd_impl.h:197-351, mf/matrix/distributed_matrix_impl.cc:24-40).
* :class:`RandomMatrix` -- a ``.rm`` random-matrix descriptor
  (mf/matrix/io/randomMatrixDescriptor.h); ``Context.set_matrix_rm`` and
  ``Context.set_factors_rm`` generate its matrices on the device.
* :class:`Batch` -- many small independent factorizations in one launch
  sequence; :class:`Mlp` and ``Context.run_controlled`` -- the learned
  step-size controller.
* :func:`read_sparse`, :func:`read_mm_array`, :func:`write_mm_coord`,
  :func:`write_mm_array`, :func:`write_blocked` -- the MatrixMarket and
  blocked ``.xml`` files of mf/matrix/io.

Example::

    import dsgdpp_b200 as P
    cfg = P.Config(m=m, n=n, rank=32, d=64, precision="fp32")
    with P.Context(cfg) as ctx:
        ctx.set_matrix(P.TRAIN, rows, cols, vals)      # 0-based coordinates
        ctx.set_matrix(P.TEST, trows, tcols, tvals)
        ctx.set_factors(W, H)                          # m x r and n x r, FP64
        ctx.seed(1)
        trace = ctx.run(50, "BoldDriver", 0.001)       # one dict per epoch
        W, H = ctx.get_factors()
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdsgdpp_b200.so")

# constants of include/dsgdpp.h
OK = 0
E_INVALID, E_CUDA, E_IO, E_UNSUPPORTED, E_STATE, E_NOMEM = -1, -2, -3, -4, -5, -6
UPDATE = {"Nzsl": 0, "Nzsl_L2": 1, "Nzsl_Nzl2": 2}
REGULARIZE = {"None": 0, "L2": 1}
LOSS = {"Nzsl": 0, "Nzsl_L2": 1, "Nzsl_Nzl2": 2}
SGD_ORDER = {"SEQ": 0, "WR": 1, "WOR": 2}
STRATUM_ORDER = {"SEQ": 0, "RSEQ": 1, "WR": 2, "WOR": 3, "COWOR": 4}
PRECISION = {"fp64": 0, "fp32": 1, "bf16": 2}
EXEC = {"replay": 0, "hogwild": 1}
LAUNCH = {"stream": 0, "graph": 1, "persistent": 2}
WRITE_MODE = {"auto": 0, "store": 1, "atomic": 2}
LAYOUT = {"shuffled": 0, "col_runs": 1, "row_runs": 2, "runs": 3}
METHOD = {"dsgdpp": 0, "dsgd": 1}
TRAIN, TEST = 0, 1
DECAY = {"Const": 0, "BoldDriver": 1}


class DsgdppError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


class _Config(C.Structure):
    _fields_ = [
        ("m", C.c_uint64), ("n", C.c_uint64), ("rank", C.c_uint32), ("d", C.c_uint32),
        ("precision", C.c_int32), ("exec", C.c_int32), ("launch", C.c_int32),
        ("update", C.c_int32), ("update_lambda", C.c_double),
        ("regularize", C.c_int32), ("regularize_lambda", C.c_double),
        ("loss", C.c_int32), ("loss_lambda", C.c_double),
        ("truncate", C.c_int32), ("truncate_min", C.c_double), ("truncate_max", C.c_double),
        ("sgd_order", C.c_int32), ("stratum_order", C.c_int32), ("device", C.c_int32),
        ("lanes_per_nnz", C.c_uint32), ("vecs_per_lane", C.c_uint32),
        ("ctas_per_sm", C.c_uint32), ("layout_seed", C.c_uint64), ("write_mode", C.c_int32),
        ("layout", C.c_int32), ("method", C.c_int32),
    ]


class _TraceRow(C.Structure):
    _fields_ = [
        ("epoch", C.c_uint64), ("loss", C.c_double), ("test_loss", C.c_double),
        ("eps", C.c_double), ("time_eps", C.c_double), ("time_epoch", C.c_double),
        ("time_loss", C.c_double), ("time_test_loss", C.c_double),
    ]


_P = C.c_void_p
_u32p = C.POINTER(C.c_uint32)


class _Problem(C.Structure):
    _fields_ = [
        ("m", C.c_uint64), ("n", C.c_uint64), ("rank", C.c_uint32), ("d", C.c_uint32),
        ("nnz", C.c_uint64), ("rows", _u32p), ("cols", _u32p), ("vals", C.POINTER(C.c_double)),
        ("nnz_test", C.c_uint64), ("trows", _u32p), ("tcols", _u32p),
        ("tvals", C.POINTER(C.c_double)), ("W", C.POINTER(C.c_double)),
        ("H", C.POINTER(C.c_double)), ("seed", C.c_uint32), ("eps0", C.c_double),
    ]


_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)
_f32p = C.POINTER(C.c_float)

# every symbol of include/dsgdpp.h with its ctypes signature
SIGNATURES = {
    "dsgdpp_config_init": (None, [C.POINTER(_Config)]),
    "dsgdpp_create": (C.c_int, [C.POINTER(_Config), C.POINTER(_P)]),
    "dsgdpp_create_error": (C.c_char_p, []),
    "dsgdpp_destroy": (None, [_P]),
    "dsgdpp_last_error": (C.c_char_p, [_P]),
    "dsgdpp_status_string": (C.c_char_p, [C.c_int]),
    "dsgdpp_abi_version": (C.c_int, []),
    "dsgdpp_set_matrix": (C.c_int, [_P, C.c_int, C.c_uint64, _u32p, _u32p, _f64p]),
    "dsgdpp_set_factors": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_get_factors": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_block_nnz": (C.c_int, [_P, C.c_int, _u64p]),
    "dsgdpp_nnz12": (C.c_int, [_P, _u64p, _u64p, _u64p]),
    "dsgdpp_seed": (C.c_int, [_P, C.c_uint32]),
    "dsgdpp_epoch": (C.c_int, [_P, C.c_double]),
    "dsgdpp_epoch_explicit": (C.c_int, [_P, C.c_double, _u32p, _u32p]),
    "dsgdpp_last_epoch_ms": (C.c_int, [_P, _f64p]),
    "dsgdpp_set_kernel_timing": (C.c_int, [_P, C.c_int]),
    "dsgdpp_kernel_timing": (C.c_int, [_P, _f64p, _u64p]),
    "dsgdpp_launch_shape": (C.c_int, [_P, _u32p, _u32p, _u32p]),
    "dsgdpp_loss": (C.c_int, [_P, _f64p]),
    "dsgdpp_nzsl": (C.c_int, [_P, C.c_int, _f64p]),
    "dsgdpp_l2": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_nzl2": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_nzsl_fp32_noalloc": (C.c_int, [_P, _P, _P, C.c_uint64, _P, _P, C.c_uint32,
                                           C.c_uint32, C.c_uint32, _P, _P]),
    "dsgdpp_run": (C.c_int, [_P, C.c_uint32, C.c_int, C.c_double, C.c_double, C.c_double,
                             C.POINTER(_TraceRow)]),
    "dsgdpp_sync": (C.c_int, [_P]),
    "dsgdpp_save_factors": (C.c_int, [_P]),
    "dsgdpp_restore_factors": (C.c_int, [_P]),
    "dsgdpp_update_norms": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(_P)]),
    "dsgdpp_mlp_destroy": (None, [_P]),
    "dsgdpp_mlp_param_count": (C.c_int, []),
    "dsgdpp_mlp_get_params": (C.c_int, [_P, _f32p]),
    "dsgdpp_mlp_set_params": (C.c_int, [_P, _f32p]),
    "dsgdpp_mlp_forward": (C.c_int, [_P, _f32p, C.c_int, _f32p]),
    "dsgdpp_mlp_gradient": (C.c_int, [_P, _f32p, _f32p, C.c_int, _f32p, _f32p]),
    "dsgdpp_mlp_train_step": (C.c_int, [_P, _f32p, _f32p, C.c_int, C.c_float, _f32p]),
    "dsgdpp_run_controlled": (C.c_int, [_P, _P, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                        C.c_double, C.POINTER(_TraceRow), _u32p, _u32p]),
    "dsgdpp_controller_features": (None, [_f64p, _f64p, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_double, _f32p]),
    "dsgdpp_autotune": (C.c_int, [C.POINTER(_Config), C.c_uint64, _u32p, _u32p, _f64p, _f64p,
                                  _f64p, _u32p, C.c_uint32, C.c_uint32, C.c_double,
                                  C.POINTER(_Config), _f64p]),
    "dsgdpp_batch_create": (C.c_int, [C.POINTER(_Config), C.c_uint32, C.POINTER(_Problem),
                                      C.POINTER(_P)]),
    "dsgdpp_batch_destroy": (None, [_P]),
    "dsgdpp_batch_last_error": (C.c_char_p, [_P]),
    "dsgdpp_batch_run": (C.c_int, [_P, C.c_uint32, C.c_double, C.c_double, _f64p, _f64p,
                                   _f64p]),
    "dsgdpp_batch_autotune": (C.c_int, [C.POINTER(_Config), C.c_uint32, C.POINTER(_Problem),
                                        C.c_uint32, C.c_uint32, _u32p, _u32p, _f64p]),
    "dsgdpp_batch_problem_d": (C.c_int, [_P, C.c_uint32, _u32p]),
    "dsgdpp_batch_get_factors": (C.c_int, [_P, C.c_uint32, _f64p, _f64p]),
    "dsgdpp_rng_create": (_P, [C.c_uint32]),
    "dsgdpp_rng_destroy": (None, [_P]),
    "dsgdpp_rng_next": (C.c_uint32, [_P]),
    "dsgdpp_rng_next_int": (C.c_uint32, [_P, C.c_uint32]),
    "dsgdpp_draw_schedule": (None, [_P, C.c_uint32, C.c_int, _u32p, _u32p]),
    "dsgdpp_dsgd_schedule": (None, [_P, C.c_uint32, C.c_uint32, C.c_int, _u32p]),
    "dsgdpp_point_orders": (C.c_uint64, [C.c_uint32, C.c_int, _u64p, _u32p, _u32p, _u32p]),
    "dsgdpp_block_offsets": (None, [C.c_uint64, C.c_uint32, _u64p]),
    "dsgdpp_philox4x32_10": (None, [_u32p, _u32p, _u32p]),
    "dsgdpp_io_error": (C.c_char_p, []),
    "dsgdpp_free": (None, [_P]),
    "dsgdpp_read_sparse": (C.c_int, [C.c_char_p, _u64p, _u64p, _u64p, C.POINTER(_u32p),
                                     C.POINTER(_u32p), C.POINTER(_f64p)]),
    "dsgdpp_write_mm_coord": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint64, C.c_uint64, _u32p,
                                        _u32p, _f64p]),
    "dsgdpp_read_mm_array": (C.c_int, [C.c_char_p, _u64p, _u64p, C.POINTER(_f64p)]),
    "dsgdpp_write_mm_array": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint64, _f64p]),
    "dsgdpp_write_blocked": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint64,
                                       C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64, _u32p,
                                       _u32p, _f64p]),
    "dsgdpp_rm_error": (C.c_char_p, []),
    "dsgdpp_rm_load": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "dsgdpp_rm_create": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64,
                                   C.c_uint64, C.c_uint32, C.c_char_p, C.c_char_p,
                                   C.POINTER(_P)]),
    "dsgdpp_rm_save": (C.c_int, [_P, C.c_char_p]),
    "dsgdpp_rm_destroy": (None, [_P]),
    "dsgdpp_rm_info": (C.c_int, [_P, _u64p]),
    "dsgdpp_rm_generate": (C.c_int, [_P, C.c_int, C.c_int, _u32p, _u32p, _f64p]),
    "dsgdpp_rm_generate_factors": (C.c_int, [_P, C.c_int, _f64p, _f64p]),
    "dsgdpp_set_matrix_rm": (C.c_int, [_P, C.c_int, _P]),
    "dsgdpp_set_blocks": (C.c_int, [_P, C.c_int, _u64p, _u32p, _u32p, _f64p]),
    "dsgdpp_epoch_part": (C.c_int, [_P, C.c_double, _u32p, _u32p, C.c_uint32, C.c_uint32]),
    "dsgdpp_h_block_bytes": (C.c_int, [_P, C.c_uint32, _u64p]),
    "dsgdpp_h_block_copy": (C.c_int, [_P, C.c_uint32, _P, C.c_int]),
    "dsgdpp_set_counts": (C.c_int, [_P, _u64p, _u64p]),
    "dsgdpp_set_wait_limit": (C.c_int, [_P, C.c_double]),
    "dsgdpp_set_tasks": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
    "dsgdpp_shard_unique_id": (C.c_int, [_P]),
    "dsgdpp_shard_create_nccl": (C.c_int, [_P, C.c_int, C.c_int, _P, C.POINTER(_P)]),
    "dsgdpp_shard_create_local": (C.c_int, [C.POINTER(_P), C.c_int, C.POINTER(_P)]),
    "dsgdpp_shard_destroy": (None, [_P]),
    "dsgdpp_shard_last_error": (C.c_char_p, [_P]),
    "dsgdpp_shard_set_wait_limit": (C.c_int, [_P, C.c_double]),
    "dsgdpp_shard_epoch": (C.c_int, [_P, C.c_double, _u32p, _u32p]),
    "dsgdpp_shard_share": (C.c_int, [_P]),
    "dsgdpp_shard_gather_w": (C.c_int, [_P]),
    "dsgdpp_shard_losses": (C.c_int, [_P, _f64p, _f64p]),
    "dsgdpp_shard_moved": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "dsgdpp_shard_set_timeline": (C.c_int, [_P, C.c_int]),
    "dsgdpp_shard_timeline": (C.c_int, [_P, C.c_uint32, _f64p, _f64p]),
    "dsgdpp_shard_plan": (C.c_uint64, [C.c_uint32, C.c_uint32, C.c_int, _u32p,
                                       C.POINTER(C.c_int32), _u32p]),
    "dsgdpp_set_factors_rm": (C.c_int, [_P, _P]),
}


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
            f"g.build()'` (make -C dsgdpp_b200/csrc)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class Config:
    """dsgdpp_config with the reference defaults (tools/mfdsgdpp.cc:429-441)."""
    m: int
    n: int
    rank: int
    d: int
    precision: str = "fp32"
    exec: str = "hogwild"
    launch: str = "graph"
    update: str = "Nzsl_L2"
    update_lambda: float = 1.0
    regularize: str = "None"
    regularize_lambda: float = 0.0
    loss: str = "Nzsl_L2"
    loss_lambda: float = 1.0
    truncate: Optional[tuple] = None
    sgd_order: str = "WOR"
    stratum_order: str = "COWOR"
    device: int = 0
    lanes_per_nnz: int = 0
    vecs_per_lane: int = 0
    ctas_per_sm: int = 0
    layout_seed: int = 0x5EED5EED
    write_mode: str = "auto"
    layout: str = "runs"
    method: str = "dsgdpp"

    def to_c(self) -> _Config:
        c = _Config()
        lib.dsgdpp_config_init(C.byref(c))
        c.m, c.n, c.rank, c.d = self.m, self.n, self.rank, self.d
        c.precision = PRECISION[self.precision]
        c.exec = EXEC[self.exec]
        c.launch = LAUNCH[self.launch]
        c.update, c.update_lambda = UPDATE[self.update], self.update_lambda
        c.regularize, c.regularize_lambda = REGULARIZE[self.regularize], self.regularize_lambda
        c.loss, c.loss_lambda = LOSS[self.loss], self.loss_lambda
        if self.truncate is not None:
            c.truncate, c.truncate_min, c.truncate_max = 1, self.truncate[0], self.truncate[1]
        c.sgd_order = SGD_ORDER[self.sgd_order]
        c.stratum_order = STRATUM_ORDER[self.stratum_order]
        c.device = self.device
        c.lanes_per_nnz, c.vecs_per_lane = self.lanes_per_nnz, self.vecs_per_lane
        c.ctas_per_sm, c.layout_seed = self.ctas_per_sm, self.layout_seed
        c.write_mode = WRITE_MODE[self.write_mode]
        c.layout = LAYOUT[self.layout]
        c.method = METHOD[self.method]
        return c


class Context:
    """One DSGD++ job on one GPU (DsgdPpJob + DsgdPpRunner)."""

    def __init__(self, config: Config):
        self.config = config
        self._cfg = config.to_c()
        h = _P()
        rc = lib.dsgdpp_create(C.byref(self._cfg), C.byref(h))
        if rc != OK:
            raise DsgdppError(rc, "dsgdpp_create: " + lib.dsgdpp_create_error().decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise DsgdppError(rc, f"{what}: {lib.dsgdpp_last_error(self._h).decode()}")

    # data -------------------------------------------------------------------
    def set_matrix(self, which: int, rows, cols, vals):
        r, c, v = _u32(rows), _u32(cols), _f64(vals)
        if not (len(r) == len(c) == len(v)):
            raise ValueError("rows, cols and vals differ in length")
        self._check(lib.dsgdpp_set_matrix(self._h, which, len(v), _ptr(r, C.c_uint32),
                                          _ptr(c, C.c_uint32), _ptr(v, C.c_double)),
                    "set_matrix")

    def set_factors(self, W, H):
        """W: m x r row-major; H: r x n column-major, passed as its n x r transpose."""
        w, h = _f64(W), _f64(H)
        self._check(lib.dsgdpp_set_factors(self._h, _ptr(w, C.c_double), _ptr(h, C.c_double)),
                    "set_factors")

    def set_blocks(self, which: int, block_nnz, local_rows, local_cols, vals):
        """Blocks one after another (row-major block order) with block-local
        coordinates, as the reference's blocked matrix holds them."""
        bn = np.ascontiguousarray(block_nnz, np.uint64)
        r, c, v = _u32(local_rows), _u32(local_cols), _f64(vals)
        self._check(lib.dsgdpp_set_blocks(self._h, which, _ptr(bn, C.c_uint64),
                                          _ptr(r, C.c_uint32), _ptr(c, C.c_uint32),
                                          _ptr(v, C.c_double)), "set_blocks")

    def set_counts(self, nnz1, nnz2):
        """Per-row and per-column training counts (weights of Nzsl_L2)."""
        a = np.ascontiguousarray(nnz1, np.uint64)
        b = np.ascontiguousarray(nnz2, np.uint64)
        self._check(lib.dsgdpp_set_counts(self._h, _ptr(a, C.c_uint64), _ptr(b, C.c_uint64)),
                    "set_counts")

    def set_matrix_rm(self, which: int, rm: "RandomMatrix"):
        """The data (TRAIN) or test (TEST) matrix of a .rm descriptor, generated
        on the device (getDataMatrices with a .rm file)."""
        self._check(lib.dsgdpp_set_matrix_rm(self._h, which, rm._h), "set_matrix_rm")

    def set_factors_rm(self, rm: "RandomMatrix"):
        """Worig and Horig of a .rm descriptor as the factors (getFactors with .rm)."""
        self._check(lib.dsgdpp_set_factors_rm(self._h, rm._h), "set_factors_rm")

    def get_factors(self):
        w = np.empty((self.config.m, self.config.rank), np.float64)
        h = np.empty((self.config.n, self.config.rank), np.float64)
        self._check(lib.dsgdpp_get_factors(self._h, _ptr(w, C.c_double), _ptr(h, C.c_double)),
                    "get_factors")
        return w, h

    def get_factors_into(self, W: np.ndarray, H: np.ndarray):
        """Reads the factors into caller-provided C-contiguous float64 arrays."""
        for a, rows in ((W, self.config.m), (H, self.config.n)):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (rows, self.config.rank):
                raise ValueError("factor buffers must be C-contiguous float64 of the factor shape")
        self._check(lib.dsgdpp_get_factors(self._h, _ptr(W, C.c_double), _ptr(H, C.c_double)),
                    "get_factors")

    def block_nnz(self, which: int = TRAIN) -> np.ndarray:
        d = self.config.d
        nb2 = d if self.config.method == "dsgd" else 2 * d  # column blocks
        out = np.empty(d * nb2, np.uint64)
        self._check(lib.dsgdpp_block_nnz(self._h, which, _ptr(out, C.c_uint64)), "block_nnz")
        return out.reshape(d, nb2)

    def nnz12(self):
        a = np.empty(self.config.m, np.uint64)
        b = np.empty(self.config.n, np.uint64)
        mx = C.c_uint64()
        self._check(lib.dsgdpp_nnz12(self._h, _ptr(a, C.c_uint64), _ptr(b, C.c_uint64),
                                     C.byref(mx)), "nnz12")
        return a, b, mx.value

    # epochs -----------------------------------------------------------------
    def seed(self, seed: int):
        self._check(lib.dsgdpp_seed(self._h, seed & 0xFFFFFFFF), "seed")

    def epoch(self, eps: float):
        self._check(lib.dsgdpp_epoch(self._h, eps), "epoch")

    def epoch_explicit(self, eps: float, schedule, task_seeds):
        s, t = _u32(schedule), _u32(task_seeds)
        self._check(lib.dsgdpp_epoch_explicit(self._h, eps, _ptr(s, C.c_uint32),
                                              _ptr(t, C.c_uint32)), "epoch_explicit")

    def epoch_part(self, eps: float, schedule, task_seeds, s_begin: int, s_end: int):
        """Sub-epochs [s_begin, s_end) of the epoch (eps, schedule, seeds)."""
        s = _u32(schedule)
        t = _u32(task_seeds)
        self._check(lib.dsgdpp_epoch_part(self._h, eps, _ptr(s, C.c_uint32), _ptr(t, C.c_uint32),
                                          s_begin, s_end), "epoch_part")

    def set_tasks(self, first: int, count: int):
        """Run tasks first .. first+count-1 only (one rank's share of the job)."""
        self._check(lib.dsgdpp_set_tasks(self._h, first, count), "set_tasks")

    def h_block_bytes(self, b2: int) -> int:
        out = C.c_uint64()
        self._check(lib.dsgdpp_h_block_bytes(self._h, b2, C.byref(out)), "h_block_bytes")
        return out.value

    def h_block_copy(self, b2: int, device_ptr: int, to_context: bool):
        """Copies H column block b2 to (to_context False) or from a device buffer
        (an address, e.g. a torch CUDA tensor's data_ptr())."""
        self._check(lib.dsgdpp_h_block_copy(self._h, b2, C.c_void_p(device_ptr), int(to_context)),
                    "h_block_copy")

    def last_epoch_ms(self) -> float:
        v = C.c_double()
        self._check(lib.dsgdpp_last_epoch_ms(self._h, C.byref(v)), "last_epoch_ms")
        return v.value

    def set_wait_limit(self, seconds: float):
        """How long a dependency wait of the persistent epoch may last."""
        self._check(lib.dsgdpp_set_wait_limit(self._h, float(seconds)), "set_wait_limit")

    def set_kernel_timing(self, on: bool):
        self._check(lib.dsgdpp_set_kernel_timing(self._h, int(on)), "set_kernel_timing")

    def kernel_timing(self):
        ms, n = C.c_double(), C.c_uint64()
        self._check(lib.dsgdpp_kernel_timing(self._h, C.byref(ms), C.byref(n)), "kernel_timing")
        return ms.value, n.value

    def launch_shape(self):
        a, b, g = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._check(lib.dsgdpp_launch_shape(self._h, C.byref(a), C.byref(b), C.byref(g)),
                    "launch_shape")
        return a.value, b.value, g.value

    def run_controlled(self, mlp: "Mlp", epochs: int, eps0: float = 0.001, decrease: float = 0.5,
                       increase: float = 1.05, target_test_loss: float = 0.0):
        rows = (_TraceRow * (epochs + 1))()
        done, fb = C.c_uint32(), C.c_uint32()
        self._check(lib.dsgdpp_run_controlled(self._h, mlp._h, epochs, eps0, decrease, increase,
                                              target_test_loss, rows, C.byref(done), C.byref(fb)),
                    "run_controlled")
        trace = [dict(epoch=r.epoch, loss=r.loss, test_loss=r.test_loss, eps=r.eps,
                      time_eps=r.time_eps, time_epoch=r.time_epoch, time_loss=r.time_loss,
                      time_test_loss=r.time_test_loss) for r in rows[:done.value + 1]]
        return trace, fb.value

    def save_factors(self):
        self._check(lib.dsgdpp_save_factors(self._h), "save_factors")

    def restore_factors(self):
        self._check(lib.dsgdpp_restore_factors(self._h), "restore_factors")

    def update_norms(self):
        a, b = C.c_double(), C.c_double()
        self._check(lib.dsgdpp_update_norms(self._h, C.byref(a), C.byref(b)), "update_norms")
        return a.value, b.value

    def sync(self):
        self._check(lib.dsgdpp_sync(self._h), "sync")

    # losses -----------------------------------------------------------------
    def loss(self) -> float:
        v = C.c_double()
        self._check(lib.dsgdpp_loss(self._h, C.byref(v)), "loss")
        return v.value

    def nzsl(self, which: int = TRAIN) -> float:
        v = C.c_double()
        self._check(lib.dsgdpp_nzsl(self._h, which, C.byref(v)), "nzsl")
        return v.value

    def l2(self):
        a, b = C.c_double(), C.c_double()
        self._check(lib.dsgdpp_l2(self._h, C.byref(a), C.byref(b)), "l2")
        return a.value, b.value

    def nzl2(self):
        a, b = C.c_double(), C.c_double()
        self._check(lib.dsgdpp_nzl2(self._h, C.byref(a), C.byref(b)), "nzl2")
        return a.value, b.value

    def run(self, epochs: int, decay: str = "BoldDriver", eps0: float = 0.001,
            decrease: float = 0.5, increase: float = 1.05):
        rows = (_TraceRow * (epochs + 1))()
        self._check(lib.dsgdpp_run(self._h, epochs, DECAY[decay], eps0, decrease, increase,
                                   rows), "run")
        return [dict(epoch=r.epoch, loss=r.loss, test_loss=r.test_loss, eps=r.eps,
                     time_eps=r.time_eps, time_epoch=r.time_epoch, time_loss=r.time_loss,
                     time_test_loss=r.time_test_loss) for r in rows]


SHARD_ID_BYTES = 128


def shard_unique_id() -> bytes:
    """A new NCCL unique id for :meth:`Shard.nccl` (made on rank 0)."""
    buf = C.create_string_buffer(SHARD_ID_BYTES)
    rc = lib.dsgdpp_shard_unique_id(C.cast(buf, C.c_void_p))
    if rc != OK:
        raise DsgdppError(rc, "shard_unique_id: NCCL is not available")
    return buf.raw


def shard_plan(d: int, nb2: int, world: int, schedule, holder):
    """The hand-off plan of one epoch (no GPU): an array of (group, block,
    from rank, to rank) rows (group 0 = before the epoch, s + 1 = after
    sub-epoch s) and the block holders after it (-1 = every rank)."""
    sch = _u32(schedule)
    h = np.ascontiguousarray(holder, np.int32).copy()
    hp = h.ctypes.data_as(C.POINTER(C.c_int32))
    n = lib.dsgdpp_shard_plan(d, nb2, world, _ptr(sch, C.c_uint32), hp, None)
    out = np.zeros((n, 4), np.uint32)
    h = np.ascontiguousarray(holder, np.int32).copy()
    hp = h.ctypes.data_as(C.POINTER(C.c_int32))
    lib.dsgdpp_shard_plan(d, nb2, world, _ptr(sch, C.c_uint32), hp, _ptr(out, C.c_uint32))
    return out, h


class Shard:
    """One DSGD++ job over several ranks (the hand-off of DsgdPpTask::run,
    mf/sgd/dsgdpp_impl.h:141-263): :meth:`nccl` for one rank per GPU and
    process, :meth:`local` for emulated ranks (contexts of this process)."""

    def __init__(self, handle, keep):
        self._h = handle
        self._keep = keep

    @classmethod
    def nccl(cls, ctx: "Context", rank: int, world: int, unique_id: bytes) -> "Shard":
        h = _P()
        buf = C.create_string_buffer(bytes(unique_id), SHARD_ID_BYTES)
        rc = lib.dsgdpp_shard_create_nccl(ctx._h, rank, world, C.cast(buf, C.c_void_p),
                                          C.byref(h))
        if rc != OK:
            raise DsgdppError(rc, "shard_create_nccl: " + lib.dsgdpp_last_error(ctx._h).decode())
        return cls(h, [ctx])

    @classmethod
    def local(cls, ctxs) -> "Shard":
        arr = (_P * len(ctxs))(*[c._h for c in ctxs])
        h = _P()
        rc = lib.dsgdpp_shard_create_local(arr, len(ctxs), C.byref(h))
        if rc != OK:
            raise DsgdppError(rc, "shard_create_local: " +
                              lib.dsgdpp_last_error(ctxs[0]._h).decode())
        return cls(h, list(ctxs))

    def close(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_shard_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != OK:
            raise DsgdppError(rc, f"{what}: {lib.dsgdpp_shard_last_error(self._h).decode()}")

    def set_wait_limit(self, seconds: float):
        self._check(lib.dsgdpp_shard_set_wait_limit(self._h, float(seconds)), "set_wait_limit")

    def epoch(self, eps: float, schedule=None, task_seeds=None):
        """One epoch on every rank: the given draws, or the master generator's."""
        if schedule is None:
            self._check(lib.dsgdpp_shard_epoch(self._h, eps, None, None), "shard_epoch")
            return
        s, t = _u32(schedule), _u32(task_seeds)
        self._check(lib.dsgdpp_shard_epoch(self._h, eps, _ptr(s, C.c_uint32),
                                           _ptr(t, C.c_uint32)), "shard_epoch")

    def share(self):
        self._check(lib.dsgdpp_shard_share(self._h), "shard_share")

    def gather_w(self):
        """Every rank's W rows to every rank (to read the result; ends the job)."""
        self._check(lib.dsgdpp_shard_gather_w(self._h), "shard_gather_w")

    def losses(self):
        """(training loss, test loss) of the whole job, after :meth:`share`."""
        a, b = C.c_double(), C.c_double()
        self._check(lib.dsgdpp_shard_losses(self._h, C.byref(a), C.byref(b)), "shard_losses")
        return a.value, b.value

    def moved(self):
        a, b = C.c_uint64(), C.c_uint64()
        self._check(lib.dsgdpp_shard_moved(self._h, C.byref(a), C.byref(b)), "shard_moved")
        return a.value, b.value

    def set_timeline(self, on: bool):
        self._check(lib.dsgdpp_shard_set_timeline(self._h, int(on)), "set_timeline")

    def timeline(self, index: int, nb2: int):
        """([nb2, 2] compute, [nb2, 2] transfer) begin/end in ms of the last epoch."""
        comp = np.zeros((nb2, 2))
        xfer = np.zeros((nb2, 2))
        self._check(lib.dsgdpp_shard_timeline(self._h, index, _ptr(comp, C.c_double),
                                              _ptr(xfer, C.c_double)), "shard_timeline")
        return comp, xfer


def _problem_array(problems):
    """ctypes array of dsgdpp_problem, and the numpy arrays it points into."""
    arr = (_Problem * len(problems))()
    keep = []
    for k, p in enumerate(problems):
        q = arr[k]
        q.m, q.n, q.rank, q.d = p["m"], p["n"], p["rank"], p.get("d", 0)
        rows, cols, vals = _u32(p["rows"]), _u32(p["cols"]), _f64(p["vals"])
        W, H = _f64(p["W"]), _f64(p["H"])
        q.nnz = len(vals)
        q.rows, q.cols = _ptr(rows, C.c_uint32), _ptr(cols, C.c_uint32)
        q.vals = _ptr(vals, C.c_double)
        q.W, q.H = _ptr(W, C.c_double), _ptr(H, C.c_double)
        keep += [rows, cols, vals, W, H]
        if p.get("tvals") is not None and len(p["tvals"]):
            tr, tc, tv = _u32(p["trows"]), _u32(p["tcols"]), _f64(p["tvals"])
            q.nnz_test = len(tv)
            q.trows, q.tcols = _ptr(tr, C.c_uint32), _ptr(tc, C.c_uint32)
            q.tvals = _ptr(tv, C.c_double)
            keep += [tr, tc, tv]
        q.seed = p.get("seed", 0)
        q.eps0 = p.get("eps0", 0.001)
    return arr, keep


class Batch:
    """Many independent factorizations advanced together (dsgdpp_batch_*).

    ``problems`` is a list of dicts with keys m, n, rank, rows, cols, vals,
    W, H and optionally d (0: chosen per problem), trows/tcols/tvals, seed,
    eps0.  ``config`` supplies everything the problems share; its m, n,
    rank and d are ignored.
    """

    def __init__(self, config: Config, problems):
        self.config = config
        self._cfg = config.to_c()
        arr, self._keep = _problem_array(problems)
        self.count = len(problems)
        self.shapes = [(p["m"], p["n"], p["rank"]) for p in problems]
        h = _P()
        rc = lib.dsgdpp_batch_create(C.byref(self._cfg), len(problems), arr, C.byref(h))
        self._keep = None  # the library holds its own copies
        if rc != OK:
            raise DsgdppError(rc, "dsgdpp_batch_create failed (details on stderr)")
        self._h = h

    @staticmethod
    def autotune(config: Config, problems, sample_stride: int = 8, epochs: int = 2):
        """The batched autotuner: (per-problem d list, CTAs per SM, sample epoch ms)."""
        arr, keep = _problem_array(problems)
        d = np.zeros(len(problems), np.uint32)
        ctas = C.c_uint32()
        ms = C.c_double()
        cfg = config.to_c()
        rc = lib.dsgdpp_batch_autotune(C.byref(cfg), len(problems), arr, sample_stride, epochs,
                                       _ptr(d, C.c_uint32), C.byref(ctas), C.byref(ms))
        del keep
        if rc != OK:
            raise DsgdppError(rc, "dsgdpp_batch_autotune failed (details on stderr)")
        return [int(v) for v in d], ctas.value, ms.value

    def _check(self, rc, what):
        if rc != OK:
            raise DsgdppError(rc, f"{what}: {lib.dsgdpp_batch_last_error(self._h).decode()}")

    def run(self, epochs: int, decrease: float = 0.5, increase: float = 1.05):
        """(train losses, test losses, summed epoch device ms) after `epochs` epochs."""
        tr = np.zeros(self.count)
        te = np.zeros(self.count)
        ms = C.c_double()
        self._check(lib.dsgdpp_batch_run(self._h, epochs, decrease, increase,
                                         _ptr(tr, C.c_double), _ptr(te, C.c_double),
                                         C.byref(ms)), "batch_run")
        return tr, te, ms.value

    def problem_d(self, p: int) -> int:
        d = C.c_uint32()
        self._check(lib.dsgdpp_batch_problem_d(self._h, p, C.byref(d)), "batch_problem_d")
        return d.value

    def get_factors(self, p: int):
        m, n, r = self.shapes[p]
        W = np.empty((m, r))
        H = np.empty((n, r))
        self._check(lib.dsgdpp_batch_get_factors(self._h, p, _ptr(W, C.c_double),
                                                 _ptr(H, C.c_double)), "batch_get_factors")
        return W, H

    def close(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(config: Config, rows, cols, vals, W, H, d_candidates=(64, 128, 256, 512),
             epochs: int = 3, eps: float = 0.001):
    """Fastest (d, lanes, vecs, CTAs/SM) for this data; returns (Config, ms)."""
    base = config.to_c()
    r, c, v = _u32(rows), _u32(cols), _f64(vals)
    w, h = _f64(W), _f64(H)
    ds = np.array(d_candidates, np.uint32)
    best = _Config()
    ms = C.c_double()
    rc = lib.dsgdpp_autotune(C.byref(base), len(v), _ptr(r, C.c_uint32), _ptr(c, C.c_uint32),
                             _ptr(v, C.c_double), _ptr(w, C.c_double), _ptr(h, C.c_double),
                             _ptr(ds, C.c_uint32), len(ds), epochs, eps, C.byref(best),
                             C.byref(ms))
    if rc != OK:
        raise DsgdppError(rc, "autotune")
    import dataclasses
    out = dataclasses.replace(config, d=best.d, lanes_per_nnz=best.lanes_per_nnz,
                              vecs_per_lane=best.vecs_per_lane, ctas_per_sm=best.ctas_per_sm)
    return out, ms.value


# ---- host utilities ---------------------------------------------------------
class Random32:
    """rg::Random32 as pinned by the library (MT19937, Boost bucket nextInt)."""

    def __init__(self, seed: int):
        self._h = lib.dsgdpp_rng_create(seed & 0xFFFFFFFF)

    def __del__(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_rng_destroy(self._h)
            self._h = None

    def next(self) -> int:
        return lib.dsgdpp_rng_next(self._h)

    def next_int(self, n: int) -> int:
        return lib.dsgdpp_rng_next_int(self._h, n)


def draw_schedule(rng: Random32, d: int, stratum_order: str = "COWOR"):
    """DsgdPpRunner::epoch draws: (2d x d schedule, d task seeds)."""
    s = np.empty((2 * d, d), np.uint32)
    t = np.empty(d, np.uint32)
    lib.dsgdpp_draw_schedule(rng._h, d, STRATUM_ORDER[stratum_order], _ptr(s, C.c_uint32),
                             _ptr(t, C.c_uint32))
    return s, t


def dsgd_schedule(rng: Random32, w: int, t: int, stratum_order: str) -> np.ndarray:
    out = np.empty((w * t, w * t), np.uint32)
    lib.dsgdpp_dsgd_schedule(rng._h, w, t, STRATUM_ORDER[stratum_order], _ptr(out, C.c_uint32))
    return out


def point_orders(d: int, sgd_order: str, block_nnz, schedule, task_seeds) -> np.ndarray:
    bn = np.ascontiguousarray(block_nnz, dtype=np.uint64).ravel()
    s, t = _u32(schedule), _u32(task_seeds)
    total = lib.dsgdpp_point_orders(d, SGD_ORDER[sgd_order], _ptr(bn, C.c_uint64),
                                    _ptr(s, C.c_uint32), _ptr(t, C.c_uint32), None)
    out = np.empty(total, np.uint32)
    lib.dsgdpp_point_orders(d, SGD_ORDER[sgd_order], _ptr(bn, C.c_uint64), _ptr(s, C.c_uint32),
                            _ptr(t, C.c_uint32), _ptr(out, C.c_uint32))
    return out


def block_offsets(size: int, blocks: int) -> np.ndarray:
    out = np.empty(blocks, np.uint64)
    lib.dsgdpp_block_offsets(size, blocks, _ptr(out, C.c_uint64))
    return out


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Mlp:
    """The step-size controller network (16 -> 64 -> 64 -> 1, GELU) on the GPU."""

    INPUTS = 16

    def __init__(self, device: int = 0, seed: int = 1):
        h = _P()
        rc = lib.dsgdpp_mlp_create(device, seed, C.byref(h))
        if rc != OK:
            raise DsgdppError(rc, "dsgdpp_mlp_create")
        self._h = h
        self.n_params = lib.dsgdpp_mlp_param_count()

    def close(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def _chk(self, rc, what):
        if rc != OK:
            raise DsgdppError(rc, what)

    @property
    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        self._chk(lib.dsgdpp_mlp_get_params(self._h, _ptr(p, C.c_float)), "mlp_get_params")
        return p

    @params.setter
    def params(self, p):
        p = _f32(p)
        self._chk(lib.dsgdpp_mlp_set_params(self._h, _ptr(p, C.c_float)), "mlp_set_params")

    def forward(self, x) -> np.ndarray:
        x = _f32(x).reshape(-1, self.INPUTS)
        out = np.empty(len(x), np.float32)
        self._chk(lib.dsgdpp_mlp_forward(self._h, _ptr(x, C.c_float), len(x), _ptr(out, C.c_float)),
                  "mlp_forward")
        return out

    def gradient(self, x, y):
        x = _f32(x).reshape(-1, self.INPUTS)
        y = _f32(y)
        g = np.empty(self.n_params, np.float32)
        loss = C.c_float()
        self._chk(lib.dsgdpp_mlp_gradient(self._h, _ptr(x, C.c_float), _ptr(y, C.c_float), len(x),
                                          C.byref(loss), _ptr(g, C.c_float)), "mlp_gradient")
        return loss.value, g

    def train_step(self, x, y, lr=1e-3) -> float:
        x = _f32(x).reshape(-1, self.INPUTS)
        y = _f32(y)
        loss = C.c_float()
        self._chk(lib.dsgdpp_mlp_train_step(self._h, _ptr(x, C.c_float), _ptr(y, C.c_float),
                                            len(x), lr, C.byref(loss)), "mlp_train_step")
        return loss.value


def controller_features(train_hist, test_hist, eps, upd_mean, upd_max, epoch_frac,
                        last_log_mult, fail_eps=0.0) -> np.ndarray:
    tr = np.full(5, np.nan)
    te = np.full(5, np.nan)
    tr[:min(5, len(train_hist))] = list(train_hist)[:5]
    te[:min(5, len(test_hist))] = list(test_hist)[:5]
    out = np.empty(16, np.float32)
    lib.dsgdpp_controller_features(_ptr(tr, C.c_double), _ptr(te, C.c_double), eps, upd_mean,
                                   upd_max, epoch_frac, last_log_mult, fail_eps,
                                   _ptr(out, C.c_float))
    return out


class IOError_(DsgdppError):
    pass


def _io(rc, what):
    if rc != OK:
        raise IOError_(rc, f"{what}: {lib.dsgdpp_io_error().decode()}")


def read_sparse(path: str):
    """.mmc or .xml-blocked sparse file -> (m, n, rows, cols, vals), 0-based."""
    m, n, nnz = C.c_uint64(), C.c_uint64(), C.c_uint64()
    r, c, v = _u32p(), _u32p(), _f64p()
    _io(lib.dsgdpp_read_sparse(path.encode(), C.byref(m), C.byref(n), C.byref(nnz), C.byref(r),
                               C.byref(c), C.byref(v)), "read_sparse")
    k = nnz.value
    try:
        rows = np.ctypeslib.as_array(r, shape=(max(k, 1),))[:k].copy()
        cols = np.ctypeslib.as_array(c, shape=(max(k, 1),))[:k].copy()
        vals = np.ctypeslib.as_array(v, shape=(max(k, 1),))[:k].copy()
    finally:
        for p in (r, c, v):
            lib.dsgdpp_free(C.cast(p, _P))
    return m.value, n.value, rows, cols, vals


def write_mm_coord(path: str, m: int, n: int, rows, cols, vals):
    r, c, v = _u32(rows), _u32(cols), _f64(vals)
    _io(lib.dsgdpp_write_mm_coord(path.encode(), m, n, len(v), _ptr(r, C.c_uint32),
                                  _ptr(c, C.c_uint32), _ptr(v, C.c_double)), "write_mm_coord")


def read_mm_array(path: str) -> np.ndarray:
    """.mma -> a size1 x size2 array (the file lists it column by column)."""
    m, n = C.c_uint64(), C.c_uint64()
    p = _f64p()
    _io(lib.dsgdpp_read_mm_array(path.encode(), C.byref(m), C.byref(n), C.byref(p)),
        "read_mm_array")
    try:
        k = m.value * n.value
        flat = np.ctypeslib.as_array(p, shape=(max(k, 1),))[:k].copy()
    finally:
        lib.dsgdpp_free(C.cast(p, _P))
    return flat.reshape(n.value, m.value).T.copy()


def write_mm_array(path: str, a):
    a = np.asarray(a, np.float64)
    flat = np.ascontiguousarray(a.T).ravel()
    _io(lib.dsgdpp_write_mm_array(path.encode(), a.shape[0], a.shape[1], _ptr(flat, C.c_double)),
        "write_mm_array")


def write_blocked(xml_path: str, directory: str, base: str, m: int, n: int, blocks1: int,
                  blocks2: int, rows, cols, vals):
    r, c, v = _u32(rows), _u32(cols), _f64(vals)
    _io(lib.dsgdpp_write_blocked(xml_path.encode(), directory.encode(), base.encode(), m, n,
                                 blocks1, blocks2, len(v), _ptr(r, C.c_uint32),
                                 _ptr(c, C.c_uint32), _ptr(v, C.c_double)), "write_blocked")


def philox4x32_10(ctr, key) -> np.ndarray:
    c, k = _u32(ctr), _u32(key)
    out = np.empty(4, np.uint32)
    lib.dsgdpp_philox4x32_10(_ptr(c, C.c_uint32), _ptr(k, C.c_uint32), _ptr(out, C.c_uint32))
    return out


class RandomMatrix:
    """A .rm random-matrix descriptor (RandomMatrixDescriptor): load one with
    RandomMatrix(path), make one with RandomMatrix.create(...)."""

    def __init__(self, path: Optional[str] = None, _handle=None):
        self._h = _handle
        if path is not None:
            h = _P()
            rc = lib.dsgdpp_rm_load(path.encode(), C.byref(h))
            if rc != OK:
                raise DsgdppError(rc, f"rm_load: {lib.dsgdpp_rm_error().decode()}")
            self._h = h

    @staticmethod
    def create(size1, size2, blocks1, blocks2, nnz, nnz_test, rank, values, noise=""):
        h = _P()
        rc = lib.dsgdpp_rm_create(size1, size2, blocks1, blocks2, nnz, nnz_test, rank,
                                  values.encode(), noise.encode(), C.byref(h))
        if rc != OK:
            raise DsgdppError(rc, f"rm_create: {lib.dsgdpp_rm_error().decode()}")
        return RandomMatrix(_handle=h)

    def _chk(self, rc, what):
        if rc != OK:
            raise DsgdppError(rc, f"{what}: {lib.dsgdpp_rm_error().decode()}")

    def save(self, path: str):
        self._chk(lib.dsgdpp_rm_save(self._h, path.encode()), "rm_save")

    def info(self) -> dict:
        out = np.zeros(9, np.uint64)
        self._chk(lib.dsgdpp_rm_info(self._h, _ptr(out, C.c_uint64)), "rm_info")
        keys = ("size1", "size2", "rank", "blocks1", "blocks2", "nnz", "nnz_test", "data_nnz",
                "test_nnz")
        return {k: int(v) for k, v in zip(keys, out)}

    def generate(self, which: int = TRAIN, device: int = 0):
        """(rows, cols, vals) of the data or test matrix, generated on the GPU."""
        n = self.info()["data_nnz" if which == TRAIN else "test_nnz"]
        rows = np.empty(n, np.uint32)
        cols = np.empty(n, np.uint32)
        vals = np.empty(n, np.float64)
        self._chk(lib.dsgdpp_rm_generate(self._h, which, device, _ptr(rows, C.c_uint32),
                                         _ptr(cols, C.c_uint32), _ptr(vals, C.c_double)),
                  "rm_generate")
        return rows, cols, vals

    def generate_factors(self, device: int = 0):
        """(Worig: size1 x rank, Horig: size2 x rank), generated on the GPU."""
        i = self.info()
        W = np.empty((i["size1"], i["rank"]), np.float64)
        H = np.empty((i["size2"], i["rank"]), np.float64)
        self._chk(lib.dsgdpp_rm_generate_factors(self._h, device, _ptr(W, C.c_double),
                                                 _ptr(H, C.c_double)), "rm_generate_factors")
        return W, H

    def close(self):
        if getattr(self, "_h", None):
            lib.dsgdpp_rm_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
