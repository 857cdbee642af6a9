"""Python binding of the B200 HPR-QP engine.

Mirrors the reference package's public surface (python/src/hprqp/__init__.py
of PolyU-IOR/HPR-QP-C): ``Model``, ``Parameters``, ``Result``,
``build_from_qabc`` / ``build_from_QAbc``, ``optimize``, ``status_name``,
``gpu_backend_available`` and the STATUS_* / SPMV_MODE_* constants, all on
top of the same ``hprqp_*`` opaque-handle C ABI.  The library is
``libhprqp.so`` built in-tree by ``hpr-qp-c_b200/build.py`` (override the
path with ``HPRQP_LIBRARY_PATH``).  There is no CPU fallback: if the library
cannot be loaded an ``OSError`` is raised, and ``use_gpu=False`` returns
``STATUS_NOT_IMPLEMENTED``.

Additions beyond the reference: ``spmv`` and ``setup_info`` (engine
diagnostics), the batched solver (``hprqp.batch``) and the differentiable
layer (``hprqp.torch_layer.QPFunction``).
"""
from __future__ import annotations

import ctypes
import math
import os
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, Optional, Sequence

import numpy as np

STATUS_OK = 0
STATUS_INVALID_ARGUMENT = 1
STATUS_ALLOCATION_FAILED = 2
STATUS_NOT_IMPLEMENTED = 3
STATUS_MAX_ITER = 4
STATUS_TIME_LIMIT = 5
STATUS_OPTIMAL = 6
STATUS_CONTINUE = 7

SPMV_MODE_AUTO = 0
SPMV_MODE_CUSPARSE = 1
SPMV_MODE_CUSTOMIZED = 2

_PKG_ROOT = Path(__file__).resolve().parents[2]  # hpr-qp-c_b200/
DEFAULT_LIBRARY = _PKG_ROOT / "lib" / "libhprqp.so"

c_size_p = ctypes.POINTER(ctypes.c_size_t)
c_double_p = ctypes.POINTER(ctypes.c_double)


@dataclass(frozen=True)
class Result:
    status_code: int
    status: str
    iter: int
    iter_4: int
    iter_6: int
    time: float
    time_4: float
    time_6: float
    objective: float
    residual: float
    gap: float
    x: list
    y: list
    z: list
    w: list


class _MatrixCSR(ctypes.Structure):
    _fields_ = [("nrow", ctypes.c_size_t), ("ncol", ctypes.c_size_t), ("nnz", ctypes.c_size_t),
                ("row_ptr", c_size_p), ("col_ind", c_size_p), ("values", c_double_p), ("owns_data", ctypes.c_int)]


class _ModelStruct(ctypes.Structure):
    _fields_ = [("Q", _MatrixCSR), ("A", _MatrixCSR), ("AT", _MatrixCSR), ("c", c_double_p),
                ("AL", c_double_p), ("AU", c_double_p), ("l", c_double_p), ("u", c_double_p),
                ("obj_constant", ctypes.c_double), ("owns_data", ctypes.c_int),
                ("num_var_cones", ctypes.c_size_t), ("var_cone_offsets", c_size_p),
                ("num_row_cones", ctypes.c_size_t), ("row_cone_offsets", c_size_p), ("soc_rhs", c_double_p)]


class _ParamsStruct(ctypes.Structure):
    _fields_ = [("stoptol", ctypes.c_double), ("max_iter", ctypes.c_size_t), ("use_gpu", ctypes.c_int),
                ("device_number", ctypes.c_int), ("time_limit", ctypes.c_double),
                ("check_iter", ctypes.c_size_t), ("print_frequency", ctypes.c_int),
                ("use_scaling", ctypes.c_int), ("verbose", ctypes.c_int), ("spmv_mode_q", ctypes.c_int),
                ("spmv_mode_a", ctypes.c_int), ("gram_mode", ctypes.c_int), ("polishing", ctypes.c_int),
                ("polish_python", ctypes.c_char_p), ("polish_worker", ctypes.c_char_p),
                ("polish_directory", ctypes.c_char_p), ("polish_keep_files", ctypes.c_int),
                ("polish_max_attempts", ctypes.c_size_t), ("polish_episode_seconds", ctypes.c_double),
                ("polish_total_seconds", ctypes.c_double), ("polish_memory_bytes", ctypes.c_size_t)]


class _Library:
    _instance: Optional[ctypes.CDLL] = None
    _path: Optional[str] = None

    @classmethod
    def load(cls) -> ctypes.CDLL:
        if cls._instance is not None:
            return cls._instance
        path = os.environ.get("HPRQP_LIBRARY_PATH") or str(DEFAULT_LIBRARY)
        if not Path(path).exists():
            raise OSError(f"libhprqp.so not found at {path}; build it with `python hpr-qp-c_b200/build.py`")
        lib = ctypes.CDLL(path)
        cls._configure(lib)
        cls._instance = lib
        cls._path = path
        return lib

    @staticmethod
    def _configure(lib: ctypes.CDLL) -> None:
        vp = ctypes.c_void_p
        lib.hprqp_solve_for_backward.argtypes = [ctypes.c_void_p] * 3 + [ctypes.POINTER(ctypes.c_void_p)]
        lib.hprqp_solve_for_backward.restype = ctypes.c_int
        lib.hprqp_backward.argtypes = [ctypes.c_void_p, c_double_p, c_double_p, ctypes.c_double, ctypes.c_longlong,
                                       ctypes.c_void_p]
        lib.hprqp_backward.restype = ctypes.c_int
        lib.hprqp_solve_state_destroy.argtypes = [ctypes.c_void_p]
        lib.hprqp_solve_state_destroy.restype = None
        lib.hprqp_status_name.argtypes = [ctypes.c_int]
        lib.hprqp_status_name.restype = ctypes.c_char_p
        lib.hprqp_gpu_backend_available.restype = ctypes.c_int
        lib.hprqp_model_create.argtypes = [ctypes.POINTER(vp)]
        lib.hprqp_model_destroy.argtypes = [vp]
        lib.hprqp_model_destroy.restype = None
        lib.hprqp_model_build_from_qabc_csr.argtypes = [
            vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, c_size_p, c_size_p, c_double_p,
            ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, c_size_p, c_size_p, c_double_p,
            c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, ctypes.c_double]
        lib.hprqp_model_num_variables.argtypes = [vp]
        lib.hprqp_model_num_variables.restype = ctypes.c_size_t
        lib.hprqp_model_num_constraints.argtypes = [vp]
        lib.hprqp_model_num_constraints.restype = ctypes.c_size_t
        lib.hprqp_params_create.argtypes = [ctypes.POINTER(vp)]
        lib.hprqp_params_destroy.argtypes = [vp]
        lib.hprqp_params_destroy.restype = None
        lib.hprqp_params_set_defaults.argtypes = [vp]
        for name, t in (("stoptol", ctypes.c_double), ("max_iter", ctypes.c_size_t), ("use_gpu", ctypes.c_int),
                        ("device_number", ctypes.c_int), ("time_limit", ctypes.c_double),
                        ("check_iter", ctypes.c_size_t), ("print_frequency", ctypes.c_int),
                        ("use_scaling", ctypes.c_int), ("verbose", ctypes.c_int), ("spmv_mode_q", ctypes.c_int),
                        ("spmv_mode_a", ctypes.c_int)):
            getattr(lib, f"hprqp_params_set_{name}").argtypes = [vp, t]
        lib.hprqp_results_create.argtypes = [ctypes.POINTER(vp)]
        lib.hprqp_results_destroy.argtypes = [vp]
        lib.hprqp_results_destroy.restype = None
        lib.hprqp_optimize.argtypes = [vp, vp, vp]
        for name in ("num_variables", "num_constraints", "iter", "iter_4", "iter_6"):
            getattr(lib, f"hprqp_results_{name}").argtypes = [vp]
            getattr(lib, f"hprqp_results_{name}").restype = ctypes.c_size_t
        for name in ("time", "time_4", "time_6", "objective", "residual", "gap"):
            getattr(lib, f"hprqp_results_{name}").argtypes = [vp]
            getattr(lib, f"hprqp_results_{name}").restype = ctypes.c_double
        for name in ("x", "y", "z", "w"):
            getattr(lib, f"hprqp_results_{name}_data").argtypes = [vp]
            getattr(lib, f"hprqp_results_{name}_data").restype = c_double_p
        lib.hprqp_b200_spmv.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, c_size_p, c_size_p,
                                        c_double_p, c_double_p, c_double_p, ctypes.c_int, c_double_p]
        lib.hprqp_b200_gather_bound.argtypes = [ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, c_size_p,
                                                c_size_p, c_double_p, c_double_p, ctypes.c_int, c_double_p,
                                                c_double_p]
        lib.hprqp_b200_setup.argtypes = [ctypes.POINTER(_ModelStruct), ctypes.POINTER(_ParamsStruct)] + \
            [c_double_p] * 11
        lib.hprqp_b200_launch_count.restype = ctypes.c_uint64
        lib.hprqp_b200_set_single_cta_max_work.argtypes = [ctypes.c_size_t]
        lib.hprqp_b200_set_single_cta_max_work.restype = ctypes.c_size_t
        lib.params_set_defaults.argtypes = [ctypes.POINTER(_ParamsStruct)]
        lib.params_set_defaults.restype = None


def _lib() -> ctypes.CDLL:
    return _Library.load()


def library_path() -> str:
    _lib()
    return str(_Library._path)


def status_name(status: int) -> str:
    return _lib().hprqp_status_name(int(status)).decode("utf-8")


def gpu_backend_available() -> bool:
    return bool(_lib().hprqp_gpu_backend_available())


def launch_count() -> int:
    return int(_lib().hprqp_b200_launch_count())


def set_single_cta_max_work(max_work: int) -> int:
    """Route solve_gpu: models without cones whose products per iteration
    touch at most ``max_work`` nonzeros (2 nnz(Q) + 2 nnz(A)) are solved in
    one CTA of the batch kernel; 0 sends every model through the host-driven
    loop.  Returns the previous value (hprqp_b200_set_single_cta_max_work)."""
    return int(_lib().hprqp_b200_set_single_cta_max_work(int(max_work)))


def _raise_for_status(code: int, context: str) -> int:
    if code != STATUS_OK:
        raise RuntimeError(f"{context} failed with status {status_name(code)}")
    return code


def _spmv_mode_code(value) -> int:
    if value in (SPMV_MODE_AUTO, "auto"):
        return SPMV_MODE_AUTO
    if value in (SPMV_MODE_CUSPARSE, "cusparse"):
        return SPMV_MODE_CUSPARSE
    if value in (SPMV_MODE_CUSTOMIZED, "customized"):
        return SPMV_MODE_CUSTOMIZED
    raise ValueError("Unsupported SpMV mode. Expected 'auto', 'cusparse', or 'customized'.")


class Model:
    def __init__(self) -> None:
        handle = ctypes.c_void_p()
        self._lib_ref = _lib()
        _raise_for_status(self._lib_ref.hprqp_model_create(ctypes.byref(handle)), "hprqp_model_create")
        self._handle = handle

    def __del__(self) -> None:
        # the library handle is read from the instance: at interpreter exit
        # the module's globals may already be gone
        handle, lib = getattr(self, "_handle", None), getattr(self, "_lib_ref", None)
        if handle is not None and handle.value and lib is not None:
            lib.hprqp_model_destroy(handle)
            handle.value = None

    @property
    def num_variables(self) -> int:
        return int(_lib().hprqp_model_num_variables(self._handle))

    @property
    def num_constraints(self) -> int:
        return int(_lib().hprqp_model_num_constraints(self._handle))

    def _struct(self) -> _ModelStruct:
        # the binding model struct starts with an HPRQPModel
        return ctypes.cast(self._handle, ctypes.POINTER(_ModelStruct)).contents

    def to_instance(self, name: str = ""):
        """Copies of the built (preprocessed) model's arrays as a
        :class:`hprqp.instances.QPInstance` -- Q, A, c, AL, AU, l, u and the
        objective constant -- e.g. to solve models read from MPS files as one
        batch (:mod:`hprqp.batch`).  Cone models are not supported."""
        from .instances import CSR, QPInstance

        st = self._struct()
        if st.num_var_cones or st.num_row_cones:
            raise ValueError("to_instance: cone models are not supported")

        def csr(M):
            nrow, nnz = int(M.nrow), int(M.nnz)
            ip = np.ctypeslib.as_array(M.row_ptr, (nrow + 1,)).astype(np.int64)
            ii = np.ctypeslib.as_array(M.col_ind, (nnz,)).astype(np.int64) if nnz else np.zeros(0, np.int64)
            dd = np.ctypeslib.as_array(M.values, (nnz,)).copy() if nnz else np.zeros(0)
            return CSR(nrow, int(M.ncol), ip, ii, dd)

        n, m = int(st.Q.nrow), int(st.A.nrow)
        vec = (lambda p, k: np.ctypeslib.as_array(p, (k,)).copy() if k else np.zeros(0))  # noqa: E731
        return QPInstance(csr(st.Q), csr(st.A), vec(st.c, n), vec(st.AL, m), vec(st.AU, m), vec(st.l, n),
                          vec(st.u, n), float(st.obj_constant), name)


class Parameters:
    def __init__(self, **kwargs) -> None:
        handle = ctypes.c_void_p()
        self._lib_ref = _lib()
        _raise_for_status(self._lib_ref.hprqp_params_create(ctypes.byref(handle)), "hprqp_params_create")
        self._handle = handle
        for name, value in kwargs.items():
            getattr(self, f"set_{name}")(value)

    def __del__(self) -> None:
        # the library handle is read from the instance: at interpreter exit
        # the module's globals may already be gone
        handle, lib = getattr(self, "_handle", None), getattr(self, "_lib_ref", None)
        if handle is not None and handle.value and lib is not None:
            lib.hprqp_params_destroy(handle)
            handle.value = None

    def _call(self, func_name: str, *args) -> "Parameters":
        _raise_for_status(getattr(_lib(), func_name)(self._handle, *args), func_name)
        return self

    def set_defaults(self):
        return self._call("hprqp_params_set_defaults")

    def set_stoptol(self, value: float):
        return self._call("hprqp_params_set_stoptol", float(value))

    def set_max_iter(self, value: int):
        return self._call("hprqp_params_set_max_iter", int(value))

    def set_use_gpu(self, value: bool):
        return self._call("hprqp_params_set_use_gpu", 1 if value else 0)

    def set_device_number(self, value: int):
        return self._call("hprqp_params_set_device_number", int(value))

    def set_time_limit(self, value: float):
        return self._call("hprqp_params_set_time_limit", float(value))

    def set_check_iter(self, value: int):
        return self._call("hprqp_params_set_check_iter", int(value))

    def set_print_frequency(self, value: int):
        return self._call("hprqp_params_set_print_frequency", int(value))

    def set_use_scaling(self, value: bool):
        return self._call("hprqp_params_set_use_scaling", 1 if value else 0)

    def set_verbose(self, value: bool):
        return self._call("hprqp_params_set_verbose", 1 if value else 0)

    def set_spmv_mode_q(self, value):
        return self._call("hprqp_params_set_spmv_mode_q", _spmv_mode_code(value))

    def set_spmv_mode_a(self, value):
        return self._call("hprqp_params_set_spmv_mode_a", _spmv_mode_code(value))

    def _struct(self) -> _ParamsStruct:
        return ctypes.cast(self._handle, ctypes.POINTER(_ParamsStruct)).contents


def read_from_mps(path) -> Model:
    model = Model()
    _raise_for_status(_lib().hprqp_model_read_from_mps(model._handle, os.fspath(path).encode()),
                      "hprqp_model_read_from_mps")
    return model


build_from_mps = read_from_mps


def _is_scipy_sparse(matrix) -> bool:
    return all(hasattr(matrix, a) for a in ("indptr", "indices", "data", "shape"))


def _matrix_to_csr(matrix):
    """(nrow, ncol, indptr, indices, data) from a dense list, a numpy array,
    a scipy sparse matrix or an instances.CSR."""
    if hasattr(matrix, "indptr") and hasattr(matrix, "nrow"):
        return (int(matrix.nrow), int(matrix.ncol), np.asarray(matrix.indptr, np.uint64),
                np.asarray(matrix.indices, np.uint64), np.asarray(matrix.data, np.float64))
    if _is_scipy_sparse(matrix):
        csr = matrix.tocsr()
        return (int(csr.shape[0]), int(csr.shape[1]), csr.indptr.astype(np.uint64), csr.indices.astype(np.uint64),
                csr.data.astype(np.float64))
    arr = np.asarray(matrix, dtype=np.float64)
    if arr.size == 0:
        return 0, 0, np.zeros(1, np.uint64), np.zeros(0, np.uint64), np.zeros(0)
    if arr.ndim != 2:
        raise TypeError("Expected a dense row-major matrix or a SciPy sparse matrix.")
    rows, cols = np.nonzero(arr)
    indptr = np.zeros(arr.shape[0] + 1, np.uint64)
    np.add.at(indptr, rows + 1, 1)
    return arr.shape[0], arr.shape[1], np.cumsum(indptr).astype(np.uint64), cols.astype(np.uint64), arr[rows, cols]


def _vec(values, n: int, name: str) -> np.ndarray:
    out = np.ascontiguousarray(np.asarray(list(values) if not isinstance(values, np.ndarray) else values,
                                          dtype=np.float64).reshape(-1))
    if out.shape[0] != n:
        raise ValueError(f"{name} length {out.shape[0]} does not match expected length {n}.")
    return out


def _ptr_sz(a: np.ndarray):
    if a.size == 0:
        a = np.zeros(1, np.uint64)
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(c_size_p)


def _ptr_db(a: np.ndarray):
    if a.size == 0:
        a = np.zeros(1)
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(c_double_p)


def build_from_qabc(Q, c, A, AL, AU, l, u, obj_constant: float = 0.0) -> Model:
    qn, qm, qp, qi, qv = _matrix_to_csr(Q)
    an, am, ap, ai, av = _matrix_to_csr(A)
    if qn != qm:
        raise ValueError("Q must be square.")
    if an == 0 and am == 0:
        am = qm
        ap = np.zeros(1, np.uint64)
    if am != qm:
        raise ValueError("A column count must match Q size.")
    c_arr = _vec(c, qm, "c")
    l_arr = _vec(l, qm, "l")
    u_arr = _vec(u, qm, "u")
    keep = []

    def sz(a):
        arr, p = _ptr_sz(a)
        keep.append(arr)
        return p

    def db(a):
        arr, p = _ptr_db(a)
        keep.append(arr)
        return p

    al = db(_vec(AL, an, "AL")) if an else None
    au = db(_vec(AU, an, "AU")) if an else None
    model = Model()
    status = _lib().hprqp_model_build_from_qabc_csr(
        model._handle, qn, qm, len(qv), sz(qp), sz(qi), db(qv), an, am, len(av), sz(ap), sz(ai), db(av),
        db(c_arr), al, au, db(l_arr), db(u_arr), float(obj_constant))
    _raise_for_status(status, "hprqp_model_build_from_qabc_csr")
    return model


build_from_QAbc = build_from_qabc


class _SOCSpec(ctypes.Structure):
    _fields_ = [("num_var_cones", ctypes.c_size_t), ("var_offsets", c_size_p), ("num_row_cones", ctypes.c_size_t),
                ("row_offsets", c_size_p), ("rhs", c_double_p)]


def build_from_qabc_soc(Q, c, A, AL, AU, l, u, var_cone_offsets=None, row_cone_offsets=None, rhs=None,
                        obj_constant: float = 0.0) -> Model:
    """QP with second-order cones (build_from_QAbc_soc, include/hprqp.h):
    variables [var_cone_offsets[0], n) and rows [row_cone_offsets[0], m) are
    split into Lorentz cones {(t, v): |v| <= t} at the offsets (count + 1
    entries each, ending at n / m); cone variables have bounds (-inf, inf);
    cone rows have AL = -inf, AU = inf and mean A x - rhs in K; rhs (m
    entries) is zero on the linear rows."""
    qn, qm, qp, qi, qv = _matrix_to_csr(Q)
    an, am, ap, ai, av = _matrix_to_csr(A)
    if an == 0 and am == 0:
        am = qm
        ap = np.zeros(1, np.uint64)
    keep = []

    def csr(nr, nc, p, i, v):
        p = np.ascontiguousarray(p, np.uint64)
        i = np.ascontiguousarray(i if len(i) else np.zeros(1), np.uint64)
        v = np.ascontiguousarray(v if len(v) else np.zeros(1), np.float64)
        keep.extend([p, i, v])
        return _MatrixCSR(nr, nc, int(p[-1]), p.ctypes.data_as(c_size_p), i.ctypes.data_as(c_size_p),
                          v.ctypes.data_as(c_double_p), 0)

    def db(a, k, name):
        arr = _vec(a, k, name) if k else np.zeros(1)
        keep.append(arr)
        return arr.ctypes.data_as(c_double_p)

    def offs(o):
        if o is None or len(o) == 0:
            return 0, None
        arr = np.ascontiguousarray(np.asarray(o, np.uint64))
        keep.append(arr)
        return len(arr) - 1, arr.ctypes.data_as(c_size_p)

    nv, vp = offs(var_cone_offsets)
    nr, rp = offs(row_cone_offsets)
    spec = _SOCSpec(nv, vp, nr, rp, db(rhs, an, "rhs") if rhs is not None else None)
    Qc, Ac = csr(qn, qm, qp, qi, qv), csr(an, am, ap, ai, av)
    model = Model()
    lib = _lib()
    lib.build_from_QAbc_soc.argtypes = [ctypes.POINTER(_MatrixCSR), ctypes.POINTER(_MatrixCSR)] + \
        [c_double_p] * 5 + [ctypes.c_double, ctypes.POINTER(_SOCSpec), ctypes.c_void_p]
    lib.build_from_QAbc_soc.restype = ctypes.c_int
    st = lib.build_from_QAbc_soc(ctypes.byref(Qc), ctypes.byref(Ac), db(c, qm, "c"),
                                 db(AL, an, "AL") if an else None, db(AU, an, "AU") if an else None,
                                 db(l, qm, "l"), db(u, qm, "u"), float(obj_constant), ctypes.byref(spec),
                                 model._handle)
    _raise_for_status(st, "build_from_QAbc_soc")
    return model


def build_from_qabc_qc(Q, c, A, AL, AU, l, u, C, constant, R=None, offsets=None, D=None,
                       obj_constant: float = 0.0) -> Model:
    """QP with convex quadratic constraints (include/shared/qcqp.h):
    row i of C with constant[i] and either the factor R_i (rows
    [offsets[i], offsets[i+1]) of R: build_from_QAbc_qc_factors) or the
    diagonal D_i (row i of D: build_from_QAbc_qc_diagonal) gives
    C_i x + 1/2 |R_i x|^2 + constant_i <= 0  (D_i = R_i' R_i).  Each is
    lifted to one second-order cone after the rows of A; solve_gpu runs the
    cone path.  The matrices may be dense or scipy sparse."""
    if (R is None) == (D is None):
        raise ValueError("give either R with offsets or D")
    keep = []

    def csr(mat):
        nr, nc, p, i, v = _matrix_to_csr(mat)
        p = np.ascontiguousarray(p if len(p) else np.zeros(1), np.uint64)
        i = np.ascontiguousarray(i if len(i) else np.zeros(1), np.uint64)
        v = np.ascontiguousarray(v if len(v) else np.zeros(1), np.float64)
        keep.extend([p, i, v])
        return _MatrixCSR(nr, nc, int(p[-1]), p.ctypes.data_as(c_size_p), i.ctypes.data_as(c_size_p),
                          v.ctypes.data_as(c_double_p), 0)

    def db(a, k, name):
        arr = _vec(a, k, name) if k else np.zeros(1)
        keep.append(arr)
        return arr.ctypes.data_as(c_double_p)

    Qc, Cc = csr(Q), csr(C)
    n = int(Qc.ncol)
    Ac = csr(A)
    if Ac.nrow == 0:
        Ac.ncol = n
    m, nq = int(Ac.nrow), int(Cc.nrow)
    lib = _lib()
    M = ctypes.POINTER(_MatrixCSR)
    head = [ctypes.byref(Qc), ctypes.byref(Ac), db(c, n, "c"), db(AL, m, "AL") if m else None,
            db(AU, m, "AU") if m else None, db(l, n, "l"), db(u, n, "u"), float(obj_constant), ctypes.byref(Cc),
            db(constant, nq, "constant")]
    model = Model()
    if D is not None:
        fn = lib.build_from_QAbc_qc_diagonal
        fn.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, M, c_double_p, M, ctypes.c_void_p]
        args = head + [ctypes.byref(csr(D)), model._handle]
    else:
        off = np.ascontiguousarray(np.asarray(offsets if offsets is not None else [], np.uint64))
        if off.shape[0] != nq + 1:
            raise ValueError(f"offsets: expected {nq + 1} entries, got {off.shape[0]}")
        keep.append(off)
        fn = lib.build_from_QAbc_qc_factors
        fn.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, M, c_double_p, M, c_size_p, ctypes.c_void_p]
        args = head + [ctypes.byref(csr(R)), off.ctypes.data_as(c_size_p), model._handle]
    fn.restype = ctypes.c_int
    _raise_for_status(fn(*args), "build_from_QAbc_qc")
    return model


def build_from_instance(inst) -> Model:
    """Model from an ``instances.QPInstance`` (CSR arrays, no copies in Python)."""
    return build_from_qabc(inst.Q, inst.c, inst.A, inst.AL, inst.AU, inst.l, inst.u, inst.obj_constant)


def _copy_vector(pointer, length: int) -> list:
    if not pointer or length == 0:
        return []
    return np.ctypeslib.as_array(pointer, shape=(length,)).copy().tolist()


def optimize(model: Model, params: Optional[Parameters] = None, as_numpy: bool = False) -> Result:
    if params is None:
        params = Parameters()
    lib = _lib()
    results_handle = ctypes.c_void_p()
    _raise_for_status(lib.hprqp_results_create(ctypes.byref(results_handle)), "hprqp_results_create")
    try:
        status_code = int(lib.hprqp_optimize(model._handle, params._handle, results_handle))
        n = int(lib.hprqp_results_num_variables(results_handle))
        m = int(lib.hprqp_results_num_constraints(results_handle))

        def vec(fn, k):
            p = fn(results_handle)
            if not p or k == 0:
                return np.zeros(0) if as_numpy else []
            arr = np.ctypeslib.as_array(p, shape=(k,)).copy()
            return arr if as_numpy else arr.tolist()

        return Result(
            status_code=status_code,
            status=status_name(status_code),
            iter=int(lib.hprqp_results_iter(results_handle)),
            iter_4=int(lib.hprqp_results_iter_4(results_handle)),
            iter_6=int(lib.hprqp_results_iter_6(results_handle)),
            time=float(lib.hprqp_results_time(results_handle)),
            time_4=float(lib.hprqp_results_time_4(results_handle)),
            time_6=float(lib.hprqp_results_time_6(results_handle)),
            objective=float(lib.hprqp_results_objective(results_handle)),
            residual=float(lib.hprqp_results_residual(results_handle)),
            gap=float(lib.hprqp_results_gap(results_handle)),
            x=vec(lib.hprqp_results_x_data, n),
            y=vec(lib.hprqp_results_y_data, m),
            z=vec(lib.hprqp_results_z_data, n),
            w=vec(lib.hprqp_results_w_data, n),
        )
    finally:
        lib.hprqp_results_destroy(results_handle)


class _ResidualsStruct(ctypes.Structure):
    _fields_ = [("is_updated", ctypes.c_int), ("err_Rp_org_bar", ctypes.c_double),
                ("err_Rd_org_bar", ctypes.c_double), ("KKTx_and_gap_org_bar", ctypes.c_double),
                ("primal_obj_bar", ctypes.c_double), ("rel_gap_bar", ctypes.c_double),
                ("dual_obj_bar", ctypes.c_double)]


def residuals(model: Model, x, y, z, iter: int = 1, params: Optional[Parameters] = None) -> dict:
    """The solver's residual kernels at a given point of the preprocessed
    model (hprqp_b200_residuals): errRp, errRd, gap, objectives, KKT."""
    if params is None:
        params = Parameters(verbose=False)
    n, m = model.num_variables, model.num_constraints
    xa = np.ascontiguousarray(np.broadcast_to(np.asarray(x, np.float64), (n,)))
    za = np.ascontiguousarray(np.broadcast_to(np.asarray(z, np.float64), (n,)))
    ya = np.ascontiguousarray(np.broadcast_to(np.asarray(y, np.float64), (m,))) if m else np.zeros(1)
    out = _ResidualsStruct()
    lib = _lib()
    lib.hprqp_b200_residuals.argtypes = [ctypes.c_void_p, ctypes.c_void_p, c_double_p, c_double_p, c_double_p,
                                         ctypes.c_size_t, ctypes.POINTER(_ResidualsStruct)]
    lib.hprqp_b200_residuals.restype = ctypes.c_int
    _raise_for_status(lib.hprqp_b200_residuals(model._handle, params._handle, xa.ctypes.data_as(c_double_p),
                                               ya.ctypes.data_as(c_double_p), za.ctypes.data_as(c_double_p),
                                               int(iter), ctypes.byref(out)), "hprqp_b200_residuals")
    return {"err_rp": out.err_Rp_org_bar, "err_rd": out.err_Rd_org_bar, "gap": out.rel_gap_bar,
            "primal_obj": out.primal_obj_bar, "dual_obj": out.dual_obj_bar, "kkt": out.KKTx_and_gap_org_bar}


class _ResultsStruct(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_size_t), ("iter_4", ctypes.c_size_t), ("iter_6", ctypes.c_size_t),
                ("time", ctypes.c_double), ("time_4", ctypes.c_double), ("time_6", ctypes.c_double),
                ("primal_obj", ctypes.c_double), ("residuals", ctypes.c_double), ("gap", ctypes.c_double),
                ("status", ctypes.c_int), ("x", c_double_p), ("y", c_double_p), ("z", c_double_p),
                ("w", c_double_p), ("polish_attempts", ctypes.c_size_t), ("polish_accepted", ctypes.c_int),
                ("gram_active", ctypes.c_int), ("total_time", ctypes.c_double)]


class _GradientsStruct(ctypes.Structure):
    _fields_ = [(k, c_double_p) for k in ("dc", "dl", "du", "dAL", "dAU", "dQ_values", "dA_values", "lam", "mu")] + \
               [("minres_iters", ctypes.c_longlong), ("minres_relres", ctypes.c_double),
                ("backward_seconds", ctypes.c_double)]


class SolveState:
    """Device state of a finished solve, kept for :meth:`backward`
    (hprqp_diff.h).  Gradients are in the space of the model (its symmetrised
    Q, the rows of A kept by preprocessing), like the solution."""

    def __init__(self, model: "Model", handle: ctypes.c_void_p):
        self._model = model  # the state reads the model: keep it alive
        self._handle = handle
        ms = model._struct()
        self.n, self.m = int(ms.Q.ncol), int(ms.A.nrow)
        self.q_nnz, self.a_nnz = int(ms.Q.nnz), int(ms.A.nnz)

    def backward(self, grad_x, grad_y=None, tol: float = 1e-12, max_iter: int = 0) -> dict:
        gx = np.ascontiguousarray(np.broadcast_to(np.asarray(grad_x, np.float64), (self.n,)))
        gy = None if grad_y is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(grad_y, np.float64), (self.m,)))
        out = {k: np.zeros(max(v, 1)) for k, v in (("dc", self.n), ("dl", self.n), ("du", self.n), ("dAL", self.m),
                                                   ("dAU", self.m), ("dQ_values", self.q_nnz),
                                                   ("dA_values", self.a_nnz), ("lam", self.n), ("mu", self.m))}
        g = _GradientsStruct(**{k: v.ctypes.data_as(c_double_p) for k, v in out.items()})
        gxp = (gx if self.n else np.zeros(1)).ctypes.data_as(c_double_p)
        gyp = None if gy is None else (gy if self.m else np.zeros(1)).ctypes.data_as(c_double_p)
        _raise_for_status(_lib().hprqp_backward(self._handle, gxp, gyp, float(tol), int(max_iter), ctypes.byref(g)),
                          "hprqp_backward")
        sizes = {"dc": self.n, "dl": self.n, "du": self.n, "dAL": self.m, "dAU": self.m, "dQ_values": self.q_nnz,
                 "dA_values": self.a_nnz, "lam": self.n, "mu": self.m}
        res = {k: out[k][:sizes[k]] for k in out}
        res.update(minres_iters=int(g.minres_iters), minres_relres=float(g.minres_relres),
                   backward_seconds=float(g.backward_seconds))
        return res

    def close(self) -> None:
        h = getattr(self, "_handle", None)
        if h is not None and h.value and _Library._instance is not None:
            _Library._instance.hprqp_solve_state_destroy(h)
            h.value = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_for_backward(model: Model, params: Optional[Parameters] = None):
    """``optimize`` that keeps the solve's device state for the adjoint:
    returns ``(Result, SolveState or None)`` (include/hprqp_diff.h)."""
    if params is None:
        params = Parameters()
    lib = _lib()
    results_handle = ctypes.c_void_p()
    _raise_for_status(lib.hprqp_results_create(ctypes.byref(results_handle)), "hprqp_results_create")
    state = ctypes.c_void_p()
    try:
        code = int(lib.hprqp_solve_for_backward(model._handle, params._handle, results_handle, ctypes.byref(state)))
        r = ctypes.cast(results_handle, ctypes.POINTER(_ResultsStruct)).contents
        n, m = model.num_variables, model.num_constraints

        def vec(ptr, k):
            return np.ctypeslib.as_array(ptr, shape=(k,)).copy() if (ptr and k) else np.zeros(0)

        res = Result(status_code=code, status=status_name(code), iter=int(r.iter), iter_4=int(r.iter_4),
                     iter_6=int(r.iter_6), time=float(r.time), time_4=float(r.time_4), time_6=float(r.time_6),
                     objective=float(r.primal_obj), residual=float(r.residuals), gap=float(r.gap),
                     x=vec(r.x, n), y=vec(r.y, m), z=vec(r.z, n), w=vec(r.w, n))
    finally:
        lib.hprqp_results_destroy(results_handle)
    return res, (SolveState(model, state) if state.value else None)


def spmv(indptr, indices, data, ncol: int, x, reps: int = 1):
    """y = M x on the GPU with the engine's row-block kernel.
    Returns (y, mean_ms_per_product)."""
    keep = []
    ip, ipp = _ptr_sz(np.asarray(indptr))
    ii, iip = _ptr_sz(np.asarray(indices))
    dd, ddp = _ptr_db(np.asarray(data))
    xx, xxp = _ptr_db(np.asarray(x, dtype=np.float64))
    nrow = len(indptr) - 1
    y = np.zeros(max(nrow, 1))
    ms = ctypes.c_double(0.0)
    st = _lib().hprqp_b200_spmv(nrow, int(ncol), int(indptr[-1]), ipp, iip, ddp, xxp, y.ctypes.data_as(c_double_p),
                                int(reps), ctypes.byref(ms))
    _raise_for_status(st, "hprqp_b200_spmv")
    return y[:nrow], ms.value


def gather_bound(indptr, indices, data, ncol: int, x, reps: int = 1):
    """The floor of any CSR product with this sparsity pattern
    (hprqp_b200_gather_bound): every index and value streamed and every
    x[col] gathered, no row structure.  Returns (sum of all products,
    mean_ms_per_pass)."""
    ip, ipp = _ptr_sz(np.asarray(indptr))
    ii, iip = _ptr_sz(np.asarray(indices))
    dd, ddp = _ptr_db(np.asarray(data))
    xx, xxp = _ptr_db(np.asarray(x, dtype=np.float64))
    ms = ctypes.c_double(0.0)
    total = ctypes.c_double(0.0)
    st = _lib().hprqp_b200_gather_bound(len(indptr) - 1, int(ncol), int(indptr[-1]), ipp, iip, ddp, xxp, int(reps),
                                        ctypes.byref(ms), ctypes.byref(total))
    _raise_for_status(st, "hprqp_b200_gather_bound")
    return total.value, ms.value


def setup_info(model: Model, params: Optional[Parameters] = None, dump: bool = False):
    """Engine setup of a built model: sigma0, lambda_max(AA'), lambda_max(Q),
    Q_is_diag, noC, norms and (dump=True) the scaled arrays."""
    if params is None:
        params = Parameters(verbose=False)
    ms = model._struct()
    n, m = int(ms.Q.ncol), int(ms.A.nrow)
    out = np.zeros(9)
    arrays = {}
    ptrs = []
    if dump:
        sizes = dict(row_norm=m, col_norm=n, q_val=int(ms.Q.nnz), a_val=int(ms.A.nnz), at_val=int(ms.A.nnz),
                     c=n, l=n, u=n, AL=m, AU=m)
        for k, sz in sizes.items():
            arrays[k] = np.zeros(max(sz, 1))
            ptrs.append(arrays[k].ctypes.data_as(c_double_p))
    else:
        ptrs = [None] * 10
    st = _lib().hprqp_b200_setup(ctypes.byref(ms), ctypes.byref(params._struct()), out.ctypes.data_as(c_double_p),
                                 *ptrs)
    _raise_for_status(st, "hprqp_b200_setup")
    info = dict(sigma=out[0], lambda_max_A=out[1], lambda_max_Q=out[2], Q_is_diag=int(out[3]), noC=int(out[4]),
                norm_b_org=out[5], norm_c_org=out[6], norm_b=out[7], norm_c=out[8])
    if dump:
        for k, sz in dict(row_norm=m, col_norm=n, q_val=int(ms.Q.nnz), a_val=int(ms.A.nnz), at_val=int(ms.A.nnz),
                          c=n, l=n, u=n, AL=m, AU=m).items():
            info[k] = arrays[k][:sz]
    return info


def model_arrays(model: Model):
    """Copy of the preprocessed model held by the library (CSR as int64)."""
    ms = model._struct()
    n, m = int(ms.Q.ncol), int(ms.A.nrow)

    def csr(c):
        nr, nnz = int(c.nrow), int(c.nnz)
        ip = np.ctypeslib.as_array(c.row_ptr, shape=(nr + 1,)).astype(np.int64)
        ii = np.ctypeslib.as_array(c.col_ind, shape=(nnz,)).astype(np.int64) if nnz else np.zeros(0, np.int64)
        dv = np.ctypeslib.as_array(c.values, shape=(nnz,)).copy() if nnz else np.zeros(0)
        return ip, ii, dv

    def vec(p, k):
        return np.ctypeslib.as_array(p, shape=(k,)).copy() if (p and k) else np.zeros(0)

    q = csr(ms.Q)
    a = csr(ms.A)
    nrc = int(ms.num_row_cones)
    return dict(n=n, m=m, q_indptr=q[0], q_indices=q[1], q_data=q[2], a_indptr=a[0], a_indices=a[1], a_data=a[2],
                c=vec(ms.c, n), l=vec(ms.l, n), u=vec(ms.u, n), AL=vec(ms.AL, m), AU=vec(ms.AU, m),
                obj_constant=float(ms.obj_constant), num_var_cones=int(ms.num_var_cones), num_row_cones=nrc,
                row_cone_offsets=(np.ctypeslib.as_array(ms.row_cone_offsets, shape=(nrc + 1,)).astype(np.int64)
                                  if nrc else np.zeros(0, np.int64)),
                soc_rhs=vec(ms.soc_rhs, m) if nrc else np.zeros(0))


def __getattr__(name):
    """``hprqp.QPFunction`` / ``hprqp.QPLayer`` (batched) and
    ``hprqp.SingleQPFunction`` (one large QP): the differentiable layers,
    imported on first use so that torch stays optional; the CVXPY bridge
    (``build_from_cvxpy_problem``, ``solve_cvxpy_problem``), likewise."""
    if name in ("QPFunction", "QPLayer", "SingleQPFunction"):
        from . import torch_layer

        return getattr(torch_layer, name)
    if name in ("CVXPYBuildInfo", "build_from_cvxpy_problem", "solve_cvxpy_problem"):
        from . import cvxpy_bridge

        return getattr(cvxpy_bridge, name)
    raise AttributeError(f"module 'hprqp' has no attribute {name!r}")


__all__ = [
    "CVXPYBuildInfo", "build_from_cvxpy_problem", "solve_cvxpy_problem",
    "QPFunction", "QPLayer", "SingleQPFunction", "SolveState", "residuals", "solve_for_backward", "Model", "Parameters", "Result", "SPMV_MODE_AUTO", "SPMV_MODE_CUSPARSE", "SPMV_MODE_CUSTOMIZED",
    "STATUS_ALLOCATION_FAILED", "STATUS_CONTINUE", "STATUS_INVALID_ARGUMENT", "STATUS_MAX_ITER",
    "STATUS_NOT_IMPLEMENTED", "STATUS_OK", "STATUS_OPTIMAL", "STATUS_TIME_LIMIT", "build_from_mps",
    "build_from_QAbc", "build_from_qabc", "build_from_qabc_soc", "build_from_instance", "gpu_backend_available", "optimize",
    "read_from_mps", "status_name", "spmv", "gather_bound", "build_from_qabc_qc", "setup_info", "model_arrays", "launch_count", "library_path",
]
