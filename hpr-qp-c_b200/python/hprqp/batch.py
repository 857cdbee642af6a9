"""Batched solves (hprqp_batch.h): many independent QPs in one persistent
kernel, each to its own tolerance with its own sigma and restarts."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _MatrixCSR, _lib, _raise_for_status, c_double_p, c_size_p

_configured = False


class BatchGradients(ctypes.Structure):
    _fields_ = [(name, ctypes.POINTER(ctypes.c_double)) for name in ("dc", "dl", "du", "dAL", "dAU", "dQ_values",
                                                                     "dA_values")] + \
               [("minres_iters", ctypes.POINTER(ctypes.c_int)), ("minres_relres", ctypes.POINTER(ctypes.c_double))]


class BatchParams(ctypes.Structure):
    _fields_ = [("stoptol", ctypes.c_double), ("max_iter", ctypes.c_size_t), ("time_limit", ctypes.c_double),
                ("check_iter", ctypes.c_size_t), ("print_frequency", ctypes.c_int), ("use_scaling", ctypes.c_int),
                ("device_number", ctypes.c_int), ("verbose", ctypes.c_int)]


def _configure():
    global _configured
    if _configured:
        return
    lib = _lib()
    vp = ctypes.c_void_p
    lib.hprqp_batch_params_set_defaults.argtypes = [ctypes.POINTER(BatchParams)]
    lib.hprqp_batch_params_set_defaults.restype = None
    lib.hprqp_batch_create.argtypes = [ctypes.c_size_t, c_size_p, c_size_p, ctypes.POINTER(_MatrixCSR),
                                       ctypes.POINTER(_MatrixCSR), c_double_p, c_double_p, c_double_p, c_double_p,
                                       c_double_p, c_double_p, ctypes.c_int, ctypes.POINTER(vp)]
    lib.hprqp_batch_solve.argtypes = [vp, ctypes.POINTER(BatchParams)]
    lib.hprqp_batch_set_warm_start.argtypes = [vp, c_double_p, c_double_p, c_double_p, c_double_p]
    lib.hprqp_batch_get_sigma.argtypes = [vp, c_double_p]
    lib.hprqp_batch_get_times.argtypes = [vp, c_double_p]
    lib.hprqp_batch_last_solve_ms.argtypes = [vp]
    lib.hprqp_batch_last_solve_ms.restype = ctypes.c_double
    lib.hprqp_batch_get_results.argtypes = [vp, ctypes.POINTER(ctypes.c_int), c_size_p, c_double_p, c_double_p,
                                            c_double_p, c_double_p, c_double_p, c_double_p, c_double_p]
    lib.hprqp_batch_backward.argtypes = [vp, c_double_p, c_double_p, ctypes.c_double,
                                         ctypes.POINTER(BatchGradients)]
    lib.hprqp_batch_last_backward_ms.argtypes = [vp]
    lib.hprqp_batch_last_backward_ms.restype = ctypes.c_double
    lib.hprqp_batch_destroy.argtypes = [vp]
    lib.hprqp_batch_destroy.restype = None
    lib.hprqp_batch_set_spmv_lanes.argtypes = [vp, ctypes.c_int]
    lib.hprqp_batch_request_abort.argtypes = [vp]
    lib.hprqp_batch_get_spmv_lanes.argtypes = [vp, ctypes.POINTER(ctypes.c_int)]
    _configured = True


def default_params(**kw) -> BatchParams:
    _configure()
    p = BatchParams()
    _lib().hprqp_batch_params_set_defaults(ctypes.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@dataclass
class Packed:
    """A list of QPs packed as one block-diagonal problem (host arrays)."""
    var_offsets: np.ndarray
    row_offsets: np.ndarray
    q_indptr: np.ndarray
    q_indices: np.ndarray
    q_data: np.ndarray
    a_indptr: np.ndarray
    a_indices: np.ndarray
    a_data: np.ndarray
    c: np.ndarray
    AL: np.ndarray
    AU: np.ndarray
    l: np.ndarray
    u: np.ndarray
    obj: np.ndarray

    @property
    def K(self) -> int:
        return len(self.var_offsets) - 1

    @property
    def nbytes(self) -> int:
        return int(sum(a.nbytes for a in (self.q_indptr, self.q_indices, self.q_data, self.a_indptr,
                                          self.a_indices, self.a_data, self.c, self.AL, self.AU, self.l, self.u)))


def pack(instances: Sequence) -> Packed:
    K = len(instances)
    var_off = np.zeros(K + 1, np.uint64)
    row_off = np.zeros(K + 1, np.uint64)
    var_off[1:] = np.cumsum([i.n for i in instances])
    row_off[1:] = np.cumsum([i.m for i in instances])
    q_ptr = [np.zeros(1, np.int64)]
    a_ptr = [np.zeros(1, np.int64)]
    qnz = anz = 0
    for inst in instances:
        q_ptr.append(np.asarray(inst.Q.indptr[1:], np.int64) + qnz)
        a_ptr.append(np.asarray(inst.A.indptr[1:], np.int64) + anz)
        qnz += inst.Q.nnz
        anz += inst.A.nnz
    q_idx = np.concatenate([np.asarray(i.Q.indices, np.int64) + int(var_off[k]) for k, i in enumerate(instances)])
    a_idx = np.concatenate([np.asarray(i.A.indices, np.int64) + int(var_off[k]) for k, i in enumerate(instances)])
    return Packed(var_off, row_off,
                  np.concatenate(q_ptr).astype(np.uint64), q_idx.astype(np.uint64),
                  np.concatenate([i.Q.data for i in instances]).astype(np.float64),
                  np.concatenate(a_ptr).astype(np.uint64), a_idx.astype(np.uint64),
                  np.concatenate([i.A.data for i in instances]).astype(np.float64),
                  np.concatenate([i.c for i in instances]).astype(np.float64),
                  np.concatenate([i.AL for i in instances]).astype(np.float64),
                  np.concatenate([i.AU for i in instances]).astype(np.float64),
                  np.concatenate([i.l for i in instances]).astype(np.float64),
                  np.concatenate([i.u for i in instances]).astype(np.float64),
                  np.array([i.obj_constant for i in instances], np.float64))


def _csr(nrow, ncol, indptr, indices, data, keep):
    ip = np.ascontiguousarray(indptr, np.uint64)
    ii = np.ascontiguousarray(indices if len(indices) else np.zeros(1), np.uint64)
    dd = np.ascontiguousarray(data if len(data) else np.zeros(1), np.float64)
    keep += [ip, ii, dd]
    return _MatrixCSR(nrow, ncol, int(ip[-1]), ip.ctypes.data_as(c_size_p), ii.ctypes.data_as(c_size_p),
                      dd.ctypes.data_as(c_double_p), 0)


@dataclass
class BatchResult:
    status: np.ndarray
    iter: np.ndarray
    objective: np.ndarray
    residual: np.ndarray
    gap: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    w: np.ndarray
    solve_ms: float
    sigma: Optional[np.ndarray] = None  # per instance, at the end of the solve
    seconds: Optional[np.ndarray] = None  # per instance, its own time on its CTA


@dataclass
class Gradients:
    """dL/d(problem data) from hprqp_batch_backward, packed like the inputs
    (dQ / dA: one value per nonzero of the caller's Q / A)."""
    dc: np.ndarray
    dl: np.ndarray
    du: np.ndarray
    dAL: np.ndarray
    dAU: np.ndarray
    dQ: np.ndarray
    dA: np.ndarray
    minres_iters: np.ndarray
    minres_relres: np.ndarray
    backward_ms: float


class Batch:
    """Device-resident batch: create once, solve many times."""

    def __init__(self, instances_or_packed, device_number: int = 0):
        _configure()
        p = instances_or_packed if isinstance(instances_or_packed, Packed) else pack(instances_or_packed)
        self.packed = p
        keep = []
        # matrix sizes from the arrays themselves (a C caller cannot be
        # checked against array lengths): the library then rejects offsets
        # that do not match them
        n = len(p.q_indptr) - 1
        m = len(p.a_indptr) - 1
        Q = _csr(n, n, p.q_indptr, p.q_indices, p.q_data, keep)
        A = _csr(m, n, p.a_indptr, p.a_indices, p.a_data, keep)

        def db(a):
            a = np.ascontiguousarray(a if len(a) else np.zeros(1), np.float64)
            keep.append(a)
            return a.ctypes.data_as(c_double_p)

        vo = np.ascontiguousarray(p.var_offsets, np.uint64)
        ro = np.ascontiguousarray(p.row_offsets, np.uint64)
        keep += [vo, ro]
        handle = ctypes.c_void_p()
        st = _lib().hprqp_batch_create(p.K, vo.ctypes.data_as(c_size_p), ro.ctypes.data_as(c_size_p),
                                       ctypes.byref(Q), ctypes.byref(A), db(p.c), db(p.AL), db(p.AU), db(p.l),
                                       db(p.u), db(p.obj), int(device_number), ctypes.byref(handle))
        _raise_for_status(st, "hprqp_batch_create")
        self._handle = handle
        self.n, self.m, self.K = n, m, p.K

    def set_warm_start(self, x0=None, y0=None, w0=None, sigma0=None):
        """Start the following solves at (x0, y0, w0) -- e.g. the x, y, w of
        a solve of a nearby batch -- instead of zero, optionally with that
        solve's per-instance sigma (:attr:`BatchResult.sigma`); ``x0=None``
        clears it (hprqp_batch_set_warm_start)."""
        if x0 is None:
            _raise_for_status(_lib().hprqp_batch_set_warm_start(self._handle, None, None, None, None),
                              "hprqp_batch_set_warm_start")
            return

        def vec(a, size, name):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.float64).reshape(-1)
            if a.shape[0] != size:
                raise ValueError(f"warm start {name}: expected {size} entries, got {a.shape[0]}")
            return a if size else np.zeros(1)

        x = vec(x0, self.n, "x0")
        y = vec(y0, self.m, "y0")
        w = vec(w0, self.n, "w0")
        sg = vec(sigma0, self.K, "sigma0")
        ptr = (lambda a: None if a is None else a.ctypes.data_as(c_double_p))
        _raise_for_status(_lib().hprqp_batch_set_warm_start(self._handle, ptr(x), ptr(y), ptr(w), ptr(sg)),
                          "hprqp_batch_set_warm_start")

    def request_abort(self):
        """Stop the solve running on this batch in another thread
        (hprqp_batch_request_abort): unfinished instances end with
        TIME_LIMIT (5)."""
        _raise_for_status(_lib().hprqp_batch_request_abort(self._handle), "hprqp_batch_request_abort")

    def spmv_lanes(self) -> np.ndarray:
        """SpMV lane-group width of every matrix, shape (K, 3): Q, A, A'
        (hprqp_batch_get_spmv_lanes)."""
        out = np.zeros(3 * max(self.K, 1), np.int32)
        _raise_for_status(_lib().hprqp_batch_get_spmv_lanes(self._handle,
                                                             out.ctypes.data_as(ctypes.POINTER(ctypes.c_int))),
                          "hprqp_batch_get_spmv_lanes")
        return out[:3 * self.K].reshape(self.K, 3)

    def set_spmv_lanes(self, lanes: int = 0):
        """Force one SpMV lane-group width (1, 2, 4, 8, 16, 32) on every
        matrix; 0 restores the autotuned widths (hprqp_batch_set_spmv_lanes)."""
        _raise_for_status(_lib().hprqp_batch_set_spmv_lanes(self._handle, int(lanes)), "hprqp_batch_set_spmv_lanes")

    def solve(self, **kw) -> float:
        params = default_params(**kw)
        _raise_for_status(_lib().hprqp_batch_solve(self._handle, ctypes.byref(params)), "hprqp_batch_solve")
        return float(_lib().hprqp_batch_last_solve_ms(self._handle))

    def results(self, vectors: bool = True) -> BatchResult:
        K = self.K
        status = np.zeros(K, np.int32)
        it = np.zeros(K, np.uint64)
        obj = np.zeros(K)
        res = np.zeros(K)
        gap = np.zeros(K)
        x = np.zeros(max(self.n, 1))
        z = np.zeros(max(self.n, 1))
        w = np.zeros(max(self.n, 1))
        y = np.zeros(max(self.m, 1))
        vec = (lambda a: a.ctypes.data_as(c_double_p)) if vectors else (lambda a: None)
        st = _lib().hprqp_batch_get_results(self._handle, status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                            it.ctypes.data_as(c_size_p), obj.ctypes.data_as(c_double_p),
                                            res.ctypes.data_as(c_double_p), gap.ctypes.data_as(c_double_p),
                                            vec(x), vec(y), vec(z), vec(w))
        _raise_for_status(st, "hprqp_batch_get_results")
        sigma = np.zeros(K)
        _raise_for_status(_lib().hprqp_batch_get_sigma(self._handle, sigma.ctypes.data_as(c_double_p)),
                          "hprqp_batch_get_sigma")
        seconds = np.zeros(K)
        _raise_for_status(_lib().hprqp_batch_get_times(self._handle, seconds.ctypes.data_as(c_double_p)),
                          "hprqp_batch_get_times")
        return BatchResult(status, it.astype(np.int64), obj, res, gap, x[:self.n], y[:self.m], z[:self.n],
                           w[:self.n], float(_lib().hprqp_batch_last_solve_ms(self._handle)), sigma, seconds)

    def backward(self, grad_x, grad_y=None, tol: float = 1e-12) -> Gradients:
        """Implicit-differentiation adjoint of the last solve (one MINRES
        solve per instance on the device); see hprqp_batch_backward."""
        gx = np.ascontiguousarray(np.broadcast_to(np.asarray(grad_x, np.float64), (self.n,)))
        gy = None if grad_y is None else np.ascontiguousarray(np.broadcast_to(np.asarray(grad_y, np.float64),
                                                                               (self.m,)))
        p = self.packed
        n1, m1 = max(self.n, 1), max(self.m, 1)
        out = {k: np.zeros(v) for k, v in (("dc", n1), ("dl", n1), ("du", n1), ("dAL", m1), ("dAU", m1),
                                           ("dQ_values", max(len(p.q_data), 1)),
                                           ("dA_values", max(len(p.a_data), 1)))}
        its = np.zeros(self.K, np.int32)
        rel = np.zeros(self.K)
        g = BatchGradients(**{k: v.ctypes.data_as(c_double_p) for k, v in out.items()},
                           minres_iters=its.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                           minres_relres=rel.ctypes.data_as(c_double_p))
        gx_buf = gx if self.n else np.zeros(1)
        gy_buf = None if gy is None else (gy if self.m else np.zeros(1))
        st = _lib().hprqp_batch_backward(self._handle, gx_buf.ctypes.data_as(c_double_p),
                                         None if gy_buf is None else gy_buf.ctypes.data_as(c_double_p),
                                         float(tol), ctypes.byref(g))
        _raise_for_status(st, "hprqp_batch_backward")
        return Gradients(out["dc"][:self.n], out["dl"][:self.n], out["du"][:self.n], out["dAL"][:self.m],
                         out["dAU"][:self.m], out["dQ_values"][:len(p.q_data)], out["dA_values"][:len(p.a_data)],
                         its, rel, float(_lib().hprqp_batch_last_backward_ms(self._handle)))

    def split(self, vec: np.ndarray, kind: str) -> List[np.ndarray]:
        off = self.packed.var_offsets if kind == "x" else self.packed.row_offsets
        return [vec[int(off[k]):int(off[k + 1])] for k in range(self.K)]

    def close(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            _lib().hprqp_batch_destroy(h)
            h.value = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch(instances, **kw) -> BatchResult:
    b = Batch(instances, device_number=kw.pop("device_number", 0))
    try:
        b.solve(**kw)
        return b.results()
    finally:
        b.close()
