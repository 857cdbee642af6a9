"""ctypes access to the CPU checkers (test infrastructure only).

* ``liboracle.so``: this project's serial C restatement of the reference
  algorithm (oracle/hprqp_oracle.c), built by ``make -C oracle``.
* ``_ref/libhprqp_ref_cpu.so``: the reference's own CPU backend compiled from
  its sources by ``make -C oracle ref`` (only possible where the reference
  sources exist; the built library travels with the repository snapshot).
* ``_ref/libhprqp_ref_gpu.so``: the reference's own CUDA backend
  (cuSPARSE/cuBLAS), ``make -C oracle ref-gpu``; called through its C API
  (``solve_gpu``) with polishing and the Gram path off.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "lib" / "liboracle.so"
REF_CPU_LIB = HERE / "_ref" / "libhprqp_ref_cpu.so"
REF_GPU_LIB = HERE / "_ref" / "libhprqp_ref_gpu.so"

MODE_GPU_REF = 0
MODE_CPU_REF = 1

c_size_p = ctypes.POINTER(ctypes.c_size_t)
c_double_p = ctypes.POINTER(ctypes.c_double)


class _OracleResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("iter", ctypes.c_size_t),
        ("iter_4", ctypes.c_size_t),
        ("iter_6", ctypes.c_size_t),
        ("primal_obj", ctypes.c_double),
        ("residuals", ctypes.c_double),
        ("gap", ctypes.c_double),
        ("err_rp", ctypes.c_double),
        ("err_rd", ctypes.c_double),
        ("dual_obj", ctypes.c_double),
        ("sigma", ctypes.c_double),
        ("lambda_max_A", ctypes.c_double),
        ("lambda_max_Q", ctypes.c_double),
        ("Q_is_diag", ctypes.c_int),
        ("noC", ctypes.c_int),
        ("restarts", ctypes.c_size_t),
        ("time", ctypes.c_double),
    ]


class _OracleParams(ctypes.Structure):
    _fields_ = [
        ("stoptol", ctypes.c_double),
        ("max_iter", ctypes.c_size_t),
        ("time_limit", ctypes.c_double),
        ("check_iter", ctypes.c_size_t),
        ("print_frequency", ctypes.c_int),
        ("use_scaling", ctypes.c_int),
        ("mode", ctypes.c_int),
    ]


_lib: Optional[ctypes.CDLL] = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build_oracle()
        _lib = ctypes.CDLL(str(ORACLE_LIB))
        _lib.oracle_build.restype = ctypes.c_int
        _lib.oracle_solve.restype = ctypes.c_int
        _lib.oracle_solve_from.restype = ctypes.c_int
        _lib.oracle_model_n.restype = ctypes.c_size_t
        _lib.oracle_model_m.restype = ctypes.c_size_t
        _lib.oracle_model_q_nnz.restype = ctypes.c_size_t
        _lib.oracle_model_a_nnz.restype = ctypes.c_size_t
        for name in ("oracle_model_n", "oracle_model_m", "oracle_model_q_nnz", "oracle_model_a_nnz",
                     "oracle_model_free"):
            getattr(_lib, name).argtypes = [ctypes.c_void_p]
    return _lib


def _sz(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a, a.ctypes.data_as(c_size_p)


def _db(a: Optional[np.ndarray]):
    if a is None:
        return None, None
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(c_double_p)


class OracleModel:
    """A preprocessed model inside the C oracle."""

    def __init__(self, inst):
        L = lib()
        keep = []

        def sz(a):
            arr, p = _sz(a)
            keep.append(arr)
            return p

        def db(a):
            arr, p = _db(a)
            keep.append(arr)
            return p

        handle = ctypes.c_void_p()
        st = L.oracle_build(
            ctypes.c_size_t(inst.n), ctypes.c_size_t(inst.Q.nnz), sz(inst.Q.indptr), sz(inst.Q.indices),
            db(inst.Q.data), ctypes.c_size_t(inst.m), ctypes.c_size_t(inst.A.nnz), sz(inst.A.indptr),
            sz(inst.A.indices), db(inst.A.data), db(inst.c), db(inst.AL if inst.m else np.zeros(1)),
            db(inst.AU if inst.m else np.zeros(1)), db(inst.l), db(inst.u),
            ctypes.c_double(inst.obj_constant), ctypes.byref(handle))
        if st != 0:
            raise ValueError(f"oracle_build failed with status {st}")
        self.handle = handle
        self.n = int(L.oracle_model_n(handle))
        self.m = int(L.oracle_model_m(handle))

    def __del__(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            lib().oracle_model_free(self.handle)
            self.handle = None

    def export(self):
        L = lib()
        qn = int(L.oracle_model_q_nnz(self.handle))
        an = int(L.oracle_model_a_nnz(self.handle))
        q_rp = np.zeros(self.n + 1, np.uint64)
        q_ci = np.zeros(max(qn, 1), np.uint64)
        q_v = np.zeros(max(qn, 1))
        a_rp = np.zeros(self.m + 1, np.uint64)
        a_ci = np.zeros(max(an, 1), np.uint64)
        a_v = np.zeros(max(an, 1))
        c = np.zeros(self.n)
        l = np.zeros(self.n)
        u = np.zeros(self.n)
        AL = np.zeros(max(self.m, 1))
        AU = np.zeros(max(self.m, 1))
        L.oracle_model_export(self.handle, *[a.ctypes.data_as(c_size_p if a.dtype == np.uint64 else c_double_p)
                                             for a in (q_rp, q_ci, q_v, a_rp, a_ci, a_v, c, AL, AU, l, u)])
        return dict(q_indptr=q_rp.astype(np.int64), q_indices=q_ci[:qn].astype(np.int64), q_data=q_v[:qn],
                    a_indptr=a_rp.astype(np.int64), a_indices=a_ci[:an].astype(np.int64), a_data=a_v[:an],
                    c=c, l=l, u=u, AL=AL[:self.m], AU=AU[:self.m])

    def solve(self, stoptol=1e-8, max_iter=2147483647, time_limit=3600.0, check_iter=100,
              print_frequency=-1, use_scaling=True, mode=MODE_GPU_REF, x0=None, y0=None, w0=None, sigma0=0.0):
        """Solve; with x0 (n), optionally y0 (m rows of the preprocessed
        model), w0 (n) and sigma0 > 0, from that warm start
        (oracle_solve_from)."""
        p = _OracleParams(stoptol, max_iter, time_limit, check_iter, print_frequency, int(use_scaling), mode)
        r = _OracleResult()
        x = np.zeros(max(self.n, 1))
        w = np.zeros(max(self.n, 1))
        z = np.zeros(max(self.n, 1))
        y = np.zeros(max(self.m, 1))

        def start(a, size):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, np.float64).reshape(-1)
            if a.shape[0] != size:
                raise ValueError(f"warm start: expected {size} entries, got {a.shape[0]}")
            a = a if size else np.zeros(1)
            return a, a.ctypes.data_as(c_double_p)

        (xa, xp), (ya, yp), (wa, wp) = start(x0, self.n), start(y0, self.m), start(w0, self.n)
        lib().oracle_solve_from(self.handle, ctypes.byref(p), xp, yp, wp, ctypes.c_double(sigma0), ctypes.byref(r),
                                x.ctypes.data_as(c_double_p), y.ctypes.data_as(c_double_p),
                                z.ctypes.data_as(c_double_p), w.ctypes.data_as(c_double_p))
        out = {name: getattr(r, name) for name, _ in _OracleResult._fields_}
        out.update(x=x[:self.n], y=y[:self.m], z=z[:self.n], w=w[:self.n])
        return out

    def setup(self, use_scaling=True, mode=MODE_GPU_REF):
        out = np.zeros(5)
        st = lib().oracle_setup(self.handle, int(use_scaling), mode, out.ctypes.data_as(c_double_p))
        if st != 0:
            raise ValueError(st)
        return dict(sigma=out[0], lambda_max_A=out[1], lambda_max_Q=out[2], Q_is_diag=int(out[3]), noC=int(out[4]))

    def scale(self, use_scaling=True, mode=MODE_GPU_REF):
        L = lib()
        qn = int(L.oracle_model_q_nnz(self.handle))
        an = int(L.oracle_model_a_nnz(self.handle))
        arrs = dict(row_norm=np.zeros(max(self.m, 1)), col_norm=np.zeros(max(self.n, 1)),
                    q_data=np.zeros(max(qn, 1)), a_data=np.zeros(max(an, 1)), c=np.zeros(max(self.n, 1)),
                    l=np.zeros(max(self.n, 1)), u=np.zeros(max(self.n, 1)), AL=np.zeros(max(self.m, 1)),
                    AU=np.zeros(max(self.m, 1)), scalars=np.zeros(4))
        st = L.oracle_scale(self.handle, int(use_scaling), mode,
                            *[arrs[k].ctypes.data_as(c_double_p) for k in
                              ("row_norm", "col_norm", "q_data", "a_data", "c", "l", "u", "AL", "AU", "scalars")])
        if st != 0:
            raise ValueError(st)
        arrs["row_norm"] = arrs["row_norm"][:self.m]
        arrs["AL"] = arrs["AL"][:self.m]
        arrs["AU"] = arrs["AU"][:self.m]
        arrs["q_data"] = arrs["q_data"][:qn]
        arrs["a_data"] = arrs["a_data"][:an]
        return arrs

    def kkt(self, x, y, z):
        out = np.zeros(6)
        xa, xp = _db(x)
        ya, yp = _db(y if self.m else np.zeros(1))
        za, zp = _db(z)
        lib().oracle_kkt(self.handle, xp, yp, zp, out.ctypes.data_as(c_double_p))
        return dict(err_rp=out[0], err_rd=out[1], gap=out[2], primal_obj=out[3], dual_obj=out[4], kkt=out[5])


def kkt_adjoint_dense(inst, x, y, z, grad_x, grad_y=None):
    """Dense FP64 implicit-differentiation adjoint of a QP solution.

    The reference (PolyU-IOR/HPR-QP-C) has no adjoint; this is the checker
    for the device MINRES adjoint.  Its sign conventions are the reference's
    KKT conditions (src/gpu/residuals.cu: Qx + c - A'y - z = 0, y_r > 0 at the
    lower row bound, z_i > 0 at the lower variable bound).  Active sets:
    F = {i : z_i == 0}, R = {r : y_r != 0}.  Solves
    [[Q_FF, A_RF'], [A_RF, 0]] [lam_F; mu_R] = [g_F; -gy_R] with numpy's
    dense solver (least squares when singular) and returns every gradient.
    ``y``/``grad_y`` cover all of the instance's rows (removed rows: y = 0).
    """
    Q = inst.Q.dense()
    Q = 0.5 * (Q + Q.T)
    A = inst.A.dense()
    n, m = Q.shape[0], A.shape[0]
    x, y, z = (np.asarray(v, np.float64) for v in (x, y, z))
    gx = np.asarray(grad_x, np.float64)
    gy = np.zeros(m) if grad_y is None else np.asarray(grad_y, np.float64)
    F = np.nonzero(z == 0.0)[0]
    R = np.nonzero(y != 0.0)[0]
    nf, nr = len(F), len(R)
    K = np.zeros((nf + nr, nf + nr))
    K[:nf, :nf] = Q[np.ix_(F, F)]
    K[:nf, nf:] = A[np.ix_(R, F)].T
    K[nf:, :nf] = A[np.ix_(R, F)]
    rhs = np.concatenate([gx[F], -gy[R]])
    try:
        sol = np.linalg.solve(K, rhs)
    except np.linalg.LinAlgError:
        sol = np.linalg.lstsq(K, rhs, rcond=None)[0]
    lam = np.zeros(n)
    mu = np.zeros(m)
    lam[F] = sol[:nf]
    mu[R] = sol[nf:]
    db = gx - Q @ lam - A.T @ mu
    qi, qj = _coo(inst.Q)
    ai, aj = _coo(inst.A)
    return dict(lam=lam, mu=mu, dc=-lam, dl=np.where(z > 0.0, db, 0.0), du=np.where(z < 0.0, db, 0.0),
                dAL=np.where(y > 0.0, mu, 0.0), dAU=np.where(y < 0.0, mu, 0.0),
                dQ=-0.5 * (lam[qi] * x[qj] + lam[qj] * x[qi]), dA=-mu[ai] * x[aj] + lam[aj] * y[ai])


def _coo(csr):
    indptr = np.asarray(csr.indptr, np.int64)
    rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    return rows, np.asarray(csr.indices, np.int64)


def matvec(indptr, indices, data, x):
    indptr_a, ip = _sz(indptr)
    indices_a, ii = _sz(indices if len(indices) else np.zeros(1))
    data_a, dp = _db(data if len(data) else np.zeros(1))
    xa, xp = _db(x if len(x) else np.zeros(1))
    nrow = len(indptr) - 1
    y = np.zeros(max(nrow, 1))
    lib().oracle_csr_matvec(ctypes.c_size_t(nrow), ip, ii, dp, xp, y.ctypes.data_as(c_double_p))
    return y[:nrow]


# --------------------------------------------------------------------------
# the reference's own CPU library (oracle/_ref), through its hprqp_* ABI
# --------------------------------------------------------------------------

_ref: Optional[ctypes.CDLL] = None


def ref_available() -> bool:
    return REF_CPU_LIB.exists()


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(str(REF_CPU_LIB))
        _ref.hprqp_status_name.restype = ctypes.c_char_p
        for name in ("hprqp_results_x_data", "hprqp_results_y_data", "hprqp_results_z_data",
                     "hprqp_results_w_data"):
            getattr(_ref, name).restype = c_double_p
            getattr(_ref, name).argtypes = [ctypes.c_void_p]
        for name in ("hprqp_results_iter", "hprqp_results_iter_4", "hprqp_results_iter_6",
                     "hprqp_results_num_variables", "hprqp_results_num_constraints"):
            getattr(_ref, name).restype = ctypes.c_size_t
            getattr(_ref, name).argtypes = [ctypes.c_void_p]
        for name in ("hprqp_results_time", "hprqp_results_objective", "hprqp_results_residual",
                     "hprqp_results_gap"):
            getattr(_ref, name).restype = ctypes.c_double
            getattr(_ref, name).argtypes = [ctypes.c_void_p]
        _ref.hprqp_params_set_stoptol.argtypes = [ctypes.c_void_p, ctypes.c_double]
        _ref.hprqp_params_set_time_limit.argtypes = [ctypes.c_void_p, ctypes.c_double]
        for name in ("hprqp_params_set_max_iter", "hprqp_params_set_check_iter"):
            getattr(_ref, name).argtypes = [ctypes.c_void_p, ctypes.c_size_t]
        for name in ("hprqp_params_set_use_gpu", "hprqp_params_set_verbose", "hprqp_params_set_use_scaling",
                     "hprqp_params_set_print_frequency"):
            getattr(_ref, name).argtypes = [ctypes.c_void_p, ctypes.c_int]
        _ref.hprqp_optimize.argtypes = [ctypes.c_void_p] * 3
    return _ref


def ref_solve(inst, stoptol=1e-8, max_iter=2147483647, use_scaling=True, check_iter=100,
              print_frequency=-1, time_limit=3600.0):
    """Solve with the reference CPU library (use_gpu=0, polishing off)."""
    L = ref_lib()
    keep = []

    def sz(a):
        arr, p = _sz(a if len(a) else np.zeros(1))
        keep.append(arr)
        return p

    def db(a):
        arr, p = _db(a if len(a) else np.zeros(1))
        keep.append(arr)
        return p

    model = ctypes.c_void_p()
    params = ctypes.c_void_p()
    res = ctypes.c_void_p()
    L.hprqp_model_create(ctypes.byref(model))
    st = L.hprqp_model_build_from_qabc_csr(
        model, ctypes.c_size_t(inst.n), ctypes.c_size_t(inst.n), ctypes.c_size_t(inst.Q.nnz), sz(inst.Q.indptr),
        sz(inst.Q.indices), db(inst.Q.data), ctypes.c_size_t(inst.m), ctypes.c_size_t(inst.n),
        ctypes.c_size_t(inst.A.nnz), sz(inst.A.indptr), sz(inst.A.indices), db(inst.A.data), db(inst.c),
        db(inst.AL) if inst.m else None, db(inst.AU) if inst.m else None, db(inst.l), db(inst.u),
        ctypes.c_double(inst.obj_constant))
    if st != 0:
        L.hprqp_model_destroy(model)
        raise ValueError(f"reference build failed: {st}")
    L.hprqp_params_create(ctypes.byref(params))
    L.hprqp_params_set_use_gpu(params, 0)
    L.hprqp_params_set_verbose(params, 0)
    L.hprqp_params_set_stoptol(params, stoptol)
    L.hprqp_params_set_max_iter(params, max_iter)
    L.hprqp_params_set_use_scaling(params, int(use_scaling))
    L.hprqp_params_set_check_iter(params, check_iter)
    L.hprqp_params_set_print_frequency(params, print_frequency)
    L.hprqp_params_set_time_limit(params, time_limit)
    L.hprqp_results_create(ctypes.byref(res))
    status = L.hprqp_optimize(model, params, res)
    n = int(L.hprqp_results_num_variables(res))
    m = int(L.hprqp_results_num_constraints(res))

    def vec(fn, k):
        p = fn(res)
        return np.array([p[i] for i in range(k)]) if (p and k) else np.zeros(0)

    out = dict(status=status, iter=int(L.hprqp_results_iter(res)), iter_4=int(L.hprqp_results_iter_4(res)),
               iter_6=int(L.hprqp_results_iter_6(res)), primal_obj=L.hprqp_results_objective(res),
               residuals=L.hprqp_results_residual(res), gap=L.hprqp_results_gap(res),
               time=L.hprqp_results_time(res),
               x=vec(L.hprqp_results_x_data, n), y=vec(L.hprqp_results_y_data, m),
               z=vec(L.hprqp_results_z_data, n), w=vec(L.hprqp_results_w_data, n))
    L.hprqp_results_destroy(res)
    L.hprqp_params_destroy(params)
    L.hprqp_model_destroy(model)
    return out


# --------------------------------------------------------------------------
# the reference's own GPU library (oracle/_ref), through its C API
# --------------------------------------------------------------------------
# Struct layouts of the reference's include/shared/types.h:10-214 (an ABI,
# so they must match field for field).

class _RefCSR(ctypes.Structure):
    _fields_ = [("nrow", ctypes.c_size_t), ("ncol", ctypes.c_size_t), ("nnz", ctypes.c_size_t),
                ("row_ptr", c_size_p), ("col_ind", c_size_p), ("values", c_double_p), ("owns_data", ctypes.c_int)]


class _RefModel(ctypes.Structure):
    _fields_ = [("Q", _RefCSR), ("A", _RefCSR), ("AT", _RefCSR), ("c", c_double_p), ("AL", c_double_p),
                ("AU", c_double_p), ("l", c_double_p), ("u", c_double_p), ("obj_constant", ctypes.c_double),
                ("owns_data", ctypes.c_int), ("num_var_cones", ctypes.c_size_t), ("var_cone_offsets", c_size_p),
                ("num_row_cones", ctypes.c_size_t), ("row_cone_offsets", c_size_p), ("soc_rhs", c_double_p)]


class _RefParams(ctypes.Structure):
    _fields_ = [("stoptol", ctypes.c_double), ("max_iter", ctypes.c_size_t), ("use_gpu", ctypes.c_int),
                ("device_number", ctypes.c_int), ("time_limit", ctypes.c_double),
                ("check_iter", ctypes.c_size_t), ("print_frequency", ctypes.c_int),
                ("use_scaling", ctypes.c_int), ("verbose", ctypes.c_int), ("spmv_mode_q", ctypes.c_int),
                ("spmv_mode_a", ctypes.c_int), ("gram_mode", ctypes.c_int), ("polishing", ctypes.c_int),
                ("polish_python", ctypes.c_char_p), ("polish_worker", ctypes.c_char_p),
                ("polish_directory", ctypes.c_char_p), ("polish_keep_files", ctypes.c_int),
                ("polish_max_attempts", ctypes.c_size_t), ("polish_episode_seconds", ctypes.c_double),
                ("polish_total_seconds", ctypes.c_double), ("polish_memory_bytes", ctypes.c_size_t)]


class _RefResults(ctypes.Structure):
    _fields_ = [("iter", ctypes.c_size_t), ("iter_4", ctypes.c_size_t), ("iter_6", ctypes.c_size_t),
                ("time", ctypes.c_double), ("time_4", ctypes.c_double), ("time_6", ctypes.c_double),
                ("primal_obj", ctypes.c_double), ("residuals", ctypes.c_double), ("gap", ctypes.c_double),
                ("status", ctypes.c_int), ("x", c_double_p), ("y", c_double_p), ("z", c_double_p),
                ("w", c_double_p), ("polish_attempts", ctypes.c_size_t), ("polish_accepted", ctypes.c_int),
                ("gram_active", ctypes.c_int), ("total_time", ctypes.c_double)]


_ref_gpu: Optional[ctypes.CDLL] = None


def ref_gpu_available() -> bool:
    return REF_GPU_LIB.exists()


def ref_gpu_lib() -> ctypes.CDLL:
    global _ref_gpu
    if _ref_gpu is None:
        L = ctypes.CDLL(str(REF_GPU_LIB))
        L.model_init.argtypes = [ctypes.POINTER(_RefModel)]
        L.model_free.argtypes = [ctypes.POINTER(_RefModel)]
        L.build_from_QAbc.argtypes = [ctypes.POINTER(_RefCSR), ctypes.POINTER(_RefCSR)] + [c_double_p] * 5 + \
            [ctypes.c_double, ctypes.POINTER(_RefModel)]
        L.params_set_defaults.argtypes = [ctypes.POINTER(_RefParams)]
        L.results_init.argtypes = [ctypes.POINTER(_RefResults)]
        L.results_free.argtypes = [ctypes.POINTER(_RefResults)]
        L.solve_gpu.argtypes = [ctypes.POINTER(_RefModel), ctypes.POINTER(_RefParams), ctypes.POINTER(_RefResults)]
        L.gpu_backend_available.restype = ctypes.c_int
        _ref_gpu = L
    return _ref_gpu


class _RefSOC(ctypes.Structure):
    _fields_ = [("num_var_cones", ctypes.c_size_t), ("var_offsets", c_size_p), ("num_row_cones", ctypes.c_size_t),
                ("row_offsets", c_size_p), ("rhs", c_double_p)]


class RefGpuModel:
    """A model built by the reference's own ``build_from_QAbc`` (or
    ``build_from_QAbc_soc`` when ``soc = (var_offsets, row_offsets, rhs)``)
    inside the reference GPU library; ``solve`` runs its ``solve_gpu``
    (polishing 0, Gram off: the reference with ``--polishing 0 --gram off``)."""

    def __init__(self, inst, soc=None):
        L = ref_gpu_lib()
        self._keep = []

        def csr(nrow, ncol, m):
            ip, pp = _sz(np.asarray(m.indptr))
            ii, pi = _sz(np.asarray(m.indices) if m.nnz else np.zeros(1))
            dd, pd = _db(np.asarray(m.data) if m.nnz else np.zeros(1))
            self._keep += [ip, ii, dd]
            return _RefCSR(nrow, ncol, m.nnz, pp, pi, pd, 0)

        def db(a):
            arr, p = _db(a if len(a) else np.zeros(1))
            self._keep.append(arr)
            return p

        Q = csr(inst.n, inst.n, inst.Q)
        A = csr(inst.m, inst.n, inst.A)
        self.model = _RefModel()
        L.model_init(ctypes.byref(self.model))
        if soc is None:
            st = L.build_from_QAbc(ctypes.byref(Q), ctypes.byref(A), db(inst.c), db(inst.AL), db(inst.AU),
                                   db(inst.l), db(inst.u), float(inst.obj_constant), ctypes.byref(self.model))
        else:
            vo, ro, rhs = soc

            def offs(o):
                if o is None:
                    return 0, None
                arr, p = _sz(np.asarray(o))
                self._keep.append(arr)
                return len(o) - 1, p

            nv, vp = offs(vo)
            nr, rp = offs(ro)
            spec = _RefSOC(nv, vp, nr, rp, db(rhs) if rhs is not None else None)
            L.build_from_QAbc_soc.argtypes = [ctypes.POINTER(_RefCSR), ctypes.POINTER(_RefCSR)] + [c_double_p] * 5 + \
                [ctypes.c_double, ctypes.POINTER(_RefSOC), ctypes.POINTER(_RefModel)]
            st = L.build_from_QAbc_soc(ctypes.byref(Q), ctypes.byref(A), db(inst.c), db(inst.AL), db(inst.AU),
                                       db(inst.l), db(inst.u), float(inst.obj_constant), ctypes.byref(spec),
                                       ctypes.byref(self.model))
        if st != 0:
            raise ValueError(f"reference build_from_QAbc failed: {st}")
        self.n = int(self.model.Q.ncol)
        self.m = int(self.model.A.nrow)

    def solve(self, stoptol=1e-6, max_iter=2147483647, time_limit=3600.0, device=0):
        L = ref_gpu_lib()
        p = _RefParams()
        L.params_set_defaults(ctypes.byref(p))
        p.stoptol = stoptol
        p.max_iter = max_iter
        p.time_limit = time_limit
        p.use_gpu = 1
        p.device_number = device
        p.verbose = 0
        p.polishing = 0
        p.gram_mode = 0
        r = _RefResults()
        L.results_init(ctypes.byref(r))
        st = L.solve_gpu(ctypes.byref(self.model), ctypes.byref(p), ctypes.byref(r))

        def vec(ptr, k):
            return np.ctypeslib.as_array(ptr, shape=(k,)).copy() if (ptr and k) else np.zeros(0)

        out = dict(ret=st, status=r.status, iter=int(r.iter), primal_obj=r.primal_obj, residuals=r.residuals,
                   gap=r.gap, time=r.time, x=vec(r.x, self.n), y=vec(r.y, self.m), z=vec(r.z, self.n),
                   w=vec(r.w, self.n))
        L.results_free(ctypes.byref(r))
        return out

    def __del__(self):
        try:
            ref_gpu_lib().model_free(ctypes.byref(self.model))
        except Exception:
            pass


# --------------------------------------------------------------------------
# the reference's MPS reader (its CPU library's build_from_mps)
# --------------------------------------------------------------------------

def _model_arrays(ms) -> dict:
    def csr(c):
        nr, nnz = int(c.nrow), int(c.nnz)
        ip = np.ctypeslib.as_array(c.row_ptr, shape=(nr + 1,)).astype(np.int64).copy()
        ii = np.ctypeslib.as_array(c.col_ind, shape=(nnz,)).astype(np.int64).copy() if nnz else np.zeros(0, np.int64)
        dv = np.ctypeslib.as_array(c.values, shape=(nnz,)).copy() if nnz else np.zeros(0)
        return ip, ii, dv

    n, m = int(ms.Q.ncol), int(ms.A.nrow)

    def vec(ptr, k):
        return np.ctypeslib.as_array(ptr, shape=(k,)).copy() if (ptr and k) else np.zeros(0)

    q, a = csr(ms.Q), csr(ms.A)
    return dict(n=n, m=m, q_indptr=q[0], q_indices=q[1], q_data=q[2], a_indptr=a[0], a_indices=a[1], a_data=a[2],
                c=vec(ms.c, n), l=vec(ms.l, n), u=vec(ms.u, n), AL=vec(ms.AL, m), AU=vec(ms.AU, m),
                obj_constant=float(ms.obj_constant))


_REF_MPS_SCRIPT = r"""
import ctypes, json, sys
L = ctypes.CDLL(sys.argv[1])   # loaded before anything else: see ref_build_from_mps
szp, dp = ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_double)
class CSR(ctypes.Structure):
    _fields_ = [("nrow", ctypes.c_size_t), ("ncol", ctypes.c_size_t), ("nnz", ctypes.c_size_t),
                ("row_ptr", szp), ("col_ind", szp), ("values", dp), ("owns_data", ctypes.c_int)]
class Model(ctypes.Structure):
    _fields_ = [("Q", CSR), ("A", CSR), ("AT", CSR), ("c", dp), ("AL", dp), ("AU", dp), ("l", dp), ("u", dp),
                ("obj_constant", ctypes.c_double), ("owns_data", ctypes.c_int), ("num_var_cones", ctypes.c_size_t),
                ("var_cone_offsets", szp), ("num_row_cones", ctypes.c_size_t), ("row_cone_offsets", szp),
                ("soc_rhs", dp)]
ms = Model()
L.model_init(ctypes.byref(ms))
st = L.build_from_mps(sys.argv[2].encode(), ctypes.byref(ms))
out = {"status": st}
if st == 0:
    n, m = ms.Q.ncol, ms.A.nrow
    h = lambda p, k: [float(p[i]).hex() for i in range(k)]
    ii = lambda p, k: [int(p[i]) for i in range(k)]
    out.update(n=n, m=m, q_indptr=ii(ms.Q.row_ptr, n + 1), q_indices=ii(ms.Q.col_ind, ms.Q.nnz),
               q_data=h(ms.Q.values, ms.Q.nnz), a_indptr=ii(ms.A.row_ptr, m + 1), a_indices=ii(ms.A.col_ind, ms.A.nnz),
               a_data=h(ms.A.values, ms.A.nnz), c=h(ms.c, n), l=h(ms.l, n), u=h(ms.u, n), AL=h(ms.AL, m),
               AU=h(ms.AU, m), obj_constant=float(ms.obj_constant).hex(),
               num_row_cones=int(ms.num_row_cones),
               row_cone_offsets=ii(ms.row_cone_offsets, ms.num_row_cones + 1) if ms.num_row_cones else [],
               soc_rhs=h(ms.soc_rhs, m) if ms.num_row_cones else [], num_var_cones=int(ms.num_var_cones))
    L.model_free(ctypes.byref(ms))
print("@@" + json.dumps(out))
"""


def ref_build_from_mps(path) -> dict:
    """Parse an MPS file with the reference's own reader (its CPU library's
    build_from_mps: src/shared/mps_qp.cpp, mps_reader.cpp) and return its
    HPRQPModel arrays, or {"status": code}.

    Runs in a fresh interpreter that loads the reference library before any
    other extension: in a process that has imported numpy first, the
    reference reader's std::cerr warnings (second objective row, second RHS
    or BOUNDS set) crashed inside libstdc++ here."""
    import json as _json
    import sys as _sys

    r = subprocess.run([_sys.executable, "-c", _REF_MPS_SCRIPT, str(REF_CPU_LIB), str(path)],
                       capture_output=True, text=True, timeout=120)
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("@@")]
    if not line:
        return {"status": -1, "stderr": r.stderr[-2000:]}
    d = _json.loads(line[0][2:])
    if d["status"] != 0:
        return {"status": int(d["status"])}
    out = {"status": 0, "n": d["n"], "m": d["m"], "obj_constant": float.fromhex(d["obj_constant"])}
    for k in ("q_indptr", "q_indices", "a_indptr", "a_indices"):
        out[k] = np.asarray(d[k], np.int64)
    for k in ("q_data", "a_data", "c", "l", "u", "AL", "AU"):
        out[k] = np.array([float.fromhex(v) for v in d[k]], np.float64)
    out["num_var_cones"] = int(d.get("num_var_cones", 0))
    out["num_row_cones"] = int(d.get("num_row_cones", 0))
    out["row_cone_offsets"] = np.asarray(d.get("row_cone_offsets", []), np.int64)
    out["soc_rhs"] = np.array([float.fromhex(v) for v in d.get("soc_rhs", [])], np.float64)
    return out
