"""build_from_QAbc_qc_factors / build_from_QAbc_qc_diagonal (include/shared/
qcqp.h) against the reference's own builders (its CPU library, reference
src/shared/qcqp.c) on the same inputs: identical models (arrays, cone
offsets, rhs) and the same rejections."""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

import pyoracle

pytestmark = pytest.mark.skipif(not pyoracle.ref_available(), reason="reference CPU library not built")

c_size_p = ctypes.POINTER(ctypes.c_size_t)
c_double_p = ctypes.POINTER(ctypes.c_double)


def _setup(L, hprqp):
    M, Mo = ctypes.POINTER(hprqp._MatrixCSR), ctypes.POINTER(hprqp._ModelStruct)
    for f in ("build_from_QAbc_qc_factors", "build_from_QAbc_qc_diagonal"):
        getattr(L, f).restype = ctypes.c_int
    L.build_from_QAbc_qc_factors.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, M, c_double_p, M,
                                                                         c_size_p, Mo]
    L.build_from_QAbc_qc_diagonal.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, M, c_double_p, M, Mo]
    L.model_init.argtypes = [Mo]
    L.model_init.restype = None
    L.model_free.argtypes = [Mo]
    L.model_free.restype = None
    return L


@pytest.fixture(scope="module")
def libs(engine_lib):
    # private handles: the argument types set here must not leak into the
    # shared library objects other tests configure differently
    hprqp = engine_lib
    pyoracle.ref_lib()
    return (hprqp, _setup(ctypes.CDLL(hprqp.library_path()), hprqp),
            _setup(ctypes.CDLL(str(pyoracle.REF_CPU_LIB)), hprqp))


class _Keep(list):
    def csr(self, hprqp, dense):
        dense = np.atleast_2d(np.asarray(dense, float))
        nrow, ncol = dense.shape
        rp, ci, v = [0], [], []
        for r in range(nrow):
            for j in range(ncol):
                if dense[r, j] != 0.0:
                    ci.append(j)
                    v.append(dense[r, j])
            rp.append(len(ci))
        rp = np.asarray(rp, np.uint64)
        ci = np.asarray(ci or [0], np.uint64)
        v = np.asarray(v or [0.0], np.float64)
        self += [rp, ci, v]
        return hprqp._MatrixCSR(nrow, ncol, int(rp[-1]), rp.ctypes.data_as(c_size_p), ci.ctypes.data_as(c_size_p),
                                v.ctypes.data_as(c_double_p), 0)

    def vec(self, a, dtype=np.float64, ptr=c_double_p):
        a = np.ascontiguousarray(a if len(a) else [0], dtype)
        self.append(a)
        return a.ctypes.data_as(ptr)


def _arrays(ms):
    n, m, nrc = int(ms.Q.ncol), int(ms.A.nrow), int(ms.num_row_cones)
    get = (lambda p, k: np.ctypeslib.as_array(p, (k,)).copy() if k else np.zeros(0))  # noqa: E731
    out = {"n": n, "m": m, "nrc": nrc, "obj": ms.obj_constant}
    for name, M in (("Q", ms.Q), ("A", ms.A), ("AT", ms.AT)):
        out[name] = (get(M.row_ptr, int(M.nrow) + 1), get(M.col_ind, int(M.nnz)), get(M.values, int(M.nnz)))
    for name in ("c", "l", "u"):
        out[name] = get(getattr(ms, name), n)
    for name in ("AL", "AU"):
        out[name] = get(getattr(ms, name), m)
    out["offsets"] = get(ms.row_cone_offsets, nrc + 1) if nrc else np.zeros(0)
    out["rhs"] = get(ms.soc_rhs, m) if nrc else np.zeros(0)
    return out


def _build(hprqp, L, fn, args):
    ms = hprqp._ModelStruct()
    L.model_init(ctypes.byref(ms))
    st = getattr(L, fn)(*args, ctypes.byref(ms))
    out = _arrays(ms) if st == 0 else None
    L.model_free(ctypes.byref(ms))
    return st, out


def _same(a, b):
    assert (a["n"], a["m"], a["nrc"], a["obj"]) == (b["n"], b["m"], b["nrc"], b["obj"])
    for k in ("Q", "A", "AT"):
        for x, y in zip(a[k], b[k]):
            assert np.array_equal(x, y), k
    for k in ("c", "l", "u", "AL", "AU", "offsets", "rhs"):
        assert np.array_equal(a[k], b[k]), k


def _problem(seed):
    rng = np.random.default_rng(seed)
    n = 7
    Q = np.diag(rng.random(n) + 0.5)
    A = (rng.random((4, n)) < 0.5) * rng.standard_normal((4, n))
    A[2] = 0.0  # an empty linear row: kept, as in every cone model
    AL, AU = np.array([-1.0, -np.inf, 0.0, -np.inf]), np.array([1.0, 2.0, 0.0, np.inf])
    l, u = np.full(n, -np.inf), np.full(n, np.inf)
    l[:3], u[:3] = -1.0, 1.0
    C = rng.standard_normal((3, n)) * (rng.random((3, n)) < 0.6)
    const = -1.0 - rng.random(3)
    R = rng.standard_normal((4, n)) * (rng.random((4, n)) < 0.7)
    offsets = np.array([0, 2, 2, 4], np.uint64)  # the second constraint has no factor rows
    return Q, A, rng.standard_normal(n), AL, AU, l, u, C, const, R, offsets


@pytest.mark.parametrize("seed", range(4))
def test_factors_identical_to_reference(libs, seed):
    hprqp, ours, ref = libs
    Q, A, c, AL, AU, l, u, C, const, R, offsets = _problem(seed)
    k = _Keep()
    args = (ctypes.byref(k.csr(hprqp, Q)), ctypes.byref(k.csr(hprqp, A)), k.vec(c), k.vec(AL), k.vec(AU), k.vec(l),
            k.vec(u), 0.75, ctypes.byref(k.csr(hprqp, C)), k.vec(const), ctypes.byref(k.csr(hprqp, R)),
            k.vec(offsets, np.uint64, c_size_p))
    s1, a = _build(hprqp, ours, "build_from_QAbc_qc_factors", args)
    s2, b = _build(hprqp, ref, "build_from_QAbc_qc_factors", args)
    assert s1 == s2 == 0
    _same(a, b)
    assert a["m"] == 4 + 2 * 3 + 4 and list(a["offsets"]) == [4, 8, 10, 14]


@pytest.mark.parametrize("seed", range(3))
def test_diagonal_identical_to_reference(libs, seed):
    hprqp, ours, ref = libs
    Q, A, c, AL, AU, l, u, C, const, _, _ = _problem(seed)
    rng = np.random.default_rng(100 + seed)
    D = rng.random((3, Q.shape[0])) * (rng.random((3, Q.shape[0])) < 0.5)
    k = _Keep()
    args = (ctypes.byref(k.csr(hprqp, Q)), ctypes.byref(k.csr(hprqp, A)), k.vec(c), k.vec(AL), k.vec(AU), k.vec(l),
            k.vec(u), 0.0, ctypes.byref(k.csr(hprqp, C)), k.vec(const), ctypes.byref(k.csr(hprqp, D)))
    s1, a = _build(hprqp, ours, "build_from_QAbc_qc_diagonal", args)
    s2, b = _build(hprqp, ref, "build_from_QAbc_qc_diagonal", args)
    assert s1 == s2 == 0
    _same(a, b)


def test_same_rejections(libs):
    hprqp, ours, ref = libs
    Q, A, c, AL, AU, l, u, C, const, R, offsets = _problem(0)
    k = _Keep()
    base = [ctypes.byref(k.csr(hprqp, Q)), ctypes.byref(k.csr(hprqp, A)), k.vec(c), k.vec(AL), k.vec(AU), k.vec(l),
            k.vec(u), 0.0]
    cases = {
        "negative_diagonal": ("build_from_QAbc_qc_diagonal",
                              base + [ctypes.byref(k.csr(hprqp, C)), k.vec(const),
                                      ctypes.byref(k.csr(hprqp, -np.abs(C) - 0.1))]),
        "wrong_columns": ("build_from_QAbc_qc_factors",
                          base + [ctypes.byref(k.csr(hprqp, C[:, :-1])), k.vec(const),
                                  ctypes.byref(k.csr(hprqp, R)), k.vec(offsets, np.uint64, c_size_p)]),
        "bad_offsets": ("build_from_QAbc_qc_factors",
                        base + [ctypes.byref(k.csr(hprqp, C)), k.vec(const), ctypes.byref(k.csr(hprqp, R)),
                                k.vec(np.array([0, 3, 2, 4], np.uint64), np.uint64, c_size_p)]),
        "nonfinite_constant": ("build_from_QAbc_qc_factors",
                               base + [ctypes.byref(k.csr(hprqp, C)), k.vec([math.nan, 0.0, 0.0]),
                                       ctypes.byref(k.csr(hprqp, R)), k.vec(offsets, np.uint64, c_size_p)]),
    }
    for name, (fn, args) in cases.items():
        s1, _ = _build(hprqp, ours, fn, tuple(args))
        s2, _ = _build(hprqp, ref, fn, tuple(args))
        assert s1 == s2 == hprqp.STATUS_INVALID_ARGUMENT, name
