"""Host-side C entry points of the builder and the sparse/vector helpers, on
CPU, with the reference's own known answers: tests/test_builder_preprocess.c
(row deletion, Q symmetrisation) and tests/test_sparse_helpers.c (matvec,
transpose matvec, box projection, model copy)."""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

c_size_p = ctypes.POINTER(ctypes.c_size_t)
c_double_p = ctypes.POINTER(ctypes.c_double)


@pytest.fixture(scope="module")
def lib(engine_lib):
    hprqp = engine_lib
    L = hprqp._lib()
    M, Mo = ctypes.POINTER(hprqp._MatrixCSR), ctypes.POINTER(hprqp._ModelStruct)
    L.build_model_from_arrays.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, Mo]
    L.build_from_QAbc.argtypes = [M, M] + [c_double_p] * 5 + [ctypes.c_double, Mo]
    L.preprocess_model.argtypes = [Mo]
    L.model_validate_soc.argtypes = [Mo]
    L.model_init.argtypes = [Mo]
    L.model_init.restype = None
    L.model_free.argtypes = [Mo]
    L.model_free.restype = None
    L.matrix_csr_matvec.argtypes = [M, c_double_p, c_double_p]
    L.matrix_csr_transpose_matvec.argtypes = [M, c_double_p, c_double_p]
    L.vec_project_box.argtypes = [c_double_p] * 4 + [ctypes.c_size_t]
    L.vec_project_box.restype = None
    L.vec_axpby.argtypes = [c_double_p, c_double_p, ctypes.c_size_t, ctypes.c_double, ctypes.c_double]
    L.vec_axpby.restype = None
    L.vec_fill.argtypes = [c_double_p, ctypes.c_size_t, ctypes.c_double]
    L.vec_fill.restype = None
    L.vec_copy.argtypes = [c_double_p, c_double_p, ctypes.c_size_t]
    L.vec_copy.restype = None
    for f in ("vec_dot",):
        getattr(L, f).argtypes = [c_double_p, c_double_p, ctypes.c_size_t]
        getattr(L, f).restype = ctypes.c_double
    for f in ("vec_norm2", "vec_norm_inf"):
        getattr(L, f).argtypes = [c_double_p, ctypes.c_size_t]
        getattr(L, f).restype = ctypes.c_double
    return hprqp, L


class _Keep(list):
    def csr(self, hprqp, nrow, ncol, rp, ci, v):
        rp = np.ascontiguousarray(rp, np.uint64)
        ci = np.ascontiguousarray(ci if len(ci) else [0], np.uint64)
        v = np.ascontiguousarray(v if len(v) else [0.0], np.float64)
        self += [rp, ci, v]
        return hprqp._MatrixCSR(nrow, ncol, int(rp[-1]), rp.ctypes.data_as(c_size_p), ci.ctypes.data_as(c_size_p),
                                v.ctypes.data_as(c_double_p), 0)

    def vec(self, values):
        a = np.ascontiguousarray(values, np.float64)
        self.append(a)
        return a.ctypes.data_as(c_double_p)


def _arr(p, n):
    return np.ctypeslib.as_array(p, (n,)).copy() if n else np.zeros(0)


def test_builder_preprocess_reference_case(lib):
    """tests/test_builder_preprocess.c:21-96"""
    hprqp, L = lib
    k = _Keep()
    Q = k.csr(hprqp, 2, 2, [0, 2, 3], [0, 1, 1], [2.0, 6.0, 4.0])
    A = k.csr(hprqp, 3, 2, [0, 2, 2, 2], [0, 1], [1.0, -1.0])
    model = hprqp._ModelStruct()
    L.model_init(ctypes.byref(model))
    st = L.build_model_from_arrays(ctypes.byref(Q), ctypes.byref(A), k.vec([1.0, 2.0]), k.vec([0.0, -1.0, -math.inf]),
                                   k.vec([3.0, 1.0, math.inf]), k.vec([-2.0, -2.0]), k.vec([2.0, 2.0]), 0.0,
                                   ctypes.byref(model))
    assert st == 0
    assert model.A.nrow == 1 and model.AT.ncol == 1 and model.Q.nnz == 4
    qv = _arr(model.Q.values, 4)
    assert abs(qv[1] - 3.0) < 1e-12 and abs(qv[2] - 3.0) < 1e-12
    assert model.AL[0] == 0.0 and model.AU[0] == 3.0
    # preprocessing a built model again changes nothing
    before = (_arr(model.Q.values, 4), model.A.nrow, model.AT.nnz)
    assert L.preprocess_model(ctypes.byref(model)) == 0
    assert np.array_equal(_arr(model.Q.values, 4), before[0]) and model.A.nrow == 1 and model.AT.nnz == before[2]
    assert L.model_validate_soc(ctypes.byref(model)) == 0
    L.model_free(ctypes.byref(model))


def test_sparse_helpers_reference_case(lib):
    """tests/test_sparse_helpers.c:11-124"""
    hprqp, L = lib
    k = _Keep()
    M = k.csr(hprqp, 2, 3, [0, 2, 4], [0, 2, 1, 2], [1.0, 4.0, 2.0, 5.0])
    x = np.array([1.0, 2.0, 3.0])
    y = np.zeros(2)
    assert L.matrix_csr_matvec(ctypes.byref(M), x.ctypes.data_as(c_double_p), y.ctypes.data_as(c_double_p)) == 0
    assert y.tolist() == [13.0, 19.0]
    yt = np.zeros(3)
    assert L.matrix_csr_transpose_matvec(ctypes.byref(M), y.ctypes.data_as(c_double_p),
                                         yt.ctypes.data_as(c_double_p)) == 0
    assert yt.tolist() == [13.0, 38.0, 147.0]
    proj = np.zeros(3)
    L.vec_project_box(proj.ctypes.data_as(c_double_p), x.ctypes.data_as(c_double_p), k.vec([0.0, 1.5, 2.5]),
                      k.vec([1.0, 2.5, 2.8]), 3)
    assert proj.tolist() == [1.0, 2.0, 2.8]
    Q = k.csr(hprqp, 3, 3, [0, 1, 2, 3], [0, 1, 2], [2.0, 3.0, 4.0])
    model = hprqp._ModelStruct()
    L.model_init(ctypes.byref(model))
    assert L.build_from_QAbc(ctypes.byref(Q), ctypes.byref(M), k.vec([1.0, -1.0, 0.5]), k.vec([-1.0, 0.0]),
                             k.vec([2.0, 3.0]), k.vec([-2.0] * 3), k.vec([2.0] * 3), 1.5, ctypes.byref(model)) == 0
    assert (model.AT.nrow, model.AT.ncol, model.AT.nnz) == (3, 2, 4)
    assert model.obj_constant == 1.5 and model.c[1] == -1.0 and model.AL[1] == 0.0
    L.model_free(ctypes.byref(model))


def test_vector_helpers(lib):
    _, L = lib
    p = (lambda a: a.ctypes.data_as(c_double_p))  # noqa: E731
    x, y = np.array([1.0, -2.0, 3.0]), np.array([4.0, 5.0, -6.0])
    assert L.vec_dot(p(x), p(y), 3) == 1.0 * 4.0 + (-2.0) * 5.0 + 3.0 * -6.0
    assert L.vec_norm2(p(x), 3) == math.sqrt(14.0)
    assert L.vec_norm_inf(p(np.array([1.0, np.nan, -7.5, 2.0])), 4) == 7.5
    z = y.copy()
    L.vec_axpby(p(z), p(x), 3, 2.0, -1.0)
    assert z.tolist() == (2.0 * x - y).tolist()
    L.vec_fill(p(z), 3, 0.25)
    assert z.tolist() == [0.25] * 3
    L.vec_copy(p(z), p(x), 3)
    assert z.tolist() == x.tolist()
    out = np.zeros(2)
    # lower above upper: the upper bound wins, as in the reference
    L.vec_project_box(p(out), p(np.array([0.0, 9.0])), p(np.array([1.0, 5.0])), p(np.array([0.5, 6.0])), 2)
    assert out.tolist() == [0.5, 6.0]


def test_preprocess_rejects_models_it_does_not_own(lib):
    hprqp, L = lib
    model = hprqp._ModelStruct()
    L.model_init(ctypes.byref(model))
    assert L.preprocess_model(ctypes.byref(model)) == hprqp.STATUS_INVALID_ARGUMENT
    assert L.preprocess_model(None) == hprqp.STATUS_INVALID_ARGUMENT
    assert L.model_validate_soc(None) == hprqp.STATUS_INVALID_ARGUMENT


def test_preprocess_keeps_cone_rows(lib):
    """a cone model keeps every row and its cone blocks through preprocessing"""
    hprqp, L = lib
    m = hprqp.build_from_qabc_soc(np.eye(3), [1.0, 0.0, 0.0], [[1.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.0, 1.0]],
                                  [0.0, -math.inf, -math.inf], [1.0, math.inf, math.inf], [-math.inf] * 3,
                                  [math.inf] * 3, row_cone_offsets=[1, 3], rhs=[0.0, 1.0, 0.0])
    st = m._struct()
    assert st.A.nrow == 3
    assert L.preprocess_model(ctypes.byref(st)) == 0
    st = m._struct()
    assert st.A.nrow == 3 and st.num_row_cones == 1 and list(_arr(st.soc_rhs, 3)) == [0.0, 1.0, 0.0]
