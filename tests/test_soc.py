"""Second-order cones: the model builder against the reference's
(build_from_QAbc_soc of its CPU library) on CPU, and the GPU solve against
the reference's own GPU solve_gpu on the same cone models."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import pyoracle
from hprqp import instances

CASES = [(0, {}), (1, {}), (2, {"cone": 0}), (3, {"row_cone": 0}), (4, {"n_lin": 60, "cone": 12, "m_lin": 20,
                                                                        "row_cone": 8})]


def _build(hprqp, sc):
    q = sc.qp
    return hprqp.build_from_qabc_soc(q.Q, q.c, q.A, q.AL, q.AU, q.l, q.u, sc.var_offsets, sc.row_offsets, sc.rhs)


@pytest.mark.parametrize("seed,kw", CASES)
def test_soc_model_matches_reference_builder(engine_lib, seed, kw):
    hprqp = engine_lib
    if not pyoracle.ref_available():
        pytest.skip("reference CPU library not built")
    sc = instances.soc_case(seed, **kw)
    ours = hprqp.model_arrays(_build(hprqp, sc))
    ref = _ref_soc_model(pyoracle.ref_lib(), sc)
    for k in ("q_indptr", "q_indices", "q_data", "a_indptr", "a_indices", "a_data", "c", "l", "u", "AL", "AU"):
        assert np.array_equal(np.asarray(ours[k]), np.asarray(ref[k])), k


def _ref_soc_model(L, sc):
    q = sc.qp
    keep = []

    def sz(a):
        arr = np.ascontiguousarray(np.asarray(a if len(a) else np.zeros(1), np.uint64))
        keep.append(arr)
        return arr.ctypes.data_as(pyoracle.c_size_p)

    def db(a):
        arr = np.ascontiguousarray(np.asarray(a if len(a) else np.zeros(1), np.float64))
        keep.append(arr)
        return arr.ctypes.data_as(pyoracle.c_double_p)

    Qc = pyoracle._RefCSR(q.n, q.n, q.Q.nnz, sz(q.Q.indptr), sz(q.Q.indices), db(q.Q.data), 0)
    Ac = pyoracle._RefCSR(q.m, q.n, q.A.nnz, sz(q.A.indptr), sz(q.A.indices), db(q.A.data), 0)
    nv = 0 if sc.var_offsets is None else len(sc.var_offsets) - 1
    nr = 0 if sc.row_offsets is None else len(sc.row_offsets) - 1
    spec = pyoracle._RefSOC(nv, sz(sc.var_offsets) if nv else None, nr, sz(sc.row_offsets) if nr else None,
                            db(sc.rhs) if nr else None)
    ms = pyoracle._RefModel()
    L.model_init(ctypes.byref(ms))
    L.build_from_QAbc_soc.argtypes = [ctypes.POINTER(pyoracle._RefCSR)] * 2 + [pyoracle.c_double_p] * 5 + \
        [ctypes.c_double, ctypes.POINTER(pyoracle._RefSOC), ctypes.POINTER(pyoracle._RefModel)]
    st = L.build_from_QAbc_soc(ctypes.byref(Qc), ctypes.byref(Ac), db(q.c), db(q.AL), db(q.AU), db(q.l), db(q.u),
                               0.0, ctypes.byref(spec), ctypes.byref(ms))
    assert st == 0
    out = pyoracle._model_arrays(ms)
    L.model_free(ctypes.byref(ms))
    return out


def test_soc_invalid_specs_rejected(engine_lib):
    hprqp = engine_lib
    sc = instances.soc_case(0)
    q = sc.qp
    bad = []
    bad.append(dict(var_offsets=[q.n - 3, q.n - 1], row_offsets=sc.row_offsets, rhs=sc.rhs))  # does not end at n
    l2 = q.l.copy()
    l2[-1] = -5.0  # a cone variable with a finite bound
    bad.append(dict(l=l2))
    rhs2 = sc.rhs.copy()
    rhs2[0] = 1.0  # rhs on a linear row
    bad.append(dict(rhs=rhs2))
    bad.append(dict(row_offsets=[sc.row_offsets[0], sc.row_offsets[0], q.m]))  # empty cone
    for b in bad:
        args = dict(var_offsets=sc.var_offsets, row_offsets=sc.row_offsets, rhs=sc.rhs, l=q.l)
        args.update(b)
        with pytest.raises(RuntimeError):
            hprqp.build_from_qabc_soc(q.Q, q.c, q.A, q.AL, q.AU, args["l"], q.u, args["var_offsets"],
                                      args["row_offsets"], args["rhs"])


def _feasible(sc, x, tol):
    q = sc.qp
    A = q.A.dense()
    ax = A @ x
    n_lin = len(x) if sc.var_offsets is None else sc.var_offsets[0]
    ok = bool(np.all(x[:n_lin] <= q.u[:n_lin] + tol) and np.all(x[:n_lin] >= q.l[:n_lin] - tol))
    m_lin = q.m if sc.row_offsets is None else sc.row_offsets[0]
    lo, up, v = q.AL[:m_lin], q.AU[:m_lin], ax[:m_lin]
    ok &= bool(np.all(v >= lo - tol * (1 + np.abs(lo))) and np.all(v <= up + tol * (1 + np.abs(up))))
    if sc.var_offsets is not None:
        b, e = sc.var_offsets[0], sc.var_offsets[1]
        ok &= np.linalg.norm(x[b + 1:e]) <= x[b] + tol * (1 + abs(x[b]))
    if sc.row_offsets is not None:
        b, e = sc.row_offsets[0], sc.row_offsets[1]
        r = ax[b:e] - sc.rhs[b:e]
        ok &= np.linalg.norm(r[1:]) <= r[0] + tol * (1 + abs(r[0]))
    return bool(ok)


@pytest.mark.gpu
@pytest.mark.parametrize("stoptol", [1e-6, 1e-8])
@pytest.mark.parametrize("seed,kw", CASES)
def test_soc_solve_matches_reference_gpu(engine_lib, seed, kw, stoptol):
    hprqp = engine_lib
    if not pyoracle.ref_gpu_available():
        pytest.skip("reference GPU library not built")
    sc = instances.soc_case(seed, **kw)
    ref = pyoracle.RefGpuModel(sc.qp, soc=(sc.var_offsets, sc.row_offsets, sc.rhs)).solve(stoptol=stoptol)
    assert ref["status"] == hprqp.STATUS_OPTIMAL
    r = hprqp.optimize(_build(hprqp, sc), hprqp.Parameters(verbose=False, stoptol=stoptol), as_numpy=True)
    assert r.status_code == hprqp.STATUS_OPTIMAL
    assert r.residual <= stoptol
    assert abs(r.objective - ref["primal_obj"]) <= 1e-6 * max(1.0, abs(ref["primal_obj"]))
    assert _feasible(sc, r.x, 10 * stoptol)
    assert abs(r.iter - ref["iter"]) <= max(20, ref["iter"] // 5)
