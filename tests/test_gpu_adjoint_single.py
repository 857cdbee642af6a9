"""Single-solve adjoint (hprqp_diff.h: solve_gpu that keeps its device state,
then MINRES on the device-wide SpMV kernels) against the dense FP64 KKT
adjoint, against the batched adjoint, and, at a size the dense solve cannot
take, through the residual of the same active-set KKT system assembled with
scipy on the host."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = pytest.mark.gpu

OPTIMAL = 6


def _close(got, ref, tol=1e-5):
    got, ref = np.asarray(got, float), np.asarray(ref, float)
    if ref.size == 0:
        return True
    return float(np.max(np.abs(got - ref))) <= tol * max(1.0, float(np.max(np.abs(ref))))


def _model_instance(hprqp, model):
    """the preprocessed model as a QPInstance (its symmetrised Q, kept rows)"""
    a = hprqp.model_arrays(model)
    n, m = a["n"], a["m"]
    Q = instances.CSR(n, n, a["q_indptr"], a["q_indices"], a["q_data"])
    A = instances.CSR(m, n, a["a_indptr"], a["a_indices"], a["a_data"])
    return instances.QPInstance(Q, A, a["c"], a["AL"], a["AU"], a["l"], a["u"], a["obj_constant"])


def _solve(hprqp, inst, stoptol=1e-11):
    model = hprqp.build_from_instance(inst)
    r, state = hprqp.solve_for_backward(model, hprqp.Parameters(verbose=False, stoptol=stoptol))
    assert state is not None
    return model, r, state


@pytest.mark.parametrize("case", [0, 1, 2, 3])
@pytest.mark.parametrize("with_gy", [True, False])
def test_single_adjoint_vs_dense_kkt(engine_lib, case, with_gy):
    hprqp = engine_lib
    inst = instances.adjoint_case(case)
    model, r, state = _solve(hprqp, inst)
    try:
        assert r.status_code == OPTIMAL
        mi = _model_instance(hprqp, model)
        rng = np.random.default_rng(40 + case)
        gx = rng.standard_normal(mi.n)
        gy = rng.standard_normal(mi.m) if with_gy else None
        g = state.backward(gx, gy, tol=1e-13)
        ref = pyoracle.kkt_adjoint_dense(mi, r.x, r.y, r.z, gx, gy)
        for k_ours, k_ref in (("dc", "dc"), ("dl", "dl"), ("du", "du"), ("dAL", "dAL"), ("dAU", "dAU"),
                              ("dQ_values", "dQ"), ("dA_values", "dA"), ("lam", "lam"), ("mu", "mu")):
            assert _close(g[k_ours], ref[k_ref]), (k_ours, np.max(np.abs(g[k_ours] - ref[k_ref])))
        assert g["minres_relres"] <= 1e-10
        # a second backward on the same state gives the same gradients
        g2 = state.backward(gx, gy, tol=1e-13)
        assert np.array_equal(g["dc"], g2["dc"]) and np.array_equal(g["dA_values"], g2["dA_values"])
    finally:
        state.close()


def test_single_adjoint_matches_batched(engine_lib):
    hprqp = engine_lib
    from hprqp import batch

    inst = instances.adjoint_case(5)
    model, r, state = _solve(hprqp, inst)
    try:
        gx = np.random.default_rng(3).standard_normal(inst.n)
        g = state.backward(gx, tol=1e-13)
    finally:
        state.close()
    b = batch.Batch([inst])
    b.solve(stoptol=1e-11)
    gb = b.backward(gx, tol=1e-13)
    b.close()
    assert _close(g["dc"], gb.dc, 1e-6) and _close(g["dl"], gb.dl, 1e-6) and _close(g["du"], gb.du, 1e-6)
    assert _close(g["dAL"], gb.dAL, 1e-6) and _close(g["dAU"], gb.dAU, 1e-6)


def test_single_adjoint_no_rows_and_free_variables(engine_lib):
    hprqp = engine_lib
    tiny = {i.name: i for i in instances.tiny_cases()}
    for name in ("empty_a", "standard_noC", "standard"):
        inst = tiny[name]
        model, r, state = _solve(hprqp, inst, 1e-10)
        try:
            mi = _model_instance(hprqp, model)
            gx = np.linspace(-1.0, 1.0, mi.n)
            g = state.backward(gx)
            ref = pyoracle.kkt_adjoint_dense(mi, r.x, r.y, r.z, gx)
            assert _close(g["dc"], ref["dc"]) and _close(g["dAL"], ref["dAL"]), name
        finally:
            state.close()


def test_single_adjoint_large_kkt_residual(engine_lib):
    """The large power-law recipe shrunk to n = 10,000: the device MINRES
    solution satisfies the active-set KKT system assembled on the host
    (scipy) to 1e-8 relative, and is zero off the active sets.  (scipy's
    SuperLU fails to factorize this KKT matrix, so no direct solution is
    compared here; the residual check does not need one.)"""
    import scipy.sparse as sp

    hprqp = engine_lib
    inst = instances.config1(scale=0.01)
    model = hprqp.build_from_instance(inst)
    r, state = hprqp.solve_for_backward(model, hprqp.Parameters(verbose=False, stoptol=1e-8, time_limit=60.0))
    assert state is not None
    try:
        mi = _model_instance(hprqp, model)
        rng = np.random.default_rng(11)
        gx = rng.standard_normal(mi.n)
        g = state.backward(gx, tol=1e-12)
    finally:
        state.close()
    F = np.nonzero(r.z == 0.0)[0]
    R = np.nonzero(r.y != 0.0)[0]
    Q = mi.Q.to_scipy()
    A = mi.A.to_scipy()
    K = sp.bmat([[Q[F][:, F], A[R][:, F].T], [A[R][:, F], None]], format="csc")
    rhs = np.concatenate([gx[F], np.zeros(len(R))])
    sol = np.concatenate([g["lam"][F], g["mu"][R]])
    assert np.linalg.norm(K @ sol - rhs) <= 1e-8 * np.linalg.norm(rhs)
    assert np.all(g["lam"][r.z != 0.0] == 0.0) and np.all(g["mu"][r.y == 0.0] == 0.0)


def test_single_adjoint_at_large_qp_size_converges(engine_lib):
    """The single large backward at the large QP's sizes (n = 1e6, m = 5e5,
    nnz(A) = 1e7, nnz(Q) ~ 3.2e7; the plain recipe, whose forward reaches
    1e-8): the forward solve is OPTIMAL, MINRES reaches a relative residual
    of 1e-10, and the adjoint satisfies the active-set KKT system assembled
    on the host to 1e-7 relative (MINRES runs on the scaled system)."""
    import scipy.sparse as sp

    hprqp = engine_lib
    inst = instances.config1_sized_plain()
    model = hprqp.build_from_instance(inst)
    r, state = hprqp.solve_for_backward(model, hprqp.Parameters(verbose=False, stoptol=1e-8, time_limit=300.0))
    assert r.status_code == hprqp.STATUS_OPTIMAL and r.residual < 1e-8
    assert state is not None
    try:
        gx = np.random.default_rng(1).standard_normal(inst.n)
        g = state.backward(gx, tol=1e-10, max_iter=50000)
    finally:
        state.close()
    assert g["minres_relres"] <= 1e-10, g["minres_relres"]
    mi = _model_instance(hprqp, model)
    F = np.nonzero(r.z == 0.0)[0]
    R = np.nonzero(r.y != 0.0)[0]
    Q = mi.Q.to_scipy()
    A = mi.A.to_scipy()
    AF = A[R][:, F]
    res = np.concatenate([Q[F][:, F] @ g["lam"][F] + AF.T @ g["mu"][R] - gx[F], AF @ g["lam"][F]])
    assert np.linalg.norm(res) <= 1e-7 * np.linalg.norm(gx[F]), np.linalg.norm(res) / np.linalg.norm(gx[F])


def test_torch_single_qp_function_matches_batched_layer(engine_lib):
    """hprqp.SingleQPFunction (solve_gpu + device-wide adjoint) and the
    batched QPFunction give the same gradients for the same QP, on CUDA
    tensors; a row removed by preprocessing gets zero gradients."""
    import torch

    import hprqp
    from hprqp import batch

    inst = instances.adjoint_case(2)
    # add an empty row (removed by preprocessing) at the end
    A = inst.A
    inst.A = instances.CSR(A.nrow + 1, A.ncol, np.append(A.indptr, A.indptr[-1]), A.indices, A.data)
    inst.AL = np.append(inst.AL, -1.0)
    inst.AU = np.append(inst.AU, 1.0)
    dev = "cuda"
    t = lambda a: torch.tensor(np.asarray(a, float), dtype=torch.float64, device=dev, requires_grad=True)  # noqa
    rng = np.random.default_rng(21)
    wx = torch.tensor(rng.standard_normal(inst.n), device=dev)
    wy = torch.tensor(rng.standard_normal(inst.m), device=dev)
    grads = []
    for which in ("single", "batched"):
        tensors = [t(v) for v in (inst.Q.data, inst.A.data, inst.c, inst.AL, inst.AU, inst.l, inst.u)]
        if which == "single":
            structure = (inst.n, inst.m, inst.Q.indptr, inst.Q.indices, inst.A.indptr, inst.A.indices)
            x, y = hprqp.SingleQPFunction.apply(structure, {"stoptol": 1e-11}, 1e-13, *tensors)
        else:
            layer = hprqp.QPLayer(batch.pack([inst]), backward_tol=1e-13, stoptol=1e-11)
            x, y = layer(*tensors)
        ((wx * x).sum() + (wy * y).sum()).backward()
        grads.append([tt.grad.cpu().numpy() for tt in tensors])
        assert float(y[-1]) == 0.0
    for gs, gb in zip(*grads):
        assert _close(gs, gb, 1e-6)
    assert grads[0][3][-1] == 0.0 and grads[0][4][-1] == 0.0  # dAL, dAU of the removed row
