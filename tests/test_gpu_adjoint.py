"""Device adjoint (hprqp_batch_backward: MINRES on the active-set KKT system,
one instance per CTA) against the dense FP64 KKT adjoint of the same
solution, against central finite differences of the GPU solver, and the
PyTorch layer built on it.

Bar: every gradient within 1e-5 (relative to max(1, |reference|)) of the
dense solve; the dense solve itself is pinned to finite differences of the
CPU oracle in test_adjoint_oracle.py."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-5
OPTIMAL = 6  # HPRQP_STATUS_OPTIMAL


def _close(got, ref, tol=GRAD_TOL):
    got, ref = np.asarray(got, float), np.asarray(ref, float)
    if ref.size == 0:
        return True
    return float(np.max(np.abs(got - ref))) <= tol * max(1.0, float(np.max(np.abs(ref))))


def _nz_range(packed, k, kind):
    ptr = packed.q_indptr if kind == "Q" else packed.a_indptr
    off = packed.var_offsets if kind == "Q" else packed.row_offsets
    return int(ptr[int(off[k])]), int(ptr[int(off[k + 1])])


def _check_batch(insts, seed, with_gy=True, stoptol=1e-11):
    from hprqp import batch

    b = batch.Batch(insts)
    try:
        b.solve(stoptol=stoptol, max_iter=200000)
        r = b.results()
        assert np.all(r.status == OPTIMAL), r.status
        rng = np.random.default_rng(seed)
        gx = rng.standard_normal(b.n)
        gy = rng.standard_normal(b.m) if with_gy else None
        g = b.backward(gx, gy, tol=1e-13)
        xs, ys, zs = b.split(r.x, "x"), b.split(r.y, "y"), b.split(r.z, "x")
        gxs = b.split(gx, "x")
        gys = b.split(gy, "y") if with_gy else [None] * len(insts)
        for k, inst in enumerate(insts):
            ref = pyoracle.kkt_adjoint_dense(inst, xs[k], ys[k], zs[k], gxs[k], gys[k])
            for name, got in (("dc", b.split(g.dc, "x")[k]), ("dl", b.split(g.dl, "x")[k]),
                              ("du", b.split(g.du, "x")[k]), ("dAL", b.split(g.dAL, "y")[k]),
                              ("dAU", b.split(g.dAU, "y")[k])):
                assert _close(got, ref[name]), (inst.name, name, np.max(np.abs(got - ref[name])))
            q0, q1 = _nz_range(b.packed, k, "Q")
            a0, a1 = _nz_range(b.packed, k, "A")
            assert _close(g.dQ[q0:q1], ref["dQ"]), (inst.name, "dQ")
            assert _close(g.dA[a0:a1], ref["dA"]), (inst.name, "dA")
            assert g.minres_relres[k] <= 1e-10, (inst.name, g.minres_relres[k], g.minres_iters[k])
        assert g.backward_ms > 0.0
        return g
    finally:
        b.close()


@pytest.mark.parametrize("with_gy", [True, False])
def test_adjoint_vs_dense_kkt(engine_lib, with_gy):
    _check_batch([instances.adjoint_case(i) for i in range(6)], 3 + int(with_gy), with_gy)


def test_adjoint_mixed_sizes(engine_lib):
    insts = [instances.adjoint_case(10, n=20, m=8), instances.adjoint_case(11, n=150, m=90),
             instances.adjoint_case(12, n=300, m=40), instances.adjoint_case(13, n=40, m=60)]
    _check_batch(insts, 7)


def test_adjoint_differentiation_batch_members(engine_lib):
    """Members of the 256-instance differentiation batch (n=500, m=300,
    150 equality rows; one has an empty row removed by preprocessing)."""
    _check_batch([instances.config4_instance(i) for i in (0, 3, 5)], 13, stoptol=1e-10)


def test_adjoint_no_rows_and_unconstrained(engine_lib):
    """m = 0, equality-only and all-interior instances (for the last the
    adjoint is Q^-1 g)."""
    tiny = {i.name: i for i in instances.tiny_cases()}
    _check_batch([tiny["empty_a"], tiny["standard_noC"], tiny["standard"], tiny["dense_q"]], 11)


def test_adjoint_zero_gradient(engine_lib):
    from hprqp import batch

    insts = [instances.adjoint_case(i) for i in range(2)]
    b = batch.Batch(insts)
    try:
        b.solve(stoptol=1e-10)
        g = b.backward(np.zeros(b.n), np.zeros(b.m))
        for a in (g.dc, g.dl, g.du, g.dAL, g.dAU, g.dQ, g.dA):
            assert np.all(a == 0.0)
        assert np.all(g.minres_iters == 0)
    finally:
        b.close()


def test_adjoint_repeated_calls_identical(engine_lib):
    from hprqp import batch

    insts = [instances.adjoint_case(i) for i in range(4)]
    b = batch.Batch(insts)
    try:
        b.solve(stoptol=1e-10)
        gx = np.random.default_rng(2).standard_normal(b.n)
        g1 = b.backward(gx)
        g2 = b.backward(gx)
        for a1, a2 in zip((g1.dc, g1.dl, g1.du, g1.dAL, g1.dAU, g1.dQ, g1.dA),
                          (g2.dc, g2.dl, g2.du, g2.dAL, g2.dAU, g2.dQ, g2.dA)):
            assert np.array_equal(a1, a2)
    finally:
        b.close()


def _perturb(p, field, idx, delta):
    if field == "row":  # equality row: both sides move
        p.AL[idx] += delta
        p.AU[idx] += delta
    else:
        getattr(p, {"Q": "q_data", "A": "a_data"}.get(field, field))[idx] += delta


def _unpack(p):
    """a one-instance Packed back into a QPInstance"""
    n = int(p.var_offsets[-1])
    m = int(p.row_offsets[-1])
    Q = instances.CSR(n, n, p.q_indptr.astype(np.int64), p.q_indices.astype(np.int64), p.q_data)
    A = instances.CSR(m, n, p.a_indptr.astype(np.int64), p.a_indices.astype(np.int64), p.a_data)
    return instances.QPInstance(Q, A, p.c, p.AL, p.AU, p.l, p.u, float(p.obj[0]))


@pytest.mark.parametrize("which", [0, 3])
def test_adjoint_finite_difference_through_gpu(engine_lib, which):
    """The differentiation workload's check: L = sum g.x*, g ~ N(0,1); central
    differences (eps 1e-6, FP64) of the batched GPU solver itself on 20
    random coordinates of one n=500, m=300 instance (c, active bounds of
    variables and rows, nonzeros of Q and A).  All 40 perturbed QPs are
    solved as one batch, to 1e-10 (tighter tolerances stall on some of these
    instances in the reference algorithm's sigma/restart logic; at 1e-10 the
    difference quotient is good to about 4e-6 relative, measured with the
    CPU oracle)."""
    from hprqp import batch

    inst = instances.config4_instance(which)
    eps = 1e-6
    rng = np.random.default_rng(100 + which)
    gx = rng.standard_normal(inst.n)
    b = batch.Batch([inst])
    b.solve(stoptol=1e-10, max_iter=200000)
    r = b.results()
    assert r.status[0] == OPTIMAL
    g = b.backward(gx, tol=1e-13)
    b.close()
    ranged = inst.AL < inst.AU
    pools = [("c", np.arange(inst.n), g.dc),
             ("l", np.nonzero(r.z > 0)[0], g.dl), ("u", np.nonzero(r.z < 0)[0], g.du),
             ("AL", np.nonzero((r.y > 0) & ranged)[0], g.dAL), ("AU", np.nonzero((r.y < 0) & ranged)[0], g.dAU),
             ("row", np.nonzero((r.y != 0) & ~ranged)[0], g.dAL + g.dAU),
             ("Q", np.arange(inst.Q.nnz), g.dQ), ("A", np.arange(inst.A.nnz), g.dA)]
    pools = [pl for pl in pools if len(pl[1])]
    coords = []
    for j in range(20):
        field, idx, grad = pools[j % len(pools)]
        i = int(rng.choice(idx))
        coords.append((field, i, float(grad[i])))
    perturbed = []
    for field, i, _ in coords:
        for sgn in (1.0, -1.0):
            p = batch.pack([inst])
            _perturb(p, field, i, sgn * eps)
            perturbed.append(_unpack(p))
    bb = batch.Batch(perturbed)
    bb.solve(stoptol=1e-10, max_iter=200000)
    rr = bb.results()
    bb.close()
    assert np.all(rr.status == OPTIMAL), rr.status
    xs = bb.split(rr.x, "x")
    for j, (field, i, an) in enumerate(coords):
        fd = (gx @ xs[2 * j] - gx @ xs[2 * j + 1]) / (2 * eps)
        assert abs(fd - an) <= 1e-4 * max(1.0, abs(fd)), (field, i, fd, an)


def test_torch_layer_matches_adjoint(engine_lib):
    import torch

    import hprqp
    from hprqp import batch

    insts = [instances.adjoint_case(i) for i in range(3)]
    p = batch.pack(insts)
    layer = hprqp.QPLayer(p, stoptol=1e-11)
    dev = "cuda"
    t = lambda a: torch.tensor(a, dtype=torch.float64, device=dev, requires_grad=True)  # noqa: E731
    q, a, c, AL, AU, l, u = (t(v) for v in (p.q_data, p.a_data, p.c, p.AL, p.AU, p.l, p.u))
    x, y = layer(q, a, c, AL, AU, l, u)
    assert x.device.type == "cuda" and x.shape == (int(p.var_offsets[-1]),)
    rng = np.random.default_rng(9)
    wx = torch.tensor(rng.standard_normal(x.shape[0]), device=dev)
    wy = torch.tensor(rng.standard_normal(y.shape[0]), device=dev)
    loss = (wx * x).sum() + (wy * y).sum()
    loss.backward()
    b = batch.Batch(p)
    b.solve(stoptol=1e-11)
    g = b.backward(wx.cpu().numpy(), wy.cpu().numpy(), tol=1e-12)
    b.close()
    for tensor, ref in ((c, g.dc), (l, g.dl), (u, g.du), (AL, g.dAL), (AU, g.dAU), (q, g.dQ), (a, g.dA)):
        assert tensor.grad is not None
        assert _close(tensor.grad.cpu().numpy(), ref, 1e-7)
