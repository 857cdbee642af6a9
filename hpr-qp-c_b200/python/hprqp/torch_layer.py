"""Differentiable batched QP layer for PyTorch.

    min_x  1/2 x'Qx + c'x   s.t.  AL <= Ax <= AU,  l <= x <= u

for a batch of QPs that share one sparsity structure (given once as a
:class:`hprqp.batch.Packed`), with the numeric data passed as tensors.  The
forward pass runs the batched persistent solver (hprqp_batch_solve); the
backward pass runs the implicit-differentiation adjoint
(hprqp_batch_backward): one MINRES solve per instance on the active-set KKT
system

    [[Q_FF, A_RF'], [A_RF, 0]] [lam_F; mu_R] = [dL/dx_F; -dL/dy_R]

(F: variables off their bounds, R: rows at a bound), then

    dL/dc = -lam,  dL/dAL_r = mu_r (y_r > 0),  dL/dAU_r = mu_r (y_r < 0),
    dL/dl_i (z_i > 0), dL/du_i (z_i < 0) = dL/dx_i - (Q lam)_i - (A' mu)_i,
    dL/dQ_ij = -(lam_i x_j + lam_j x_i) / 2,  dL/dA_rj = -mu_r x_j + lam_j y_r.

The reference (PolyU-IOR/HPR-QP-C) has no differentiable layer; this module
is an addition.  The solve and the adjoint run on the GPU; tensors cross the
C ABI as host float64 arrays, and results come back on the inputs' device.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Optional

import numpy as np
import torch

from .batch import Batch, Packed


def _np(t: torch.Tensor) -> np.ndarray:
    return t.detach().to("cpu", torch.float64).contiguous().numpy()


class QPFunction(torch.autograd.Function):
    """``QPFunction.apply(structure, solve_kw, backward_tol, q_data, a_data,
    c, AL, AU, l, u) -> (x, y)``; ``structure`` fixes offsets and CSR index
    arrays, the tensors give the values in the same packing."""

    @staticmethod
    def forward(ctx, structure: Packed, solve_kw: dict, backward_tol: float, q_data, a_data, c, AL, AU, l, u):
        packed = replace(structure, q_data=_np(q_data), a_data=_np(a_data), c=_np(c), AL=_np(AL), AU=_np(AU),
                         l=_np(l), u=_np(u))
        kw = dict(solve_kw)
        start = kw.pop("warm_start", None)
        store = kw.pop("_warm_store", None)
        batch = Batch(packed, device_number=kw.pop("device_number", 0))
        try:
            if start is not None:
                batch.set_warm_start(*start)
            batch.solve(**kw)
            res = batch.results()
        except Exception:
            batch.close()
            raise
        if store is not None:
            store["point"] = (res.x.copy(), res.y.copy(), res.w.copy(), res.sigma.copy())
        ctx.batch = batch
        ctx.backward_tol = backward_tol
        ctx.device = c.device
        ctx.status = res.status
        x = torch.from_numpy(res.x.copy()).to(c.device)
        y = torch.from_numpy(res.y.copy()).to(c.device)
        return x, y

    @staticmethod
    def backward(ctx, gx, gy):
        batch: Optional[Batch] = getattr(ctx, "batch", None)
        if batch is None:
            raise RuntimeError("hprqp QPFunction: backward called twice (retain_graph is not supported)")
        try:
            g = batch.backward(_np(gx) if gx is not None else np.zeros(batch.n),
                               _np(gy) if gy is not None else None, tol=ctx.backward_tol)
        finally:
            batch.close()
            ctx.batch = None
        dev = ctx.device
        t = lambda a: torch.from_numpy(a.copy()).to(dev)  # noqa: E731
        return (None, None, None, t(g.dQ), t(g.dA), t(g.dc), t(g.dAL), t(g.dAU), t(g.dl), t(g.du))


class SingleQPFunction(torch.autograd.Function):
    """One (large) QP through solve_gpu + the device-wide adjoint
    (hprqp_diff.h).  ``SingleQPFunction.apply(structure, solve_kw,
    backward_tol, q_data, a_data, c, AL, AU, l, u) -> (x, y)`` with
    ``structure = (n, m, q_indptr, q_indices, a_indptr, a_indices)`` (CSR
    index arrays of the caller's Q and A); y has one entry per caller row
    (rows removed by preprocessing -- empty, or free on both sides -- get 0)."""

    @staticmethod
    def forward(ctx, structure, solve_kw: dict, backward_tol: float, q_data, a_data, c, AL, AU, l, u):
        from . import Parameters, build_from_qabc, solve_for_backward
        import scipy.sparse as sp

        n, m, qi, qj, ai, aj = structure
        qv, av = _np(q_data), _np(a_data)
        Q = sp.csr_matrix((qv, qj, qi), shape=(n, n))
        A = sp.csr_matrix((av, aj, ai), shape=(m, n))
        ALn, AUn = _np(AL), _np(AU)
        model = build_from_qabc(Q, _np(c), A, ALn, AUn, _np(l), _np(u))
        kw = dict(solve_kw)
        r, state = solve_for_backward(model, Parameters(verbose=False, **kw))
        if state is None:
            raise RuntimeError(f"hprqp SingleQPFunction: solve ended with status {r.status}")
        lens = np.diff(np.asarray(ai))
        kept = np.nonzero((lens > 0) & ~(np.isneginf(ALn) & np.isposinf(AUn)))[0]
        if len(kept) != len(r.y):
            state.close()
            raise RuntimeError("hprqp SingleQPFunction: unexpected row preprocessing")
        y = np.zeros(m)
        y[kept] = r.y
        ctx.state, ctx.model, ctx.kept, ctx.tol = state, model, kept, backward_tol
        ctx.x, ctx.y, ctx.structure, ctx.device = r.x, y, structure, c.device
        return torch.from_numpy(r.x.copy()).to(c.device), torch.from_numpy(y).to(c.device)

    @staticmethod
    def backward(ctx, gx, gy):
        state = getattr(ctx, "state", None)
        if state is None:
            raise RuntimeError("hprqp SingleQPFunction: backward called twice (retain_graph is not supported)")
        n, m, qi, qj, ai, aj = ctx.structure
        gxn = _np(gx) if gx is not None else np.zeros(n)
        gyk = _np(gy)[ctx.kept] if gy is not None else None
        try:
            g = state.backward(gxn, gyk, tol=ctx.tol)
        finally:
            state.close()
            ctx.state = None
        lam = g["lam"]
        mu = np.zeros(m)
        mu[ctx.kept] = g["mu"]
        x, y = ctx.x, ctx.y
        qrow = np.repeat(np.arange(n), np.diff(np.asarray(qi)))
        qcol = np.asarray(qj)
        arow = np.repeat(np.arange(m), np.diff(np.asarray(ai)))
        acol = np.asarray(aj)
        dQ = -0.5 * (lam[qrow] * x[qcol] + lam[qcol] * x[qrow])
        dA = -mu[arow] * x[acol] + lam[acol] * y[arow]
        dAL = np.zeros(m)
        dAU = np.zeros(m)
        dAL[ctx.kept] = g["dAL"]
        dAU[ctx.kept] = g["dAU"]
        dev = ctx.device
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        return (None, None, None, t(dQ), t(dA), t(g["dc"]), t(dAL), t(dAU), t(g["dl"]), t(g["du"]))


class QPLayer(torch.nn.Module):
    """Batched QP layer.  ``structure`` fixes the offsets and the CSR index
    arrays of Q and A (its numeric arrays are ignored); ``forward`` takes the
    data tensors packed the same way and returns ``(x, y)``.  Solver
    parameters (``stoptol``, default 1e-8, ``max_iter``, ...) are passed as
    keywords.  With ``warm_start=True`` every forward after the first starts
    the solver at the previous forward's solution and sigma
    (hprqp_batch_set_warm_start):
    in a training loop the data move a little per step, so the new solution
    is near the old one.  The gradients do not depend on the starting point."""

    def __init__(self, structure: Packed, backward_tol: float = 1e-12, warm_start: bool = False, **solve_kw):
        super().__init__()
        self.structure = structure
        self.backward_tol = backward_tol
        self.warm_start = warm_start
        self.solve_kw = {"stoptol": 1e-8, **solve_kw}
        self._warm = {}  # (x, y, w, sigma) of the last forward

    def forward(self, q_data, a_data, c, AL, AU, l, u):
        kw = self.solve_kw
        if self.warm_start:
            kw = {**kw, "warm_start": self._warm.get("point"), "_warm_store": self._warm}
        return QPFunction.apply(self.structure, kw, self.backward_tol, q_data, a_data, c, AL, AU, l, u)
