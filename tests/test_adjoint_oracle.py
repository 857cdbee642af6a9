"""The dense KKT adjoint (the checker for the device adjoint) against central
finite differences of the CPU oracle solved to 1e-12.

The reference has no adjoint, so the adjoint checker is pinned here by
differentiating the reference algorithm's own solutions numerically."""
from __future__ import annotations

import copy

import numpy as np
import pytest

import pyoracle
from hprqp import instances

TOL = 1e-12
EPS = 1e-5
OPTIMAL = 6  # HPRQP_STATUS_OPTIMAL


def _solve(inst):
    o = pyoracle.OracleModel(inst).solve(stoptol=TOL, mode=pyoracle.MODE_GPU_REF)
    assert o["status"] == OPTIMAL
    return o


def _loss(inst, gx, gy):
    o = _solve(inst)
    return float(gx @ o["x"] + gy @ o["y"])


def _perturbed(inst, field, idx, delta):
    p = copy.deepcopy(inst)
    if field == "row":  # equality row: move both sides
        p.AL = p.AL.copy()
        p.AU = p.AU.copy()
        p.AL[idx] += delta
        p.AU[idx] += delta
    elif field in ("Q", "A"):
        mat = getattr(p, field)
        mat.data = mat.data.copy()
        mat.data[idx] += delta
    else:
        arr = getattr(p, field).copy()
        arr[idx] += delta
        setattr(p, field, arr)
    return p


def _fd(inst, field, idx, gx, gy):
    return (_loss(_perturbed(inst, field, idx, EPS), gx, gy) -
            _loss(_perturbed(inst, field, idx, -EPS), gx, gy)) / (2 * EPS)


@pytest.mark.parametrize("case", [0, 1])
def test_dense_adjoint_matches_finite_differences(case):
    inst = instances.adjoint_case(case)
    o = _solve(inst)
    x, y, z = o["x"], o["y"], o["z"]
    assert len(y) == inst.m  # no row removed by preprocessing in this recipe
    ax = inst.A.dense() @ x
    # sign conventions: y > 0 at the lower row bound, z > 0 at the lower variable bound
    assert np.all(np.abs(ax[y > 0] - inst.AL[y > 0]) < 1e-8)
    assert np.all(np.abs(ax[y < 0] - inst.AU[y < 0]) < 1e-8)
    assert np.all(np.abs(x[z > 0] - inst.l[z > 0]) < 1e-8)
    assert np.all(np.abs(x[z < 0] - inst.u[z < 0]) < 1e-8)
    nb = int(np.sum(z != 0))
    nr = int(np.sum(y != 0))
    assert 0 < nb < inst.n and 0 < nr <= inst.m  # both active sets non-trivial
    rng = np.random.default_rng(17 + case)
    gx = rng.standard_normal(inst.n)
    gy = rng.standard_normal(inst.m)
    g = pyoracle.kkt_adjoint_dense(inst, x, y, z, gx, gy)
    free = np.nonzero(z == 0)[0]
    checks = [("c", int(i), g["dc"][i]) for i in free[:3]]
    lo = np.nonzero(z > 0)[0]
    hi = np.nonzero(z < 0)[0]
    checks += [("l", int(i), g["dl"][i]) for i in lo[:2]] + [("u", int(i), g["du"][i]) for i in hi[:2]]
    ranged = inst.AL < inst.AU
    rlo = np.nonzero((y > 0) & ranged)[0]
    rhi = np.nonzero((y < 0) & ranged)[0]
    req = np.nonzero((y != 0) & ~ranged)[0]
    checks += [("row", int(r), g["dAL"][r] + g["dAU"][r]) for r in req[:2]]
    checks += [("AL", int(r), g["dAL"][r]) for r in rlo[:2]] + [("AU", int(r), g["dAU"][r]) for r in rhi[:2]]
    checks += [("Q", e, g["dQ"][e]) for e in (0, inst.Q.nnz // 2, inst.Q.nnz - 1)]
    checks += [("A", e, g["dA"][e]) for e in (0, inst.A.nnz // 3, inst.A.nnz - 1)]
    assert len(checks) >= 12
    for field, idx, analytic in checks:
        fd = _fd(inst, field, idx, gx, gy)
        assert abs(fd - analytic) <= 1e-4 * max(1.0, abs(fd)), (field, idx, fd, analytic)
