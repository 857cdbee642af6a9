"""The oracle's warm start (oracle_solve_from), on CPU: a zero start is the
cold solve bit for bit, a start at the oracle's own solution re-converges
to it in a fraction of the iterations, and sigma0 is taken."""
from __future__ import annotations

import numpy as np

import pyoracle
from hprqp import instances


def _same(a, b):
    for key in ("status", "iter", "iter_4", "iter_6", "primal_obj", "residuals", "sigma", "restarts"):
        assert a[key] == b[key], key
    for key in ("x", "y", "z", "w"):
        assert np.array_equal(a[key], b[key]), key


def _cases():
    free = instances.plain_qp(0x48505251 + 91100, n=50, m=20, a_density=0.1, m_rows=10, m_density=0.1, n_eq=12)
    free.l[:] = -np.inf
    free.u[:] = np.inf  # the noC path
    return [instances.config3_instance(40), instances.adjoint_case(3), free] + \
        [i for i in instances.tiny_cases() if i.name in ("standard", "dense_q")]


def test_zero_start_is_the_cold_solve():
    for inst in _cases():
        om = pyoracle.OracleModel(inst)
        cold = om.solve(stoptol=1e-8)
        warm = om.solve(stoptol=1e-8, x0=np.zeros(om.n), y0=np.zeros(om.m), w0=np.zeros(om.n))
        if cold["iter"] == 0:
            # optimal at the zero point: a warm start is never accepted before
            # the first step, so it stops at the next check instead
            assert warm["status"] == cold["status"] == 6 and warm["iter"] >= 1, inst.name
            assert warm["primal_obj"] == cold["primal_obj"]
            continue
        _same(cold, warm)
        assert om.solve(stoptol=1e-8, x0=np.zeros(om.n), sigma0=0.0)["iter"] == cold["iter"]


def test_restart_at_own_solution():
    for inst in _cases():
        om = pyoracle.OracleModel(inst)
        cold = om.solve(stoptol=1e-8)
        assert cold["status"] == 6
        warm = om.solve(stoptol=1e-8, x0=cold["x"], y0=cold["y"], w0=cold["w"], sigma0=cold["sigma"])
        assert warm["status"] == 6
        assert 1 <= warm["iter"] <= max(10, cold["iter"] // 4), (inst.name, warm["iter"], cold["iter"])
        assert abs(warm["primal_obj"] - cold["primal_obj"]) <= 1e-7 * max(1.0, abs(cold["primal_obj"]))


def test_sigma0_changes_the_run():
    om = pyoracle.OracleModel(instances.config3_instance(41))
    a = om.solve(stoptol=1e-6, x0=np.zeros(om.n))
    b = om.solve(stoptol=1e-6, x0=np.zeros(om.n), sigma0=10.0 * a["sigma"])
    assert a["iter"] != b["iter"] or a["primal_obj"] != b["primal_obj"]
    assert b["status"] == 6
