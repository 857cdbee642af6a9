"""The CPU oracle against the reference's own answers (no GPU).

Pins: (1) the closed-form one-step values of the reference's
tests/cpu/test_iteration.c:53-56; (2) the analytic optimum of the reference's
python/tests/test_hprqp.py:26-42; (3) golden vectors produced by the
reference CPU backend itself (tests/golden/reference_cpu.json, see
make_golden.py) -- the oracle in CPU-reference mode must reproduce them
bit for bit, and in GPU-reference mode to within rounding.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import pyoracle
from hprqp import instances

CASES = {inst.name: inst for inst in instances.tiny_cases()}


def _small(name):
    if name in CASES:
        return CASES[name]
    if name == "small_free":
        inst = instances.plain_qp(0x48505251 + 90100, n=50, m=20, a_density=0.1, m_rows=10, m_density=0.1,
                                  n_eq=12, name="small_free")
        inst.l[:] = -np.inf
        inst.u[:] = np.inf
        return inst
    k = int(name.split("_")[1])
    return instances.plain_qp(0x48505251 + 90000 + k, n=60, m=30, a_density=0.1, m_rows=12, m_density=0.1,
                              n_eq=18, name=name)


def test_one_step_closed_form():
    """tests/cpu/test_iteration.c:53-91 (STANDARD case, no scaling, one full step)."""
    om = pyoracle.OracleModel(CASES["standard"])
    r = om.solve(max_iter=1, print_frequency=1, use_scaling=False, mode=pyoracle.MODE_CPU_REF)
    sigma = 2.0 / math.sqrt(5.0)
    ybar = 2.0 / (2.1 * sigma)
    assert abs(r["x"][0]) < 1e-12 and abs(r["x"][1]) < 1e-12
    assert abs(r["z"][0] - 2.0) < 1e-12 and abs(r["z"][1] - 1.0) < 1e-12
    assert abs(r["y"][0] - ybar) < 1e-12
    assert abs(r["w"][0] - sigma / (1 + 2 * sigma) * ybar) < 1e-12
    assert abs(r["w"][1] - sigma / (1 + 4 * sigma) * ybar) < 1e-12


def test_python_analytic_optimum():
    """python/tests/test_hprqp.py:26-42: min x1^2 + x2^2 - 4x1 - 2x2 -> -5 at (2, 1)."""
    inst = instances.tiny_cases()[0]
    Q = instances.CSR(2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([2.0, 2.0]))
    A = instances.CSR(0, 2, np.array([0]), np.zeros(0, np.int64), np.zeros(0))
    q = instances.QPInstance(Q, A, np.array([-4.0, -2.0]), np.zeros(0), np.zeros(0), np.full(2, -np.inf),
                             np.full(2, np.inf))
    for mode in (pyoracle.MODE_CPU_REF, pyoracle.MODE_GPU_REF):
        r = pyoracle.OracleModel(q).solve(stoptol=1e-8, mode=mode)
        assert r["status"] == 6
        assert abs(r["primal_obj"] + 5.0) < 1e-6
        assert abs(r["x"][0] - 2.0) < 1e-6 and abs(r["x"][1] - 1.0) < 1e-6


def _check(rec, r, tol):
    assert r["status"] == rec["status"], (rec["name"], rec["max_iter"])
    assert r["iter"] == rec["iter"]
    for key in ("x", "y", "z", "w"):
        a, b = np.asarray(r[key]), np.asarray(rec[key])
        assert a.shape == b.shape
        if a.size:
            assert np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(b))), (rec["name"], key)
    assert abs(r["primal_obj"] - rec["objective"]) <= tol * max(1.0, abs(rec["objective"]))


def test_oracle_cpu_mode_bit_exact(golden):
    for rec in golden:
        inst = _small(rec["name"])
        cap = rec["max_iter"] if rec["max_iter"] is not None else 2147483647
        r = pyoracle.OracleModel(inst).solve(stoptol=rec["stoptol"], max_iter=cap, mode=pyoracle.MODE_CPU_REF)
        _check(rec, r, 0.0)
        assert r["iter_4"] == rec["iter_4"] and r["iter_6"] == rec["iter_6"]


def test_oracle_gpu_mode_close(golden):
    """GPU-reference semantics differ from the CPU backend only in rounding
    details and in which bars a non-check step refreshes, so converged
    answers agree to the solve tolerance."""
    for rec in golden:
        if rec["max_iter"] is not None:
            continue
        inst = _small(rec["name"])
        r = pyoracle.OracleModel(inst).solve(stoptol=rec["stoptol"], mode=pyoracle.MODE_GPU_REF)
        assert r["status"] == rec["status"] == 6
        assert abs(r["primal_obj"] - rec["objective"]) <= 1e-6 * max(1.0, abs(rec["objective"]))


def test_kkt_recompute_matches_solver_residual(golden):
    """The host FP64 KKT recomputation in the original space reproduces the
    solver's own residual bookkeeping (src/cpu/residuals.c:123-189)."""
    for rec in golden:
        if rec["max_iter"] is not None or rec["name"] in ("tall_diag",):
            continue
        inst = _small(rec["name"])
        om = pyoracle.OracleModel(inst)
        r = om.solve(stoptol=rec["stoptol"], mode=pyoracle.MODE_GPU_REF)
        k = om.kkt(r["x"], r["y"], r["z"])
        assert k["kkt"] <= 1.5 * rec["stoptol"] + 1e-14, (rec["name"], k)
        assert abs(k["primal_obj"] - r["primal_obj"]) <= 1e-9 * max(1.0, abs(r["primal_obj"]))


def test_oracle_rejects_invalid_models():
    inst = CASES["standard"]
    bad = instances.QPInstance(inst.Q, inst.A, inst.c.copy(), inst.AL.copy(), inst.AU.copy(), inst.l.copy(),
                               inst.u.copy())
    bad.l[0] = 20.0  # l > u
    with pytest.raises(ValueError):
        pyoracle.OracleModel(bad)
    bad2 = instances.QPInstance(inst.Q, inst.A, inst.c.copy(), inst.AL.copy(), inst.AU.copy(), inst.l.copy(),
                                inst.u.copy())
    bad2.c[1] = np.nan
    with pytest.raises(ValueError):
        pyoracle.OracleModel(bad2)
