"""CVXPY bridge on the GPU: the reference test's known answers
(python/tests/test_cvxpy_integration.py:48-57: objective 7, x = (1, 2),
y = 3, values written into the variables) and, for its second problem
(lines 59-80, where the reference compares its CPU and GPU paths), the
oracle's solve of the same model.  cvxpy is not installed here: the
canonical data come from tests/cvxpy_standin.py."""
from __future__ import annotations

import sys

import numpy as np
import pytest

import cvxpy_standin as cs
import pyoracle

pytestmark = pytest.mark.gpu


@pytest.fixture
def cvxpy(monkeypatch):
    monkeypatch.setitem(sys.modules, "cvxpy", cs.module())


def test_solve_assigns_values(engine_lib, cvxpy):
    hprqp = engine_lib
    prob, x, y = cs.reference_example()
    r = hprqp.solve_cvxpy_problem(prob, hprqp.Parameters(verbose=False, stoptol=1e-9))
    assert r.status_code == hprqp.STATUS_OPTIMAL
    assert r.objective == pytest.approx(7.0, abs=1e-6)
    assert x.value == pytest.approx([1.0, 2.0], abs=1e-6)
    assert float(y.value) == pytest.approx(3.0, abs=1e-6)


def test_second_problem_against_oracle(engine_lib, cvxpy):
    hprqp = engine_lib
    x = cs.Variable(2)
    prob = cs.Problem([x], [[2.0, 0.0], [0.0, 4.0]], [2.0, 1.0], 0.0, A=[[1.0, 1.0]], b=[2.0], F=-np.eye(2),
                      G=[0.0, 0.0])
    r = hprqp.solve_cvxpy_problem(prob, hprqp.Parameters(verbose=False, stoptol=1e-9), assign_values=False)
    assert x.value is None
    model, _ = hprqp.build_from_cvxpy_problem(prob)
    o = pyoracle.OracleModel(model.to_instance()).solve(stoptol=1e-9)
    assert r.status_code == o["status"] == hprqp.STATUS_OPTIMAL
    assert r.objective == pytest.approx(o["primal_obj"], abs=1e-6)
    assert np.allclose(r.x, o["x"], atol=1e-6)
    # the analytic optimum: x = (7/6, 5/6)
    assert np.allclose(r.x, [7.0 / 6.0, 5.0 / 6.0], atol=1e-6)
