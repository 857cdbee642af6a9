"""hprqp.cvxpy_bridge on CPU: the canonical OSQP data of a CVXPY problem
become the HPR model (rows [A; F], bounds [b, b] and [-inf, G], free
variables, the objective at zero as constant), with the reference's checks
(python/src/hprqp/__init__.py:441-573).  cvxpy is not installed here, so a
stand-in module (tests/cvxpy_standin.py) supplies the canonical data of the
reference's own test problem."""
from __future__ import annotations

import sys

import numpy as np
import pytest

import cvxpy_standin as cs


@pytest.fixture
def cvxpy(monkeypatch):
    mod = cs.module()
    monkeypatch.setitem(sys.modules, "cvxpy", mod)
    return mod


def test_build_matches_the_reference_test_expectations(engine_lib, cvxpy):
    hprqp = engine_lib
    prob, x, y = cs.reference_example()
    x.value = np.array([5.0, 6.0])  # restored after the constant is evaluated
    model, info = hprqp.build_from_cvxpy_problem(prob)
    assert (model.num_variables, model.num_constraints) == (info.num_variables, info.num_constraints) == (3, 3)
    assert info.variable_offsets == {x.id: 0, y.id: 2}
    assert info.variable_shapes == {x.id: (2,), y.id: ()}
    assert info.objective_constant == pytest.approx(21.0)
    assert np.array_equal(x.value, [5.0, 6.0]) and y.value is None
    inst = model.to_instance()
    assert np.allclose(inst.Q.dense(), np.diag([2.0, 2.0, 2.0]))
    assert np.array_equal(inst.c, [-2.0, -4.0, -6.0])
    assert np.array_equal(inst.A.dense(), [[1, 0, 1], [0, -1, 0], [0, 0, -1]])
    assert np.array_equal(inst.AL, [4.0, -np.inf, -np.inf]) and np.array_equal(inst.AU, [4.0, -1.0, -0.5])
    assert np.all(np.isneginf(inst.l)) and np.all(np.isposinf(inst.u))
    assert inst.obj_constant == 21.0


def test_rejections(engine_lib, cvxpy):
    hprqp = engine_lib
    x = cs.Variable(2)
    P, q = np.eye(2), np.ones(2)
    with pytest.raises(ValueError, match="minimisation"):
        hprqp.build_from_cvxpy_problem(cs.Problem([x], P, q, 0.0, sense="maximize"))
    with pytest.raises(ValueError, match="auxiliary"):
        hprqp.build_from_cvxpy_problem(cs.Problem([x], np.eye(3), np.ones(3), 0.0, extra_columns=1))
    with pytest.raises(ValueError, match="mixed-integer"):
        hprqp.build_from_cvxpy_problem(cs.Problem([x], P, q, 0.0, int_idx=[0]))
    with pytest.raises(TypeError):
        hprqp.build_from_cvxpy_problem(object())


def test_missing_cvxpy_is_a_clear_error(engine_lib, monkeypatch):
    hprqp = engine_lib
    monkeypatch.setitem(sys.modules, "cvxpy", None)
    with pytest.raises(RuntimeError, match="cvxpy"):
        hprqp.build_from_cvxpy_problem(cs.reference_example()[0])


def test_values_written_column_major(engine_lib, cvxpy):
    from hprqp import cvxpy_bridge

    M, s = cs.Variable((2, 3)), cs.Variable()
    prob = cs.Problem([s, M], np.eye(7), np.zeros(7), 0.0)
    info = cvxpy_bridge.CVXPYBuildInfo({s.id: 0, M.id: 1}, {s.id: (), M.id: (2, 3)}, 7, 0, 0.0)
    cvxpy_bridge.write_values(prob, info, np.arange(7.0))
    assert s.value == 0.0
    assert np.array_equal(M.value, np.array([[1.0, 3.0, 5.0], [2.0, 4.0, 6.0]]))
