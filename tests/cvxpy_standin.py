"""A stand-in for the few parts of CVXPY that hprqp.cvxpy_bridge touches,
for tests only (cvxpy is not installed here).  A ``Problem`` is given by
its canonical OSQP data -- minimize 1/2 z'Pz + q'z + const subject to
A z = b and F z <= G over the problem's variables stacked column-major --
and answers ``get_problem_data(OSQP)`` with the dict CVXPY returns for
such a problem (keys P, q, A, b, F, G, n_var, param_prob.var_id_to_col,
bool_vars_idx, int_vars_idx).  Installed as ``sys.modules["cvxpy"]`` by
the tests that use it."""
from __future__ import annotations

import itertools
import types

import numpy as np
import scipy.sparse as sp

_ids = itertools.count(101)


class Variable:
    def __init__(self, shape=()):
        self.shape = (shape,) if isinstance(shape, int) else tuple(shape)
        self.size = int(np.prod(self.shape)) if self.shape else 1
        self.id = next(_ids)
        self.value = None


class _Expr:
    def __init__(self, fn):
        self._fn = fn

    @property
    def value(self):
        return self._fn()


class _Objective:
    def __init__(self, name, fn):
        self.NAME = name
        self.expr = _Expr(fn)


class _ParamProb:
    def __init__(self, var_id_to_col):
        self.var_id_to_col = var_id_to_col


class Problem:
    def __init__(self, variables, P, q, const, A=None, b=(), F=None, G=(), sense="minimize", extra_columns=0,
                 int_idx=()):
        self._vars = list(variables)
        cols, off = {}, 0
        for v in self._vars:
            cols[v.id] = off
            off += v.size
        n = off + extra_columns
        P = np.asarray(P, float)
        q = np.asarray(q, float)
        self._data = {"P": sp.csc_matrix(P), "q": q,
                      "A": sp.csc_matrix(np.zeros((0, n)) if A is None else np.asarray(A, float)),
                      "b": np.asarray(b, float),
                      "F": sp.csc_matrix(np.zeros((0, n)) if F is None else np.asarray(F, float)),
                      "G": np.asarray(G, float), "n_var": n, "param_prob": _ParamProb(cols),
                      "bool_vars_idx": [], "int_vars_idx": list(int_idx)}

        def objective():
            if any(v.value is None for v in self._vars):
                return None
            z = np.concatenate([np.ravel(np.asarray(v.value, float), order="F") for v in self._vars])
            return 0.5 * z @ (P[:off, :off] @ z) + q[:off] @ z + const

        self.objective = _Objective(sense, objective)

    def variables(self):
        return list(self._vars)

    def is_qp(self):
        return True

    def get_problem_data(self, solver):
        assert solver == "OSQP"
        return self._data, None, None


def module():
    m = types.ModuleType("cvxpy")
    m.OSQP = "OSQP"
    m.Variable = Variable
    m.Problem = Problem
    return m


def reference_example():
    """The reference's own CVXPY test problem (python/tests/
    test_cvxpy_integration.py:16-30): minimize 1/2 x'diag(2,2)x - [2,4]x +
    y^2 - 6y + 21 s.t. x0 + y = 4, x1 >= 1, y >= 0.5; optimum x = (1, 2),
    y = 3, objective 7."""
    x, y = Variable(2), Variable()
    P = np.diag([2.0, 2.0, 2.0])
    q = [-2.0, -4.0, -6.0]
    prob = Problem([x, y], P, q, 21.0, A=[[1.0, 0.0, 1.0]], b=[4.0], F=[[0.0, -1.0, 0.0], [0.0, 0.0, -1.0]],
                   G=[-1.0, -0.5])
    return prob, x, y
