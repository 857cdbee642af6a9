"""CVXPY problems in, solutions out (the reference binding's CVXPY bridge,
python/src/hprqp/__init__.py:441-573, with the same functions and rules).

A ``cvxpy.Problem`` is canonicalised by CVXPY for OSQP, whose data are

    minimize 1/2 x'Px + q'x   s.t.   A x = b,   F x <= G

over the problem's own variables stacked in one vector.  That is an HPR QP
with free variables and the rows [A; F] bounded by [b; -inf] and [b; G];
the objective constant is the objective's value at x = 0.  The reference
rejects problems CVXPY had to extend with auxiliary variables (their
values could not be handed back), maximisation, non-QP and mixed-integer
problems; so does this bridge.  CVXPY is imported only when a function of
this module is called.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Dict, Optional, Sequence, Tuple


@dataclass(frozen=True)
class CVXPYBuildInfo:
    """Where each CVXPY variable sits in the solver's vector."""
    variable_offsets: Dict[int, int]
    variable_shapes: Dict[int, Tuple[int, ...]]
    num_variables: int
    num_constraints: int
    objective_constant: float


def _cvxpy():
    try:
        import cvxpy
    except ImportError as exc:
        raise RuntimeError("CVXPY support needs the cvxpy package, which is not installed") from exc
    return cvxpy


def _osqp_data(problem, cp) -> Dict[str, Any]:
    for attr in ("get_problem_data", "variables", "objective"):
        if not hasattr(problem, attr):
            raise TypeError("expected a cvxpy.Problem")
    if str(getattr(problem.objective, "NAME", "")).lower() != "minimize":
        raise ValueError("only minimisation problems are supported")
    if hasattr(problem, "is_qp") and not problem.is_qp():
        raise ValueError("only convex quadratic problems are supported")
    out = problem.get_problem_data(cp.OSQP)
    data = out[0] if isinstance(out, tuple) else out
    if not isinstance(data, dict):
        raise RuntimeError("unexpected output of CVXPY's canonicalisation")
    if len(data.get("bool_vars_idx") or ()) or len(data.get("int_vars_idx") or ()):
        raise ValueError("mixed-integer problems are not supported")
    return data


def _constant_at_zero(problem) -> float:
    """The objective at x = 0, every variable's value restored afterwards."""
    import numpy as np

    variables = list(problem.variables())
    saved = [None if v.value is None else np.array(v.value, copy=True) for v in variables]
    try:
        for v in variables:
            v.value = 0.0 if v.shape == () else np.zeros(v.shape, order="F")
        value = problem.objective.expr.value
        if value is None:
            raise RuntimeError("the objective could not be evaluated at zero")
        return float(value)
    finally:
        for v, old in zip(variables, saved):
            v.value = old


def build_from_cvxpy_problem(problem) -> Tuple["Model", CVXPYBuildInfo]:  # noqa: F821
    """(model, info) for a CVXPY QP; see the module docstring."""
    import scipy.sparse as sp

    from . import build_from_qabc

    cp = _cvxpy()
    data = _osqp_data(problem, cp)
    variables = list(problem.variables())
    n = int(data["n_var"])
    if n != sum(int(v.size) for v in variables):
        raise ValueError("CVXPY added auxiliary variables to this problem; write it as a QP in its own variables "
                         "(explicit quadratic and affine terms)")
    to_col = {int(k): int(c) for k, c in data["param_prob"].var_id_to_col.items()}
    if any(int(v.id) not in to_col for v in variables):
        raise ValueError("a CVXPY variable has no column in the canonical data")
    P = sp.csr_matrix(data["P"])
    A_eq, F = sp.csr_matrix(data["A"]), sp.csr_matrix(data["F"])
    b, G = [float(v) for v in data["b"]], [float(v) for v in data["G"]]
    blocks = [M for M in (A_eq, F) if M.shape[0] > 0]
    A = sp.vstack(blocks, format="csr") if blocks else sp.csr_matrix((0, n))
    AL = b + [-math.inf] * F.shape[0]
    AU = b + G
    const = _constant_at_zero(problem)
    model = build_from_qabc(P, data["q"], A, AL, AU, [-math.inf] * n, [math.inf] * n, obj_constant=const)
    info = CVXPYBuildInfo({int(v.id): to_col[int(v.id)] for v in variables},
                          {int(v.id): tuple(int(d) for d in v.shape) for v in variables}, n, int(A.shape[0]), const)
    return model, info


def write_values(problem, info: CVXPYBuildInfo, x: Sequence[float]) -> None:
    """Write a solution vector back into the problem's variables
    (column-major, as CVXPY vectorises)."""
    import numpy as np

    x = np.asarray(x, dtype=float)
    for v in problem.variables():
        start = info.variable_offsets[int(v.id)]
        part = x[start:start + int(v.size)]
        v.value = float(part[0]) if v.shape == () else part.reshape(v.shape, order="F")


def solve_cvxpy_problem(problem, params: Optional["Parameters"] = None,  # noqa: F821
                        assign_values: bool = True) -> "Result":  # noqa: F821
    """Build, solve with solve_gpu, and (by default) write the solution into
    the problem's variables; ``assign_values=False`` leaves them alone."""
    from . import optimize

    model, info = build_from_cvxpy_problem(problem)
    result = optimize(model, params)
    if assign_values:
        write_values(problem, info, result.x)
    return result
