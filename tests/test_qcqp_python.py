"""hprqp.build_from_qabc_qc on CPU: the same QCQP built from arrays (with the
diagonal D or with factors R) and read from an MPS file with QCMATRIX rows
gives the same lifted model (for a row  a x + x'Hx <= u  the reader uses
C = a, D = 2H, constant = -u)."""
from __future__ import annotations

import numpy as np
import pytest


def _mps():
    return "\n".join([
        "NAME QCPY", "ROWS", " N obj", " L lin", " L q1", " L q2", "COLUMNS",
        "    x obj 1.5 lin 1", "    x q1 0.5", "    y obj -1 lin 1", "    y q2 -0.25", "    z obj 0.5 q1 1",
        "RHS", "    rhs lin 2 q1 3", "    rhs q2 1.5", "BOUNDS", " FR b x", " FR b y", " LO b z -1", " UP b z 4",
        "QUADOBJ", "    x x 2", "    y y 1", "    z z 3",
        "QCMATRIX q1", "    x x 1", "    z z 0.5", "QCMATRIX q2", "    y y 2", "ENDATA"]) + "\n"


def _arrays(hprqp, model):
    a = hprqp.model_arrays(model)
    return {k: np.asarray(v) for k, v in a.items()}


@pytest.mark.parametrize("form", ["diagonal", "factors"])
def test_python_builder_equals_mps_reader(engine_lib, tmp_path, form):
    hprqp = engine_lib
    p = tmp_path / "q.mps"
    p.write_text(_mps())
    ref = _arrays(hprqp, hprqp.read_from_mps(p))
    inf = np.inf
    Q = np.diag([2.0, 1.0, 3.0])
    A = [[1.0, 1.0, 0.0]]
    C = [[0.5, 0.0, 1.0], [0.0, -0.25, 0.0]]
    kw = dict(Q=Q, c=[1.5, -1.0, 0.5], A=A, AL=[-inf], AU=[2.0], l=[-inf, -inf, -1.0], u=[inf, inf, 4.0], C=C,
              constant=[-3.0, -1.5])
    if form == "diagonal":
        m = hprqp.build_from_qabc_qc(D=[[2.0, 0.0, 1.0], [0.0, 4.0, 0.0]], **kw)
    else:  # R_i rows sqrt(d) e_j, as the diagonal form builds them
        R = [[np.sqrt(2.0), 0, 0], [0, 0, 1.0], [0, np.sqrt(4.0), 0]]
        m = hprqp.build_from_qabc_qc(R=R, offsets=[0, 2, 3], **kw)
    got = _arrays(hprqp, m)
    for k in ref:
        assert np.array_equal(got[k], ref[k]), k
    assert int(got["num_row_cones"]) == 2


def test_python_builder_arguments(engine_lib):
    hprqp = engine_lib
    with pytest.raises(ValueError):
        hprqp.build_from_qabc_qc(np.eye(2), [0, 0], [], [], [], [0, 0], [1, 1], [[1.0, 0.0]], [0.0])
    with pytest.raises(ValueError):
        hprqp.build_from_qabc_qc(np.eye(2), [0, 0], [], [], [], [0, 0], [1, 1], [[1.0, 0.0]], [0.0],
                                 R=[[1.0, 0.0]], offsets=[0])
    with pytest.raises(RuntimeError, match="INVALID_ARGUMENT"):  # a negative diagonal is not convex
        hprqp.build_from_qabc_qc(np.eye(2), [0, 0], [], [], [], [0, 0], [1, 1], [[1.0, 0.0]], [0.0],
                                 D=[[-1.0, 0.0]])
