"""build_from_mps against the reference's own MPS reader (its CPU library,
oracle/_ref) on seeded MPS files written by tests/mps_cases.py: the two
libraries must return bit-identical models, and reject the same malformed
files."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import pyoracle
from mps_cases import malformed, malformed_qcqp, random_mps, random_qcqp_mps

needs_ref = pytest.mark.skipif(not pyoracle.ref_available(), reason="reference CPU library not built")


def _ours(hprqp, path):
    try:
        model = hprqp.build_from_mps(path)
    except RuntimeError as err:
        return {"status": str(err)}
    out = hprqp.model_arrays(model)
    out["status"] = 0
    return out


def _same(a, b):
    for k in ("n", "m", "obj_constant", "num_var_cones", "num_row_cones"):
        assert a[k] == b[k], k
    for k in ("q_indptr", "q_indices", "q_data", "a_indptr", "a_indices", "a_data", "c", "l", "u", "AL", "AU",
              "row_cone_offsets", "soc_rhs"):
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert x.shape == y.shape, k
        assert np.array_equal(x, y, equal_nan=True), k


@needs_ref
@pytest.mark.parametrize("quad", ["QUADOBJ", "QMATRIX", ""])
@pytest.mark.parametrize("seed", range(6))
def test_models_identical_to_reference(engine_lib, tmp_path, seed, quad):
    p = tmp_path / f"g{seed}.mps"
    p.write_text(random_mps(seed, n=10 + seed, m=6 + seed, quad=quad))
    ref = pyoracle.ref_build_from_mps(p)
    assert ref["status"] == 0
    ours = _ours(engine_lib, p)
    assert ours["status"] == 0
    _same(ours, ref)


@needs_ref
@pytest.mark.parametrize("name", sorted(malformed()))
def test_malformed_rejected_like_reference(engine_lib, tmp_path, name):
    p = tmp_path / f"{name}.mps"
    p.write_text(malformed()[name])
    ref = pyoracle.ref_build_from_mps(p)
    ours = _ours(engine_lib, p)
    assert ref["status"] != 0
    assert ours["status"] != 0


def test_missing_file(engine_lib, tmp_path):
    assert _ours(engine_lib, tmp_path / "absent.mps")["status"] != 0


@pytest.mark.gpu
def test_solve_from_mps_matches_arrays(engine_lib, tmp_path):
    """The n=1000 seeded QP written as MPS, read back and solved on the GPU:
    same model (up to the ranged rows' AL + (AU - AL) rounding) and the same
    objective as the model built from the arrays."""
    from mps_cases import write_instance

    from hprqp import instances

    hprqp = engine_lib
    inst = instances.config0()
    p = tmp_path / "config0.mps"
    p.write_text(write_instance(inst))
    m1 = hprqp.build_from_mps(p)
    m2 = hprqp.build_from_instance(inst)
    a1, a2 = hprqp.model_arrays(m1), hprqp.model_arrays(m2)
    for k in ("q_indptr", "q_indices", "q_data", "a_indptr", "a_indices", "a_data", "c", "l", "u", "AL"):
        assert np.array_equal(a1[k], a2[k]), k
    assert np.allclose(a1["AU"], a2["AU"], rtol=1e-12, atol=1e-14)
    r1 = hprqp.optimize(m1, hprqp.Parameters(verbose=False, stoptol=1e-6))
    r2 = hprqp.optimize(m2, hprqp.Parameters(verbose=False, stoptol=1e-6))
    assert r1.status_code == r2.status_code == hprqp.STATUS_OPTIMAL
    assert abs(r1.objective - r2.objective) <= 1e-6 * abs(r2.objective)


def test_reference_fixture_model(engine_lib):
    """the reference's own tests/data/simple_qp.mps: the model equals what
    the reference's reader built from it (tests/golden/simple_qp.json, made
    by tests/golden/make_reference_fixtures.py)"""
    import json

    golden = Path(__file__).resolve().parent / "golden"
    ref = json.loads((golden / "simple_qp.json").read_text())["model"]
    got = engine_lib.read_from_mps(golden / "simple_qp.mps").to_instance()
    assert (got.n, got.m) == (ref["n"], ref["m"]) and got.obj_constant == ref["obj_constant"]
    for mine, key in ((got.Q.indptr, "q_indptr"), (got.Q.indices, "q_indices"), (got.Q.data, "q_data"),
                      (got.A.indptr, "a_indptr"), (got.A.indices, "a_indices"), (got.A.data, "a_data"),
                      (got.c, "c"), (got.l, "l"), (got.u, "u"), (got.AL, "AL"), (got.AU, "AU")):
        assert np.array_equal(np.asarray(mine, float), np.asarray(ref[key], float)), key


@needs_ref
@pytest.mark.parametrize("seed", range(6))
def test_qcqp_models_identical_to_reference(engine_lib, tmp_path, seed):
    """QCMATRIX rows lifted to second-order cones exactly as the reference's
    reader and builder do (src/shared/mps_qp.cpp:119-206, qcqp.c)"""
    p = tmp_path / f"qc{seed}.mps"
    p.write_text(random_qcqp_mps(seed, n=8 + seed, m=6 + seed % 3))
    ref = pyoracle.ref_build_from_mps(p)
    assert ref["status"] == 0 and ref["num_row_cones"] == 4
    ours = _ours(engine_lib, p)
    assert ours["status"] == 0
    _same(ours, ref)


@needs_ref
@pytest.mark.parametrize("name", sorted(malformed_qcqp()))
def test_qcqp_malformed_rejected_like_reference(engine_lib, tmp_path, name):
    p = tmp_path / f"{name}.mps"
    p.write_text(malformed_qcqp()[name])
    assert pyoracle.ref_build_from_mps(p)["status"] != 0
    assert _ours(engine_lib, p)["status"] != 0
