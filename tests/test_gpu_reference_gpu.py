"""The plain GPU path against the reference's own GPU backend.

The reference's CUDA solver (cuSPARSE SpMV, cuBLAS reductions; built from
its sources for sm_100a by ``make -C oracle ref-gpu``, polishing and the
Gram path off) and this engine's ``solve_gpu`` solve the same seeded
instances: both must reach the tolerance, the objectives must agree within
1e-6 relative, and the KKT residual of this engine's solution, recomputed in
FP64 on the host from the original model, must be below the tolerance.
Iterates are not compared entry by entry: the two SpMVs round differently
(cuSPARSE's summation order is not ours), so trajectories drift apart
within rounding and then converge to the same optimum."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not pyoracle.ref_gpu_available(),
                                 reason="reference GPU library not built (make -C oracle ref-gpu)")]

CASES = [instances.config0(), instances.config3_instance(0), instances.config3_instance(7),
         instances.config3_instance(21), instances.config4_instance(0), instances.adjoint_case(0)]
TINY = [i for i in instances.tiny_cases() if i.name not in ("tall_diag", "zero_1d")]


def _ours(hprqp, inst, stoptol):
    model = hprqp.build_from_instance(inst)
    return hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=stoptol), as_numpy=True)


@pytest.mark.parametrize("stoptol", [1e-6, 1e-8])
@pytest.mark.parametrize("inst", CASES, ids=[i.name for i in CASES])
def test_plain_matches_reference_gpu(engine_lib, inst, stoptol):
    ref = pyoracle.RefGpuModel(inst).solve(stoptol=stoptol)
    assert ref["ret"] == ref["status"] == engine_lib.STATUS_OPTIMAL, ref["status"]
    r = _ours(engine_lib, inst, stoptol)
    assert r.status_code == engine_lib.STATUS_OPTIMAL
    assert abs(r.objective - ref["primal_obj"]) <= 1e-6 * max(1.0, abs(ref["primal_obj"]))
    k = pyoracle.OracleModel(inst).kkt(r.x, r.y, r.z)
    assert k["kkt"] <= stoptol * 1.01
    # the reference's own solution satisfies the same host check
    kr = pyoracle.OracleModel(inst).kkt(ref["x"], ref["y"], ref["z"])
    assert kr["kkt"] <= stoptol * 1.01


@pytest.mark.parametrize("inst", TINY, ids=[i.name for i in TINY])
def test_fixture_models_match_reference_gpu(engine_lib, inst):
    ref = pyoracle.RefGpuModel(inst).solve(stoptol=1e-8)
    r = _ours(engine_lib, inst, 1e-8)
    assert r.status_code == ref["status"] == engine_lib.STATUS_OPTIMAL
    assert abs(r.objective - ref["primal_obj"]) <= 1e-6 * max(1.0, abs(ref["primal_obj"]))
    assert np.max(np.abs(r.x - ref["x"]), initial=0.0) <= 1e-5 * max(1.0, float(np.max(np.abs(ref["x"]),
                                                                                        initial=0.0)))


def test_batched_matches_reference_gpu(engine_lib):
    """The batched solver against the reference GPU solve of each member."""
    from hprqp import batch

    insts = [instances.config3_instance(i) for i in range(8)]
    r = batch.solve_batch(insts, stoptol=1e-6)
    for k, inst in enumerate(insts):
        ref = pyoracle.RefGpuModel(inst).solve(stoptol=1e-6)
        assert r.status[k] == ref["status"] == engine_lib.STATUS_OPTIMAL
        assert abs(r.objective[k] - ref["primal_obj"]) <= 1e-6 * max(1.0, abs(ref["primal_obj"]))
