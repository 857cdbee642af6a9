"""Convex QCQPs from MPS (diagonal QCMATRIX rows lifted to second-order
cones) solved on the GPU: this engine against the reference's own GPU build
(its solve_gpu on the model its own reader built from the same file), and
every quadratic constraint of the file checked at the solution."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp.instances import CSR, QPInstance
from mps_cases import random_qcqp_mps

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (pyoracle.ref_available() and pyoracle.ref_gpu_available()),
                                 reason="reference libraries not built")]


@pytest.mark.parametrize("seed", range(3))
def test_qcqp_mps_matches_reference_gpu(engine_lib, tmp_path, seed):
    hprqp = engine_lib
    p = tmp_path / f"qc{seed}.mps"
    p.write_text(random_qcqp_mps(seed))
    r = hprqp.optimize(hprqp.read_from_mps(p), hprqp.Parameters(verbose=False, stoptol=1e-8))
    assert r.status_code == hprqp.STATUS_OPTIMAL
    m = pyoracle.ref_build_from_mps(p)
    inst = QPInstance(CSR(m["n"], m["n"], m["q_indptr"], m["q_indices"], m["q_data"]),
                      CSR(m["m"], m["n"], m["a_indptr"], m["a_indices"], m["a_data"]),
                      m["c"], m["AL"], m["AU"], m["l"], m["u"], m["obj_constant"])
    ref = pyoracle.RefGpuModel(inst, soc=(None, m["row_cone_offsets"], m["soc_rhs"])).solve(stoptol=1e-8)
    assert ref["status"] == hprqp.STATUS_OPTIMAL
    assert abs(r.objective - ref["primal_obj"]) <= 1e-6 * max(1.0, abs(ref["primal_obj"]))
    x = np.asarray(r.x)
    assert np.allclose(x, ref["x"], atol=1e-4)
    # each lifted cone: t >= |v| at the solution, i.e. the quadratic row holds
    A = inst.A.to_scipy()
    s = A @ x - m["soc_rhs"]
    off = m["row_cone_offsets"]
    for k in range(len(off) - 1):
        t, v = s[off[k]], s[off[k] + 1:off[k + 1]]
        assert np.linalg.norm(v) <= t + 1e-6 * max(1.0, abs(t)), k
