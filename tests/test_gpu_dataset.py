"""The dataset runner on real MPS files: per file (solve_gpu) and as one
batch (hprqp_batch.h).  Both tables must hold the same optima as a direct
solve of each file, rejected files must carry the reader's status, and the
summary rows must count the solved files."""
from __future__ import annotations

import numpy as np
import pytest

import mps_cases
from hprqp import dataset, instances

pytestmark = pytest.mark.gpu


def _folder(tmp_path):
    data = tmp_path / "data"
    data.mkdir()
    for k in range(3):
        (data / f"qp{k}.mps").write_text(mps_cases.write_instance(instances.adjoint_case(k)))
    (data / "bad.mps").write_text(mps_cases.malformed()["bad_number"])
    (data / "quad_rows.mps").write_text(mps_cases.random_qcqp_mps(3))  # second-order cones after the lift
    (data / "nonconvex.mps").write_text(mps_cases.malformed_qcqp()["nonconvex_le"])
    return data


def test_dataset_runner_per_file_and_batched(engine_lib, tmp_path):
    hprqp = engine_lib
    data = _folder(tmp_path)
    tables = {}
    for mode, extra in (("each", []), ("batch", ["--batch"])):
        out = tmp_path / mode
        assert dataset.main([str(data), str(out), "--stoptol", "1e-8"] + extra) == 0
        tables[mode] = {r["name"]: r for r in dataset.read_table(out / dataset.CSV_NAME)}
        lines = (out / dataset.CSV_NAME).read_text().splitlines()
        assert lines[-2].startswith("SGM10,") and lines[-1].startswith("solved,,4,")
        assert "qp0.mps" in (out / dataset.LOG_NAME).read_text()
    for mode, rows in tables.items():
        assert sorted(rows) == ["bad.mps", "nonconvex.mps", "qp0.mps", "qp1.mps", "qp2.mps", "quad_rows.mps"]
        assert rows["bad.mps"]["status"] == rows["nonconvex.mps"]["status"] == "INVALID_ARGUMENT"
        assert rows["quad_rows.mps"]["status"] == "OPTIMAL" and rows["quad_rows.mps"]["row_cones"] == "4"
        direct = hprqp.optimize(hprqp.read_from_mps(data / "quad_rows.mps"),
                                hprqp.Parameters(verbose=False, stoptol=1e-8))
        tol = 1e-6 * max(1.0, abs(direct.objective))
        assert abs(float(rows["quad_rows.mps"]["primal_obj"]) - direct.objective) <= tol
        for k in range(3):
            r = rows[f"qp{k}.mps"]
            assert r["status"] == "OPTIMAL", (mode, r)
            direct = hprqp.optimize(hprqp.read_from_mps(data / f"qp{k}.mps"),
                                    hprqp.Parameters(verbose=False, stoptol=1e-8))
            assert abs(float(r["primal_obj"]) - direct.objective) <= 1e-6 * max(1.0, abs(direct.objective))
            assert float(r["alg_time"]) > 0 and float(r["res"]) < 1e-8
    # the per-file path runs solve_gpu itself: same iteration counts
    for k in range(3):
        direct = hprqp.optimize(hprqp.read_from_mps(data / f"qp{k}.mps"),
                                hprqp.Parameters(verbose=False, stoptol=1e-8))
        assert int(tables["each"][f"qp{k}.mps"]["iter"]) == direct.iter


def test_batch_instance_times(engine_lib):
    from hprqp import batch

    b = batch.Batch([instances.config3_instance(k) for k in range(90, 96)])
    ms = b.solve(stoptol=1e-6)
    r = b.results(vectors=False)
    b.close()
    assert np.all(r.seconds > 0)
    assert np.all(r.seconds <= ms / 1e3 * 1.01 + 1e-3)


def test_model_to_instance_round_trip(engine_lib):
    """a built model's arrays, solved as a batch of one, give the model's own solve"""
    hprqp = engine_lib
    from hprqp import batch

    inst = instances.adjoint_case(5)
    model = hprqp.build_from_instance(inst)
    again = model.to_instance("x")
    assert again.n == inst.n and again.m <= inst.m
    direct = hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=1e-8))
    r = batch.solve_batch([again], stoptol=1e-8)
    assert r.status[0] == 6
    assert abs(r.objective[0] - direct.objective) <= 1e-6 * max(1.0, abs(direct.objective))
