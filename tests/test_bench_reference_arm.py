"""bench.py --impl reference on CPU (it runs the reference's own CPU build,
oracle/_ref, on a bounded sample): one JSON line with the contract's keys,
the metric and config of the GPU arm, impl "reference", a cpu_baseline
describing the run and an e2e block with zero transfer bytes."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import pytest

import pyoracle

ROOT = Path(__file__).resolve().parents[1]


@pytest.mark.skipif(not pyoracle.ref_available(), reason="reference CPU library not built")
def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup",
                          "0", "--cpu-sample", "8"], capture_output=True, text=True, timeout=600, check=True,
                         cwd=ROOT).stdout
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0 and d["higher_is_better"]
    assert d["config"]["global_batch"] == 4096 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and "sample" in cb
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_objective_agreement_counts_only_both_optimal():
    sys.path.insert(0, str(ROOT))
    import numpy as np

    import bench

    got = bench.objective_agreement(np.array([6, 6, 4]), np.array([1.0, -2.0, 3.0]),
                                    [(0, 6, 1.0 + 1e-7), (1, 6, -2.0), (2, 6, 30.0)])
    assert got["instances"] == 3 and got["both_optimal"] == 2
    assert abs(got["max_rel_objective_diff"] - 1e-7) < 1e-12
    assert bench.objective_agreement(np.array([4]), np.array([0.0]), [(0, 6, 1.0)])["max_rel_objective_diff"] is None


def test_plain_call_stats_names_the_slowest_call_and_its_route():
    sys.path.insert(0, str(ROOT))
    import bench

    got = bench.plain_call_stats([0.05, 0.06, 0.7, 0.055], [1000, 150000, 300000, 5000])
    assert got["calls"] == 4 and got["max_instance"] == 2 and got["max_route"] == "host loop"
    assert got["max_ms"] == 700.0 and got["median_ms"] == 57.5 and got["host_loop_calls"] == 1
    assert bench.plain_call_stats([0.01], [200000])["max_route"] == "one CTA"
    assert bench.plain_call_stats([], []) == {"calls": 0}

