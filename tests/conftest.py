"""Shared test setup: import paths, the `gpu` marker, fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "hpr-qp-c_b200" / "python"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import json

    return json.loads((ROOT / "tests" / "golden" / "reference_cpu.json").read_text())["records"]


@pytest.fixture(scope="session")
def engine_lib():
    """Builds the engine library if needed and returns the hprqp module."""
    lib = ROOT / "hpr-qp-c_b200" / "lib" / "libhprqp.so"
    if not lib.exists():
        import subprocess

        subprocess.run([sys.executable, str(ROOT / "hpr-qp-c_b200" / "build.py")], check=True)
    import hprqp

    return hprqp


@pytest.fixture(params=["host_loop", "single_cta"])
def plain_path(request, engine_lib):
    """Runs a plain-path test through both routes of solve_gpu: the
    host-driven loop of fused device passes, and the whole solve in one CTA
    of the batch kernel (hprqp_b200_set_single_cta_max_work)."""
    big = 1 << 40
    old = engine_lib.set_single_cta_max_work(0 if request.param == "host_loop" else big)
    yield request.param
    engine_lib.set_single_cta_max_work(old)
