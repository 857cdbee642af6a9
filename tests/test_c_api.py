"""The host-side C entry points from a C program (tests/native/c_api_probe.c,
compiled as pedantic C99 against include/ and linked to the library): the headers are
valid C and the builders work without a GPU."""
from __future__ import annotations

import json
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_c_caller(engine_lib, tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lib = Path(engine_lib.library_path())
    exe = tmp_path / "c_api_probe"
    env = {k: v for k, v in os.environ.items() if k != "LD_PRELOAD"}
    subprocess.run([cc, "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", f"-I{ROOT / 'include'}", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "c_api_probe.c"), f"-L{lib.parent}", f"-l:{lib.name}",
                    f"-Wl,-rpath,{lib.parent}", "-lm"], check=True, env=env)
    mps = ROOT / "tests" / "golden" / "simple_qp.mps"
    out = json.loads(subprocess.run([str(exe), str(mps)], capture_output=True, text=True, check=True,
                                    env=env).stdout)
    assert out["build"] == out["qc"] == out["pre"] == out["matvec"] == out["soc"] == 0
    assert out["y"] == 2.0 and out["dot"] == 2.0
    # one linear row, then one cone: 2 head rows + 2 factor rows
    assert out["m_qp"] == 1 and out["m_qc"] == 1 + 4 and out["cones"] == 1
    assert out["bind"] == 0 and (out["bn"], out["bm"]) == (2, 1)
    # cones and MPS input through the C entry points (reference tests/test_binding_api.c:16-118
    # reads the same file: 2 variables, 2 rows, Q with 3 stored upper-triangle entries symmetrised)
    assert out["soc_build"] == 0 and (out["soc_var_cones"], out["soc_row_cones"]) == (1, 1)
    assert out["mps"] == 0 and (out["mps_n"], out["mps_m"]) == (2, 2) and out["mps_nnz_q"] == 4
    assert out["bind_mps"] == 0 and out["bind_mps_n"] == 2
    if not out["gpu"]:
        assert out["solve"] == engine_lib.STATUS_NOT_IMPLEMENTED  # no CPU fallback
