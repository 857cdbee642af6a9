"""C-ABI surface and host logic of libhprqp.so (no GPU needed).

* every function declared in include/*.h is exported by the library;
* the host preprocessing (Q symmetrisation, empty/free row deletion,
  validation) produces exactly the oracle's preprocessed model, which restates
  the reference builder (src/shared/build.c:137-400);
* error behaviour of the reference-facing entry points.
"""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import pyoracle
from hprqp import instances

ROOT = Path(__file__).resolve().parents[1]


def _declared_functions():
    names = set()
    for h in (ROOT / "include").rglob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-z_][a-z0-9_]*)\s*\(", text, flags=re.M):
            if m.group(1) not in ("if", "while", "for", "return", "sizeof"):
                names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(engine_lib):
    lib = ctypes.CDLL(engine_lib.library_path())
    names = _declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def _model_matches_oracle(hprqp, inst):
    model = hprqp.build_from_instance(inst)
    ours = hprqp.model_arrays(model)
    ref = pyoracle.OracleModel(inst).export()
    assert ours["n"] == len(ref["c"]) and ours["m"] == len(ref["AL"])
    for key in ("q_indptr", "q_indices", "a_indptr", "a_indices"):
        assert np.array_equal(ours[key], ref[key]), key
    for key in ("q_data", "a_data", "c", "l", "u", "AL", "AU"):
        assert np.array_equal(ours[key], ref[key]), key


def test_preprocessing_matches_oracle_tiny(engine_lib):
    for inst in instances.tiny_cases():
        _model_matches_oracle(engine_lib, inst)


def test_preprocessing_matches_oracle_seeded(engine_lib):
    _model_matches_oracle(engine_lib, instances.config0())
    inst = instances.config3_instance(7)
    _model_matches_oracle(engine_lib, inst)


def test_preprocessing_symmetrises_and_deletes_rows(engine_lib):
    hprqp = engine_lib
    inf = np.inf
    # upper-triangular Q input, one empty A row, one free row
    Q = [[2.0, 1.0], [0.0, 4.0]]
    A = [[1.0, 1.0], [0.0, 0.0], [1.0, -1.0]]
    model = hprqp.build_from_qabc(Q, [1.0, 1.0], A, [1.0, 0.0, -inf], [1.0, 0.0, inf], [-1, -1], [1, 1])
    arr = hprqp.model_arrays(model)
    assert arr["m"] == 1
    dense = np.zeros((2, 2))
    for r in range(2):
        for k in range(arr["q_indptr"][r], arr["q_indptr"][r + 1]):
            dense[r, arr["q_indices"][k]] = arr["q_data"][k]
    assert np.array_equal(dense, np.array([[2.0, 0.5], [0.5, 4.0]]))


def test_invalid_arguments(engine_lib):
    hprqp = engine_lib
    with pytest.raises(RuntimeError, match="INVALID_ARGUMENT"):
        hprqp.build_from_qabc([[1.0]], [0.0], [[1.0]], [2.0], [1.0], [-1.0], [1.0])  # AL > AU
    with pytest.raises(RuntimeError, match="INVALID_ARGUMENT"):
        hprqp.build_from_qabc([[1.0]], [np.nan], [], [], [], [-1.0], [1.0])
    with pytest.raises(RuntimeError, match="INVALID_ARGUMENT"):
        hprqp.build_from_qabc([[1.0]], [0.0], [], [], [], [2.0], [1.0])  # l > u


def test_no_cpu_fallback(engine_lib):
    hprqp = engine_lib
    model = hprqp.build_from_instance(instances.tiny_cases()[0])
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, use_gpu=False))
    assert r.status_code == hprqp.STATUS_NOT_IMPLEMENTED


def test_status_names_and_defaults(engine_lib):
    hprqp = engine_lib
    assert hprqp.status_name(hprqp.STATUS_OPTIMAL) == "OPTIMAL"
    assert hprqp.status_name(99) == "UNKNOWN"
    p = hprqp.Parameters()
    s = p._struct()
    # src/shared/solver.c:133-157 (tests/test_defaults.c of the reference)
    assert s.stoptol == 1e-8 and s.max_iter == 2147483647 and s.check_iter == 100
    assert s.print_frequency == -1 and s.use_scaling == 1 and s.time_limit == 3600.0
    assert s.gram_mode == 1 and s.polishing == 1


def test_no_host_stub_exits(engine_lib):
    """nvcc turns a host-side call of a __device__-only function into an
    exit(1) stub; the library must contain no call to exit at all."""
    import subprocess

    out = subprocess.run(["nm", "-D", "--undefined-only", engine_lib.library_path()], capture_output=True,
                         text=True).stdout
    names = {line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip()}
    assert "exit" not in names and "_exit" not in names


def test_batch_rejects_bad_packing(engine_lib):
    """hprqp_batch_create validates the block-diagonal packing on the host."""
    import hprqp
    from hprqp import batch

    insts = instances.tiny_cases()[:2]
    p = batch.pack(insts)
    p.var_offsets = p.var_offsets.copy()
    p.var_offsets[-1] += 1  # does not end at n
    with pytest.raises(RuntimeError, match="INVALID_ARGUMENT"):
        batch.Batch(p)


def test_reference_wrappers_find_every_symbol(engine_lib):
    """every hprqp_* symbol the reference's Python and Julia packages bind
    (tests/golden/reference_ffi_symbols.json, from
    tests/golden/make_ffi_symbols.py) is exported, so both load this library
    through HPRQP_LIBRARY_PATH unchanged"""
    import ctypes
    import json

    lib = ctypes.CDLL(engine_lib.library_path())
    data = json.loads((ROOT / "tests" / "golden" / "reference_ffi_symbols.json").read_text())
    assert data["python"] and data["julia"]
    missing = [s for names in data.values() for s in names if not hasattr(lib, s)]
    assert not missing, missing
