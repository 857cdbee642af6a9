"""Copy the reference's own MPS test fixture (tests/data/simple_qp.mps, used
by its tests/test_binding_api.c:16-118) and record what the reference makes
of it: its reader's model arrays (its CPU library's build_from_mps) and its
CPU solver's result at max_iter 0 and at stoptol 1e-8.  Writes simple_qp.mps
and simple_qp.json beside this file.

    make -C oracle ref REF_ROOT=<reference checkout> && python tests/golden/make_reference_fixtures.py <reference checkout>
"""
from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path[:0] = [str(ROOT / "oracle"), str(ROOT / "hpr-qp-c_b200" / "python")]

import pyoracle  # noqa: E402
from hprqp.instances import CSR, QPInstance  # noqa: E402


def main(ref: Path) -> None:
    mps = HERE / "simple_qp.mps"
    shutil.copyfile(ref / "tests" / "data" / "simple_qp.mps", mps)
    m = pyoracle.ref_build_from_mps(mps)
    assert m["status"] == 0, m
    inst = QPInstance(CSR(m["n"], m["n"], m["q_indptr"], m["q_indices"], m["q_data"]),
                      CSR(m["m"], m["n"], m["a_indptr"], m["a_indices"], m["a_data"]),
                      m["c"], m["AL"], m["AU"], m["l"], m["u"], m["obj_constant"], "simple_qp")
    out = {"model": {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in m.items()}}
    for key, kw in (("max_iter0", dict(max_iter=0)), ("solve_1e-8", dict(stoptol=1e-8))):
        r = pyoracle.ref_solve(inst, **kw)
        out[key] = {k: (v.tolist() if isinstance(v, np.ndarray) else v) for k, v in r.items() if k != "time"}
    (HERE / "simple_qp.json").write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", mps, HERE / "simple_qp.json")


if __name__ == "__main__":
    main(Path(sys.argv[1]))
