"""Regenerate tests/golden/reference_cpu.json from the reference itself.

Runs the reference's own CPU backend (oracle/_ref/libhprqp_ref_cpu.so,
compiled from the reference sources by ``make -C oracle ref``) through its
hprqp_* C ABI on the reference's twelve fixture models (restated in
hprqp.instances.tiny_cases) and on small seeded QPs, at several iteration
caps and tolerances, and records what it returns.  The fixtures pin the
oracle (tests/test_oracle_golden.py) without needing the reference at test
time.

    make -C oracle ref REF_ROOT=<reference checkout> && python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "hpr-qp-c_b200" / "python"))

import pyoracle  # noqa: E402
from hprqp import instances  # noqa: E402


def cases():
    out = []
    for inst in instances.tiny_cases():
        caps = [0, 1, 7, 10, 100, 250, 1000]
        if inst.name != "tall_diag":
            caps.append(None)
        for cap in caps:
            out.append((inst, dict(stoptol=1e-8, max_iter=cap)))
    # small seeded QPs with the plain recipe (reduced sizes) and one noC model
    small = [instances.plain_qp(0x48505251 + 90000 + k, n=60, m=30, a_density=0.1, m_rows=12, m_density=0.1,
                                n_eq=18, name=f"small_{k}") for k in range(4)]
    free = instances.plain_qp(0x48505251 + 90100, n=50, m=20, a_density=0.1, m_rows=10, m_density=0.1, n_eq=12,
                              name="small_free")
    free.l[:] = -float("inf")
    free.u[:] = float("inf")
    small.append(free)
    for inst in small:
        for cap in (10, 100, 300, None):
            out.append((inst, dict(stoptol=1e-6, max_iter=cap)))
    return out


def main() -> None:
    records = []
    for inst, kw in cases():
        cap = kw["max_iter"]
        r = pyoracle.ref_solve(inst, stoptol=kw["stoptol"], max_iter=cap if cap is not None else 2147483647)
        records.append(dict(
            name=inst.name, stoptol=kw["stoptol"], max_iter=cap,
            status=int(r["status"]), iter=int(r["iter"]), iter_4=int(r["iter_4"]), iter_6=int(r["iter_6"]),
            objective=r["primal_obj"], residual=r["residuals"], gap=r["gap"],
            x=list(map(float, r["x"])), y=list(map(float, r["y"])), z=list(map(float, r["z"])),
            w=list(map(float, r["w"])),
        ))
    path = Path(__file__).resolve().parent / "reference_cpu.json"
    path.write_text(json.dumps(dict(generator="reference CPU backend (use_gpu=0), hprqp_* ABI",
                                    records=records), indent=0))
    print(f"wrote {len(records)} records to {path}")


if __name__ == "__main__":
    main()
