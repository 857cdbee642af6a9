"""Time this engine's plain solve_gpu against the reference's own solve_gpu
(oracle/_ref/libhprqp_ref_gpu.so: cuSPARSE SpMV, cuBLAS reductions, built
from the reference sources for sm_100a; polishing and the Gram path off) on
the same seeded instances, on one GPU.  Test infrastructure: prints one JSON
object per workload.

    python oracle/compare_reference_gpu.py [--sample 16] [--large-iters 3000]

* plain QP (n=1000, m=500), stoptol 1e-6: call time incl. setup, loop time;
* batch-recipe sample, stoptol 1e-6: plain solves/s of both, and this
  engine's batched solver on the same instances;
* portfolio QP (n=200,200), stoptol 1e-6;
* large power-law QP (n=1e6), stoptol 1e-8, a fixed iteration budget:
  iterations/s of both loops.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path[:0] = [str(ROOT / "oracle"), str(ROOT / "hpr-qp-c_b200" / "python")]

import pyoracle  # noqa: E402
import hprqp  # noqa: E402
from hprqp import batch, instances  # noqa: E402


def ours(inst, stoptol, max_iter=2147483647):
    model = hprqp.build_from_instance(inst)
    t0 = time.perf_counter()
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=stoptol, max_iter=max_iter), as_numpy=True)
    return {"status": r.status_code, "iter": int(r.iter), "loop_s": r.time, "call_s": time.perf_counter() - t0,
            "objective": r.objective}


def ref(inst, stoptol, max_iter=2147483647):
    m = pyoracle.RefGpuModel(inst)
    t0 = time.perf_counter()
    o = m.solve(stoptol=stoptol, max_iter=max_iter)
    return {"status": o["status"], "iter": o["iter"], "loop_s": o["time"], "call_s": time.perf_counter() - t0,
            "objective": o["primal_obj"]}


def pair(name, inst, stoptol, max_iter=2147483647):
    ours(inst, stoptol, 10)  # load the kernels once
    ref(inst, stoptol, 10)
    a = ours(inst, stoptol, max_iter)
    b = ref(inst, stoptol, max_iter)
    out = {"workload": name, "stoptol": stoptol, "ours": a, "reference_gpu": b,
           "loop_speedup": b["loop_s"] / a["loop_s"] if a["loop_s"] > 0 else None,
           "call_speedup": b["call_s"] / a["call_s"],
           "iters_per_s": {"ours": a["iter"] / a["loop_s"], "reference_gpu": b["iter"] / b["loop_s"]}}
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sample", type=int, default=16)
    ap.add_argument("--large-iters", type=int, default=3000)
    ap.add_argument("--skip-large", action="store_true")
    args = ap.parse_args()
    if not pyoracle.ref_gpu_available():
        print(json.dumps({"unavailable": "oracle/_ref/libhprqp_ref_gpu.so not built (make -C oracle ref-gpu)"}))
        return
    pair("plain QP n=1000 m=500", instances.config0(), 1e-6)
    insts = instances.config3(args.sample)
    ours(insts[0], 1e-6, 10)
    ref(insts[0], 1e-6, 10)
    ta = sum(ours(i, 1e-6)["call_s"] for i in insts)
    tb = sum(ref(i, 1e-6)["call_s"] for i in insts)
    b = batch.Batch(insts)
    b.solve(stoptol=1e-6)
    ms = b.solve(stoptol=1e-6)
    b.close()
    print(json.dumps({"workload": f"batch-recipe sample of {len(insts)} QPs, stoptol 1e-6",
                      "plain_solves_per_s": {"ours": len(insts) / ta, "reference_gpu": len(insts) / tb},
                      "batched_solves_per_s_ours": len(insts) / (ms / 1e3)}), flush=True)
    pair("portfolio n=200,200", instances.config2(), 1e-6)
    if not args.skip_large:
        pair("large power-law QP n=1e6 (fixed iterations)", instances.config1(), 1e-8, args.large_iters)


if __name__ == "__main__":
    main()
