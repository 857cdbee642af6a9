"""Benchmark of the HPR-QP engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: solves/s to 1e-6 relative KKT on the 4096-QP batch workload
(n ~ U{50..2000}, m ~ U{ceil(n/4)..n}, A density U(0.5%,5%), Q = M'M + 0.01 I
with nnz(Q) ~ dQ n^2, dQ ~ U(0.1%,2%), 60% equality rows, seeded), next to
looping the plain one-QP-per-call solve over the same instances, plus the
SpMV bandwidth on the large power-law QP (n=1e6, m=5e5, nnz(A)~1e7,
nnz(Q)~3.2e7) against the measured HBM peak.

One step = one batched solve of the whole 4096-instance batch.  ``value`` is
measured with the batch resident on the device (CUDA-event time of the solve
kernel); ``e2e`` goes through the one-call C ABI (hprqp_solve_batch) from
host buffers, so host preprocessing, upload and read-back of all solutions
are inside the timed region.  Multi-GPU runs are replicas: every rank solves
its own batch (different seeds), the time is the max over ranks.

``--impl reference`` times the reference's own CPU implementation
(oracle/_ref/libhprqp_ref_cpu.so, compiled from the reference sources; the C
oracle port if that library is absent) on the host cores, one process per
core, on a bounded sample of the same instances per step.
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "hpr-qp-c_b200" / "python"))
sys.path.insert(0, str(ROOT / "oracle"))

# DRAM bytes moved per algorithmic byte by k_batch_solve: ncu on a 300-QP
# solve of this workload in the bench's kernel shapes (a 640-thread launch
# for its 85 instances of n, m <= 640, a 1024-thread launch for the rest, one
# instance per SM at a time, no shared-memory pool) read+wrote 0.009 +
# 394.424 GB (dram__bytes_read.sum + dram__bytes_write.sum of both launches)
# for 512.257 GB of algorithmic bytes; traffic grows with instance-iterations,
# so the bench scales this ratio by its own solve's algorithmic bytes.
BATCH_DRAM_PER_ALGO_BYTE = 394.433e9 / 512.257e9
METRIC = "solves/s to 1e-6 rel-KKT, batched vs plain on 1 B200; SpMV GB/s vs HBM peak"
STOPTOL = 1e-6
BATCH = 4096


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.smi_id = self.physical_id(device)
        self.proc = None
        self.path = Path("/tmp") / f"hprqp_clocks_{os.getpid()}.csv"

    @staticmethod
    def physical_id(device: int, visible: str | None = None) -> str:
        """nvidia-smi's id of CUDA device `device`: CUDA_VISIBLE_DEVICES
        renumbers devices (its entries are indices or UUIDs, both of which
        nvidia-smi --id takes); without it the CUDA index is the physical one."""
        if visible is None:
            visible = os.environ.get("CUDA_VISIBLE_DEVICES")
        if visible:
            ids = [v.strip() for v in visible.split(",") if v.strip()]
            if 0 <= device < len(ids):
                return ids[device]
        return str(device)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.smi_id}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        if self.path.exists():
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# workload
# --------------------------------------------------------------------------
def rank_first_instance(rank: int) -> int:
    """First instance id of a rank's batch: replicas solve disjoint seeded
    batches (rank r: ids 100000 r ...), so per-GPU work is fixed as N grows."""
    return 100000 * rank


def max_over_ranks(v: float, dist=None, device: str = "cuda") -> float:
    """Max of a per-rank time over all ranks (every rank calls it in the same
    order; identity when no process group is initialised)."""
    if dist is None or not dist.is_initialized():
        return v
    import torch

    t = torch.tensor([v], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(per_rank: int, world: int, steps: int, seconds: float) -> float:
    """Solves/s of the whole job: all ranks' instances over the slowest rank's time."""
    return per_rank * world * steps / seconds


def batch_instances(count: int, start: int = 0):
    from hprqp import instances

    return instances.config3(count, start)


def bytes_per_iter(inst) -> float:
    """B_iter = 2 S(Q) + S(A) + S(A') + 8 (24 n + 7 m), S(M) = 12 nnz + 4 (nrow+1)."""
    n, m = inst.n, inst.m
    sq = 12 * inst.Q.nnz + 4 * (n + 1)
    sa = 12 * inst.A.nnz + 4 * (m + 1)
    sat = 12 * inst.A.nnz + 4 * (n + 1)
    return 2 * sq + sa + sat + 8 * (24 * n + 7 * m)


def _ref_worker(args):
    inst_ids, stoptol = args
    import pyoracle

    out = []
    for k in inst_ids:
        inst = batch_instances(1, k)[0]
        if pyoracle.ref_available():
            r = pyoracle.ref_solve(inst, stoptol=stoptol)
        else:
            r = pyoracle.OracleModel(inst).solve(stoptol=stoptol, mode=pyoracle.MODE_CPU_REF)
        out.append((int(k), int(r["status"]), float(r["primal_obj"])))
    return out


def _ref_single_core(_):
    """One core, reference CPU library (or the oracle port): the n=1000 QP to
    1e-6 and 16 members of the differentiation batch (n=500, m=300) to 1e-8."""
    import pyoracle
    from hprqp import instances

    def solve(inst, tol):
        if pyoracle.ref_available():
            return pyoracle.ref_solve(inst, stoptol=tol)
        return pyoracle.OracleModel(inst).solve(stoptol=tol, mode=pyoracle.MODE_CPU_REF)

    inst = instances.config0()
    t0 = time.perf_counter()
    r = solve(inst, 1e-6)
    c0 = time.perf_counter() - t0
    sample = [instances.config4_instance(i) for i in range(16)]
    t0 = time.perf_counter()
    st4 = [int(solve(i, 1e-8)["status"]) for i in sample]
    c4 = (time.perf_counter() - t0) / len(sample)
    return {"plain_qp_n1000_s": round(c0, 4), "plain_qp_status": int(r["status"]),
            "diff_batch_member_s": round(c4, 4), "diff_batch_sample": len(sample),
            "diff_batch_optimal": int(sum(s == 6 for s in st4)), "cores": 1}


def cpu_single_core_timings():
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.map(_ref_single_core, [0])[0]


def cpu_reference_rate(ids, cores: int):
    """Reference CPU solves/s over the given batch instances on `cores`
    spawned processes."""
    import pyoracle

    kind = "reference" if pyoracle.ref_available() else "port"
    chunks = [ids[i::cores] for i in range(cores)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(int, range(cores))  # start the workers outside the timed region
        t0 = time.perf_counter()
        solved = sum(pool.map(_ref_worker, [(c, STOPTOL) for c in chunks if c]), [])
        dt = time.perf_counter() - t0
    # (instance id, status, primal objective), in instance order
    return len(ids) / dt, kind, dt, sorted(solved)


def objective_agreement(ours_status, ours_obj, ref_solved):
    """The batch's objectives against the reference CPU solves of the same
    instances: both OPTIMAL, largest |ours - ref| / max(1, |ref|)."""
    diffs, both = [], 0
    for k, st, obj in ref_solved:
        if st == 6 and int(ours_status[k]) == 6:
            both += 1
            diffs.append(abs(float(ours_obj[k]) - obj) / max(1.0, abs(obj)))
    return {"instances": len(ref_solved), "both_optimal": both,
            "max_rel_objective_diff": float(max(diffs)) if diffs else None}


def plain_call_stats(seconds, product_nnz, one_cta_limit: int = 200000):
    """Per-call summary of the plain loop: median and slowest call, and the
    slowest call's instance and route (solve_gpu runs a model without cones
    on one CTA of the batch kernel when 2 nnz(Q) + 2 nnz(A) <= the limit,
    else through the host-driven loop)."""
    ms = [1e3 * float(t) for t in seconds]
    if not ms:
        return {"calls": 0}
    k = int(np.argmax(ms))
    route = lambda w: "one CTA" if w <= one_cta_limit else "host loop"  # noqa: E731
    return {"calls": len(ms), "median_ms": round(float(np.median(ms)), 2), "max_ms": round(ms[k], 2),
            "max_instance": k, "max_route": route(int(product_nnz[k])),
            "host_loop_calls": int(sum(int(w) > one_cta_limit for w in product_nnz))}


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_gpu_leg(device: int, sample: int = 32, large_iters: int = 1000):
    """The reference's own GPU solve_gpu (its CUDA build: cuSPARSE SpMV and
    cuBLAS reductions, polishing 0, Gram off) beside this engine's solve_gpu
    on the same seeded instances and the same GPU: the n=1000 QP, a sample
    of the batch recipe (and the batched kernel on it), the portfolio QP and
    the large power-law QP at a fixed iteration budget.  A baseline, like
    cpu_baseline: the reference measured, never this engine."""
    import hprqp
    import pyoracle
    from hprqp import batch as hb
    from hprqp import instances

    if not pyoracle.ref_gpu_available():
        return {"unavailable": "the reference GPU library (oracle/_ref/libhprqp_ref_gpu.so) is not built"}

    def ours(inst, stoptol, max_iter=2147483647, model=None):
        model = model or hprqp.build_from_instance(inst)
        t0 = time.perf_counter()
        r = hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=stoptol, max_iter=max_iter,
                                                   device_number=device), as_numpy=True)
        return {"status": r.status_code, "iter": int(r.iter), "loop_s": r.time,
                "call_s": time.perf_counter() - t0, "objective": r.objective}

    def ref(inst, stoptol, max_iter=2147483647, model=None):
        model = model or pyoracle.RefGpuModel(inst)
        t0 = time.perf_counter()
        o = model.solve(stoptol=stoptol, max_iter=max_iter, device=device)
        return {"status": int(o["status"]), "iter": int(o["iter"]), "loop_s": float(o["time"]),
                "call_s": time.perf_counter() - t0, "objective": float(o["primal_obj"])}

    def pair(name, inst, stoptol, max_iter=2147483647):
        om, rm = hprqp.build_from_instance(inst), pyoracle.RefGpuModel(inst)
        ours(inst, stoptol, 10, om)  # load both libraries' kernels outside the timings
        ref(inst, stoptol, 10, rm)
        a, b = ours(inst, stoptol, max_iter, om), ref(inst, stoptol, max_iter, rm)
        return {"workload": name, "stoptol": stoptol, "ours": a, "reference_gpu": b,
                "iters_per_s": {"ours": a["iter"] / a["loop_s"], "reference_gpu": b["iter"] / b["loop_s"]},
                "loop_speedup": (b["loop_s"] / b["iter"]) / (a["loop_s"] / a["iter"]),
                "call_speedup": b["call_s"] / a["call_s"],
                "rel_objective_diff": abs(a["objective"] - b["objective"]) / max(1.0, abs(b["objective"]))}

    out = {"plain_qp_n1000": pair("plain QP n=1000 m=500 (1% A density)", instances.config0(), 1e-6)}
    insts = batch_instances(sample, 0)
    om = [hprqp.build_from_instance(i) for i in insts]
    rm = [pyoracle.RefGpuModel(i) for i in insts]
    ours(insts[0], STOPTOL, 10, om[0])
    ref(insts[0], STOPTOL, 10, rm[0])
    ra = [ours(i, STOPTOL, model=m) for i, m in zip(insts, om)]
    rb = [ref(i, STOPTOL, model=m) for i, m in zip(insts, rm)]
    b = hb.Batch(insts, device_number=device)
    b.solve(stoptol=STOPTOL)
    bms = b.solve(stoptol=STOPTOL)
    b.close()
    ta, tb = sum(x["call_s"] for x in ra), sum(x["call_s"] for x in rb)
    out["batch_sample"] = {
        "workload": f"{sample} instances of the batch recipe, stoptol {STOPTOL:g}, one solve_gpu call each",
        "solves_per_s": {"ours_plain": sample / ta, "reference_gpu_plain": sample / tb,
                         "ours_batched": sample / (bms / 1e3)},
        "plain_speedup": tb / ta,
        "optimal": {"ours": sum(x["status"] == 6 for x in ra), "reference_gpu": sum(x["status"] == 6 for x in rb)},
        "max_rel_objective_diff": max(abs(x["objective"] - y["objective"]) / max(1.0, abs(y["objective"]))
                                      for x, y in zip(ra, rb))}
    out["portfolio"] = pair("portfolio n=200,200 (k=200 factors, 500 sectors)", instances.config2(), 1e-6)
    out["large_qp"] = pair(f"power-law QP n=1e6 m=5e5, stoptol 1e-8, {large_iters} iterations",
                           instances.config1(), 1e-8, large_iters)
    return out


def spmv_leg(peak_gbs: float, reps: int = 10, scale: float = 1.0):
    """Row-tiled SpMV on the large power-law QP's A and Q (device timing),
    beside the gather bound of the same matrix (hprqp_b200_gather_bound)."""
    import hprqp
    from hprqp import instances

    inst = instances.config1(scale=scale)
    rng = np.random.default_rng(5)
    out = {}
    for name, (ip, ii, dd, nrow, ncol) in {
        "A": (inst.A.indptr, inst.A.indices, inst.A.data, inst.m, inst.n),
        "Q": (inst.Q.indptr, inst.Q.indices, inst.Q.data, inst.n, inst.n),
    }.items():
        x = rng.standard_normal(ncol)
        y, ms = hprqp.spmv(ip, ii, dd, ncol, x, reps=reps)
        total, bound_ms = hprqp.gather_bound(ip, ii, dd, ncol, x, reps=reps)
        if abs(total - float(np.sum(y))) > 1e-9 * max(1.0, float(np.sum(np.abs(y)))):
            raise RuntimeError(f"gather bound checksum {total} != sum(M x) {np.sum(y)}")
        nnz = int(ip[-1])
        algo = 12 * nnz + 4 * (nrow + 1) + 8 * ncol + 8 * nrow
        gbs = algo / (ms * 1e-3) / 1e9
        out[name] = {"nnz": nnz, "ms": round(ms, 4), "GB/s": round(gbs, 1), "frac": round(gbs / peak_gbs, 4),
                     "bytes": algo,
                     # the same bytes over the time of a pass with no row structure at all:
                     # what any CSR kernel can reach on this column pattern
                     "gather_bound": {"ms": round(bound_ms, 4), "GB/s": round(algo / (bound_ms * 1e-3) / 1e9, 1),
                                      "frac": round(algo / (bound_ms * 1e-3) / 1e9 / peak_gbs, 4),
                                      "spmv_over_bound": round(bound_ms / ms, 4)}}
    return out


def large_qp_leg(peak_gbs: float, iters: int = 3000, minres_iters: int = 2000, scale: float = 1.0):
    """Plain solve_gpu on the large power-law QP (n=1e6, m=5e5, nnz(A)~1e7,
    nnz(Q)~3.2e7, stoptol 1e-8) for a fixed iteration budget (it does not
    reach 1e-8 within minutes, neither here nor with the reference's GPU
    build): HPR iterations/s of the solve loop and the HBM roofline of its
    algorithmic bytes (B_iter per iteration); then the single-instance
    adjoint (hprqp_diff.h) on that unconverged iterate for a fixed MINRES
    budget (time per MINRES iteration; large_backward_leg has the converged
    case)."""
    import hprqp
    from hprqp import instances

    inst = instances.config1(scale=scale)
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, stoptol=1e-8, max_iter=iters)
    t0 = time.perf_counter()
    r, state = hprqp.solve_for_backward(model, params)
    wall = time.perf_counter() - t0
    ips = r.iter / r.time
    gbs = bytes_per_iter(inst) * ips / 1e9
    out = {"workload": "n=1e6 m=5e5 power-law QP, stoptol 1e-8", "iterations": int(r.iter),
           "loop_s": round(r.time, 4), "call_s": round(wall, 3), "iters_per_s": round(ips, 1),
           "bytes_per_iter": bytes_per_iter(inst), "GB/s": round(gbs, 1), "frac": round(gbs / peak_gbs, 4),
           "kkt": float(r.residual), "status": r.status}
    if state is not None:
        # single-instance backward at this size: L = g.x*, g ~ N(0,1), on the
        # active set of the iterate above, a fixed MINRES budget
        g = state.backward(np.random.default_rng(1).standard_normal(r.x.shape[0]), tol=1e-10,
                           max_iter=minres_iters)
        state.close()
        out["backward"] = {"minres_iters": g["minres_iters"], "relres": g["minres_relres"],
                           "seconds": round(g["backward_seconds"], 3),
                           "ms_per_minres_iter": round(1e3 * g["backward_seconds"] / max(g["minres_iters"], 1), 4)}
    return out


def large_backward_leg(scale: float = 1.0, tol: float = 1e-10, max_minres: int = 50000):
    """The single large backward at the large QP's sizes (n=1e6, m=5e5,
    nnz(A)=1e7, nnz(Q)~3.2e7) on the plain recipe, whose forward solve reaches
    1e-8 (the power-law recipe does not within minutes): forward
    solve_for_backward to 1e-8, then hprqp_backward with MINRES to a relative
    residual of 1e-10; times of both calls and their ratio."""
    import hprqp
    from hprqp import instances

    inst = instances.config1_sized_plain(scale=scale)
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, stoptol=1e-8, time_limit=300.0)
    t0 = time.perf_counter()
    r, state = hprqp.solve_for_backward(model, params)
    fwd = time.perf_counter() - t0
    out = {"workload": f"plain recipe at n={inst.n} m={inst.m} nnz(A)={inst.A.nnz} nnz(Q)={inst.Q.nnz}, stoptol 1e-8",
           "status": r.status, "iterations": int(r.iter), "kkt": float(r.residual), "forward_call_s": round(fwd, 3),
           "forward_loop_s": round(r.time, 3)}
    if state is not None:
        g = state.backward(np.random.default_rng(1).standard_normal(inst.n), tol=tol, max_iter=max_minres)
        state.close()
        out.update(minres_iters=int(g["minres_iters"]), minres_relres=float(g["minres_relres"]),
                   backward_s=round(g["backward_seconds"], 3),
                   ms_per_minres_iter=round(1e3 * g["backward_seconds"] / max(g["minres_iters"], 1), 4),
                   backward_over_forward=round(g["backward_seconds"] / fwd, 3))
    return out


def portfolio_leg():
    """Plain solve_gpu on the factor-structured portfolio QP (n=200,200,
    200 dense factor rows, diagonal Q) to 1e-6."""
    import hprqp
    from hprqp import instances

    inst = instances.config2()
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, stoptol=1e-6)
    hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=1e-6, max_iter=10), as_numpy=True)
    t0 = time.perf_counter()
    r = hprqp.optimize(model, params, as_numpy=True)
    wall = time.perf_counter() - t0
    return {"workload": "portfolio n=200,200 (k=200 factors, 500 sectors), stoptol 1e-6", "status": r.status,
            "iterations": int(r.iter), "loop_s": round(r.time, 4), "call_s": round(wall, 3),
            "iters_per_s": round(r.iter / r.time, 1), "objective": r.objective, "kkt": float(r.residual)}


def adjoint_leg(device: int, count: int = 256, reps: int = 3):
    """Differentiation workload: 256 QPs (n=500, m=300, 150 equality rows),
    forward solve to 1e-8, loss L = sum g.x* with g ~ N(0,1) per instance,
    backward through the device adjoint (MINRES on the active-set KKT
    system).  Device times of the solve kernel and of the adjoint kernel,
    plus host wall time of the whole backward call (adjoint + gradient
    assembly for c, l, u, AL, AU and the nonzeros of Q and A)."""
    from hprqp import batch as hb
    from hprqp import instances

    insts = instances.config4(count)
    b = hb.Batch(insts, device_number=device)
    rng = np.random.default_rng(4)
    gx = rng.standard_normal(b.n)
    fwd, bwd, bwd_wall = [], [], []
    for _ in range(reps + 1):
        fwd.append(b.solve(stoptol=1e-8))
        t0 = time.perf_counter()
        g = b.backward(gx)
        bwd_wall.append(1e3 * (time.perf_counter() - t0))
        bwd.append(g.backward_ms)
    res = b.results(vectors=False)
    b.close()
    f = statistics.median(fwd[1:])
    k = statistics.median(bwd[1:])
    w = statistics.median(bwd_wall[1:])
    return {"workload": f"{count} QPs n=500 m=300 (150 equality), stoptol 1e-8, L = sum g.x*",
            "forward_kernel_ms": round(f, 3), "backward_kernel_ms": round(k, 3), "backward_call_ms": round(w, 3),
            "backward_over_forward": round(w / f, 4), "backward_kernel_over_forward": round(k / f, 4),
            "optimal": int(np.sum(res.status == 6)), "mean_solve_iters": float(res.iter.mean()),
            "mean_minres_iters": float(g.minres_iters.mean()), "max_minres_relres": float(g.minres_relres.max())}


def warm_start_leg(packed, base_results, device: int, reps: int = 2):
    """Training-loop re-solve: the batch's linear costs move by 1% (c_i *
    (1 + 0.01 N(0,1)), seeded) after a solve; the moved batch is solved cold
    (from zero, as the reference does), warm (hprqp_batch_set_warm_start at
    the previous solution) and warm with the previous solve's sigma.  Device time of the solve kernel and iterations of
    each, and the largest objective difference between them."""
    from dataclasses import replace

    from hprqp import batch as hb

    rng = np.random.default_rng(11)
    moved = replace(packed, c=packed.c * (1.0 + 0.01 * rng.standard_normal(packed.c.shape[0])))
    b = hb.Batch(moved, device_number=device)
    cold_ms, warm_ms = [], []
    for _ in range(reps):
        b.set_warm_start(None)
        cold_ms.append(b.solve(stoptol=STOPTOL))
    cold = b.results(vectors=False)
    b.set_warm_start(base_results.x, base_results.y, base_results.w)
    for _ in range(reps):
        warm_ms.append(b.solve(stoptol=STOPTOL))
    warm = b.results(vectors=False)
    b.set_warm_start(base_results.x, base_results.y, base_results.w, base_results.sigma)
    ws_ms = []
    for _ in range(reps):
        ws_ms.append(b.solve(stoptol=STOPTOL))
    warm_s = b.results(vectors=False)
    b.close()
    K = packed.K
    cm, wm = min(cold_ms), min(warm_ms)
    scale = np.maximum(1.0, np.abs(cold.objective))
    return {"workload": f"{K} QPs of the batch, c moved by 1%, stoptol {STOPTOL:g}",
            "cold": {"solves_per_s": K / (cm / 1e3), "kernel_ms": round(cm, 3), "mean_iters": float(cold.iter.mean()),
                     "optimal": int(np.sum(cold.status == 6))},
            "warm": {"solves_per_s": K / (wm / 1e3), "kernel_ms": round(wm, 3), "mean_iters": float(warm.iter.mean()),
                     "optimal": int(np.sum(warm.status == 6))},
            "warm_sigma": {"solves_per_s": K / (min(ws_ms) / 1e3), "kernel_ms": round(min(ws_ms), 3),
                           "mean_iters": float(warm_s.iter.mean()), "optimal": int(np.sum(warm_s.status == 6))},
            "warm_over_cold_speed": round(cm / wm, 3), "warm_sigma_over_cold_speed": round(cm / min(ws_ms), 3),
            "max_rel_objective_diff": float(max(np.max(np.abs(warm.objective - cold.objective) / scale),
                                                np.max(np.abs(warm_s.objective - cold.objective) / scale)))}


def e2e_step(packed, device: int):
    """One call of hprqp_solve_batch from host buffers; returns seconds."""
    from hprqp import batch as hb
    import hprqp

    lib = hprqp._lib()
    hb._configure()
    fn = lib.hprqp_solve_batch
    c_size_p = ctypes.POINTER(ctypes.c_size_t)
    c_double_p = ctypes.POINTER(ctypes.c_double)
    fn.argtypes = [ctypes.c_size_t, c_size_p, c_size_p, ctypes.POINTER(hprqp._MatrixCSR),
                   ctypes.POINTER(hprqp._MatrixCSR), c_double_p, c_double_p, c_double_p, c_double_p, c_double_p,
                   c_double_p, ctypes.POINTER(hb.BatchParams), ctypes.POINTER(ctypes.c_int), c_size_p, c_double_p,
                   c_double_p, c_double_p, c_double_p, c_double_p, c_double_p, c_double_p]
    p = packed
    K = p.K
    n = int(p.var_offsets[-1])
    m = int(p.row_offsets[-1])
    keep = []
    Q = hb._csr(n, n, p.q_indptr, p.q_indices, p.q_data, keep)
    A = hb._csr(m, n, p.a_indptr, p.a_indices, p.a_data, keep)
    dp = lambda a: a.ctypes.data_as(c_double_p)  # noqa: E731
    status = np.zeros(K, np.int32)
    it = np.zeros(K, np.uint64)
    obj = np.zeros(K)
    res = np.zeros(K)
    gap = np.zeros(K)
    x = np.zeros(n)
    y = np.zeros(max(m, 1))
    z = np.zeros(n)
    w = np.zeros(n)
    params = hb.default_params(stoptol=STOPTOL, device_number=device)
    vo = np.ascontiguousarray(p.var_offsets, np.uint64)
    ro = np.ascontiguousarray(p.row_offsets, np.uint64)
    t0 = time.perf_counter()
    st = fn(K, vo.ctypes.data_as(c_size_p), ro.ctypes.data_as(c_size_p), ctypes.byref(Q), ctypes.byref(A), dp(p.c),
            dp(p.AL), dp(p.AU), dp(p.l), dp(p.u), dp(p.obj), ctypes.byref(params),
            status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), it.ctypes.data_as(c_size_p), dp(obj), dp(res),
            dp(gap), dp(x), dp(y), dp(z), dp(w))
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(f"hprqp_solve_batch failed: {st}")
    d2h = status.nbytes + it.nbytes + obj.nbytes + res.nbytes + gap.nbytes + x.nbytes + 8 * m + z.nbytes + w.nbytes
    return dt, int(np.sum(status == 6)), d2h


# --------------------------------------------------------------------------
# main
# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=BATCH, help="instances per step")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--cpu-sample", type=int, default=256)
    ap.add_argument("--no-spmv", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-plain-large", action="store_true")
    ap.add_argument("--no-warm", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--only", choices=["spmv", "batch", "adjoint", "large", "large_backward", "portfolio", "warm",
                                       "reference_gpu"],
                    default=None,
                    help="sub-runs: only the large-QP SpMV leg, the batched solve, the adjoint, the large-QP "
                         "plain solve, the portfolio plain solve, the warm-start re-solve or the reference GPU "
                         "build beside the plain path")
    ap.add_argument("--spmv-reps", type=int, default=10)
    ap.add_argument("--scale", type=float, default=1.0,
                    help="--only spmv / --only large: the large power-law QP recipe with every dimension scaled "
                         "(small cases for kernel profiles)")
    ap.add_argument("--large-iters", type=int, default=3000, help="--only large: HPR iteration budget")
    ap.add_argument("--minres-iters", type=int, default=2000, help="--only large: MINRES iteration budget")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1
    config = {"workload": f"batch of {args.batch} seeded QPs per GPU: n~U{{50..2000}}, m~U{{ceil(n/4)..n}}, "
                          f"A density U(0.5%,5%), nnz(Q)~U(0.1%,2%) n^2, 60% equality rows; stoptol {STOPTOL:g}",
              "global_batch": args.batch * world, "parallelism": f"replicas x{world} (instance-sharded)",
              "l2": "inputs larger than L2: the batch holds ~3 GB of matrices"}

    if args.impl == "reference":
        if rank != 0:
            return
        sample = min(args.cpu_sample, args.batch)
        rates = []
        t_total = 0.0
        kind = "port"
        for step in range(args.steps):
            ids = list(range(step * sample, (step + 1) * sample))
            rate, kind, dt, _ = cpu_reference_rate(ids, cores)
            rates.append(rate)
            t_total += dt
        value = float(statistics.median(rates))
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators)",
                "config": config, "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind,
                                 "cpu_model": cpu_model(),
                                 "sample": f"{sample} batch instances per step, one process per core"},
                "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=900))
    import hprqp
    from hprqp import batch as hb

    peak, peak_kind = _peaks()
    if args.only == "spmv":
        print(json.dumps({"spmv": spmv_leg(peak, args.spmv_reps, args.scale)}), flush=True)
        return
    if args.only == "adjoint":
        print(json.dumps({"adjoint": adjoint_leg(local_rank)}), flush=True)
        return
    if args.only == "large":
        print(json.dumps({"large_qp": large_qp_leg(peak, args.large_iters, args.minres_iters, args.scale)}),
              flush=True)
        return
    if args.only == "large_backward":
        print(json.dumps({"large_backward": large_backward_leg(args.scale)}), flush=True)
        return
    if args.only == "portfolio":
        print(json.dumps({"portfolio": portfolio_leg()}), flush=True)
        return
    if args.only == "reference_gpu":
        print(json.dumps({"reference_gpu": reference_gpu_leg(local_rank)}), flush=True)
        return
    insts = batch_instances(args.batch, rank_first_instance(rank))
    packed = hb.pack(insts)
    bytes_algo_per_inst = np.array([bytes_per_iter(i) for i in insts])
    b = hb.Batch(packed, device_number=local_rank)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        b.solve(stoptol=STOPTOL)
    launches0 = hprqp.launch_count()
    kernel_ms = []
    with ClockSampler(local_rank) as clk:
        barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            kernel_ms.append(b.solve(stoptol=STOPTOL))
        barrier()
        wall = time.perf_counter() - t0
    launches = hprqp.launch_count() - launches0
    res = b.results(vectors=not args.no_warm and rank == 0)
    dev_s = max_over_ranks(sum(kernel_ms) / 1e3, dist)
    wall = max_over_ranks(wall, dist)
    value = whole_job_rate(args.batch, world, args.steps, dev_s)
    iters = res.iter.astype(np.float64)
    algo_bytes = float(np.sum(iters * bytes_algo_per_inst))
    achieved = algo_bytes / (statistics.mean(kernel_ms) / 1e3) / 1e9
    b.close()
    if args.only == "batch":
        print(json.dumps({"value": value, "unit": "solves/s", "kernel_ms": kernel_ms, "achieved_GBs": achieved,
                          "algorithmic_bytes_per_launch": algo_bytes, "mean_iters": float(iters.mean())}), flush=True)
        return
    if args.only == "warm":
        print(json.dumps({"warm_start": warm_start_leg(packed, res, local_rank)}), flush=True)
        return

    # end to end through the C ABI from host buffers
    e2e_times = []
    d2h = 0
    e2e_ok = 0
    barrier()
    for _ in range(args.e2e_steps):
        dt, ok, d2h = e2e_step(packed, local_rank)
        e2e_times.append(dt)
        e2e_ok = ok
    e2e_s = max_over_ranks(sum(e2e_times), dist)
    e2e_value = whole_job_rate(args.batch, world, args.e2e_steps, e2e_s)
    h2d = int(packed.q_indptr.size * 4 + packed.q_indices.size * 4 + packed.q_data.nbytes +
              2 * (packed.a_indices.size * 4 + packed.a_data.nbytes) + 4 * (packed.a_indptr.size + packed.q_indptr.size)
              + packed.c.nbytes + packed.l.nbytes + packed.u.nbytes + packed.AL.nbytes + packed.AU.nbytes)

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators)",
            "config": config, "clocks": clk.summary(), "gpu_launches": int(launches),
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(d2h),
                    "optimal": e2e_ok},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": algo_bytes * BATCH_DRAM_PER_ALGO_BYTE,
                         "traffic_source": "ncu DRAM bytes of a 300-QP solve of this workload (same kernel "
                                           "shapes), scaled by algorithmic bytes (instance-iterations)",
                         "kernel": "k_batch_solve (one solve: a 640-thread launch for the instances of "
                                   "n, m <= 640 and a 1024-thread launch for the rest, concurrent; "
                                   "achieved over their span)",
                         "algorithmic_bytes_per_launch": algo_bytes, "peak_kind": peak_kind},
            "solved_optimal": int(np.sum(res.status == 6)), "mean_iters": float(iters.mean())}

    if rank == 0:
        # plain path: one solve_gpu call per QP over a sample of the same batch
        sample = insts[:args.plain_sample]
        models = [hprqp.build_from_instance(i) for i in sample]
        params = hprqp.Parameters(verbose=False, stoptol=STOPTOL, device_number=local_rank)
        hprqp.optimize(models[0], params)
        call_s = []
        t0 = time.perf_counter()
        for mdl in models:
            t1 = time.perf_counter()
            hprqp.optimize(mdl, params)
            call_s.append(time.perf_counter() - t1)
        plain_rate = len(models) / (time.perf_counter() - t0)
        calls = plain_call_stats(call_s, [2 * (i.Q.nnz + i.A.nnz) for i in sample])
        # the same loop through the host-driven route of solve_gpu (every
        # iteration launched from the host), which small QPs no longer take
        old_route = hprqp.set_single_cta_max_work(0)
        try:
            hprqp.optimize(models[0], params)
            t0 = time.perf_counter()
            for mdl in models:
                hprqp.optimize(mdl, params)
            host_loop_rate = len(models) / (time.perf_counter() - t0)
        finally:
            hprqp.set_single_cta_max_work(old_route)
        line["plain"] = {"value": plain_rate, "unit": "solves/s", "sample": f"{len(models)} instances of the batch",
                         "route": "one CTA of the batch kernel per solve_gpu call (small models)",
                         "host_loop": host_loop_rate, "calls": calls}
        line["batched_over_plain"] = value / world / plain_rate
        line["batched_over_plain_host_loop"] = value / world / host_loop_rate
        if not args.no_spmv:
            line["spmv"] = spmv_leg(peak)
        if not args.no_adjoint:
            line["adjoint"] = adjoint_leg(local_rank)
        if not args.no_warm:
            line["warm_start"] = warm_start_leg(packed, res, local_rank)
        if not args.no_plain_large:
            line["large_qp"] = large_qp_leg(peak)
            line["large_backward"] = large_backward_leg()
            line["portfolio"] = portfolio_leg()
        if not args.no_reference_gpu:
            line["reference_gpu"] = reference_gpu_leg(local_rank)
        ids = list(range(min(args.cpu_sample, args.batch)))
        rate, kind, cdt, ref_solved = cpu_reference_rate(ids, cores)
        line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": cores, "kind": kind,
                                "cpu_model": cpu_model(),
                                "sample": f"{len(ids)} batch instances, one process per core",
                                "single_core": cpu_single_core_timings()}
        # parity of the timed batch itself: its objectives against the
        # reference CPU solves of the same instances
        line["vs_reference_cpu"] = objective_agreement(res.status, res.objective, ref_solved)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
