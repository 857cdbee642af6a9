"""Benchmark of the HPR-QP engine on one node.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload batch|plain]

Metric (the project's headline): solves/s to 1e-6 relative KKT on the
4096-instance batch workload (n ~ U{50..2000}, m ~ U{n/4..n}, seeded), next
to the plain one-QP-per-call path, plus the SpMV bandwidth of the large
power-law QP (n=1e6, m=5e5, nnz(A)~1e7, nnz(Q)~3.2e7) against the measured
HBM peak.

One step = one pass of the solver over the whole batch of synthetic QPs.
``value`` is measured with the inputs already resident on the device;
``e2e`` goes through the C ABI with host buffers (host->device copies and the
read-back of the solutions inside the timed region).  Multi-GPU runs are
replicas: every rank solves its own copy of the batch (weak scaling), and the
time is the max over ranks.

``--impl reference`` times the reference's own CPU implementation of the path
(oracle/_ref/libhprqp_ref_cpu.so, compiled from the reference sources; the
C oracle when that library is absent) on the host cores, on a bounded sample
of the same workload.
"""
from __future__ import annotations

import argparse
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

METRIC = "solves/s to 1e-6 rel-KKT, batched vs plain on 1 B200; SpMV GB/s vs HBM peak"
STOPTOL = 1e-6


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# --------------------------------------------------------------------------
# clocks sampling during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = Path("/tmp") / f"hprqp_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
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
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# --------------------------------------------------------------------------
# workloads
# --------------------------------------------------------------------------
def batch_instances(count: int, start: int = 0):
    from hprqp import instances

    return instances.config3(count, start)


def algorithmic_bytes_per_iter(inst) -> float:
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
        out.append(int(r["status"]))
    return out


def cpu_reference_rate(sample: int, cores: int):
    """Reference CPU solves/s over `sample` batch instances on `cores` host
    processes (spawned, one instance at a time per process)."""
    import pyoracle

    kind = "reference" if pyoracle.ref_available() else "port"
    ids = list(range(sample))
    chunks = [ids[i::cores] for i in range(cores)]
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(cores) as pool:
        statuses = sum(pool.map(_ref_worker, [(c, STOPTOL) for c in chunks if c]), [])
    dt = time.perf_counter() - t0
    return sample / dt, kind, dt, statuses


def spmv_roofline(peak_gbs: float):
    """Row-block SpMV on the large power-law QP's A, A' and Q."""
    import hprqp
    from hprqp import instances

    inst = instances.config1()
    rng = np.random.default_rng(5)
    out = {}
    for name, (ip, ii, dd, nrow, ncol) in {
        "A": (inst.A.indptr, inst.A.indices, inst.A.data, inst.m, inst.n),
        "Q": (inst.Q.indptr, inst.Q.indices, inst.Q.data, inst.n, inst.n),
    }.items():
        x = rng.standard_normal(ncol)
        _, ms = hprqp.spmv(ip, ii, dd, ncol, x, reps=10)
        nnz = int(ip[-1])
        algo = 12 * nnz + 4 * (nrow + 1) + 8 * ncol + 8 * nrow
        gbs = algo / (ms * 1e-3) / 1e9
        out[name] = {"nnz": nnz, "ms": ms, "GB/s": gbs, "frac": gbs / peak_gbs, "bytes": algo}
    return out


def run_plain(instances_list, params_kw):
    import hprqp

    models = [hprqp.build_from_instance(inst) for inst in instances_list]
    params = hprqp.Parameters(verbose=False, stoptol=STOPTOL, **params_kw)
    iters = []
    ok = 0
    for mdl in models:
        r = hprqp.optimize(mdl, params, as_numpy=True)
        iters.append(r.iter)
        ok += r.status_code == hprqp.STATUS_OPTIMAL
    return iters, ok


# --------------------------------------------------------------------------
# main
# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=["plain"])
    ap.add_argument("--batch", type=int, default=64, help="instances per step")
    ap.add_argument("--cpu-sample", type=int, default=64)
    ap.add_argument("--no-spmv", action="store_true")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cores = os.cpu_count() or 1

    config = {"workload": f"config3 batch: {args.batch} seeded QPs, n~U{{50..2000}}, m~U{{n/4..n}}, "
                          f"stoptol {STOPTOL:g}",
              "global_batch": args.batch * world, "parallelism": f"replicas x{world}",
              "l2": "inputs larger than L2 (126 MB) across a step"}

    if args.impl == "reference":
        if rank != 0:
            return
        rates = []
        kind = "port"
        for _ in range(args.warmup):
            pass  # the CPU reference has no warm-up state; warm-up steps are skipped
        t_total = 0.0
        for _ in range(args.steps):
            rate, kind, dt, _ = cpu_reference_rate(args.cpu_sample, cores)
            rates.append(rate)
            t_total += dt
        value = float(statistics.median(rates))
        line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
                "config": config, "impl": "reference",
                "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": kind,
                                 "sample": f"{args.cpu_sample} batch instances per step"},
                "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    import hprqp

    peak, peak_kind = _peaks()
    insts = batch_instances(args.batch, 1000 * rank)
    params_kw = {"device_number": local_rank}
    for _ in range(args.warmup):
        run_plain(insts, params_kw)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    launches0 = hprqp.launch_count()
    with ClockSampler(local_rank) as clk:
        barrier()
        t0 = time.perf_counter()
        iters_all = []
        for _ in range(args.steps):
            iters, ok = run_plain(insts, params_kw)
            iters_all.extend(iters)
        barrier()
        dt = time.perf_counter() - t0
    launches = hprqp.launch_count() - launches0
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([dt], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dt = float(t.item())
    value = args.batch * world * args.steps / dt

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators)",
            "config": config, "clocks": clk.summary(), "gpu_launches": int(launches),
            "e2e": {"value": value, "unit": "solves/s",
                    "h2d_bytes_per_step": int(sum(12 * i.Q.nnz + 12 * i.A.nnz + 8 * (3 * i.n + 2 * i.m)
                                                  for i in insts)),
                    "d2h_bytes_per_step": int(sum(8 * (3 * i.n + i.m) for i in insts))},
            "mean_iters": float(np.mean(iters_all))}
    if rank == 0 and not args.no_spmv:
        sp = spmv_roofline(peak)
        line["roofline"] = {"bound": "hbm", "achieved": sp["Q"]["GB/s"], "peak": peak, "unit": "GB/s",
                            "frac": sp["Q"]["GB/s"] / peak, "traffic": None,
                            "kernel": "k_rowblock<EpiStore> (y = Q x, n=1e6, nnz 3.2e7)",
                            "peak_kind": peak_kind}
        line["spmv"] = sp
    if rank == 0:
        rate, kind, cdt, _ = cpu_reference_rate(min(args.cpu_sample, 32), cores)
        line["cpu_baseline"] = {"value": rate, "unit": "solves/s", "cores": cores, "kind": kind,
                                "sample": f"{min(args.cpu_sample, 32)} batch instances"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
