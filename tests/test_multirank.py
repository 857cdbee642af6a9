"""Multi-rank host logic of bench.py on CPU: two gloo ranks (world size 2,
127.0.0.1), as `bench.py --gpus 2` runs them under torchrun with NCCL.

Replicas: every rank solves its own disjoint seeded batch, the time is the
max over ranks, and the whole-job rate counts all ranks' instances."""
from __future__ import annotations

import json
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    sys.path[:0] = [str(ROOT), str(ROOT / "hpr-qp-c_b200" / "python"), str(ROOT / "oracle")]
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        per_rank_seconds = 1.0 + rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(per_rank_seconds, dist, device="cpu")
        first = bench.rank_first_instance(rank)
        ids = list(range(first, first + 4096))
        insts = bench.batch_instances(2, first)
        rate = bench.whole_job_rate(4096, world, 3, slowest)
        # every rank takes the same collective steps: a second reduction
        again = bench.max_over_ranks(0.5 * (rank + 1), dist, device="cpu")
        out = {"rank": rank, "slowest": slowest, "again": again, "ids": [ids[0], ids[-1]], "rate": rate,
               "n0": insts[0].n, "c0": float(insts[0].c[0])}
        Path(out_dir, f"rank{rank}.json").write_text(json.dumps(out))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as tmp

    port = _free_port()
    tmp.spawn(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r = [json.loads((tmp_path / f"rank{k}.json").read_text()) for k in range(2)]
    # max over ranks, identical on both ranks
    assert r[0]["slowest"] == r[1]["slowest"] == 2.0
    assert r[0]["again"] == r[1]["again"] == 1.0
    # whole-job rate: all ranks' instances over the slowest rank's time
    assert r[0]["rate"] == pytest.approx(4096 * 2 * 3 / 2.0)
    # disjoint instance ranges, different data
    assert r[0]["ids"][1] < r[1]["ids"][0]
    assert (r[0]["n0"], r[0]["c0"]) != (r[1]["n0"], r[1]["c0"])


def test_single_rank_is_identity():
    sys.path[:0] = [str(ROOT)]
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.rank_first_instance(0) == 0
    assert bench.whole_job_rate(10, 1, 2, 4.0) == 5.0


def test_clock_sampler_maps_visible_devices():
    """Under torchrun each rank's CUDA device 0..N-1 is renumbered by
    CUDA_VISIBLE_DEVICES; the clock samples must come from that physical GPU."""
    sys.path[:0] = [str(ROOT)]
    import bench

    pid = bench.ClockSampler.physical_id
    assert pid(1, "") == "1"
    assert pid(0, "3,5") == "3" and pid(1, "3,5") == "5"
    assert pid(0, "GPU-8f3a, GPU-11b2") == "GPU-8f3a" and pid(1, "GPU-8f3a, GPU-11b2") == "GPU-11b2"
    assert pid(4, "3,5") == "4"  # out of range: leave the index alone
