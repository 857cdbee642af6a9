"""The SpMV setup of rowblock.cuh on CPU: tile plan, long-row chunks,
row-start bitmap, array padding and the tile-kernel choice, through a
host-only probe compiled from the same header (tests/native)."""
from __future__ import annotations

import json
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
TILE_ROWS, TILE_CAP, CHUNK = 64, 1024, 1024


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path_factory.mktemp("probe") / "tile_plan_probe"
    # a clean environment: a sanitizer runtime preloaded into the test
    # process must not reach nvcc or the probe
    env = {k: v for k, v in os.environ.items() if k != "LD_PRELOAD"}
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17",
                    f"-I{ROOT / 'hpr-qp-c_b200' / 'csrc'}", f"-I{ROOT / 'include'}", "-o", str(exe),
                    str(ROOT / "tests" / "native" / "tile_plan_probe.cu")], check=True, env=env)

    def run(indptr, indices):
        text = f"{len(indptr) - 1} {len(indices)}\n" + " ".join(map(str, indptr)) + "\n" + \
            " ".join(map(str, indices)) + "\n"
        out = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True, env=env).stdout
        return json.loads(out)

    return run


def _csr(rng, lens, ncol, contiguous=False):
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(int)
    parts = []
    for l in lens:
        if contiguous and l:
            s = rng.integers(0, ncol - l + 1)
            parts.append(np.arange(s, s + l))
        else:
            parts.append(np.sort(rng.choice(ncol, size=l, replace=False)))
    indices = np.concatenate(parts).astype(int) if parts else np.zeros(0, int)
    return indptr, indices


def _check_plan(plan, indptr):
    lens = np.diff(indptr)
    nrow = len(lens)
    covered = []
    for r0, r1, entries, zero in plan["tiles"]:
        assert zero == 0 and 0 < r1 - r0 <= TILE_ROWS
        assert entries == indptr[r1] - indptr[r0] and (entries <= TILE_CAP)
        assert np.all(lens[r0:r1] <= TILE_CAP)
        covered += list(range(r0, r1))
    long_rows = [r for r, _ in plan["long_rows"]]
    assert sorted(covered + long_rows) == list(range(nrow))
    assert long_rows == [r for r in range(nrow) if lens[r] > TILE_CAP]
    # chunks: each long row cut into consecutive <= CHUNK pieces, slots in order
    for i, (row, first) in enumerate(plan["long_rows"]):
        last = plan["long_rows"][i + 1][1] if i + 1 < len(plan["long_rows"]) else len(plan["chunks"])
        pieces = plan["chunks"][first:last]
        assert pieces[0][1] == indptr[row] and pieces[-1][2] == indptr[row + 1]
        for j, (r, k0, k1, slot) in enumerate(pieces):
            assert r == row and slot == first + j and 0 < k1 - k0 <= CHUNK
            if j:
                assert k0 == pieces[j - 1][2]
    # a tile stops only when the next row would break a limit
    for (r0, r1, entries, _), nxt in zip(plan["tiles"], plan["tiles"][1:] + [None]):
        if r1 < nrow and lens[r1] <= TILE_CAP and r1 - r0 < TILE_ROWS:
            assert entries + lens[r1] > TILE_CAP


def _check_heads(plan, indptr):
    nnz = int(indptr[-1])
    assert plan["padded_nnz"] % 8 == 0 and plan["padded_nnz"] >= nnz + 1
    assert len(plan["heads"]) == plan["padded_nnz"] // 8
    bits = np.unpackbits(np.array(plan["heads"], np.uint8), bitorder="little")
    starts = {int(indptr[r]) for r in range(len(indptr) - 1) if indptr[r + 1] > indptr[r]}
    assert set(np.nonzero(bits)[0].tolist()) == starts


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_ragged_rows(probe, seed):
    rng = np.random.default_rng(seed)
    lens = np.concatenate([np.zeros(70, int), np.ones(200, int), rng.integers(2, 60, 300),
                           [1023, 1024, 1025, 2048, 2049, 4100], rng.integers(0, 5, 130)])
    rng.shuffle(lens)
    indptr, indices = _csr(rng, lens, 6000)
    plan = probe(indptr, indices)
    _check_plan(plan, indptr)
    _check_heads(plan, indptr)
    assert plan["staged"] == 0


def test_empty_and_tiny(probe):
    plan = probe([0, 0, 0, 0], [])
    assert plan["tiles"] == [[0, 3, 0, 0]] and plan["chunks"] == [] and plan["padded_nnz"] == 8
    assert plan["heads"] == [0] and plan["staged"] == 0
    plan = probe([0, 1], [7])
    assert plan["heads"] == [1, 0] and plan["staged"] == 0


def test_kernel_choice(probe):
    rng = np.random.default_rng(4)
    lens = rng.integers(1, 300, 200)
    indptr, indices = _csr(rng, lens, 5000, contiguous=True)
    assert probe(indptr, indices)["staged"] == 1
    indptr, indices = _csr(rng, lens, 5000)
    assert probe(indptr, indices)["staged"] == 0
    # exactly half of the in-row pairs consecutive: staged
    assert probe([0, 3, 6], [0, 1, 5, 2, 4, 5])["staged"] == 1
    assert probe([0, 3, 6], [0, 2, 5, 2, 4, 5])["staged"] == 0
