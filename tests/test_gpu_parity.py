"""GPU parity of the plain HPR path against the CPU oracle.

Tolerances follow the reference's own GPU-vs-CPU tests
(tests/gpu/test_gpu_*.c): SpMV results per row within 1e-13 of the
magnitude sum; scaling within 1e-10 (test_gpu_scale.c:46-60); eigenvalues
within 1e-6 (lambda_max(AA'), test_gpu_eigs.c:37-38); iterates after K steps
within 1e-8 relative (test_gpu_solver.c:73-81 uses 1e-8 end to end);
converged objectives within 1e-6 relative (the project's acceptance
criterion) with the KKT residual recomputed in FP64 on the host.
"""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


def _spmv_check(hprqp, indptr, indices, data, ncol, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(ncol)
    y, _ = hprqp.spmv(indptr, indices, data, ncol, x)
    ref = pyoracle.matvec(indptr, indices, data, x)
    bound = np.zeros(len(indptr) - 1)
    for r in range(len(indptr) - 1):
        s, e = indptr[r], indptr[r + 1]
        bound[r] = np.sum(np.abs(data[s:e] * x[indices[s:e]]))
    assert np.all(np.abs(y - ref) <= 1e-13 * (bound + 1e-300) + 1e-300)


def _csr_from_lengths(rng, lens, ncol):
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    indices = np.concatenate([np.sort(rng.choice(ncol, size=l, replace=False)) if l else np.zeros(0, np.int64)
                              for l in lens]).astype(np.int64)
    data = rng.standard_normal(int(indptr[-1]))
    return indptr, indices, data


def test_spmv_row_length_mix(engine_lib):
    rng = np.random.default_rng(1)
    ncol = 5000
    # empty rows, singletons, medium, rows longer than one staged tile, one very long row
    lens = np.concatenate([np.zeros(50, int), np.ones(300, int), rng.integers(2, 40, 400),
                           rng.integers(100, 700, 30), [2049, 4097, 4999], np.zeros(10, int)])
    rng.shuffle(lens)
    indptr, indices, data = _csr_from_lengths(rng, lens, ncol)
    _spmv_check(engine_lib, indptr, indices, data, ncol, 2)


def test_spmv_zipf_rows(engine_lib):
    rng = np.random.default_rng(3)
    lens = np.minimum(rng.zipf(1.5, 20000), 3000)
    indptr, indices, data = _csr_from_lengths(rng, lens, 4000)
    _spmv_check(engine_lib, indptr, indices, data, 4000, 4)


def test_spmv_contiguous_runs(engine_lib):
    """rows made of consecutive columns (dense blocks) run the staged tile
    kernel; ragged lengths, empty rows and a row longer than a tile"""
    rng = np.random.default_rng(7)
    ncol = 3000
    lens = np.concatenate([rng.integers(1, 300, 500), [1500, 2999], np.zeros(5, int), np.ones(40, int)])
    rng.shuffle(lens)
    indptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    indices = np.concatenate([np.arange(s, s + l) for s, l in
                              zip((rng.integers(0, ncol - l + 1) for l in lens), lens)]).astype(np.int64)
    data = rng.standard_normal(int(indptr[-1]))
    _spmv_check(engine_lib, indptr, indices, data, ncol, 8)


def test_gather_bound_checksum(engine_lib):
    """hprqp_b200_gather_bound does the whole pass: its sum of products is
    the sum of the entries of M x"""
    rng = np.random.default_rng(9)
    lens = np.minimum(rng.zipf(1.6, 30000), 2500)
    indptr, indices, data = _csr_from_lengths(rng, lens, 6000)
    x = rng.standard_normal(6000)
    y, _ = engine_lib.spmv(indptr, indices, data, 6000, x)
    total, ms = engine_lib.gather_bound(indptr, indices, data, 6000, x, reps=3)
    assert ms > 0
    assert abs(total - float(np.sum(y))) <= 1e-12 * float(np.sum(np.abs(data * x[indices])))


def test_spmv_reference_exact_values(engine_lib):
    """tests/gpu/test_gpu_spmv_operation.cu:27-29, 47-52: exact products of
    a 3x3 CSR with two vectors."""
    indptr, indices = np.array([0, 2, 3, 5]), np.array([0, 2, 1, 0, 2])
    data = np.array([2.0, -1.0, 3.0, 4.0, 5.0])
    y, _ = engine_lib.spmv(indptr, indices, data, 3, np.array([1.0, 2.0, 3.0]))
    assert y.tolist() == [-1.0, 6.0, 19.0]
    y, _ = engine_lib.spmv(indptr, indices, data, 3, np.array([-2.0, 1.0, 4.0]))
    assert y.tolist() == [-8.0, 3.0, 12.0]


def _packed_fixture(fixture):
    """the eight row patterns of tests/gpu/test_gpu_packed_spmv.cu:18-22"""
    m = {0: 1, 1: 127, 2: 257}.get(fixture, 128)
    n = 311 if fixture == 2 else 256
    indptr, indices, data = [0], [], []
    for i in range(m):
        k = {0: 2, 1: 3, 2: 7, 3: 31, 4: 33, 6: 0}.get(fixture)
        if fixture == 5:
            k = 32 if i == 0 else 1
        if fixture == 7:
            k = 0 if i % 5 == 0 else 5
        for j in sorted({(i * 11 + t * 7) % n for t in range(k)}):
            indices.append(j)
            data.append(np.sin(1.7 * i + 0.3 * j))
        indptr.append(len(indices))
    return np.array(indptr), np.array(indices, dtype=np.int64), np.array(data), n


@pytest.mark.parametrize("fixture", range(8))
def test_spmv_reference_patterns(engine_lib, fixture):
    """tests/gpu/test_gpu_packed_spmv.cu:9-14: each pattern and its
    transpose within 1e-12 of an extended-precision sum, x_j = sin(.19 j) +
    cos(.011 j)."""
    import math

    import scipy.sparse as sp

    indptr, indices, data, n = _packed_fixture(fixture)
    M = sp.csr_matrix((data, indices, indptr), shape=(len(indptr) - 1, n))
    for mat in (M, M.T.tocsr()):
        mat.sort_indices()
        x = np.array([math.sin(0.19 * j) + math.cos(0.011 * j) for j in range(mat.shape[1])])
        y, _ = engine_lib.spmv(mat.indptr, mat.indices, mat.data, mat.shape[1], x)
        for i in range(mat.shape[0]):
            s, e = mat.indptr[i], mat.indptr[i + 1]
            ref = math.fsum(mat.data[s:e] * x[mat.indices[s:e]]) if e > s else 0.0
            assert abs(y[i] - ref) / (1.0 + abs(ref)) < 1e-12


def test_spmv_empty_matrix(engine_lib):
    indptr = np.zeros(11, np.int64)
    y, _ = engine_lib.spmv(indptr, np.zeros(0, np.int64), np.zeros(0), 5, np.ones(5))
    assert np.array_equal(y, np.zeros(10))


@pytest.mark.parametrize("name", ["standard", "scale", "dense_q", "tall_diag", "iteration_standard", "config0",
                                  "config3_5"])
def test_setup_matches_oracle(engine_lib, name):
    hprqp = engine_lib
    if name == "config0":
        inst = instances.config0()
    elif name.startswith("config3"):
        inst = instances.config3_instance(int(name.split("_")[1]))
    else:
        inst = {i.name: i for i in instances.tiny_cases()}[name]
    model = hprqp.build_from_instance(inst)
    info = hprqp.setup_info(model, dump=True)
    om = pyoracle.OracleModel(inst)
    sc = om.scale(mode=pyoracle.MODE_GPU_REF)
    st = om.setup(mode=pyoracle.MODE_GPU_REF)
    assert _rel(info["row_norm"], sc["row_norm"]) <= 1e-10
    assert _rel(info["col_norm"], sc["col_norm"]) <= 1e-10
    assert _rel(info["q_val"], sc["q_data"]) <= 1e-10
    assert _rel(info["a_val"], sc["a_data"]) <= 1e-10
    assert _rel(info["c"], sc["c"]) <= 1e-10
    assert info["Q_is_diag"] == st["Q_is_diag"] and info["noC"] == st["noC"]
    assert abs(info["sigma"] - st["sigma"]) <= 1e-10 * max(1.0, st["sigma"])
    assert abs(info["lambda_max_A"] - st["lambda_max_A"]) <= 1e-6 * max(1.0, st["lambda_max_A"])
    assert abs(info["lambda_max_Q"] - st["lambda_max_Q"]) <= 1e-4 * max(1.0, st["lambda_max_Q"])


def _solve_pair(hprqp, inst, **kw):
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, **kw)
    r = hprqp.optimize(model, params, as_numpy=True)
    o = pyoracle.OracleModel(inst).solve(mode=pyoracle.MODE_GPU_REF, **kw)
    return r, o


TINY = [i for i in instances.tiny_cases()]


@pytest.mark.parametrize("inst", TINY, ids=[i.name for i in TINY])
@pytest.mark.parametrize("cap", [1, 10, 100, 250])
def test_iterates_after_k_steps(engine_lib, plain_path, inst, cap):
    r, o = _solve_pair(engine_lib, inst, stoptol=1e-8, max_iter=cap)
    assert r.status_code == o["status"]
    assert r.iter == o["iter"]
    for key in ("x", "y", "z", "w"):
        assert _rel(getattr(r, key), o[key]) <= 1e-8, key


@pytest.mark.parametrize("inst", TINY, ids=[i.name for i in TINY])
@pytest.mark.parametrize("cap", [1, 10])
def test_steps_within_reference_iteration_tolerance(engine_lib, plain_path, inst, cap):
    """the reference's GPU-vs-CPU step tolerance, 1e-12 absolute
    (tests/gpu/test_gpu_iteration.cpp:42-90), on the whole solve after 1
    and 10 steps (setup, scaling and power iterations included); measured
    differences are at most a few 1e-16"""
    r, o = _solve_pair(engine_lib, inst, stoptol=1e-8, max_iter=cap)
    assert r.status_code == o["status"] and r.iter == o["iter"]
    for key in ("x", "y", "z", "w"):
        got, ref = np.asarray(getattr(r, key), float), np.asarray(o[key], float)
        assert got.shape == ref.shape and (got.size == 0 or np.max(np.abs(got - ref)) <= 1e-12), key


@pytest.mark.parametrize("inst", [i for i in TINY if i.name != "tall_diag"],
                         ids=[i.name for i in TINY if i.name != "tall_diag"])
def test_tiny_solves_converge_like_oracle(engine_lib, plain_path, inst):
    r, o = _solve_pair(engine_lib, inst, stoptol=1e-8)
    assert r.status_code == o["status"] == engine_lib.STATUS_OPTIMAL
    assert abs(r.objective - o["primal_obj"]) <= 1e-6 * max(1.0, abs(o["primal_obj"]))
    assert abs(r.iter - o["iter"]) <= max(10, o["iter"] // 10)


def test_config0_end_to_end(engine_lib, plain_path):
    """n=1000, m=500 seeded QP at 1e-6: same tolerance reached, objective
    within 1e-6 relative, KKT recomputed on the host in FP64."""
    inst = instances.config0()
    r, o = _solve_pair(engine_lib, inst, stoptol=1e-6)
    assert r.status_code == o["status"] == engine_lib.STATUS_OPTIMAL
    assert abs(r.objective - o["primal_obj"]) <= 1e-6 * abs(o["primal_obj"])
    k = pyoracle.OracleModel(inst).kkt(r.x, r.y, r.z)
    assert k["kkt"] <= 1e-6 * 1.01
    assert abs(r.iter - o["iter"]) <= max(20, o["iter"] // 10)


def test_single_cta_route_keeps_host_loop_bookkeeping(engine_lib, capfd):
    """The one-CTA route of solve_gpu reports what the host loop reports:
    status, iterations, the 1e-4 / 1e-6 milestones, and (verbose) the same
    printed iterations of the residual log."""
    hprqp = engine_lib
    model = hprqp.build_from_instance(instances.config0())
    out = {}
    for route, work in (("host_loop", 0), ("single_cta", 1 << 40)):
        old = hprqp.set_single_cta_max_work(work)
        try:
            capfd.readouterr()
            r = hprqp.optimize(model, hprqp.Parameters(verbose=True, stoptol=1e-6), as_numpy=True)
            text = capfd.readouterr().out
        finally:
            hprqp.set_single_cta_max_work(old)
        iters = [int(line.split()[0]) for line in text.splitlines()
                 if line.strip() and line.split()[0].isdigit() and len(line.split()) == 8]
        out[route] = (r, iters)
    (a, ia), (b, ib) = out["host_loop"], out["single_cta"]
    assert a.status_code == b.status_code == hprqp.STATUS_OPTIMAL
    assert a.iter == b.iter and a.iter_4 == b.iter_4 and a.iter_6 == b.iter_6
    assert ia == ib and ia[0] == 0 and ia[-1] == a.iter
    assert 0.0 < b.time_4 <= b.time_6 <= b.time


def test_reference_python_api_gpu_path(engine_lib, plain_path):
    """python/tests/test_hprqp.py:44-65 of the reference, GPU side."""
    hprqp = engine_lib
    assert hprqp.gpu_backend_available()
    model = hprqp.build_from_qabc([[2.0, 0.0], [0.0, 4.0]], [2.0, 1.0], [[1.0, 1.0]], [2.0], [2.0], [0.0, 0.0],
                                  [10.0, 10.0])
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, use_gpu=True, device_number=0))
    assert r.status_code == hprqp.STATUS_OPTIMAL
    assert abs(r.objective - 71.0 / 12.0) < 1e-6
    model2 = hprqp.build_from_qabc([[2.0, 0.0], [0.0, 2.0]], [-4.0, -2.0], [], [], [], [-np.inf, -np.inf],
                                   [np.inf, np.inf])
    r2 = hprqp.optimize(model2, hprqp.Parameters(verbose=False, stoptol=1e-8))
    assert r2.status_code == hprqp.STATUS_OPTIMAL
    assert abs(r2.objective + 5.0) < 1e-6 and abs(r2.x[0] - 2.0) < 1e-6 and abs(r2.x[1] - 1.0) < 1e-6
    assert r2.y == []


def test_max_iter_zero_and_invalid_device(engine_lib, plain_path):
    hprqp = engine_lib
    model = hprqp.build_from_instance(TINY[0])
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, max_iter=0))
    assert r.status_code == hprqp.STATUS_MAX_ITER and len(r.x) == 2
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, device_number=999))
    assert r.status_code == hprqp.STATUS_INVALID_ARGUMENT


def test_residual_kernels_known_answers(engine_lib):
    """The residual kernels at seeded points of the reference's residual
    fixture (tests/gpu/test_gpu_residuals.c:72-89 of the reference): pobj 3,
    dobj -1, errRd 0.46, errRp 0, gap 1, KKT 1; at iteration 0 the bound
    violation of x = (11, 1) gives errRp 1."""
    hprqp = engine_lib
    inst = {i.name: i for i in instances.tiny_cases()}["residuals"]
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, use_scaling=False)
    r = hprqp.residuals(model, [1.0, 1.0], [0.5], [0.2, 0.3], iter=1, params=params)
    for key, want in (("primal_obj", 3.0), ("dual_obj", -1.0), ("err_rd", 0.46), ("err_rp", 0.0), ("gap", 1.0),
                      ("kkt", 1.0)):
        assert abs(r[key] - want) <= 1e-8, (key, r[key])
    r0 = hprqp.residuals(model, [11.0, 1.0], [0.0], [0.0, 0.0], iter=0, params=params)
    assert abs(r0["err_rp"] - 1.0) <= 1e-8


@pytest.mark.parametrize("scaling", [True, False])
def test_residual_kernels_match_oracle(engine_lib, scaling):
    """At a random point of the n=1000 QP, with and without scaling, the
    device residuals agree with the oracle's FP64 host recomputation."""
    hprqp = engine_lib
    inst = instances.config0()
    model = hprqp.build_from_instance(inst)
    rng = np.random.default_rng(8)
    x = rng.uniform(-2, 2, inst.n)
    y = rng.standard_normal(inst.m)
    z = rng.standard_normal(inst.n)
    r = hprqp.residuals(model, x, y, z, iter=5, params=hprqp.Parameters(verbose=False, use_scaling=scaling))
    k = pyoracle.OracleModel(inst).kkt(x, y, z)
    for key in ("err_rp", "err_rd", "gap", "primal_obj", "dual_obj"):
        assert abs(r[key] - k[key]) <= 1e-10 * max(1.0, abs(k[key])), (key, r[key], k[key])


def test_reference_mps_fixture_through_binding(engine_lib, plain_path):
    """tests/test_binding_api.c:16-118 of the reference on its own
    simple_qp.mps: 2 variables and 2 rows, max_iter 0 gives MAX_ITER with
    solution vectors; solved to 1e-8 it matches the reference CPU solver's
    result recorded in tests/golden/simple_qp.json."""
    import json
    from pathlib import Path

    hprqp = engine_lib
    golden = Path(__file__).resolve().parent / "golden"
    ref = json.loads((golden / "simple_qp.json").read_text())
    model = hprqp.read_from_mps(golden / "simple_qp.mps")
    assert (model.num_variables, model.num_constraints) == (2, 2)
    r0 = hprqp.optimize(model, hprqp.Parameters(verbose=False, max_iter=0))
    assert r0.status_code == hprqp.STATUS_MAX_ITER == ref["max_iter0"]["status"]
    assert len(r0.x) == 2 and len(r0.y) == 2
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=1e-8))
    want = ref["solve_1e-8"]
    assert r.status_code == want["status"] == hprqp.STATUS_OPTIMAL
    assert abs(r.objective - want["primal_obj"]) <= 1e-6 * max(1.0, abs(want["primal_obj"]))
    assert np.allclose(r.x, want["x"], atol=1e-5) and np.allclose(r.y, want["y"], atol=1e-5)
