"""Batched persistent solver vs the CPU oracle and the plain path.

Each instance of a batch must behave like a single solve of the same QP:
same status, objective within 1e-6 relative of the oracle, iterates after K
steps within 1e-8 (the plain-path tolerance), host-recomputed KKT within the
requested tolerance."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = pytest.mark.gpu


def _kept(inst):
    """rows that survive preprocessing (non-empty, not free on both sides)"""
    lens = np.diff(np.asarray(inst.A.indptr))
    free = np.isneginf(inst.AL) & np.isposinf(inst.AU)
    return np.nonzero((lens > 0) & ~free)[0]


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if a.size == 0:
        return 0.0
    return float(np.max(np.abs(a - b)) / max(1.0, float(np.max(np.abs(b)))))


TINY = [i for i in instances.tiny_cases() if i.name != "tall_diag"]


@pytest.mark.parametrize("cap", [1, 10, 100, 250])
def test_batch_iterates_after_k_steps(engine_lib, cap):
    from hprqp import batch

    insts = instances.tiny_cases()
    b = batch.Batch(insts)
    b.solve(stoptol=1e-8, max_iter=cap)
    r = b.results()
    xs, ys, zs, ws = b.split(r.x, "x"), b.split(r.y, "y"), b.split(r.z, "x"), b.split(r.w, "x")
    for k, inst in enumerate(insts):
        om = pyoracle.OracleModel(inst)
        o = om.solve(stoptol=1e-8, max_iter=cap, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == o["status"], inst.name
        assert r.iter[k] == o["iter"], inst.name
        # rows removed by preprocessing come back as 0; the oracle reports the kept rows
        kept_y = ys[k][_kept(inst)]
        for got, ref in ((xs[k], o["x"]), (kept_y, o["y"]), (zs[k], o["z"]), (ws[k], o["w"])):
            assert _rel(got, ref) <= 1e-8, inst.name


@pytest.mark.parametrize("cap", [1, 10])
def test_batch_steps_within_reference_iteration_tolerance(engine_lib, cap):
    """the reference's GPU-vs-CPU step tolerance, 1e-12 absolute
    (tests/gpu/test_gpu_iteration.cpp:42-90), for every fixture model solved
    in one batch; measured differences are at most a few 1e-15"""
    from hprqp import batch

    insts = instances.tiny_cases()
    b = batch.Batch(insts)
    b.solve(stoptol=1e-8, max_iter=cap)
    r = b.results()
    b.close()
    xs, ys, zs, ws = b.split(r.x, "x"), b.split(r.y, "y"), b.split(r.z, "x"), b.split(r.w, "x")
    for k, inst in enumerate(insts):
        o = pyoracle.OracleModel(inst).solve(stoptol=1e-8, max_iter=cap, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == o["status"] and r.iter[k] == o["iter"], inst.name
        for got, ref in ((xs[k], o["x"]), (ys[k][_kept(inst)], o["y"]), (zs[k], o["z"]), (ws[k], o["w"])):
            assert len(ref) == 0 or np.max(np.abs(got - ref)) <= 1e-12, inst.name


@pytest.mark.parametrize("lanes", [0, 1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("cap", [1, 10])
def test_batch_spmv_lane_widths(engine_lib, lanes, cap):
    """Every SpMV lane-group width the autotuner can pick (forced on every
    matrix of every instance; 0 = the autotuned widths) gives the oracle's
    status and iteration count and its iterates within the reference's
    1e-12 step tolerance (tests/gpu/test_gpu_iteration.cpp:42-90), relative
    to the iterate's scale, on the fixture models and batch-recipe QPs."""
    from hprqp import batch

    insts = instances.tiny_cases() + [instances.config3_instance(i) for i in (1, 7, 12)]
    b = batch.Batch(insts)
    tuned = b.spmv_lanes()
    assert set(np.unique(tuned)) <= {1, 2, 4, 8, 16, 32}
    b.set_spmv_lanes(lanes)
    if lanes:
        assert np.all(b.spmv_lanes() == lanes)
    else:
        assert np.array_equal(b.spmv_lanes(), tuned)
    b.solve(stoptol=1e-8, max_iter=cap)
    r = b.results()
    b.close()
    xs, ys, zs, ws = b.split(r.x, "x"), b.split(r.y, "y"), b.split(r.z, "x"), b.split(r.w, "x")
    for k, inst in enumerate(insts):
        o = pyoracle.OracleModel(inst).solve(stoptol=1e-8, max_iter=cap, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == o["status"] and r.iter[k] == o["iter"], (inst.name, lanes)
        for got, ref in ((xs[k], o["x"]), (ys[k][_kept(inst)], o["y"]), (zs[k], o["z"]), (ws[k], o["w"])):
            if len(ref):
                assert np.max(np.abs(got - ref)) <= 1e-12 * max(1.0, float(np.max(np.abs(ref)))), (inst.name, lanes)


def test_batch_between_one_and_two_instances_per_sm(engine_lib):
    """A batch of more instances than SMs but at most two per SM runs on
    512-thread CTAs (one wave, two per SM) instead of 1024-thread ones: the
    fixture models repeated to 13 x 12 = 156 instances give the oracle's
    status, iteration count and iterates within 1e-12 after 10 steps."""
    from hprqp import batch

    tiny = instances.tiny_cases()
    insts = tiny * 13
    assert 148 < len(insts) <= 296
    b = batch.Batch(insts)
    b.solve(stoptol=1e-8, max_iter=10)
    r = b.results()
    b.close()
    xs, ys = b.split(r.x, "x"), b.split(r.y, "y")
    ref = {}
    for k, inst in enumerate(insts):
        o = ref.setdefault(inst.name, pyoracle.OracleModel(inst).solve(stoptol=1e-8, max_iter=10,
                                                                       mode=pyoracle.MODE_GPU_REF))
        assert r.status[k] == o["status"] and r.iter[k] == o["iter"], inst.name
        for got, want in ((xs[k], o["x"]), (ys[k][_kept(inst)], o["y"])):
            assert len(want) == 0 or np.max(np.abs(got - want)) <= 1e-12, inst.name


def test_batch_spmv_lanes_rejects_bad_width(engine_lib):
    from hprqp import batch

    b = batch.Batch(instances.tiny_cases()[:2])
    for bad in (3, 64, -1):
        with pytest.raises(Exception):
            b.set_spmv_lanes(bad)
    b.close()


def test_batch_tiny_converge(engine_lib):
    from hprqp import batch

    r = batch.solve_batch(TINY, stoptol=1e-8)
    for k, inst in enumerate(TINY):
        o = pyoracle.OracleModel(inst).solve(stoptol=1e-8, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == 6 == o["status"], inst.name
        assert abs(r.objective[k] - o["primal_obj"]) <= 1e-6 * max(1.0, abs(o["primal_obj"]))


def test_batch_seeded_matches_oracle_and_plain(engine_lib):
    """Instances of the 4096-QP recipe: batch == plain solve == oracle (the
    plain solve through the host-driven loop, not the one-CTA route, which
    runs the batch kernel itself)."""
    hprqp = engine_lib
    from hprqp import batch

    insts = [instances.config3_instance(k) for k in range(12)]
    b = batch.Batch(insts)
    ms = b.solve(stoptol=1e-6)
    assert ms > 0
    r = b.results()
    xs, ys, zs = b.split(r.x, "x"), b.split(r.y, "y"), b.split(r.z, "x")
    for k, inst in enumerate(insts):
        om = pyoracle.OracleModel(inst)
        o = om.solve(stoptol=1e-6, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == 6 == o["status"], k
        assert abs(r.objective[k] - o["primal_obj"]) <= 1e-6 * abs(o["primal_obj"]), k
        assert abs(int(r.iter[k]) - o["iter"]) <= max(20, o["iter"] // 10), (k, r.iter[k], o["iter"])
        kkt = om.kkt(xs[k], ys[k][_kept(inst)], zs[k])["kkt"]
        assert kkt <= 1.01e-6, (k, kkt)
        old = hprqp.set_single_cta_max_work(0)
        try:
            p = hprqp.optimize(hprqp.build_from_instance(inst), hprqp.Parameters(verbose=False, stoptol=1e-6))
        finally:
            hprqp.set_single_cta_max_work(old)
        assert abs(p.objective - r.objective[k]) <= 1e-6 * abs(p.objective)


def test_batch_resolve_is_deterministic(engine_lib):
    from hprqp import batch

    insts = [instances.config3_instance(k) for k in range(20, 28)]
    b = batch.Batch(insts)
    b.solve(stoptol=1e-6)
    r1 = b.results()
    b.solve(stoptol=1e-6)
    r2 = b.results()
    assert np.array_equal(r1.iter, r2.iter)
    assert np.array_equal(r1.x, r2.x) and np.array_equal(r1.y, r2.y)


def test_batch_noc_and_empty_rows(engine_lib):
    """free variables (noC path) and rows removed by preprocessing."""
    from hprqp import batch

    free = instances.plain_qp(0x48505251 + 90100, n=50, m=20, a_density=0.1, m_rows=10, m_density=0.1, n_eq=12)
    free.l[:] = -np.inf
    free.u[:] = np.inf
    holes = instances.plain_qp(0x48505251 + 90200, n=40, m=16, a_density=0.1, m_rows=8, m_density=0.1, n_eq=8)
    holes.AL[3] = -np.inf
    holes.AU[3] = np.inf  # a free row: deleted by preprocessing
    insts = [free, holes]
    r = batch.solve_batch(insts, stoptol=1e-6)
    for k, inst in enumerate(insts):
        o = pyoracle.OracleModel(inst).solve(stoptol=1e-6, mode=pyoracle.MODE_GPU_REF)
        assert r.status[k] == 6 == o["status"]
        assert abs(r.objective[k] - o["primal_obj"]) <= 1e-6 * max(1.0, abs(o["primal_obj"]))
    ys = np.split(r.y, np.cumsum([i.m for i in insts])[:-1])
    assert ys[1][3] == 0.0 and len(ys[1]) == holes.m


def _one_call(hprqp, packed, **kw):
    """hprqp_solve_batch (create + solve + results + destroy in one call)."""
    import ctypes

    from hprqp import batch as hb

    lib = hprqp._lib()
    hb._configure()
    fn = lib.hprqp_solve_batch
    szp, dbp = ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_double)
    fn.argtypes = [ctypes.c_size_t, szp, szp, ctypes.POINTER(hprqp._MatrixCSR), ctypes.POINTER(hprqp._MatrixCSR),
                   dbp, dbp, dbp, dbp, dbp, dbp, ctypes.POINTER(hb.BatchParams), ctypes.POINTER(ctypes.c_int), szp,
                   dbp, dbp, dbp, dbp, dbp, dbp, dbp]
    p = packed
    n, m = int(p.var_offsets[-1]), int(p.row_offsets[-1])
    keep = []
    Q = hb._csr(n, n, p.q_indptr, p.q_indices, p.q_data, keep)
    A = hb._csr(m, n, p.a_indptr, p.a_indices, p.a_data, keep)
    dp = lambda a: a.ctypes.data_as(dbp)  # noqa: E731
    out = dict(status=np.zeros(p.K, np.int32), iter=np.zeros(p.K, np.uint64), obj=np.zeros(p.K),
               res=np.zeros(p.K), gap=np.zeros(p.K), x=np.zeros(n), y=np.zeros(max(m, 1)), z=np.zeros(n),
               w=np.zeros(n))
    vo = np.ascontiguousarray(p.var_offsets, np.uint64)
    ro = np.ascontiguousarray(p.row_offsets, np.uint64)
    params = hb.default_params(**kw)
    st = fn(p.K, vo.ctypes.data_as(szp), ro.ctypes.data_as(szp), ctypes.byref(Q), ctypes.byref(A), dp(p.c),
            dp(p.AL), dp(p.AU), dp(p.l), dp(p.u), dp(p.obj), ctypes.byref(params),
            out["status"].ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out["iter"].ctypes.data_as(szp),
            dp(out["obj"]), dp(out["res"]), dp(out["gap"]), dp(out["x"]), dp(out["y"]), dp(out["z"]), dp(out["w"]))
    assert st == hprqp.STATUS_OK
    out["y"] = out["y"][:m]
    return out


@pytest.mark.parametrize("count", [12, 1100])
def test_one_call_equals_batch_handle(engine_lib, count):
    """hprqp_solve_batch gives bit for bit what a Batch handle gives on the
    same instances -- also for batches large enough that the one-call form
    builds and launches them in two parts (1100 >= 1024 instances)."""
    from hprqp import batch

    insts = [instances.config4_instance(i) for i in range(count)]
    packed = batch.pack(insts)
    one = _one_call(engine_lib, packed, stoptol=1e-6)
    b = batch.Batch(packed)
    b.solve(stoptol=1e-6)
    r = b.results()
    b.close()
    assert np.array_equal(one["status"], r.status) and np.all(r.status == 6)
    assert np.array_equal(one["iter"].astype(np.int64), r.iter)
    assert np.array_equal(one["obj"], r.objective)
    for key, ref in (("x", r.x), ("y", r.y), ("z", r.z), ("w", r.w)):
        assert np.array_equal(one[key], ref), key


def test_one_call_split_mixed_sizes(engine_lib):
    """The two-part one-call form on 1100 instances of mixed sizes (2 to 2000
    variables), a third of the small ones with a free row that preprocessing
    removes: the first part takes the smallest instances, scattered through
    the caller's order; instances of n, m <= 640 run on 640-thread CTAs and
    the batch-recipe QPs (n up to 2000) mostly on 1024-thread CTAs, in both
    parts and in the handle; every result still lands in the caller's
    packing bit for bit as a Batch handle gives it (removed rows: y = 0)."""
    import dataclasses

    from hprqp import batch

    insts = []
    for i in range(1100):
        if i % 22 == 10:
            insts.append(instances.config3_instance(i))
        elif i % 5 == 0:
            insts.append(instances.config4_instance(i))
        elif i % 5 == 1:
            insts.append(TINY[i % len(TINY)])
        else:
            inst = instances.adjoint_case(i)
            if i % 3 == 0:
                AL, AU = inst.AL.copy(), inst.AU.copy()
                AL[-1], AU[-1] = -np.inf, np.inf
                inst = dataclasses.replace(inst, AL=AL, AU=AU)
            insts.append(inst)
    packed = batch.pack(insts)
    one = _one_call(engine_lib, packed, stoptol=1e-6)
    b = batch.Batch(packed)
    b.solve(stoptol=1e-6)
    r = b.results()
    b.close()
    assert np.array_equal(one["status"], r.status)
    assert np.array_equal(one["iter"].astype(np.int64), r.iter)
    assert np.array_equal(one["obj"], r.objective)
    assert np.array_equal(one["res"], r.residual, equal_nan=True)
    assert np.array_equal(one["gap"], r.gap, equal_nan=True)
    for key, ref in (("x", r.x), ("y", r.y), ("z", r.z), ("w", r.w)):
        assert np.array_equal(one[key], ref), key
    row_end = np.asarray(packed.row_offsets)[1:]
    freed = [k for k in range(1100) if k % 22 != 10 and k % 5 >= 2 and k % 3 == 0]  # adjoint cases, last row free
    assert np.all(one["y"][row_end[freed] - 1] == 0.0)
