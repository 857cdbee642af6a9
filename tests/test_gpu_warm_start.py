"""Warm-started batch solves (hprqp_batch_set_warm_start).

The reference has no warm start (its iterates start at zero), so the checks
are: a zero warm start reproduces the cold solve exactly; a warm start at a
solution converges to the same optimum (objective of the cold solve, KKT
recomputed on the host below the tolerance) in a fraction of the
iterations; a warm start at the solution of a perturbed batch reaches the
cold solve's optimum; clearing the warm start restores the cold solve."""
from __future__ import annotations

import numpy as np
import pytest

import pyoracle
from hprqp import instances

pytestmark = pytest.mark.gpu


def _kept(inst):
    lens = np.diff(np.asarray(inst.A.indptr))
    free = np.isneginf(inst.AL) & np.isposinf(inst.AU)
    return np.nonzero((lens > 0) & ~free)[0]


def _mixed_batch():
    insts = [instances.config3_instance(k) for k in range(40, 46)]
    free = instances.plain_qp(0x48505251 + 91100, n=50, m=20, a_density=0.1, m_rows=10, m_density=0.1, n_eq=12)
    free.l[:] = -np.inf
    free.u[:] = np.inf  # noC path: Q w is carried with the iterates
    holes = instances.plain_qp(0x48505251 + 91200, n=40, m=16, a_density=0.1, m_rows=8, m_density=0.1, n_eq=8)
    holes.AL[3] = -np.inf
    holes.AU[3] = np.inf  # removed by preprocessing: y0 of that row is ignored
    return insts + [free, holes]


def _same(r1, r2):
    assert np.array_equal(r1.status, r2.status)
    assert np.array_equal(r1.iter, r2.iter)
    for a, b in ((r1.x, r2.x), (r1.y, r2.y), (r1.z, r2.z), (r1.w, r2.w), (r1.objective, r2.objective)):
        assert np.array_equal(a, b)


def test_zero_warm_start_is_the_cold_solve(engine_lib):
    from hprqp import batch

    b = batch.Batch(_mixed_batch())
    b.solve(stoptol=1e-6)
    cold = b.results()
    b.set_warm_start(np.zeros(b.n), np.zeros(b.m), np.zeros(b.n))
    b.solve(stoptol=1e-6)
    _same(cold, b.results())
    b.set_warm_start(None)  # cleared: the cold solve again
    b.solve(stoptol=1e-6)
    _same(cold, b.results())
    b.close()


def test_warm_start_at_solution(engine_lib):
    from hprqp import batch

    insts = _mixed_batch()
    b = batch.Batch(insts)
    b.solve(stoptol=1e-8)
    cold = b.results()
    assert np.all(cold.status == 6)
    b.set_warm_start(cold.x, cold.y, cold.w)
    b.solve(stoptol=1e-8)
    warm = b.results()
    b.close()
    assert np.all(warm.status == 6)
    # never accepted before the first step; far fewer steps than from zero
    assert np.all(warm.iter >= 1)
    assert warm.iter.sum() <= 0.25 * cold.iter.sum(), (warm.iter, cold.iter)
    xs, ys, zs = (np.split(v, np.cumsum([getattr(i, d) for i in insts])[:-1])
                  for v, d in ((warm.x, "n"), (warm.y, "m"), (warm.z, "n")))
    for k, inst in enumerate(insts):
        assert abs(warm.objective[k] - cold.objective[k]) <= 1e-6 * max(1.0, abs(cold.objective[k])), k
        kkt = pyoracle.OracleModel(inst).kkt(xs[k], ys[k][_kept(inst)], zs[k])["kkt"]
        assert kkt <= 1.01e-8, (k, kkt)


def test_warm_start_from_perturbed_batch(engine_lib):
    """The training-loop case: the data moved a little since the last solve."""
    from hprqp import batch

    base = [instances.config3_instance(k) for k in range(60, 68)]
    b0 = batch.Batch(base)
    b0.solve(stoptol=1e-6)
    prev = b0.results()
    b0.close()
    rng = np.random.default_rng(7)
    moved = []
    for inst in base:
        inst.c = inst.c * (1.0 + 0.01 * rng.standard_normal(inst.n))
        moved.append(inst)
    b = batch.Batch(moved)
    b.solve(stoptol=1e-6)
    cold = b.results()
    b.set_warm_start(prev.x, prev.y, prev.w)
    b.solve(stoptol=1e-6)
    warm = b.results()
    b.close()
    assert np.all(cold.status == 6) and np.all(warm.status == 6)
    for k in range(len(moved)):
        assert abs(warm.objective[k] - cold.objective[k]) <= 1e-5 * max(1.0, abs(cold.objective[k])), k
    assert warm.iter.sum() < cold.iter.sum(), (warm.iter, cold.iter)
    # with the previous solve's sigma as well
    b = batch.Batch(moved)
    b.set_warm_start(prev.x, prev.y, prev.w, prev.sigma)
    b.solve(stoptol=1e-6)
    warm_s = b.results()
    b.close()
    assert np.all(warm_s.status == 6)
    for k in range(len(moved)):
        assert abs(warm_s.objective[k] - cold.objective[k]) <= 1e-5 * max(1.0, abs(cold.objective[k])), k
    assert np.all(warm_s.sigma > 0)


def test_sigma_start_is_used(engine_lib):
    """sigma0 <= 0 keeps the data-based sigma0 (the cold solve exactly); a
    positive sigma0 changes the run."""
    from hprqp import batch

    insts = [instances.config3_instance(k) for k in range(80, 84)]
    b = batch.Batch(insts)
    b.solve(stoptol=1e-6)
    cold = b.results()
    b.set_warm_start(np.zeros(b.n), np.zeros(b.m), None, np.zeros(b.K))
    b.solve(stoptol=1e-6)
    _same(cold, b.results())
    b.set_warm_start(np.zeros(b.n), None, None, cold.sigma * 10.0)
    b.solve(stoptol=1e-6)
    other = b.results()
    b.close()
    assert np.all(other.status == 6)
    assert not np.array_equal(other.iter, cold.iter)


def test_warm_start_rejects_bad_input(engine_lib):
    from hprqp import batch

    b = batch.Batch([instances.config3_instance(70)])
    bad = np.zeros(b.n)
    bad[0] = np.nan
    with pytest.raises(Exception):
        b.set_warm_start(bad)
    with pytest.raises(ValueError):
        b.set_warm_start(np.zeros(b.n + 1))
    with pytest.raises(Exception):
        b.set_warm_start(np.zeros(b.n), None, None, np.array([np.inf]))
    b.close()


def test_qp_layer_warm_start(engine_lib):
    """QPLayer(warm_start=True): the second forward starts at the first's
    solution; solutions and gradients agree with a cold layer."""
    import torch

    from hprqp import QPLayer, batch

    insts = [instances.config4_instance(k) for k in range(4)]
    p = batch.pack(insts)
    t = lambda a: torch.tensor(a, dtype=torch.float64, requires_grad=True)  # noqa: E731
    warm_layer = QPLayer(p, warm_start=True, stoptol=1e-8)
    cold_layer = QPLayer(p, stoptol=1e-8)
    c0 = p.c.copy()
    warm_layer(*(t(a) for a in (p.q_data, p.a_data, c0, p.AL, p.AU, p.l, p.u)))
    c1 = c0 * 1.01
    outs = []
    for layer in (warm_layer, cold_layer):
        args = [t(a) for a in (p.q_data, p.a_data, c1, p.AL, p.AU, p.l, p.u)]
        x, y = layer(*args)
        x.sum().backward()
        outs.append((x.detach().numpy(), args[2].grad.numpy()))
    (xw, gw), (xc, gc) = outs
    assert np.max(np.abs(xw - xc)) <= 1e-5 * max(1.0, np.max(np.abs(xc)))
    assert np.max(np.abs(gw - gc)) <= 1e-4 * max(1.0, np.max(np.abs(gc)))


@pytest.mark.parametrize("cap", [1, 10, 100])
@pytest.mark.parametrize("with_sigma", [False, True])
def test_warm_iterates_after_k_steps_match_oracle(engine_lib, cap, with_sigma):
    """The batch's warm start against the oracle's restatement of the same
    rules (oracle_solve_from): status, iteration count and iterates after K
    steps within 1e-8, from a seeded random point (and sigma0 = 2)."""
    from hprqp import batch

    insts = _mixed_batch()
    rng = np.random.default_rng(17)
    n_tot, m_tot = sum(i.n for i in insts), sum(i.m for i in insts)
    x0, y0, w0 = rng.standard_normal(n_tot), rng.standard_normal(m_tot), rng.standard_normal(n_tot)
    sig = np.full(len(insts), 2.0) if with_sigma else None
    b = batch.Batch(insts)
    b.set_warm_start(x0, y0, w0, sig)
    b.solve(stoptol=1e-8, max_iter=cap)
    r = b.results()
    b.close()
    vo, ro = np.cumsum([0] + [i.n for i in insts]), np.cumsum([0] + [i.m for i in insts])
    for k, inst in enumerate(insts):
        xs, ws = slice(vo[k], vo[k + 1]), slice(vo[k], vo[k + 1])
        kept = _kept(inst)
        yk = y0[ro[k]:ro[k + 1]][kept]
        o = pyoracle.OracleModel(inst).solve(stoptol=1e-8, max_iter=cap, mode=pyoracle.MODE_GPU_REF,
                                             x0=x0[xs], y0=yk, w0=w0[ws], sigma0=2.0 if with_sigma else 0.0)
        assert r.status[k] == o["status"] and r.iter[k] == o["iter"], (k, r.status[k], o["status"], r.iter[k])
        got_y = r.y[ro[k]:ro[k + 1]][kept]
        for got, ref in ((r.x[xs], o["x"]), (got_y, o["y"]), (r.z[xs], o["z"]), (r.w[ws], o["w"])):
            assert np.max(np.abs(got - ref)) <= 1e-8 * max(1.0, float(np.max(np.abs(ref)))), k
