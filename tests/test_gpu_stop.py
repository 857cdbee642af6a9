"""Early stops of the batch and of the plain solve, made on the host: the
time limit (reference src/shared/solver_backend.c:192-208, 432-513: an
iterate past time_limit ends with TIME_LIMIT) and the batch's abort request
(hprqp_batch_request_abort, set from another host thread while the kernel
runs).  Nothing here faults or hangs the GPU: every solve that is meant to be
stopped also carries a time limit of a few seconds as its own bound."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

import hprqp
from hprqp import instances

pytestmark = pytest.mark.gpu

TIME_LIMIT, OPTIMAL = 5, 6


def test_plain_time_limit_zero(engine_lib, plain_path):
    model = hprqp.build_from_instance(instances.config0())
    r = hprqp.optimize(model, hprqp.Parameters(verbose=False, stoptol=1e-6, time_limit=0.0), as_numpy=True)
    assert r.status_code == TIME_LIMIT
    assert r.iter == 0
    assert np.isfinite(r.residual) and r.residual > 1e-6


def test_batch_time_limit_small_batch(engine_lib):
    """64 QPs, 1 ms: every instance has a CTA at once, is set up, and stops at
    the first status check past the limit with its residuals computed."""
    from hprqp import batch

    b = batch.Batch(instances.config3(64, 300))
    b.solve(stoptol=1e-6, time_limit=1e-3)
    r = b.results(vectors=False)
    b.close()
    assert set(np.unique(r.status)) <= {TIME_LIMIT, OPTIMAL}
    assert np.sum(r.status == TIME_LIMIT) > 0
    done = r.status == OPTIMAL
    assert np.all(r.residual[done] < 1e-6)
    assert np.all(np.isfinite(r.residual[~done]))


def test_batch_time_limit_skips_instances_not_started(engine_lib):
    """More instances than CTAs: those taken from the queue after the limit
    are not set up and report TIME_LIMIT at iteration 0, residual inf."""
    from hprqp import batch

    K = 1024
    b = batch.Batch(instances.config3(K, 400))
    b.solve(stoptol=1e-6, time_limit=1e-3)
    r = b.results()
    b.close()
    assert set(np.unique(r.status)) <= {TIME_LIMIT, OPTIMAL}
    skipped = (r.status == TIME_LIMIT) & (r.iter == 0) & np.isinf(r.residual)
    assert np.sum(skipped) > 0
    xs = b.split(r.x, "x")
    for k in np.nonzero(skipped)[0][:20]:
        assert np.all(xs[k] == 0.0)


def test_batch_abort_from_host_thread(engine_lib):
    """A solve that cannot converge (stoptol below what FP64 reaches, an
    unbounded iteration budget, a 30 s time limit as the backstop) is stopped
    from another thread after 0.5 s: it returns promptly, every unfinished
    instance reports TIME_LIMIT, and the next solve of the batch runs in full."""
    from hprqp import batch

    b = batch.Batch(instances.config3(1024, 500))
    out = {}

    def run():
        t0 = time.perf_counter()
        b.solve(stoptol=1e-30, max_iter=10**9, time_limit=30.0)
        out["seconds"] = time.perf_counter() - t0

    th = threading.Thread(target=run)
    th.start()
    time.sleep(0.5)
    b.request_abort()
    th.join(timeout=60)
    assert not th.is_alive()
    assert out["seconds"] < 10.0, out  # far below the 30 s time limit
    r = b.results(vectors=False)
    assert np.all(r.status == TIME_LIMIT)
    assert np.sum(r.iter > 0) > 0  # the instances running at the request were stopped mid-solve
    # the request ended with that solve
    b.solve(stoptol=1e-6, max_iter=10**6, time_limit=60.0)
    r2 = b.results(vectors=False)
    b.close()
    assert np.all(r2.status == OPTIMAL)
