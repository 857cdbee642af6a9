"""The no-allocation power iteration (hprqp_b200_power_lambda_noalloc).

It exists for callers that cannot allocate device memory: their GPU memory
belongs to another allocator or arena, or their host forbids device
allocation once running.  The entry point keeps its work vectors in a fixed
8 MiB array inside the library, so it must give the same lambda_max(A A')
as the allocating setup path, call after call, even though every call reuses
(and leaves dirty) the same array -- on the legacy default stream and on a
stream the caller owns, at the largest size the array admits, and without
changing the device's free memory.  This file is collected last on purpose.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from hprqp import instances

pytestmark = pytest.mark.gpu


def _entry(hprqp):
    lib = ctypes.CDLL(hprqp.library_path())
    fn = lib.hprqp_b200_power_lambda_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t] + [ctypes.c_void_p] * 7 + \
        [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    fn.restype = ctypes.c_int
    return fn


def _device_csr(torch, indptr, indices, data):
    return (torch.tensor(np.asarray(indptr, np.int32), device="cuda"),
            torch.tensor(np.asarray(indices, np.int32), device="cuda"),
            torch.tensor(np.asarray(data, np.float64), device="cuda"))


def _model_csr(hprqp, model):
    import scipy.sparse as sp

    arr = hprqp.model_arrays(model)
    m, n = arr["m"], arr["n"]
    A = sp.csr_matrix((arr["a_data"], arr["a_indices"], arr["a_indptr"]), shape=(m, n))
    AT = A.T.tocsr()
    AT.sort_indices()
    return m, n, A, AT


def _calls(hprqp, torch, model, stream=None, count=2, between=None):
    """`count` calls on the model's unscaled A (device copies made once);
    returns the lambdas.  between(i) runs before call i."""
    m, n, A, AT = _model_csr(hprqp, model)
    a = _device_csr(torch, A.indptr, A.indices, A.data)
    at = _device_csr(torch, AT.indptr, AT.indices, AT.data)
    torch.cuda.synchronize()
    fn = _entry(hprqp)
    handle = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    got = []
    for i in range(count):  # later calls run on the scratch the previous one left behind
        if between is not None:
            between(i)
        lam = ctypes.c_double(0.0)
        its = ctypes.c_int(0)
        st = fn(0, m, n, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), at[0].data_ptr(), at[1].data_ptr(),
                at[2].data_ptr(), handle, ctypes.byref(lam), ctypes.byref(its))
        assert st == hprqp.STATUS_OK
        assert its.value > 0
        got.append(lam.value)
    return got


def _setup_lambda(hprqp, model):
    # the allocating setup path on the same (unscaled) A
    return hprqp.setup_info(model, hprqp.Parameters(verbose=False, use_scaling=False))["lambda_max_A"]


@pytest.mark.parametrize("case", ["config0", "config3_9"])
def test_noalloc_lambda_matches_setup_two_calls(engine_lib, case):
    torch = pytest.importorskip("torch")
    hprqp = engine_lib
    inst = instances.config0() if case == "config0" else instances.config3_instance(9)
    model = hprqp.build_from_instance(inst)
    ref = _setup_lambda(hprqp, model)
    got = _calls(hprqp, torch, model)
    # eigenvalue tolerance of the reference's GPU eigs test (tests/gpu/test_gpu_eigs.c:37-38)
    for g in got:
        assert abs(g - ref) <= 1e-6 * abs(ref), (g, ref)
    assert got[0] == got[1]


def test_noalloc_on_caller_stream(engine_lib):
    """A stream the caller created (here torch's) instead of the legacy default stream."""
    torch = pytest.importorskip("torch")
    hprqp = engine_lib
    model = hprqp.build_from_instance(instances.config3_instance(3))
    ref = _setup_lambda(hprqp, model)
    stream = torch.cuda.Stream()
    got = _calls(hprqp, torch, model, stream=stream)
    for g in got:
        assert abs(g - ref) <= 1e-6 * abs(ref), (g, ref)
    assert got[0] == got[1]


def test_noalloc_largest_admitted_size(engine_lib):
    """2 m + n exactly at the limit of the fixed array (1,046,526 doubles)."""
    torch = pytest.importorskip("torch")
    import scipy.sparse as sp

    hprqp = engine_lib
    m, n = 262_144, 522_238
    assert 2 * m + n == 1_046_526
    rng = np.random.default_rng(2024)
    per_row = 3
    rows = np.repeat(np.arange(m), per_row)
    cols = rng.integers(0, n, size=m * per_row)
    A = sp.csr_matrix((rng.standard_normal(m * per_row), (rows, cols)), shape=(m, n))
    A.sum_duplicates()
    A.sort_indices()
    Q = sp.identity(n, format="csr")
    ones_n, ones_m = np.ones(n), np.ones(m)
    model = hprqp.build_from_qabc(Q, np.zeros(n), A, -ones_m, ones_m, -ones_n, ones_n)
    assert _model_csr(hprqp, model)[:2] == (m, n)
    ref = _setup_lambda(hprqp, model)
    got = _calls(hprqp, torch, model)
    for g in got:
        assert abs(g - ref) <= 1e-6 * abs(ref), (g, ref)
    assert got[0] == got[1]


def test_noalloc_allocates_no_device_memory(engine_lib):
    """The device's free memory does not change across calls (measured once
    the first call has loaded the library's device code, which reserves the
    array); the device copies of A and A' are made before the first call."""
    torch = pytest.importorskip("torch")
    hprqp = engine_lib
    model = hprqp.build_from_instance(instances.config0())
    free = []

    def record(i):
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])

    got = _calls(hprqp, torch, model, count=3, between=record)
    record(3)
    # free[1] is taken after the first call has loaded the device code
    assert free[1] == free[2] == free[3], free
    assert got[0] == got[1] == got[2]


def test_noalloc_empty_rows_and_bad_device(engine_lib):
    torch = pytest.importorskip("torch")
    hprqp = engine_lib
    fn = _entry(hprqp)
    lam = ctypes.c_double(-1.0)
    its = ctypes.c_int(-1)
    # m == 0: lambda 0 after no iteration, nothing read
    st = fn(0, 0, 5, None, None, None, None, None, None, None, ctypes.byref(lam), ctypes.byref(its))
    assert st == hprqp.STATUS_OK and lam.value == 0.0 and its.value == 0
    # a device index that does not exist is an argument error, not a CUDA failure
    dummy_i = torch.zeros(4, dtype=torch.int32, device="cuda")
    dummy_d = torch.zeros(4, dtype=torch.float64, device="cuda")
    before = torch.cuda.current_device()
    st = fn(torch.cuda.device_count(), 1, 1, dummy_i.data_ptr(), dummy_i.data_ptr(), dummy_d.data_ptr(),
            dummy_i.data_ptr(), dummy_i.data_ptr(), dummy_d.data_ptr(), None, ctypes.byref(lam), None)
    assert st == hprqp.STATUS_INVALID_ARGUMENT
    assert torch.cuda.current_device() == before


def test_noalloc_rejects_oversized_problem(engine_lib):
    torch = pytest.importorskip("torch")
    hprqp = engine_lib
    fn = _entry(hprqp)
    dummy_i = torch.zeros(4, dtype=torch.int32, device="cuda")
    dummy_d = torch.zeros(4, dtype=torch.float64, device="cuda")
    lam = ctypes.c_double(0.0)
    m = 600_000  # 2 m + n > 1,046,526
    st = fn(0, m, 1, dummy_i.data_ptr(), dummy_i.data_ptr(), dummy_d.data_ptr(), dummy_i.data_ptr(),
            dummy_i.data_ptr(), dummy_d.data_ptr(), None, ctypes.byref(lam), None)
    assert st == hprqp.STATUS_INVALID_ARGUMENT
