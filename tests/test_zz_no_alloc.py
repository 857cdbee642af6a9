"""The no-allocation power iteration (hprqp_b200_power_lambda_noalloc).

It exists for callers that cannot allocate device memory: their GPU memory
belongs to another allocator or arena, or their host forbids device
allocation once running.  The entry point keeps its work vectors in a fixed
8 MiB array inside the library, so it must give the same lambda_max(A A')
as the allocating setup path, call after call, even though every call reuses
(and leaves dirty) the same array.  This file is collected last on purpose.
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


@pytest.mark.parametrize("case", ["config0", "config3_9"])
def test_noalloc_lambda_matches_setup_two_calls(engine_lib, case):
    torch = pytest.importorskip("torch")
    import scipy.sparse as sp

    hprqp = engine_lib
    inst = instances.config0() if case == "config0" else instances.config3_instance(9)
    model = hprqp.build_from_instance(inst)
    params = hprqp.Parameters(verbose=False, use_scaling=False)
    ref = hprqp.setup_info(model, params)["lambda_max_A"]  # allocating path, same (unscaled) A
    arr = hprqp.model_arrays(model)
    m, n = arr["m"], arr["n"]
    A = sp.csr_matrix((arr["a_data"], arr["a_indices"], arr["a_indptr"]), shape=(m, n))
    AT = A.T.tocsr()
    AT.sort_indices()
    a = _device_csr(torch, A.indptr, A.indices, A.data)
    at = _device_csr(torch, AT.indptr, AT.indices, AT.data)
    fn = _entry(hprqp)
    got = []
    for _ in range(2):  # the second call runs on the scratch the first one left behind
        lam = ctypes.c_double(0.0)
        its = ctypes.c_int(0)
        st = fn(0, m, n, a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), at[0].data_ptr(), at[1].data_ptr(),
                at[2].data_ptr(), None, ctypes.byref(lam), ctypes.byref(its))
        assert st == hprqp.STATUS_OK
        assert its.value > 0
        got.append(lam.value)
    # eigenvalue tolerance of the reference's GPU eigs test (tests/gpu/test_gpu_eigs.c:37-38)
    for g in got:
        assert abs(g - ref) <= 1e-6 * abs(ref), (g, ref)
    assert got[0] == got[1]


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
