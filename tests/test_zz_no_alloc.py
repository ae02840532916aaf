"""The allocation-free FP64 factorization entry point, lnb_dchol_noalloc_dev.

It exists for callers that cannot call cudaMalloc: code whose device memory
belongs to another manager (a caching allocator or a fixed arena holding all
of HBM) and code on a latency-critical path where cudaMalloc's implicit
synchronization is not acceptable.  Its scratch is a fixed device array inside
the library, shared by every call.

The test calls it through the C ABI (ctypes) twice in a row on different
matrices and checks each result against the regular entry point
lnb_dchol_dev on the same input: the factors must agree to FP64 rounding of
the blocked sums, and both must meet the reference's factor bound.  The
second call would expose stale scratch contents (the status word and the
block inverses are reused).  This file sorts last so that a run that stops at
the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib(cuda):
    import linompss_b200
    L = linompss_b200.lib()
    for name in ("lnb_dchol_noalloc_dev", "lnb_dchol_dev"):
        getattr(L, name).argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        getattr(L, name).restype = C.c_int
    return L


def factor(lib, fn, A0, b, dev, free_bytes=None):
    """Factor A0 through entry point `fn`; if free_bytes is a list, append the
    device's free memory just before and just after the call."""
    import torch
    n = A0.shape[0]
    At = torch.tensor(np.ascontiguousarray(A0.T), device=dev)   # column-major view
    info = torch.full((1,), -99, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    rc = getattr(lib, fn)(n, b, At.data_ptr(), At.stride(0), info.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    assert rc == 0, rc
    return At.cpu().numpy().T, int(info.item())


@pytest.mark.parametrize("cases", [[(1000, 256, 1), (700, 100, 2)], [(512, 512, 3), (1537, 1024, 4)]])
def test_noalloc_matches_regular_entry_point_twice(lib, cuda, cases):
    eps = np.finfo(float).eps
    for call, (n, b, seed) in enumerate(cases):     # two calls in a row on different inputs
        A0 = O.spd_covariance(n, 1e-2, seed=seed)
        L_ref, info_ref = factor(lib, "lnb_dchol_dev", A0, b, cuda)
        free = []
        L_na, info_na = factor(lib, "lnb_dchol_noalloc_dev", A0, b, cuda, free)
        if call > 0:
            # the property the entry point exists for: a warm call takes no device memory
            assert free[0] == free[1], f"free device memory changed by {free[0] - free[1]} bytes"
        assert info_ref == 0 and info_na == 0
        np.testing.assert_allclose(np.tril(L_na), np.tril(L_ref), rtol=0, atol=64 * n * eps * np.abs(L_ref).max())
        np.testing.assert_array_equal(np.triu(L_na, 1), np.triu(A0, 1))
        assert O.chol_residual_np(A0, L_na) <= 10.0


def test_noalloc_reports_info_and_limits(lib, cuda):
    A0 = O.spd_diag_dominant(300, seed=9)
    A0[200, 200] = -1.0
    _, info = factor(lib, "lnb_dchol_noalloc_dev", A0, 64, cuda)
    assert info == 201
    # the next call starts from a clean status word
    _, info = factor(lib, "lnb_dchol_noalloc_dev", O.spd_diag_dominant(300, seed=10), 64, cuda)
    assert info == 0
    # tile sizes beyond the fixed scratch are rejected before any work
    import linompss_b200
    rc = lib.lnb_dchol_noalloc_dev(2048, 2048, 0, 2048, 0, 0)
    assert rc == linompss_b200.LNB_ETOOBIG
