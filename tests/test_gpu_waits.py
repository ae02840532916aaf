"""Bounded device-side waits: a dependency that is never satisfied ends in
LNB_ETIMEOUT with the site recorded, not in a hang, and the context stays
usable afterwards.  The failure is made on the host side of the kernel's
contract (the solve's ticket starts past the diagonal chain, so the update
items wait on solution blocks nobody publishes); nothing faults or traps.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def test_wait_runs_out_and_reports(lnb):
    L = lnb.lib()
    L.lnb_selftest_wait_timeout.argtypes = [C.c_longlong]
    rc = L.lnb_selftest_wait_timeout(20000)          # 20 ms limit
    assert rc == -5, (rc, lnb.last_error())
    assert "site" in lnb.last_error()


def test_context_usable_after_timeout(lnb):
    from oracle import oracle as O
    L = lnb.lib()
    L.lnb_selftest_wait_timeout.argtypes = [C.c_longlong]
    assert L.lnb_selftest_wait_timeout(5000) == -5
    m, nrhs, b = 500, 2, 64
    A0 = O.spd_diag_dominant(m, seed=3)
    B0 = np.random.default_rng(3).standard_normal((m, nrhs))
    A, B = A0.copy(order="F"), B0.copy(order="F")
    assert lnb.dspdsolv_main(m, nrhs, b, A, B) == 0
    assert O.backward_error(A0, B, B0) <= 10 * m * np.finfo(float).eps
