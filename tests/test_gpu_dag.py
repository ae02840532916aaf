"""The FP64 factorization's device-side DAG schedule (LNB_SCHED_DAG): one
persistent launch that walks the tile task DAG, against the reference's
golden outputs, the oracle and LAPACK (numpy), through the C ABI.

Covers ragged sizes (n not a multiple of the 64-wide tiles, n < 64, n = 1),
leading dimensions larger than n, the solves reusing the DAG's diagonal-block
inverses, non-SPD inputs (LAPACK info and the valid leading columns), the
device-pointer forms, agreement with the stream schedule, and the bounded
waits (a dependency that nothing satisfies ends in LNB_ETIMEOUT, and the
context stays usable).  Bars as in test_gpu_f64.py.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    linompss_b200.set_chol_schedule(linompss_b200.SCHED_DAG)
    yield linompss_b200
    linompss_b200.set_chol_schedule(linompss_b200.SCHED_AUTO)


@pytest.mark.parametrize("name", ["chol_rl_n100_b32", "chol_rl_n128_b32", "chol_rl_n199_b53",
                                  "chol_ll_n100_b32", "chol_ll_n128_b64"])
def test_dag_chol_golden(lnb, golden_dir, name):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    A = d["A"].copy(order="F")
    n, b = A.shape[0], int(d["b"])
    assert lnb.ompss_dchol_rl(n, b, b, A, n) == 0
    np.testing.assert_allclose(np.tril(A), np.tril(d["out"]), rtol=0, atol=64 * EPS * np.abs(d["out"]).max())
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(d["A"], 1))
    assert O.chol_residual_np(d["A"], A) <= 10.0


@pytest.mark.parametrize("n", [1, 2, 7, 63, 64, 65, 127, 128, 300, 1000, 2048, 2500])
def test_dag_chol_sizes(lnb, n):
    A0 = O.spd_covariance(n, 1e-2, seed=n) if n > 8 else O.spd_diag_dominant(n, seed=n)
    A = A0.copy(order="F")
    assert lnb.ompss_dchol_rl(n, 256, 256, A, n) == 0
    L = np.linalg.cholesky(A0)
    np.testing.assert_allclose(np.tril(A), L, rtol=0, atol=64 * n * EPS * np.abs(L).max())
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(A0, 1))
    assert O.chol_residual_np(A0, A) <= 10.0


def test_dag_lda_larger_than_n(lnb):
    n, lda = 333, 401
    A0 = O.spd_diag_dominant(n, seed=5)
    big = np.asfortranarray(np.full((lda, n), 7.25))
    big[:n, :] = A0
    assert lnb.ompss_dchol_rl(n, 64, 64, big, lda) == 0
    np.testing.assert_allclose(np.tril(big[:n]), np.linalg.cholesky(A0), rtol=0, atol=1e-12 * n)
    np.testing.assert_array_equal(big[n:], 7.25)


@pytest.mark.parametrize("name", ["spdsolv_m128_r1_b32", "spdsolv_m128_r3_b32", "spdsolv_m96_r8_b48"])
def test_dag_spdsolv_golden(lnb, golden_dir, name):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    A = d["A"].copy(order="F")
    B = d["B"].copy(order="F")
    m, nrhs = B.shape
    b = int(name.split("_b")[-1])
    assert lnb.dspdsolv_main(m, nrhs, b, A, B) == 0
    np.testing.assert_allclose(B, d["X"], rtol=1e-12, atol=1e-13)
    assert O.backward_error(d["A"], B, d["B"]) <= 10 * m * EPS


@pytest.mark.parametrize("m,nrhs", [(2048, 1), (2048, 64), (777, 5), (70, 9)])
def test_dag_spdsolv_sizes(lnb, m, nrhs):
    rng = np.random.default_rng(m + nrhs)
    A0 = O.spd_diag_dominant(m, seed=m)
    X0 = rng.uniform(-1, 1, (m, nrhs))
    B0 = np.asfortranarray(A0 @ X0)
    A, B = A0.copy(order="F"), B0.copy(order="F")
    assert lnb.dspdsolv_main(m, nrhs, 256, A, B) == 0
    assert O.backward_error_np(A0, B, B0) <= 10 * m * EPS / 2
    np.testing.assert_allclose(B, np.linalg.solve(A0, B0), rtol=0, atol=1e-12 * max(1, np.abs(X0).max()))


@pytest.mark.parametrize("pos", [0, 5, 40, 63, 64, 130, 299])
def test_dag_not_spd_reports_info(lnb, pos):
    n = 300
    A0 = O.spd_diag_dominant(n, seed=11)
    A0[pos, pos] = -1.0
    A1, A2 = A0.copy(order="F"), A0.copy(order="F")
    info = lnb.ompss_dchol_rl(n, 64, 64, A1, n)
    assert info == O.chol_rl(A2, 64) == pos + 1
    if pos > 0:
        np.testing.assert_allclose(np.tril(A1)[:, :pos], np.tril(A2)[:, :pos], rtol=0, atol=1e-11)


def test_dag_matches_stream_schedule(lnb):
    """config 1's inputs (n = 2048, b = 256, seed 0) through both schedules"""
    n, b = 2048, 256
    A0 = O.spd_diag_dominant(n, seed=0)
    Ad, As = A0.copy(order="F"), A0.copy(order="F")
    assert lnb.ompss_dchol_rl(n, b, b, Ad, n) == 0
    lnb.set_chol_schedule(lnb.SCHED_STREAMS)
    try:
        assert lnb.ompss_dchol_rl(n, b, b, As, n) == 0
    finally:
        lnb.set_chol_schedule(lnb.SCHED_DAG)
    np.testing.assert_allclose(np.tril(Ad), np.tril(As), rtol=0, atol=2 * n * EPS * np.abs(As).max())


def test_dag_device_forms(lnb, cuda):
    import torch
    n, nrhs = 3000, 3
    A0 = O.spd_covariance(n, 1e-2, seed=12)
    B0 = np.asfortranarray(np.random.default_rng(12).standard_normal((n, nrhs)))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    info = torch.full((1,), -1, dtype=torch.int32, device=cuda)
    lnb.dposv_dev(At, Bt, n, nrhs, 512, info=info)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    assert O.chol_residual_np(A0, At.cpu().numpy().T) <= 10.0
    assert O.backward_error_np(A0, Bt.cpu().numpy().T, B0) <= 10 * n * EPS / 2
    At2 = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    lnb.dchol_dev(At2, n, 512, info=info)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    np.testing.assert_allclose(np.tril(At2.cpu().numpy().T), np.linalg.cholesky(A0), rtol=0, atol=1e-10)


def test_dag_wait_runs_out_and_context_stays_usable(lnb):
    L = lnb.lib()
    L.lnb_selftest_chol_wait_timeout.argtypes = [C.c_longlong]
    rc = L.lnb_selftest_chol_wait_timeout(20000)
    assert rc == lnb.LNB_ETIMEOUT, (rc, lnb.last_error())
    assert "site" in lnb.last_error()
    n = 500
    A0 = O.spd_diag_dominant(n, seed=3)
    A = A0.copy(order="F")
    assert lnb.ompss_dchol_rl(n, 64, 64, A, n) == 0
    np.testing.assert_allclose(np.tril(A), np.linalg.cholesky(A0), rtol=0, atol=1e-11)
