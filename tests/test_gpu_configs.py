"""The reference configurations' paths on the GPU, through the C ABI.

Configuration 1 (plain FP64 dspdsolv_main, n = 2048, b = 256, one right-hand
side, A = (R + R^T)/2 + n I with R ~ U[0,1), x_true ~ U[-1,1), seed 0) runs at
its full size against the reference itself: the reference compiled from its
own sources (oracle/_ref/libref.so) solves the same arrays on the CPU.

Configurations 2-4 are large (n = 16384 .. 49152); their full-size runs are
measured by bench.py, which checks the factor residual and the backward error
on the device.  Here each one's path runs with the configuration's own tile
size, right-hand-side count and input distribution at an n the CPU checker
(numpy LAPACK) handles in seconds:
  2: FP64 factor + solves, b = 512, 1 and 64 right-hand sides, G G^T/n + 1e-2 I
  3: TF32x3 factor + FP64 refinement, b = 512 (the delta sweep is in
     test_gpu_mixed.py)
  4: per-tile-scaled BF16 factor, b = 1024, 8 right-hand sides,
     D (G G^T/n + delta I) D, D = diag(10^u), u ~ U[-2,2], delta 1e-2 / 1e-4

Bars: factor ||A - L L^T||_inf / (n eps ||A||_inf) <= 10 (potrf_test.c:31-36);
normwise backward error <= 10 n eps; entrywise agreement with the reference's
output to the rounding of blocked FP64 sums.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def config1_inputs():
    n = 2048
    A0 = O.spd_diag_dominant(n, seed=0)
    x_true = np.random.default_rng(0).uniform(-1, 1, (n, 1))
    return A0, np.asfortranarray(x_true), np.asfortranarray(A0 @ x_true)


def test_config1_spdsolv_against_reference_build(lnb):
    if not O.ref_available():
        pytest.skip("the reference build oracle/_ref/libref.so is not present")
    n, b = 2048, 256
    A0, x_true, B0 = config1_inputs()
    A1, B1 = A0.copy(order="F"), B0.copy(order="F")
    A2, B2 = A0.copy(order="F"), B0.copy(order="F")
    assert lnb.dspdsolv_main(n, 1, b, A1, B1) == 0
    assert O.ref_spdsolv(A2, B2, b) == 0
    # the same factor as the reference's (A is strongly diagonally dominant,
    # cond ~ 2, so two backward-stable factors agree to a few n eps)
    np.testing.assert_allclose(np.tril(A1), np.tril(A2), rtol=0, atol=2 * n * EPS * np.abs(A2).max())
    np.testing.assert_allclose(B1, B2, rtol=1e-12, atol=1e-13)
    for L in (A1, A2):
        assert O.chol_residual_np(A0, L) <= 10.0
    eps2 = EPS / 2
    assert O.backward_error_np(A0, B1, B0) <= 10 * n * eps2
    assert O.backward_error_np(A0, B2, B0) <= 10 * n * eps2
    # the GPU leaves the upper triangle as it was
    np.testing.assert_array_equal(np.triu(A1, 1), np.triu(A0, 1))
    assert np.abs(B1 - x_true).max() <= 1e-12


@pytest.mark.parametrize("nrhs", [1, 64])
def test_config2_family_fp64(lnb, cuda, nrhs):
    import torch
    n, b = 3072, 512
    A0 = O.spd_covariance(n, 1e-2, seed=21)
    B0 = np.asfortranarray(np.random.default_rng(21).standard_normal((n, nrhs)))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    info = torch.full((1,), -1, dtype=torch.int32, device=cuda)
    lnb.dposv_dev(At, Bt, n, nrhs, b, info=info)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    L = At.cpu().numpy().T
    X = Bt.cpu().numpy().T
    assert O.chol_residual_np(A0, L) <= 10.0
    assert O.backward_error_np(A0, X, B0) <= 10 * n * EPS / 2
    Xref = np.linalg.solve(A0, B0)
    bound = 2 * np.linalg.cond(A0, np.inf) * 10 * n * EPS
    assert np.abs(X - Xref).max() / np.abs(Xref).max() <= bound


@pytest.mark.parametrize("n", [4096, 5000])
@pytest.mark.parametrize("delta", [1e-2, 1e-4])
def test_config4_family_bf16_b1024(lnb, n, delta):
    """b = 1024 tiles: nested diagonal factor, 1024-wide panel solve and BF16
    operand copies of K = 1024; 5000 leaves a ragged last tile of 904."""
    b, nrhs = 1024, 8
    rng = np.random.default_rng(40 + n)
    D = 10.0 ** rng.uniform(-2, 2, n)
    A0 = O.fortran(D[:, None] * O.spd_covariance(n, delta, seed=n) * D[None, :])
    B0 = np.asfortranarray(rng.standard_normal((n, nrhs)))
    opts = lnb.ir_opts(factor=lnb.FACTOR_BF16, max_iter=40, pcg_max_iter=400)
    rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    assert rc == 0, (rc, res, lnb.last_error())
    be = O.backward_error_np(A0, X, B0)
    assert be <= 10 * n * EPS / 2, (be, res)
    assert res["backward_error"] <= 10 * n * EPS / 2


def test_config3_family_tf32x3_forward_error(lnb):
    n, b = 4096, 512
    A0 = O.spd_covariance(n, 1e-3, seed=31)
    B0 = np.asfortranarray(np.random.default_rng(31).standard_normal((n, 1)))
    opts = lnb.ir_opts(factor=lnb.FACTOR_TF32X3)
    rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    assert rc == 0, (rc, res)
    Xref = np.linalg.solve(A0, B0)
    bound = 2 * np.linalg.cond(A0, np.inf) * 10 * n * EPS / 2
    assert np.abs(X - Xref).max() / np.abs(Xref).max() <= bound
    assert res["iterations"] <= 6 and not res["used_pcg"]
