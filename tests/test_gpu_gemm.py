"""task_dgemm / task_dsyrk on the DMMA GEMM against numpy FP64: all four
transpose cases of gemm_test (task_gemm.c:55-58 calls cblas_dgemm with the
reference's transa/transb), ragged m, n, k around the 64 x 64 x 16 tiling,
padded and odd leading dimensions (the 8-byte copy path), beta = 0 with NaN
in C (C is not read), and both triangles of SYRK with the other triangle
left untouched."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def padded(rng, rows, cols, ld):
    M = np.full((ld, cols), np.nan, order="F")
    M[:rows] = rng.standard_normal((rows, cols))
    return M


@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("tb", ["N", "T"])
@pytest.mark.parametrize("m,n,k,pad", [(64, 64, 16, 0), (1, 1, 1, 0), (70, 33, 17, 3), (129, 257, 100, 1),
                                       (200, 64, 513, 2), (37, 300, 5, 0)])
def test_task_dgemm_all_transposes(lnb, ta, tb, m, n, k, pad):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    A = padded(rng, ar, ac, ar + pad)
    B = padded(rng, br, bc, br + pad)
    C = padded(rng, m, n, m + pad)
    C0 = C.copy(order="F")
    alpha, beta = 13.44, -9.877
    lnb.task_dgemm(ta, tb, m, n, k, alpha, A, ar + pad, B, br + pad, beta, C, m + pad)
    opA = A[:ar] if ta == "N" else A[:ar].T
    opB = B[:br] if tb == "N" else B[:br].T
    ref = alpha * opA @ opB + beta * C0[:m]
    np.testing.assert_allclose(C[:m], ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert np.isnan(C[m:]).all()                         # padding rows untouched


def test_task_dgemm_beta_zero_ignores_c(lnb):
    rng = np.random.default_rng(1)
    m, n, k = 90, 75, 40
    A = np.asfortranarray(rng.standard_normal((m, k)))
    B = np.asfortranarray(rng.standard_normal((k, n)))
    C = np.full((m, n), np.nan, order="F")
    lnb.task_dgemm("N", "N", m, n, k, 2.0, A, m, B, k, 0.0, C, m)
    np.testing.assert_allclose(C, 2.0 * A @ B, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k", [(70, 33), (130, 257), (1, 5)])
def test_task_dsyrk_both_triangles(lnb, uplo, trans, n, k):
    rng = np.random.default_rng(n + k)
    A = np.asfortranarray(rng.standard_normal((n, k) if trans == "N" else (k, n)))
    C0 = np.asfortranarray(rng.standard_normal((n, n)))
    C = C0.copy(order="F")
    lnb.task_dsyrk(uplo, trans, n, k, 1.5, A, A.shape[0], -0.5, C, n)
    P = A @ A.T if trans == "N" else A.T @ A
    ref = 1.5 * P - 0.5 * C0
    tri = np.tril if uplo == "L" else np.triu
    other = (lambda X: np.triu(X, 1)) if uplo == "L" else (lambda X: np.tril(X, -1))
    np.testing.assert_allclose(tri(C), tri(ref), rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    np.testing.assert_array_equal(other(C), other(C0))


def test_device_gemm_and_syrk(lnb, cuda):
    import torch
    g = torch.Generator(device="cuda").manual_seed(3)
    m, n, k = 300, 200, 129
    At = torch.randn(m, k, dtype=torch.float64, device=cuda, generator=g)   # (cols, ld): op(A) = A^T is m x k
    Bt = torch.randn(n, k, dtype=torch.float64, device=cuda, generator=g)   # B stored k x n, ld k
    Ct = torch.randn(n, m, dtype=torch.float64, device=cuda, generator=g)
    C0 = Ct.clone()
    lnb.dgemm_dev("T", "N", m, n, k, 2.0, At, Bt, 0.5, Ct)
    A = At.T.cpu().numpy()      # k x m stored
    B = Bt.T.cpu().numpy()      # k x n stored
    ref = 2.0 * A.T @ B + 0.5 * C0.T.cpu().numpy()
    np.testing.assert_allclose(Ct.T.cpu().numpy(), ref, rtol=1e-12, atol=1e-11)
    St = torch.randn(m, m, dtype=torch.float64, device=cuda, generator=g)
    S0 = St.clone()
    lnb.dsyrk_dev("L", "T", m, k, -1.0, At, 1.0, St)
    refS = S0.T.cpu().numpy() - A.T @ A
    got = St.T.cpu().numpy()
    np.testing.assert_allclose(np.tril(got), np.tril(refS), rtol=1e-12, atol=1e-11)
    np.testing.assert_array_equal(np.triu(got, 1), np.triu(S0.T.cpu().numpy(), 1))


@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m,nrhs,alpha", [(300, 200, 13.44), (1000, 256, -0.5), (64, 192, 1.0), (65, 193, 2.0),
                                          (130, 40, 3.0)])
def test_dtrsm_many_rhs_gemm_path(lnb, cuda, uplo, trans, diag, m, nrhs, alpha):
    """192 or more right-hand sides take the blocked DMMA GEMM solve (40: the DAG walk)"""
    import torch
    rng = np.random.default_rng(m + nrhs)
    T = rng.standard_normal((m, m)) / np.sqrt(m) + 4 * np.eye(m)
    T = np.tril(T) if uplo == "L" else np.triu(T)
    Tnan = T.copy()
    Tnan[np.triu_indices(m, 1) if uplo == "L" else np.tril_indices(m, -1)] = np.nan   # the other triangle is not read
    if diag == "U":
        np.fill_diagonal(T, 1.0)
        np.fill_diagonal(Tnan, np.nan)
    B0 = rng.standard_normal((m, nrhs))
    Tt = torch.tensor(np.ascontiguousarray(Tnan.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    lnb.dtrsm_dev(uplo, trans, diag, m, nrhs, alpha, Tt, Bt)
    X = Bt.cpu().numpy().T
    op = T if trans == "N" else T.T
    berr = np.abs(op @ X - alpha * B0).max() / (np.abs(op).sum(1).max() * np.abs(X).max() + abs(alpha) * np.abs(B0).max())
    assert berr < 10 * m * np.finfo(float).eps / 2, berr


@pytest.mark.parametrize("nrhs", [3, 64, 200])
def test_dtrsm_alpha_zero(lnb, cuda, nrhs):
    """alpha = 0 sets B to zero without reading T (BLAS), on every schedule"""
    import torch
    m = 200
    Tt = torch.full((m, m), float("nan"), dtype=torch.float64, device=cuda)
    Bt = torch.randn(nrhs, m, dtype=torch.float64, device=cuda)
    lnb.dtrsm_dev("L", "N", "N", m, nrhs, 0.0, Tt, Bt)
    assert int((Bt != 0).sum().item()) == 0
