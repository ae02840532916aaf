"""Tile LU with partial pivoting and the general solve on the GPU, through the
C ABI:
  * against the reference's own outputs (tests/golden/lu_*, gensolv_*: its
    ompss_dgetrf and dgensolv_main on its GENMAT_IP matrix distribution);
  * against LAPACK (scipy) on matrices where pivoting happens: the same pivot
    sequence and factor for every panel width, ragged last panels, tall,
    wide, and tall enough that a panel spans a cluster of several CTAs (each
    panel shape: 32 columns to 4096 rows, 16 to 8192, 8 to 16384, 4 to 32768);
  * exactly singular columns: LAPACK's info, the factorization completed;
  * FP32 twins, the _ll drivers, and the device entry points.
Tolerances: blocked FP64 sums in another order agree to ~1e-12 relative."""
import os

import numpy as np
import pytest
import scipy.linalg as sl
import scipy.linalg.lapack as la

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps / 2


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def global_pivots(ipiv_local, b):
    return np.arange(len(ipiv_local)) // b * b + ipiv_local


@pytest.mark.parametrize("name", ["lu_m200_n200_b33", "lu_m240_n160_b64"])
@pytest.mark.parametrize("ll", [False, True])
def test_getrf_matches_reference(lnb, golden_dir, name, ll):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    A = d["A"].copy(order="F")
    info, ipiv = lnb.ompss_getrf(A, int(d["b"]), ll=ll)
    assert info == 0
    np.testing.assert_array_equal(ipiv, d["ipiv"])
    np.testing.assert_allclose(A, d["LU"], rtol=0, atol=1e-12 * np.abs(d["LU"]).max())


def test_gensolv_matches_reference(lnb, golden_dir):
    d = np.load(os.path.join(golden_dir, "gensolv_m128_b48.npz"))
    A, B = d["A"].copy(order="F"), d["B"].copy(order="F")
    assert lnb.gensolv(A, B, int(d["b"])) == 0
    np.testing.assert_allclose(A, d["LU"], rtol=0, atol=1e-12 * np.abs(d["LU"]).max())
    np.testing.assert_allclose(B, d["X"], rtol=0, atol=1e-12 * np.abs(d["X"]).max())


@pytest.mark.parametrize("m,n,b", [(300, 300, 64), (300, 300, 50), (1000, 1000, 121), (700, 400, 100),
                                   (257, 257, 256), (200, 300, 64), (3000, 600, 256), (7000, 300, 128),
                                   (9000, 40, 16), (1, 1, 1), (33, 1, 8)])
def test_getrf_pivoting_matches_lapack(lnb, m, n, b):
    A0 = np.asfortranarray(np.random.default_rng(m + 3 * n + b).standard_normal((m, n)))
    lu, piv, info_l = la.dgetrf(A0)
    A = A0.copy(order="F")
    info, ipiv = lnb.ompss_getrf(A, b)
    assert info == info_l == 0
    np.testing.assert_array_equal(global_pivots(ipiv, b), piv + 1)
    np.testing.assert_allclose(A, lu, rtol=0, atol=1e-11 * max(1.0, np.abs(lu).max()))
    perm, L, U = O.lu_unpack(A, ipiv, b)
    np.testing.assert_allclose(A0[perm], L @ U, rtol=0, atol=1e-12 * np.abs(A0).max() * max(m, n))


def test_getrf_singular_column_info(lnb):
    A0 = np.asfortranarray(np.random.default_rng(9).standard_normal((150, 150)))
    A0[:, 70] = 0.0
    _, _, info_l = la.dgetrf(A0)
    A = A0.copy(order="F")
    info, ipiv = lnb.ompss_getrf(A, 32)
    assert info == info_l == 71
    assert np.isfinite(A).all()


def test_sgetrf_and_sgensolv(lnb):
    m, b = 260, 64
    A0 = O.genmat_ip(m, m, 21).astype(np.float32, order="F")
    A = A0.copy(order="F")
    info, ipiv = lnb.ompss_getrf(A, b)
    assert info == 0 and (ipiv == np.arange(m) % b + 1).all()
    lu, _, _ = la.sgetrf(A0)
    np.testing.assert_allclose(A, lu, rtol=0, atol=1e-5 * np.abs(lu).max())
    A = A0.copy(order="F")
    B0 = np.asfortranarray(np.random.default_rng(22).random((m, 5)).astype(np.float32))
    B = B0.copy(order="F")
    assert lnb.gensolv(A, B, b) == 0
    X = np.linalg.solve(A0.astype(np.float64), B0.astype(np.float64))
    np.testing.assert_allclose(B, X, rtol=0, atol=1e-5 * np.abs(X).max())


@pytest.mark.parametrize("m,nrhs,b", [(500, 7, 64), (1200, 300, 121)])
def test_gensolv_with_pivoting(lnb, m, nrhs, b):
    rng = np.random.default_rng(m + nrhs)
    A0 = np.asfortranarray(rng.standard_normal((m, m)))
    B0 = np.asfortranarray(rng.standard_normal((m, nrhs)))
    A, B = A0.copy(order="F"), B0.copy(order="F")
    assert lnb.gensolv(A, B, b) == 0
    berr = np.abs(A0 @ B - B0).max() / (np.abs(A0).sum(1).max() * np.abs(B).max() + np.abs(B0).max())
    assert berr < 10 * m * EPS, berr


def test_device_getrf_getrs(lnb, cuda):
    import torch
    n, nrhs = 900, 20
    rng = np.random.default_rng(31)
    A0 = rng.standard_normal((n, n))
    B0 = rng.standard_normal((n, nrhs))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    ipiv = torch.zeros(n, dtype=torch.int32, device=cuda)
    info = torch.full((1,), -7, dtype=torch.int32, device=cuda)
    lnb.dgetrf_dev(At, n, n, ipiv, info=info)
    lnb.dgetrs_dev(At, ipiv, Bt, n, nrhs)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    _, piv, _ = la.dgetrf(A0)
    np.testing.assert_array_equal(ipiv.cpu().numpy(), piv + 1)
    np.testing.assert_allclose(Bt.cpu().numpy().T, np.linalg.solve(A0, B0), rtol=0, atol=1e-10)


def test_getrf_errors(lnb):
    A = np.asfortranarray(np.eye(4))
    with pytest.raises(lnb.LinompssError):
        lnb.ompss_getrf(A, 0)


def test_getrf_rows_limit(lnb):
    """more rows than a panel cluster holds: LNB_ETOOBIG before any device work"""
    A = np.asfortranarray(np.ones((32769, 2)))
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_getrf(A, 2)
    assert e.value.code == lnb.LNB_ETOOBIG
    A = np.asfortranarray(np.random.default_rng(3).standard_normal((32768, 4)))
    lu, piv, _ = la.dgetrf(A)
    info, ipiv = lnb.ompss_getrf(A, 4)
    assert info == 0
    np.testing.assert_array_equal(global_pivots(ipiv, 4), piv + 1)
    np.testing.assert_allclose(A, lu, rtol=0, atol=1e-12)
