"""Entry points of the C ABI not covered by the other GPU files, each against
the oracle (or LAPACK through numpy for the FP32 factors):

  ompss_dchol_nhrl / ompss_dchol_nhll   nested hypermatrix forms (chol_nrlmain.c,
                                        chol_nllmain.c): same factor as hrl/hll
  ompss_schol_ll, ompss_schol_hll        FP32 twins of the left-looking drivers
  ompss_schol_hrl                        in every factor mode
  lnb_dpotrs_dev                         'N', 'T' and 'B' alone
  lnb_dtrsm_dev                          the four triangle/transpose cases, unit
                                         diagonal, alpha, few and many columns
  lnb_spotrs_dev                         'N' and 'T' alone
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps
U32 = np.finfo(np.float32).eps / 2
MODES = {"fp32": 1, "tf32x3": 2, "bf16": 3, "tf32": 4}
RESID = {"fp32": 10 * U32, "tf32x3": 10 * U32, "tf32": 2.0 ** -11, "bf16": 2.0 ** -8}


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    yield linompss_b200
    linompss_b200.set_factor_mode(linompss_b200.FACTOR_TF32X3)


def to_tiles(A, mt, b, dtype):
    tiles = np.zeros((mt, mt, b, b), dtype=dtype)
    for j in range(mt):
        for i in range(mt):
            tiles[j, i] = A[i * b:(i + 1) * b, j * b:(j + 1) * b].T
    return tiles


@pytest.mark.parametrize("name", ["chol_hrl_mt4_b16", "chol_hll_mt4_b16", "chol_hrl_mt3_b24"])
@pytest.mark.parametrize("variant", ["nhrl", "nhll"])
def test_nested_hypermatrix_golden(lnb, golden_dir, name, variant):
    """The nested drivers compute the same factor as hrl/hll; the golden
    outputs of the reference's hrl/hll pin it."""
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    tiles = d["tiles_in"].copy()
    mt, b = tiles.shape[0], tiles.shape[2]
    assert getattr(lnb, "ompss_dchol_" + variant)(mt, b, b, tiles) == 0
    for j in range(mt):
        for i in range(j, mt):
            ref, got = d["tiles_out"][j, i].T, tiles[j, i].T
            if i == j:
                ref, got = np.tril(ref), np.tril(got)
            np.testing.assert_allclose(got, ref, rtol=0, atol=64 * EPS * 64)
        for i in range(j):
            np.testing.assert_array_equal(tiles[j, i], d["tiles_in"][j, i])


def resid32(A0, L):
    n = A0.shape[0]
    Lt = np.tril(L.astype(np.float64))
    R = Lt @ Lt.T - A0.astype(np.float64)
    return np.abs(R).sum(axis=1).max() / (np.abs(A0).sum(axis=1).max() * n)


@pytest.mark.parametrize("mode", ["fp32", "tf32x3", "tf32", "bf16"])
def test_schol_hrl_every_mode(lnb, mode):
    lnb.set_factor_mode(MODES[mode])
    mt, b = 5, 128
    n = mt * b
    A0 = O.spd_covariance(n, 1.0, seed=50).astype(np.float32)
    tiles = to_tiles(A0, mt, b, np.float32)
    assert lnb.ompss_schol_hrl(mt, b, b, tiles) == 0
    L = np.zeros((n, n), dtype=np.float32)
    for j in range(mt):
        for i in range(j, mt):
            L[i * b:(i + 1) * b, j * b:(j + 1) * b] = tiles[j, i].T
    assert resid32(A0, L) <= RESID[mode]
    if mode in ("fp32", "tf32x3"):
        L64 = np.linalg.cholesky(A0.astype(np.float64))
        np.testing.assert_allclose(np.tril(L), L64, rtol=0, atol=2e-5 * np.abs(L64).max())
    orig = to_tiles(A0, mt, b, np.float32)
    for j in range(mt):
        for i in range(j):
            np.testing.assert_array_equal(tiles[j, i], orig[j, i])


@pytest.mark.parametrize("mode", ["fp32", "tf32x3"])
def test_schol_ll_and_hll(lnb, mode):
    lnb.set_factor_mode(MODES[mode])
    n, b = 777, 128
    A0 = O.spd_covariance(n, 1.0, seed=51).astype(np.float32)
    A = np.asfortranarray(A0.copy())
    assert lnb.ompss_schol_ll(n, b, b, A, n) == 0
    L64 = np.linalg.cholesky(A0.astype(np.float64))
    np.testing.assert_allclose(np.tril(A), L64, rtol=0, atol=2e-5 * np.abs(L64).max())
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(A0, 1))
    mt, bh = 4, 96
    nh = mt * bh
    Ah = O.spd_covariance(nh, 1.0, seed=52).astype(np.float32)
    tiles = to_tiles(Ah, mt, bh, np.float32)
    assert lnb.ompss_schol_hll(mt, bh, bh, tiles) == 0
    L64 = np.linalg.cholesky(Ah.astype(np.float64))
    for j in range(mt):
        for i in range(j, mt):
            got = tiles[j, i].T.astype(np.float64)
            ref = L64[i * bh:(i + 1) * bh, j * bh:(j + 1) * bh]
            if i == j:
                got, ref = np.tril(got), np.tril(ref)
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5 * np.abs(L64).max())


def dev_cols(M, cuda):
    """a column-major matrix as a (cols, rows) tensor on the device"""
    import torch
    return torch.tensor(np.ascontiguousarray(M.T), device=cuda)


@pytest.mark.parametrize("which", ["N", "T", "B"])
@pytest.mark.parametrize("n,nrhs", [(1000, 1), (1000, 5), (777, 20)])
def test_dpotrs_dev_each_direction(lnb, cuda, which, n, nrhs):
    import torch
    A0 = O.spd_covariance(n, 1e-1, seed=n + nrhs)
    L = np.linalg.cholesky(A0)
    B0 = np.asfortranarray(np.random.default_rng(n).standard_normal((n, nrhs)))
    Lt, Bt = dev_cols(L, cuda), dev_cols(B0, cuda)
    lnb.dpotrs_dev(Lt, Bt, n, nrhs, which)
    torch.cuda.synchronize()
    X = Bt.cpu().numpy().T
    ref = B0.copy(order="F")
    if which in ("N", "B"):
        O.ltrsm("L", "N", "N", 64, 1.0, O.fortran(L), ref)
    if which in ("T", "B"):
        O.ltrsm("L", "T", "N", 64, 1.0, O.fortran(L), ref)
    np.testing.assert_allclose(X, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("L", "T", "U"), ("U", "N", "N"), ("U", "T", "U")])
@pytest.mark.parametrize("m,n", [(300, 1), (513, 7), (640, 33)])
def test_dtrsm_dev_vs_oracle(lnb, cuda, uplo, trans, diag, m, n):
    import torch
    rng = np.random.default_rng(m * 3 + n)
    T = np.asfortranarray(rng.uniform(-1, 1, (m, m)) / np.sqrt(m) + (1.0 if diag == "U" else 3.0) * np.eye(m))
    B0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    Tt, Bt = dev_cols(T, cuda), dev_cols(B0, cuda)
    lnb.dtrsm_dev(uplo, trans, diag, m, n, -0.75, Tt, Bt)
    torch.cuda.synchronize()
    ref = B0.copy(order="F")
    O.ltrsm(uplo, trans, diag, 64, -0.75, T, ref)
    np.testing.assert_allclose(Bt.cpu().numpy().T, ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("which", ["N", "T"])
@pytest.mark.parametrize("n,nrhs", [(900, 1), (900, 3), (500, 12)])
def test_spotrs_dev_each_direction(lnb, cuda, which, n, nrhs):
    """FP32 factor and right-hand sides; the solve computes in FP64 and rounds
    the result once, so it matches the FP64 solve with the FP32 factor to FP32
    rounding of the result."""
    import torch
    A0 = O.spd_covariance(n, 1e-1, seed=2 * n + nrhs)
    L32 = np.linalg.cholesky(A0).astype(np.float32)
    B32 = np.random.default_rng(n).standard_normal((n, nrhs)).astype(np.float32)
    Lt, Bt = dev_cols(L32, cuda), dev_cols(B32, cuda)
    lnb.spotrs_dev(Lt, Bt, n, nrhs, which)
    torch.cuda.synchronize()
    ref = np.asfortranarray(B32.astype(np.float64))
    O.ltrsm("L", which, "N", 64, 1.0, O.fortran(L32.astype(np.float64)), ref)
    got = Bt.cpu().numpy().T.astype(np.float64)
    np.testing.assert_allclose(got, ref, rtol=4 * U32, atol=4 * U32 * np.abs(ref).max())
