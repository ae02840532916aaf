"""GPU parity of the FP32 tile Cholesky (ompss_schol_rl, the reference's
schol_rl) in each update mode, through the C ABI.

Tolerances are per mode, stated against the FP32 unit roundoff u32:
  FP32 (SIMT) and TF32x3 (tcgen05, hi/lo split): FP32-level factor,
      ||A - L L^T|| / (n u32 ||A||) <= 10 and entrywise close to the
      reference's own FP32 output (golden) / the FP64 factor
  TF32 (one product, 10-bit mantissa operands) and BF16 (8-bit):
      the factor is a preconditioner-grade approximation; bounds scale with
      the operand precision (2^-11, 2^-8).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
U32 = np.finfo(np.float32).eps / 2

MODES = {"fp32": 1, "tf32x3": 2, "bf16": 3, "tf32": 4}
# bound on ||A - L L^T||_inf / (||A||_inf n) per mode
RESID = {"fp32": 10 * U32, "tf32x3": 10 * U32, "tf32": 2.0 ** -11, "bf16": 2.0 ** -8}


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    yield linompss_b200
    linompss_b200.set_factor_mode(linompss_b200.FACTOR_TF32X3)


def resid32(A0, L):
    n = A0.shape[0]
    Lt = np.tril(L.astype(np.float64))
    R = Lt @ Lt.T - A0.astype(np.float64)
    return np.abs(R).sum(axis=1).max() / (np.abs(A0).sum(axis=1).max() * n)


@pytest.mark.parametrize("mode", ["fp32", "tf32x3", "tf32", "bf16"])
def test_schol_golden(lnb, golden_dir, mode):
    d = np.load(os.path.join(golden_dir, "schol_rl_n96_b32.npz"))
    lnb.set_factor_mode(MODES[mode])
    A = np.asfortranarray(d["A"].copy())
    assert lnb.ompss_schol_rl(96, 32, 32, A, 96) == 0
    assert resid32(d["A"], A) <= RESID[mode]
    if mode in ("fp32", "tf32x3"):
        np.testing.assert_allclose(np.tril(A), np.tril(d["out"]), rtol=0,
                                   atol=64 * U32 * np.abs(d["out"]).max())
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(d["A"], 1))


@pytest.mark.parametrize("mode", ["fp32", "tf32x3", "tf32", "bf16"])
@pytest.mark.parametrize("n,b", [(130, 64), (300, 128), (1000, 256), (1024, 512), (2048, 256), (777, 200)])
def test_schol_modes_sizes(lnb, mode, n, b):
    lnb.set_factor_mode(MODES[mode])
    A0 = O.spd_covariance(n, 1.0, seed=n + b)
    A = np.asfortranarray(A0.astype(np.float32))
    assert lnb.ompss_schol_rl(n, b, b, A, n) == 0
    r = resid32(A0, A)
    assert r <= RESID[mode], r
    if mode in ("fp32", "tf32x3"):
        L = np.linalg.cholesky(A0)
        np.testing.assert_allclose(np.tril(A), L, rtol=0, atol=2e-5 * np.abs(L).max())


def test_tf32x3_matches_fp32_simt(lnb):
    """The split product recovers FP32-level accuracy: measured against the
    FP64 factor of the same (FP32-valued) matrix, the TF32x3 factor's error is
    at the level of the SIMT FP32 factor's, and a single TF32 product's is
    several times larger.  (The factors differ in accumulation order, so the
    comparison is made against the FP64 factor, not between the modes.)"""
    n, b = 1536, 256
    A0 = O.spd_covariance(n, 0.1, seed=7).astype(np.float32)
    L64 = np.linalg.cholesky(A0.astype(np.float64))
    scale = np.abs(L64).max()
    err = {}
    for mode in ("fp32", "tf32x3", "tf32"):
        lnb.set_factor_mode(MODES[mode])
        A = np.asfortranarray(A0.copy())
        assert lnb.ompss_schol_rl(n, b, b, A, n) == 0
        err[mode] = np.abs(np.tril(A).astype(np.float64) - L64).max() / scale
    assert err["tf32x3"] <= max(4 * err["fp32"], 2e-5), err
    assert err["tf32"] >= 4 * err["tf32x3"], err


def test_schol_hypermatrix(lnb):
    lnb.set_factor_mode(MODES["tf32x3"])
    mt, b = 4, 64
    n = mt * b
    A0 = O.spd_covariance(n, 1.0, seed=3).astype(np.float32)
    tiles = np.zeros((mt, mt, b, b), dtype=np.float32)
    for j in range(mt):
        for i in range(mt):
            tiles[j, i] = A0[i * b:(i + 1) * b, j * b:(j + 1) * b].T
    assert lnb.ompss_schol_hrl(mt, b, b, tiles) == 0
    L = np.linalg.cholesky(A0.astype(np.float64))
    for j in range(mt):
        for i in range(j, mt):
            got = tiles[j, i].T.astype(np.float64)
            ref = L[i * b:(i + 1) * b, j * b:(j + 1) * b]
            if i == j:
                got, ref = np.tril(got), np.tril(ref)
            np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5 * np.abs(L).max())


@pytest.mark.parametrize("mode", ["fp32", "tf32x3"])
@pytest.mark.parametrize("n,b,bad", [(400, 128, 300), (1200, 512, 700), (1200, 512, 520), (1200, 512, 1100),
                                       (1000, 200, 450), (256, 256, 0)])
def test_schol_not_spd(lnb, mode, n, b, bad):
    """A negative pivot is reported 1-based from every diagonal-tile path: the
    cluster factor (whole 32-blocks: b = 512, 256), the leaf (b <= 128, the
    ragged last tile) and the nested path (lda % 4 != 0)."""
    lnb.set_factor_mode(MODES[mode])
    lda = n + 1 if b == 200 else n
    A0 = O.spd_diag_dominant(n, seed=2).astype(np.float32)
    A0[bad, bad] = -5.0
    A = np.zeros((lda, n), dtype=np.float32, order="F")
    A[:n] = A0
    assert lnb.ompss_schol_rl(n, b, b, A, lda) == bad + 1


@pytest.mark.parametrize("n,nrhs", [(3001, 1), (3001, 8), (4096, 2), (8192, 3), (9000, 8)])
def test_spotrs_chain_matches_fp64_solve(lnb, cuda, n, nrhs):
    """FP32-stored factor, FP64 right-hand sides and arithmetic: the solve
    equals an FP64 triangular solve with the same (FP32-valued) factor.  From
    n = 1024 the solve runs on the inverses of 512-wide diagonal blocks (9000:
    a ragged last block)."""
    import torch
    rng = np.random.default_rng(n + nrhs)
    L = np.tril(rng.uniform(-1, 1, (n, n)) / np.sqrt(n)).astype(np.float32)
    L[np.diag_indices(n)] = (2.0 + rng.uniform(0, 1, n)).astype(np.float32)
    B0 = rng.standard_normal((n, nrhs))
    Lt = torch.tensor(np.ascontiguousarray(L.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T).astype(np.float32), device=cuda)
    lnb.spotrs_dev(Lt, Bt, n, nrhs, "B")
    torch.cuda.synchronize()
    L64 = L.astype(np.float64)
    import scipy.linalg as sl
    Y = sl.solve_triangular(L64, B0.astype(np.float32).astype(np.float64), lower=True)
    X = sl.solve_triangular(L64.T, Y, lower=False)
    got = Bt.cpu().numpy().T.astype(np.float64)
    # the device result is rounded to FP32 on the way out
    np.testing.assert_allclose(got, X, rtol=0, atol=2e-7 * np.abs(X).max())


@pytest.mark.parametrize("mode", ["tf32x3", "tf32", "bf16"])
@pytest.mark.parametrize("n,b", [(2048, 512), (1000, 256), (777, 200)])
def test_update_cta_pairs_match_single_cta(lnb, monkeypatch, mode, n, b):
    """The trailing update runs on 2-CTA clusters (256 x 256 tiles, cta_group::2
    MMAs) by default; LNB_TC_PAIR=0 selects the single-CTA 128 x 128 kernel.
    Both compute the same products in a different accumulation order, so the
    factors agree to the precision of the mode and meet the same residual bound."""
    A0 = O.spd_covariance(n, 1.0, seed=n + 11)
    out = {}
    for pair in ("1", "0"):
        monkeypatch.setenv("LNB_TC_PAIR", pair)
        lnb.set_factor_mode(MODES[mode])
        A = np.asfortranarray(A0.astype(np.float32))
        assert lnb.ompss_schol_rl(n, b, b, A, n) == 0
        assert resid32(A0, A) <= RESID[mode]
        out[pair] = np.tril(A).astype(np.float64)
    tol = {"tf32x3": 2e-5, "tf32": 2e-3, "bf16": 2e-2}[mode]
    np.testing.assert_allclose(out["1"], out["0"], rtol=0, atol=tol * np.abs(out["0"]).max())


@pytest.mark.parametrize("bs", [64, 96, 160, 352, 480, 512])
def test_cluster_diagonal_factor_single_tile(lnb, bs):
    """One diagonal tile (n = b, whole 32-blocks): the 8-CTA cluster factor alone,
    for odd and even block counts (block rows q and 15 - q per CTA).  The factor
    meets the FP32 residual bound and matches the FP64 Cholesky; the upper
    triangle keeps its input values."""
    lnb.set_factor_mode(MODES["tf32x3"])
    A0 = O.spd_covariance(bs, 0.5, seed=bs)
    A = np.asfortranarray(A0.astype(np.float32))
    upper = np.triu(A, 1).copy()
    assert lnb.ompss_schol_rl(bs, bs, bs, A, bs) == 0
    assert resid32(A0, A) <= RESID["tf32x3"]
    L = np.linalg.cholesky(A0)
    np.testing.assert_allclose(np.tril(A), L, rtol=0, atol=2e-5 * np.abs(L).max())
    np.testing.assert_array_equal(np.triu(A, 1), upper)


@pytest.mark.parametrize("bs,bad", [(512, 0), (512, 31), (512, 32), (512, 300), (512, 511), (160, 100)])
def test_cluster_diagonal_factor_reports_pivot(lnb, bs, bad):
    """A non-positive pivot inside a single cluster-factored tile is reported
    1-based, from the first block (step before the sweep) to the last one."""
    lnb.set_factor_mode(MODES["tf32x3"])
    A0 = O.spd_diag_dominant(bs, seed=bs + bad).astype(np.float32)
    A0[bad, bad] = -5.0
    A = np.asfortranarray(A0.copy())
    assert lnb.ompss_schol_rl(bs, bs, bs, A, bs) == bad + 1
