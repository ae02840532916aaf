"""GPU parity of the FP64 path against the oracle and the reference's golden
outputs.  Every call goes through the C ABI (liblinompss_b200.so).

Bars (from the reference's own checks):
  factor: ||A - L L^T||_inf / (||A||_inf n eps) <= 10   (potrf_test.c:31-36)
  solve : normwise backward error <= 10 n eps
  vs oracle/golden: entrywise, to the rounding of blocked FP64 sums
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


def factor_ok(A0, L):
    return O.chol_residual_np(A0, L) <= 10.0


# ---------------------------------------------------------------- factor
@pytest.mark.parametrize("name", ["chol_rl_n100_b32", "chol_rl_n128_b32", "chol_rl_n199_b53",
                                  "chol_ll_n100_b32", "chol_ll_n128_b64"])
def test_chol_golden(lnb, golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    n, b = A.shape[0], int(d["b"])
    f = lnb.ompss_dchol_rl if "_rl_" in name else lnb.ompss_dchol_ll
    assert f(n, b, b, A, n) == 0
    np.testing.assert_allclose(np.tril(A), np.tril(d["out"]), rtol=0,
                               atol=64 * EPS * np.abs(d["out"]).max())
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(d["A"], 1))  # upper untouched
    assert factor_ok(d["A"], A)


@pytest.mark.parametrize("name", ["chol_hrl_mt4_b16", "chol_hll_mt4_b16", "chol_hrl_mt3_b24"])
def test_chol_hypermatrix_golden(lnb, golden_dir, name):
    d = load(golden_dir, name)
    tiles = d["tiles_in"].copy()
    mt, b = tiles.shape[0], tiles.shape[2]
    f = lnb.ompss_dchol_hrl if "_hrl_" in name else lnb.ompss_dchol_hll
    assert f(mt, b, b, tiles) == 0
    for j in range(mt):
        for i in range(j, mt):
            ref, got = d["tiles_out"][j, i].T, tiles[j, i].T
            if i == j:
                ref, got = np.tril(ref), np.tril(got)
            np.testing.assert_allclose(got, ref, rtol=0, atol=64 * EPS * 64)
        for i in range(j):  # strictly-upper tiles never touched
            np.testing.assert_array_equal(tiles[j, i], d["tiles_in"][j, i])


@pytest.mark.parametrize("n,b", [(1, 1), (7, 16), (31, 32), (64, 32), (65, 32), (300, 100), (257, 256),
                                 (513, 128), (1000, 250), (2048, 256)])
def test_chol_sizes_vs_oracle(lnb, n, b):
    A0 = O.spd_diag_dominant(n, seed=n * 7 + b)
    A = A0.copy(order="F")
    assert lnb.ompss_dchol_rl(n, b, b, A, n) == 0
    L = np.linalg.cholesky(A0)
    np.testing.assert_allclose(np.tril(A), L, rtol=0, atol=256 * EPS * np.abs(L).max())
    assert factor_ok(A0, A)


def test_chol_lda_larger_than_n(lnb):
    n, b, lda = 200, 64, 237
    A0 = O.spd_diag_dominant(n, seed=5)
    big = np.asfortranarray(np.full((lda, n), 7.25))
    big[:n, :] = A0
    assert lnb.ompss_dchol_rl(n, b, b, big, lda) == 0
    np.testing.assert_allclose(np.tril(big[:n]), np.linalg.cholesky(A0), rtol=0, atol=1e-12 * n)
    np.testing.assert_array_equal(big[n:], 7.25)   # rows past n untouched


def test_chol_covariance_matches_oracle(lnb):
    n, b = 384, 128
    A0 = O.spd_covariance(n, 1e-2, seed=3)
    A1, A2 = A0.copy(order="F"), A0.copy(order="F")
    assert lnb.ompss_dchol_rl(n, b, b, A1, n) == 0
    assert O.chol_rl(A2, b) == 0
    np.testing.assert_allclose(np.tril(A1), np.tril(A2), rtol=0, atol=1e-11)
    assert O.chol_residual(A0, A1) <= 10.0


@pytest.mark.parametrize("pos", [0, 5, 40, 130, 299])
def test_chol_not_spd_reports_info(lnb, pos):
    n, b = 300, 64
    A0 = O.spd_diag_dominant(n, seed=11)
    A0[pos, pos] = -1.0
    A1, A2 = A0.copy(order="F"), A0.copy(order="F")
    info = lnb.ompss_dchol_rl(n, b, b, A1, n)
    assert info == O.chol_rl(A2, b) == pos + 1
    # columns before the failing one are the (valid) factor
    if pos > 0:
        np.testing.assert_allclose(np.tril(A1)[:, :pos], np.tril(A2)[:, :pos], rtol=0, atol=1e-11)


# ---------------------------------------------------------------- solves
@pytest.mark.parametrize("name", ["spdsolv_m128_r1_b32", "spdsolv_m128_r3_b32", "spdsolv_m96_r8_b48"])
def test_spdsolv_golden(lnb, golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    B = d["B"].copy(order="F")
    m, nrhs = B.shape
    b = int(name.split("_b")[-1])
    assert lnb.dspdsolv_main(m, nrhs, b, A, B) == 0
    np.testing.assert_allclose(B, d["X"], rtol=1e-12, atol=1e-13)
    assert O.backward_error(d["A"], B, d["B"]) <= 10 * m * EPS


@pytest.mark.parametrize("m,nrhs,b", [(1, 1, 4), (100, 1, 32), (333, 5, 64), (1024, 64, 256), (2048, 1, 256),
                                      (2048, 64, 256), (700, 130, 100)])
def test_spdsolv_sizes(lnb, m, nrhs, b):
    rng = np.random.default_rng(m + nrhs)
    A0 = O.spd_diag_dominant(m, seed=m)
    X0 = rng.uniform(-1, 1, (m, nrhs))
    B0 = np.asfortranarray(A0 @ X0)
    A, B = A0.copy(order="F"), B0.copy(order="F")
    assert lnb.dspdsolv_main(m, nrhs, b, A, B) == 0
    assert O.backward_error_np(A0, B, B0) <= 10 * m * EPS
    np.testing.assert_allclose(B, np.linalg.solve(A0, B0), rtol=0, atol=1e-12 * max(1, np.abs(X0).max()))


@pytest.mark.parametrize("case", ["LLN", "LLT", "LUN", "LUT"])
def test_dtrsm_golden(lnb, golden_dir, case):
    d = load(golden_dir, "dtrsm_" + case)
    M, N, bb, alpha = int(d["M"]), int(d["N"]), int(d["bb"]), float(d["alpha"])
    A = d["A"].copy(order="F")
    B = d["B"].copy(order="F")
    lnb.ompss_dtrsm("L", case[1], case[2], "N", M, N, bb, alpha, A, A.shape[0], B, B.shape[0])
    ref = d["out"]
    relerr = np.abs(B[:M, :N] - ref[:M, :N]).sum(axis=0).max() / np.abs(ref[:M, :N]).sum(axis=0).max()
    assert relerr < 1e-12
    np.testing.assert_array_equal(B[M:], d["B"][M:])


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("L", "T", "N"), ("U", "N", "U"), ("U", "T", "N")])
def test_dtrsm_vs_oracle_ragged(lnb, uplo, trans, diag):
    rng = np.random.default_rng(1)
    m, n = 203, 17
    # well conditioned for both diagonal kinds: small off-diagonal entries
    T = np.asfortranarray(rng.uniform(-1, 1, (m, m)) / m + (1.0 if diag == "U" else 2.0) * np.eye(m))
    B0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    B1, B2 = B0.copy(order="F"), B0.copy(order="F")
    lnb.ompss_dtrsm("L", uplo, trans, diag, m, n, 64, 0.5, T, m, B1, m)
    O.ltrsm(uplo, trans, diag, 64, 0.5, T, B2)
    np.testing.assert_allclose(B1, B2, rtol=1e-13, atol=1e-15)


@pytest.mark.parametrize("uplo,trans,diag", [("L", "N", "N"), ("L", "T", "N"), ("U", "N", "U"), ("U", "T", "N")])
@pytest.mark.parametrize("m,n", [(64, 1), (65, 2), (700, 3), (2500, 1), (2500, 8), (1999, 5)])
def test_dtrsm_few_rhs_vs_oracle(lnb, uplo, trans, diag, m, n):
    """1..8 right-hand sides take the diagonal-chain launch: every band width
    and worker-item shape, ragged last block, all four triangle/transpose cases."""
    rng = np.random.default_rng(m + 7 * n)
    T = np.asfortranarray(rng.uniform(-1, 1, (m, m)) / np.sqrt(m) + (1.0 if diag == "U" else 3.0) * np.eye(m))
    B0 = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    B1, B2 = B0.copy(order="F"), B0.copy(order="F")
    lnb.ompss_dtrsm("L", uplo, trans, diag, m, n, 64, 1.0, T, m, B1, m)
    O.ltrsm(uplo, trans, diag, 64, 1.0, T, B2)
    np.testing.assert_allclose(B1, B2, rtol=1e-12, atol=1e-13 * np.abs(B2).max())


# ---------------------------------------------------------------- tile tasks
def test_task_potrf_lower_and_upper(lnb):
    n = 150
    A0 = O.spd_diag_dominant(n, seed=4)
    A = A0.copy(order="F")
    assert lnb.task_dpotrf("L", n, A, n) == 0
    np.testing.assert_allclose(np.tril(A), np.linalg.cholesky(A0), rtol=0, atol=1e-11)
    U = A0.copy(order="F")
    assert lnb.task_dpotrf("U", n, U, n) == 0
    np.testing.assert_allclose(np.triu(U), np.linalg.cholesky(A0).T, rtol=0, atol=1e-11)


@pytest.mark.parametrize("side,uplo,trans", [("R", "L", "T"), ("L", "L", "N"), ("R", "U", "N"), ("L", "U", "T")])
def test_task_trsm(lnb, side, uplo, trans):
    rng = np.random.default_rng(2)
    bm, bn = 48, 40
    na = bm if side == "L" else bn
    A = np.asfortranarray(rng.uniform(-1, 1, (na, na)) + 3 * na * np.eye(na))
    B0 = np.asfortranarray(rng.uniform(-1, 1, (bm, bn)))
    B1 = B0.copy(order="F")
    B2 = B0.copy(order="F")
    lnb.task_dtrsm(side, uplo, trans, "N", bm, bn, 2.0, A, na, B1, bm)
    O.lib().orc_dtrsm(*[O.C.c_char(x.encode()) for x in (side, uplo, trans, "N")], O._i64(bm), O._i64(bn),
                      O.C.c_double(2.0), O._ptr(A), O._i64(na), O._ptr(B2), O._i64(bm))
    np.testing.assert_allclose(B1, B2, rtol=1e-13, atol=1e-14)


def test_task_syrk_gemm(lnb):
    rng = np.random.default_rng(3)
    n, k = 70, 33
    A = np.asfortranarray(rng.standard_normal((n, k)))
    C0 = np.asfortranarray(rng.standard_normal((n, n)))
    C1 = C0.copy(order="F")
    lnb.task_dsyrk("L", "N", n, k, -1.0, A, n, 1.0, C1, n)
    ref = C0 - A @ A.T
    np.testing.assert_allclose(np.tril(C1), np.tril(ref), rtol=0, atol=1e-12)
    np.testing.assert_array_equal(np.triu(C1, 1), np.triu(C0, 1))
    Bm = np.asfortranarray(rng.standard_normal((40, k)))
    C2 = np.asfortranarray(rng.standard_normal((n, 40)))
    C3 = C2.copy(order="F")
    lnb.task_dgemm("N", "T", n, 40, k, -1.0, A, n, Bm, 40, 1.0, C3, n)
    np.testing.assert_allclose(C3, C2 - A @ Bm.T, rtol=0, atol=1e-12)


# ---------------------------------------------------------------- device API
def test_device_chol_and_potrs(lnb, cuda):
    import torch
    n, nrhs, b = 1536, 3, 256
    A0 = O.spd_covariance(n, 1e-2, seed=9)
    B0 = np.asfortranarray(np.random.default_rng(9).standard_normal((n, nrhs)))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)     # column-major view
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    info = torch.zeros(1, dtype=torch.int32, device=cuda)
    lnb.dposv_dev(At, Bt, n, nrhs, b, info=info)
    torch.cuda.synchronize()
    assert int(info.item()) == 0
    X = Bt.cpu().numpy().T
    assert O.backward_error_np(A0, X, B0) <= 10 * n * EPS


# ---------------------------------------------------------------- itref
@pytest.mark.parametrize("name", ["dcg_n64_bm16_s8", "dcg_n64_bm16_s200", "dcg_n100_bm32_s300"])
def test_dcg_golden(lnb, golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    n = A.shape[0]
    x = np.zeros(n)
    rc = lnb.ompss_dcg(n, int(d["bm"]), A, n, d["rhs"].copy(), x, float(d["tol"]), int(d["steps"]))
    assert rc == int(d["rc"])
    np.testing.assert_allclose(x, d["x"], rtol=0, atol=1e-11 * max(1.0, np.abs(d["x"]).max()))


@pytest.mark.parametrize("name", ["itref_n64_bm16", "itref_n96_bm32"])
def test_itref_golden(lnb, golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    n = A.shape[0]
    x = np.zeros(n)
    norms = np.zeros(int(d["refit"]))
    k = lnb.ompss_ditref(n, int(d["bm"]), A, n, d["rhs"].copy(), x, float(d["prec"]), int(d["refit"]),
                         int(d["it"]), norms)
    ko, xo, no = O.itref(d["A"], d["rhs"], int(d["bm"]), float(d["prec"]), int(d["refit"]), int(d["it"]))
    assert k == ko
    assert norms[0] == pytest.approx(d["norms_logged"][0], rel=1e-6)
    assert norms[k - 1] <= float(d["prec"])
    np.testing.assert_allclose(x, xo, rtol=0, atol=1e-12)
    assert O.backward_error(d["A"], x, d["rhs"]) <= 10 * n * EPS


@pytest.mark.parametrize("case", ["LN_b", "LN_b0", "LT_b", "UN_b", "UT_b"])
def test_ompss_dsyrk_golden(lnb, golden_dir, case):
    """ompss_dsyrk against the reference's blocked SYRK (syrk_main.c): ragged
    n and k against the tile size, padded lda/ldc, beta 0; the other triangle
    and the rows past n stay as they were."""
    d = load(golden_dir, "dsyrk_" + case)
    n, k, bb = int(d["n"]), int(d["k"]), int(d["bb"])
    alpha, beta = float(d["alpha"]), float(d["beta"])
    A = d["A"].copy(order="F")
    Cm = d["C"].copy(order="F")
    assert lnb.ompss_dsyrk(case[0], case[1], bb, n, k, alpha, A, A.shape[0], Cm, Cm.shape[0], beta=beta) == 0
    ref = d["out"]
    np.testing.assert_allclose(Cm, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    if beta != 0.0:
        np.testing.assert_array_equal(Cm[n:], d["C"][n:])


@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_ompss_ssyrk_vs_fp64(lnb, uplo, trans):
    """The FP32 twin computes in FP64 and rounds once: within FP32 rounding of
    the exact result of its FP32 inputs; the other triangle untouched."""
    rng = np.random.default_rng(5)
    n, k = 300, 130
    A = np.asfortranarray(rng.standard_normal((n, k) if trans == "N" else (k, n)).astype(np.float32))
    C0 = np.asfortranarray(rng.standard_normal((n, n)).astype(np.float32))
    Cm = C0.copy(order="F")
    assert lnb.ompss_ssyrk(uplo, trans, 64, n, k, 0.5, A, A.shape[0], Cm, n, beta=-1.0) == 0
    op = A.astype(np.float64) if trans == "N" else A.astype(np.float64).T
    ref = -1.0 * C0.astype(np.float64) + 0.5 * op @ op.T
    tri = np.tril if uplo == "L" else np.triu
    np.testing.assert_allclose(tri(Cm.astype(np.float64)), tri(ref), rtol=0,
                               atol=2 * np.finfo(np.float32).eps * np.abs(ref).max())
    other = (lambda x: np.triu(x, 1)) if uplo == "L" else (lambda x: np.tril(x, -1))
    np.testing.assert_array_equal(other(Cm), other(C0))


def test_ompss_dsyrk_rejects_bad_arguments(lnb):
    A = np.zeros((4, 4), order="F")
    Cm = np.zeros((4, 4), order="F")
    with pytest.raises(lnb.LinompssError):
        lnb.ompss_dsyrk("X", "N", 2, 4, 4, 1.0, A, 4, Cm, 4)
    with pytest.raises(lnb.LinompssError):
        lnb.ompss_dsyrk("L", "N", 0, 4, 4, 1.0, A, 4, Cm, 4)


def test_ompss_ssyrk_golden(lnb, golden_dir):
    """ompss_ssyrk against the reference's FP32 blocked SYRK: the library sums in
    FP64 and rounds once, so it differs from the reference's FP32 sums by their
    rounding; the other triangle and the rows past n are untouched."""
    d = load(golden_dir, "ssyrk_LN_b")
    n, k, bb = int(d["n"]), int(d["k"]), int(d["bb"])
    A = d["A"].copy(order="F")
    Cm = d["C"].copy(order="F")
    assert lnb.ompss_ssyrk("L", "N", bb, n, k, float(d["alpha"]), A, A.shape[0], Cm, Cm.shape[0],
                           beta=float(d["beta"])) == 0
    tol = 4 * k * np.finfo(np.float32).eps * np.abs(d["out"]).max()
    np.testing.assert_allclose(Cm, d["out"], rtol=0, atol=tol)
    np.testing.assert_array_equal(np.triu(Cm[:n], 1), np.triu(d["C"][:n], 1))
    np.testing.assert_array_equal(Cm[n:], d["C"][n:])
