"""Pin the CPU oracle against the reference's own outputs (tests/golden/).

The fixtures were recorded from the reference compiled from its sources
(tests/golden/make_golden.py).  The reference delegates every tile to an
external BLAS/LAPACK (OpenBLAS here), whose summation order differs from the
oracle's triple loops, so agreement is to rounding, with tolerances scaled
by the problem's conditioning.  Only the lower triangle is compared for the
factorizations: that is the output contract, and the reference writes stray
values into the unused upper triangle when n % b != 0 (chol_rlmain.c:36).
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name + ".npz"))


@pytest.mark.parametrize("name", ["chol_rl_n100_b32", "chol_rl_n128_b32", "chol_rl_n199_b53",
                                  "chol_ll_n100_b32", "chol_ll_n128_b64"])
def test_chol_colmajor(golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    b = int(d["b"])
    info = O.chol_rl(A, b) if "_rl_" in name else O.chol_ll(A, b)
    assert info == int(d["info"]) == 0
    ref = np.tril(d["out"])
    got = np.tril(A)
    np.testing.assert_allclose(got, ref, rtol=0, atol=64 * np.finfo(float).eps * np.abs(ref).max())
    assert O.chol_residual(d["A"], A) <= 10.0
    assert O.chol_residual(d["A"], d["out"]) <= 10.0


def test_chol_rl_upper_untouched_by_oracle(golden_dir):
    d = load(golden_dir, "chol_rl_n199_b53")
    A = d["A"].copy(order="F")
    O.chol_rl(A, 53)
    np.testing.assert_array_equal(np.triu(A, 1), np.triu(d["A"], 1))


@pytest.mark.parametrize("name", ["chol_hrl_mt4_b16", "chol_hll_mt4_b16", "chol_hrl_mt3_b24"])
def test_chol_hypermatrix(golden_dir, name):
    d = load(golden_dir, name)
    tiles = d["tiles_in"].copy()
    info = O.chol_hrl(tiles) if "_hrl_" in name else O.chol_hll(tiles)
    assert info == int(d["info"]) == 0
    mt = tiles.shape[0]
    for j in range(mt):
        for i in range(j, mt):
            ref = d["tiles_out"][j, i].T  # stored column-major
            got = tiles[j, i].T
            if i == j:
                ref, got = np.tril(ref), np.tril(got)
            np.testing.assert_allclose(got, ref, rtol=0, atol=64 * np.finfo(float).eps * 64)


def test_schol_rl(golden_dir):
    d = load(golden_dir, "schol_rl_n96_b32")
    A = np.asfortranarray(d["A"].copy())
    info = O.schol_rl(A, 32)
    assert info == 0
    np.testing.assert_allclose(np.tril(A), np.tril(d["out"]), rtol=0,
                               atol=64 * np.finfo(np.float32).eps * np.abs(d["out"]).max())


@pytest.mark.parametrize("name", ["spdsolv_m128_r1_b32", "spdsolv_m128_r3_b32", "spdsolv_m96_r8_b48"])
def test_spdsolv(golden_dir, name):
    d = load(golden_dir, name)
    A = d["A"].copy(order="F")
    B = d["B"].copy(order="F")
    b = int(name.split("_b")[-1])
    assert O.spdsolv(A, B, b) == 0
    np.testing.assert_allclose(B, d["X"], rtol=1e-12, atol=1e-13)
    assert O.backward_error(d["A"], B, d["B"]) <= 10 * A.shape[0] * np.finfo(float).eps


@pytest.mark.parametrize("case", ["LLN", "LLT", "LUN", "LUT"])
def test_blocked_dtrsm(golden_dir, case):
    d = load(golden_dir, "dtrsm_" + case)
    M, N, bb, alpha = int(d["M"]), int(d["N"]), int(d["bb"]), float(d["alpha"])
    A = d["A"]
    B = d["B"].copy(order="F")
    Bv = B[:M, :N]
    work = np.asfortranarray(Bv.copy())
    O.ltrsm(case[1], case[2], "N", bb, alpha, np.asfortranarray(A[:M, :M]), work)
    ref = d["out"][:M, :N]
    # trsm_test.c:9-14 uses the 1-norm relative error with threshold 1e-15
    # against MKL; the oracle's loops and OpenBLAS round differently, and a
    # triangle with every entry ~100 amplifies that, so the bound here is 1e-12
    relerr = np.abs(work - ref).sum(axis=0).max() / np.abs(ref).sum(axis=0).max()
    assert relerr < 1e-12
    # rows beyond M and columns beyond N are untouched
    np.testing.assert_array_equal(d["out"][M:, :], d["B"][M:, :])


@pytest.mark.parametrize("name", ["dcg_n64_bm16_s8", "dcg_n64_bm16_s200", "dcg_n100_bm32_s300"])
def test_dcg_matches_reference_recurrence(golden_dir, name):
    d = load(golden_dir, name)
    rc, x, _ = O.cg(d["A"], d["rhs"], int(d["bm"]), float(d["tol"]), int(d["steps"]))
    assert rc == int(d["rc"])
    np.testing.assert_allclose(x, d["x"], rtol=0, atol=1e-12 * max(1.0, np.abs(d["x"]).max()))


@pytest.mark.parametrize("name", ["itref_n64_bm16", "itref_n96_bm32"])
def test_itref_loop(golden_dir, name):
    d = load(golden_dir, name)
    k, x, norms = O.itref(d["A"], d["rhs"], int(d["bm"]), float(d["prec"]), int(d["refit"]), int(d["it"]))
    logged = d["norms_logged"][:k]
    # entry 0 is sqrt(DBL_MAX) in both (the initial residual is never dotted)
    assert norms[0] == pytest.approx(logged[0], rel=1e-6)
    # the loop stops at the same outer iteration, below prec in both
    assert logged[k - 1] <= float(d["prec"]) and norms[k - 1] <= float(d["prec"])
    assert all(v > float(d["prec"]) for v in logged[:k - 1])
    assert O.backward_error(d["A"], x, d["rhs"]) <= 10 * d["A"].shape[0] * np.finfo(float).eps


def test_every_fixture_is_covered(golden_dir):
    names = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(golden_dir, "*.npz")))
    assert len(names) >= 20


@pytest.mark.skipif(not O.ref_available(), reason="reference not built here")
def test_oracle_vs_live_reference_ragged():
    """Where the reference build exists, check one fresh seeded case live."""
    A0 = O.spd_diag_dominant(77, 99)
    A1, A2 = A0.copy(order="F"), A0.copy(order="F")
    O.chol_rl(A1, 20)
    O.ref_chol("rl", A2, 20)
    np.testing.assert_allclose(np.tril(A1), np.tril(A2), rtol=0, atol=1e-12)


@pytest.mark.parametrize("case", ["LN_b", "LN_b0", "LT_b", "UN_b", "UT_b"])
def test_blocked_dsyrk(golden_dir, case):
    """The oracle's SYRK against the reference's own blocked ompss_dsyrk
    (syrk_main.c): the requested triangle, the other one untouched."""
    d = load(golden_dir, "dsyrk_" + case)
    n, k, alpha, beta = int(d["n"]), int(d["k"]), float(d["alpha"]), float(d["beta"])
    uplo, trans = case[0], case[1]
    Cm = d["C"].copy(order="F")
    O.syrk(uplo, trans, n, k, alpha, np.asfortranarray(d["A"]), beta, Cm)
    np.testing.assert_allclose(Cm, d["out"], rtol=0, atol=1e-12 * np.abs(d["out"]).max())


def test_blocked_ssyrk(golden_dir):
    """The oracle's FP32 SYRK against the reference's ompss_ssyrk: FP32 sums in a
    different order, so within FP32 rounding of the k-term dot products."""
    d = load(golden_dir, "ssyrk_LN_b")
    n, k = int(d["n"]), int(d["k"])
    Cm = d["C"].copy(order="F")
    O.syrk("L", "N", n, k, float(d["alpha"]), np.asfortranarray(d["A"]), float(d["beta"]), Cm)
    tol = 4 * k * np.finfo(np.float32).eps * np.abs(d["out"]).max()
    np.testing.assert_allclose(Cm, d["out"], rtol=0, atol=tol)


# ---------------------------------------------------------------- sparse refinement
# The reference's sparse matrix product is MKL's mkl_dcsrmv (fpsblas.h defines
# SBLAS_csrmv empty without MKL, and task_csrmm.c does not compile in the
# non-MKL configuration), so the sparse restatement is pinned piece by piece:
# its block-Jacobi against the reference's own CSparse preconditioner, and its
# recurrence against the reference's dense dcg_pure on the same matrix as CSR.
@pytest.mark.parametrize("name", ["sparse_bj_n150_bm32", "sparse_bj_n200_bm48"])
def test_oracle_block_jacobi_matches_reference(golden_dir, name):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    bm = int(d["bm"])
    rc, F = O.bj_setup(d["vptr"], d["vpos"], d["vval"], bm)
    assert rc == 0
    z = O.bj_apply(F, bm, d["r"])
    np.testing.assert_allclose(z, d["z"], rtol=1e-13, atol=1e-15 * np.abs(d["z"]).max())


@pytest.mark.parametrize("name", ["dcg_n64_bm16_s8", "dcg_n64_bm16_s200", "dcg_n100_bm32_s300"])
@pytest.mark.parametrize("base", [0, 1])
def test_oracle_sparse_cg_reproduces_reference_dense_cg(golden_dir, name, base):
    """a dense matrix given as CSR: the sparse dcg_pure takes the reference's dense iterates"""
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    vptr, vpos, vval = O.csr_from_dense(d["A"], base)
    rc, x, _ = O.scg(vptr, vpos, vval, d["rhs"], int(d["bm"]), float(d["tol"]), int(d["steps"]), False)
    assert rc == int(d["rc"])
    np.testing.assert_allclose(x, d["x"], rtol=1e-12, atol=1e-14)


def test_oracle_sparse_refinement_converges_with_block_jacobi():
    A = O.spd_sparse(300, seed=3)
    vptr, vpos, vval = O.csr_from_dense(A)
    x_true = np.random.default_rng(3).standard_normal(300)
    k, x, norms = O.sitref(vptr, vpos, vval, A @ x_true, 64, 1e-12, 10, 300, True)
    assert 1 <= k <= 10
    np.testing.assert_allclose(x, x_true, rtol=0, atol=1e-10)


def test_mm_reader_matches_scipy(tmp_path):
    """the library's MatrixMarket reader (host code, no device needed)"""
    import scipy.io
    import scipy.sparse

    import linompss_b200 as lnb
    A = O.spd_sparse(80, seed=4)
    for kind in ("symmetric", "general"):
        path = str(tmp_path / f"a_{kind}.mtx")
        M = scipy.sparse.coo_matrix(np.tril(A) if kind == "symmetric" else A)
        scipy.io.mmwrite(path, M, symmetry=kind)
        n, vptr, vpos, vval = lnb.mm_read_csr(path)
        assert n == 80
        ref = scipy.sparse.csr_matrix(scipy.io.mmread(path)).toarray()
        got = np.zeros((n, n))
        for i in range(n):
            for p in range(vptr[i], vptr[i + 1]):
                got[i, vpos[p]] += vval[p]
            assert np.all(np.diff(vpos[vptr[i]:vptr[i + 1]]) > 0)
        np.testing.assert_allclose(got, A, rtol=0, atol=1e-15)
        np.testing.assert_allclose(ref if kind == "general" else A, A)


# ---------------------------------------------------------------- LU / gensolv
@pytest.mark.parametrize("name", ["lu_m200_n200_b33", "lu_m240_n160_b64"])
def test_oracle_lu_matches_reference(golden_dir, name):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    A = d["A"].copy(order="F")
    info, ipiv = O.getrf(A, int(d["b"]))
    assert info == 0
    np.testing.assert_array_equal(ipiv, d["ipiv"])
    np.testing.assert_allclose(A, d["LU"], rtol=0, atol=1e-12 * np.abs(d["LU"]).max())


def test_oracle_gensolv_matches_reference(golden_dir):
    d = np.load(os.path.join(golden_dir, "gensolv_m128_b48.npz"))
    A, B = d["A"].copy(order="F"), d["B"].copy(order="F")
    assert O.gensolv(A, B, int(d["b"])) == 0
    np.testing.assert_allclose(A, d["LU"], rtol=0, atol=1e-12 * np.abs(d["LU"]).max())
    np.testing.assert_allclose(B, d["X"], rtol=0, atol=1e-13 * np.abs(d["X"]).max())


def test_oracle_lu_with_pivoting_matches_lapack_when_panels_align():
    """partial pivoting over every row below: the same pivots and factor as LAPACK dgetrf"""
    import scipy.linalg as sl
    A0 = np.asfortranarray(np.random.default_rng(5).standard_normal((300, 300)))
    lu, piv = sl.lu_factor(A0)
    A = A0.copy(order="F")
    info, ipiv = O.getrf(A, 50)
    assert info == 0
    np.testing.assert_array_equal(np.arange(300) // 50 * 50 + ipiv, piv + 1)
    np.testing.assert_allclose(A, lu, rtol=0, atol=1e-11)
    perm, L, U = O.lu_unpack(A, ipiv, 50)
    np.testing.assert_allclose(A0[perm], L @ U, rtol=0, atol=1e-12)


def test_oracle_lu_ragged_last_panel_quirk():
    """the reference swaps only dimC columns of the earlier blocks for a ragged last panel
    (lu_main.c TASK_LASWP(j, dimC, ...)): with pivoting there, P A != L U.  The oracle keeps it
    (it restates the reference); the library factors correctly (tests/test_gpu_lu.py)"""
    A0 = np.asfortranarray(np.random.default_rng(5).standard_normal((300, 300)))
    A = A0.copy(order="F")
    _, ipiv = O.getrf(A, 64)
    A2 = A0.copy(order="F")
    if O.ref_available():
        assert (O.ref_getrf(A2, 64) == ipiv).all()
        np.testing.assert_allclose(A, A2, rtol=0, atol=1e-12)
    perm, L, U = O.lu_unpack(A, ipiv, 64)
    assert np.abs(A0[perm] - L @ U).max() > 1.0
