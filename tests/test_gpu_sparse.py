"""Sparse refinement on the GPU (ompss_dscg, ompss_dsitref: itref.c built
with USE_SPARSE), through the C ABI, against the oracle and the reference's
own dense dcg_pure outputs.

  * the dense dcg fixtures given as CSR (zero- and one-based): the device's
    sparse CG takes the reference's iterates
  * a fixed number of steps with and without the block-Jacobi preconditioner
    against the oracle's iterates (no stopping, so both run the same steps)
  * the refinement loop to convergence, ragged last block, several bm
  * a large 2D Poisson-like system (n = 40000, bm = 512) by its residual
  * a MatrixMarket file read by the library and solved
  * errors: a diagonal block that is not positive definite, bm > 512
Tolerances: FP64 dot products and CSR sums run in a different order on the
device, so iterates agree to ~1e-10 relative after tens of steps.
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


@pytest.mark.parametrize("name", ["dcg_n64_bm16_s8", "dcg_n64_bm16_s200", "dcg_n100_bm32_s300"])
@pytest.mark.parametrize("base", [0, 1])
def test_sparse_cg_matches_reference_dense_cg(lnb, golden_dir, name, base):
    d = np.load(os.path.join(golden_dir, name + ".npz"))
    n = d["A"].shape[0]
    vptr, vpos, vval = O.csr_from_dense(d["A"], base)
    x = np.zeros(n)
    rc = lnb.ompss_dscg(n, int(d["bm"]), vptr, vpos, vval, np.ascontiguousarray(d["rhs"]), x, float(d["tol"]),
                        int(d["steps"]), 0)
    assert rc == int(d["rc"])
    np.testing.assert_allclose(x, d["x"], rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("n,bm", [(300, 64), (333, 100), (257, 512)])
def test_sparse_cg_fixed_steps_vs_oracle(lnb, precond, n, bm):
    A = O.spd_sparse(n, seed=n + bm)
    vptr, vpos, vval = O.csr_from_dense(A)
    rhs = np.random.default_rng(n).standard_normal(n)
    steps = 25
    rc_o, x_o, _ = O.scg(vptr, vpos, vval, rhs, bm, 0.0, steps, bool(precond))
    x = np.zeros(n)
    rc = lnb.ompss_dscg(n, bm, vptr, vpos, vval, rhs, x, 0.0, steps, precond)
    assert rc == rc_o == steps
    np.testing.assert_allclose(x, x_o, rtol=0, atol=1e-10 * np.abs(x_o).max())


@pytest.mark.parametrize("precond", [0, 1])
@pytest.mark.parametrize("base", [0, 1])
def test_sparse_refinement_vs_oracle(lnb, precond, base):
    n, bm = 400, 96                          # ragged last block of 16
    A = O.spd_sparse(n, seed=7)
    vptr, vpos, vval = O.csr_from_dense(A, base)
    x_true = np.random.default_rng(7).standard_normal(n)
    rhs = A @ x_true
    k_o, x_o, norms_o = O.sitref(vptr, vpos, vval, rhs, bm, 1e-12, 10, n, bool(precond))
    x = np.zeros(n)
    norms = np.zeros(10)
    k = lnb.ompss_dsitref(n, bm, vptr, vpos, vval, rhs, x, 1e-12, 10, n, precond, norms)
    assert abs(k - k_o) <= 1
    np.testing.assert_allclose(x, x_true, rtol=0, atol=1e-10)
    np.testing.assert_allclose(x, x_o, rtol=0, atol=1e-10)


def poisson_csr(m, shift=0.05):
    """5-point Laplacian on an m x m grid plus shift I, zero-based CSR"""
    import scipy.sparse as sp
    T = sp.diags([-1.0, 2.0 + shift / 2, -1.0], [-1, 0, 1], shape=(m, m))
    I = sp.identity(m)
    A = (sp.kron(I, T) + sp.kron(T, I)).tocsr()
    A.sort_indices()
    return A


def test_sparse_refinement_large_poisson(lnb):
    m = 200
    A = poisson_csr(m)
    n = A.shape[0]
    x_true = np.random.default_rng(11).standard_normal(n)
    rhs = A @ x_true
    x = np.zeros(n)
    k = lnb.ompss_dsitref(n, 512, A.indptr, A.indices, A.data, rhs, x, 1e-10, 6, 3000, 1)
    assert k >= 1
    r = rhs - A @ x
    assert np.linalg.norm(r) <= 1e-9 * np.linalg.norm(rhs)


def test_sparse_from_matrix_market(lnb, tmp_path):
    import scipy.io
    import scipy.sparse
    A = O.spd_sparse(500, seed=12)
    path = str(tmp_path / "A.mtx")
    scipy.io.mmwrite(path, scipy.sparse.coo_matrix(np.tril(A)), symmetry="symmetric")
    n, vptr, vpos, vval = lnb.mm_read_csr(path)
    x_true = np.ones(n)
    rhs = A @ x_true
    x = np.zeros(n)
    k = lnb.ompss_dsitref(n, 128, vptr, vpos, vval, rhs, x, 1e-12, 8, n, 1)
    assert k >= 1
    np.testing.assert_allclose(x, x_true, rtol=0, atol=1e-10)


def test_sparse_errors(lnb):
    A = O.spd_sparse(100, seed=13)
    A[70, 70] = -5.0
    vptr, vpos, vval = O.csr_from_dense(A)
    x = np.zeros(100)
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dsitref(100, 32, vptr, vpos, vval, np.ones(100), x, 1e-12, 4, 100, 1)
    assert e.value.code == lnb.LNB_EINVAL and "block 2" in str(e.value)
    B = O.spd_sparse(100, seed=14)
    vptr, vpos, vval = O.csr_from_dense(B)
    with pytest.raises(lnb.LinompssError) as e:
        lnb.ompss_dsitref(100, 1024, vptr, vpos, vval, np.ones(100), x, 1e-12, 4, 100, 1)
    assert e.value.code == lnb.LNB_EINVAL
