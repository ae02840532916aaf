"""The refinement's symmetric product Y = A X (lnb_dsymv_dev) against a torch
FP64 product of the symmetrised lower triangle.  NaN fills the strict upper
triangle and the padding rows below n, so any read outside the lower
triangle shows.  Sizes cover partial 64-row tiles, odd n (the last 16-byte
copy of a column is half a row), odd lda (the strip kernel), and 1..16
right-hand sides (tensor-core passes of 8 and a tail)."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def run(lnb, n, nrhs, lda, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    At = torch.full((n, lda), float("nan"), dtype=torch.float64, device="cuda")   # column-major n x n, ld lda
    M = torch.randn(n, n, generator=g, dtype=torch.float64, device="cuda")
    L = torch.tril(M)                                                             # L[r, c], r >= c
    At[:, :n] = torch.where(torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda")), L, At[:, :n]).T
    X = torch.randn(nrhs, n, generator=g, dtype=torch.float64, device="cuda")
    Y = torch.full((nrhs, n), 7.0, dtype=torch.float64, device="cuda")
    lnb.dsymv_dev(At, X, Y, n, nrhs)
    torch.cuda.synchronize()
    S = L + torch.tril(L, -1).T
    ref = (S @ X.T).T
    scale = (S.abs() @ X.abs().T).T
    err = ((Y - ref).abs() / scale.clamp_min(1e-300)).max().item()
    return err


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 255, 256, 257, 700, 1031])
@pytest.mark.parametrize("nrhs", [1, 2, 3, 8, 9, 16])
def test_dsymv_matches_fp64(lnb, n, nrhs):
    lda = n + (n % 2)                       # even: the tensor-core path
    assert run(lnb, n, nrhs, lda, n * 31 + nrhs) < 1e-13


@pytest.mark.parametrize("n,nrhs", [(257, 8), (513, 3)])
def test_dsymv_odd_lda(lnb, n, nrhs):
    assert run(lnb, n, nrhs, n + 2 if n % 2 == 0 else n, 5) < 1e-13


def test_dsymv_large(lnb):
    assert run(lnb, 4100, 8, 4102, 9) < 1e-12


def test_dsymv_rejects_bad_lda(lnb):
    import ctypes as C
    A = torch.zeros(4, 4, dtype=torch.float64, device="cuda")
    X = torch.zeros(1, 4, dtype=torch.float64, device="cuda")
    f = lnb.lib().lnb_dsymv_dev
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    assert f(4, 1, lnb._p(A), 3, lnb._p(X), lnb._p(X), None) == lnb.LNB_EINVAL
