"""Mixed precision: low-precision factor + FP64 refinement (lnb_dsposv_ir).

The bar is the north star's: FP64-level normwise backward error
||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 10 n eps (eps = 2^-53),
reached from an FP32 / TF32x3 / BF16 factor; the forward error against the
FP64 solution is bounded by cond(A) times that.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps / 2


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def check(lnb, A0, B0, b, factor, **kw):
    n = A0.shape[0]
    opts = lnb.ir_opts(factor=factor, **kw)
    rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    assert rc == 0, (rc, res, lnb.last_error())
    be = O.backward_error_np(A0, X, B0)
    assert be <= 10 * n * EPS, (be, res)
    assert res["backward_error"] <= 10 * n * EPS
    return X, res


@pytest.mark.parametrize("factor", ["FACTOR_TF32X3", "FACTOR_FP32", "FACTOR_BF16", "FACTOR_TF32"])
def test_ir_well_conditioned(lnb, factor):
    n, b = 2048, 256
    A0 = O.spd_covariance(n, 1e-1, seed=1)
    B0 = np.asfortranarray(np.random.default_rng(1).standard_normal((n, 1)))
    X, res = check(lnb, A0, B0, b, getattr(lnb, factor))
    Xref = np.linalg.solve(A0, B0)
    # refinement stops at an inf-norm normwise backward error <= 10 n eps, so
    # the forward error is bounded by cond_inf(A) times that (2x margin)
    bound = 2 * np.linalg.cond(A0, np.inf) * 10 * n * EPS
    assert np.abs(X - Xref).max() / np.abs(Xref).max() <= bound
    if factor in ("FACTOR_TF32X3", "FACTOR_FP32"):
        assert res["iterations"] <= 4 and not res["used_pcg"]


@pytest.mark.parametrize("delta", [1e-1, 1e-3, 1e-5])
def test_ir_tf32x3_delta_sweep(lnb, delta):
    """configs[2]'s matrix family G G^T/n + delta I at reduced n (cond ~4e1..4e5)."""
    n, b = 3072, 512
    A0 = O.spd_covariance(n, delta, seed=2)
    B0 = np.asfortranarray(np.random.default_rng(2).standard_normal((n, 1)))
    X, res = check(lnb, A0, B0, b, lnb.FACTOR_TF32X3)
    assert res["iterations"] <= 12


def test_ir_bf16_badly_scaled_multi_rhs(lnb):
    """configs[3]'s family D (G G^T/n + delta I) D, D = diag(10^u), u ~ U[-2,2],
    8 right-hand sides, at reduced n; BF16 factor + equilibration + PCG fallback."""
    n, b, nrhs = 2048, 512, 8
    rng = np.random.default_rng(3)
    D = 10.0 ** rng.uniform(-2, 2, n)
    A0 = O.fortran(D[:, None] * O.spd_covariance(n, 1e-4, seed=3) * D[None, :])
    B0 = np.asfortranarray(rng.standard_normal((n, nrhs)))
    X, res = check(lnb, A0, B0, b, lnb.FACTOR_BF16, max_iter=40, pcg_max_iter=400)


def test_ir_bf16_without_equilibration_still_refines(lnb):
    n, b = 1024, 256
    A0 = O.spd_covariance(n, 1e-2, seed=4)
    B0 = np.asfortranarray(np.random.default_rng(4).standard_normal((n, 2)))
    check(lnb, A0, B0, b, lnb.FACTOR_BF16, equilibrate=0, max_iter=40)


def test_ir_pcg_fallback_triggers(lnb):
    """A BF16 factor of a cond ~4e5 matrix cannot refine plainly (cond * u_bf16 >> 1):
    the stall detector must switch to PCG, which then converges."""
    n, b = 2048, 256
    A0 = O.spd_covariance(n, 1e-5, seed=5)
    B0 = np.asfortranarray(np.random.default_rng(5).standard_normal((n, 1)))
    X, res = check(lnb, A0, B0, b, lnb.FACTOR_BF16, max_iter=30, pcg_max_iter=800)
    assert res["used_pcg"] == 1 and res["pcg_iterations"] > 0


def test_ir_reports_noconv_when_disallowed(lnb):
    n, b = 1024, 256
    A0 = O.spd_covariance(n, 1e-6, seed=6)
    B0 = np.asfortranarray(np.random.default_rng(6).standard_normal((n, 1)))
    opts = lnb.ir_opts(factor=lnb.FACTOR_BF16, allow_pcg=0, max_iter=3)
    rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    assert rc == lnb.LNB_ENOCONV
    assert res["iterations"] == 3 and res["backward_error"] > 10 * n * EPS


def test_ir_device_api_leaves_A_untouched(lnb, cuda):
    import torch
    n, b, nrhs = 1536, 256, 3
    A0 = O.spd_covariance(n, 1e-2, seed=7)
    B0 = np.random.default_rng(7).standard_normal((n, nrhs))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    Xt = torch.zeros_like(Bt)
    A_before = At.clone()
    rc, res = lnb.dsposv_ir_dev(At, Bt, Xt, n, nrhs, b, lnb.ir_opts(factor=lnb.FACTOR_TF32X3))
    torch.cuda.synchronize()
    assert rc == 0
    assert torch.equal(At, A_before)
    X = Xt.cpu().numpy().T
    assert O.backward_error_np(A0, X, B0) <= 10 * n * EPS
    assert res["factor_ms"] > 0 and res["solve_ms"] > 0


@pytest.mark.parametrize("ahead", [None, "0", "1"])
@pytest.mark.parametrize("factor,n,b", [("FACTOR_TF32X3", 6000, 512), ("FACTOR_TF32", 3000, 256)])
def test_ir_streamed_host_path(lnb, cuda, monkeypatch, ahead, factor, n, b):
    """The host entry point factors while A is still arriving: block columns
    join the right-looking schedule through a catch-up update with every
    finished panel.  LNB_STREAM_AHEAD = 0 forces a catch-up at every step (K
    growing to n), 1 a mix; unset, columns join as soon as they land.  Every
    variant refines to the FP64 bar and agrees with the device entry point."""
    import torch
    if ahead is None:
        monkeypatch.delenv("LNB_STREAM_AHEAD", raising=False)
    else:
        monkeypatch.setenv("LNB_STREAM_AHEAD", ahead)
    A0 = O.spd_covariance(n, 1e-3, seed=n)
    B0 = np.asfortranarray(np.random.default_rng(n).standard_normal((n, 2)))
    X, res = check(lnb, A0, B0, b, getattr(lnb, factor))
    assert not res["used_pcg"] and res["refactored_tiles"] == 0
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    Xt = torch.zeros_like(Bt)
    rc, res_d = lnb.dsposv_ir_dev(At, Bt, Xt, n, 2, b, lnb.ir_opts(factor=getattr(lnb, factor)))
    torch.cuda.synchronize()
    assert rc == 0
    Xd = Xt.cpu().numpy().T
    bound = 2 * np.linalg.cond(A0, np.inf) * 10 * n * EPS
    assert np.abs(X - Xd).max() / np.abs(Xd).max() <= 2 * bound
    assert abs(res["iterations"] - res_d["iterations"]) <= 1


def near_singular_pair(n, i, eps):
    """I with the 2 x 2 principal block [[1, 1 - eps], [1 - eps, 1]] at (i, i):
    SPD (eigenvalues eps and 2 - eps), but 1 - eps rounds to 1 in FP32, so the
    low-precision pivot of row i + 1 is exactly zero."""
    A = np.eye(n)
    A[i, i + 1] = A[i + 1, i] = 1.0 - eps
    return np.asfortranarray(A)


@pytest.mark.parametrize("api", ["host", "device"])
def test_ir_fp64_refactor_of_failed_tile(lnb, cuda, api):
    """A low-precision pivot that fails on an SPD matrix: the diagonal tile is
    rebuilt in FP64 from the original matrix and refactored, and the solve
    still reaches the FP64 bar (with the PCG fallback if refinement stalls)."""
    import torch
    n, b = 1024, 256
    A0 = near_singular_pair(n, 300, 1e-9)
    B0 = np.asfortranarray(np.random.default_rng(8).standard_normal((n, 1)))
    opts = lnb.ir_opts(factor=lnb.FACTOR_TF32X3, max_iter=10, pcg_max_iter=100)
    if api == "host":
        rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    else:
        At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
        Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
        Xt = torch.zeros_like(Bt)
        rc, res = lnb.dsposv_ir_dev(At, Bt, Xt, n, 1, b, opts)
        torch.cuda.synchronize()
        X = Xt.cpu().numpy().T
    assert rc == 0, (rc, res, lnb.last_error())
    assert res["refactored_tiles"] >= 1
    assert O.backward_error_np(A0, X, B0) <= 10 * n * EPS


@pytest.mark.parametrize("depth", ["1", "2", "3"])
def test_ir_device_path_panel_grouping(lnb, cuda, monkeypatch, depth):
    """The device entry point keeps every panel's operand copies, so columns
    beyond the look-ahead can take their panels `depth` at a time (one update
    with K = depth * b, LNB_UPD_DEPTH).  Every grouping refines to the FP64 bar
    in the same number of iterations, give or take one."""
    import torch
    monkeypatch.setenv("LNB_UPD_DEPTH", depth)
    n, b, nrhs = 5120, 512, 2
    A0 = O.spd_covariance(n, 1e-3, seed=31)
    B0 = np.random.default_rng(31).standard_normal((n, nrhs))
    At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    Xt = torch.zeros_like(Bt)
    rc, res = lnb.dsposv_ir_dev(At, Bt, Xt, n, nrhs, b, lnb.ir_opts(factor=lnb.FACTOR_TF32X3))
    torch.cuda.synchronize()
    assert rc == 0, (res, lnb.last_error())
    assert O.backward_error_np(A0, Xt.cpu().numpy().T, B0) <= 10 * n * EPS
    assert res["iterations"] <= 4 and not res["used_pcg"]


@pytest.mark.parametrize("api,n", [("host", 2048), ("host", 1999), ("device", 2048), ("device", 1999)])
def test_ir_reported_backward_error(lnb, cuda, api, n):
    """The backward error the solver reports after one refinement step equals
    the oracle's on the returned X: ||A||_inf comes from the row sums of |A|
    that the FP32 conversion accumulates (both triangles of the symmetric A
    from its lower one), on the streamed host path and the device path, with
    an even and an odd leading dimension.  After one step the residual is far
    above its rounding noise, so the two agree to ~1e-8 relative."""
    import torch
    b = 256
    rng = np.random.default_rng(n + 40)
    d = 10.0 ** rng.uniform(-1, 1, n)
    A0 = np.asfortranarray(O.spd_covariance(n, 1e-2, seed=n) * d[:, None] * d[None, :])
    B0 = np.asfortranarray(rng.standard_normal((n, 1)))   # one column: the oracle's max is over all
    opts = lnb.ir_opts(factor=lnb.FACTOR_TF32X3, max_iter=1, allow_pcg=0)
    if api == "host":
        rc, X, res = lnb.dsposv_ir(A0.copy(order="F"), B0, b, opts)
    else:
        At = torch.tensor(np.ascontiguousarray(A0.T), device=cuda)
        Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
        Xt = torch.zeros_like(Bt)
        rc, res = lnb.dsposv_ir_dev(At, Bt, Xt, n, 1, b, opts)
        torch.cuda.synchronize()
        X = Xt.cpu().numpy().T
    assert rc in (0, lnb.LNB_ENOCONV), (rc, lnb.last_error())
    be = O.backward_error_np(A0, X, B0)
    assert be > 1e3 * n * EPS, be          # far from the rounding level of the residual
    assert abs(res["backward_error"] - be) <= 1e-6 * be, (res["backward_error"], be)
