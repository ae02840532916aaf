"""Batched uneven SPD solves (lnb_batched_posv_dev): many independent systems
of orders 16..512 with 1..8 right-hand sides in one persistent launch.

Bar per system: the FP64 normwise backward error <= 10 n eps, reached from an
FP32 factor by FP64 refinement (mode FP32) or directly (mode FP64); results
agree with numpy's FP64 solve.  Also: the launch is capturable in a CUDA
graph and replays to the same answer, sizes beyond the kernel's capacity are
reported per system, and the autotuner picks one of its candidates.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps / 2


@pytest.fixture(scope="module")
def lnb(cuda):
    import linompss_b200
    return linompss_b200


def make_batch(count, seed, nmin=16, nmax=512, rmax=8, delta=1e-2):
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, count)
    rs = rng.integers(1, rmax + 1, count)
    As, Bs = [], []
    for n, r in zip(ns, rs):
        G = rng.standard_normal((n, n))
        As.append(G @ G.T / n + delta * np.eye(n))
        Bs.append(rng.standard_normal((n, r)))
    return ns, rs, As, Bs


def to_device(ns, rs, As, Bs, dev):
    import torch
    a_off = np.concatenate([[0], np.cumsum(ns.astype(np.int64) ** 2)[:-1]])
    b_off = np.concatenate([[0], np.cumsum(ns.astype(np.int64) * rs)[:-1]])
    Aflat = np.concatenate([A.ravel(order="F") for A in As])
    Bflat = np.concatenate([B.ravel(order="F") for B in Bs])
    t = lambda x, dt: torch.tensor(x, dtype=dt, device=dev)
    return (t(ns.astype(np.int32), torch.int32), t(rs.astype(np.int32), torch.int32), t(a_off, torch.int64),
            t(b_off, torch.int64), t(Aflat, torch.float64), t(Bflat, torch.float64), b_off)


def check(ns, rs, As, Bs, Xflat, b_off):
    worst = 0.0
    for k, (n, r) in enumerate(zip(ns, rs)):
        X = Xflat[b_off[k]:b_off[k] + n * r].reshape(n, r, order="F")
        A, B = As[k], Bs[k]
        R = B - A @ X
        be = np.abs(R).max() / (np.abs(A).sum(axis=1).max() * np.abs(X).max() + np.abs(B).max())
        worst = max(worst, be / (n * EPS))
        # forward error vs numpy's FP64 solve, bounded by cond(A) times the backward error bar
        Xref = np.linalg.solve(A, B)
        cond = np.linalg.cond(A)
        assert np.abs(X - Xref).max() / np.abs(Xref).max() <= 4 * cond * 10 * n * EPS + 1e-15
    return worst


@pytest.mark.parametrize("mode", ["FACTOR_FP32", "FACTOR_FP64"])
def test_batched_uneven(lnb, cuda, mode):
    import torch
    ns, rs, As, Bs = make_batch(200, seed=1)
    nd, rd, ao, bo, dA, dB, b_off = to_device(ns, rs, As, Bs, cuda)
    dX = torch.zeros_like(dB)
    info = torch.full((len(ns),), -99, dtype=torch.int32, device=cuda)
    iters = torch.zeros(len(ns), dtype=torch.int32, device=cuda)
    lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, getattr(lnb, mode), 10, info, iters)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    assert check(ns, rs, As, Bs, dX.cpu().numpy(), b_off) <= 10.0
    it = iters.cpu().numpy()
    assert it.min() >= 1 and it.max() <= (10 if mode == "FACTOR_FP32" else 1)


def test_batched_edge_sizes_and_capacity(lnb, cuda):
    import torch
    ns = np.array([1, 2, 16, 17, 31, 33, 127, 129, 511, 512])
    rng = np.random.default_rng(5)
    rs = np.array([1, 8, 3, 1, 2, 8, 1, 4, 2, 1])
    As, Bs = [], []
    for n, r in zip(ns, rs):
        G = rng.standard_normal((n, n))
        As.append(G @ G.T / n + 0.1 * np.eye(n))
        Bs.append(rng.standard_normal((n, r)))
    nd, rd, ao, bo, dA, dB, b_off = to_device(ns, rs, As, Bs, cuda)
    dX = torch.zeros_like(dB)
    info = torch.full((len(ns),), -99, dtype=torch.int32, device=cuda)
    lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, info)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    assert check(ns, rs, As, Bs, dX.cpu().numpy(), b_off) <= 10.0
    # a system beyond the kernel's capacity (n > 512 or nrhs > 8) is flagged, others still solved
    nd2 = nd.clone()
    rd2 = rd.clone()
    rd2[1] = 9
    info.fill_(-99)
    lnb.batched_posv_dev(nd2, rd2, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, info)
    torch.cuda.synchronize()
    got = info.cpu().numpy()
    assert got[1] == -7 and (np.delete(got, 1) == 0).all()


@pytest.mark.parametrize("mode", ["FACTOR_FP32", "FACTOR_FP64"])
def test_batched_not_spd_reports_info(lnb, cuda, mode):
    import torch
    ns, rs, As, Bs = make_batch(20, seed=3, nmax=200)
    As[7] = As[7].copy()
    As[7][5, 5] = -1.0
    nd, rd, ao, bo, dA, dB, b_off = to_device(ns, rs, As, Bs, cuda)
    dX = torch.zeros_like(dB)
    info = torch.full((len(ns),), -99, dtype=torch.int32, device=cuda)
    lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, getattr(lnb, mode), 10, info)
    torch.cuda.synchronize()
    got = info.cpu().numpy()
    assert got[7] == 6 and (np.delete(got, 7) == 0).all()


def test_batched_graph_capture_and_autotune(lnb, cuda):
    import torch
    ns, rs, As, Bs = make_batch(300, seed=4)
    nd, rd, ao, bo, dA, dB, b_off = to_device(ns, rs, As, Bs, cuda)
    dX = torch.zeros_like(dB)
    pw = lnb.batched_autotune(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10)
    assert pw in (256, 512)
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, stream=s)   # workspace exists
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=s):
            lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, lnb.FACTOR_FP32, 10, stream=s)
    dX.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert check(ns, rs, As, Bs, dX.cpu().numpy(), b_off) <= 10.0


def test_sspdsolv_and_spotrs(lnb, cuda):
    import torch
    from oracle import oracle as O
    m, nrhs, b = 640, 3, 128
    A0 = O.spd_covariance(m, 1.0, seed=8).astype(np.float32)
    B0 = np.random.default_rng(8).standard_normal((m, nrhs)).astype(np.float32)
    A = np.asfortranarray(A0.copy())
    B = np.asfortranarray(B0.copy())
    assert lnb.sspdsolv_main(m, nrhs, b, A, B) == 0
    Xref = np.linalg.solve(A0.astype(np.float64), B0.astype(np.float64))
    assert np.abs(B - Xref).max() / np.abs(Xref).max() < 1e-4
    # device FP32 solve with the FP32 factor just computed
    Lt = torch.tensor(np.ascontiguousarray(A.T), device=cuda)
    Bt = torch.tensor(np.ascontiguousarray(B0.T), device=cuda)
    lnb.spotrs_dev(Lt, Bt, m, nrhs, "B")
    torch.cuda.synchronize()
    np.testing.assert_allclose(Bt.cpu().numpy().T, B, rtol=0, atol=1e-5 * np.abs(B).max())


@pytest.mark.parametrize("mode", ["FACTOR_FP32", "FACTOR_FP64"])
def test_batched_not_spd_at_every_panel_position(lnb, cuda, mode):
    """A non-positive pivot at the first, last and a middle column of the first,
    a middle and a ragged last 32-column panel: each system reports its own
    column (LAPACK info) and the others are solved."""
    import torch
    bad_cols = [0, 5, 31, 32, 63, 80, 95, 99]
    ns, rs, As, Bs = make_batch(len(bad_cols) + 3, seed=11, nmin=100, nmax=100)
    for k, c in enumerate(bad_cols):
        As[k] = As[k].copy()
        As[k][c, c] = -1.0
    nd, rd, ao, bo, dA, dB, b_off = to_device(ns, rs, As, Bs, cuda)
    dX = torch.zeros_like(dB)
    info = torch.full((len(ns),), -99, dtype=torch.int32, device=cuda)
    lnb.batched_posv_dev(nd, rd, ao, bo, dA, dB, dX, getattr(lnb, mode), 10, info)
    torch.cuda.synchronize()
    got = info.cpu().numpy()
    assert list(got[:len(bad_cols)]) == [c + 1 for c in bad_cols]
    assert (got[len(bad_cols):] == 0).all()
