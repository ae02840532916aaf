"""ctypes bindings for the CPU oracle (oracle/liboracle.so) and the reference
build (oracle/_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product package never
imports this module.

All matrices are numpy float64 arrays in column-major (Fortran) order, as the
reference stores them.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = None
_REF = None

_i64 = C.c_int64
_dp = C.POINTER(C.c_double)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def lib():
    """The C restatement (built by `make -C oracle`)."""
    global _ORC
    if _ORC is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
        _ORC = C.CDLL(path)
        for name in ("orc_chol_residual", "orc_backward_error"):
            getattr(_ORC, name).restype = C.c_double
    return _ORC


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libref.so"))


def ref():
    """The reference compiled from its own sources (built by `make -C oracle ref`)."""
    global _REF
    if _REF is None:
        _REF = C.CDLL(os.path.join(_HERE, "_ref", "libref.so"))
    return _REF


def fortran(a) -> np.ndarray:
    return np.asfortranarray(np.array(a, dtype=np.float64, copy=True))


# --------------------------------------------------------------------------
# seeded inputs with the shapes/distributions of the reference's generators
# --------------------------------------------------------------------------
def spd_diag_dominant(n: int, seed: int = 0) -> np.ndarray:
    """A = (R + R^T)/2 + n I with R ~ U[0,1): the distribution of dgenmat_spd
    (genmat.c:49-70, symmetric U[0,1) plus n on the diagonal)."""
    rng = np.random.default_rng(seed)
    R = rng.random((n, n))
    return fortran((R + R.T) / 2 + n * np.eye(n))


def spd_covariance(n: int, delta: float, seed: int = 0) -> np.ndarray:
    """A = G G^T / n + delta I with G ~ N(0,1)."""
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((n, n))
    return fortran(G @ G.T / n + delta * np.eye(n))


# --------------------------------------------------------------------------
# oracle wrappers (operate in place, return info / codes like the reference)
# --------------------------------------------------------------------------
def chol_rl(A: np.ndarray, b: int) -> int:
    n = A.shape[0]
    return lib().orc_dchol_rl(_i64(n), _i64(b), _ptr(A), _i64(A.shape[0]))


def chol_ll(A: np.ndarray, b: int) -> int:
    n = A.shape[0]
    return lib().orc_dchol_ll(_i64(n), _i64(b), _ptr(A), _i64(A.shape[0]))


def schol_rl(A: np.ndarray, b: int) -> int:
    n = A.shape[0]
    return lib().orc_schol_rl(_i64(n), _i64(b), _ptr(A), _i64(A.shape[0]))


def _tile_table(tiles: np.ndarray):
    """tiles: (mt, mt, b, b) array, tiles[j, i] is tile (i, j) stored column-major."""
    mt = tiles.shape[0]
    arr = (C.c_void_p * (mt * mt))()
    for j in range(mt):
        for i in range(mt):
            arr[j * mt + i] = tiles[j, i].ctypes.data
    return arr


def chol_hrl(tiles: np.ndarray) -> int:
    mt, b = tiles.shape[0], tiles.shape[2]
    return lib().orc_dchol_hrl(_i64(mt), _i64(b), _tile_table(tiles))


def chol_hll(tiles: np.ndarray) -> int:
    mt, b = tiles.shape[0], tiles.shape[2]
    return lib().orc_dchol_hll(_i64(mt), _i64(b), _tile_table(tiles))


def ltrsm(uplo: str, trans: str, diag: str, bm: int, alpha: float, A: np.ndarray,
          B: np.ndarray) -> None:
    m, n = B.shape
    lib().orc_dltrsm(C.c_char(uplo.encode()), C.c_char(trans.encode()), C.c_char(diag.encode()),
                     _i64(bm), _i64(m), _i64(n), C.c_double(alpha), _ptr(A), _i64(A.shape[0]),
                     _ptr(B), _i64(B.shape[0]))


def syrk(uplo: str, trans: str, n: int, k: int, alpha: float, A: np.ndarray, beta: float, Cm: np.ndarray) -> None:
    """Cm = alpha op(A) op(A)^T + beta Cm on triangle `uplo` (orc_dsyrk, or orc_ssyrk for FP32), in place"""
    single = Cm.dtype == np.float32
    f = lib().orc_ssyrk if single else lib().orc_dsyrk
    T = C.c_float if single else C.c_double
    f(C.c_char(uplo.encode()), C.c_char(trans.encode()), _i64(n), _i64(k), T(alpha), _ptr(A), _i64(A.shape[0]),
      T(beta), _ptr(Cm), _i64(Cm.shape[0]))


def spdsolv(A: np.ndarray, B: np.ndarray, b: int) -> int:
    m, nrhs = B.shape
    return lib().orc_dspdsolv(_i64(m), _i64(nrhs), _i64(b), _ptr(A), _ptr(B))


def getrf(A: np.ndarray, b: int):
    """dlu_main restated (orc_dgetrf), A (m x n, m >= n, column-major) in place; returns (info, ipiv) with
    the reference's pivots: 1-based, relative to the first row of each b-wide panel"""
    m, n = A.shape
    ipiv = np.zeros(max(m, n), dtype=np.int32)
    info = lib().orc_dgetrf(_i64(m), _i64(n), _i64(b), _ptr(A), _i64(m), ipiv.ctypes.data_as(C.c_void_p))
    return info, ipiv[:min(m, n)]


def gensolv(A: np.ndarray, B: np.ndarray, b: int) -> int:
    """dgensolv_main restated (orc_dgensolv): A -> LU, B -> X, in place"""
    m, n = B.shape
    return lib().orc_dgensolv(_i64(m), _i64(n), _i64(b), _ptr(A), _ptr(B))


def genmat_ip(m: int, n: int, seed: int, scale: float = 100.0) -> np.ndarray:
    """GENMAT_IP (genmat.c:131-144) with a seeded generator: uniform [0, 1) entries plus `scale` on the
    diagonal, the distribution of the reference's LU and gensolv programs"""
    A = np.random.default_rng(seed).random((m, n))
    k = min(m, n)
    A[np.arange(k), np.arange(k)] += scale
    return np.asfortranarray(A)


def lu_unpack(LU: np.ndarray, ipiv_local: np.ndarray, b: int):
    """(P, L, U) with P A = L U from a getrf result in the reference's pivot convention"""
    m, n = LU.shape
    k = min(m, n)
    perm = np.arange(m)
    for i in range(k):
        p = (i // b) * b + int(ipiv_local[i]) - 1
        perm[[i, p]] = perm[[p, i]]
    L = np.tril(LU[:, :k], -1) + np.eye(m, k)
    U = np.triu(LU[:k, :])
    return perm, L, U


def cg(A: np.ndarray, rhs: np.ndarray, bm: int, tol: float, steps: int):
    n = A.shape[0]
    x = np.zeros(n)
    log = np.zeros(max(steps, 1))
    rc = lib().orc_dcg(_i64(n), _i64(bm), _ptr(A), _i64(n), _ptr(rhs), _ptr(x),
                       C.c_double(tol), C.c_int(steps), _ptr(log))
    return rc, x, log


def itref(A: np.ndarray, rhs: np.ndarray, bm: int, prec: float, refit: int, it: int):
    n = A.shape[0]
    x = np.zeros(n)
    norms = np.zeros(max(refit, 1))
    k = lib().orc_ditref(_i64(n), _i64(bm), _ptr(A), _ptr(rhs), _ptr(x), C.c_double(prec),
                         C.c_int(refit), C.c_int(it), _ptr(norms))
    return k, x, norms[:k]


def chol_residual(A0: np.ndarray, L: np.ndarray) -> float:
    n = A0.shape[0]
    return lib().orc_chol_residual(_i64(n), _ptr(A0), _i64(A0.shape[0]), _ptr(L), _i64(L.shape[0]))


def backward_error(A: np.ndarray, X: np.ndarray, B: np.ndarray) -> float:
    n = A.shape[0]
    X = fortran(X.reshape(n, -1))
    B = fortran(B.reshape(n, -1))
    return lib().orc_backward_error(_i64(n), _i64(X.shape[1]), _ptr(A), _i64(n), _ptr(X), _i64(n),
                                    _ptr(B), _i64(n))


# numpy helpers for big cases (vectorised, same definitions as above)
def chol_residual_np(A0: np.ndarray, L: np.ndarray) -> float:
    n = A0.shape[0]
    Lt = np.tril(L)
    R = Lt @ Lt.T - A0
    return float(np.abs(R).sum(axis=1).max() / (np.abs(A0).sum(axis=1).max() * n * np.finfo(float).eps / 2))


def backward_error_np(A: np.ndarray, X: np.ndarray, B: np.ndarray) -> float:
    X = X.reshape(A.shape[0], -1)
    B = B.reshape(A.shape[0], -1)
    R = B - A @ X
    return float(np.abs(R).max() / (np.abs(A).sum(axis=1).max() * np.abs(X).max() + np.abs(B).max()))


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref/libref.so)
# --------------------------------------------------------------------------
class _OmpssBlas(C.Union):
    """ompssblas_t (fpmatr.h:14-17), non-MKL form: .s points at "L"/"R"/"T"/..."""
    _fields_ = [("e", C.c_int), ("s", C.c_char_p)]


_KEEP = {}


def ref_opt(ch: str) -> _OmpssBlas:
    if ch not in _KEEP:
        _KEEP[ch] = C.c_char_p(ch.encode())
    u = _OmpssBlas()
    u.s = _KEEP[ch].value
    return u


def ref_chol(variant: str, A: np.ndarray, b: int) -> int:
    f = getattr(ref(), "ompss_dchol_" + variant)
    n = A.shape[0]
    return f(C.c_int(n), C.c_int(b), C.c_int(b), _ptr(A), C.c_int(A.shape[0]))


def ref_chol_h(variant: str, tiles: np.ndarray) -> int:
    f = getattr(ref(), "ompss_dchol_" + variant)
    mt, b = tiles.shape[0], tiles.shape[2]
    return f(C.c_int(mt), C.c_int(b), C.c_int(b), _tile_table(tiles))


def ref_spdsolv(A: np.ndarray, B: np.ndarray, b: int) -> int:
    m, nrhs = B.shape
    return ref().dspdsolv_main(C.c_int(m), C.c_int(nrhs), C.c_int(b), _ptr(A), _ptr(B))


def ref_getrf(A: np.ndarray, b: int, single: bool = False) -> np.ndarray:
    """the reference's ompss_dgetrf / ompss_sgetrf (dlu_main), A in place; returns its IPIV"""
    m, n = A.shape
    ipiv = np.zeros(max(m, n), dtype=np.int32)
    f = ref().ompss_sgetrf if single else ref().ompss_dgetrf
    f(C.c_int(m), C.c_int(n), C.c_int(b), _ptr(A), C.c_int(m), ipiv.ctypes.data_as(C.c_void_p))
    return ipiv[:min(m, n)]


def ref_gensolv(A: np.ndarray, B: np.ndarray, b: int, single: bool = False) -> None:
    """the reference's dgensolv_main / sgensolv_main: A -> LU, B -> X (B has as many columns as A rows:
    its IPIV is allocated with the column count)"""
    m, n = B.shape
    f = ref().sgensolv_main if single else ref().dgensolv_main
    f(C.c_int(m), C.c_int(n), C.c_int(b), _ptr(A), _ptr(B))


def ref_dtrsm(side, uplo, trans, diag, m, n, b, alpha, A, lda, B, ldb) -> None:
    f = ref().ompss_dtrsm
    f.argtypes = [_OmpssBlas] * 4 + [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                                     C.c_void_p, C.c_int]
    f(ref_opt(side), ref_opt(uplo), ref_opt(trans), ref_opt(diag), m, n, b, alpha,
      _ptr(A), lda, _ptr(B), ldb)


def ref_dsyrk(uplo, trans, b, n, k, alpha, A, lda, beta, Cm, ldc) -> None:
    """the reference's own blocked ompss_dsyrk (syrk_main.c), Cm updated in place"""
    f = ref().ompss_dsyrk
    f.argtypes = [_OmpssBlas] * 2 + [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_double,
                                     C.c_void_p, C.c_int]
    f(ref_opt(uplo), ref_opt(trans), b, n, k, alpha, _ptr(A), lda, beta, _ptr(Cm), ldc)


def ref_ssyrk(uplo, trans, b, n, k, alpha, A, lda, beta, Cm, ldc) -> None:
    """the reference's own blocked ompss_ssyrk (syrk_main.c, FP32), Cm updated in place"""
    f = ref().ompss_ssyrk
    f.argtypes = [_OmpssBlas] * 2 + [C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int, C.c_float,
                                     C.c_void_p, C.c_int]
    f(ref_opt(uplo), ref_opt(trans), b, n, k, alpha, _ptr(A), lda, beta, _ptr(Cm), ldc)


def ref_cg(A: np.ndarray, rhs: np.ndarray, bm: int, tol: float, steps: int):
    n = A.shape[0]
    x = np.zeros(n)
    rc = ref().lnbref_dcg(C.c_int(n), C.c_int(bm), _ptr(A), _ptr(np.ascontiguousarray(rhs)),
                          _ptr(x), C.c_double(tol), C.c_int(steps))
    return rc, x


# --------------------------------------------------------------------------
# sparse refinement (itref.c built with USE_SPARSE); CSR with base = vptr[0]
# --------------------------------------------------------------------------
def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def csr_from_dense(A: np.ndarray, base: int = 0):
    """CSR (vptr, vpos, vval) of the nonzeros of A, rows in order, columns
    ascending within a row; base 0 or 1 (the reference's one2zero offset)."""
    n = A.shape[0]
    vptr, vpos, vval = [base], [], []
    for i in range(n):
        cols = np.nonzero(A[i])[0]
        vpos.extend(cols + base)
        vval.extend(A[i, cols])
        vptr.append(vptr[-1] + len(cols))
    return _i32(vptr), _i32(vpos), np.ascontiguousarray(vval, dtype=np.float64)


def csrmv(vptr, vpos, vval, x, alpha=1.0, beta=0.0, y=None):
    n = len(vptr) - 1
    y = np.zeros(n) if y is None else np.ascontiguousarray(y, dtype=np.float64).copy()
    x = np.ascontiguousarray(x, dtype=np.float64)
    lib().orc_csrmv(_i64(n), C.c_int(int(vptr[0])), _ptr(vptr), _ptr(vpos), _ptr(vval), _ptr(x),
                    C.c_double(alpha), C.c_double(beta), _ptr(y))
    return y


def bj_setup(vptr, vpos, vval, bm: int):
    """block-Jacobi factors (n/bm blocks of bm x bm, column-major); returns (rc, F)"""
    n = len(vptr) - 1
    nblk = (n + bm - 1) // bm
    F = np.zeros(nblk * bm * bm)
    rc = lib().orc_bj_setup(_i64(n), _i64(bm), C.c_int(int(vptr[0])), _ptr(vptr), _ptr(vpos), _ptr(vval), _ptr(F))
    return rc, F


def bj_apply(F, bm: int, r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.zeros_like(r)
    lib().orc_bj_apply(_i64(len(r)), _i64(bm), _ptr(F), _ptr(r), _ptr(z))
    return z


def scg(vptr, vpos, vval, rhs, bm: int, tol: float, steps: int, precond: bool):
    n = len(vptr) - 1
    F = bj_setup(vptr, vpos, vval, bm)[1] if precond else None
    x = np.zeros(n)
    log = np.zeros(max(steps, 1))
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    rc = lib().orc_dscg(_i64(n), _i64(bm), C.c_int(int(vptr[0])), _ptr(vptr), _ptr(vpos), _ptr(vval),
                        _ptr(F) if F is not None else None, _ptr(rhs), _ptr(x), C.c_double(tol), C.c_int(steps),
                        _ptr(log))
    return rc, x, log


def sitref(vptr, vpos, vval, rhs, bm: int, prec: float, refit: int, it: int, precond: bool):
    n = len(vptr) - 1
    F = bj_setup(vptr, vpos, vval, bm)[1] if precond else None
    x = np.zeros(n)
    norms = np.zeros(max(refit, 1))
    rhs = np.ascontiguousarray(rhs, dtype=np.float64)
    k = lib().orc_dsitref(_i64(n), _i64(bm), C.c_int(int(vptr[0])), _ptr(vptr), _ptr(vpos), _ptr(vval),
                          _ptr(F) if F is not None else None, _ptr(rhs), _ptr(x), C.c_double(prec), C.c_int(refit),
                          C.c_int(it), _ptr(norms))
    return k, x, norms[:k]


def ref_bj_apply(vptr, vpos, vval, bm: int, r):
    """the reference's own block-Jacobi preconditioner (CSparse, itref_setup.c:55-93)
    applied to r; zero-based CSR.  Returns (rc, z)."""
    n = len(vptr) - 1
    vptr, vpos = _i32(vptr).copy(), _i32(vpos).copy()
    vval = np.ascontiguousarray(vval, dtype=np.float64).copy()
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.zeros(n)
    rc = ref().lnbref_bj_apply(C.c_int(n), C.c_int(bm), _ptr(vptr), _ptr(vpos), _ptr(vval), _ptr(r), _ptr(z))
    return rc, z


def spd_sparse(n: int, seed: int = 0, density: float = 0.02, shift: float = 1.0) -> np.ndarray:
    """a sparse SPD test matrix: the 5-point Laplacian of a near-square grid plus
    a symmetric random sparse perturbation, made diagonally dominant"""
    rng = np.random.default_rng(seed)
    m = int(np.ceil(np.sqrt(n)))
    A = np.zeros((n, n))
    for i in range(n):
        A[i, i] = 4.0
        for j in (i - 1, i + 1, i - m, i + m):
            if 0 <= j < n and (abs(i - j) != 1 or (i // m) == (j // m)):
                A[i, j] = -1.0
    R = (rng.random((n, n)) < density) * rng.uniform(-0.5, 0.5, (n, n))
    R = np.triu(R, 1)
    A += R + R.T
    A[np.diag_indices(n)] += np.abs(A).sum(axis=1) - np.abs(np.diag(A)) + shift - np.diag(A) + 4.0
    return A
