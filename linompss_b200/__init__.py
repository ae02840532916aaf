"""linompss_b200 -- B200 (sm_100a) tiled SPD solve with the Linompss C interface.

The product is the shared library ``liblinompss_b200.so`` (C host code plus
sm_100a CUDA kernels) whose C ABI is ``include/linompss_b200.h``.  This module
is a thin ctypes binding over that ABI, mirroring the reference's entry points
(same names, argument meaning and return codes) for Python callers and for
the tests:

  * host (numpy, column-major) forms: ``ompss_dchol_rl``, ``ompss_dchol_ll``,
    ``ompss_dchol_hrl``, ``ompss_dchol_hll``, ``dspdsolv_main``, ``ompss_dtrsm``,
    ``task_dpotrf``/``task_dtrsm``/``task_dsyrk``/``task_dgemm``, ``ompss_dcg``,
    ``ompss_ditref``;
  * device (torch CUDA tensor) forms: ``dchol_dev``, ``dpotrs_dev``, ``dposv_dev``,
    ``dtrsm_dev`` and the mixed-precision / batched solvers.

There is no CPU fallback: if the library is missing, importing the binding
raises, and on a machine without an sm_100 GPU every call returns LNB_ENODEV.

Device matrices are column-major like the reference's: an n x n matrix with
leading dimension ld is held in a torch tensor ``At`` of shape (n, ld) whose
row j is column j (i.e. ``At = A.T`` stored contiguously).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblinompss_b200.so")

LNB_OK, LNB_EINVAL, LNB_ENODEV, LNB_ECUDA, LNB_ENOMEM, LNB_ETIMEOUT, LNB_ENOCONV, LNB_ETOOBIG = (
    0, -1, -2, -3, -4, -5, -6, -7)
FACTOR_FP64, FACTOR_FP32, FACTOR_TF32X3, FACTOR_BF16, FACTOR_TF32 = 0, 1, 2, 3, 4
SCHED_AUTO, SCHED_STREAMS, SCHED_DAG = 0, 1, 2


class LinompssError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib() -> C.CDLL:
    """Load the in-tree library; raise loudly if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built: run `make -C linompss_b200/csrc` "
                              "(or __graft_entry__.build())")
        _lib = C.CDLL(LIB_PATH)
        _lib.lnb_last_error.restype = C.c_char_p
        _lib.lnb_version.restype = C.c_char_p
    return _lib


def last_error() -> str:
    return lib().lnb_last_error().decode()


def _chk(rc: int) -> int:
    """negative return codes are LNB_E* errors"""
    if rc < 0:
        raise LinompssError(rc, last_error())
    return rc


def _p(a) -> C.c_void_p:
    if a is None:
        return C.c_void_p(0)
    if isinstance(a, np.ndarray):
        return C.c_void_p(a.ctypes.data)
    return C.c_void_p(a.data_ptr())  # torch tensor


def _colmajor(A: np.ndarray, dtype=np.float64):
    if A.dtype != dtype or not A.flags.f_contiguous:
        raise ValueError("matrix must be a Fortran-ordered (column-major) %s array" % np.dtype(dtype).name)
    return A


# --------------------------------------------------------------------------
# ompssblas_t (fpmatr.h:14-17), non-MKL form
# --------------------------------------------------------------------------
class ompssblas_t(C.Union):
    _fields_ = [("e", C.c_int), ("s", C.c_char_p)]


_OPT_STRINGS = {}


def opt(ch: str) -> ompssblas_t:
    """OMPSSBLAS_* descriptor whose .s starts with `ch` ('L','R','U','N','T')."""
    if ch not in _OPT_STRINGS:
        _OPT_STRINGS[ch] = C.create_string_buffer(ch.encode())
    u = ompssblas_t()
    u.s = C.cast(_OPT_STRINGS[ch], C.c_char_p)
    return u


# --------------------------------------------------------------------------
# host entry points (numpy, in place, like the reference)
# --------------------------------------------------------------------------
def ompss_dchol_rl(n: int, b: int, t: int, A: np.ndarray, lda: int) -> int:
    _colmajor(A)
    return _chk(lib().ompss_dchol_rl(C.c_int(n), C.c_int(b), C.c_int(t), _p(A), C.c_int(lda)))


def ompss_dchol_ll(n: int, b: int, t: int, A: np.ndarray, lda: int) -> int:
    _colmajor(A)
    return _chk(lib().ompss_dchol_ll(C.c_int(n), C.c_int(b), C.c_int(t), _p(A), C.c_int(lda)))


def _tile_table(tiles):
    mt = tiles.shape[0]
    arr = (C.c_void_p * (mt * mt))()
    for j in range(mt):
        for i in range(mt):
            arr[j * mt + i] = tiles[j, i].ctypes.data
    return arr


def ompss_dchol_hrl(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    """tiles: (mt, mt, b, b) C-ordered array; tiles[j, i] is tile (i, j) column-major."""
    return _chk(lib().ompss_dchol_hrl(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def ompss_dchol_hll(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    return _chk(lib().ompss_dchol_hll(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def ompss_dchol_nhrl(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    return _chk(lib().ompss_dchol_nhrl(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def ompss_dchol_nhll(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    return _chk(lib().ompss_dchol_nhll(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def set_factor_mode(mode: int) -> None:
    """Update path of the FP32 factorizations: FACTOR_FP32, FACTOR_TF32X3, FACTOR_TF32, FACTOR_BF16."""
    lib().lnb_set_factor_mode(C.c_int(mode))


def ompss_schol_rl(n: int, b: int, t: int, A: np.ndarray, lda: int) -> int:
    _colmajor(A, np.float32)
    return _chk(lib().ompss_schol_rl(C.c_int(n), C.c_int(b), C.c_int(t), _p(A), C.c_int(lda)))


def ompss_schol_ll(n: int, b: int, t: int, A: np.ndarray, lda: int) -> int:
    _colmajor(A, np.float32)
    return _chk(lib().ompss_schol_ll(C.c_int(n), C.c_int(b), C.c_int(t), _p(A), C.c_int(lda)))


def ompss_schol_hrl(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    return _chk(lib().ompss_schol_hrl(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def ompss_schol_hll(mt: int, b: int, t: int, tiles: np.ndarray) -> int:
    return _chk(lib().ompss_schol_hll(C.c_int(mt), C.c_int(b), C.c_int(t), _tile_table(tiles)))


def schol_dev(At, n: int, b: int, info=None, stream=None) -> int:
    return _chk(lib().lnb_schol_dev(C.c_int(n), C.c_int(b), _p(At), C.c_int(_ld(At)), _p(info), _stream(stream)))


def dspdsolv_main(m: int, n: int, b: int, A: np.ndarray, B: np.ndarray) -> int:
    _colmajor(A)
    _colmajor(B)
    return _chk(lib().dspdsolv_main(C.c_int(m), C.c_int(n), C.c_int(b), _p(A), _p(B)))


def ompss_dtrsm(side, uplo, trans, diag, m, n, b, alpha, A, lda, B, ldb) -> int:
    f = lib().ompss_dtrsm
    f.argtypes = [ompssblas_t] * 4 + [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_int]
    return _chk(f(opt(side), opt(uplo), opt(trans), opt(diag), m, n, b, alpha, _p(A), lda, _p(B), ldb))


def ompss_dsyrk(uplo, trans, b, n, k, alpha, A, lda, Cm, ldc, beta=1.0) -> int:
    """Cm = alpha op(A) op(A)^T + beta Cm on the triangle `uplo` of Cm (in place)."""
    _colmajor(A)
    _colmajor(Cm)
    f = lib().ompss_dsyrk
    f.argtypes = [ompssblas_t, ompssblas_t, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                  C.c_double, C.c_void_p, C.c_int]
    return _chk(f(opt(uplo), opt(trans), b, n, k, alpha, _p(A), lda, beta, _p(Cm), ldc))


def ompss_ssyrk(uplo, trans, b, n, k, alpha, A, lda, Cm, ldc, beta=1.0) -> int:
    _colmajor(A, np.float32)
    _colmajor(Cm, np.float32)
    f = lib().ompss_ssyrk
    f.argtypes = [ompssblas_t, ompssblas_t, C.c_int, C.c_int, C.c_int, C.c_float, C.c_void_p, C.c_int,
                  C.c_float, C.c_void_p, C.c_int]
    return _chk(f(opt(uplo), opt(trans), b, n, k, alpha, _p(A), lda, beta, _p(Cm), ldc))


def task_dpotrf(uplo: str, n: int, A: np.ndarray, lda: int, p: int = 0) -> int:
    f = lib().task_dpotrf
    f.argtypes = [ompssblas_t, C.c_int, C.c_void_p, C.c_int, C.c_int]
    return _chk(f(opt(uplo), n, _p(A), lda, p))


def task_dtrsm(side, uplo, trans, diag, bm, bn, alpha, A, lda, B, ldb, p=0) -> int:
    f = lib().task_dtrsm
    f.argtypes = [ompssblas_t] * 4 + [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_int, C.c_int]
    return _chk(f(opt(side), opt(uplo), opt(trans), opt(diag), bm, bn, alpha, _p(A), lda, _p(B), ldb, p))


def task_dsyrk(uplo, trans, n, k, alpha, A, lda, beta, Cm, ldc, p=0) -> int:
    f = lib().task_dsyrk
    f.argtypes = [ompssblas_t] * 2 + [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_double,
                                      C.c_void_p, C.c_int, C.c_int]
    return _chk(f(opt(uplo), opt(trans), n, k, alpha, _p(A), lda, beta, _p(Cm), ldc, p))


def task_dgemm(transa, transb, bm, bn, bk, alpha, A, lda, B, ldb, beta, Cm, ldc, p=0) -> int:
    f = lib().task_dgemm
    f.argtypes = [ompssblas_t] * 2 + [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_int]
    return _chk(f(opt(transa), opt(transb), bm, bn, bk, alpha, _p(A), lda, _p(B), ldb, beta, _p(Cm), ldc, p))


def ompss_dcg(n, bm, A, lda, b, x, tol, steps) -> int:
    """Returns -1 if converged, else the number of steps (itref.c:922-924)."""
    f = lib().ompss_dcg
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int]
    rc = f(n, bm, _p(A), lda, _p(b), _p(x), tol, steps)
    if rc < -1:
        raise LinompssError(rc, last_error())
    return rc


def ompss_ditref(n, bm, A, lda, b, x, prec, refit, it, norms=None) -> int:
    f = lib().ompss_ditref
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                  C.c_int, C.c_void_p]
    return _chk(f(n, bm, _p(A), lda, _p(b), _p(x), prec, refit, it, _p(norms)))


def _csr(vptr, vpos, vval):
    return (np.ascontiguousarray(vptr, dtype=np.int32), np.ascontiguousarray(vpos, dtype=np.int32),
            np.ascontiguousarray(vval, dtype=np.float64))


def ompss_dscg(n, bm, vptr, vpos, vval, b, x, tol, steps, is_precond=1) -> int:
    """Sparse dcg_pure (x: start vector in, iterate out).  Returns -1 if converged, else the steps."""
    vptr, vpos, vval = _csr(vptr, vpos, vval)
    f = lib().ompss_dscg
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                  C.c_int, C.c_int]
    rc = f(n, bm, _p(vptr), _p(vpos), _p(vval), _p(b), _p(x), tol, steps, is_precond)
    if rc < -1:
        raise LinompssError(rc, last_error())
    return rc


def ompss_dsitref(n, bm, vptr, vpos, vval, b, x, prec, refit, it, is_precond=1, norms=None) -> int:
    vptr, vpos, vval = _csr(vptr, vpos, vval)
    f = lib().ompss_dsitref
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                  C.c_int, C.c_int, C.c_int, C.c_void_p]
    return _chk(f(n, bm, _p(vptr), _p(vpos), _p(vval), _p(b), _p(x), prec, refit, it, is_precond, _p(norms)))


def mm_read_csr(path: str):
    """MatrixMarket coordinate file -> (n, vptr, vpos, vval) zero-based CSR (numpy copies)."""
    L = lib()
    L.lnb_mm_read_csr.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int)),
                                  C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_double))]
    L.lnb_mm_free.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    n = C.c_int()
    vp, vq, vv = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_double)()
    _chk(L.lnb_mm_read_csr(path.encode(), C.byref(n), C.byref(vp), C.byref(vq), C.byref(vv)))
    nnz = vp[n.value]
    out = (n.value, np.ctypeslib.as_array(vp, (n.value + 1,)).copy(),
           np.ctypeslib.as_array(vq, (max(nnz, 1),))[:nnz].copy(), np.ctypeslib.as_array(vv, (max(nnz, 1),))[:nnz].copy())
    L.lnb_mm_free(vp, vq, vv)
    return out


# --------------------------------------------------------------------------
# device entry points (torch CUDA tensors, column-major as (ncols, ld))
# --------------------------------------------------------------------------
def _stream(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _ld(t) -> int:
    # a (cols, rows) row-major tensor holds a column-major rows x cols matrix;
    # torch reports stride 1 for a size-1 leading dimension, whose ld is rows
    if t.dim() > 1 and t.size(0) == 1:
        return max(int(t.size(1)), 1)
    return int(t.stride(0))


def dchol_dev(At, n: int, b: int, info=None, stream=None) -> int:
    return _chk(lib().lnb_dchol_dev(C.c_int(n), C.c_int(b), _p(At), C.c_int(_ld(At)), _p(info), _stream(stream)))


def dposv_dev(At, Bt, n: int, nrhs: int, b: int, info=None, stream=None) -> int:
    return _chk(lib().lnb_dposv_dev(C.c_int(n), C.c_int(nrhs), C.c_int(b), _p(At), C.c_int(_ld(At)), _p(Bt),
                                    C.c_int(_ld(Bt)), _p(info), _stream(stream)))


def dpotrs_dev(Lt, Bt, n: int, nrhs: int, which: str = "B", stream=None) -> int:
    return _chk(lib().lnb_dpotrs_dev(C.c_int(n), C.c_int(nrhs), _p(Lt), C.c_int(_ld(Lt)), _p(Bt),
                                     C.c_int(_ld(Bt)), C.c_char(which.encode()), _stream(stream)))


def ompss_getrf(A, b: int, ll: bool = False) -> tuple:
    """P A = L U in place (ompss_dgetrf / ompss_sgetrf by A's dtype, column-major); returns (info, IPIV) with the
    reference's panel-relative pivots"""
    single = A.dtype == np.float32
    _colmajor(A, np.float32 if single else np.float64)
    m, n = A.shape
    name = ("ompss_sgetrf" if single else "ompss_dgetrf") + ("_ll" if ll else "")
    f = getattr(lib(), name)
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]
    ipiv = np.zeros(max(min(m, n), 1), dtype=np.int32)
    info = _chk(f(m, n, b, _p(A), m, _p(ipiv)))
    return info, ipiv[:min(m, n)]


def gensolv(A, B, b: int) -> int:
    """dgensolv_main / sgensolv_main: A (m x m) -> LU, B (m x n) -> A^-1 B, in place, column-major"""
    single = A.dtype == np.float32
    _colmajor(A, np.float32 if single else np.float64)
    _colmajor(B, np.float32 if single else np.float64)
    m, n = B.shape
    f = lib().sgensolv_main if single else lib().dgensolv_main
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    return _chk(f(m, n, b, _p(A), _p(B)))


def dgetrf_dev(At, m: int, n: int, ipiv_dev, info=None, stream=None) -> int:
    f = lib().lnb_dgetrf_dev
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return _chk(f(m, n, _p(At), _ld(At), _p(ipiv_dev), _p(info), _stream(stream)))


def dgetrs_dev(LUt, ipiv_dev, Bt, n: int, nrhs: int, stream=None) -> int:
    f = lib().lnb_dgetrs_dev
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return _chk(f(n, nrhs, _p(LUt), _ld(LUt), _p(ipiv_dev), _p(Bt), _ld(Bt), _stream(stream)))


def dgemm_dev(transa: str, transb: str, m: int, n: int, k: int, alpha: float, At, Bt, beta: float, Ct,
              stream=None) -> int:
    """C = alpha op(A) op(B) + beta C on device tensors (column-major as (cols, ld))."""
    f = lib().lnb_dgemm_dev
    f.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p,
                  C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    return _chk(f(transa.encode(), transb.encode(), m, n, k, alpha, _p(At), _ld(At), _p(Bt), _ld(Bt), beta, _p(Ct),
                  _ld(Ct), _stream(stream)))


def dsyrk_dev(uplo: str, trans: str, n: int, k: int, alpha: float, At, beta: float, Ct, stream=None) -> int:
    """C = alpha op(A) op(A)^T + beta C on triangle `uplo` of the device tensor Ct."""
    f = lib().lnb_dsyrk_dev
    f.argtypes = [C.c_char, C.c_char, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int, C.c_double, C.c_void_p,
                  C.c_int, C.c_void_p]
    return _chk(f(uplo.encode(), trans.encode(), n, k, alpha, _p(At), _ld(At), beta, _p(Ct), _ld(Ct),
                  _stream(stream)))


def dsymv_dev(At, Xt, Yt, n: int, nrhs: int, stream=None) -> int:
    """Y = A X from the lower triangle of A; Xt, Yt as (nrhs, n) contiguous tensors (ld n)."""
    f = lib().lnb_dsymv_dev
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return _chk(f(n, nrhs, _p(At), _ld(At), _p(Xt), _p(Yt), _stream(stream)))


def dtrsm_dev(uplo: str, trans: str, diag: str, m: int, n: int, alpha: float, At, Bt, stream=None) -> int:
    f = lib().lnb_dtrsm_dev
    f.argtypes = [C.c_char, C.c_char, C.c_char, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_int,
                  C.c_void_p, C.c_int, C.c_void_p]
    return _chk(f(uplo.encode(), trans.encode(), diag.encode(), m, n, alpha, _p(At), _ld(At), _p(Bt), _ld(Bt),
                  _stream(stream)))


class IrOpts(C.Structure):
    """lnb_ir_opts"""
    _fields_ = [("factor", C.c_int), ("max_iter", C.c_int), ("tol", C.c_double), ("equilibrate", C.c_int),
                ("allow_pcg", C.c_int), ("pcg_max_iter", C.c_int)]


class IrResult(C.Structure):
    """lnb_ir_result"""
    _fields_ = [("iterations", C.c_int), ("pcg_iterations", C.c_int), ("used_pcg", C.c_int),
                ("refactored_tiles", C.c_int), ("backward_error", C.c_double), ("factor_ms", C.c_double),
                ("solve_ms", C.c_double), ("info", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def ir_opts(**kw) -> IrOpts:
    o = IrOpts()
    lib().lnb_ir_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def dsposv_ir(A: np.ndarray, B: np.ndarray, b: int, opts: IrOpts | None = None):
    """Mixed-precision solve A X = B (host arrays, column-major).  Returns
    (rc, X, result dict); rc is 0 or LNB_ENOCONV (the call still returns X)."""
    _colmajor(A)
    B = np.asfortranarray(B.reshape(A.shape[0], -1))
    n, nrhs = B.shape
    X = np.zeros((n, nrhs), order="F")
    res = IrResult()
    rc = lib().lnb_dsposv_ir(C.c_int(n), C.c_int(nrhs), C.c_int(b), _p(A), C.c_int(A.shape[0]), _p(B),
                             C.c_int(n), _p(X), C.c_int(n), C.byref(opts) if opts is not None else None,
                             C.byref(res))
    if rc < 0 and rc != LNB_ENOCONV:
        raise LinompssError(rc, last_error())
    return rc, X, res.as_dict()


def dsposv_ir_dev(At, Bt, Xt, n: int, nrhs: int, b: int, opts: IrOpts | None = None, stream=None):
    res = IrResult()
    rc = lib().lnb_dsposv_ir_dev(C.c_int(n), C.c_int(nrhs), C.c_int(b), _p(At), C.c_int(_ld(At)), _p(Bt),
                                 C.c_int(_ld(Bt)), _p(Xt), C.c_int(_ld(Xt)),
                                 C.byref(opts) if opts is not None else None, C.byref(res), _stream(stream))
    if rc < 0 and rc != LNB_ENOCONV:
        raise LinompssError(rc, last_error())
    return rc, res.as_dict()


def _batched_args(n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode, max_iter):
    count = int(n_dev.numel())
    return [C.c_int(count), _p(n_dev), _p(nrhs_dev), _p(a_off_dev), _p(b_off_dev), _p(dA), _p(dB), _p(dX),
            C.c_int(mode), C.c_int(max_iter)]


def batched_posv_dev(n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode=FACTOR_FP32, max_iter=10,
                     info=None, iters=None, stream=None) -> int:
    """count = n_dev.numel() systems; int32 sizes, int64 offsets (elements) into the flat
    FP64 buffers dA (n x n each, full symmetric) and dB/dX (n x nrhs each)."""
    args = _batched_args(n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode, max_iter)
    return _chk(lib().lnb_batched_posv_dev(*args, _p(info), _p(iters), _stream(stream)))


def batched_partition(ns, rs, parts: int):
    """Split one batch over `parts` GPUs, longest-processing-time first on the
    estimated cost n^3/3 + 2 n^2 nrhs (lnb_batched_partition).  Returns
    (owner, load): the part of each system and the estimated flops per part."""
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    rs = np.ascontiguousarray(rs, dtype=np.int32)
    if ns.shape != rs.shape:
        raise ValueError("n and nrhs must have the same length")
    owner = np.empty(ns.size, dtype=np.int32)
    load = np.empty(max(parts, 1), dtype=np.float64)
    _chk(lib().lnb_batched_partition(C.c_int(ns.size), _p(ns), _p(rs), C.c_int(parts), _p(owner), _p(load)))
    return owner, load


def batched_autotune(n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode=FACTOR_FP32, max_iter=10,
                     stream=None) -> int:
    """Times the solver's launch shapes on this batch (CTA size, systems per SM, order), keeps the fastest for
    later calls in this process and returns its CTA size (256 or 512 threads)."""
    args = _batched_args(n_dev, nrhs_dev, a_off_dev, b_off_dev, dA, dB, dX, mode, max_iter)
    return _chk(lib().lnb_batched_autotune(*args, _stream(stream)))


def batched_config(mode=FACTOR_FP32) -> dict:
    """the launch shape the batched solver uses for `mode` (after autotuning, the chosen one)"""
    v = [C.c_int(), C.c_int(), C.c_int()]
    lib().lnb_batched_config(mode, C.byref(v[0]), C.byref(v[1]), C.byref(v[2]))
    return {"cta_threads": v[0].value, "ctas_per_sm": v[1].value, "order": "interleaved" if v[2].value else
            "largest first"}


def spotrs_dev(Lt, Bt, n: int, nrhs: int, which: str = "B", stream=None) -> int:
    return _chk(lib().lnb_spotrs_dev(C.c_int(n), C.c_int(nrhs), _p(Lt), C.c_int(_ld(Lt)), _p(Bt),
                                     C.c_int(_ld(Bt)), C.c_char(which.encode()), _stream(stream)))


def sspdsolv_main(m: int, n: int, b: int, A: np.ndarray, B: np.ndarray) -> int:
    _colmajor(A, np.float32)
    _colmajor(B, np.float32)
    return _chk(lib().sspdsolv_main(C.c_int(m), C.c_int(n), C.c_int(b), _p(A), _p(B)))


def set_chol_schedule(sched: int) -> None:
    """Schedule of the FP64 factorizations: SCHED_AUTO, SCHED_STREAMS (host-issued
    look-ahead on two streams) or SCHED_DAG (one persistent launch walking the
    tile DAG on the device)."""
    lib().lnb_set_chol_schedule(C.c_int(sched))


def set_wait_limit_us(us: int) -> None:
    lib().lnb_set_wait_limit_us(C.c_longlong(us))


def release_workspace() -> None:
    lib().lnb_release_workspace()


def version() -> str:
    return lib().lnb_version().decode()
