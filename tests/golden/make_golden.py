"""Record golden input/output vectors from the reference itself.

Run in a container that has the Linompss source tree (the reference is built
from its own sources by `make -C oracle ref`):

    make -C oracle ref && python tests/golden/make_golden.py

Every fixture is produced by calling the reference's compiled code on seeded
inputs; nothing here computes an expected value by other means.  The
reference publishes no golden vectors of its own and its CLIs seed from
time(NULL), so the sizes and seeds below follow the reference tests' shapes
scaled down to a few hundred KB in total:

  chol_*      tests/dense_tests/potrf_test.c (SPD = U[0,1) symmetric + n I;
              a ragged n % b != 0 case like N=1989, b=533)
  spdsolv_*   spdsolv.c / spdsolv_setup.c (B = A X with X ~ U[0,1))
  dsyrk_*     the reference's ompss_dsyrk (syrk_main.c): 4 uplo/trans cases and beta 0,
              ragged n and k against b, lda and ldc padded; ssyrk_* its FP32 twin
  dtrsm_*     tests/dense_tests/trsm_test.c (4 left cases, lda != m, ldb != m,
              alpha = -2.11, entries U[0,1) + 100 -- scaled to M=60, N=50, b=13)
  dcg_*       itref.c dcg_pure on a G G^T/n + I matrix
  itref_*     the refinement loop of itref.c main(), driven through its argv
              with A and RHS passed as files (itref_config.c:130-222)
  sparse_bj_* the block-Jacobi preconditioner of the sparse refinement, built
              by the reference's own code (hb_sym_diag_block + CSparse
              cs_schol/cs_chol/cs_cholsol2, itref_setup.c:55-93) on a sparse
              SPD matrix in zero-based CSR, applied to a vector
  lu_*        the reference's ompss_dgetrf (dlu_main, lu_main.c) on GENMAT_IP
              matrices (U[0,1) + 100 on the diagonal, as lu_test.c and the dlu
              program), square with a ragged last panel and tall rectangular
  gensolv_*   dgensolv_main (gensolv_main.c) on the same distribution, B ~
              U[0,1) with as many columns as rows (its IPIV is sized by them)

    python tests/golden/make_golden.py [group ...]   (default: every group)
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print("wrote", name)


def chol_cases():
    for variant, n, b, seed in (("rl", 100, 32, 1), ("rl", 128, 32, 2), ("rl", 199, 53, 3),
                                ("ll", 100, 32, 4), ("ll", 128, 64, 5)):
        A0 = O.spd_diag_dominant(n, seed)
        A = A0.copy(order="F")
        info = O.ref_chol(variant, A, b)
        save(f"chol_{variant}_n{n}_b{b}", A=A0, out=A, info=np.int64(info), b=np.int64(b))
    for variant, mt, b, seed in (("hrl", 4, 16, 6), ("hll", 4, 16, 7), ("hrl", 3, 24, 8)):
        n = mt * b
        A0 = O.spd_diag_dominant(n, seed)
        tiles = np.zeros((mt, mt, b, b), order="C")
        for j in range(mt):
            for i in range(mt):
                tiles[j, i] = A0[i * b:(i + 1) * b, j * b:(j + 1) * b].T  # column-major tile
        tiles0 = tiles.copy()
        info = O.ref_chol_h(variant, tiles)
        save(f"chol_{variant}_mt{mt}_b{b}", tiles_in=tiles0, tiles_out=tiles, info=np.int64(info))


def schol_case():
    import ctypes as C
    n, b = 96, 32
    A0 = O.spd_diag_dominant(n, 9).astype(np.float32)
    A = np.asfortranarray(A0.copy())
    info = O.ref().ompss_schol_rl(C.c_int(n), C.c_int(b), C.c_int(b), A.ctypes.data_as(C.c_void_p),
                                  C.c_int(n))
    save(f"schol_rl_n{n}_b{b}", A=A0, out=A, info=np.int64(info))


def spdsolv_cases():
    for m, nrhs, b, seed in ((128, 1, 32, 10), (128, 3, 32, 11), (96, 8, 48, 12)):
        rng = np.random.default_rng(seed)
        A0 = O.spd_diag_dominant(m, seed)
        X = np.asfortranarray(rng.random((m, nrhs)))
        B0 = np.asfortranarray(A0 @ X)
        A = A0.copy(order="F")
        B = B0.copy(order="F")
        O.ref_spdsolv(A, B, b)
        save(f"spdsolv_m{m}_r{nrhs}_b{b}", A=A0, B=B0, X=B, L=A)


def dtrsm_cases():
    M, N, BB, LDA, LDC, alpha = 60, 50, 13, 65, 62, -2.11
    rng = np.random.default_rng(13)
    A = np.asfortranarray(rng.random((LDA, M)) + 100.0)
    C0 = np.asfortranarray(rng.random((LDC, N)) + 100.0)
    for uplo in "LU":
        for trans in "NT":
            D = C0.copy(order="F")
            O.ref_dtrsm("L", uplo, trans, "N", M, N, BB, alpha, A, LDA, D, LDC)
            save(f"dtrsm_L{uplo}{trans}", A=A, B=C0, out=D, M=np.int64(M), N=np.int64(N),
                 bb=np.int64(BB), alpha=np.float64(alpha))


def dsyrk_cases():
    # blocked ompss_dsyrk (syrk_main.c): ragged n and k against the tile size,
    # lda and ldc larger than the matrices, all four uplo/trans cases, and beta 0
    n, k, b, alpha = 70, 40, 16, -1.3
    rng = np.random.default_rng(21)
    for uplo in "LU":
        for trans in "NT":
            for beta in (0.7, 0.0):
                if beta == 0.0 and (uplo, trans) != ("L", "N"):
                    continue
                lda = (n if trans == "N" else k) + 5
                A = np.asfortranarray(rng.standard_normal((lda, k if trans == "N" else n)))
                C0 = np.asfortranarray(rng.standard_normal((n + 3, n)))
                D = C0.copy(order="F")
                O.ref_dsyrk(uplo, trans, b, n, k, alpha, A, lda, beta, D, n + 3)
                tag = "b0" if beta == 0.0 else "b"
                save(f"dsyrk_{uplo}{trans}_{tag}", A=A, C=C0, out=D, n=np.int64(n), k=np.int64(k),
                     bb=np.int64(b), alpha=np.float64(alpha), beta=np.float64(beta))


def ssyrk_case():
    # the FP32 twin ompss_ssyrk, lower and no transpose, ragged n and k against b
    n, k, b, alpha, beta = 70, 40, 16, -1.3, 0.7
    rng = np.random.default_rng(22)
    A = np.asfortranarray(rng.standard_normal((n + 5, k)).astype(np.float32))
    C0 = np.asfortranarray(rng.standard_normal((n + 3, n)).astype(np.float32))
    D = C0.copy(order="F")
    O.ref_ssyrk("L", "N", b, n, k, alpha, A, n + 5, beta, D, n + 3)
    save("ssyrk_LN_b", A=A, C=C0, out=D, n=np.int64(n), k=np.int64(k), bb=np.int64(b),
         alpha=np.float64(alpha), beta=np.float64(beta))


def dcg_cases():
    for n, bm, steps, tol, seed in ((64, 16, 8, 1e-10, 14), (64, 16, 200, 1e-10, 14),
                                    (100, 32, 300, 1e-12, 15)):
        A = O.spd_covariance(n, 1.0, seed)
        rhs = np.random.default_rng(seed + 100).random(n)
        rc, x = O.ref_cg(A, rhs, bm, tol, steps)
        save(f"dcg_n{n}_bm{bm}_s{steps}", A=A, rhs=rhs, x=x, rc=np.int64(rc),
             bm=np.int64(bm), steps=np.int64(steps), tol=np.float64(tol))


_ITREF_CHILD = r"""
import ctypes as C, sys
lib = C.CDLL(sys.argv[1])
args = sys.argv[2:]
argv = (C.c_char_p * (len(args) + 1))(*[a.encode() for a in args], None)
sys.exit(lib.lnbref_itref_main(len(args), argv))
"""


def itref_cases():
    lib = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    for n, bm, refit, it, prec, seed in ((64, 16, 6, 64, 1e-12, 16), (96, 32, 8, 96, 1e-13, 17)):
        A = O.spd_covariance(n, 1.0, seed)
        rhs = np.random.default_rng(seed + 100).random(n)
        with tempfile.TemporaryDirectory() as tmp:
            with open(os.path.join(tmp, "A.txt"), "w") as f:
                f.write("# A, column-major\n" + "".join(f"{v:.17e}\n" for v in A.ravel(order="F")))
            with open(os.path.join(tmp, "RHS.txt"), "w") as f:
                f.write("# rhs\n" + "".join(f"{v:.17e}\n" for v in rhs))
            # itref n bm interval corrections refit it prec is_precond async profile rep warmup
            #       release icriteria ii_distance orth_fac A B cglog_level
            argv = ["itref", str(n), str(bm), "1", "0", str(refit), str(it), repr(prec), "0", "0",
                    "1.0", "1", "0", "1", "1e-5", "1e-2", "1.0", "A.txt", "RHS.txt", "0"]
            subprocess.run([sys.executable, "-c", _ITREF_CHILD, lib] + argv, cwd=tmp, check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            with open(os.path.join(tmp, "itref_norms.log")) as f:
                lines = f.read().splitlines()[1:]
        norms = []
        for line in lines:
            parts = line.split()
            norms.append(float(parts[1]))
        save(f"itref_n{n}_bm{bm}", A=A, rhs=rhs, norms_logged=np.array(norms), refit=np.int64(refit),
             it=np.int64(it), prec=np.float64(prec), bm=np.int64(bm))


def sparse_bj_cases():
    for n, bm, seed in ((150, 32, 1), (200, 48, 2)):
        A = O.spd_sparse(n, seed=seed)
        vptr, vpos, vval = O.csr_from_dense(A)
        r = np.random.default_rng(seed + 50).standard_normal(n)
        rc, z = O.ref_bj_apply(vptr, vpos, vval, bm, r)
        assert rc == 0
        save(f"sparse_bj_n{n}_bm{bm}", A=A, vptr=vptr, vpos=vpos, vval=vval, r=r, z=z, bm=np.int64(bm))


def lu_cases():
    """the reference's ompss_dgetrf (dlu_main) and dgensolv_main on its own matrix distribution (GENMAT_IP:
    uniform [0, 1) plus 100 on the diagonal, seeded here), as lu_test.c and the dlu/dgensolv programs run it"""
    for m, n, b, seed in ((200, 200, 33, 11), (240, 160, 64, 12)):
        A = O.genmat_ip(m, n, seed)
        LU = A.copy(order="F")
        ipiv = O.ref_getrf(LU, b)
        save(f"lu_m{m}_n{n}_b{b}", A=A, LU=LU, ipiv=ipiv, b=np.int64(b))
    m, b = 128, 48
    A = O.genmat_ip(m, m, 13)
    B = np.asfortranarray(np.random.default_rng(14).random((m, m)))
    LU, X = A.copy(order="F"), B.copy(order="F")
    O.ref_gensolv(LU, X, b)
    save(f"gensolv_m{m}_b{b}", A=A, B=B, LU=LU, X=X, b=np.int64(b))


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("build the reference first: make -C oracle ref")
    if len(sys.argv) > 1:
        for group in sys.argv[1:]:
            globals()[group + "_cases"]()
        sys.exit(0)
    chol_cases()
    schol_case()
    spdsolv_cases()
    dtrsm_cases()
    dsyrk_cases()
    ssyrk_case()
    dcg_cases()
    itref_cases()
    sparse_bj_cases()
    lu_cases()
