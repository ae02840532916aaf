/*
 * ref_harness.c -- call shims for the reference library built by ref.mk.
 *
 * TEST INFRASTRUCTURE ONLY.  Linked into oracle/_ref/libref.so next to the
 * reference's own objects; used by tests/golden/make_golden.py to record the
 * reference's outputs, and by bench.py's CPU-baseline leg to time the
 * reference.  The factor/solve entry points of the reference are called
 * directly through ctypes; this file only wraps what cannot be called that
 * way:
 *   - dcg_pure (itref.c:690) needs a work buffer laid out as
 *     itref_setup.c:202-213 does it, a row-block energy vector
 *     (itref_setup.c:127-130) and a bitmap;
 *   - the refinement loop lives in main() (itref.c:928), which ref.mk renames
 *     to linompss_ref_itref_main so that it can be called with an argv.
 */
#include <stdlib.h>
#include <string.h>

#include "async_struct.h"
#include "dcsparse.h"
#include "hb.h"

/* dcsparse.c defines cs_cholsol2 as cs_cholsol2_double; the header declares only the short name */
int cs_cholsol2_double(int n, css *S, csn *N, double *b, double *x);

int dcg_pure(int bm, int bn, int n, void *A, int s, void *b, void *xbuff, int *offs, double tol,
             int steps, void *work, unsigned long works, int async, double profile, int warmup,
             int cglog, int release, double orth_fac, double *mat_energy, int is_precond,
             void *zbuff, void *Acs, void **S, void **N, int *bm_p);
double dmat_energy_sym(int n, int lda, int bs, double *mat, double *dist);
int linompss_ref_itref_main(int argc, char *argv[]);

/* x (length n) receives the CG iterate started from x = 0.  Returns dcg_pure's
 * code: -1 when converged, else the step count. */
int lnbref_dcg(int n, int bm, double *A, double *b, double *x, double tol, int steps)
{
    int s = 1, dupl = 4;
    unsigned long ns = (unsigned long)n * s;
    unsigned long nsalgn = ((ns + 0x7f) >> 7) << 7;
    unsigned long salgn = ((s + 0x7f) >> 7) << 7;
    unsigned long tmps = nsalgn * dupl * 4 + 3 * salgn * dupl;
    size_t works = 3 * sizeof(async_t) + sizeof(double) * (tmps + 16);
    void *work = NULL;
    if (posix_memalign(&work, 128, works)) return -1000;
    memset(work, 0, works);
    async_setup((async_t *)work);
    async_setup((async_t *)work + 1);
    async_setup((async_t *)work + 2);

    int szeb = (n + bm - 1) / bm;
    double *energy = calloc(szeb + 1, sizeof(double));
    energy[szeb] = dmat_energy_sym(n, n, bm, A, energy);
    int *bm_p = calloc(szeb, sizeof(int));
    double *xbuff = calloc(4 * ns, sizeof(double));
    int offs = 0;

    int rc = dcg_pure(bm, 1, n, A, s, b, xbuff, &offs, tol, steps, work, tmps, 0, 1.0, 0, 0, 1,
                      1.0, energy, 0, NULL, NULL, NULL, NULL, bm_p);
    memcpy(x, xbuff, sizeof(double) * n);
    free(xbuff); free(bm_p); free(energy); free(work);
    return rc;
}

int lnbref_itref_main(int argc, char **argv)
{
    return linompss_ref_itref_main(argc, argv);
}

/* The reference's block-Jacobi preconditioner of the sparse refinement,
 * built exactly as itref_setup.c:55-93 builds it and applied as
 * bsblas_dcholsolv2 (bsblas_csrmm.h:498-513) applies it: the complete bm x bm
 * diagonal blocks of the zero-based CSR matrix (hb_sym_diag_block, hb.c:512),
 * each handed to CSparse as a compressed matrix, analysed with natural
 * ordering (cs_schol(A, 0)), factored (cs_chol) and solved
 * (cs_cholsol2: z = L^-T L^-1 r).  Returns 0, or 1 + the first block whose
 * factor failed. */
int lnbref_bj_apply(int n, int bm, int *vptr, int *vpos, double *vval, const double *r, double *z)
{
    hbmat_t A;
    memset(&A, 0, sizeof A);
    A.m = A.n = n;
    A.elemc = vptr[n];
    A.vptr = vptr;
    A.vpos = vpos;
    A.vval = vval;
    const int bs = (n + bm - 1) / bm;
    hbmat_t *blocks = calloc((size_t)bs, sizeof(hbmat_t));
    hb_sym_diag_block_double(&A, bm, blocks);
    int rc = 0;
    for (int i = 0, i0 = 0; i < bs; ++i, i0 += bm) {
        hbmat_t *d = &blocks[i];
        cs c;
        c.nz = -1;
        c.nzmax = d->elemc;
        c.n = c.m = d->m;
        c.p = d->vptr;
        c.i = d->vpos;
        c.x = d->vval;
        css *S = cs_schol_double(&c, 0);
        csn *N = S ? cs_chol_double(&c, S) : NULL;
        if (!N) {
            if (!rc) rc = 1 + i;
        } else {
            cs_cholsol2_double(d->m, S, N, (double *)r + i0, z + i0);
        }
        free(d->vptr); free(d->vpos); free(d->vval);
    }
    free(blocks);
    return rc;
}
