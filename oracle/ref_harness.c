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

struct cs_sparse;
struct css_s;
struct csn_s;

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
