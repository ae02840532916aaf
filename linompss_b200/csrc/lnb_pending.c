/*
 * lnb_pending.c -- entry points declared in linompss_b200.h whose kernels
 * are not in this build yet.  Each returns LNB_EINVAL with a message; none
 * computes anything on the CPU.
 */
#include "lnb_host.h"

#define PENDING(name) lnb_set_error(LNB_EINVAL, "%s: not available in this build", name)

int sspdsolv_main(int m, int nrhs, int b, float *A, float *B) { (void)m; (void)nrhs; (void)b; (void)A; (void)B; return PENDING("sspdsolv_main"); }
int lnb_spotrs_dev(int n, int nrhs, const float *dL, int lda, float *dB, int ldb, char which, void *stream) { (void)n; (void)nrhs; (void)dL; (void)lda; (void)dB; (void)ldb; (void)which; (void)stream; return PENDING("lnb_spotrs_dev"); }
int lnb_batched_posv_dev(int count, const int *n_dev, const int *nrhs_dev, const int64_t *a_off_dev, const int64_t *b_off_dev, const double *dA, const double *dB, double *dX, int mode, int max_iter, int *info_dev, int *iters_dev, void *stream) { (void)count; (void)n_dev; (void)nrhs_dev; (void)a_off_dev; (void)b_off_dev; (void)dA; (void)dB; (void)dX; (void)mode; (void)max_iter; (void)info_dev; (void)iters_dev; (void)stream; return PENDING("lnb_batched_posv_dev"); }
