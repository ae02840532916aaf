/*
 * lnb_pending.c -- entry points declared in linompss_b200.h whose kernels
 * are not in this build yet.  Each returns LNB_EINVAL with a message; none
 * computes anything on the CPU.
 */
#include "lnb_host.h"

#define PENDING(name) lnb_set_error(LNB_EINVAL, "%s: not available in this build", name)

int ompss_schol_rl(int n, int b, int t, float *A, int lda) { (void)n; (void)b; (void)t; (void)A; (void)lda; return PENDING("ompss_schol_rl"); }
int ompss_schol_ll(int n, int b, int t, float *A, int lda) { (void)n; (void)b; (void)t; (void)A; (void)lda; return PENDING("ompss_schol_ll"); }
int ompss_schol_hrl(int mt, int b, int t, float **Ah) { (void)mt; (void)b; (void)t; (void)Ah; return PENDING("ompss_schol_hrl"); }
int ompss_schol_hll(int mt, int b, int t, float **Ah) { (void)mt; (void)b; (void)t; (void)Ah; return PENDING("ompss_schol_hll"); }
int sspdsolv_main(int m, int nrhs, int b, float *A, float *B) { (void)m; (void)nrhs; (void)b; (void)A; (void)B; return PENDING("sspdsolv_main"); }
int lnb_schol_dev(int n, int b, float *dA, int lda, int *info_dev, void *stream) { (void)n; (void)b; (void)dA; (void)lda; (void)info_dev; (void)stream; return PENDING("lnb_schol_dev"); }
int lnb_spotrs_dev(int n, int nrhs, const float *dL, int lda, float *dB, int ldb, char which, void *stream) { (void)n; (void)nrhs; (void)dL; (void)lda; (void)dB; (void)ldb; (void)which; (void)stream; return PENDING("lnb_spotrs_dev"); }
void lnb_ir_default_opts(lnb_ir_opts *o) { if (o) { o->factor = LNB_FACTOR_TF32X3; o->max_iter = 30; o->tol = 0; o->equilibrate = 1; o->allow_pcg = 1; o->pcg_max_iter = 200; } }
int lnb_dsposv_ir_dev(int n, int nrhs, int b, const double *dA, int lda, const double *dB, int ldb, double *dX, int ldx, const lnb_ir_opts *opts, lnb_ir_result *res, void *stream) { (void)n; (void)nrhs; (void)b; (void)dA; (void)lda; (void)dB; (void)ldb; (void)dX; (void)ldx; (void)opts; (void)res; (void)stream; return PENDING("lnb_dsposv_ir_dev"); }
int lnb_dsposv_ir(int n, int nrhs, int b, const double *A, int lda, const double *B, int ldb, double *X, int ldx, const lnb_ir_opts *opts, lnb_ir_result *res) { (void)n; (void)nrhs; (void)b; (void)A; (void)lda; (void)B; (void)ldb; (void)X; (void)ldx; (void)opts; (void)res; return PENDING("lnb_dsposv_ir"); }
int lnb_batched_posv_dev(int count, const int *n_dev, const int *nrhs_dev, const int64_t *a_off_dev, const int64_t *b_off_dev, const double *dA, const double *dB, double *dX, int mode, int max_iter, int *info_dev, int *iters_dev, void *stream) { (void)count; (void)n_dev; (void)nrhs_dev; (void)a_off_dev; (void)b_off_dev; (void)dA; (void)dB; (void)dX; (void)mode; (void)max_iter; (void)info_dev; (void)iters_dev; (void)stream; return PENDING("lnb_batched_posv_dev"); }
