# Build recipe for the reference's own hot-path code (test infrastructure).
#
# Compiles the Linompss sources in place (read-only tree, objects go to
# oracle/_ref/) with plain gcc and no -fopenmp, so the OmpSs pragmas are inert
# and every tile task runs inline in program order.  Each precision-generic
# file is compiled twice (-DDOUBLE_PRECISION / -DSINGLE_PRECISION) because
# ompss_dense_chol.c references both the d* and s* drivers.  itref.c's main()
# is renamed so the refinement loop can be called as a function.
#
# Invoked by `make -C oracle ref`; never run the reference's own autotools.

REF_SRC ?=
ifeq ($(strip $(REF_SRC)),)
$(error set REF_SRC to the reference's src/ directory)
endif
OUT     := _ref
CC      ?= gcc
RCFLAGS := -O2 -w -fPIC -DHAVE_CONFIG_H -I$(OUT) \
           -I$(REF_SRC)/fp -I$(REF_SRC)/blas -I$(REF_SRC)/blocked_blas -I$(REF_SRC)/matutil \
           -I$(REF_SRC)/util -I$(REF_SRC)/cholesky/dense -I$(REF_SRC)/spdsolv -I$(REF_SRC)/trsm \
           -I$(REF_SRC)/syrk \
           -I$(REF_SRC)/csparse -I$(REF_SRC)/itref -I$(REF_SRC)/lu -I$(REF_SRC)/gensolv

# precision-generic sources (built for both precisions)
GEN := cholesky/dense/chol_rlmain.c cholesky/dense/chol_llmain.c cholesky/dense/chol_hrlmain.c \
       cholesky/dense/chol_hllmain.c cholesky/dense/chol_nrlmain.c cholesky/dense/chol_nllmain.c \
       blocked_blas/tasks_potrf.c blocked_blas/tasks_trsm.c blocked_blas/tasks_syrk.c \
       blocked_blas/task_gemm.c blocked_blas/tasks_nested_potrf.c blocked_blas/tasks_nested_trsm.c \
       blocked_blas/tasks_nested_syrk.c blocked_blas/tasks_nested_gemm.c \
       spdsolv/spdsolv_main.c trsm/trsm_main.c syrk/syrk_main.c \
       lu/lu_main.c lu/lull_main.c lu/lu_kernels.c gensolv/gensolv_main.c
# double-only sources: the dense itref program and what it links
DBL := itref/itref.c itref/itref_config.c itref/itref_setup.c fp/fptype.c \
       blocked_blas/task_dot.c blocked_blas/task_axpy.c blocked_blas/task_axpy_async.c \
       blocked_blas/task_copy.c blocked_blas/task_util.c blocked_blas/task_convert.c \
       blocked_blas/task_dot_async.c blocked_blas/task_gemv.c util/as_man.c util/async_struct.c \
       util/task_log.c util/prof.c util/file_log.c util/strutil.c util/ompss_apps.c \
       util/ompss_options.c matutil/matfprint.c matutil/matfread.c matutil/genmat.c \
       matutil/genmat_config.c matutil/densutil.c csparse/dcsparse.c matutil/hb.c
# precision-independent sources
COM := fp/fpmatr.c cholesky/dense/ompss_dense_chol.c trsm/ompss_trsm.c syrk/ompss_syrk.c lu/ompss_lu.c

GEN_D := $(patsubst %.c,$(OUT)/d/%.o,$(GEN))
GEN_S := $(patsubst %.c,$(OUT)/s/%.o,$(GEN))
DBL_O := $(patsubst %.c,$(OUT)/d/%.o,$(DBL))
COM_O := $(patsubst %.c,$(OUT)/c/%.o,$(COM))

$(OUT)/libref.so: $(GEN_D) $(GEN_S) $(DBL_O) $(COM_O) $(OUT)/ref_harness.o
	$(CC) -shared -o $@ $^ -L$(OPENBLAS_DIR) -l:$(OPENBLAS_LIB) \
	      -Wl,--disable-new-dtags,-rpath,$(OPENBLAS_DIR) -lm -lpthread

$(OUT)/config.h:
	@mkdir -p $(OUT)
	printf '#define USE_MKL 0\n' > $@

# itref.c calls cblas_ddot without a prototype in non-MKL builds (implicit
# int); the forced include gives it the right return type.
$(OUT)/cblas_proto.h:
	@mkdir -p $(OUT)
	printf 'double cblas_ddot(int, const double *, int, const double *, int);\n' > $@

$(OUT)/d/%.o: $(REF_SRC)/%.c $(OUT)/config.h $(OUT)/cblas_proto.h
	@mkdir -p $(dir $@)
	$(CC) $(RCFLAGS) -DDOUBLE_PRECISION -Dmain=linompss_ref_itref_main -include math.h \
	      -include $(OUT)/cblas_proto.h -c $< -o $@

$(OUT)/s/%.o: $(REF_SRC)/%.c $(OUT)/config.h
	@mkdir -p $(dir $@)
	$(CC) $(RCFLAGS) -DSINGLE_PRECISION -c $< -o $@

$(OUT)/c/%.o: $(REF_SRC)/%.c $(OUT)/config.h
	@mkdir -p $(dir $@)
	$(CC) $(RCFLAGS) -DDOUBLE_PRECISION -c $< -o $@

$(OUT)/ref_harness.o: ref_harness.c $(OUT)/config.h
	$(CC) $(RCFLAGS) -DDOUBLE_PRECISION -c $< -o $@
