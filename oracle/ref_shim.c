/*
 * Link shim for building the reference HDSDP CPU solver as a test oracle.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product library links or calls this
 * file; it exists so that the unmodified reference sources can be compiled and
 * run on this machine as the parity oracle and as the CPU baseline.
 *
 * The reference links Intel MKL (BLAS/LAPACK names without the trailing
 * underscore, linalg/def_hdsdp_linsolver.h:182-210, linalg/vec_opts.c:12-18,
 * linalg/dense_opts.c; MKL thread control at interface/hdsdp_utils.c:466-479,
 * Pardiso at linalg/hdsdp_linsolver.c:47-450). MKL is not installed, so:
 *
 *  - every BLAS/LAPACK symbol is forwarded to the LP64 "scipy_<name>_" entry
 *    points of the OpenBLAS build shipped with scipy;
 *  - MKL_{Get_Max,Set_Num}_Threads map to OpenBLAS thread control;
 *  - pardisoinit/pardiso/pardiso_getdiag are a DENSE stand-in: the lower CSC
 *    matrix is expanded to a full column-major array and factorised with
 *    dpotrf. Phases follow the reference's use: 11 (symbolic, no-op),
 *    22 (factorise, -4 when not positive definite, matching
 *    linsolver.c:229-266), 331/333/33 (forward / backward / full solve),
 *    -1 (free). pardiso_getdiag returns L_ii^2 because the reference takes a
 *    square root of it (linsolver.c:386-388). No fill-reducing ordering and no
 *    pivot perturbation (iparm[9]=13 in the reference) are applied: same
 *    mathematics, different rounding and Krylov basis for Lanczos.
 */
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stddef.h>

/* ---- OpenBLAS (scipy build) LP64 entry points -------------------------------- */
extern double scipy_dnrm2_(const int *, const double *, const int *);
extern void scipy_daxpy_(const int *, const double *, const double *, const int *, double *, const int *);
extern double scipy_ddot_(const int *, const double *, const int *, const double *, const int *);
extern void scipy_dscal_(const int *, const double *, double *, const int *);
extern void scipy_drscl_(const int *, const double *, double *, const int *);
extern void scipy_dsyr_(const char *, const int *, const double *, const double *, const int *,
                        double *, const int *, size_t);
extern void scipy_dgemv_(const char *, const int *, const int *, const double *, const double *,
                         const int *, const double *, const int *, const double *, double *,
                         const int *, size_t);
extern void scipy_dger_(const int *, const int *, const double *, const double *, const int *,
                        const double *, const int *, double *, const int *);
extern void scipy_dspmv_(const char *, const int *, const double *, const double *, const double *,
                         const int *, const double *, double *, const int *, size_t);
extern void scipy_dsymv_(const char *, const int *, const double *, const double *, const int *,
                         const double *, const int *, const double *, double *, const int *, size_t);
extern void scipy_dsymm_(const char *, const char *, const int *, const int *, const double *,
                         const double *, const int *, const double *, const int *, const double *,
                         double *, const int *, size_t, size_t);
extern void scipy_dtrsm_(const char *, const char *, const char *, const char *, const int *,
                         const int *, const double *, const double *, const int *, double *,
                         const int *, size_t, size_t, size_t, size_t);
extern void scipy_dpotrf_(const char *, const int *, double *, const int *, int *, size_t);
extern void scipy_dpotri_(const char *, const int *, double *, const int *, int *, size_t);
extern void scipy_dpotrs_(const char *, const int *, const int *, const double *, const int *,
                          double *, const int *, int *, size_t);
extern void scipy_dsytrf_(const char *, const int *, double *, const int *, int *, double *,
                          const int *, int *, size_t);
extern void scipy_dsytrs_(const char *, const int *, const int *, const double *, const int *,
                          const int *, double *, const int *, int *, size_t);
extern void scipy_dsyevr_(const char *, const char *, const char *, const int *, double *, const int *,
                          const double *, const double *, const int *, const int *, const double *,
                          int *, double *, double *, const int *, int *, double *, const int *,
                          int *, const int *, int *, size_t, size_t, size_t);
extern void scipy_openblas_set_num_threads(int);
extern int scipy_openblas_get_num_threads(void);

/* ---- MKL-style names used by the reference ----------------------------------- */
double dnrm2(int *n, double *x, int *incx) { return scipy_dnrm2_(n, x, incx); }
void daxpy(int *n, double *a, double *x, int *incx, double *y, int *incy) { scipy_daxpy_(n, a, x, incx, y, incy); }
double ddot(int *n, double *x, int *incx, double *y, int *incy) { return scipy_ddot_(n, x, incx, y, incy); }
void dscal(int *n, double *a, double *x, int *incx) { scipy_dscal_(n, a, x, incx); }
void drscl(int *n, double *a, double *x, int *incx) { scipy_drscl_(n, a, x, incx); }
void dsyr(char *uplo, int *n, double *alpha, double *x, int *incx, double *a, int *lda) {
    scipy_dsyr_(uplo, n, alpha, x, incx, a, lda, 1);
}
void dgemv(char *t, int *m, int *n, double *alpha, double *a, int *lda, double *x, int *incx,
           double *beta, double *y, int *incy) {
    scipy_dgemv_(t, m, n, alpha, a, lda, x, incx, beta, y, incy, 1);
}
void dger(int *m, int *n, double *alpha, double *x, int *incx, double *y, int *incy, double *a, int *lda) {
    scipy_dger_(m, n, alpha, x, incx, y, incy, a, lda);
}
void dspmv(char *uplo, int *n, double *alpha, double *ap, double *x, int *incx, double *beta,
           double *y, int *incy) {
    scipy_dspmv_(uplo, n, alpha, ap, x, incx, beta, y, incy, 1);
}
void dsymv(char *uplo, int *n, double *alpha, double *a, int *lda, double *x, int *incx,
           double *beta, double *y, int *incy) {
    scipy_dsymv_(uplo, n, alpha, a, lda, x, incx, beta, y, incy, 1);
}
void dsymm(char *side, char *uplo, int *m, int *n, double *alpha, double *a, int *lda, double *b,
           int *ldb, double *beta, double *c, int *ldc) {
    scipy_dsymm_(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, 1, 1);
}
void dtrsm(const char *side, const char *uplo, const char *transa, const char *diag, const int *m,
           const int *n, const double *alpha, const double *a, const int *lda, double *b, const int *ldb) {
    scipy_dtrsm_(side, uplo, transa, diag, m, n, alpha, a, lda, b, ldb, 1, 1, 1, 1);
}
void dpotrf(const char *uplo, const int *n, double *a, const int *lda, int *info) {
    scipy_dpotrf_(uplo, n, a, lda, info, 1);
}
void dpotri(const char *uplo, const int *n, double *a, const int *lda, int *info) {
    scipy_dpotri_(uplo, n, a, lda, info, 1);
}
void dpotrs(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda,
            double *b, const int *ldb, int *info) {
    scipy_dpotrs_(uplo, n, nrhs, a, lda, b, ldb, info, 1);
}
void dsytrf(const char *uplo, const int *n, double *a, const int *lda, int *ipiv, double *work,
            const int *lwork, int *info) {
    scipy_dsytrf_(uplo, n, a, lda, ipiv, work, lwork, info, 1);
}
void dsytrs(const char *uplo, const int *n, const int *nrhs, const double *a, const int *lda,
            const int *ipiv, double *b, const int *ldb, int *info) {
    scipy_dsytrs_(uplo, n, nrhs, a, lda, ipiv, b, ldb, info, 1);
}
void dsyevr(char *jobz, char *range, char *uplo, int *n, double *a, int *lda, double *vl, double *vu,
            int *il, int *iu, double *abstol, int *m, double *w, double *z, int *ldz, int *isuppz,
            double *work, int *lwork, int *iwork, int *liwork, int *info) {
    scipy_dsyevr_(jobz, range, uplo, n, a, lda, vl, vu, il, iu, abstol, m, w, z, ldz, isuppz, work,
                  lwork, iwork, liwork, info, 1, 1, 1);
}

int MKL_Get_Max_Threads(void) { return scipy_openblas_get_num_threads(); }
int MKL_Set_Num_Threads(int nth) { scipy_openblas_set_num_threads(nth); return nth; }

/* ---- Dense stand-in for the Pardiso calls ------------------------------------- */
typedef struct {
    int n;
    double *L;      /* full column-major, lower Cholesky factor */
    double *work;
    int ok;
} dense_pds;

void pardisoinit(void *pt, int *mtype, int *iparm) {
    (void) mtype;
    void **handle = (void **) pt;
    handle[0] = NULL;
    (void) iparm;
}

static dense_pds *pds_get(void *pt, int n) {
    void **handle = (void **) pt;
    dense_pds *d = (dense_pds *) handle[0];
    if (!d) {
        d = (dense_pds *) calloc(1, sizeof(dense_pds));
        d->n = n;
        d->L = (double *) calloc((size_t) n * n, sizeof(double));
        d->work = (double *) calloc((size_t) n, sizeof(double));
        handle[0] = d;
    }
    return d;
}

static void pds_solve_lower(dense_pds *d, int trans, int nrhs, double *b) {
    const char side = 'L', uplo = 'L', diag = 'N';
    const char tr = trans ? 'T' : 'N';
    const double one = 1.0;
    dtrsm(&side, &uplo, &tr, &diag, &d->n, &nrhs, &one, d->L, &d->n, b, &d->n);
}

void pardiso(void *pt, int *maxfct, int *mnum, int *mtype, int *phase, int *n, double *a, int *ia,
             int *ja, int *perm, int *nrhs, int *iparm, int *msglvl, double *b, double *x, int *error) {
    (void) maxfct; (void) mnum; (void) mtype; (void) perm; (void) msglvl;
    *error = 0;
    if (*phase == -1) {
        void **handle = (void **) pt;
        dense_pds *d = (dense_pds *) handle[0];
        if (d) { free(d->L); free(d->work); free(d); handle[0] = NULL; }
        return;
    }
    dense_pds *d = pds_get(pt, *n);
    int nn = d->n;
    if (*phase == 11) {
        /* Symbolic analysis: report a fill estimate equal to the dense lower triangle */
        iparm[17] = nn * (nn + 1) / 2;
        return;
    }
    if (*phase == 22 || *phase == 12) {
        memset(d->L, 0, sizeof(double) * (size_t) nn * nn);
        for (int j = 0; j < nn; ++j)
            for (int k = ia[j]; k < ia[j + 1]; ++k)
                d->L[(size_t) j * nn + ja[k]] = a[k];
        int info = 0;
        const char lo = 'L';
        dpotrf(&lo, &nn, d->L, &nn, &info);
        d->ok = (info == 0);
        *error = (info == 0) ? 0 : -4;
        return;
    }
    int nr = nrhs ? *nrhs : 1;
    /* iparm[5] == 1: the solution overwrites b */
    double *target = b;
    if (!iparm[5]) {
        memcpy(x, b, sizeof(double) * (size_t) nn * nr);
        target = x;
    }
    if (*phase == 331) {
        pds_solve_lower(d, 0, nr, target);
    } else if (*phase == 333) {
        pds_solve_lower(d, 1, nr, target);
    } else if (*phase == 33) {
        pds_solve_lower(d, 0, nr, target);
        pds_solve_lower(d, 1, nr, target);
    } else {
        *error = -1;
    }
}

void pardiso_getdiag(const void *pt, void *df, void *da, const int *mnum, int *error) {
    (void) da; (void) mnum;
    void **handle = (void **) pt;
    dense_pds *d = (dense_pds *) handle[0];
    double *out = (double *) df;
    *error = 0;
    if (!d) { *error = -1; return; }
    for (int i = 0; i < d->n; ++i) {
        double l = d->L[(size_t) i * d->n + i];
        out[i] = l * l;
    }
}
