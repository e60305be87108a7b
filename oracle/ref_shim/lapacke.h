/* TEST INFRASTRUCTURE ONLY (oracle/_ref build).  LAPACKE prototypes (the
 * standard netlib LAPACKE interface, 32-bit lapack_int) for exactly the
 * routines the reference calls, resolved to the "scipy_"-prefixed exports of
 * the OpenBLAS library that ships inside scipy. */
#ifndef FRANK_ORACLE_LAPACKE_SHIM_H
#define FRANK_ORACLE_LAPACKE_SHIM_H

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102
typedef int lapack_int;

#ifdef __cplusplus
extern "C" {
#endif

lapack_int scipy_LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv);
lapack_int scipy_LAPACKE_dgeqrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, double* tau);
lapack_int scipy_LAPACKE_dorgqr(int layout, lapack_int m, lapack_int n, lapack_int k, double* a, lapack_int lda,
                                const double* tau);
lapack_int scipy_LAPACKE_dgerqf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, double* tau);
lapack_int scipy_LAPACKE_dorgrq(int layout, lapack_int m, lapack_int n, lapack_int k, double* a, lapack_int lda,
                                const double* tau);
lapack_int scipy_LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double* a,
                                lapack_int lda, double* s, double* u, lapack_int ldu, double* vt, lapack_int ldvt,
                                double* superb);
lapack_int scipy_LAPACKE_dgeqp3(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* jpvt,
                                double* tau);
lapack_int scipy_LAPACKE_dlarfg(lapack_int n, double* alpha, double* x, lapack_int incx, double* tau);
double scipy_LAPACKE_dlamch(char cmach);
double scipy_LAPACKE_dlange(int layout, char norm, lapack_int m, lapack_int n, const double* a, lapack_int lda);
lapack_int scipy_LAPACKE_dlatms(int layout, lapack_int m, lapack_int n, char dist, lapack_int* iseed, char sym,
                                double* d, lapack_int mode, double cond, double dmax, lapack_int kl, lapack_int ku,
                                char pack, double* a, lapack_int lda);
lapack_int scipy_LAPACKE_dtpqrt2(int layout, lapack_int m, lapack_int n, lapack_int l, double* a, lapack_int lda,
                                 double* b, lapack_int ldb, double* t, lapack_int ldt);
lapack_int scipy_LAPACKE_dgeqrt3(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, double* t,
                                 lapack_int ldt);
lapack_int scipy_LAPACKE_dlarfb(int layout, char side, char trans, char direct, char storev, lapack_int m,
                                lapack_int n, lapack_int k, const double* v, lapack_int ldv, const double* t,
                                lapack_int ldt, double* c, lapack_int ldc);
lapack_int scipy_LAPACKE_dtprfb(int layout, char side, char trans, char direct, char storev, lapack_int m,
                                lapack_int n, lapack_int k, lapack_int l, const double* v, lapack_int ldv,
                                const double* t, lapack_int ldt, double* a, lapack_int lda, double* b,
                                lapack_int ldb);

#ifdef __cplusplus
}
#endif

#define LAPACKE_dgetrf scipy_LAPACKE_dgetrf
#define LAPACKE_dgeqrf scipy_LAPACKE_dgeqrf
#define LAPACKE_dorgqr scipy_LAPACKE_dorgqr
#define LAPACKE_dgerqf scipy_LAPACKE_dgerqf
#define LAPACKE_dorgrq scipy_LAPACKE_dorgrq
#define LAPACKE_dgesvd scipy_LAPACKE_dgesvd
#define LAPACKE_dgeqp3 scipy_LAPACKE_dgeqp3
#define LAPACKE_dlarfg scipy_LAPACKE_dlarfg
#define LAPACKE_dlamch scipy_LAPACKE_dlamch
#define LAPACKE_dlange scipy_LAPACKE_dlange
#define LAPACKE_dlatms scipy_LAPACKE_dlatms
#define LAPACKE_dtpqrt2 scipy_LAPACKE_dtpqrt2
#define LAPACKE_dgeqrt3 scipy_LAPACKE_dgeqrt3
#define LAPACKE_dlarfb scipy_LAPACKE_dlarfb
#define LAPACKE_dtprfb scipy_LAPACKE_dtprfb

#endif
