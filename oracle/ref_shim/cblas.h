/* TEST INFRASTRUCTURE ONLY (oracle/_ref build).  CBLAS prototypes (the
 * standard netlib CBLAS interface) for exactly the routines the reference
 * calls, resolved to the "scipy_"-prefixed exports of the OpenBLAS library
 * that ships inside scipy (no system BLAS exists here).  Optionally counts
 * the calls when FRANK_ORACLE_COUNT is defined. */
#ifndef FRANK_ORACLE_CBLAS_SHIM_H
#define FRANK_ORACLE_CBLAS_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

void scipy_cblas_dswap(const int n, double* x, const int incx, double* y, const int incy);
void scipy_cblas_dcopy(const int n, const double* x, const int incx, double* y, const int incy);
void scipy_cblas_dscal(const int n, const double alpha, double* x, const int incx);
double scipy_cblas_ddot(const int n, const double* x, const int incx, const double* y, const int incy);
void scipy_cblas_daxpy(const int n, const double alpha, const double* x, const int incx, double* y, const int incy);
double scipy_cblas_dnrm2(const int n, const double* x, const int incx);
void scipy_cblas_dgemv(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE trans, const int m, const int n,
                       const double alpha, const double* a, const int lda, const double* x, const int incx,
                       const double beta, double* y, const int incy);
void scipy_cblas_dger(const enum CBLAS_ORDER order, const int m, const int n, const double alpha, const double* x,
                      const int incx, const double* y, const int incy, double* a, const int lda);
void scipy_cblas_dgemm(const enum CBLAS_ORDER order, const enum CBLAS_TRANSPOSE ta, const enum CBLAS_TRANSPOSE tb,
                       const int m, const int n, const int k, const double alpha, const double* a, const int lda,
                       const double* b, const int ldb, const double beta, double* c, const int ldc);
void scipy_cblas_dtrmm(const enum CBLAS_ORDER order, const enum CBLAS_SIDE side, const enum CBLAS_UPLO uplo,
                       const enum CBLAS_TRANSPOSE ta, const enum CBLAS_DIAG diag, const int m, const int n,
                       const double alpha, const double* a, const int lda, double* b, const int ldb);
void scipy_cblas_dtrsm(const enum CBLAS_ORDER order, const enum CBLAS_SIDE side, const enum CBLAS_UPLO uplo,
                       const enum CBLAS_TRANSPOSE ta, const enum CBLAS_DIAG diag, const int m, const int n,
                       const double alpha, const double* a, const int lda, double* b, const int ldb);
void scipy_openblas_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#define cblas_dswap scipy_cblas_dswap
#define cblas_dcopy scipy_cblas_dcopy
#define cblas_dscal scipy_cblas_dscal
#define cblas_ddot scipy_cblas_ddot
#define cblas_daxpy scipy_cblas_daxpy
#define cblas_dnrm2 scipy_cblas_dnrm2
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_dger scipy_cblas_dger
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dtrmm scipy_cblas_dtrmm
#define cblas_dtrsm scipy_cblas_dtrsm

#endif
