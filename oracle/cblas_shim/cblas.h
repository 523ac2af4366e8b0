/*
 * Minimal CBLAS declarations for building the reference's cblas linalg
 * backend (libtensor/linalg/cblas/cblas_h.h includes <cblas.h>).  No cblas.h
 * is installed in this image; the symbols come from the OpenBLAS shared
 * library shipped inside the Python environment.  Test infrastructure only.
 */
#ifndef LTG_ORACLE_CBLAS_SHIM_H
#define LTG_ORACLE_CBLAS_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_ORDER CBLAS_LAYOUT;
void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
                 const int, const int, const int, const double, const double *,
                 const int, const double *, const int, const double, double *,
                 const int);
void cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, const int, const int,
                 const double, const double *, const int, const double *,
                 const int, const double, double *, const int);
void cblas_dger(enum CBLAS_ORDER, const int, const int, const double,
                const double *, const int, const double *, const int, double *,
                const int);
double cblas_ddot(const int, const double *, const int, const double *, const int);
void cblas_daxpy(const int, const double, const double *, const int, double *, const int);
void cblas_dcopy(const int, const double *, const int, double *, const int);
void cblas_dscal(const int, const double, double *, const int);
void openblas_set_num_threads(int);
#ifdef __cplusplus
}
#endif
#endif
