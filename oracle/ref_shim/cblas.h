/* cblas.h shim for compiling the reference against the scipy-bundled
 * OpenBLAS, whose exported symbols are prefixed with `scipy_`.  Declares only
 * what the reference's streaming driver calls (cblas_dgemm / cblas_sgemm). */
#ifndef ORACLE_CBLAS_SHIM_H
#define ORACLE_CBLAS_SHIM_H
#ifdef __cplusplus
extern "C" {
#endif
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void scipy_cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
    int, int, int, double, const double *, int, const double *, int, double,
    double *, int);
void scipy_cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,
    int, int, int, float, const float *, int, const float *, int, float,
    float *, int);
#ifdef __cplusplus
}
#endif
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_sgemm scipy_cblas_sgemm
#endif
