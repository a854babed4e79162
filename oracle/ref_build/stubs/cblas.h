/* Type-only CBLAS declarations for building the reference library as a test
 * oracle.  Only the enum values and the prototypes that the reference's sources
 * name are declared; the symbols resolve to the OpenBLAS build that ships inside
 * scipy (exported with a "scipy_" prefix), hence the renaming macros. */
#ifndef ORACLE_STUB_CBLAS_H
#define ORACLE_STUB_CBLAS_H
#include <stddef.h>
enum CBLAS_ORDER {CblasRowMajor = 101, CblasColMajor = 102};
enum CBLAS_TRANSPOSE {CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113};
enum CBLAS_UPLO {CblasUpper = 121, CblasLower = 122};
enum CBLAS_DIAG {CblasNonUnit = 131, CblasUnit = 132};
enum CBLAS_SIDE {CblasLeft = 141, CblasRight = 142};
typedef enum CBLAS_ORDER CBLAS_LAYOUT;

#define cblas_dtrmm scipy_cblas_dtrmm
#define cblas_ztrmm scipy_cblas_ztrmm
#define cblas_dtrmv scipy_cblas_dtrmv
#define cblas_dtrsm scipy_cblas_dtrsm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_sgemv scipy_cblas_sgemv
#define cblas_strmm scipy_cblas_strmm
#define cblas_strsm scipy_cblas_strsm

void cblas_dtrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const int, const double, const double *, const int, double *, const int);
void cblas_strmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const int, const float, const float *, const int, float *, const int);
void cblas_ztrmm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const int, const void *, const void *, const int, void *, const int);
void cblas_dtrsm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const int, const double, const double *, const int, double *, const int);
void cblas_strsm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const int, const float, const float *, const int, float *, const int);
void cblas_dtrmv(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, enum CBLAS_DIAG,
                 const int, const double *, const int, double *, const int);
void cblas_dgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, const int, const int, const int,
                 const double, const double *, const int, const double *, const int, const double, double *, const int);
void cblas_sgemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE, const int, const int, const int,
                 const float, const float *, const int, const float *, const int, const float, float *, const int);
void cblas_dgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, const int, const int, const double, const double *, const int,
                 const double *, const int, const double, double *, const int);
void cblas_sgemv(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, const int, const int, const float, const float *, const int,
                 const float *, const int, const float, float *, const int);
#endif
