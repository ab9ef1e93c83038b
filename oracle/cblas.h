/*
 * Minimal CBLAS declarations for building the reference tlib::ttm headers
 * against the OpenBLAS shared library that ships inside the
 * opencv-python-headless wheel (which has no header of its own).
 *
 * TEST INFRASTRUCTURE ONLY: used by oracle/Makefile to compile the reference
 * into oracle/_ref/. Nothing in the product path includes this file.
 *
 * The enum values are the ones fixed by the CBLAS standard (netlib cblas.h).
 * The reference's mtm.h:53-66 names the layout type CBLAS_LAYOUT (and
 * CBLAS_ORDER under BLIS), so both names are provided.
 */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

typedef enum { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_LAYOUT;
typedef CBLAS_LAYOUT CBLAS_ORDER;
typedef enum { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 } CBLAS_TRANSPOSE;

void cblas_sgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, float alpha, const float* a, int lda,
                 const float* b, int ldb, float beta, float* c, int ldc);
void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb,
                 int m, int n, int k, double alpha, const double* a, int lda,
                 const double* b, int ldb, double beta, double* c, int ldc);
void cblas_sgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, int m, int n,
                 float alpha, const float* a, int lda, const float* x, int incx,
                 float beta, float* y, int incy);
void cblas_dgemv(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, int m, int n,
                 double alpha, const double* a, int lda, const double* x, int incx,
                 double beta, double* y, int incy);

void openblas_set_num_threads(int num_threads);
int  openblas_get_num_threads(void);

#ifdef __cplusplus
}
#endif
