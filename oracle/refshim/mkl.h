// TEST INFRASTRUCTURE ONLY -- used to compile the reference's own sources into
// oracle/_ref/ (the checker); nothing in the product includes it.
//
// The subset of oneMKL's CBLAS / LAPACKE interface that the reference calls:
//   cblas_zgemm, cblas_dgemm          src/LinearAlgebra/gemm.hpp:12-29
//   cblas_zgemm_batch_strided         src/Operator/BlockMatrix_definitions.hpp:160-170
//   LAPACKE_zheevd ('V','U')          src/Geometry/Matrix.cpp:9-23
//   LAPACKE_[dz]getrf / [dz]getri     src/Geometry/Matrix.cpp:25-98
//   LAPACKE_dgesvd ('A','A')          src/Geometry/Matrix.cpp:100-126
//   mkl_get_max_threads / set         src/initialize.cpp:33-47
// Row-major layout only (the only one the reference uses).  The callers
// define MKL_Complex16 as std::complex<double> before including this file.
#pragma once
#include <complex>

#ifndef MKL_Complex16
#define MKL_Complex16 std::complex<double>
#endif
#ifndef MKL_Complex8
#define MKL_Complex8 std::complex<float>
#endif

typedef int lapack_int;
typedef int MKL_INT;

enum CBLAS_LAYOUT { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
typedef enum CBLAS_LAYOUT CBLAS_ORDER;

#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

void cblas_dgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m, MKL_INT n, MKL_INT k,
                 double alpha, const double* a, MKL_INT lda, const double* b, MKL_INT ldb, double beta,
                 double* c, MKL_INT ldc);
void cblas_zgemm(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m, MKL_INT n, MKL_INT k,
                 const void* alpha, const void* a, MKL_INT lda, const void* b, MKL_INT ldb, const void* beta,
                 void* c, MKL_INT ldc);
void cblas_zgemm_batch_strided(CBLAS_LAYOUT layout, CBLAS_TRANSPOSE ta, CBLAS_TRANSPOSE tb, MKL_INT m,
                               MKL_INT n, MKL_INT k, const void* alpha, const void* a, MKL_INT lda,
                               MKL_INT stridea, const void* b, MKL_INT ldb, MKL_INT strideb, const void* beta,
                               void* c, MKL_INT ldc, MKL_INT stridec, MKL_INT batch);

lapack_int LAPACKE_zheevd(int layout, char jobz, char uplo, lapack_int n, MKL_Complex16* a, lapack_int lda,
                          double* w);
lapack_int LAPACKE_dsyev(int layout, char jobz, char uplo, lapack_int n, double* a, lapack_int lda, double* w);
lapack_int LAPACKE_dgetrf(int layout, lapack_int m, lapack_int n, double* a, lapack_int lda, lapack_int* ipiv);
lapack_int LAPACKE_dgetri(int layout, lapack_int n, double* a, lapack_int lda, const lapack_int* ipiv);
lapack_int LAPACKE_zgetrf(int layout, lapack_int m, lapack_int n, MKL_Complex16* a, lapack_int lda,
                          lapack_int* ipiv);
lapack_int LAPACKE_zgetri(int layout, lapack_int n, MKL_Complex16* a, lapack_int lda, const lapack_int* ipiv);
lapack_int LAPACKE_dgesvd(int layout, char jobu, char jobvt, lapack_int m, lapack_int n, double* a,
                          lapack_int lda, double* s, double* u, lapack_int ldu, double* vt, lapack_int ldvt,
                          double* superb);

int mkl_get_max_threads(void);
void mkl_set_num_threads(int n);
