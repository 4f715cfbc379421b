/*
 * hcblaslib.h -- C++ class API of hcblas-b200 (GEMM hot path of hcBLAS).
 *
 * Mirrors `struct Hcblaslibrary` of the reference (lib/include/hcblaslib.h:
 * 67-479): the same public fields (tests read handle->Order,
 * handle->currentAccl, handle->currentAcclView: test/unit-api/test-blas.cpp:
 * 1869,1877,1922) and the same hcblas_{s,d,h,c,z}gemm method signatures,
 * including the row-major order, the element offsets aOffset/bOffset/cOffset
 * and the batched overloads.  Methods return HCBLAS_SUCCEEDS or
 * HCBLAS_INVALID exactly where the reference does (quick return on a NULL
 * matrix or M, N or K == 0: sgemm_array_wrapper.cpp:307-309).
 *
 * B200 additions live behind `impl` (math mode, workspace, tuned-config
 * cache); they do not change the public layout the reference exposes.
 */
#ifndef HCBLAS_B200_HCBLASLIB_H_
#define HCBLAS_B200_HCBLASLIB_H_

#include <stdint.h>

#include "hc_compat.h"

/* Reference: lib/include/hcblaslib.h:44-51. */
enum hcblasStatus { HCBLAS_SUCCEEDS = 0, HCBLAS_INVALID = -1 };
enum hcblasOrder : unsigned short { RowMajor, ColMajor };
/* 'c' (conjugate transpose) is an extension; the reference maps every non-N
 * operation to 't' (lib/src/hcblas.cpp:1318-1319). */
enum hcblasTranspose { NoTrans = 'n', Trans = 't', ConjTrans = 'c' };

struct HcblasB200State;

struct Hcblaslibrary {
 public:
  /* Reference: lib/include/hcblaslib.h:70-83.  Checks that the view's device
   * exists; Order starts as ColMajor. */
  explicit Hcblaslibrary(hc::accelerator_view *av);
  ~Hcblaslibrary();
  Hcblaslibrary(const Hcblaslibrary &) = delete;
  Hcblaslibrary &operator=(const Hcblaslibrary &) = delete;

  hc::accelerator currentAccl;
  bool initialized = false;
  hc::accelerator_view currentAcclView;
  void *currentStream = nullptr;
  hcblasOrder Order;

  /* B200 state: math mode, workspaces, tuned configs, last path taken. */
  HcblasB200State *impl = nullptr;

  /* SGEMM (reference: hcblaslib.h:215-222) */
  hcblasStatus hcblas_sgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const float &alpha, float *A,
                            const int64_t lda, float *B, const int64_t ldb, const float &beta,
                            float *C, const int64_t ldc, const int64_t aOffset,
                            const int64_t bOffset, const int64_t cOffset);

  /* DGEMM (reference: hcblaslib.h:224-231) */
  hcblasStatus hcblas_dgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const double &alpha, double *A,
                            const int64_t lda, double *B, const int64_t ldb,
                            const double &beta, double *C, const int64_t ldc,
                            const int64_t aOffset, const int64_t bOffset,
                            const int64_t cOffset);

  /* HGEMM (reference: hcblaslib.h:233-241) */
  hcblasStatus hcblas_hgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::half &alpha, hc::half *A,
                            const int64_t lda, hc::half *B, const int64_t ldb,
                            const hc::half &beta, hc::half *C, const int64_t ldc,
                            const int64_t aOffset, const int64_t bOffset,
                            const int64_t cOffset);

  /* Batched overloads (reference: hcblaslib.h:244-266).  Matrix i is
   * X[i] + xOffset + i * X_batchOffset: with distinct pointers and
   * X_batchOffset = 0 this is the reference's pointer-array batch; with one
   * repeated base pointer and X_batchOffset = stride it is a strided batch. */
  hcblasStatus hcblas_sgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const float &alpha, float *A[],
                            const int64_t lda, const int64_t A_batchOffset, float *B[],
                            const int64_t ldb, const int64_t B_batchOffset, const float &beta,
                            float *C[], const int64_t ldc, const int64_t C_batchOffset,
                            const int64_t aOffset, const int64_t bOffset,
                            const int64_t cOffset, const int batchSize);

  hcblasStatus hcblas_dgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const double &alpha, double *A[],
                            const int64_t lda, const int64_t A_batchOffset, double *B[],
                            const int64_t ldb, const int64_t B_batchOffset,
                            const double &beta, double *C[], const int64_t ldc,
                            const int64_t C_batchOffset, const int64_t aOffset,
                            const int64_t bOffset, const int64_t cOffset,
                            const int batchSize);

  /* Extension: HGEMM batch (compiled but unreachable in the reference). */
  hcblasStatus hcblas_hgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::half &alpha, hc::half *A[],
                            const int64_t lda, const int64_t A_batchOffset, hc::half *B[],
                            const int64_t ldb, const int64_t B_batchOffset,
                            const hc::half &beta, hc::half *C[], const int64_t ldc,
                            const int64_t C_batchOffset, const int64_t aOffset,
                            const int64_t bOffset, const int64_t cOffset,
                            const int batchSize);

  /* CGEMM / ZGEMM (reference: hcblaslib.h:269-291); note the complex
   * argument order (X, xOffset, ldx). */
  hcblasStatus hcblas_cgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::short_vector::float_2 &alpha,
                            hc::short_vector::float_2 *A, const int64_t aOffset,
                            const int64_t lda, hc::short_vector::float_2 *B,
                            const int64_t bOffset, const int64_t ldb,
                            const hc::short_vector::float_2 &beta,
                            hc::short_vector::float_2 *C, const int64_t cOffset,
                            const int64_t ldc);

  hcblasStatus hcblas_zgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::short_vector::double_2 &alpha,
                            hc::short_vector::double_2 *A, const int64_t aOffset,
                            const int64_t lda, hc::short_vector::double_2 *B,
                            const int64_t bOffset, const int64_t ldb,
                            const hc::short_vector::double_2 &beta,
                            hc::short_vector::double_2 *C, const int64_t cOffset,
                            const int64_t ldc);

  /* Complex batched (reference: hcblaslib.h:294-315). */
  hcblasStatus hcblas_cgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::short_vector::float_2 &alpha,
                            hc::short_vector::float_2 *A[], const int64_t aOffset,
                            const int64_t A_batchOffset, const int64_t lda,
                            hc::short_vector::float_2 *B[], const int64_t bOffset,
                            const int64_t B_batchOffset, const int64_t ldb,
                            const hc::short_vector::float_2 &beta,
                            hc::short_vector::float_2 *C[], const int64_t cOffset,
                            const int64_t C_batchOffset, const int64_t ldc,
                            const int batchSize);

  hcblasStatus hcblas_zgemm(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose typeA, hcblasTranspose typeB, const int M,
                            const int N, const int K, const hc::short_vector::double_2 &alpha,
                            hc::short_vector::double_2 *A[], const int64_t aOffset,
                            const int64_t A_batchOffset, const int64_t lda,
                            hc::short_vector::double_2 *B[], const int64_t bOffset,
                            const int64_t B_batchOffset, const int64_t ldb,
                            const hc::short_vector::double_2 &beta,
                            hc::short_vector::double_2 *C[], const int64_t cOffset,
                            const int64_t C_batchOffset, const int64_t ldc,
                            const int batchSize);

  /* GEMV / GER (reference lib/include/hcblaslib.h:140-230): y = alpha op(A) x
   * + beta y and A = alpha x y^T + A, element offsets, strided batches with
   * explicit batch offsets.  Quick returns as the reference's
   * (sgemv_array.cpp:833-836, sger_array.cpp:134-141): a NULL vector or
   * matrix, M or N <= 0, or (GEMV) an increment <= 0 / (GER) == 0 ->
   * HCBLAS_INVALID; GER with alpha == 0 leaves A untouched.  Unlike the
   * reference, lda is honoured (the reference assumes lda == M). */
  hcblasStatus hcblas_sgemv(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose type, const int M, const int N, const float &alpha,
                            float *A, const int64_t aOffset, const int lda, float *X,
                            const int64_t xOffset, const int incX, const float &beta, float *Y,
                            const int64_t yOffset, const int incY);
  hcblasStatus hcblas_sgemv(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose type, const int M, const int N, const float &alpha,
                            float *A, const int64_t aOffset, const int64_t A_batchOffset,
                            const int lda, float *X, const int64_t xOffset,
                            const int64_t X_batchOffset, const int incX, const float &beta,
                            float *Y, const int64_t yOffset, const int64_t Y_batchOffset,
                            const int incY, const int batchSize);
  hcblasStatus hcblas_dgemv(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose type, const int M, const int N, const double &alpha,
                            double *A, const int64_t aOffset, const int lda, double *X,
                            const int64_t xOffset, const int incX, const double &beta,
                            double *Y, const int64_t yOffset, const int incY);
  hcblasStatus hcblas_dgemv(hc::accelerator_view accl_view, hcblasOrder order,
                            hcblasTranspose type, const int M, const int N, const double &alpha,
                            double *A, const int64_t aOffset, const int64_t A_batchOffset,
                            const int lda, double *X, const int64_t xOffset,
                            const int64_t X_batchOffset, const int incX, const double &beta,
                            double *Y, const int64_t yOffset, const int64_t Y_batchOffset,
                            const int incY, const int batchSize);
  hcblasStatus hcblas_sger(hc::accelerator_view accl_view, hcblasOrder order, const int M,
                           const int N, const float &alpha, const float *X,
                           const int64_t xOffset, const int incX, const float *Y,
                           const int64_t yOffset, const int incY, float *A,
                           const int64_t aOffset, const int lda);
  hcblasStatus hcblas_sger(hc::accelerator_view accl_view, hcblasOrder order, const int M,
                           const int N, const float &alpha, const float *X,
                           const int64_t xOffset, const int64_t X_batchOffset, const int incX,
                           const float *Y, const int64_t yOffset, const int64_t Y_batchOffset,
                           const int incY, float *A, const int64_t aOffset,
                           const int64_t A_batchOffset, const int lda, const int batchSize);
  hcblasStatus hcblas_dger(hc::accelerator_view accl_view, hcblasOrder order, const int M,
                           const int N, const double &alpha, const double *X,
                           const int64_t xOffset, const int incX, const double *Y,
                           const int64_t yOffset, const int incY, double *A,
                           const int64_t aOffset, const int lda);
  hcblasStatus hcblas_dger(hc::accelerator_view accl_view, hcblasOrder order, const int M,
                           const int N, const double &alpha, const double *X,
                           const int64_t xOffset, const int64_t X_batchOffset, const int incX,
                           const double *Y, const int64_t yOffset, const int64_t Y_batchOffset,
                           const int incY, double *A, const int64_t aOffset,
                           const int64_t A_batchOffset, const int lda, const int batchSize);
};

#endif /* HCBLAS_B200_HCBLASLIB_H_ */
