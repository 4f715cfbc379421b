/*
 * hipblas.h -- the hipBLAS-style C API of hcblas-b200: the GEMM subset of the
 * reference's hipBLAS-on-hcBLAS layer (lib/include/hipblas.h,
 * lib/include/hcc_detail/hip_blas.h, lib/src/hcc_detail/hipblas.cpp), so
 * that HIP-style callers of that layer switch by relinking.  Every function
 * forwards to the hcblas C API (hcblas.h) and maps its status.
 *
 * Streams are CUDA streams (hipStream_t is a cudaStream_t here); handles are
 * hcblas handles.  Divergence from the reference: hipblasCreate(NULL) returns
 * HIPBLAS_STATUS_INVALID_VALUE (the reference allocates a handle it then
 * loses, hipblas.cpp:34-36).
 */
#ifndef HCBLAS_B200_HIPBLAS_H_
#define HCBLAS_B200_HIPBLAS_H_

#include "hcblas.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Reference: lib/include/hcc_detail/hip_blas.h:39. */
typedef hcblasHandle_t hipblasHandle_t;
typedef void *hipStream_t;
typedef hcComplex hipComplex;
typedef hcDoubleComplex hipDoubleComplex;
typedef hcblasHalf hipblasHalf;

/* Reference: lib/include/hipblas.h:38-51 (values in declaration order). */
typedef enum {
  HIPBLAS_STATUS_SUCCESS = 0,
  HIPBLAS_STATUS_NOT_INITIALIZED = 1,
  HIPBLAS_STATUS_ALLOC_FAILED = 2,
  HIPBLAS_STATUS_INVALID_VALUE = 3,
  HIPBLAS_STATUS_ARCH_MISMATCH = 4,
  HIPBLAS_STATUS_MAPPING_ERROR = 5,
  HIPBLAS_STATUS_EXECUTION_FAILED = 6,
  HIPBLAS_STATUS_INTERNAL_ERROR = 7,
  HIPBLAS_STATUS_NOT_SUPPORTED = 8
} hipblasStatus_t;

typedef enum { HIPBLAS_OP_N = 0, HIPBLAS_OP_T = 1, HIPBLAS_OP_C = 2 } hipblasOperation_t;

/* Reference: hipblas.cpp:29-73, 128-130: a handle on the current device's
 * default stream; Set/GetStream bind / read the handle's stream. */
hipblasStatus_t hipblasCreate(hipblasHandle_t *handle);
hipblasStatus_t hipblasDestroy(hipblasHandle_t handle);
hipblasStatus_t hipblasSetStream(hipblasHandle_t handle, hipStream_t stream);
hipblasStatus_t hipblasGetStream(hipblasHandle_t handle, hipStream_t *stream);

/* Reference: hipblas.cpp:132-182 (a temporary handle per call). */
hipblasStatus_t hipblasSetVector(int n, int elemSize, const void *x, int incx, void *y,
                                 int incy);
hipblasStatus_t hipblasGetVector(int n, int elemSize, const void *x, int incx, void *y,
                                 int incy);
hipblasStatus_t hipblasSetMatrix(int rows, int cols, int elemSize, const void *A, int lda,
                                 void *B, int ldb);
hipblasStatus_t hipblasGetMatrix(int rows, int cols, int elemSize, const void *A, int lda,
                                 void *B, int ldb);

/* Reference: hipblas.cpp:428-500 (column-major; forwards to hcblasXgemm). */
hipblasStatus_t hipblasSgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k, const float *alpha,
                             const float *A, int lda, const float *B, int ldb, const float *beta,
                             float *C, int ldc);
hipblasStatus_t hipblasDgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k, const double *alpha,
                             const double *A, int lda, const double *B, int ldb,
                             const double *beta, double *C, int ldc);
hipblasStatus_t hipblasCgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipComplex *alpha, const hipComplex *A, int lda,
                             const hipComplex *B, int ldb, const hipComplex *beta,
                             hipComplex *C, int ldc);
hipblasStatus_t hipblasZgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipDoubleComplex *alpha, const hipDoubleComplex *A, int lda,
                             const hipDoubleComplex *B, int ldb, const hipDoubleComplex *beta,
                             hipDoubleComplex *C, int ldc);
hipblasStatus_t hipblasHgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipblasHalf *alpha, const hipblasHalf *A, int lda,
                             const hipblasHalf *B, int ldb, const hipblasHalf *beta,
                             hipblasHalf *C, int ldc);

/* Reference: hipblas.cpp:501-553 (device-resident pointer arrays). */
hipblasStatus_t hipblasSgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const float *alpha, const float *A[], int lda,
                                    const float *B[], int ldb, const float *beta, float *C[],
                                    int ldc, int batchCount);
hipblasStatus_t hipblasDgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const double *alpha, const double *A[], int lda,
                                    const double *B[], int ldb, const double *beta,
                                    double *C[], int ldc, int batchCount);
hipblasStatus_t hipblasCgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const hipComplex *alpha, const hipComplex *A[], int lda,
                                    const hipComplex *B[], int ldb, const hipComplex *beta,
                                    hipComplex *C[], int ldc, int batchCount);
hipblasStatus_t hipblasZgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const hipDoubleComplex *alpha, const hipDoubleComplex *A[],
                                    int lda, const hipDoubleComplex *B[], int ldb,
                                    const hipDoubleComplex *beta, hipDoubleComplex *C[],
                                    int ldc, int batchCount);

/* Extension (later hipBLAS releases have it; the reference layer does not):
 * strided batches, forwarding to hcblasXgemmStridedBatched. */
hipblasStatus_t hipblasSgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const float *alpha, const float *A, int lda,
                                           long long strideA, const float *B, int ldb,
                                           long long strideB, const float *beta, float *C,
                                           int ldc, long long strideC, int batchCount);
hipblasStatus_t hipblasDgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const double *alpha, const double *A, int lda,
                                           long long strideA, const double *B, int ldb,
                                           long long strideB, const double *beta, double *C,
                                           int ldc, long long strideC, int batchCount);
hipblasStatus_t hipblasHgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const hipblasHalf *alpha, const hipblasHalf *A,
                                           int lda, long long strideA, const hipblasHalf *B,
                                           int ldb, long long strideB, const hipblasHalf *beta,
                                           hipblasHalf *C, int ldc, long long strideC,
                                           int batchCount);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* HCBLAS_B200_HIPBLAS_H_ */
