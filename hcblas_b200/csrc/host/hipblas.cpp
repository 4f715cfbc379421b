/*
 * hipblas.cpp -- the hipBLAS-style GEMM API (include/hipblas.h) over the
 * hcblas C API: operation and status codes are translated, everything else
 * is forwarded unchanged (reference layer: lib/src/hcc_detail/hipblas.cpp).
 */
#include <cuda_runtime.h>

#include "../../../include/hipblas.h"

namespace {

hcblasOperation_t to_hc(hipblasOperation_t op) {
  switch (op) {
    case HIPBLAS_OP_N: return HCBLAS_OP_N;
    case HIPBLAS_OP_T: return HCBLAS_OP_T;
    default: return HCBLAS_OP_C;
  }
}

bool op_ok(hipblasOperation_t op) {
  return op == HIPBLAS_OP_N || op == HIPBLAS_OP_T || op == HIPBLAS_OP_C;
}

/* reference: hipblas.cpp:107-126 */
hipblasStatus_t to_hip(hcblasStatus_t s) {
  switch (s) {
    case HCBLAS_STATUS_SUCCESS: return HIPBLAS_STATUS_SUCCESS;
    case HCBLAS_STATUS_NOT_INITIALIZED: return HIPBLAS_STATUS_NOT_INITIALIZED;
    case HCBLAS_STATUS_ALLOC_FAILED: return HIPBLAS_STATUS_ALLOC_FAILED;
    case HCBLAS_STATUS_INVALID_VALUE: return HIPBLAS_STATUS_INVALID_VALUE;
    case HCBLAS_STATUS_MAPPING_ERROR: return HIPBLAS_STATUS_MAPPING_ERROR;
    case HCBLAS_STATUS_EXECUTION_FAILED: return HIPBLAS_STATUS_EXECUTION_FAILED;
    case HCBLAS_STATUS_INTERNAL_ERROR: return HIPBLAS_STATUS_INTERNAL_ERROR;
    default: return HIPBLAS_STATUS_INTERNAL_ERROR;
  }
}

/* run `fn(handle)` on a temporary handle (the reference's host-copy helpers) */
template <typename F>
hipblasStatus_t with_temp_handle(F &&fn) {
  hipblasHandle_t h = nullptr;
  hipblasStatus_t s = hipblasCreate(&h);
  if (s == HIPBLAS_STATUS_SUCCESS) s = to_hip(fn(h));
  if (h) hipblasDestroy(h);
  return s;
}

}  // namespace

#define HIP_OPS_CHECK()                                 \
  if (!op_ok(transa) || !op_ok(transb)) return HIPBLAS_STATUS_INVALID_VALUE;

extern "C" {

hipblasStatus_t hipblasCreate(hipblasHandle_t *handle) {
  if (handle == nullptr) return HIPBLAS_STATUS_INVALID_VALUE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    *handle = nullptr;
    return HIPBLAS_STATUS_NOT_INITIALIZED;
  }
  hcblas_accl_view_t view;
  view.device_id = dev;
  view.stream = nullptr;
  return to_hip(hcblasCreate(handle, &view));
}

hipblasStatus_t hipblasDestroy(hipblasHandle_t handle) {
  if (handle == nullptr) return HIPBLAS_STATUS_NOT_INITIALIZED;
  return to_hip(hcblasDestroy(&handle));
}

hipblasStatus_t hipblasSetStream(hipblasHandle_t handle, hipStream_t stream) {
  if (handle == nullptr) return HIPBLAS_STATUS_NOT_INITIALIZED;
  return to_hip(hcblasSetStream(handle, stream));
}

hipblasStatus_t hipblasGetStream(hipblasHandle_t handle, hipStream_t *stream) {
  if (handle == nullptr) return HIPBLAS_STATUS_NOT_INITIALIZED;
  if (stream == nullptr) return HIPBLAS_STATUS_INVALID_VALUE;
  hcblas_accl_view_t *view = nullptr;
  return to_hip(hcblasGetAcclView(handle, &view, stream));
}

hipblasStatus_t hipblasSetVector(int n, int elemSize, const void *x, int incx, void *y,
                                 int incy) {
  return with_temp_handle(
      [&](hipblasHandle_t h) { return hcblasSetVector(h, n, elemSize, x, incx, y, incy); });
}

hipblasStatus_t hipblasGetVector(int n, int elemSize, const void *x, int incx, void *y,
                                 int incy) {
  return with_temp_handle(
      [&](hipblasHandle_t h) { return hcblasGetVector(h, n, elemSize, x, incx, y, incy); });
}

hipblasStatus_t hipblasSetMatrix(int rows, int cols, int elemSize, const void *A, int lda,
                                 void *B, int ldb) {
  return with_temp_handle([&](hipblasHandle_t h) {
    return hcblasSetMatrix(h, rows, cols, elemSize, A, lda, B, ldb);
  });
}

hipblasStatus_t hipblasGetMatrix(int rows, int cols, int elemSize, const void *A, int lda,
                                 void *B, int ldb) {
  return with_temp_handle([&](hipblasHandle_t h) {
    return hcblasGetMatrix(h, rows, cols, elemSize, A, lda, B, ldb);
  });
}

hipblasStatus_t hipblasSgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k, const float *alpha,
                             const float *A, int lda, const float *B, int ldb, const float *beta,
                             float *C, int ldc) {
  HIP_OPS_CHECK()
  return to_hip(hcblasSgemm(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                            const_cast<float *>(A), lda, const_cast<float *>(B), ldb, beta, C,
                            ldc));
}

hipblasStatus_t hipblasDgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k, const double *alpha,
                             const double *A, int lda, const double *B, int ldb,
                             const double *beta, double *C, int ldc) {
  HIP_OPS_CHECK()
  return to_hip(hcblasDgemm(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                            const_cast<double *>(A), lda, const_cast<double *>(B), ldb, beta, C,
                            ldc));
}

hipblasStatus_t hipblasCgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipComplex *alpha, const hipComplex *A, int lda,
                             const hipComplex *B, int ldb, const hipComplex *beta,
                             hipComplex *C, int ldc) {
  HIP_OPS_CHECK()
  return to_hip(hcblasCgemm(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                            const_cast<hipComplex *>(A), lda, const_cast<hipComplex *>(B), ldb,
                            beta, C, ldc));
}

hipblasStatus_t hipblasZgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipDoubleComplex *alpha, const hipDoubleComplex *A, int lda,
                             const hipDoubleComplex *B, int ldb, const hipDoubleComplex *beta,
                             hipDoubleComplex *C, int ldc) {
  HIP_OPS_CHECK()
  return to_hip(hcblasZgemm(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                            const_cast<hipDoubleComplex *>(A), lda,
                            const_cast<hipDoubleComplex *>(B), ldb, beta, C, ldc));
}

hipblasStatus_t hipblasHgemm(hipblasHandle_t handle, hipblasOperation_t transa,
                             hipblasOperation_t transb, int m, int n, int k,
                             const hipblasHalf *alpha, const hipblasHalf *A, int lda,
                             const hipblasHalf *B, int ldb, const hipblasHalf *beta,
                             hipblasHalf *C, int ldc) {
  HIP_OPS_CHECK()
  return to_hip(hcblasHgemm(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                            const_cast<hipblasHalf *>(A), lda, const_cast<hipblasHalf *>(B), ldb,
                            beta, C, ldc));
}

hipblasStatus_t hipblasSgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const float *alpha, const float *A[], int lda,
                                    const float *B[], int ldb, const float *beta, float *C[],
                                    int ldc, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasSgemmBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                   const_cast<float **>(A), lda, const_cast<float **>(B), ldb,
                                   beta, C, ldc, batchCount));
}

hipblasStatus_t hipblasDgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const double *alpha, const double *A[], int lda,
                                    const double *B[], int ldb, const double *beta,
                                    double *C[], int ldc, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasDgemmBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                   const_cast<double **>(A), lda, const_cast<double **>(B), ldb,
                                   beta, C, ldc, batchCount));
}

hipblasStatus_t hipblasCgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const hipComplex *alpha, const hipComplex *A[], int lda,
                                    const hipComplex *B[], int ldb, const hipComplex *beta,
                                    hipComplex *C[], int ldc, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasCgemmBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                   const_cast<hipComplex **>(A), lda,
                                   const_cast<hipComplex **>(B), ldb, beta, C, ldc, batchCount));
}

hipblasStatus_t hipblasZgemmBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                    hipblasOperation_t transb, int m, int n, int k,
                                    const hipDoubleComplex *alpha, const hipDoubleComplex *A[],
                                    int lda, const hipDoubleComplex *B[], int ldb,
                                    const hipDoubleComplex *beta, hipDoubleComplex *C[],
                                    int ldc, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasZgemmBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                   const_cast<hipDoubleComplex **>(A), lda,
                                   const_cast<hipDoubleComplex **>(B), ldb, beta, C, ldc,
                                   batchCount));
}

hipblasStatus_t hipblasSgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const float *alpha, const float *A, int lda,
                                           long long strideA, const float *B, int ldb,
                                           long long strideB, const float *beta, float *C,
                                           int ldc, long long strideC, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasSgemmStridedBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                          A, lda, strideA, B, ldb, strideB, beta, C, ldc,
                                          strideC, batchCount));
}

hipblasStatus_t hipblasDgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const double *alpha, const double *A, int lda,
                                           long long strideA, const double *B, int ldb,
                                           long long strideB, const double *beta, double *C,
                                           int ldc, long long strideC, int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasDgemmStridedBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                          A, lda, strideA, B, ldb, strideB, beta, C, ldc,
                                          strideC, batchCount));
}

hipblasStatus_t hipblasHgemmStridedBatched(hipblasHandle_t handle, hipblasOperation_t transa,
                                           hipblasOperation_t transb, int m, int n, int k,
                                           const hipblasHalf *alpha, const hipblasHalf *A,
                                           int lda, long long strideA, const hipblasHalf *B,
                                           int ldb, long long strideB, const hipblasHalf *beta,
                                           hipblasHalf *C, int ldc, long long strideC,
                                           int batchCount) {
  HIP_OPS_CHECK()
  return to_hip(hcblasHgemmStridedBatched(handle, to_hc(transa), to_hc(transb), m, n, k, alpha,
                                          A, lda, strideA, B, ldb, strideB, beta, C, ldc,
                                          strideC, batchCount));
}

}  // extern "C"
