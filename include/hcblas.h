/*
 * hcblas.h -- C ABI of hcblas-b200, a B200 (sm_100a) drop-in for the GEMM
 * hot path of hcBLAS.
 *
 * Every entry point below keeps the name, parameter list, argument meaning
 * and status codes of the hcBLAS C API it replaces (lib/include/hcblas.h of
 * the reference; file:line given per function).  The functions are exported
 * with C linkage (plain pointers and sizes), so the same symbols serve C++
 * callers that include this header, C callers, and FFI bindings (ctypes,
 * cffi, JNI, cgo) alike.  Entries marked "extension" have no counterpart in
 * the reference's C API.
 *
 * Semantics.  hcblas{S,D,C,Z,H}gemm compute C := alpha*op(A)*op(B) + beta*C
 * in column-major order (the reference's handle order, hcblaslib.h:82) with
 * CBLAS numerics: HCBLAS_OP_C is a true conjugate transpose, beta == 0 means
 * C is not read.  Status codes follow the reference exactly
 * (lib/src/hcblas.cpp:1304-1327): NULL/destroyed handle -> NOT_INITIALIZED;
 * m, n, k (or batchCount) < 0 -> INVALID_VALUE; m, n or k == 0, or a NULL
 * matrix -> EXECUTION_FAILED (the class layer's HCBLAS_INVALID quick return,
 * sgemm_array_wrapper.cpp:307-309); launch failure -> EXECUTION_FAILED.
 * Calls are asynchronous on the handle's stream.
 */
#ifndef HCBLAS_B200_HCBLAS_H_
#define HCBLAS_B200_HCBLAS_H_

#include <stddef.h>
#include <stdint.h>

#include "hc_compat.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque library context (reference: lib/include/hcblas.h:46). */
typedef struct Hcblaslibrary *hcblasHandle_t;

/* Status and operation codes (reference: lib/include/hcblas.h:56-78).  The
 * reference declares them as C++ enums with unsigned short storage; the C
 * view uses the same storage type so both sides share one ABI. */
#ifdef __cplusplus
enum hcblasStatus_t : unsigned short {
#else
typedef unsigned short hcblasStatus_t;
enum {
#endif
  HCBLAS_STATUS_SUCCESS = 0,
  HCBLAS_STATUS_NOT_INITIALIZED = 1,
  HCBLAS_STATUS_ALLOC_FAILED = 2,
  HCBLAS_STATUS_INVALID_VALUE = 3,
  HCBLAS_STATUS_MAPPING_ERROR = 4,
  HCBLAS_STATUS_EXECUTION_FAILED = 5,
  HCBLAS_STATUS_INTERNAL_ERROR = 6
};

#ifdef __cplusplus
enum hcblasOperation_t : unsigned short {
#else
typedef unsigned short hcblasOperation_t;
enum {
#endif
  HCBLAS_OP_N = 0,
  HCBLAS_OP_T = 1,
  HCBLAS_OP_C = 2
};

/* Complex scalars, interleaved {re, im} (reference: lib/include/hcblas.h:80-97). */
typedef struct float_2_ {
  float x;
  float y;
} float_2_;
typedef struct double_2_ {
  double x;
  double y;
} double_2_;
typedef float_2_ hcFloatComplex;
typedef hcFloatComplex hcComplex;
typedef double_2_ hcDoubleComplex;

#ifdef __cplusplus
typedef hc::half hcblasHalf;
#else
typedef hcblas_half_t hcblasHalf;
#endif

/* ---------------------------------------------------------------- handle -- */

/* Reference: hcblasCreate, lib/include/hcblas.h:112.  `av` selects the device
 * and stream; NULL means the current device's default stream (extension: the
 * reference requires a view).  Allocates the handle only: no device memory is
 * touched until the first call that needs workspace. */
hcblasStatus_t hcblasCreate(hcblasHandle_t *handle, hcblas_accl_view_t *av);

/* Reference: hcblasDestroy, lib/include/hcblas.h:125. */
hcblasStatus_t hcblasDestroy(hcblasHandle_t *handle);

/* Reference: hcblasSetAcclView, lib/include/hcblas.h:140 (C++ callers pass an
 * hc::accelerator_view& through the overload below).  A non-NULL `stream`
 * (a cudaStream_t) overrides the view's own stream. */
hcblasStatus_t hcblasSetAcclView(hcblasHandle_t handle, hcblas_accl_view_t *accl_view,
                                 void *stream);

/* Reference: hcblasGetAcclView, lib/include/hcblas.h:155. */
hcblasStatus_t hcblasGetAcclView(hcblasHandle_t handle, hcblas_accl_view_t **accl_view,
                                 void **stream);

/* Extension: bind a raw cudaStream_t (cuBLAS-style). */
hcblasStatus_t hcblasSetStream(hcblasHandle_t handle, void *stream);

/* ------------------------------------------------------- host <-> device -- */

/* Reference: lib/include/hcblas.h:174-233.  The reference copies
 * rows*cols*elemSize contiguous bytes and ignores lda/ldb
 * (lib/src/hcblas.cpp:260,309); its own tests pass lda = ldb = 1.  Here a
 * leading dimension >= rows (incx/incy == 1 for vectors) is honoured as a
 * strided copy, while a smaller one reproduces the reference's contiguous
 * copy.  Copies are synchronous with respect to the host, like the
 * reference's accelerator_view::copy. */
hcblasStatus_t hcblasSetVector(hcblasHandle_t handle, int n, int elemSize, const void *x,
                               int incx, void *y, int incy);
hcblasStatus_t hcblasGetVector(hcblasHandle_t handle, int n, int elemSize, const void *x,
                               int incx, void *y, int incy);
hcblasStatus_t hcblasSetMatrix(hcblasHandle_t handle, int rows, int cols, int elemSize,
                               const void *A, int lda, void *B, int ldb);
hcblasStatus_t hcblasGetMatrix(hcblasHandle_t handle, int rows, int cols, int elemSize,
                               const void *A, int lda, void *B, int ldb);

/* Extension with no counterpart in the reference (cuBLAS-style): the same
 * copies enqueued on `stream` (the handle's stream when null) without
 * waiting, so that a caller streaming many GEMMs overlaps the next inputs'
 * host->device copy and the last result's device->host copy with the
 * current GEMM.  Host memory must be pinned for the copy to be asynchronous;
 * ordering against the GEMM's stream is the caller's (events). */
hcblasStatus_t hcblasSetMatrixAsync(hcblasHandle_t handle, int rows, int cols, int elemSize,
                                    const void *A, int lda, void *B, int ldb, void *stream);
hcblasStatus_t hcblasGetMatrixAsync(hcblasHandle_t handle, int rows, int cols, int elemSize,
                                    const void *A, int lda, void *B, int ldb, void *stream);

/* ------------------------------------------------------------------ GEMM -- */

/* Reference: lib/include/hcblas.h:662-665, lib/src/hcblas.cpp:1304-1327. */
hcblasStatus_t hcblasSgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                           hcblasOperation_t transb, int m, int n, int k, const float *alpha,
                           float *A, int lda, float *B, int ldb, const float *beta, float *C,
                           int ldc);

/* Reference: lib/include/hcblas.h:667-670, lib/src/hcblas.cpp:1363-1386. */
hcblasStatus_t hcblasDgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                           hcblasOperation_t transb, int m, int n, int k, const double *alpha,
                           double *A, int lda, double *B, int ldb, const double *beta,
                           double *C, int ldc);

/* Reference: lib/include/hcblas.h:672-676, lib/src/hcblas.cpp:1329-1361. */
hcblasStatus_t hcblasCgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                           hcblasOperation_t transb, int m, int n, int k,
                           const hcComplex *alpha, hcComplex *A, int lda, hcComplex *B,
                           int ldb, const hcComplex *beta, hcComplex *C, int ldc);

/* Reference: lib/include/hcblas.h:678-683, lib/src/hcblas.cpp:1388-1421. */
hcblasStatus_t hcblasZgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                           hcblasOperation_t transb, int m, int n, int k,
                           const hcDoubleComplex *alpha, hcDoubleComplex *A, int lda,
                           hcDoubleComplex *B, int ldb, const hcDoubleComplex *beta,
                           hcDoubleComplex *C, int ldc);

/* Reference: lib/include/hcblas.h:685-689, lib/src/hcblas.cpp:1423-1450.
 * FP16 storage; accumulation is FP32 (the reference accumulates in half). */
hcblasStatus_t hcblasHgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                           hcblasOperation_t transb, int m, int n, int k,
                           const hcblasHalf *alpha, hcblasHalf *A, int lda, hcblasHalf *B,
                           int ldb, const hcblasHalf *beta, hcblasHalf *C, int ldc);

/* Pointer-array batched GEMM: C[i] := alpha*op(A[i])*op(B[i]) + beta*C[i].
 * Aarray/Barray/Carray are DEVICE-resident arrays of device pointers, as in
 * the reference tests (test/unit-api/test-blas.cpp:1969-1971).
 * Reference: lib/include/hcblas.h:762-790, lib/src/hcblas.cpp:1523-1675. */
hcblasStatus_t hcblasSgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                  hcblasOperation_t transb, int m, int n, int k,
                                  const float *alpha, float *Aarray[], int lda, float *Barray[],
                                  int ldb, const float *beta, float *Carray[], int ldc,
                                  int batchCount);
hcblasStatus_t hcblasCgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                  hcblasOperation_t transb, int m, int n, int k,
                                  const hcComplex *alpha, hcComplex *Aarray[], int lda,
                                  hcComplex *Barray[], int ldb, const hcComplex *beta,
                                  hcComplex *Carray[], int ldc, int batchCount);
hcblasStatus_t hcblasDgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                  hcblasOperation_t transb, int m, int n, int k,
                                  const double *alpha, double *Aarray[], int lda,
                                  double *Barray[], int ldb, const double *beta,
                                  double *Carray[], int ldc, int batchCount);
hcblasStatus_t hcblasZgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                  hcblasOperation_t transb, int m, int n, int k,
                                  const hcDoubleComplex *alpha, hcDoubleComplex *Aarray[],
                                  int lda, hcDoubleComplex *Barray[], int ldb,
                                  const hcDoubleComplex *beta, hcDoubleComplex *Carray[],
                                  int ldc, int batchCount);

/* Extension: HGEMM pointer-array batch (the reference compiles an HGEMM batch
 * path but leaves it unreachable, hgemm_array_wrapper.cpp:315-370). */
hcblasStatus_t hcblasHgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                  hcblasOperation_t transb, int m, int n, int k,
                                  const hcblasHalf *alpha, hcblasHalf *Aarray[], int lda,
                                  hcblasHalf *Barray[], int ldb, const hcblasHalf *beta,
                                  hcblasHalf *Carray[], int ldc, int batchCount);

/* Extension: strided batched GEMM, X_i = X + i * strideX (elements).  The
 * reference's closest form is its row-major batch kernel addressing
 * `A_batchOffset * elt` (sgemm_array_kernels_rMajor_batch.cpp:67), which its
 * wrapper never reaches (sgemm_array_wrapper.cpp:113-151).  Under an
 * emulated math mode every element runs on that mode's path: split-BF16
 * SGEMM batches on the grouped kernel, CRT DGEMM batches with a norm-scaled
 * plan (a moduli count below the full width, or an accuracy target) as one
 * pass of each CRT kernel over the batch, the others element by element. */
hcblasStatus_t hcblasSgemmStridedBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                         hcblasOperation_t transb, int m, int n, int k,
                                         const float *alpha, const float *A, int lda,
                                         long long strideA, const float *B, int ldb,
                                         long long strideB, const float *beta, float *C,
                                         int ldc, long long strideC, int batchCount);
hcblasStatus_t hcblasDgemmStridedBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                         hcblasOperation_t transb, int m, int n, int k,
                                         const double *alpha, const double *A, int lda,
                                         long long strideA, const double *B, int ldb,
                                         long long strideB, const double *beta, double *C,
                                         int ldc, long long strideC, int batchCount);
hcblasStatus_t hcblasCgemmStridedBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                         hcblasOperation_t transb, int m, int n, int k,
                                         const hcComplex *alpha, const hcComplex *A, int lda,
                                         long long strideA, const hcComplex *B, int ldb,
                                         long long strideB, const hcComplex *beta,
                                         hcComplex *C, int ldc, long long strideC,
                                         int batchCount);
hcblasStatus_t hcblasZgemmStridedBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                         hcblasOperation_t transb, int m, int n, int k,
                                         const hcDoubleComplex *alpha, const hcDoubleComplex *A,
                                         int lda, long long strideA, const hcDoubleComplex *B,
                                         int ldb, long long strideB,
                                         const hcDoubleComplex *beta, hcDoubleComplex *C,
                                         int ldc, long long strideC, int batchCount);
hcblasStatus_t hcblasHgemmStridedBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                         hcblasOperation_t transb, int m, int n, int k,
                                         const hcblasHalf *alpha, const hcblasHalf *A, int lda,
                                         long long strideA, const hcblasHalf *B, int ldb,
                                         long long strideB, const hcblasHalf *beta,
                                         hcblasHalf *C, int ldc, long long strideC,
                                         int batchCount);

/* ------------------------------------------------------- GEMV and GER -- */

/* Reference: lib/include/hcblas.h:516-534, lib/src/hcblas.cpp:967-1060.
 * y := alpha*op(A)*x + beta*y, A m x n in the handle's order; op(A) = A for
 * HCBLAS_OP_N, A^T otherwise.  Status: NULL handle -> NOT_INITIALIZED;
 * m, n < 0 or incx, incy == 0 -> INVALID_VALUE; m or n == 0, a NULL array or
 * a negative increment -> EXECUTION_FAILED (the class layer's quick return,
 * sgemv_array.cpp:833-836).  Batched: batchCount problems at the reference's
 * implicit batch offsets -- A: m*n, x: length of x, y: length of y (in
 * elements, whatever the increments; hcblas.cpp:1009-1019).  Unlike the
 * reference, lda is honoured (the reference assumes lda == m). */
hcblasStatus_t hcblasSgemv(hcblasHandle_t handle, hcblasOperation_t trans, int m, int n,
                           const float *alpha, float *A, int lda, float *x, int incx,
                           const float *beta, float *y, int incy);
hcblasStatus_t hcblasSgemvBatched(hcblasHandle_t handle, hcblasOperation_t trans, int m, int n,
                                  const float *alpha, float *A, int lda, float *x, int incx,
                                  const float *beta, float *y, int incy, int batchCount);
hcblasStatus_t hcblasDgemv(hcblasHandle_t handle, hcblasOperation_t trans, int m, int n,
                           const double *alpha, double *A, int lda, double *x, int incx,
                           const double *beta, double *y, int incy);
hcblasStatus_t hcblasDgemvBatched(hcblasHandle_t handle, hcblasOperation_t trans, int m, int n,
                                  const double *alpha, double *A, int lda, double *x, int incx,
                                  const double *beta, double *y, int incy, int batchCount);

/* Reference: lib/include/hcblas.h:573-586, lib/src/hcblas.cpp:1130-1230.
 * A := alpha*x*y^T + A (m x n, handle's order).  Status as GEMV except that a
 * negative increment is allowed (BLAS: the vector runs backwards from its
 * last stored element); alpha == 0 leaves A untouched.  Batched offsets:
 * x: m, y: n, A: m*n elements. */
hcblasStatus_t hcblasSger(hcblasHandle_t handle, int m, int n, const float *alpha,
                          const float *x, int incx, const float *y, int incy, float *A, int lda);
hcblasStatus_t hcblasDger(hcblasHandle_t handle, int m, int n, const double *alpha,
                          const double *x, int incx, const double *y, int incy, double *A,
                          int lda);
hcblasStatus_t hcblasSgerBatched(hcblasHandle_t handle, int m, int n, const float *alpha,
                                 const float *x, int incx, const float *y, int incy, float *A,
                                 int lda, int batchCount);
hcblasStatus_t hcblasDgerBatched(hcblasHandle_t handle, int m, int n, const double *alpha,
                                 const double *x, int incx, const double *y, int incy,
                                 double *A, int lda, int batchCount);

/* Extension (no counterpart in the reference's C API): grouped GEMM --
 * one call computes many independent, unevenly sized f16 GEMMs
 *   C_i := alpha * op(A_i) * op(B_i) + beta * C_i,  i = 0 .. count-1
 * in the handle's order (column-major by default), each problem with its own
 * transposes, sizes, leading dimensions and device pointers; FP32
 * accumulation.  One persistent tcgen05 kernel walks all problems' tiles
 * from a device-side problem table; problems whose operands TMA cannot
 * address (a base address not 16-byte aligned, or lda/ldb not a multiple of
 * 8) run as single calls after it.  An identical follow-up call (same
 * problem array contents) reuses the uploaded table.
 * Status: NULL/uninitialised handle -> NOT_INITIALIZED; count < 0, a NULL
 * problem array with count > 0, NULL alpha/beta, or a negative size ->
 * INVALID_VALUE; a problem with a zero size or a NULL matrix ->
 * EXECUTION_FAILED (the single-call rule); count == 0 -> SUCCESS. */
typedef struct hcblasGemmProblem {
  hcblasOperation_t transa, transb;
  int m, n, k;
  const void *A;
  int lda;
  const void *B;
  int ldb;
  void *C;
  int ldc;
} hcblasGemmProblem;
hcblasStatus_t hcblasHgemmGrouped(hcblasHandle_t handle, int count,
                                  const hcblasGemmProblem *problems, const hcblasHalf *alpha,
                                  const hcblasHalf *beta);

/* Extension (no counterpart in the reference): the grouped GEMM for f32
 * problems (the same hcblasGemmProblem array, f32 device matrices), computed
 * on the tensor cores by the split-BF16 scheme -- every problem's op(A) and
 * op(B) are split into bf16 planes by one packing launch, then one
 * persistent kernel walks all problems' 128 x 128 tiles with 6 plane
 * products (3 when the handle's math mode is HCBLAS_MATH_SPLIT_BF16 with
 * param 3), its f32 sums promoted into registers every 64 K, so the error
 * stays at or below plain FP32's.  Any alignment and leading dimension; the
 * plan (plane layout, tables) is cached per handle for an identical
 * follow-up problem array.  Status rules as hcblasHgemmGrouped. */
hcblasStatus_t hcblasSgemmGrouped(hcblasHandle_t handle, int count,
                                  const hcblasGemmProblem *problems, const float *alpha,
                                  const float *beta);

/* Extension (no counterpart in the reference; the reference's batched
 * D/C/Z entry points lib/src/hcblas.cpp:1600-1675 take uniform problems):
 * grouped GEMM for FP64, complex FP32 and complex FP64 problems (the same
 * hcblasGemmProblem array; device matrices of the call's type; complex
 * problems honour HCBLAS_OP_C as the conjugate transpose), computed in the
 * type's own arithmetic by one persistent CUDA-core kernel that walks every
 * problem's 64 x 64 tiles from a device-side problem table (problems ordered
 * by decreasing work).  Any alignment and leading dimension.  An identical
 * follow-up call (same problem array contents) reuses the uploaded table.
 * Status rules as hcblasHgemmGrouped. */
hcblasStatus_t hcblasDgemmGrouped(hcblasHandle_t handle, int count,
                                  const hcblasGemmProblem *problems, const double *alpha,
                                  const double *beta);
hcblasStatus_t hcblasCgemmGrouped(hcblasHandle_t handle, int count,
                                  const hcblasGemmProblem *problems, const hcComplex *alpha,
                                  const hcComplex *beta);
hcblasStatus_t hcblasZgemmGrouped(hcblasHandle_t handle, int count,
                                  const hcblasGemmProblem *problems,
                                  const hcDoubleComplex *alpha, const hcDoubleComplex *beta);

/* ------------------------------------------------ class-API C shims -- */

/* C-ABI forms of the Hcblaslibrary::hcblas_Xgemm methods (include/hcblaslib.h;
 * reference lib/include/hcblaslib.h:215-315) for FFI callers that cannot call
 * C++ member functions.  Same arguments in the same order: `order` is
 * RowMajor = 0 / ColMajor = 1, typeA/typeB are 'n', 't' or 'c', offsets are
 * in elements; scalars are passed by pointer; the handle's current view (its
 * stream) is used.  Return HCBLAS_SUCCEEDS (0) or HCBLAS_INVALID (-1) as the
 * methods do.  Batched forms take device-resident pointer arrays; matrix i
 * is X[i] + xOffset + i * X_batchOffset. */
int hcblasLibSgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N, int K,
                   const float *alpha, float *A, int64_t lda, float *B, int64_t ldb,
                   const float *beta, float *C, int64_t ldc, int64_t aOffset, int64_t bOffset,
                   int64_t cOffset);
int hcblasLibDgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N, int K,
                   const double *alpha, double *A, int64_t lda, double *B, int64_t ldb,
                   const double *beta, double *C, int64_t ldc, int64_t aOffset, int64_t bOffset,
                   int64_t cOffset);
int hcblasLibHgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N, int K,
                   const hcblasHalf *alpha, hcblasHalf *A, int64_t lda, hcblasHalf *B,
                   int64_t ldb, const hcblasHalf *beta, hcblasHalf *C, int64_t ldc,
                   int64_t aOffset, int64_t bOffset, int64_t cOffset);
int hcblasLibCgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N, int K,
                   const hcComplex *alpha, hcComplex *A, int64_t aOffset, int64_t lda,
                   hcComplex *B, int64_t bOffset, int64_t ldb, const hcComplex *beta,
                   hcComplex *C, int64_t cOffset, int64_t ldc);
int hcblasLibZgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N, int K,
                   const hcDoubleComplex *alpha, hcDoubleComplex *A, int64_t aOffset,
                   int64_t lda, hcDoubleComplex *B, int64_t bOffset, int64_t ldb,
                   const hcDoubleComplex *beta, hcDoubleComplex *C, int64_t cOffset,
                   int64_t ldc);
/* batched: (A[], lda, A_batchOffset, B[], ldb, B_batchOffset, beta, C[], ldc,
 * C_batchOffset, aOffset, bOffset, cOffset, batchSize) as
 * hcblaslib.h:244-266; dtype: 0 = S, 1 = D, 2 = C, 3 = Z, 4 = H. */
int hcblasLibGemmBatched(hcblasHandle_t h, int dtype, int order, char typeA, char typeB, int M,
                         int N, int K, const void *alpha, void **A, int64_t lda,
                         int64_t A_batchOffset, void **B, int64_t ldb, int64_t B_batchOffset,
                         const void *beta, void **C, int64_t ldc, int64_t C_batchOffset,
                         int64_t aOffset, int64_t bOffset, int64_t cOffset, int batchSize);

/* ----------------------------------------------------------- math modes -- */

/* Extension: how the S/C and D/Z entry points compute.
 *   HCBLAS_MATH_NATIVE     plain FP32 / FP64 arithmetic (default)
 *   HCBLAS_MATH_SPLIT_BF16 S/C: FP32 operands split into bf16 hi/lo terms,
 *                          products on tcgen05 tensor cores, FP32 accumulate
 *                          (`param` = number of terms: 3, or 6 for a 3-way split);
 *                          C runs 3M: Ar Br, Ai Bi, (Ar+Ai)(Br+Bi)
 *   HCBLAS_MATH_OZAKI_INT8 D/S: Ozaki scheme, operands scaled per row/col and
 *                          sliced into `param` INT8 slices; for every slice
 *                          weight one INT32 GEMM (exact) over the concatenated
 *                          K of its slice pairs on the int8 tensor cores, then
 *                          an FP64 weighting pass (`param` = 3..8 slices of 7
 *                          bits; 0 = 7 slices for D, 4 for S).  S widens its
 *                          FP32 operands to FP64 first and rounds the FP64
 *                          result once into C.
 *   HCBLAS_MATH_OZAKI_F16  D: the same scheme with 8-bit integer slices held
 *                          in binary16, products on the tcgen05 f16 path with
 *                          FP32 sums kept exact (integers < 2^24) and promoted
 *                          to FP64 per 32-element K slab (`param` = 3..7
 *                          slices of 8 bits; 0 = 7 slices, 56 bits)
 *   HCBLAS_MATH_OZAKI_CRT  D/Z: integer-modular (CRT) scheme: operands scaled
 *                          per row/column to integers of up to 53 bits,
 *                          residues modulo pairwise-coprime odd moduli <= 255
 *                          as int8 (tuning knob "crt_i8"), all moduli's exact
 *                          GEMMs in one int8 tensor-core launch, reconstruction
 *                          by the CRT weighted sum in binary64 chunks
 *                          (`param` = number of moduli 8..20; 0 = the fewest
 *                          keeping all 53 bits of every row for the call's
 *                          K).  With fewer moduli each row is scaled so that
 *                          its norm fits the range (Cauchy-Schwarz); 14 moduli
 *                          match native FP64 accuracy at K = 4096-8192.  Z runs
 *                          3M in modular arithmetic (three exact GEMMs per
 *                          modulus), its complex rows planned like real rows
 *                          of 2K entries. */
enum {
  HCBLAS_MATH_NATIVE = 0,
  HCBLAS_MATH_SPLIT_BF16 = 1,
  HCBLAS_MATH_OZAKI_INT8 = 2,
  HCBLAS_MATH_OZAKI_F16 = 3,
  HCBLAS_MATH_OZAKI_CRT = 4
};
hcblasStatus_t hcblasSetMathMode(hcblasHandle_t handle, int mode, int param);
hcblasStatus_t hcblasGetMathMode(hcblasHandle_t handle, int *mode, int *param);

/* Extension: requested accuracy of the emulated math modes.  When the math
 * mode's `param` is 0, the count (split-BF16 terms, Ozaki slices, CRT
 * moduli) is the smallest whose model error reaches `bits`:
 *     RMS(error of c_ij) <= 2^-bits * ||row i of op(A)||_2 * ||col j of op(B)||_2,
 * the error level of a dot product accumulated in a binary format with a
 * bits-bit significand, so 53 asks for native FP64 accuracy and 24 for
 * native FP32.  HCBLAS_ACCURACY_NATIVE (-1) means 53 for D/Z and 24 for S/C;
 * HCBLAS_ACCURACY_DEFAULT (0, the initial value) keeps each mode's default
 * count (CRT: the fewest moduli keeping every row's full 53 bits; Ozaki-I:
 * 7 slices for D, 4 for S; split-BF16: 3 terms).  Model per scheme: CRT
 * with norm-scaled rows keeps nb bits whatever the data and K (14 moduli:
 * nb = 54); Ozaki-I keeps b*s - log2(1.33 sqrt(K (s-1)) + 1.63) bits in the
 * worst case over the data; split-BF16 keeps 15 (3 terms) or 24 (6 terms).
 * A target no count reaches gets the mode's largest count.
 * Status: NOT_INITIALIZED for a bad handle; INVALID_VALUE outside -1..64. */
#define HCBLAS_ACCURACY_DEFAULT 0
#define HCBLAS_ACCURACY_NATIVE (-1)
hcblasStatus_t hcblasSetAccuracyTarget(hcblasHandle_t handle, int bits);
hcblasStatus_t hcblasGetAccuracyTarget(hcblasHandle_t handle, int *bits);
/* The plan without a handle or a GPU: the count a call of `dtype` (0 = S,
 * 1 = D, 2 = C, 3 = Z) with inner dimension k takes under math mode `mode`
 * with parameter `param` and accuracy target `bits`, and that count's model
 * accuracy in bits (+inf when the scheme represents the operands exactly).
 * INVALID_VALUE when the mode does not emulate that dtype. */
hcblasStatus_t hcblasPlanEmulation(int mode, int param, int bits, int dtype, long long k,
                                   int *count, double *model_bits);

/* Extension: set a named tuning knob on the handle.
 *   "split_promote_kb"  split-BF16 paths: 64-element K-slabs accumulated in
 *                       TMEM before each promotion to the IEEE f32
 *                       accumulator (1 or 4; default 1).
 *   "autotune"          1: the first call in each size bucket (kernel family,
 *                       type, transposes, ceil(log2) of M, N, K) times every
 *                       candidate configuration (SIMT tile; HGEMM 128x128 /
 *                       128x256 / CTA-pair 256x256; CRT modular GEMM the
 *                       same three; split-BF16 and Ozaki-I slice-group GEMMs
 *                       with or without CTA pairs; the grouped f16 kernel at
 *                       one or two CTAs per SM, bucketed by problem count,
 *                       tiles and work) and keeps the fastest, for this
 *                       process and, when HCBLAS_AUTOTUNE_CACHE names a file,
 *                       for later ones.  Only tiling and placement are
 *                       tuned, never the arithmetic (promotion interval,
 *                       slice and moduli counts stay as set).  With beta != 0 the
 *                       candidates write a scratch matrix of C's shape
 *                       (allocated stream-ordered while tuning), so C is
 *                       updated once; grouped calls are tuned on a beta == 0
 *                       call; 0 (default): size heuristics.
 *   "graphs"            1: a call identical to an earlier one (same
 *                       arguments, pointers, math mode and knobs, same
 *                       non-default stream) replays a CUDA graph captured
 *                       from the earlier call's launch sequence instead of
 *                       launching each kernel; 0 (default) launches directly.
 *                       Graphs are dropped when the handle's workspace moves.
 *   "tc_pair"           tensor-core paths (HGEMM, split-BF16, CRT): CTA-pair
 *                       kernels (tcgen05 cta_group::2, 256-row tiles over two
 *                       SMs): 0 never, 1 when the problem fills every SM pair
 *                       (default), 2 always.
 *   "crt_i8"            CRT DGEMM / ZGEMM (HCBLAS_MATH_OZAKI_CRT): 1 (default) int8
 *                       residue planes on the int8 tensor cores with INT32
 *                       sums exact over all of K (K <= 131072, else as 0);
 *                       0 binary16 residue planes on the f16 tensor cores,
 *                       sums reduced mod p every 1024 K.  Both give
 *                       bit-identical results.
 *   "grouped_ctas"      grouped / batched HGEMM kernel: 2 (default) CTAs per SM
 *                       with 3-stage rings, whose per-tile latencies overlap,
 *                       or 1 CTA per SM with a 6-stage ring.
 *   "grouped_c_tma"     grouped / batched HGEMM kernel: 1 (default) writes C
 *                       through shared-memory boxes and TMA stores where C's
 *                       shape allows, 0 by direct stores from registers
 *                       (within 1 % of each other on 4096 uneven problems).
 *   "aux_stream"        1 (default): independent passes of one call (the
 *                       CRT DGEMM's and ZGEMM's row-scale and residue
 *                       passes of op(B))
 *                       run on a second stream of the handle, forked from
 *                       and joined back into the call's stream with events
 *                       (also inside a captured CUDA graph); 0 keeps every
 *                       launch on the call's stream.  Results are identical.
 *   "dgemm_dmma"        native DGEMM and ZGEMM (HCBLAS_MATH_NATIVE): 1
 *                       (default) on the FP64 tensor path (warp-level
 *                       mma.sync .f64; ZGEMM as four real products), 0 on the
 *                       CUDA cores (DFMA); both accumulate in binary64.
 *   "workspace_mb"      upper limit of the handle's device workspace in MiB
 *                       (0, the default: none).  A call whose path needs more
 *                       returns HCBLAS_STATUS_EXECUTION_FAILED without
 *                       launching anything.  The workspace is allocated and
 *                       released stream-ordered (cudaMallocAsync /
 *                       cudaFreeAsync on the call's stream); it cannot grow
 *                       while that stream is being captured (the call then
 *                       fails the same way).
 *   "wait_timeout_us"   limit of every bounded pipeline wait in the
 *                       tensor-core kernels, in microseconds (0, the default:
 *                       2 s).  A wait that runs out records its code in the
 *                       handle's device error flag (hcblasGetDeviceError)
 *                       and the kernel unwinds, leaving C incomplete.
 *   "inject_timeout"    failure-detection testing: 1 arms the handle's next
 *                       HGEMM call to run its tensor-core pipeline with the
 *                       first operand load withheld, so that a pipeline wait
 *                       runs out; only a single 128 x 128 tile of one 64-wide
 *                       K block with beta == 0 is accepted (anything else
 *                       returns EXECUTION_FAILED).  Disarmed after that call. */
hcblasStatus_t hcblasSetTuningParam(hcblasHandle_t handle, const char *name, int value);

/* Extension: the path the last GEMM call on this handle took (a short static
 * string such as "simt.d.128x128" or "tc.h.256x256.pair"). */
const char *hcblasGetLastPath(hcblasHandle_t handle);

/* Extension: library version string. */
const char *hcblasGetVersionString(void);

/* Extension: diagnostics.
 *   hcblasGetKernelLaunchCount: kernels this library has launched in this
 *     process (all handles).
 *   hcblasSetProfiling: on != 0 brackets every kernel the handle launches
 *     with CUDA events on its stream; any value clears the records.
 *   hcblasGetProfile: writes "name launches total_ms\n" lines (synchronising
 *     on the recorded events) into buf; returns the full text length. */
long long hcblasGetKernelLaunchCount(void);
/* Extension: waits for the handle's stream, then returns and clears the
 * device error code set by a tensor-core kernel whose pipeline wait timed out
 * (0 = none; such a kernel exits early and leaves C incomplete). */
int hcblasGetDeviceError(hcblasHandle_t handle);
hcblasStatus_t hcblasSetProfiling(hcblasHandle_t handle, int on);
int hcblasGetProfile(hcblasHandle_t handle, char *buf, int cap);

/* Extension with no counterpart in the reference: split-BF16 SGEMM that
 * allocates nothing, for callers that cannot let a library call cudaMalloc
 * (applications whose own pool allocator owns all device memory and forbids
 * hidden allocations, plug-ins hosted inside a framework that accounts for
 * every device byte itself, services that allocate everything at start-up
 * so that no later call can fail for memory or stall on the allocator's
 * implicit synchronisation).
 *
 * Computes C = alpha * op(A) op(B) + beta * C, column-major, like
 * hcblasSgemm under HCBLAS_MATH_SPLIT_BF16 with `terms` = 3 or 6 bf16
 * products, on `stream` (a cudaStream_t; NULL = the legacy default stream)
 * of the current device.  No handle is involved.  Its scratch is one static
 * device array of HCBLAS_NOALLOC_SCRATCH_BYTES per GPU that loads the
 * library (64 MiB), held until the process exits; a problem whose bf16
 * planes need more -- (terms == 6 ? 3 : 2) * (round1024(m*kp*2) +
 * round1024(n*kp*2)) bytes with kp = k rounded up to a multiple of 8, e.g.
 * m = n = k = 2048 takes 32 MiB at 3 terms and 48 MiB at 6 -- is rejected
 * with HCBLAS_STATUS_INVALID_VALUE.
 * Status rules otherwise follow hcblasSgemm (negative sizes or NULL
 * alpha/beta: INVALID_VALUE; an empty problem or a NULL matrix:
 * EXECUTION_FAILED).
 *
 * The first call in each CUDA context of a device looks up the array's
 * device address (cudaGetSymbolAddress, with that device current) and
 * caches it with the context; make that first call before any stream
 * capture begins.  All calls on a device share the array and it keeps the
 * last call's contents, so calls that overlap on the GPU (other streams,
 * other host threads) race and must be serialised by the caller. */
#define HCBLAS_NOALLOC_SCRATCH_BYTES (64u << 20)
hcblasStatus_t hcblasSgemmSplitBF16NoAlloc(void *stream, hcblasOperation_t transa,
                                           hcblasOperation_t transb, int m, int n, int k,
                                           const float *alpha, const float *A, int lda,
                                           const float *B, int ldb, const float *beta, float *C,
                                           int ldc, int terms);
/* Extension with no counterpart in the reference: the outcome of the most
 * recent hcblasSgemmSplitBF16NoAlloc call on the current device.  Waits for
 * `stream`, then returns 0 when that call's tensor-core pipeline finished,
 * the pipeline-timeout code (> 0; C is then incomplete) when one of its
 * bounded waits gave up, or -1 when the state cannot be read.  Allocates
 * nothing; each no-allocation call clears the code when it starts. */
int hcblasSgemmSplitBF16NoAllocStatus(void *stream);

#ifdef __cplusplus
} /* extern "C" */

/* C++ conveniences with the reference's exact parameter types.
 * (hcblasCreate needs none: hc::accelerator_view* converts to
 * hcblas_accl_view_t*.) */
inline hcblasStatus_t hcblasSetAcclView(hcblasHandle_t handle, hc::accelerator_view &accl_view,
                                        void *stream = nullptr) {
  return hcblasSetAcclView(handle, static_cast<hcblas_accl_view_t *>(&accl_view), stream);
}
inline hcblasStatus_t hcblasGetAcclView(hcblasHandle_t handle,
                                        hc::accelerator_view *(&accl_view), void **stream) {
  hcblas_accl_view_t *v = nullptr;
  hcblasStatus_t s = hcblasGetAcclView(handle, &v, stream);
  accl_view = static_cast<hc::accelerator_view *>(v);
  return s;
}
#endif

#endif /* HCBLAS_B200_HCBLAS_H_ */
