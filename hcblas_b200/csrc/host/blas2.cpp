/*
 * blas2.cpp -- GEMV and GER: the hcblas{S,D}gemv[Batched] and
 * hcblas{S,D}ger[Batched] C entry points and the Hcblaslibrary methods
 * behind them (reference: lib/src/hcblas.cpp:967-1230,
 * lib/src/blas/sgemv/sgemv_array.cpp, lib/src/blas/sger/sger_array.cpp).
 * Row-major calls are rewritten as their column-major transposes; the
 * kernels are in csrc/kernels/blas2.cu.
 */
#include <cuda_runtime.h>

#include <cstring>

#include "dispatch.h"

namespace hcblas_b200 {
namespace {

constexpr int kMaxSplits = 64;

template <typename T>
constexpr int dtype_of() {
  return sizeof(T) == 4 ? HCBK_S : HCBK_D;
}

/* one GEMV, column-major canonical form, alpha/beta already in binary64 */
template <typename T>
hcblasStatus gemv_one(Hcblaslibrary *h, const hc::accelerator_view &view, hcblasOrder order,
                      hcblasTranspose type, int M, int N, double alpha, const T *A, int lda,
                      const T *X, int incX, double beta, T *Y, int incY) {
  HcblasB200State *st = h->impl;
  void *stream = view.stream;
  int trans = type != NoTrans;
  int64_t m = M, n = N;
  if (order == RowMajor) { /* row-major M x N == column-major N x M */
    trans = !trans;
    m = N;
    n = M;
  }
  const int64_t leny = trans ? n : m;
  int rc;
  if (alpha == 0.0) { /* y := beta*y, A and x not referenced */
    hcbk_gemm_args a;
    std::memset(&a, 0, sizeof(a));
    a.dtype = dtype_of<T>();
    a.m = 1;
    a.n = leny;
    a.k = 1;
    a.c = Y;
    a.ldc = incY;
    a.batch = 1;
    a.beta_re = beta;
    rc = timed_launch(st, stream, "blas2.scale", [&] { return hcbk_scale_c(&a, stream); });
  } else {
    const int64_t elems = hcbk_gemv_workspace_elems(m, n, trans, kMaxSplits);
    void *ws = ensure_workspace(st, (size_t)elems * sizeof(T), stream);
    if (!ws) return HCBLAS_INVALID;
    hcbk_gemv_args g;
    g.dtype = dtype_of<T>();
    g.trans = trans;
    g.m = m;
    g.n = n;
    g.a = A;
    g.lda = lda;
    g.x = X;
    g.incx = incX;
    g.y = Y;
    g.incy = incY;
    g.alpha = alpha;
    g.beta = beta;
    g.workspace = ws;
    g.max_splits = kMaxSplits;
    rc = timed_launch(st, stream, trans ? "blas2.gemv_t" : "blas2.gemv_n",
                      [&] { return hcbk_gemv(&g, stream); }, 2 /* partial sums + finish */);
  }
  st->last_path = alpha == 0.0 ? "blas2.scale" : (trans ? "blas2.gemv_t" : "blas2.gemv_n");
  return rc == HCBK_OK ? HCBLAS_SUCCEEDS : HCBLAS_INVALID;
}

template <typename T>
hcblasStatus gemv_api(Hcblaslibrary *h, const hc::accelerator_view &view, hcblasOrder order,
                      hcblasTranspose type, int M, int N, double alpha, T *A, int64_t aOffset,
                      int64_t A_bo, int lda, T *X, int64_t xOffset, int64_t X_bo, int incX,
                      double beta, T *Y, int64_t yOffset, int64_t Y_bo, int incY, int batch) {
  if (X == nullptr || Y == nullptr || A == nullptr || M <= 0 || N <= 0 || incX <= 0 ||
      incY <= 0 || batch < 0)
    return HCBLAS_INVALID;
  if (h == nullptr || !h->initialized || h->impl == nullptr) return HCBLAS_INVALID;
  DeviceGuard dev(view.device_id);
  if (!dev.ok()) return HCBLAS_INVALID;
  for (int b = 0; b < batch; ++b) {
    const hcblasStatus s = gemv_one<T>(h, view, order, type, M, N, alpha, A + aOffset + b * A_bo,
                                       lda, X + xOffset + b * X_bo, incX, beta,
                                       Y + yOffset + b * Y_bo, incY);
    if (s != HCBLAS_SUCCEEDS) return s;
  }
  return HCBLAS_SUCCEEDS;
}

/* A := alpha x y^T + A; negative increments address the vector backwards
 * from its last stored element (BLAS) */
template <typename T>
hcblasStatus ger_api(Hcblaslibrary *h, const hc::accelerator_view &view, hcblasOrder order,
                     int M, int N, double alpha, const T *X, int64_t xOffset, int64_t X_bo,
                     int incX, const T *Y, int64_t yOffset, int64_t Y_bo, int incY, T *A,
                     int64_t aOffset, int64_t A_bo, int lda, int batch) {
  if (X == nullptr || Y == nullptr || A == nullptr || M <= 0 || N <= 0 || incX == 0 ||
      incY == 0 || batch < 0)
    return HCBLAS_INVALID;
  if (alpha == 0.0) return HCBLAS_SUCCEEDS;
  if (h == nullptr || !h->initialized || h->impl == nullptr) return HCBLAS_INVALID;
  DeviceGuard dev(view.device_id);
  if (!dev.ok()) return HCBLAS_INVALID;
  HcblasB200State *st = h->impl;
  void *stream = view.stream;
  for (int b = 0; b < batch; ++b) {
    const T *x = X + xOffset + b * X_bo;
    const T *y = Y + yOffset + b * Y_bo;
    if (incX < 0) x += (int64_t)(1 - M) * incX;
    if (incY < 0) y += (int64_t)(1 - N) * incY;
    hcbk_ger_args g;
    g.dtype = dtype_of<T>();
    g.alpha = alpha;
    g.a = A + aOffset + b * A_bo;
    g.lda = lda;
    if (order == RowMajor) { /* row-major A == column-major A^T: A^T += alpha y x^T */
      g.m = N;
      g.n = M;
      g.x = y;
      g.incx = incY;
      g.y = x;
      g.incy = incX;
    } else {
      g.m = M;
      g.n = N;
      g.x = x;
      g.incx = incX;
      g.y = y;
      g.incy = incY;
    }
    const int rc = timed_launch(st, stream, "blas2.ger", [&] { return hcbk_ger(&g, stream); });
    if (rc != HCBK_OK) return HCBLAS_INVALID;
  }
  st->last_path = "blas2.ger";
  return HCBLAS_SUCCEEDS;
}

hcblasTranspose to_trans(hcblasOperation_t op) { return op == HCBLAS_OP_N ? NoTrans : Trans; }

hcblasStatus_t to_status(hcblasStatus s) {
  return s == HCBLAS_SUCCEEDS ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_EXECUTION_FAILED;
}

bool handle_ok(hcblasHandle_t h) { return h != nullptr && h->initialized && h->impl != nullptr; }

}  // namespace
}  // namespace hcblas_b200

using namespace hcblas_b200;

/* ----------------------------------------------------- class methods -- */

hcblasStatus Hcblaslibrary::hcblas_sgemv(hc::accelerator_view av, hcblasOrder order,
                                         hcblasTranspose type, const int M, const int N,
                                         const float &alpha, float *A, const int64_t aOffset,
                                         const int lda, float *X, const int64_t xOffset,
                                         const int incX, const float &beta, float *Y,
                                         const int64_t yOffset, const int incY) {
  return gemv_api<float>(this, av, order, type, M, N, alpha, A, aOffset, 0, lda, X, xOffset, 0,
                         incX, beta, Y, yOffset, 0, incY, 1);
}

hcblasStatus Hcblaslibrary::hcblas_sgemv(hc::accelerator_view av, hcblasOrder order,
                                         hcblasTranspose type, const int M, const int N,
                                         const float &alpha, float *A, const int64_t aOffset,
                                         const int64_t A_batchOffset, const int lda, float *X,
                                         const int64_t xOffset, const int64_t X_batchOffset,
                                         const int incX, const float &beta, float *Y,
                                         const int64_t yOffset, const int64_t Y_batchOffset,
                                         const int incY, const int batchSize) {
  return gemv_api<float>(this, av, order, type, M, N, alpha, A, aOffset, A_batchOffset, lda, X,
                         xOffset, X_batchOffset, incX, beta, Y, yOffset, Y_batchOffset, incY,
                         batchSize);
}

hcblasStatus Hcblaslibrary::hcblas_dgemv(hc::accelerator_view av, hcblasOrder order,
                                         hcblasTranspose type, const int M, const int N,
                                         const double &alpha, double *A, const int64_t aOffset,
                                         const int lda, double *X, const int64_t xOffset,
                                         const int incX, const double &beta, double *Y,
                                         const int64_t yOffset, const int incY) {
  return gemv_api<double>(this, av, order, type, M, N, alpha, A, aOffset, 0, lda, X, xOffset, 0,
                          incX, beta, Y, yOffset, 0, incY, 1);
}

hcblasStatus Hcblaslibrary::hcblas_dgemv(hc::accelerator_view av, hcblasOrder order,
                                         hcblasTranspose type, const int M, const int N,
                                         const double &alpha, double *A, const int64_t aOffset,
                                         const int64_t A_batchOffset, const int lda, double *X,
                                         const int64_t xOffset, const int64_t X_batchOffset,
                                         const int incX, const double &beta, double *Y,
                                         const int64_t yOffset, const int64_t Y_batchOffset,
                                         const int incY, const int batchSize) {
  return gemv_api<double>(this, av, order, type, M, N, alpha, A, aOffset, A_batchOffset, lda, X,
                          xOffset, X_batchOffset, incX, beta, Y, yOffset, Y_batchOffset, incY,
                          batchSize);
}

hcblasStatus Hcblaslibrary::hcblas_sger(hc::accelerator_view av, hcblasOrder order, const int M,
                                        const int N, const float &alpha, const float *X,
                                        const int64_t xOffset, const int incX, const float *Y,
                                        const int64_t yOffset, const int incY, float *A,
                                        const int64_t aOffset, const int lda) {
  return ger_api<float>(this, av, order, M, N, alpha, X, xOffset, 0, incX, Y, yOffset, 0, incY,
                        A, aOffset, 0, lda, 1);
}

hcblasStatus Hcblaslibrary::hcblas_sger(hc::accelerator_view av, hcblasOrder order, const int M,
                                        const int N, const float &alpha, const float *X,
                                        const int64_t xOffset, const int64_t X_batchOffset,
                                        const int incX, const float *Y, const int64_t yOffset,
                                        const int64_t Y_batchOffset, const int incY, float *A,
                                        const int64_t aOffset, const int64_t A_batchOffset,
                                        const int lda, const int batchSize) {
  return ger_api<float>(this, av, order, M, N, alpha, X, xOffset, X_batchOffset, incX, Y,
                        yOffset, Y_batchOffset, incY, A, aOffset, A_batchOffset, lda, batchSize);
}

hcblasStatus Hcblaslibrary::hcblas_dger(hc::accelerator_view av, hcblasOrder order, const int M,
                                        const int N, const double &alpha, const double *X,
                                        const int64_t xOffset, const int incX, const double *Y,
                                        const int64_t yOffset, const int incY, double *A,
                                        const int64_t aOffset, const int lda) {
  return ger_api<double>(this, av, order, M, N, alpha, X, xOffset, 0, incX, Y, yOffset, 0, incY,
                         A, aOffset, 0, lda, 1);
}

hcblasStatus Hcblaslibrary::hcblas_dger(hc::accelerator_view av, hcblasOrder order, const int M,
                                        const int N, const double &alpha, const double *X,
                                        const int64_t xOffset, const int64_t X_batchOffset,
                                        const int incX, const double *Y, const int64_t yOffset,
                                        const int64_t Y_batchOffset, const int incY, double *A,
                                        const int64_t aOffset, const int64_t A_batchOffset,
                                        const int lda, const int batchSize) {
  return ger_api<double>(this, av, order, M, N, alpha, X, xOffset, X_batchOffset, incX, Y,
                         yOffset, Y_batchOffset, incY, A, aOffset, A_batchOffset, lda, batchSize);
}

/* ------------------------------------------------------------- C API -- */

#define HCBLAS2_CHECK()                                                            \
  if (!handle_ok(handle)) return HCBLAS_STATUS_NOT_INITIALIZED;                    \
  if (m < 0 || n < 0 || incx == 0 || incy == 0) return HCBLAS_STATUS_INVALID_VALUE; \
  if (alpha == nullptr) return HCBLAS_STATUS_INVALID_VALUE;

extern "C" hcblasStatus_t hcblasSgemv(hcblasHandle_t handle, hcblasOperation_t trans, int m,
                                      int n, const float *alpha, float *A, int lda, float *x,
                                      int incx, const float *beta, float *y, int incy) {
  HCBLAS2_CHECK()
  if (beta == nullptr) return HCBLAS_STATUS_INVALID_VALUE;
  return to_status(handle->hcblas_sgemv(handle->currentAcclView, handle->Order, to_trans(trans),
                                        m, n, *alpha, A, 0, lda, x, 0, incx, *beta, y, 0, incy));
}

extern "C" hcblasStatus_t hcblasDgemv(hcblasHandle_t handle, hcblasOperation_t trans, int m,
                                      int n, const double *alpha, double *A, int lda, double *x,
                                      int incx, const double *beta, double *y, int incy) {
  HCBLAS2_CHECK()
  if (beta == nullptr) return HCBLAS_STATUS_INVALID_VALUE;
  return to_status(handle->hcblas_dgemv(handle->currentAcclView, handle->Order, to_trans(trans),
                                        m, n, *alpha, A, 0, lda, x, 0, incx, *beta, y, 0, incy));
}

extern "C" hcblasStatus_t hcblasSgemvBatched(hcblasHandle_t handle, hcblasOperation_t trans,
                                             int m, int n, const float *alpha, float *A,
                                             int lda, float *x, int incx, const float *beta,
                                             float *y, int incy, int batchCount) {
  HCBLAS2_CHECK()
  if (beta == nullptr || batchCount < 0) return HCBLAS_STATUS_INVALID_VALUE;
  const int64_t lx = trans == HCBLAS_OP_N ? n : m, ly = trans == HCBLAS_OP_N ? m : n;
  return to_status(handle->hcblas_sgemv(handle->currentAcclView, handle->Order, to_trans(trans),
                                        m, n, *alpha, A, 0, (int64_t)m * n, lda, x, 0, lx, incx,
                                        *beta, y, 0, ly, incy, batchCount));
}

extern "C" hcblasStatus_t hcblasDgemvBatched(hcblasHandle_t handle, hcblasOperation_t trans,
                                             int m, int n, const double *alpha, double *A,
                                             int lda, double *x, int incx, const double *beta,
                                             double *y, int incy, int batchCount) {
  HCBLAS2_CHECK()
  if (beta == nullptr || batchCount < 0) return HCBLAS_STATUS_INVALID_VALUE;
  const int64_t lx = trans == HCBLAS_OP_N ? n : m, ly = trans == HCBLAS_OP_N ? m : n;
  return to_status(handle->hcblas_dgemv(handle->currentAcclView, handle->Order, to_trans(trans),
                                        m, n, *alpha, A, 0, (int64_t)m * n, lda, x, 0, lx, incx,
                                        *beta, y, 0, ly, incy, batchCount));
}

extern "C" hcblasStatus_t hcblasSger(hcblasHandle_t handle, int m, int n, const float *alpha,
                                     const float *x, int incx, const float *y, int incy,
                                     float *A, int lda) {
  HCBLAS2_CHECK()
  return to_status(handle->hcblas_sger(handle->currentAcclView, handle->Order, m, n, *alpha, x, 0,
                                       incx, y, 0, incy, A, 0, lda));
}

extern "C" hcblasStatus_t hcblasDger(hcblasHandle_t handle, int m, int n, const double *alpha,
                                     const double *x, int incx, const double *y, int incy,
                                     double *A, int lda) {
  HCBLAS2_CHECK()
  return to_status(handle->hcblas_dger(handle->currentAcclView, handle->Order, m, n, *alpha, x, 0,
                                       incx, y, 0, incy, A, 0, lda));
}

extern "C" hcblasStatus_t hcblasSgerBatched(hcblasHandle_t handle, int m, int n,
                                            const float *alpha, const float *x, int incx,
                                            const float *y, int incy, float *A, int lda,
                                            int batchCount) {
  HCBLAS2_CHECK()
  if (batchCount < 0) return HCBLAS_STATUS_INVALID_VALUE;
  return to_status(handle->hcblas_sger(handle->currentAcclView, handle->Order, m, n, *alpha, x, 0,
                                       m, incx, y, 0, n, incy, A, 0, (int64_t)m * n, lda,
                                       batchCount));
}

extern "C" hcblasStatus_t hcblasDgerBatched(hcblasHandle_t handle, int m, int n,
                                            const double *alpha, const double *x, int incx,
                                            const double *y, int incy, double *A, int lda,
                                            int batchCount) {
  HCBLAS2_CHECK()
  if (batchCount < 0) return HCBLAS_STATUS_INVALID_VALUE;
  return to_status(handle->hcblas_dger(handle->currentAcclView, handle->Order, m, n, *alpha, x, 0,
                                       m, incx, y, 0, n, incy, A, 0, (int64_t)m * n, lda,
                                       batchCount));
}
