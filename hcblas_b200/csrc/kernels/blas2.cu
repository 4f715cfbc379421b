/*
 * blas2.cu -- GEMV and GER (the N = 1 and K = 1 limits of GEMM), HBM-bound:
 * every kernel streams the matrix once with coalesced accesses, and the
 * reductions are deterministic (fixed-order two-pass sums, no atomics).
 *
 *   gemv N:  y(i) = alpha * sum_j A(i, j) x(j) + beta * y(i)
 *            threads along rows (consecutive threads read consecutive
 *            addresses of a column); the columns are cut into `splits`
 *            slices whose partial sums land in a workspace and are added in
 *            slice order by the finishing kernel
 *   gemv T:  y(j) = alpha * sum_i A(i, j) x(i) + beta * y(j)
 *            one warp per (column, row slice): lanes stride down the
 *            contiguous column, warp-shuffle reduction, partials per slice
 *   ger:     A(i, j) += alpha * x(i) * y(j), threads along rows
 * Column-major A with leading dimension lda.  Vector element r sits at
 * v[r * inc]; GER accepts negative increments (the caller passes the
 * address of the logical first element, BLAS style), GEMV positive ones.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "hcbk.h"

namespace {

/* 16-byte vector of T (float4 / double2) */
template <typename T> struct Vec16;
template <> struct Vec16<float> {
  using V = float4;
  static constexpr int N = 4;
  static __device__ __forceinline__ float get(const float4 &v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
  }
  static __device__ __forceinline__ void set(float4 &v, int i, float a) {
    if (i == 0) v.x = a;
    else if (i == 1) v.y = a;
    else if (i == 2) v.z = a;
    else v.w = a;
  }
};
template <> struct Vec16<double> {
  using V = double2;
  static constexpr int N = 2;
  static __device__ __forceinline__ double get(const double2 &v, int i) {
    return i == 0 ? v.x : v.y;
  }
  static __device__ __forceinline__ void set(double2 &v, int i, double a) {
    if (i == 0) v.x = a;
    else v.y = a;
  }
};

/* vectorised gemv N: each thread owns VN consecutive rows (16-byte loads);
 * needs m, lda multiples of VN and a 16-byte aligned A */
template <typename T>
__global__ void gemv_n_partial_vec(const T *A, int64_t lda, const T *x, int64_t incx, int64_t m,
                                   int64_t n, int64_t cols_per_split, T *part) {
  using VT = Vec16<T>;
  constexpr int VN = VT::N;
  const int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * VN;
  const int64_t j0 = (int64_t)blockIdx.y * cols_per_split;
  const int64_t j1 = (j0 + cols_per_split < n) ? j0 + cols_per_split : n;
  if (i0 >= m) return;
  T s[4][VN]; /* four columns in flight */
#pragma unroll
  for (int r = 0; r < VN; ++r) s[0][r] = s[1][r] = s[2][r] = s[3][r] = 0;
  int64_t j = j0;
  for (; j + 4 <= j1; j += 4) {
    typename VT::V a[4];
    T xv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = *reinterpret_cast<const typename VT::V *>(A + i0 + (j + u) * lda);
      xv[u] = x[(j + u) * incx];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int r = 0; r < VN; ++r) s[u][r] += VT::get(a[u], r) * xv[u];
  }
  for (; j < j1; ++j) {
    const typename VT::V a0 = *reinterpret_cast<const typename VT::V *>(A + i0 + j * lda);
    const T x0 = x[j * incx];
#pragma unroll
    for (int r = 0; r < VN; ++r) s[0][r] += VT::get(a0, r) * x0;
  }
  typename VT::V o;
#pragma unroll
  for (int r = 0; r < VN; ++r) VT::set(o, r, (s[0][r] + s[1][r]) + (s[2][r] + s[3][r]));
  *reinterpret_cast<typename VT::V *>(part + (int64_t)blockIdx.y * m + i0) = o;
}

/* vectorised gemv T: every lane reads VN consecutive rows of the column */
template <typename T>
__global__ void gemv_t_partial_vec(const T *A, int64_t lda, const T *x, int64_t incx, int64_t m,
                                   int64_t n, int64_t rows_per_split, T *part) {
  using VT = Vec16<T>;
  constexpr int VN = VT::N;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (j >= n) return;
  const int64_t i0 = (int64_t)blockIdx.y * rows_per_split;
  const int64_t i1 = (i0 + rows_per_split < m) ? i0 + rows_per_split : m;
  const T *col = A + j * lda;
  T sv[4] = {0, 0, 0, 0};
  int64_t i = i0 + lane * VN;
  constexpr int64_t W = 32 * VN; /* elements one warp covers per load */
  if (incx == 1 && (reinterpret_cast<uintptr_t>(x) & 15) == 0) {
    /* unit-stride x: 16-byte loads of x as well */
    for (; i + 3 * W < i1; i += 4 * W) { /* four loads in flight per lane */
      typename VT::V a[4], xv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = *reinterpret_cast<const typename VT::V *>(col + i + u * W);
        xv[u] = *reinterpret_cast<const typename VT::V *>(x + i + u * W);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int r = 0; r < VN; ++r) sv[u] += VT::get(a[u], r) * VT::get(xv[u], r);
    }
  }
  for (; i + 3 * W < i1; i += 4 * W) { /* four loads in flight per lane */
    typename VT::V a[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = *reinterpret_cast<const typename VT::V *>(col + i + u * W);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int r = 0; r < VN; ++r) sv[u] += VT::get(a[u], r) * x[(i + u * W + r) * incx];
  }
  for (; i < i1; i += W) {
    const typename VT::V a0 = *reinterpret_cast<const typename VT::V *>(col + i);
#pragma unroll
    for (int r = 0; r < VN; ++r) sv[0] += VT::get(a0, r) * x[(i + r) * incx];
  }
  T sum = (sv[0] + sv[1]) + (sv[2] + sv[3]);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, off);
  if (lane == 0) part[(int64_t)blockIdx.y * n + j] = sum;
}

/* vectorised ger: each thread updates VN consecutive rows of a column */
template <typename T>
__global__ void ger_kernel_vec(int64_t m, int64_t n, T alpha, const T *x, int64_t incx,
                               const T *y, int64_t incy, T *A, int64_t lda) {
  using VT = Vec16<T>;
  constexpr int VN = VT::N;
  const int64_t i0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * VN;
  if (i0 >= m) return;
  T xi[VN];
#pragma unroll
  for (int r = 0; r < VN; ++r) xi[r] = alpha * x[(i0 + r) * incx];
  int64_t j = blockIdx.y;
  const int64_t step = gridDim.y;
  for (; j + 3 * step < n; j += 4 * step) { /* four columns in flight */
    typename VT::V a[4];
    T yj[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a[u] = *reinterpret_cast<const typename VT::V *>(A + i0 + (j + u * step) * lda);
      yj[u] = y[(j + u * step) * incy];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int r = 0; r < VN; ++r) VT::set(a[u], r, VT::get(a[u], r) + xi[r] * yj[u]);
      *reinterpret_cast<typename VT::V *>(A + i0 + (j + u * step) * lda) = a[u];
    }
  }
  for (; j < n; j += step) {
    typename VT::V *p = reinterpret_cast<typename VT::V *>(A + i0 + j * lda);
    typename VT::V a = *p;
    const T yj = y[j * incy];
#pragma unroll
    for (int r = 0; r < VN; ++r) VT::set(a, r, VT::get(a, r) + xi[r] * yj);
    *p = a;
  }
}

template <typename T>
__global__ void gemv_n_partial(const T *A, int64_t lda, const T *x, int64_t incx, int64_t m,
                               int64_t n, int64_t cols_per_split, T *part) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t j0 = (int64_t)blockIdx.y * cols_per_split;
  const int64_t j1 = (j0 + cols_per_split < n) ? j0 + cols_per_split : n;
  if (i >= m) return;
  T s0 = 0, s1 = 0, s2 = 0, s3 = 0; /* four independent chains for ILP */
  int64_t j = j0;
  for (; j + 4 <= j1; j += 4) {
    s0 += A[i + j * lda] * x[j * incx];
    s1 += A[i + (j + 1) * lda] * x[(j + 1) * incx];
    s2 += A[i + (j + 2) * lda] * x[(j + 2) * incx];
    s3 += A[i + (j + 3) * lda] * x[(j + 3) * incx];
  }
  for (; j < j1; ++j) s0 += A[i + j * lda] * x[j * incx];
  part[(int64_t)blockIdx.y * m + i] = (s0 + s1) + (s2 + s3);
}

template <typename T>
__global__ void gemv_t_partial(const T *A, int64_t lda, const T *x, int64_t incx, int64_t m,
                               int64_t n, int64_t rows_per_split, T *part) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t j = (int64_t)blockIdx.x * (blockDim.x >> 5) + warp;
  if (j >= n) return;
  const int64_t i0 = (int64_t)blockIdx.y * rows_per_split;
  const int64_t i1 = (i0 + rows_per_split < m) ? i0 + rows_per_split : m;
  const T *col = A + j * lda;
  T s0 = 0, s1 = 0;
  int64_t i = i0 + lane;
  for (; i + 32 < i1; i += 64) {
    s0 += col[i] * x[i * incx];
    s1 += col[i + 32] * x[(i + 32) * incx];
  }
  if (i < i1) s0 += col[i] * x[i * incx];
  T s = s0 + s1;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) part[(int64_t)blockIdx.y * n + j] = s;
}

/* y(r) = alpha * sum_s part[s][r] + beta * y(r); beta == 0: y not read */
template <typename T>
__global__ void gemv_finish(const T *part, int splits, int64_t len, T alpha, T beta, T *y,
                            int64_t incy) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= len) return;
  T s = 0;
  for (int k = 0; k < splits; ++k) s += part[(int64_t)k * len + r];
  T o = alpha * s;
  if (beta != T(0)) o += beta * y[r * incy];
  y[r * incy] = o;
}

template <typename T>
__global__ void ger_kernel(int64_t m, int64_t n, T alpha, const T *x, int64_t incx, const T *y,
                           int64_t incy, T *A, int64_t lda) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const T xi = alpha * x[i * incx];
  for (int64_t j = blockIdx.y; j < n; j += gridDim.y) A[i + j * lda] += xi * y[j * incy];
}

/* 16-byte vector access is legal: aligned base, and every column (and every
 * `rows` boundary) starts on a 16-byte boundary */
template <typename T>
bool vec_ok(const T *A, int64_t lda, int64_t rows) {
  constexpr int VN = 16 / sizeof(T);
  return (reinterpret_cast<uintptr_t>(A) & 15) == 0 && lda % VN == 0 && rows % VN == 0;
}

template <typename T>
int gemv_impl(const hcbk_gemv_args *g, cudaStream_t st) {
  const T *A = static_cast<const T *>(g->a);
  const T *x = static_cast<const T *>(g->x);
  T *y = static_cast<T *>(g->y);
  T *part = static_cast<T *>(g->workspace);
  const int sms = hcbk_sm_count();
  const T alpha = (T)g->alpha, beta = (T)g->beta;
  if (!g->trans) {
    const bool vec = vec_ok<T>(A, g->lda, g->m);
    const int64_t rb = vec ? (g->m / Vec16<T>::N + 255) / 256 : (g->m + 255) / 256;
    /* enough (row block, column slice) blocks for ~8 resident per SM: the
     * kernel is bound by memory-level parallelism */
    int64_t splits = (rb >= 8 * sms) ? 1 : (8 * sms + rb - 1) / rb;
    if (splits > g->n) splits = g->n;
    if (splits > g->max_splits) splits = g->max_splits;
    if (splits < 1) splits = 1;
    const int64_t cps = (g->n + splits - 1) / splits;
    splits = (g->n + cps - 1) / cps;
    if (vec)
      gemv_n_partial_vec<T><<<dim3((unsigned)rb, (unsigned)splits), 256, 0, st>>>(
          A, g->lda, x, g->incx, g->m, g->n, cps, part);
    else
      gemv_n_partial<T><<<dim3((unsigned)rb, (unsigned)splits), 256, 0, st>>>(
          A, g->lda, x, g->incx, g->m, g->n, cps, part);
    gemv_finish<T><<<(unsigned)((g->m + 255) / 256), 256, 0, st>>>(part, (int)splits, g->m,
                                                                  alpha, beta, y, g->incy);
  } else {
    const int64_t cb = (g->n + 7) / 8; /* 8 warps = 8 columns per block */
    int64_t splits = (cb >= 8 * sms) ? 1 : (8 * sms + cb - 1) / cb;
    const int64_t max_by_rows = (g->m + 1023) / 1024; /* keep >= 1024 rows per slice */
    if (splits > max_by_rows) splits = max_by_rows;
    if (splits > g->max_splits) splits = g->max_splits;
    if (splits < 1) splits = 1;
    const int64_t rps = (g->m + splits - 1) / splits;
    splits = (g->m + rps - 1) / rps;
    if (vec_ok<T>(A, g->lda, rps) && vec_ok<T>(A, g->lda, g->m))
      gemv_t_partial_vec<T><<<dim3((unsigned)cb, (unsigned)splits), 256, 0, st>>>(
          A, g->lda, x, g->incx, g->m, g->n, rps, part);
    else
      gemv_t_partial<T><<<dim3((unsigned)cb, (unsigned)splits), 256, 0, st>>>(
          A, g->lda, x, g->incx, g->m, g->n, rps, part);
    gemv_finish<T><<<(unsigned)((g->n + 255) / 256), 256, 0, st>>>(part, (int)splits, g->n,
                                                                  alpha, beta, y, g->incy);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

}  // namespace

extern "C" int64_t hcbk_gemv_workspace_elems(int64_t m, int64_t n, int trans, int max_splits) {
  return (int64_t)max_splits * (trans ? n : m);
}

extern "C" int hcbk_gemv(const hcbk_gemv_args *g, void *stream) {
  if (g->m <= 0 || g->n <= 0 || g->incx <= 0 || g->incy <= 0 || g->max_splits < 1 ||
      (g->m + 255) / 256 > 0x7fffffff || g->max_splits > 65535)
    return HCBK_ERR_ARGS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (g->dtype == HCBK_S) return gemv_impl<float>(g, st);
  if (g->dtype == HCBK_D) return gemv_impl<double>(g, st);
  return HCBK_ERR_ARGS;
}

extern "C" int hcbk_ger(const hcbk_ger_args *g, void *stream) {
  if (g->m <= 0 || g->n <= 0 || g->incx == 0 || g->incy == 0) return HCBK_ERR_ARGS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int64_t rb = (g->m + 255) / 256;
  int64_t gy = ((int64_t)hcbk_sm_count() * 8 + rb - 1) / rb;
  if (gy > g->n) gy = g->n;
  if (gy > 65535) gy = 65535;
  if (gy < 1) gy = 1;
  if (g->dtype == HCBK_S) {
    float *A = static_cast<float *>(g->a);
    if (vec_ok<float>(A, g->lda, g->m))
      ger_kernel_vec<float><<<dim3((unsigned)((g->m / 4 + 255) / 256), (unsigned)gy), 256, 0,
                              st>>>(g->m, g->n, (float)g->alpha,
                                    static_cast<const float *>(g->x), g->incx,
                                    static_cast<const float *>(g->y), g->incy, A, g->lda);
    else
      ger_kernel<float><<<dim3((unsigned)rb, (unsigned)gy), 256, 0, st>>>(
          g->m, g->n, (float)g->alpha, static_cast<const float *>(g->x), g->incx,
          static_cast<const float *>(g->y), g->incy, A, g->lda);
  } else if (g->dtype == HCBK_D) {
    double *A = static_cast<double *>(g->a);
    if (vec_ok<double>(A, g->lda, g->m))
      ger_kernel_vec<double><<<dim3((unsigned)((g->m / 2 + 255) / 256), (unsigned)gy), 256, 0,
                               st>>>(g->m, g->n, g->alpha, static_cast<const double *>(g->x),
                                     g->incx, static_cast<const double *>(g->y), g->incy, A,
                                     g->lda);
    else
      ger_kernel<double><<<dim3((unsigned)rb, (unsigned)gy), 256, 0, st>>>(
          g->m, g->n, g->alpha, static_cast<const double *>(g->x), g->incx,
          static_cast<const double *>(g->y), g->incy, A, g->lda);
  } else {
    return HCBK_ERR_ARGS;
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
