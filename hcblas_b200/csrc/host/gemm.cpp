/*
 * gemm.cpp -- the GEMM hot path's host side: hcBLAS's C API and class API
 * entry points, argument checks with the reference's status conventions,
 * row-major -> column-major canonicalisation, and dispatch to the sm_100a
 * kernels through the hcbk_* C-ABI shim.
 *
 * Reference call chain being replaced (lib/src/hcblas.cpp:1304-1675 ->
 * lib/src/blas/<x>gemm/<x>gemm_array_wrapper.cpp -> size-bucket dispatchers
 * -> ~40 HCC tile kernels).  Here:
 *   C API (status mapping)  ->  class method (quick-return checks)  ->
 *   run_gemm (canonicalise, alpha == 0, path choice)  ->  hcbk_* launcher.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>
#include <utility>

#include "../../../include/hcblas.h"
#include "../../../include/hcblaslib.h"
#include "../kernels/hcbk.h"
#include "dispatch.h"
#include "state.h"

namespace hcblas_b200 {

int op_from_char(hcblasTranspose t) {
  if (t == NoTrans || t == 'N') return HCBK_OP_N;
  if (t == ConjTrans || t == 'C') return HCBK_OP_C;
  return HCBK_OP_T; /* the reference treats every non-'n' value as 't' */
}

hcblasTranspose char_from_op(hcblasOperation_t op) {
  if (op == HCBLAS_OP_N) return NoTrans;
  if (op == HCBLAS_OP_C) return ConjTrans;
  return Trans; /* reference: anything but OP_N is a transpose */
}

static bool is_complex(int dtype) { return dtype == HCBK_C || dtype == HCBK_Z; }

/* Replay a captured CUDA graph of an identical earlier call, or run the call
 * eagerly and capture its launch sequence for the next time.  The capture
 * happens after the eager run, so every buffer, tensor map and attribute it
 * needs already exists and nothing is allocated while capturing. */
int dispatch_with_graph(HcblasB200State *st, const hcbk_gemm_args *a, void *stream,
                        const char **path) {
  int dev = 0;
  cudaGetDevice(&dev);
  const int knobs[10] = {st->math_mode, st->math_param,  st->split_promote_kb,
                         st->tc_pair,   dev,             (int)st->workspace_epoch,
                         st->crt_i8,    st->grouped_ctas, st->grouped_c_tma,
                         st->use_aux};
  std::vector<unsigned char> key(sizeof(*a) + sizeof(knobs) + sizeof(stream));
  std::memcpy(key.data(), a, sizeof(*a));
  std::memcpy(key.data() + sizeof(*a), knobs, sizeof(knobs));
  std::memcpy(key.data() + sizeof(*a) + sizeof(knobs), &stream, sizeof(stream));
  for (auto &e : st->graph_cache) {
    if (e.key == key) {
      if (cudaGraphLaunch(static_cast<cudaGraphExec_t>(e.exec), static_cast<cudaStream_t>(stream)) !=
          cudaSuccess) {
        cudaGetLastError();
        return HCBK_ERR_LAUNCH;
      }
      count_launch((int)e.launches);
      *path = e.path;
      return HCBK_OK;
    }
  }
  int rc = dispatch_gemm(st, a, stream, path);
  if (rc != HCBK_OK) return rc;
  const unsigned epoch = st->workspace_epoch;
  const long long before = launch_count();
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    cudaGetLastError();
    return HCBK_OK;
  }
  const char *p2 = nullptr;
  const int rc2 = dispatch_gemm(st, a, stream, &p2);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
  const long long captured = launch_count() - before;
  count_launch((int)-captured); /* nothing ran while capturing */
  cudaGraphExec_t exec = nullptr;
  if (rc2 == HCBK_OK && ce == cudaSuccess && graph && st->workspace_epoch == epoch &&
      cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
    if (st->graph_cache.size() >= 16) {
      cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(st->graph_cache.front().exec));
      st->graph_cache.erase(st->graph_cache.begin());
    }
    HcblasGraphEntry e;
    e.key = key;
    e.exec = exec;
    e.launches = captured;
    e.path = *path;
    st->graph_cache.push_back(std::move(e));
  } else {
    cudaGetLastError();
  }
  if (graph) cudaGraphDestroy(graph);
  return HCBK_OK;
}

hcblasStatus run_gemm(Hcblaslibrary *h, const hc::accelerator_view &view, GemmCall g) {
  /* quick return, exactly as the reference's class methods
   * (sgemm_array_wrapper.cpp:307-309 and :341-343) */
  const bool ptrs_missing = g.a_arr ? (g.a_arr == nullptr || g.b_arr == nullptr || g.c_arr == nullptr)
                                    : (g.a == nullptr || g.b == nullptr || g.c == nullptr);
  if (ptrs_missing || g.m == 0 || g.n == 0 || g.k == 0) return HCBLAS_INVALID;
  if (g.m < 0 || g.n < 0 || g.k < 0 || g.batch < 0) return HCBLAS_INVALID;
  if (g.batch == 0) return HCBLAS_SUCCEEDS;
  if (h == nullptr || !h->initialized || h->impl == nullptr) return HCBLAS_INVALID;

  DeviceGuard dev(view.device_id);
  if (!dev.ok()) return HCBLAS_INVALID;

  /* row-major C = op(A) op(B)  <=>  column-major C^T = op(B)^T op(A)^T */
  if (g.order == RowMajor) {
    std::swap(g.a, g.b);
    std::swap(g.a_arr, g.b_arr);
    std::swap(g.lda, g.ldb);
    std::swap(g.a_off, g.b_off);
    std::swap(g.stride_a, g.stride_b);
    std::swap(g.op_a, g.op_b);
    std::swap(g.m, g.n);
    g.order = ColMajor;
  }
  if (!is_complex(g.dtype)) {
    if (g.op_a == HCBK_OP_C) g.op_a = HCBK_OP_T;
    if (g.op_b == HCBK_OP_C) g.op_b = HCBK_OP_T;
  }

  hcbk_gemm_args a;
  std::memset(&a, 0, sizeof(a));
  a.dtype = g.dtype;
  a.op_a = g.op_a;
  a.op_b = g.op_b;
  a.m = g.m;
  a.n = g.n;
  a.k = g.k;
  a.a = g.a;
  a.lda = g.lda;
  a.stride_a = g.stride_a;
  a.a_off = g.a_off;
  a.b = g.b;
  a.ldb = g.ldb;
  a.stride_b = g.stride_b;
  a.b_off = g.b_off;
  a.c = g.c;
  a.ldc = g.ldc;
  a.stride_c = g.stride_c;
  a.c_off = g.c_off;
  a.a_array = g.a_arr;
  a.b_array = g.b_arr;
  a.c_array = g.c_arr;
  a.batch = g.batch;
  a.alpha_re = g.alpha_re;
  a.alpha_im = is_complex(g.dtype) ? g.alpha_im : 0.0;
  a.beta_re = g.beta_re;
  a.beta_im = is_complex(g.dtype) ? g.beta_im : 0.0;

  void *stream = view.stream;
  int rc;
  const char *path;
  if (a.alpha_re == 0.0 && a.alpha_im == 0.0) {
    /* alpha == 0: C := beta*C, A and B are not referenced (CBLAS) */
    path = "scale";
    rc = timed_launch(h->impl, stream, path, [&] { return hcbk_scale_c(&a, stream); });
  } else if (h->impl->graphs && !h->impl->profiling && !h->impl->inject_timeout &&
             stream != nullptr) {
    rc = dispatch_with_graph(h->impl, &a, stream, &path);
  } else {
    rc = dispatch_gemm(h->impl, &a, stream, &path);
  }
  h->impl->last_path = path;
  if (log_enabled())
    std::fprintf(stderr, "[hcblas] dt=%d op=%d%d m=%lld n=%lld k=%lld batch=%lld path=%s rc=%d\n",
                 a.dtype, a.op_a, a.op_b, (long long)a.m, (long long)a.n, (long long)a.k,
                 (long long)a.batch, path, rc);
  return rc == HCBK_OK ? HCBLAS_SUCCEEDS : HCBLAS_INVALID;
}

}  // namespace hcblas_b200

using hcblas_b200::char_from_op;
using hcblas_b200::GemmCall;
using hcblas_b200::op_from_char;
using hcblas_b200::run_gemm;

namespace {

GemmCall make_call(int dtype, hcblasOrder order, hcblasTranspose ta, hcblasTranspose tb, int M,
                   int N, int K, double ar, double ai, double br, double bi) {
  GemmCall g;
  std::memset(&g, 0, sizeof(g));
  g.dtype = dtype;
  g.order = order;
  g.op_a = op_from_char(ta);
  g.op_b = op_from_char(tb);
  g.m = M;
  g.n = N;
  g.k = K;
  g.alpha_re = ar;
  g.alpha_im = ai;
  g.beta_re = br;
  g.beta_im = bi;
  g.batch = 1;
  return g;
}

void set_single(GemmCall &g, const void *A, int64_t lda, int64_t aoff, const void *B, int64_t ldb,
                int64_t boff, void *C, int64_t ldc, int64_t coff) {
  g.a = A;
  g.lda = lda;
  g.a_off = aoff;
  g.b = B;
  g.ldb = ldb;
  g.b_off = boff;
  g.c = C;
  g.ldc = ldc;
  g.c_off = coff;
}

void set_batched(GemmCall &g, void *const *A, int64_t lda, int64_t aoff, int64_t abo,
                 void *const *B, int64_t ldb, int64_t boff, int64_t bbo, void *const *C,
                 int64_t ldc, int64_t coff, int64_t cbo, int batch) {
  g.a_arr = reinterpret_cast<const void *const *>(A);
  g.lda = lda;
  g.a_off = aoff;
  g.stride_a = abo;
  g.b_arr = reinterpret_cast<const void *const *>(B);
  g.ldb = ldb;
  g.b_off = boff;
  g.stride_b = bbo;
  g.c_arr = C;
  g.ldc = ldc;
  g.c_off = coff;
  g.stride_c = cbo;
  g.batch = batch;
}

}  // namespace

/* ------------------------------------------------------ class methods -- */

hcblasStatus Hcblaslibrary::hcblas_sgemm(hc::accelerator_view accl_view, hcblasOrder order,
                                         hcblasTranspose typeA, hcblasTranspose typeB,
                                         const int M, const int N, const int K,
                                         const float &alpha, float *A, const int64_t lda,
                                         float *B, const int64_t ldb, const float &beta,
                                         float *C, const int64_t ldc, const int64_t aOffset,
                                         const int64_t bOffset, const int64_t cOffset) {
  GemmCall g = make_call(HCBK_S, order, typeA, typeB, M, N, K, alpha, 0, beta, 0);
  set_single(g, A, lda, aOffset, B, ldb, bOffset, C, ldc, cOffset);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_dgemm(hc::accelerator_view accl_view, hcblasOrder order,
                                         hcblasTranspose typeA, hcblasTranspose typeB,
                                         const int M, const int N, const int K,
                                         const double &alpha, double *A, const int64_t lda,
                                         double *B, const int64_t ldb, const double &beta,
                                         double *C, const int64_t ldc, const int64_t aOffset,
                                         const int64_t bOffset, const int64_t cOffset) {
  GemmCall g = make_call(HCBK_D, order, typeA, typeB, M, N, K, alpha, 0, beta, 0);
  set_single(g, A, lda, aOffset, B, ldb, bOffset, C, ldc, cOffset);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_hgemm(hc::accelerator_view accl_view, hcblasOrder order,
                                         hcblasTranspose typeA, hcblasTranspose typeB,
                                         const int M, const int N, const int K,
                                         const hc::half &alpha, hc::half *A, const int64_t lda,
                                         hc::half *B, const int64_t ldb, const hc::half &beta,
                                         hc::half *C, const int64_t ldc, const int64_t aOffset,
                                         const int64_t bOffset, const int64_t cOffset) {
  GemmCall g = make_call(HCBK_H, order, typeA, typeB, M, N, K, (float)alpha, 0, (float)beta, 0);
  set_single(g, A, lda, aOffset, B, ldb, bOffset, C, ldc, cOffset);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_sgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K, const float &alpha, float *A[],
    const int64_t lda, const int64_t A_batchOffset, float *B[], const int64_t ldb,
    const int64_t B_batchOffset, const float &beta, float *C[], const int64_t ldc,
    const int64_t C_batchOffset, const int64_t aOffset, const int64_t bOffset,
    const int64_t cOffset, const int batchSize) {
  GemmCall g = make_call(HCBK_S, order, typeA, typeB, M, N, K, alpha, 0, beta, 0);
  set_batched(g, reinterpret_cast<void *const *>(A), lda, aOffset, A_batchOffset,
              reinterpret_cast<void *const *>(B), ldb, bOffset, B_batchOffset,
              reinterpret_cast<void *const *>(C), ldc, cOffset, C_batchOffset, batchSize);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_dgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K, const double &alpha,
    double *A[], const int64_t lda, const int64_t A_batchOffset, double *B[], const int64_t ldb,
    const int64_t B_batchOffset, const double &beta, double *C[], const int64_t ldc,
    const int64_t C_batchOffset, const int64_t aOffset, const int64_t bOffset,
    const int64_t cOffset, const int batchSize) {
  GemmCall g = make_call(HCBK_D, order, typeA, typeB, M, N, K, alpha, 0, beta, 0);
  set_batched(g, reinterpret_cast<void *const *>(A), lda, aOffset, A_batchOffset,
              reinterpret_cast<void *const *>(B), ldb, bOffset, B_batchOffset,
              reinterpret_cast<void *const *>(C), ldc, cOffset, C_batchOffset, batchSize);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_hgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K, const hc::half &alpha,
    hc::half *A[], const int64_t lda, const int64_t A_batchOffset, hc::half *B[],
    const int64_t ldb, const int64_t B_batchOffset, const hc::half &beta, hc::half *C[],
    const int64_t ldc, const int64_t C_batchOffset, const int64_t aOffset,
    const int64_t bOffset, const int64_t cOffset, const int batchSize) {
  GemmCall g = make_call(HCBK_H, order, typeA, typeB, M, N, K, (float)alpha, 0, (float)beta, 0);
  set_batched(g, reinterpret_cast<void *const *>(A), lda, aOffset, A_batchOffset,
              reinterpret_cast<void *const *>(B), ldb, bOffset, B_batchOffset,
              reinterpret_cast<void *const *>(C), ldc, cOffset, C_batchOffset, batchSize);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_cgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K,
    const hc::short_vector::float_2 &alpha, hc::short_vector::float_2 *A, const int64_t aOffset,
    const int64_t lda, hc::short_vector::float_2 *B, const int64_t bOffset, const int64_t ldb,
    const hc::short_vector::float_2 &beta, hc::short_vector::float_2 *C, const int64_t cOffset,
    const int64_t ldc) {
  GemmCall g = make_call(HCBK_C, order, typeA, typeB, M, N, K, alpha.x, alpha.y, beta.x, beta.y);
  set_single(g, A, lda, aOffset, B, ldb, bOffset, C, ldc, cOffset);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_zgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K,
    const hc::short_vector::double_2 &alpha, hc::short_vector::double_2 *A,
    const int64_t aOffset, const int64_t lda, hc::short_vector::double_2 *B,
    const int64_t bOffset, const int64_t ldb, const hc::short_vector::double_2 &beta,
    hc::short_vector::double_2 *C, const int64_t cOffset, const int64_t ldc) {
  GemmCall g = make_call(HCBK_Z, order, typeA, typeB, M, N, K, alpha.x, alpha.y, beta.x, beta.y);
  set_single(g, A, lda, aOffset, B, ldb, bOffset, C, ldc, cOffset);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_cgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K,
    const hc::short_vector::float_2 &alpha, hc::short_vector::float_2 *A[],
    const int64_t aOffset, const int64_t A_batchOffset, const int64_t lda,
    hc::short_vector::float_2 *B[], const int64_t bOffset, const int64_t B_batchOffset,
    const int64_t ldb, const hc::short_vector::float_2 &beta, hc::short_vector::float_2 *C[],
    const int64_t cOffset, const int64_t C_batchOffset, const int64_t ldc,
    const int batchSize) {
  GemmCall g = make_call(HCBK_C, order, typeA, typeB, M, N, K, alpha.x, alpha.y, beta.x, beta.y);
  set_batched(g, reinterpret_cast<void *const *>(A), lda, aOffset, A_batchOffset,
              reinterpret_cast<void *const *>(B), ldb, bOffset, B_batchOffset,
              reinterpret_cast<void *const *>(C), ldc, cOffset, C_batchOffset, batchSize);
  return run_gemm(this, accl_view, g);
}

hcblasStatus Hcblaslibrary::hcblas_zgemm(
    hc::accelerator_view accl_view, hcblasOrder order, hcblasTranspose typeA,
    hcblasTranspose typeB, const int M, const int N, const int K,
    const hc::short_vector::double_2 &alpha, hc::short_vector::double_2 *A[],
    const int64_t aOffset, const int64_t A_batchOffset, const int64_t lda,
    hc::short_vector::double_2 *B[], const int64_t bOffset, const int64_t B_batchOffset,
    const int64_t ldb, const hc::short_vector::double_2 &beta, hc::short_vector::double_2 *C[],
    const int64_t cOffset, const int64_t C_batchOffset, const int64_t ldc,
    const int batchSize) {
  GemmCall g = make_call(HCBK_Z, order, typeA, typeB, M, N, K, alpha.x, alpha.y, beta.x, beta.y);
  set_batched(g, reinterpret_cast<void *const *>(A), lda, aOffset, A_batchOffset,
              reinterpret_cast<void *const *>(B), ldb, bOffset, B_batchOffset,
              reinterpret_cast<void *const *>(C), ldc, cOffset, C_batchOffset, batchSize);
  return run_gemm(this, accl_view, g);
}

/* ----------------------------------------------------------------- C API -- */

namespace {

inline bool handle_ok(hcblasHandle_t h) { return h != nullptr && h->initialized; }

inline hcblasStatus_t to_status(hcblasStatus s) {
  return s == HCBLAS_SUCCEEDS ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_EXECUTION_FAILED;
}

/* Shared body of hcblas{S,D,C,Z,H}gemm (lib/src/hcblas.cpp:1304-1450):
 * handle check, m/n/k < 0 check, zero offsets, host-side alpha/beta. */
hcblasStatus_t c_gemm(hcblasHandle_t handle, int dtype, hcblasOperation_t transa,
                      hcblasOperation_t transb, int m, int n, int k, double ar, double ai,
                      const void *A, int lda, const void *B, int ldb, double br, double bi,
                      void *C, int ldc) {
  GemmCall g = make_call(dtype, handle->Order, char_from_op(transa), char_from_op(transb), m, n,
                         k, ar, ai, br, bi);
  set_single(g, A, lda, 0, B, ldb, 0, C, ldc, 0);
  return to_status(run_gemm(handle, handle->currentAcclView, g));
}

hcblasStatus_t c_gemm_batched(hcblasHandle_t handle, int dtype, hcblasOperation_t transa,
                              hcblasOperation_t transb, int m, int n, int k, double ar,
                              double ai, void *const *A, int lda, void *const *B, int ldb,
                              double br, double bi, void *const *C, int ldc, int batch) {
  GemmCall g = make_call(dtype, handle->Order, char_from_op(transa), char_from_op(transb), m, n,
                         k, ar, ai, br, bi);
  /* The reference passes C_batchOffset = m*n for C/Z (lib/src/hcblas.cpp:1576,
   * 1653), which its pointer-array kernels never read
   * (cgemm_array_kernels_batch.cpp:143-157 index C[elt] + cOffset only): every
   * batch offset is 0 here. */
  set_batched(g, A, lda, 0, 0, B, ldb, 0, 0, C, ldc, 0, 0, batch);
  return to_status(run_gemm(handle, handle->currentAcclView, g));
}

hcblasStatus_t c_gemm_strided(hcblasHandle_t handle, int dtype, hcblasOperation_t transa,
                              hcblasOperation_t transb, int m, int n, int k, double ar,
                              double ai, const void *A, int lda, long long sA, const void *B,
                              int ldb, long long sB, double br, double bi, void *C, int ldc,
                              long long sC, int batch) {
  GemmCall g = make_call(dtype, handle->Order, char_from_op(transa), char_from_op(transb), m, n,
                         k, ar, ai, br, bi);
  set_single(g, A, lda, 0, B, ldb, 0, C, ldc, 0);
  g.stride_a = sA;
  g.stride_b = sB;
  g.stride_c = sC;
  g.batch = batch;
  return to_status(run_gemm(handle, handle->currentAcclView, g));
}

}  // namespace

#define HCBLAS_CHECK_ARGS(extra)                                       \
  if (!handle_ok(handle)) return HCBLAS_STATUS_NOT_INITIALIZED;        \
  if (m < 0 || n < 0 || k < 0 extra) return HCBLAS_STATUS_INVALID_VALUE; \
  if (alpha == nullptr || beta == nullptr) return HCBLAS_STATUS_INVALID_VALUE;

extern "C" hcblasStatus_t hcblasSgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                                      hcblasOperation_t transb, int m, int n, int k,
                                      const float *alpha, float *A, int lda, float *B, int ldb,
                                      const float *beta, float *C, int ldc) {
  HCBLAS_CHECK_ARGS()
  return c_gemm(handle, HCBK_S, transa, transb, m, n, k, *alpha, 0, A, lda, B, ldb, *beta, 0, C,
                ldc);
}

extern "C" hcblasStatus_t hcblasDgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                                      hcblasOperation_t transb, int m, int n, int k,
                                      const double *alpha, double *A, int lda, double *B,
                                      int ldb, const double *beta, double *C, int ldc) {
  HCBLAS_CHECK_ARGS()
  return c_gemm(handle, HCBK_D, transa, transb, m, n, k, *alpha, 0, A, lda, B, ldb, *beta, 0, C,
                ldc);
}

extern "C" hcblasStatus_t hcblasCgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                                      hcblasOperation_t transb, int m, int n, int k,
                                      const hcComplex *alpha, hcComplex *A, int lda,
                                      hcComplex *B, int ldb, const hcComplex *beta,
                                      hcComplex *C, int ldc) {
  HCBLAS_CHECK_ARGS()
  return c_gemm(handle, HCBK_C, transa, transb, m, n, k, alpha->x, alpha->y, A, lda, B, ldb,
                beta->x, beta->y, C, ldc);
}

extern "C" hcblasStatus_t hcblasZgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                                      hcblasOperation_t transb, int m, int n, int k,
                                      const hcDoubleComplex *alpha, hcDoubleComplex *A, int lda,
                                      hcDoubleComplex *B, int ldb, const hcDoubleComplex *beta,
                                      hcDoubleComplex *C, int ldc) {
  HCBLAS_CHECK_ARGS()
  return c_gemm(handle, HCBK_Z, transa, transb, m, n, k, alpha->x, alpha->y, A, lda, B, ldb,
                beta->x, beta->y, C, ldc);
}

extern "C" hcblasStatus_t hcblasHgemm(hcblasHandle_t handle, hcblasOperation_t transa,
                                      hcblasOperation_t transb, int m, int n, int k,
                                      const hcblasHalf *alpha, hcblasHalf *A, int lda,
                                      hcblasHalf *B, int ldb, const hcblasHalf *beta,
                                      hcblasHalf *C, int ldc) {
  HCBLAS_CHECK_ARGS()
  return c_gemm(handle, HCBK_H, transa, transb, m, n, k, hc::half::to_float(alpha->bits), 0, A,
                lda, B, ldb, hc::half::to_float(beta->bits), 0, C, ldc);
}

extern "C" hcblasStatus_t hcblasSgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                             hcblasOperation_t transb, int m, int n, int k,
                                             const float *alpha, float *Aarray[], int lda,
                                             float *Barray[], int ldb, const float *beta,
                                             float *Carray[], int ldc, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_batched(handle, HCBK_S, transa, transb, m, n, k, *alpha, 0,
                        reinterpret_cast<void *const *>(Aarray), lda,
                        reinterpret_cast<void *const *>(Barray), ldb, *beta, 0,
                        reinterpret_cast<void *const *>(Carray), ldc, batchCount);
}

extern "C" hcblasStatus_t hcblasCgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                             hcblasOperation_t transb, int m, int n, int k,
                                             const hcComplex *alpha, hcComplex *Aarray[],
                                             int lda, hcComplex *Barray[], int ldb,
                                             const hcComplex *beta, hcComplex *Carray[], int ldc,
                                             int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_batched(handle, HCBK_C, transa, transb, m, n, k, alpha->x, alpha->y,
                        reinterpret_cast<void *const *>(Aarray), lda,
                        reinterpret_cast<void *const *>(Barray), ldb, beta->x, beta->y,
                        reinterpret_cast<void *const *>(Carray), ldc, batchCount);
}

extern "C" hcblasStatus_t hcblasDgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                             hcblasOperation_t transb, int m, int n, int k,
                                             const double *alpha, double *Aarray[], int lda,
                                             double *Barray[], int ldb, const double *beta,
                                             double *Carray[], int ldc, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_batched(handle, HCBK_D, transa, transb, m, n, k, *alpha, 0,
                        reinterpret_cast<void *const *>(Aarray), lda,
                        reinterpret_cast<void *const *>(Barray), ldb, *beta, 0,
                        reinterpret_cast<void *const *>(Carray), ldc, batchCount);
}

extern "C" hcblasStatus_t hcblasZgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                             hcblasOperation_t transb, int m, int n, int k,
                                             const hcDoubleComplex *alpha,
                                             hcDoubleComplex *Aarray[], int lda,
                                             hcDoubleComplex *Barray[], int ldb,
                                             const hcDoubleComplex *beta,
                                             hcDoubleComplex *Carray[], int ldc, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_batched(handle, HCBK_Z, transa, transb, m, n, k, alpha->x, alpha->y,
                        reinterpret_cast<void *const *>(Aarray), lda,
                        reinterpret_cast<void *const *>(Barray), ldb, beta->x, beta->y,
                        reinterpret_cast<void *const *>(Carray), ldc, batchCount);
}

extern "C" hcblasStatus_t hcblasHgemmBatched(hcblasHandle_t handle, hcblasOperation_t transa,
                                             hcblasOperation_t transb, int m, int n, int k,
                                             const hcblasHalf *alpha, hcblasHalf *Aarray[],
                                             int lda, hcblasHalf *Barray[], int ldb,
                                             const hcblasHalf *beta, hcblasHalf *Carray[],
                                             int ldc, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_batched(handle, HCBK_H, transa, transb, m, n, k,
                        hc::half::to_float(alpha->bits), 0,
                        reinterpret_cast<void *const *>(Aarray), lda,
                        reinterpret_cast<void *const *>(Barray), ldb,
                        hc::half::to_float(beta->bits), 0,
                        reinterpret_cast<void *const *>(Carray), ldc, batchCount);
}

extern "C" hcblasStatus_t hcblasSgemmStridedBatched(
    hcblasHandle_t handle, hcblasOperation_t transa, hcblasOperation_t transb, int m, int n,
    int k, const float *alpha, const float *A, int lda, long long strideA, const float *B,
    int ldb, long long strideB, const float *beta, float *C, int ldc, long long strideC,
    int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_strided(handle, HCBK_S, transa, transb, m, n, k, *alpha, 0, A, lda, strideA, B,
                        ldb, strideB, *beta, 0, C, ldc, strideC, batchCount);
}

extern "C" hcblasStatus_t hcblasDgemmStridedBatched(
    hcblasHandle_t handle, hcblasOperation_t transa, hcblasOperation_t transb, int m, int n,
    int k, const double *alpha, const double *A, int lda, long long strideA, const double *B,
    int ldb, long long strideB, const double *beta, double *C, int ldc, long long strideC,
    int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_strided(handle, HCBK_D, transa, transb, m, n, k, *alpha, 0, A, lda, strideA, B,
                        ldb, strideB, *beta, 0, C, ldc, strideC, batchCount);
}

extern "C" hcblasStatus_t hcblasCgemmStridedBatched(
    hcblasHandle_t handle, hcblasOperation_t transa, hcblasOperation_t transb, int m, int n,
    int k, const hcComplex *alpha, const hcComplex *A, int lda, long long strideA,
    const hcComplex *B, int ldb, long long strideB, const hcComplex *beta, hcComplex *C,
    int ldc, long long strideC, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_strided(handle, HCBK_C, transa, transb, m, n, k, alpha->x, alpha->y, A, lda,
                        strideA, B, ldb, strideB, beta->x, beta->y, C, ldc, strideC, batchCount);
}

extern "C" hcblasStatus_t hcblasZgemmStridedBatched(
    hcblasHandle_t handle, hcblasOperation_t transa, hcblasOperation_t transb, int m, int n,
    int k, const hcDoubleComplex *alpha, const hcDoubleComplex *A, int lda, long long strideA,
    const hcDoubleComplex *B, int ldb, long long strideB, const hcDoubleComplex *beta,
    hcDoubleComplex *C, int ldc, long long strideC, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_strided(handle, HCBK_Z, transa, transb, m, n, k, alpha->x, alpha->y, A, lda,
                        strideA, B, ldb, strideB, beta->x, beta->y, C, ldc, strideC, batchCount);
}

extern "C" hcblasStatus_t hcblasHgemmStridedBatched(
    hcblasHandle_t handle, hcblasOperation_t transa, hcblasOperation_t transb, int m, int n,
    int k, const hcblasHalf *alpha, const hcblasHalf *A, int lda, long long strideA,
    const hcblasHalf *B, int ldb, long long strideB, const hcblasHalf *beta, hcblasHalf *C,
    int ldc, long long strideC, int batchCount) {
  HCBLAS_CHECK_ARGS(|| batchCount < 0)
  return c_gemm_strided(handle, HCBK_H, transa, transb, m, n, k, hc::half::to_float(alpha->bits),
                        0, A, lda, strideA, B, ldb, strideB, hc::half::to_float(beta->bits), 0, C,
                        ldc, strideC, batchCount);
}

/* ------------------------------------------------- class-API C shims -- */

namespace {

hcblasTranspose tchar(char c) {
  if (c == 'n' || c == 'N') return NoTrans;
  if (c == 'c' || c == 'C') return ConjTrans;
  return Trans;
}

hcblasOrder ord(int o) { return o == 0 ? RowMajor : ColMajor; }

}  // namespace

extern "C" int hcblasLibSgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N,
                              int K, const float *alpha, float *A, int64_t lda, float *B,
                              int64_t ldb, const float *beta, float *C, int64_t ldc,
                              int64_t aOffset, int64_t bOffset, int64_t cOffset) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  return h->hcblas_sgemm(h->currentAcclView, ord(order), tchar(typeA), tchar(typeB), M, N, K,
                         *alpha, A, lda, B, ldb, *beta, C, ldc, aOffset, bOffset, cOffset);
}

extern "C" int hcblasLibDgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N,
                              int K, const double *alpha, double *A, int64_t lda, double *B,
                              int64_t ldb, const double *beta, double *C, int64_t ldc,
                              int64_t aOffset, int64_t bOffset, int64_t cOffset) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  return h->hcblas_dgemm(h->currentAcclView, ord(order), tchar(typeA), tchar(typeB), M, N, K,
                         *alpha, A, lda, B, ldb, *beta, C, ldc, aOffset, bOffset, cOffset);
}

extern "C" int hcblasLibHgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N,
                              int K, const hcblasHalf *alpha, hcblasHalf *A, int64_t lda,
                              hcblasHalf *B, int64_t ldb, const hcblasHalf *beta, hcblasHalf *C,
                              int64_t ldc, int64_t aOffset, int64_t bOffset, int64_t cOffset) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  return h->hcblas_hgemm(h->currentAcclView, ord(order), tchar(typeA), tchar(typeB), M, N, K,
                         *alpha, A, lda, B, ldb, *beta, C, ldc, aOffset, bOffset, cOffset);
}

extern "C" int hcblasLibCgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N,
                              int K, const hcComplex *alpha, hcComplex *A, int64_t aOffset,
                              int64_t lda, hcComplex *B, int64_t bOffset, int64_t ldb,
                              const hcComplex *beta, hcComplex *C, int64_t cOffset,
                              int64_t ldc) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  hc::short_vector::float_2 al(alpha->x, alpha->y), be(beta->x, beta->y);
  return h->hcblas_cgemm(h->currentAcclView, ord(order), tchar(typeA), tchar(typeB), M, N, K, al,
                         reinterpret_cast<hc::short_vector::float_2 *>(A), aOffset, lda,
                         reinterpret_cast<hc::short_vector::float_2 *>(B), bOffset, ldb, be,
                         reinterpret_cast<hc::short_vector::float_2 *>(C), cOffset, ldc);
}

extern "C" int hcblasLibZgemm(hcblasHandle_t h, int order, char typeA, char typeB, int M, int N,
                              int K, const hcDoubleComplex *alpha, hcDoubleComplex *A,
                              int64_t aOffset, int64_t lda, hcDoubleComplex *B, int64_t bOffset,
                              int64_t ldb, const hcDoubleComplex *beta, hcDoubleComplex *C,
                              int64_t cOffset, int64_t ldc) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  hc::short_vector::double_2 al(alpha->x, alpha->y), be(beta->x, beta->y);
  return h->hcblas_zgemm(h->currentAcclView, ord(order), tchar(typeA), tchar(typeB), M, N, K, al,
                         reinterpret_cast<hc::short_vector::double_2 *>(A), aOffset, lda,
                         reinterpret_cast<hc::short_vector::double_2 *>(B), bOffset, ldb, be,
                         reinterpret_cast<hc::short_vector::double_2 *>(C), cOffset, ldc);
}

extern "C" int hcblasLibGemmBatched(hcblasHandle_t h, int dtype, int order, char typeA,
                                    char typeB, int M, int N, int K, const void *alpha, void **A,
                                    int64_t lda, int64_t A_batchOffset, void **B, int64_t ldb,
                                    int64_t B_batchOffset, const void *beta, void **C,
                                    int64_t ldc, int64_t C_batchOffset, int64_t aOffset,
                                    int64_t bOffset, int64_t cOffset, int batchSize) {
  if (!handle_ok(h) || !alpha || !beta) return HCBLAS_INVALID;
  double ar = 0, ai = 0, br = 0, bi = 0;
  switch (dtype) {
    case HCBK_S: ar = *(const float *)alpha; br = *(const float *)beta; break;
    case HCBK_D: ar = *(const double *)alpha; br = *(const double *)beta; break;
    case HCBK_C:
      ar = ((const float *)alpha)[0]; ai = ((const float *)alpha)[1];
      br = ((const float *)beta)[0]; bi = ((const float *)beta)[1];
      break;
    case HCBK_Z:
      ar = ((const double *)alpha)[0]; ai = ((const double *)alpha)[1];
      br = ((const double *)beta)[0]; bi = ((const double *)beta)[1];
      break;
    case HCBK_H:
      ar = hc::half::to_float(((const hcblas_half_t *)alpha)->bits);
      br = hc::half::to_float(((const hcblas_half_t *)beta)->bits);
      break;
    default: return HCBLAS_INVALID;
  }
  GemmCall g = make_call(dtype, ord(order), tchar(typeA), tchar(typeB), M, N, K, ar, ai, br, bi);
  set_batched(g, A, lda, aOffset, A_batchOffset, B, ldb, bOffset, B_batchOffset, C, ldc, cOffset,
              C_batchOffset, batchSize);
  return run_gemm(h, h->currentAcclView, g);
}
