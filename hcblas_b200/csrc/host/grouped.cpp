/*
 * grouped.cpp -- host side of the grouped (uneven batch) HGEMM: builds the
 * device problem table the persistent kernel walks (csrc/kernels/grouped.cu),
 * caches it per handle, and runs the problems the table cannot hold as
 * single calls.
 *
 * Plan: every problem is canonicalised to column-major (row-major handles
 * swap A and B, as run_gemm does), its tensor maps are encoded, and problems
 * are ordered by decreasing work (tiles x K-slabs) so that the kernel's
 * round-robin tile walk ends on the cheapest tiles.  The table (entries, then
 * the count + 1 tile prefix sums) is written into a pinned staging buffer and
 * copied to the device on the handle's stream.  A follow-up call with a
 * byte-identical problem array (and the same order and device) reuses the
 * device table as it is: no encoding, no copy.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "dispatch.h"

namespace hcblas_b200 {
namespace {

struct Canon {
  int op_a, op_b;
  int64_t m, n, k;
  const void *a;
  int64_t lda;
  const void *b;
  int64_t ldb;
  void *c;
  int64_t ldc;
};

/* column-major form; for real data the conjugate transpose is the transpose */
Canon canonical(const hcblasGemmProblem &p, hcblasOrder order) {
  Canon c;
  c.op_a = p.transa == HCBLAS_OP_N ? HCBK_OP_N : HCBK_OP_T;
  c.op_b = p.transb == HCBLAS_OP_N ? HCBK_OP_N : HCBK_OP_T;
  c.m = p.m;
  c.n = p.n;
  c.k = p.k;
  c.a = p.A;
  c.lda = p.lda;
  c.b = p.B;
  c.ldb = p.ldb;
  c.c = p.C;
  c.ldc = p.ldc;
  if (order == RowMajor) { /* C^T = op(B)^T op(A)^T */
    std::swap(c.a, c.b);
    std::swap(c.lda, c.ldb);
    std::swap(c.op_a, c.op_b);
    std::swap(c.m, c.n);
  }
  return c;
}

bool ensure_table(HcblasGroupedPlan &gp, size_t bytes, void *stream) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (gp.table && gp.table_bytes >= bytes && gp.table_device == dev) return true;
  if (gp.table) {
    /* queued kernels (or captured graphs) may still read the old table */
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    DeviceGuard g(gp.table_device);
    cudaFree(gp.table);
    gp.table = nullptr;
    gp.table_bytes = 0;
  }
  size_t want = bytes < (size_t)(1u << 20) ? (size_t)(1u << 20) : bytes;
  if (cudaMalloc(&gp.table, want) != cudaSuccess) {
    cudaGetLastError();
    gp.table = nullptr;
    return false;
  }
  gp.table_bytes = want;
  gp.table_device = dev;
  return true;
}

bool ensure_staging(HcblasGroupedPlan &gp, size_t bytes) {
  if (gp.upload_done) /* the previous upload still reads the staging buffer */
    cudaEventSynchronize(static_cast<cudaEvent_t>(gp.upload_done));
  if (gp.staging && gp.staging_bytes >= bytes) return true;
  if (gp.staging) cudaFreeHost(gp.staging);
  gp.staging = nullptr;
  gp.staging_bytes = 0;
  size_t want = bytes < (size_t)(1u << 20) ? (size_t)(1u << 20) : bytes;
  if (cudaHostAlloc(&gp.staging, want, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    gp.staging = nullptr;
    return false;
  }
  gp.staging_bytes = want;
  return true;
}

}  // namespace

/* Build (or reuse) the plan and run every problem; HCBK_* code. */
int grouped_hgemm(HcblasB200State *st, void *stream, hcblasOrder order, int count,
                  const hcblasGemmProblem *probs, float alpha, float beta) {
  if (alpha == 0.0f) { /* C_i := beta*C_i, A and B not referenced (CBLAS) */
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order);
      hcbk_gemm_args a;
      std::memset(&a, 0, sizeof(a));
      a.dtype = HCBK_H;
      a.m = c.m;
      a.n = c.n;
      a.k = c.k;
      a.c = c.c;
      a.ldc = c.ldc;
      a.batch = 1;
      a.beta_re = beta;
      int rc = timed_launch(st, stream, "scale", [&] { return hcbk_scale_c(&a, stream); });
      if (rc) return rc;
    }
    st->last_path = "scale";
    return HCBK_OK;
  }
  HcblasGroupedPlan &gp = st->grouped;
  int dev = 0;
  cudaGetDevice(&dev);
  std::vector<unsigned char> key(sizeof(hcblasGemmProblem) * (size_t)count + 2);
  std::memcpy(key.data(), probs, sizeof(hcblasGemmProblem) * (size_t)count);
  key[key.size() - 2] = static_cast<unsigned char>(order);
  key[key.size() - 1] = static_cast<unsigned char>(dev);
  const bool reuse = gp.table && gp.table_device == dev && key == gp.key;

  if (!reuse) {
    /* captured graphs of earlier grouped calls read this table: drop them */
    if (!st->graph_cache.empty()) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      clear_graph_cache(st);
    }
    gp.key.clear();
    std::vector<hcbk_grouped_entry> ent((size_t)count);
    std::vector<int> ok_idx;
    std::vector<int> fallback;
    ok_idx.reserve(count);
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order);
      int rc = hcbk_grouped_encode(&ent[i], c.op_a, c.op_b, c.m, c.n, c.k, c.a, c.lda, c.b,
                                   c.ldb, c.c, c.ldc);
      if (rc == HCBK_OK) ok_idx.push_back(i);
      else if (rc == HCBK_ERR_ALIGN || rc == HCBK_ERR_ARGS) fallback.push_back(i);
      else return rc;
    }
    auto work = [&](int i) {
      const hcbk_grouped_entry &e = ent[i];
      return (int64_t)e.tiles_m * ((e.n + 127) / 128) * ((e.k + 63) / 64);
    };
    std::stable_sort(ok_idx.begin(), ok_idx.end(),
                     [&](int x, int y) { return work(x) > work(y); });
    const int nt = (int)ok_idx.size();
    const size_t ent_bytes = sizeof(hcbk_grouped_entry) * (size_t)nt;
    const size_t ts_off = (ent_bytes + 255) & ~size_t(255);
    const size_t bytes = ts_off + sizeof(int32_t) * ((size_t)nt + 1);
    int64_t total = 0;
    if (nt > 0) {
      if (!ensure_table(gp, bytes, stream) || !ensure_staging(gp, bytes)) return HCBK_ERR_NOMEM;
      unsigned char *stg = static_cast<unsigned char *>(gp.staging);
      auto *dst = reinterpret_cast<hcbk_grouped_entry *>(stg);
      auto *ts = reinterpret_cast<int32_t *>(stg + ts_off);
      for (int j = 0; j < nt; ++j) {
        const hcbk_grouped_entry &e = ent[ok_idx[j]];
        std::memcpy(&dst[j], &e, sizeof(e));
        ts[j] = (int32_t)total;
        total += (int64_t)e.tiles_m * ((e.n + 127) / 128);
        if (total > 0x7fffffff) return HCBK_ERR_ARGS;
      }
      ts[nt] = (int32_t)total;
      if (cudaMemcpyAsync(gp.table, stg, bytes, cudaMemcpyHostToDevice,
                          static_cast<cudaStream_t>(stream)) != cudaSuccess)
        return HCBK_ERR_LAUNCH;
      if (!gp.upload_done &&
          cudaEventCreateWithFlags(reinterpret_cast<cudaEvent_t *>(&gp.upload_done),
                                   cudaEventDisableTiming) != cudaSuccess) {
        gp.upload_done = nullptr;
        cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      } else {
        cudaEventRecord(static_cast<cudaEvent_t>(gp.upload_done),
                        static_cast<cudaStream_t>(stream));
      }
    }
    gp.count = nt;
    gp.total_tiles = (int)total;
    gp.tile_start_offset = ts_off;
    gp.fallback = fallback;
    gp.key = key;
  }

  int *err = device_error_flag(st);
  if (!err) return HCBK_ERR_NOMEM;
  if (gp.count > 0) {
    hcbk_grouped_args g;
    g.table = static_cast<const hcbk_grouped_entry *>(gp.table);
    g.tile_start =
        reinterpret_cast<const int32_t *>(static_cast<char *>(gp.table) + gp.tile_start_offset);
    g.count = gp.count;
    g.total_tiles = gp.total_tiles;
    g.alpha = alpha;
    g.beta = beta;
    int rc = timed_launch(st, stream, "tc.h.grouped",
                          [&] { return hcbk_hgemm_grouped_tc(&g, err, stream); });
    if (rc) return rc;
  }
  for (int i : gp.fallback) {
    const Canon c = canonical(probs[i], order);
    hcbk_gemm_args a;
    std::memset(&a, 0, sizeof(a));
    a.dtype = HCBK_H;
    a.op_a = c.op_a;
    a.op_b = c.op_b;
    a.m = c.m;
    a.n = c.n;
    a.k = c.k;
    a.a = c.a;
    a.lda = c.lda;
    a.b = c.b;
    a.ldb = c.ldb;
    a.c = c.c;
    a.ldc = c.ldc;
    a.batch = 1;
    a.alpha_re = alpha;
    a.beta_re = beta;
    const char *path = nullptr;
    int rc = dispatch_gemm(st, &a, stream, &path);
    if (rc) return rc;
  }
  st->last_path = gp.fallback.empty() ? "tc.h.grouped" : "tc.h.grouped+single";
  return HCBK_OK;
}

}  // namespace hcblas_b200

extern "C" hcblasStatus_t hcblasHgemmGrouped(hcblasHandle_t handle, int count,
                                             const hcblasGemmProblem *problems,
                                             const hcblasHalf *alpha, const hcblasHalf *beta) {
  using namespace hcblas_b200;
  if (handle == nullptr || !handle->initialized || handle->impl == nullptr)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (count < 0 || (count > 0 && problems == nullptr) || alpha == nullptr || beta == nullptr)
    return HCBLAS_STATUS_INVALID_VALUE;
  for (int i = 0; i < count; ++i)
    if (problems[i].m < 0 || problems[i].n < 0 || problems[i].k < 0)
      return HCBLAS_STATUS_INVALID_VALUE;
  for (int i = 0; i < count; ++i) {
    const hcblasGemmProblem &p = problems[i];
    if (p.m == 0 || p.n == 0 || p.k == 0 || p.A == nullptr || p.B == nullptr || p.C == nullptr)
      return HCBLAS_STATUS_EXECUTION_FAILED;
  }
  if (count == 0) return HCBLAS_STATUS_SUCCESS;
  DeviceGuard dev(handle->currentAcclView.device_id);
  if (!dev.ok()) return HCBLAS_STATUS_EXECUTION_FAILED;
  const float a = hc::half::to_float(alpha->bits), b = hc::half::to_float(beta->bits);
  int rc = grouped_hgemm(handle->impl, handle->currentAcclView.stream, handle->Order, count,
                         problems, a, b);
  if (log_enabled())
    std::fprintf(stderr, "[hcblas] grouped count=%d path=%s rc=%d\n", count,
                 handle->impl->last_path, rc);
  return rc == HCBK_OK ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_EXECUTION_FAILED;
}
