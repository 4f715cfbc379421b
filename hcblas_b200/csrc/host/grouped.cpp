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

/* column-major form; for real data the conjugate transpose is the
 * transpose, complex data keeps it */
Canon canonical(const hcblasGemmProblem &p, hcblasOrder order, bool cplx = false) {
  Canon c;
  auto op = [&](hcblasOperation_t t) {
    return t == HCBLAS_OP_N ? HCBK_OP_N : (cplx && t == HCBLAS_OP_C) ? HCBK_OP_C : HCBK_OP_T;
  };
  c.op_a = op(p.transa);
  c.op_b = op(p.transb);
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

bool grouped_ensure_table(HcblasGroupedPlan &gp, size_t bytes, void *stream) {
  return ensure_table(gp, bytes, stream);
}

/* Build (or reuse) the plan and run every problem; HCBK_* code. */
bool grouped_hgemm_compact_match(HcblasB200State *st, const std::vector<unsigned char> &compact) {
  const HcblasGroupedPlan &gp = st->grouped;
  int dev = 0;
  cudaGetDevice(&dev);
  return gp.table && gp.table_device == dev && !gp.compact_key.empty() &&
         gp.fallback.empty() && compact == gp.compact_key;
}

int grouped_hgemm(HcblasB200State *st, void *stream, hcblasOrder order, int count,
                  const hcblasGemmProblem *probs, float alpha, float beta,
                  const std::vector<unsigned char> *compact) {
  if (!probs && (alpha == 0.0f || !compact || !grouped_hgemm_compact_match(st, *compact)))
    return HCBK_ERR_ARGS;
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
  std::vector<unsigned char> key;
  bool reuse = compact && grouped_hgemm_compact_match(st, *compact);
  if (!reuse) {
    key.resize(sizeof(hcblasGemmProblem) * (size_t)count + 3);
    std::memcpy(key.data(), probs, sizeof(hcblasGemmProblem) * (size_t)count);
    key[key.size() - 3] = static_cast<unsigned char>(st->grouped_c_tma);
    key[key.size() - 2] = static_cast<unsigned char>(order);
    key[key.size() - 1] = static_cast<unsigned char>(dev);
    reuse = gp.table && gp.table_device == dev && key == gp.key;
  }

  if (!reuse) {
    /* captured graphs of earlier grouped calls read this table: drop them */
    if (!st->graph_cache.empty()) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      clear_graph_cache(st);
    }
    gp.key.clear();
    gp.compact_key.clear();
    std::vector<hcbk_grouped_entry> ent((size_t)count);
    std::vector<int> ok_idx;
    std::vector<int> fallback;
    ok_idx.reserve(count);
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order);
      int rc = hcbk_grouped_encode(&ent[i], c.op_a, c.op_b, c.m, c.n, c.k, c.a, c.lda, c.b,
                                   c.ldb, c.c, c.ldc);
      if (rc == HCBK_OK && !st->grouped_c_tma) ent[i].c_tma = 0; /* direct stores */
      if (rc == HCBK_OK) ok_idx.push_back(i);
      else if (rc == HCBK_ERR_ALIGN || rc == HCBK_ERR_ARGS) fallback.push_back(i);
      else return rc;
    }
    auto work = [&](int i) { /* tensor work of a problem's padded tiles */
      const hcbk_grouped_entry &e = ent[i];
      return (int64_t)hcbk_grouped_tiles(&e) * e.bn * ((e.k + 63) / 64);
    };
    std::stable_sort(ok_idx.begin(), ok_idx.end(),
                     [&](int x, int y) { return work(x) > work(y); });
    const int nt = (int)ok_idx.size();
    if (nt >= (1 << 24)) return HCBK_ERR_ARGS;
    int64_t total = 0, all_work = 0;
    for (int j = 0; j < nt; ++j) {
      total += (int64_t)hcbk_grouped_tiles(&ent[ok_idx[j]]);
      all_work += work(ok_idx[j]);
      if (total > 0x7fffffff) return HCBK_ERR_ARGS;
    }
    /* table: entries | tile prefix sums | per-tile descriptors */
    const size_t ent_bytes = sizeof(hcbk_grouped_entry) * (size_t)nt;
    const size_t ts_off = (ent_bytes + 255) & ~size_t(255);
    const size_t td_off = (ts_off + sizeof(int32_t) * ((size_t)nt + 1) + 255) & ~size_t(255);
    const size_t bytes = td_off + 4 * sizeof(int32_t) * (size_t)total;
    total = 0;
    if (nt > 0) {
      if (!ensure_table(gp, bytes, stream) || !ensure_staging(gp, bytes)) return HCBK_ERR_NOMEM;
      unsigned char *stg = static_cast<unsigned char *>(gp.staging);
      auto *dst = reinterpret_cast<hcbk_grouped_entry *>(stg);
      auto *ts = reinterpret_cast<int32_t *>(stg + ts_off);
      auto *td = reinterpret_cast<int32_t *>(stg + td_off);
      for (int j = 0; j < nt; ++j) {
        const hcbk_grouped_entry &e = ent[ok_idx[j]];
        std::memcpy(&dst[j], &e, sizeof(e));
        ts[j] = (int32_t)total;
        hcbk_grouped_fill_tiles(&e, j, td + 4 * total);
        total += (int64_t)hcbk_grouped_tiles(&e);
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
    gp.tile_desc_offset = td_off;
    gp.fallback = fallback;
    gp.work = all_work;
    gp.tuned_ctas = 0;
    gp.key = key;
  }
  if (compact) gp.compact_key = *compact; /* the table built or matched holds these problems */

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
    g.device_maps = 0;
    g.tile_desc =
        reinterpret_cast<const int32_t *>(static_cast<char *>(gp.table) + gp.tile_desc_offset);
    g.uniform_tiles = 0;
    g.u_tiles_m = g.u_k = g.u_flags = 0;
    g.ctas_per_sm = st->grouped_ctas;
    if (st->autotune) {
      /* one or two CTAs per SM, per bucket of problem count, tiles and
       * tensor work; tuned on a beta == 0 call, where every candidate
       * writes what the final launch rewrites, then kept with the plan */
      if (!gp.tuned_ctas && beta == 0.0f) {
        auto lg = [](int64_t v) {
          int r = 0;
          while (((int64_t)1 << r) < v && r < 62) ++r;
          return r;
        };
        char shape[96];
        std::snprintf(shape, sizeof(shape), "count%d|tiles%d|work%d", lg(gp.count),
                      lg(gp.total_tiles), lg(gp.work));
        gp.tuned_ctas = 1 + tune_choice(st, stream, tune_key_shape("grouped_h", shape), 2,
                                        [&](int i) {
                                          hcbk_grouped_args gi = g;
                                          gi.ctas_per_sm = 1 + i;
                                          return hcbk_hgemm_grouped_tc(&gi, err, stream);
                                        },
                                        st->grouped_ctas - 1);
      }
      if (gp.tuned_ctas) g.ctas_per_sm = gp.tuned_ctas;
    }
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

/* Grouped FP32 GEMM, split-BF16: the plan holds every problem's bf16 plane
 * layout (one device allocation), the pack jobs that fill it and the GEMM
 * table whose 3-D maps read it; each call packs the current operands (one
 * launch) and runs the grouped tensor-core kernel (one launch). */
int grouped_sgemm_split(HcblasB200State *st, void *stream, hcblasOrder order, int count,
                        const hcblasGemmProblem *probs, float alpha, float beta, int terms,
                        const PtrBatch *ptrs) {
  if (alpha == 0.0f) { /* C_i := beta*C_i, A and B not referenced (CBLAS) */
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order);
      hcbk_gemm_args a;
      std::memset(&a, 0, sizeof(a));
      a.dtype = HCBK_S;
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
  const int nplanes = terms == 6 ? 3 : 2;
  HcblasGroupedPlan &gp = st->grouped_split;
  int dev = 0;
  cudaGetDevice(&dev);
  std::vector<unsigned char> key(sizeof(hcblasGemmProblem) * (size_t)count + 3);
  std::memcpy(key.data(), probs, sizeof(hcblasGemmProblem) * (size_t)count);
  key[key.size() - 3] = static_cast<unsigned char>(order);
  key[key.size() - 2] = static_cast<unsigned char>(dev);
  key[key.size() - 1] = static_cast<unsigned char>(terms);
  const bool reuse = gp.table && gp.planes && gp.table_device == dev && key == gp.key;

  if (!reuse) {
    if (!st->graph_cache.empty()) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      clear_graph_cache(st);
    }
    gp.key.clear();
    /* plane layout: per problem, A planes then B planes, each plane
     * rows x kp bf16 (kp = K rounded up to 16: rows on 32-byte sectors),
     * problems 1 KiB aligned */
    std::vector<Canon> cn((size_t)count);
    std::vector<size_t> a_off((size_t)count), b_off((size_t)count);
    size_t total_planes = 0;
    for (int i = 0; i < count; ++i) {
      cn[i] = canonical(probs[i], order);
      const int64_t kp = (cn[i].k + 15) & ~int64_t(15);
      a_off[i] = total_planes;
      total_planes += (size_t)nplanes * cn[i].m * kp * 2;
      b_off[i] = total_planes;
      total_planes += (size_t)nplanes * cn[i].n * kp * 2;
      total_planes = (total_planes + 1023) & ~size_t(1023);
    }
    if (gp.planes && (gp.planes_bytes < total_planes || gp.table_device != dev)) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      DeviceGuard g(gp.table_device);
      cudaFree(gp.planes);
      gp.planes = nullptr;
      gp.planes_bytes = 0;
    }
    if (!gp.planes) {
      if (cudaMalloc(&gp.planes, total_planes) != cudaSuccess) {
        cudaGetLastError();
        gp.planes = nullptr;
        return HCBK_ERR_NOMEM;
      }
      gp.planes_bytes = total_planes;
    }
    char *pl = static_cast<char *>(gp.planes);
    std::vector<hcbk_grouped_entry> ent((size_t)count);
    std::vector<hcbk_gpack_job> jobs((size_t)count * 2);
    for (int i = 0; i < count; ++i) {
      const Canon &c = cn[i];
      const int64_t kp = (c.k + 15) & ~int64_t(15);
      if (c.m > 0x7fffffff || c.n > 0x7fffffff || c.k > 0x7fffffff) return HCBK_ERR_ARGS;
      hcbk_grouped_entry &e = ent[i];
      std::memset(&e, 0, sizeof(e));
      int rc = hcbk_encode_tma_3d_planes(e.map_a, 1, pl + a_off[i], c.k, c.m, nplanes, kp,
                                         (uint64_t)c.m * kp * 2, 128);
      if (!rc)
        rc = hcbk_encode_tma_3d_planes(e.map_b, 1, pl + b_off[i], c.k, c.n, nplanes, kp,
                                       (uint64_t)c.n * kp * 2, 128);
      if (rc) return rc;
      e.c = c.c;
      e.ldc = c.ldc;
      e.m = (int32_t)c.m;
      e.n = (int32_t)c.n;
      e.k = (int32_t)c.k;
      e.tiles_m = (int32_t)((c.m + 127) / 128);
      e.bn = 128; /* the split kernel's tile: 128 x 128 over K-major planes */
      /* op(A) rows m: column-major A is M-contiguous for N, K-contiguous for T;
       * op(B) rows n: B is K-contiguous for N, N-contiguous for T */
      for (int side = 0; side < 2; ++side) {
        hcbk_gpack_job &j = jobs[2 * i + side];
        std::memset(&j, 0, sizeof(j));
        j.src = static_cast<const float *>(side ? c.b : c.a);
        j.ld = side ? c.ldb : c.lda;
        j.k_contig = side ? (c.op_b == HCBK_OP_N) : (c.op_a != HCBK_OP_N);
        j.rows = (int32_t)(side ? c.n : c.m);
        j.kdim = (int32_t)c.k;
        j.ld_dst = (int32_t)kp;
        j.planes = pl + (side ? b_off[i] : a_off[i]);
        j.plane_stride = (int64_t)j.rows * kp;
        j.tiles_r = (j.rows + 31) / 32;
      }
    }
    std::vector<int> order_idx((size_t)count);
    for (int i = 0; i < count; ++i) order_idx[i] = i;
    auto work = [&](int i) {
      const hcbk_grouped_entry &e = ent[i];
      return (int64_t)e.tiles_m * ((e.n + 127) / 128) * ((e.k + 63) / 64);
    };
    std::stable_sort(order_idx.begin(), order_idx.end(),
                     [&](int x, int y) { return work(x) > work(y); });
    if (count >= (1 << 24)) return HCBK_ERR_ARGS;
    int64_t total_est = 0;
    for (int i = 0; i < count; ++i) {
      total_est += (int64_t)hcbk_grouped_tiles(&ent[i]);
      if (total_est > 0x7fffffff) return HCBK_ERR_ARGS;
    }
    /* table: entries | tile prefix | pack jobs | pack tile prefix | tile descriptors */
    const size_t ent_bytes = sizeof(hcbk_grouped_entry) * (size_t)count;
    const size_t ts_off = (ent_bytes + 255) & ~size_t(255);
    const size_t job_off = (ts_off + sizeof(int32_t) * ((size_t)count + 1) + 255) & ~size_t(255);
    const size_t njobs = (size_t)count * 2;
    const size_t jts_off = (job_off + sizeof(hcbk_gpack_job) * njobs + 255) & ~size_t(255);
    const size_t td_off = (jts_off + sizeof(int32_t) * (njobs + 1) + 255) & ~size_t(255);
    const size_t bytes = td_off + 4 * sizeof(int32_t) * (size_t)total_est;
    if (!ensure_table(gp, bytes, stream) || !ensure_staging(gp, bytes)) return HCBK_ERR_NOMEM;
    unsigned char *stg = static_cast<unsigned char *>(gp.staging);
    auto *dst = reinterpret_cast<hcbk_grouped_entry *>(stg);
    auto *ts = reinterpret_cast<int32_t *>(stg + ts_off);
    auto *jdst = reinterpret_cast<hcbk_gpack_job *>(stg + job_off);
    auto *jts = reinterpret_cast<int32_t *>(stg + jts_off);
    auto *td = reinterpret_cast<int32_t *>(stg + td_off);
    int64_t total = 0;
    for (int x = 0; x < count; ++x) {
      const hcbk_grouped_entry &e = ent[order_idx[x]];
      std::memcpy(&dst[x], &e, sizeof(e));
      ts[x] = (int32_t)total;
      hcbk_grouped_fill_tiles(&e, x, td + 4 * total);
      total += (int64_t)hcbk_grouped_tiles(&e);
    }
    ts[count] = (int32_t)total;
    int64_t ptotal = 0;
    for (size_t x = 0; x < njobs; ++x) {
      jdst[x] = jobs[x];
      jts[x] = (int32_t)ptotal;
      ptotal += (int64_t)jobs[x].tiles_r * ((jobs[x].kdim + 63) / 64);
      if (ptotal > 0x7fffffff) return HCBK_ERR_ARGS;
    }
    jts[njobs] = (int32_t)ptotal;
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
    gp.count = count;
    gp.total_tiles = (int)total;
    gp.tile_start_offset = ts_off;
    gp.pack_count = (int)njobs;
    gp.pack_tiles = (int)ptotal;
    gp.pack_offset = job_off;
    gp.pack_ts_offset = jts_off;
    gp.tile_desc_offset = td_off;
    gp.fallback.clear();
    gp.key = key;
  }

  int *err = device_error_flag(st);
  if (!err) return HCBK_ERR_NOMEM;
  char *tb = static_cast<char *>(gp.table);
  int rc = HCBK_OK;
  if (ptrs) { /* the batch's operands and C from its device pointer arrays */
    rc = timed_launch(st, stream, "pack.ptr_patch", [&] {
      return hcbk_grouped_split_patch(reinterpret_cast<hcbk_gpack_job *>(tb + gp.pack_offset),
                                      reinterpret_cast<hcbk_grouped_entry *>(tb), ptrs->a,
                                      ptrs->b, ptrs->c, ptrs->a_off, ptrs->b_off, ptrs->c_off,
                                      ptrs->sa, ptrs->sb, ptrs->sc, count, stream);
    });
    if (rc) return rc;
  }
  rc = timed_launch(st, stream, "pack.split_bf16.grouped", [&] {
    return hcbk_grouped_pack(reinterpret_cast<const hcbk_gpack_job *>(tb + gp.pack_offset),
                             reinterpret_cast<const int32_t *>(tb + gp.pack_ts_offset),
                             gp.pack_count, gp.pack_tiles, nplanes, stream);
  });
  if (rc) return rc;
  hcbk_grouped_args g;
  g.table = reinterpret_cast<const hcbk_grouped_entry *>(tb);
  g.tile_start = reinterpret_cast<const int32_t *>(tb + gp.tile_start_offset);
  g.count = gp.count;
  g.total_tiles = gp.total_tiles;
  g.alpha = alpha;
  g.beta = beta;
  g.device_maps = 0;
  g.tile_desc = reinterpret_cast<const int32_t *>(tb + gp.tile_desc_offset);
  g.uniform_tiles = 0;
  g.u_tiles_m = g.u_k = g.u_flags = 0;
  g.ctas_per_sm = 1;
  const char *path = terms == 6 ? "tc.s.grouped_split_bf16x6" : "tc.s.grouped_split_bf16x3";
  rc = timed_launch(st, stream, path,
                    [&] { return hcbk_sgemm_grouped_split_tc(&g, terms, err, stream); });
  if (rc) return rc;
  st->last_path = path;
  return HCBK_OK;
}

/* Grouped GEMM on the CUDA cores for S/D/C/Z in their own arithmetic: one
 * persistent launch over the device problem table (hcbk_gemm_simt_grouped),
 * problems ordered by decreasing work; the table is cached per handle for
 * a byte-identical follow-up problem array. */
int grouped_simt(HcblasB200State *st, void *stream, int dtype, hcblasOrder order, int count,
                 const hcblasGemmProblem *probs, double alpha_re, double alpha_im,
                 double beta_re, double beta_im) {
  const bool cplx = dtype == HCBK_C || dtype == HCBK_Z;
  if (alpha_re == 0.0 && alpha_im == 0.0) { /* C_i := beta*C_i, A and B not referenced */
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order, cplx);
      hcbk_gemm_args a;
      std::memset(&a, 0, sizeof(a));
      a.dtype = dtype;
      a.m = c.m;
      a.n = c.n;
      a.k = c.k;
      a.c = c.c;
      a.ldc = c.ldc;
      a.batch = 1;
      a.beta_re = beta_re;
      a.beta_im = beta_im;
      int rc = timed_launch(st, stream, "scale", [&] { return hcbk_scale_c(&a, stream); });
      if (rc) return rc;
    }
    st->last_path = "scale";
    return HCBK_OK;
  }
  int bm = 0, bn = 0;
  if (hcbk_simt_grouped_tile(dtype, &bm, &bn) != HCBK_OK) return HCBK_ERR_ARGS;
  HcblasGroupedPlan &gp = st->grouped_simt;
  int dev = 0;
  cudaGetDevice(&dev);
  std::vector<unsigned char> key(sizeof(hcblasGemmProblem) * (size_t)count + 3);
  std::memcpy(key.data(), probs, sizeof(hcblasGemmProblem) * (size_t)count);
  key[key.size() - 3] = static_cast<unsigned char>(order);
  key[key.size() - 2] = static_cast<unsigned char>(dev);
  key[key.size() - 1] = static_cast<unsigned char>(dtype);
  const bool reuse = gp.table && gp.table_device == dev && key == gp.key;
  if (!reuse) {
    if (!st->graph_cache.empty()) {
      cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
      clear_graph_cache(st);
    }
    gp.key.clear();
    std::vector<hcbk_simt_entry> ent((size_t)count);
    std::vector<int> order_idx((size_t)count);
    for (int i = 0; i < count; ++i) {
      const Canon c = canonical(probs[i], order, cplx);
      if (c.m > 0x7fffffff || c.n > 0x7fffffff || c.k > 0x7fffffff) return HCBK_ERR_ARGS;
      hcbk_simt_entry &e = ent[i];
      e.a = c.a;
      e.b = c.b;
      e.c = c.c;
      e.lda = c.lda;
      e.ldb = c.ldb;
      e.ldc = c.ldc;
      e.m = (int32_t)c.m;
      e.n = (int32_t)c.n;
      e.k = (int32_t)c.k;
      e.op_a = c.op_a;
      e.op_b = c.op_b;
      e.tiles_m = (int32_t)((c.m + bm - 1) / bm);
      order_idx[i] = i;
    }
    auto work = [&](int i) {
      const hcbk_simt_entry &e = ent[i];
      return (int64_t)e.tiles_m * ((e.n + bn - 1) / bn) * (int64_t)e.k;
    };
    std::stable_sort(order_idx.begin(), order_idx.end(),
                     [&](int x, int y) { return work(x) > work(y); });
    const size_t ent_bytes = sizeof(hcbk_simt_entry) * (size_t)count;
    const size_t ts_off = (ent_bytes + 255) & ~size_t(255);
    const size_t bytes = ts_off + sizeof(int32_t) * ((size_t)count + 1);
    if (!ensure_table(gp, bytes, stream) || !ensure_staging(gp, bytes)) return HCBK_ERR_NOMEM;
    unsigned char *stg = static_cast<unsigned char *>(gp.staging);
    auto *dst = reinterpret_cast<hcbk_simt_entry *>(stg);
    auto *ts = reinterpret_cast<int32_t *>(stg + ts_off);
    int64_t total = 0;
    for (int j = 0; j < count; ++j) {
      const hcbk_simt_entry &e = ent[order_idx[j]];
      dst[j] = e;
      ts[j] = (int32_t)total;
      total += (int64_t)e.tiles_m * ((e.n + bn - 1) / bn);
      if (total > 0x7fffffff) return HCBK_ERR_ARGS;
    }
    ts[count] = (int32_t)total;
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
    gp.count = count;
    gp.total_tiles = (int)total;
    gp.tile_start_offset = ts_off;
    gp.key = key;
  }
  hcbk_simt_grouped_args g;
  g.dtype = dtype;
  g.table = static_cast<const hcbk_simt_entry *>(gp.table);
  g.tile_start =
      reinterpret_cast<const int32_t *>(static_cast<char *>(gp.table) + gp.tile_start_offset);
  g.count = gp.count;
  g.total_tiles = gp.total_tiles;
  g.alpha_re = alpha_re;
  g.alpha_im = cplx ? alpha_im : 0.0;
  g.beta_re = beta_re;
  g.beta_im = cplx ? beta_im : 0.0;
  static const char *names[4] = {"simt.s.grouped", "simt.d.grouped", "simt.c.grouped",
                                 "simt.z.grouped"};
  st->last_path = names[dtype];
  return timed_launch(st, stream, names[dtype],
                      [&] { return hcbk_gemm_simt_grouped(&g, stream); });
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

extern "C" hcblasStatus_t hcblasSgemmGrouped(hcblasHandle_t handle, int count,
                                             const hcblasGemmProblem *problems,
                                             const float *alpha, const float *beta) {
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
  /* 3 products when the handle asks for the 3-term split, else 6 (error no
   * worse than plain FP32) */
  const HcblasB200State *st = handle->impl;
  const int terms = (st->math_mode == HCBLAS_MATH_SPLIT_BF16 && st->math_param == 3) ? 3 : 6;
  int rc = grouped_sgemm_split(handle->impl, handle->currentAcclView.stream, handle->Order, count,
                               problems, *alpha, *beta, terms);
  if (log_enabled())
    std::fprintf(stderr, "[hcblas] grouped sgemm count=%d path=%s rc=%d\n", count,
                 handle->impl->last_path, rc);
  return rc == HCBK_OK ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_EXECUTION_FAILED;
}

namespace {

/* the status rules of hcblasHgemmGrouped, then the SIMT grouped kernel */
hcblasStatus_t simt_grouped_call(hcblasHandle_t handle, int dtype, int count,
                                 const hcblasGemmProblem *problems, const void *alpha,
                                 const void *beta) {
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
  double ar = 0, ai = 0, br = 0, bi = 0;
  switch (dtype) {
    case HCBK_D:
      ar = *static_cast<const double *>(alpha);
      br = *static_cast<const double *>(beta);
      break;
    case HCBK_C: {
      const hcComplex *a = static_cast<const hcComplex *>(alpha);
      const hcComplex *b = static_cast<const hcComplex *>(beta);
      ar = a->x, ai = a->y, br = b->x, bi = b->y;
      break;
    }
    default: {
      const hcDoubleComplex *a = static_cast<const hcDoubleComplex *>(alpha);
      const hcDoubleComplex *b = static_cast<const hcDoubleComplex *>(beta);
      ar = a->x, ai = a->y, br = b->x, bi = b->y;
      break;
    }
  }
  int rc = grouped_simt(handle->impl, handle->currentAcclView.stream, dtype, handle->Order, count,
                        problems, ar, ai, br, bi);
  if (log_enabled())
    std::fprintf(stderr, "[hcblas] grouped dtype=%d count=%d path=%s rc=%d\n", dtype, count,
                 handle->impl->last_path, rc);
  return rc == HCBK_OK ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_EXECUTION_FAILED;
}

}  // namespace

extern "C" hcblasStatus_t hcblasDgemmGrouped(hcblasHandle_t handle, int count,
                                             const hcblasGemmProblem *problems,
                                             const double *alpha, const double *beta) {
  return simt_grouped_call(handle, HCBK_D, count, problems, alpha, beta);
}

extern "C" hcblasStatus_t hcblasCgemmGrouped(hcblasHandle_t handle, int count,
                                             const hcblasGemmProblem *problems,
                                             const hcComplex *alpha, const hcComplex *beta) {
  return simt_grouped_call(handle, HCBK_C, count, problems, alpha, beta);
}

extern "C" hcblasStatus_t hcblasZgemmGrouped(hcblasHandle_t handle, int count,
                                             const hcblasGemmProblem *problems,
                                             const hcDoubleComplex *alpha,
                                             const hcDoubleComplex *beta) {
  return simt_grouped_call(handle, HCBK_Z, count, problems, alpha, beta);
}
