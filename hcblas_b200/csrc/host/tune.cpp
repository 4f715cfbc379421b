/*
 * tune.cpp -- the autotuner (tuning knob "autotune"): per size bucket, time
 * every candidate tile configuration of a kernel family once on the call
 * that first lands in the bucket, keep the fastest.
 *
 * Bucket key: the library version, the driver version, the device (name and
 * ordinal), family, dtype, transposes, ceil(log2) of M, N and K; a decision
 * made by another library or driver version is never reused.  Cache lines
 * that do not parse, or whose choice is out of range for the family, are
 * ignored and the bucket is tuned again.  The cache is process-wide; when the
 * environment variable HCBLAS_AUTOTUNE_CACHE names a file, the cache is read
 * from it on first use and every new decision is appended to it, so later
 * processes start tuned.  Candidates run through the kernels' own C entry
 * points (not counted, not profiled) bracketed by CUDA events on the call's
 * stream; nothing is tuned while the stream is being captured into a graph.
 * Candidates write either outputs that the final run overwrites completely
 * (beta == 0, workspace planes) or, for beta != 0, a scratch copy of C's
 * shape (TuneTarget), so tuning never changes a result.
 */
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <mutex>
#include <string>
#include <unordered_map>

#include "dispatch.h"

namespace hcblas_b200 {
namespace {

std::mutex g_tune_mutex;
std::unordered_map<std::string, int> g_tune;
bool g_tune_loaded = false;

const char *cache_path() {
  const char *p = std::getenv("HCBLAS_AUTOTUNE_CACHE");
  return (p && p[0]) ? p : nullptr;
}

void load_locked() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  const char *path = cache_path();
  if (!path) return;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    /* "<key> <choice>"; malformed lines are ignored */
    const size_t sp = line.rfind(' ');
    if (sp == std::string::npos || sp == 0) continue;
    char *end = nullptr;
    const long v = std::strtol(line.c_str() + sp + 1, &end, 10);
    if (end == line.c_str() + sp + 1 || v < 0 || v > 64) continue;
    g_tune[line.substr(0, sp)] = (int)v;
  }
}

void store_locked(const std::string &key, int choice) {
  g_tune[key] = choice;
  const char *path = cache_path();
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  if (f) f << key << ' ' << choice << '\n';
}

int ilog2_ceil(int64_t v) {
  int r = 0;
  while (((int64_t)1 << r) < v && r < 62) ++r;
  return r;
}

}  // namespace

std::string tune_key(const char *family, const hcbk_gemm_args *a) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  std::memset(&prop, 0, sizeof(prop));
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) cudaGetLastError();
  for (char *c = prop.name; *c; ++c)
    if (*c == ' ') *c = '_';
  int drv = 0;
  if (cudaDriverGetVersion(&drv) != cudaSuccess) cudaGetLastError();
  char buf[320];
  std::snprintf(buf, sizeof(buf), "v2|%s|drv%d|%s|%d|%s|dt%d|op%d%d|m%d|n%d|k%d|b%d",
                HCBLAS_B200_VERSION, drv, prop.name, dev, family, a->dtype, a->op_a, a->op_b,
                ilog2_ceil(a->m), ilog2_ceil(a->n), ilog2_ceil(a->k), a->batch > 1 ? 1 : 0);
  return buf;
}

std::string tune_key_shape(const char *family, const char *shape) {
  hcbk_gemm_args none;
  std::memset(&none, 0, sizeof(none));
  std::string k = tune_key(family, &none);
  const size_t cut = k.find("|dt");
  return (cut == std::string::npos ? k : k.substr(0, cut)) + "|" + shape;
}

namespace {
size_t elem_bytes(int dtype) {
  switch (dtype) {
    case HCBK_S: return 4;
    case HCBK_D: return 8;
    case HCBK_C: return 8;
    case HCBK_Z: return 16;
    default: return 2;
  }
}
}  // namespace

TuneTarget::TuneTarget(const hcbk_gemm_args *a, void *stream) : t_(*a), a_(a), stream_(stream) {
  usable_ = a->batch == 1 && !a->a_array && a->m > 0 && a->n > 0 && a->ldc >= a->m;
}

const hcbk_gemm_args *TuneTarget::args() {
  if (!usable_ || failed_) return nullptr;
  if (a_->beta_re == 0.0 && a_->beta_im == 0.0) return a_;
  if (!scratch_) {
    const size_t esz = elem_bytes(a_->dtype);
    const int64_t phase = a_->c_off % (int64_t)(256 / esz); /* same 256-byte alignment phase */
    const size_t bytes = ((size_t)a_->ldc * (size_t)(a_->n - 1) + (size_t)a_->m + phase) * esz;
    if (cudaMallocAsync(&scratch_, bytes, static_cast<cudaStream_t>(stream_)) != cudaSuccess) {
      cudaGetLastError();
      scratch_ = nullptr;
      failed_ = true;
      return nullptr;
    }
    /* finite contents: beta * C reads them */
    cudaMemsetAsync(scratch_, 0, bytes, static_cast<cudaStream_t>(stream_));
    t_.c = scratch_;
    t_.c_off = phase;
  }
  return &t_;
}

TuneTarget::~TuneTarget() {
  if (scratch_) cudaFreeAsync(scratch_, static_cast<cudaStream_t>(stream_));
}

int tune_choice(HcblasB200State *st, void *stream, const std::string &key, int ncand,
                const std::function<int(int)> &run, int fallback) {
  if (!st->autotune) return fallback;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    load_locked();
    auto it = g_tune.find(key);
    if (it != g_tune.end() && it->second < ncand) return it->second;
  }
  cudaStream_t cs = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(cs, &cap) != cudaSuccess) {
    cudaGetLastError();
    return fallback;
  }
  if (cap != cudaStreamCaptureStatusNone) return fallback;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    cudaGetLastError();
    if (e0) cudaEventDestroy(e0);
    return fallback;
  }
  int best = fallback;
  float best_ms = 1e30f;
  bool timed_any = false;
  for (int i = 0; i < ncand; ++i) {
    if (run(i) != HCBK_OK) { /* candidate not applicable to this call */
      cudaGetLastError();
      continue;
    }
    cudaEventRecord(e0, cs);
    bool ok = true;
    for (int r = 0; r < 2 && ok; ++r) ok = run(i) == HCBK_OK;
    cudaEventRecord(e1, cs);
    float ms = 0.f;
    if (!ok || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    timed_any = true;
    if (ms < best_ms) {
      best_ms = ms;
      best = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!timed_any) return fallback; /* nothing ran: decide again on a later call */
  if (log_enabled())
    std::fprintf(stderr, "[hcblas] autotune %s -> %d (%.4f ms)\n", key.c_str(), best, best_ms);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  store_locked(key, best);
  return best;
}

}  // namespace hcblas_b200
