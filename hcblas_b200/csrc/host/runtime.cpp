/*
 * runtime.cpp -- handle lifecycle, accelerator views (streams), device memory
 * and host<->device copies: the parts of hcBLAS's C API around GEMM
 * (lib/src/hcblas.cpp:39-312) and of its HCC runtime usage (hc::am_alloc,
 * accelerator_view::copy) re-expressed on the CUDA runtime.
 */
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <string>

#include "../../../include/hcblas.h"
#include "../../../include/hcblaslib.h"
#include "../kernels/hcbk.h"
#include "state.h"

namespace hcblas_b200 {

DeviceGuard::DeviceGuard(int dev) {
  if (cudaGetDevice(&prev_) != cudaSuccess) {
    prev_ = -1;
    ok_ = false;
    return;
  }
  if (dev == prev_) {
    ok_ = true;
    return;
  }
  ok_ = cudaSetDevice(dev) == cudaSuccess;
}

DeviceGuard::~DeviceGuard() {
  int cur = -1;
  if (prev_ >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev_) cudaSetDevice(prev_);
}

/* Order `stream` after the last work that used the workspace on another
 * stream (class-API calls may name a different accelerator view per call). */
static void order_after_last_use(HcblasB200State *st, cudaStream_t stream) {
  cudaStream_t last = static_cast<cudaStream_t>(st->workspace_stream);
  if (last == stream) return;
  if (!st->workspace_event &&
      cudaEventCreateWithFlags(reinterpret_cast<cudaEvent_t *>(&st->workspace_event),
                               cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    st->workspace_event = nullptr;
  }
  cudaEvent_t ev = static_cast<cudaEvent_t>(st->workspace_event);
  if (!ev || cudaEventRecord(ev, last) != cudaSuccess ||
      cudaStreamWaitEvent(stream, ev, 0) != cudaSuccess) {
    /* the earlier stream is gone (destroyed by the caller): its work can
     * only be waited for as a whole */
    cudaGetLastError();
    cudaDeviceSynchronize();
  }
}

void *ensure_workspace(HcblasB200State *st, size_t bytes, void *stream_v) {
  cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
  int dev = 0;
  cudaGetDevice(&dev);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) {
    cudaGetLastError();
    cap = cudaStreamCaptureStatusNone;
  }
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (st->workspace && st->workspace_device == dev) {
    if (!capturing) order_after_last_use(st, stream);
    if (st->workspace_bytes >= bytes) {
      st->workspace_stream = stream;
      return st->workspace;
    }
  }
  /* growing: not while the stream is being captured (an allocation would
   * belong to the graph), and never beyond the handle's limit */
  if (capturing || (st->workspace_limit && bytes > st->workspace_limit)) {
    if (log_enabled())
      std::fprintf(stderr, "[hcblas] workspace of %zu bytes refused (%s)\n", bytes,
                   capturing ? "stream capture in progress" : "over the handle's limit");
    return nullptr;
  }
  if (st->workspace) {
    /* stream-ordered release: queued kernels that still read the old
     * workspace finish before the memory is reused; no device-wide wait */
    clear_graph_cache(st);
    if (st->workspace_device == dev) {
      cudaFreeAsync(st->workspace, stream);
    } else {
      DeviceGuard g(st->workspace_device);
      cudaFreeAsync(st->workspace, static_cast<cudaStream_t>(st->workspace_stream));
    }
    cudaGetLastError();
    st->workspace = nullptr;
    st->workspace_bytes = 0;
  }
  size_t want = bytes < (size_t)(64u << 20) ? (size_t)(64u << 20) : bytes;
  if (st->workspace_limit && want > st->workspace_limit) want = bytes;
  void *p = nullptr;
  if (cudaMallocAsync(&p, want, stream) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  st->workspace = p;
  st->workspace_bytes = want;
  st->workspace_device = dev;
  st->workspace_stream = stream;
  return p;
}

void clear_graph_cache(HcblasB200State *st) {
  for (auto &e : st->graph_cache)
    if (e.exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(e.exec));
  st->graph_cache.clear();
  ++st->workspace_epoch;
}

int *device_error_flag(HcblasB200State *st) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (st->dev_err && st->dev_err_device == dev) return st->dev_err;
  if (st->dev_err) {
    clear_graph_cache(st);
    DeviceGuard g(st->dev_err_device);
    cudaFree(st->dev_err);
    st->dev_err = nullptr;
  }
  /* the device error block: int 0 the code, ints 2-3 the wait limit (ns) */
  void *p = nullptr;
  if (cudaMalloc(&p, 4 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  int block[4] = {0, 0, 0, 0};
  std::memcpy(block + 2, &st->wait_limit_ns, sizeof(st->wait_limit_ns));
  if (cudaMemcpy(p, block, sizeof(block), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(p);
    return nullptr;
  }
  st->dev_err = static_cast<int *>(p);
  st->dev_err_device = dev;
  return st->dev_err;
}

static std::atomic<long long> g_launches{0};

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void *prof_event(HcblasB200State *st) {
  if (!st->event_pool.empty()) {
    void *e = st->event_pool.back();
    st->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void prof_record(void *ev, void *stream) {
  cudaEventRecord(static_cast<cudaEvent_t>(ev), static_cast<cudaStream_t>(stream));
}

void *aux_fork(HcblasB200State *st, void *stream) {
  if (!st->use_aux) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (st->aux_stream && st->aux_device != dev) return nullptr; /* created for another device */
  if (!st->aux_stream) {
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&f, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&j, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      if (s) cudaStreamDestroy(s);
      if (f) cudaEventDestroy(f);
      return nullptr;
    }
    st->aux_stream = s;
    st->aux_fork = f;
    st->aux_join = j;
    st->aux_device = dev;
  }
  if (cudaEventRecord(static_cast<cudaEvent_t>(st->aux_fork), static_cast<cudaStream_t>(stream)) !=
          cudaSuccess ||
      cudaStreamWaitEvent(static_cast<cudaStream_t>(st->aux_stream),
                          static_cast<cudaEvent_t>(st->aux_fork), 0) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return st->aux_stream;
}

int aux_join(HcblasB200State *st, void *stream) {
  if (cudaEventRecord(static_cast<cudaEvent_t>(st->aux_join),
                      static_cast<cudaStream_t>(st->aux_stream)) != cudaSuccess ||
      cudaStreamWaitEvent(static_cast<cudaStream_t>(stream), static_cast<cudaEvent_t>(st->aux_join),
                          0) != cudaSuccess) {
    cudaGetLastError();
    return HCBK_ERR_LAUNCH;
  }
  return HCBK_OK;
}

bool log_enabled() {
  static int v = -1;
  if (v < 0) {
    const char *e = std::getenv("HCBLAS_LOG");
    v = (e && e[0] == '1') ? 1 : 0;
  }
  return v == 1;
}

}  // namespace hcblas_b200

using hcblas_b200::DeviceGuard;

/* ---------------------------------------------------- hc_compat services -- */

extern "C" void *hcblas_am_alloc(size_t bytes, int device_id, unsigned flags) {
  (void)flags;
  DeviceGuard g(device_id);
  if (!g.ok()) return nullptr;
  void *p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

extern "C" int hcblas_am_free(void *ptr) {
  if (!ptr) return 0;
  return cudaFree(ptr) == cudaSuccess ? 0 : -1;
}

extern "C" int hcblas_am_copy(hcblas_accl_view_t view, const void *src, void *dst,
                              size_t bytes) {
  DeviceGuard g(view.device_id);
  cudaStream_t s = static_cast<cudaStream_t>(view.stream);
  if (cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, s) != cudaSuccess) return -1;
  return cudaStreamSynchronize(s) == cudaSuccess ? 0 : -1;
}

extern "C" int hcblas_view_wait(hcblas_accl_view_t view) {
  DeviceGuard g(view.device_id);
  return cudaStreamSynchronize(static_cast<cudaStream_t>(view.stream)) == cudaSuccess ? 0 : -1;
}

extern "C" int hcblas_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" int hcblas_current_device(void) {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return d;
}

/* ------------------------------------------------------- Hcblaslibrary -- */

Hcblaslibrary::Hcblaslibrary(hc::accelerator_view *av)
    : currentAccl(av ? av->device_id : hcblas_current_device()),
      currentAcclView(av ? *av : hc::accelerator_view()) {
  const int n = hcblas_device_count();
  const int dev = currentAccl.get_device_id();
  initialized = (dev >= 0 && dev < n);
  currentStream = currentAcclView.stream;
  Order = ColMajor;
  impl = new (std::nothrow) HcblasB200State();
  if (!impl) initialized = false;
}

Hcblaslibrary::~Hcblaslibrary() {
  initialized = false;
  if (impl) {
    if (impl->workspace) {
      DeviceGuard g(impl->workspace_device);
      cudaStream_t ws = static_cast<cudaStream_t>(impl->workspace_stream);
      if (cudaFreeAsync(impl->workspace, ws) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeAsync(impl->workspace, nullptr);
      }
      if (cudaStreamSynchronize(ws) != cudaSuccess) cudaGetLastError();
    }
    if (impl->workspace_event) cudaEventDestroy(static_cast<cudaEvent_t>(impl->workspace_event));
    if (impl->aux_stream) {
      DeviceGuard g(impl->aux_device);
      cudaStreamSynchronize(static_cast<cudaStream_t>(impl->aux_stream));
      cudaStreamDestroy(static_cast<cudaStream_t>(impl->aux_stream));
      cudaEventDestroy(static_cast<cudaEvent_t>(impl->aux_fork));
      cudaEventDestroy(static_cast<cudaEvent_t>(impl->aux_join));
    }
    for (auto &r : impl->prof) {
      cudaEventDestroy(static_cast<cudaEvent_t>(r.ev0));
      cudaEventDestroy(static_cast<cudaEvent_t>(r.ev1));
    }
    for (void *e : impl->event_pool) cudaEventDestroy(static_cast<cudaEvent_t>(e));
    if (impl->dev_err) {
      DeviceGuard g(impl->dev_err_device);
      cudaFree(impl->dev_err);
    }
    cudaStreamSynchronize(static_cast<cudaStream_t>(currentAcclView.stream));
    hcblas_b200::clear_graph_cache(impl);
    for (HcblasGroupedPlan *pp :
         {&impl->grouped, &impl->grouped_split, &impl->grouped_simt, &impl->grouped_ptr}) {
      HcblasGroupedPlan &gp = *pp;
      if (gp.upload_done) {
        cudaEventSynchronize(static_cast<cudaEvent_t>(gp.upload_done));
        cudaEventDestroy(static_cast<cudaEvent_t>(gp.upload_done));
      }
      if (gp.table || gp.planes) {
        DeviceGuard g(gp.table_device);
        cudaStreamSynchronize(static_cast<cudaStream_t>(currentAcclView.stream));
        if (gp.table) cudaFree(gp.table);
        if (gp.planes) cudaFree(gp.planes);
      }
      if (gp.staging) cudaFreeHost(gp.staging);
    }
    delete impl;
    impl = nullptr;
  }
}

/* ------------------------------------------------------------- C API -- */

extern "C" hcblasStatus_t hcblasCreate(hcblasHandle_t *handle, hcblas_accl_view_t *av) {
  if (handle == nullptr) return HCBLAS_STATUS_INVALID_VALUE;
  hc::accelerator_view view;
  if (av) {
    view.device_id = av->device_id;
    view.stream = av->stream;
  }
  Hcblaslibrary *h = new (std::nothrow) Hcblaslibrary(&view);
  if (h == nullptr) return HCBLAS_STATUS_ALLOC_FAILED;
  if (!h->initialized) {
    delete h;
    *handle = nullptr;
    return HCBLAS_STATUS_NOT_INITIALIZED;
  }
  *handle = h;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasDestroy(hcblasHandle_t *handle) {
  if (handle == nullptr || *handle == nullptr || !(*handle)->initialized)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  delete *handle;
  *handle = nullptr;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasSetAcclView(hcblasHandle_t handle, hcblas_accl_view_t *accl_view,
                                            void *stream) {
  if (handle == nullptr || !handle->initialized) return HCBLAS_STATUS_NOT_INITIALIZED;
  if (accl_view) {
    handle->currentAcclView.device_id = accl_view->device_id;
    handle->currentAcclView.stream = accl_view->stream;
    handle->currentAccl = hc::accelerator(accl_view->device_id);
  }
  if (stream) handle->currentAcclView.stream = stream;
  handle->currentStream = handle->currentAcclView.stream;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasGetAcclView(hcblasHandle_t handle, hcblas_accl_view_t **accl_view,
                                            void **stream) {
  if (handle == nullptr) return HCBLAS_STATUS_NOT_INITIALIZED;
  if (accl_view) *accl_view = &handle->currentAcclView;
  if (stream) *stream = handle->currentStream;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasSetStream(hcblasHandle_t handle, void *stream) {
  if (handle == nullptr || !handle->initialized) return HCBLAS_STATUS_NOT_INITIALIZED;
  handle->currentAcclView.stream = stream;
  handle->currentStream = stream;
  return HCBLAS_STATUS_SUCCESS;
}

namespace {

/* 2-D copy of `cols` columns of `rows` elements, then wait on the stream. */
/* one pitched copy on `stream` (the handle's stream when null); waits for it
 * unless `async` */
hcblasStatus_t copy2d(hcblasHandle_t h, const void *src, size_t spitch, void *dst,
                      size_t dpitch, size_t width, size_t height, void *stream = nullptr,
                      bool async = false) {
  DeviceGuard g(h->currentAcclView.device_id);
  cudaStream_t s = static_cast<cudaStream_t>(stream ? stream : h->currentAcclView.stream);
  cudaError_t e;
  if (spitch == width && dpitch == width)
    e = cudaMemcpyAsync(dst, src, width * height, cudaMemcpyDefault, s);
  else
    e = cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDefault, s);
  if (e == cudaSuccess && !async) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return HCBLAS_STATUS_MAPPING_ERROR;
  }
  return HCBLAS_STATUS_SUCCESS;
}

hcblasStatus_t copy_matrix(hcblasHandle_t handle, int rows, int cols, int elemSize,
                           const void *A, int lda, void *B, int ldb, void *stream = nullptr,
                           bool async = false) {
  if (handle == nullptr || !handle->initialized) return HCBLAS_STATUS_NOT_INITIALIZED;
  if (rows < 0 || cols < 0 || lda <= 0 || ldb <= 0 || elemSize <= 0)
    return HCBLAS_STATUS_INVALID_VALUE;
  if (rows == 0 || cols == 0) return HCBLAS_STATUS_SUCCESS;
  if (A == nullptr || B == nullptr) return HCBLAS_STATUS_MAPPING_ERROR;
  const size_t es = (size_t)elemSize;
  if (lda >= rows && ldb >= rows)
    return copy2d(handle, A, (size_t)lda * es, B, (size_t)ldb * es, (size_t)rows * es,
                  (size_t)cols, stream, async);
  /* the reference's behaviour: rows*cols contiguous elements */
  const size_t w = (size_t)rows * (size_t)cols * es;
  return copy2d(handle, A, w, B, w, w, 1, stream, async);
}

hcblasStatus_t copy_vector(hcblasHandle_t handle, int n, int elemSize, const void *x, int incx,
                           void *y, int incy) {
  if (handle == nullptr || !handle->initialized) return HCBLAS_STATUS_NOT_INITIALIZED;
  if (n < 0 || elemSize <= 0 || incx <= 0 || incy <= 0) return HCBLAS_STATUS_INVALID_VALUE;
  if (n == 0) return HCBLAS_STATUS_SUCCESS;
  if (x == nullptr || y == nullptr) return HCBLAS_STATUS_MAPPING_ERROR;
  const size_t es = (size_t)elemSize;
  return copy2d(handle, x, (size_t)incx * es, y, (size_t)incy * es, es, (size_t)n);
}

}  // namespace

extern "C" hcblasStatus_t hcblasSetVector(hcblasHandle_t handle, int n, int elemSize,
                                          const void *x, int incx, void *y, int incy) {
  return copy_vector(handle, n, elemSize, x, incx, y, incy);
}

extern "C" hcblasStatus_t hcblasGetVector(hcblasHandle_t handle, int n, int elemSize,
                                          const void *x, int incx, void *y, int incy) {
  return copy_vector(handle, n, elemSize, x, incx, y, incy);
}

extern "C" hcblasStatus_t hcblasSetMatrix(hcblasHandle_t handle, int rows, int cols, int elemSize,
                                          const void *A, int lda, void *B, int ldb) {
  return copy_matrix(handle, rows, cols, elemSize, A, lda, B, ldb);
}

extern "C" hcblasStatus_t hcblasGetMatrix(hcblasHandle_t handle, int rows, int cols, int elemSize,
                                          const void *A, int lda, void *B, int ldb) {
  return copy_matrix(handle, rows, cols, elemSize, A, lda, B, ldb);
}

extern "C" hcblasStatus_t hcblasSetMatrixAsync(hcblasHandle_t handle, int rows, int cols,
                                               int elemSize, const void *A, int lda, void *B,
                                               int ldb, void *stream) {
  return copy_matrix(handle, rows, cols, elemSize, A, lda, B, ldb, stream, true);
}

extern "C" hcblasStatus_t hcblasGetMatrixAsync(hcblasHandle_t handle, int rows, int cols,
                                               int elemSize, const void *A, int lda, void *B,
                                               int ldb, void *stream) {
  return copy_matrix(handle, rows, cols, elemSize, A, lda, B, ldb, stream, true);
}

extern "C" hcblasStatus_t hcblasSetMathMode(hcblasHandle_t handle, int mode, int param) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (mode < HCBLAS_MATH_NATIVE || mode > HCBLAS_MATH_OZAKI_CRT)
    return HCBLAS_STATUS_INVALID_VALUE;
  if (mode == HCBLAS_MATH_OZAKI_CRT && (param < 0 || param > HCBK_CRT_MAX_MODULI || (param > 0 && param < 8)))
    return HCBLAS_STATUS_INVALID_VALUE;
  if (mode == HCBLAS_MATH_SPLIT_BF16 && !(param == 0 || param == 3 || param == 6))
    return HCBLAS_STATUS_INVALID_VALUE;
  if (mode == HCBLAS_MATH_OZAKI_INT8 && (param < 0 || param > 8 || (param > 0 && param < 3)))
    return HCBLAS_STATUS_INVALID_VALUE;
  if (mode == HCBLAS_MATH_OZAKI_F16 && (param < 0 || param > 7 || (param > 0 && param < 3)))
    return HCBLAS_STATUS_INVALID_VALUE;
  handle->impl->math_mode = mode;
  handle->impl->math_param = param;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasGetMathMode(hcblasHandle_t handle, int *mode, int *param) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (mode) *mode = handle->impl->math_mode;
  if (param) *param = handle->impl->math_param;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasSetTuningParam(hcblasHandle_t handle, const char *name,
                                               int value) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (name == nullptr) return HCBLAS_STATUS_INVALID_VALUE;
  if (std::strcmp(name, "split_promote_kb") == 0) {
    if (value != 1 && value != 4) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->split_promote_kb = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "autotune") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->autotune = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "graphs") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->graphs = value;
    if (!value) hcblas_b200::clear_graph_cache(handle->impl);
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "tc_pair") == 0) {
    if (value < 0 || value > 2) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->tc_pair = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "crt_i8") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->crt_i8 = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "grouped_ctas") == 0) {
    if (value != 1 && value != 2) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->grouped_ctas = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "grouped_c_tma") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->grouped_c_tma = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "aux_stream") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->use_aux = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "dgemm_dmma") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->dgemm_dmma = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "workspace_mb") == 0) {
    if (value < 0) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->workspace_limit = (size_t)value << 20;
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "wait_timeout_us") == 0) {
    if (value < 0) return HCBLAS_STATUS_INVALID_VALUE;
    HcblasB200State *st = handle->impl;
    st->wait_limit_ns = (unsigned long long)value * 1000ull;
    if (st->dev_err) {
      /* ordered after the handle's queued work, like a kernel argument */
      DeviceGuard g(st->dev_err_device);
      cudaStream_t cs = static_cast<cudaStream_t>(handle->currentAcclView.stream);
      if (cudaStreamSynchronize(cs) != cudaSuccess ||
          cudaMemcpy(st->dev_err + 2, &st->wait_limit_ns, sizeof(st->wait_limit_ns),
                     cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        return HCBLAS_STATUS_EXECUTION_FAILED;
      }
    }
    return HCBLAS_STATUS_SUCCESS;
  }
  if (std::strcmp(name, "inject_timeout") == 0) {
    if (value != 0 && value != 1) return HCBLAS_STATUS_INVALID_VALUE;
    handle->impl->inject_timeout = value;
    return HCBLAS_STATUS_SUCCESS;
  }
  return HCBLAS_STATUS_INVALID_VALUE;
}

extern "C" const char *hcblasGetLastPath(hcblasHandle_t handle) {
  if (handle == nullptr || !handle->impl) return "none";
  return handle->impl->last_path;
}

extern "C" const char *hcblasGetVersionString(void) {
  return "hcblas-b200 " HCBLAS_B200_VERSION " (sm_100a)";
}

extern "C" long long hcblasGetKernelLaunchCount(void) { return hcblas_b200::launch_count(); }

extern "C" int hcblasGetDeviceError(hcblasHandle_t handle) {
  if (handle == nullptr || !handle->initialized || !handle->impl) return -1;
  HcblasB200State *st = handle->impl;
  if (!st->dev_err) return 0;
  DeviceGuard g(st->dev_err_device);
  int v = 0;
  cudaStreamSynchronize(static_cast<cudaStream_t>(handle->currentAcclView.stream));
  if (cudaMemcpy(&v, st->dev_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return -2;
  }
  if (v) cudaMemset(st->dev_err, 0, sizeof(int));
  return v;
}

extern "C" hcblasStatus_t hcblasSetProfiling(hcblasHandle_t handle, int on) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  HcblasB200State *st = handle->impl;
  st->profiling = on != 0;
  for (auto &r : st->prof) {
    st->event_pool.push_back(r.ev0);
    st->event_pool.push_back(r.ev1);
  }
  st->prof.clear();
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" int hcblasGetProfile(hcblasHandle_t handle, char *buf, int cap) {
  if (handle == nullptr || !handle->initialized || !handle->impl) return -1;
  HcblasB200State *st = handle->impl;
  DeviceGuard g(handle->currentAcclView.device_id);
  std::map<std::string, std::pair<long long, double>> agg;
  for (auto &r : st->prof) {
    cudaEventSynchronize(static_cast<cudaEvent_t>(r.ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, static_cast<cudaEvent_t>(r.ev0), static_cast<cudaEvent_t>(r.ev1));
    auto &a = agg[r.name];
    a.first += 1;
    a.second += ms;
  }
  std::string out;
  char line[256];
  for (auto &kv : agg) {
    std::snprintf(line, sizeof(line), "%s %lld %.6f\n", kv.first.c_str(), kv.second.first,
                  kv.second.second);
    out += line;
  }
  if (buf && cap > 0) {
    std::strncpy(buf, out.c_str(), (size_t)cap - 1);
    buf[cap - 1] = '\0';
  }
  return (int)out.size();
}
