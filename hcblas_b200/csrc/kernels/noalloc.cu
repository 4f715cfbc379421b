/*
 * noalloc.cu -- split-BF16 SGEMM for callers that must not allocate device
 * memory.
 *
 * The split-BF16 path (hcblasSgemm with HCBLAS_MATH_SPLIT_BF16) needs scratch
 * memory for the bf16 planes of both operands; the handle-based entry point
 * takes it from a workspace it grows with cudaMalloc.  Some callers cannot
 * let a library call cudaMalloc: applications with their own pool allocator
 * that own every device byte and forbid hidden allocations, plug-ins hosted
 * inside another framework that accounts for all device memory itself, and
 * real-time or inference services that allocate everything once at start-up
 * so that no call can fail later for want of memory or stall on the
 * allocator's implicit synchronisation.
 *
 * hcblasSgemmSplitBF16NoAlloc serves them: its scratch is one file-scope
 * static __device__ array of HCBLAS_NOALLOC_SCRATCH_BYTES (64 MiB), created
 * with the module on every GPU that loads the library and held until the
 * process exits.  The entry point calls no cudaMalloc, cudaFree or other
 * allocating routine; the caller passes the inputs and outputs.  Calls whose
 * planes do not fit are rejected with HCBLAS_STATUS_INVALID_VALUE.
 *
 * The host code never dereferences the array's name (in host code it only
 * stands in for the symbol): the first call in each CUDA context of a
 * device, with that device current, asks the runtime for the array's device
 * address with cudaGetSymbolAddress and caches it together with the context
 * it belongs to; a call from another context (for example after
 * cudaDeviceReset) looks the address up again.  That first call should come
 * before any stream capture begins.
 *
 * Every call on a device shares the one array, and the array keeps the last
 * call's contents.  The pack kernel rewrites every plane element the GEMM
 * reads, and the pipeline-timeout flag (the only state that must start at
 * zero) is cleared on the caller's stream at the start of each call;
 * hcblasSgemmSplitBF16NoAllocStatus reads it back after the call.  Calls
 * that overlap on the GPU -- on different streams, or from several host
 * threads -- race on the array and must be serialised by the caller.
 */
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../../include/hcblas.h"
#include "hcbk.h"

namespace {

constexpr size_t kScratchBytes = HCBLAS_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

/* the scratch and the device error block of the tensor-core kernels
 * (int 0: the pipeline-timeout code; ints 2-3: the wait limit, 0 = the
 * kernels' default); device addresses come from cudaGetSymbolAddress, never
 * from taking these names' addresses on the host */
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];
static __device__ __align__(256) int g_timeout_flag[4];

struct DeviceScratch {
  bool ready;
  CUcontext ctx; /* the context the cached addresses belong to */
  unsigned char *scratch;
  int *flag;
};

std::mutex g_setup_mutex;
DeviceScratch g_dev[kMaxDevices];

/* the current CUDA context, through the driver entry point the runtime
 * exposes (nullptr if it cannot be found) */
CUcontext current_context() {
  typedef CUresult (*PFN_ctx_get)(CUcontext *);
  static PFN_ctx_get fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_ctx_get>(ptr);
    else
      cudaGetLastError();
    looked = true;
  }
  CUcontext c = nullptr;
  if (fn == nullptr || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

/* once per device and context, with that device current */
bool device_scratch(int dev, DeviceScratch *out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  const CUcontext ctx = current_context();
  DeviceScratch &d = g_dev[dev];
  if (!d.ready || d.ctx != ctx) {
    void *s = nullptr, *f = nullptr;
    d.ready = false;
    if (cudaGetSymbolAddress(&s, g_scratch) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (cudaGetSymbolAddress(&f, g_timeout_flag) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    d.scratch = static_cast<unsigned char *>(s);
    d.flag = static_cast<int *>(f);
    d.ctx = current_context(); /* the symbol lookup may have created the primary context */
    d.ready = true;
  }
  *out = d;
  return true;
}

size_t round_1k(size_t v) { return (v + 1023) & ~size_t(1023); }

}  // namespace

extern "C" hcblasStatus_t hcblasSgemmSplitBF16NoAlloc(void *stream, hcblasOperation_t transa,
                                                      hcblasOperation_t transb, int m, int n,
                                                      int k, const float *alpha, const float *A,
                                                      int lda, const float *B, int ldb,
                                                      const float *beta, float *C, int ldc,
                                                      int terms) {
  if (m < 0 || n < 0 || k < 0 || alpha == nullptr || beta == nullptr ||
      (terms != 3 && terms != 6) || transa > HCBLAS_OP_C || transb > HCBLAS_OP_C)
    return HCBLAS_STATUS_INVALID_VALUE;
  /* the library's quick-return rule: empty problems and missing matrices
   * fail, as in hcblasSgemm */
  if (m == 0 || n == 0 || k == 0 || A == nullptr || B == nullptr || C == nullptr)
    return HCBLAS_STATUS_EXECUTION_FAILED;

  const int nplanes = terms == 6 ? 3 : 2;
  const int64_t kp = ((int64_t)k + 7) & ~int64_t(7); /* 16-byte plane row pitch */
  /* m, n, kp < 2^31: each plane's size fits size_t; reject either operand
   * alone before the sum and the plane count are applied, so that nothing
   * below can wrap */
  const size_t a_bytes = round_1k((size_t)m * kp * 2), b_bytes = round_1k((size_t)n * kp * 2);
  if (a_bytes > kScratchBytes || b_bytes > kScratchBytes ||
      (a_bytes + b_bytes) * nplanes > kScratchBytes)
    return HCBLAS_STATUS_INVALID_VALUE;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return HCBLAS_STATUS_EXECUTION_FAILED;
  }
  DeviceScratch ds;
  if (!device_scratch(dev, &ds)) return HCBLAS_STATUS_EXECUTION_FAILED;
  if (cudaMemsetAsync(ds.flag, 0, sizeof(int), static_cast<cudaStream_t>(stream)) != cudaSuccess)
    return HCBLAS_STATUS_EXECUTION_FAILED;

  /* column-major; for real data the conjugate transpose is the transpose */
  const int op_a = transa == HCBLAS_OP_N ? HCBK_OP_N : HCBK_OP_T;
  const int op_b = transb == HCBLAS_OP_N ? HCBK_OP_N : HCBK_OP_T;

  if (*alpha == 0.0f) { /* C := beta*C, A and B not referenced */
    hcbk_gemm_args a;
    memset(&a, 0, sizeof(a));
    a.dtype = HCBK_S;
    a.m = m;
    a.n = n;
    a.k = k;
    a.c = C;
    a.ldc = ldc;
    a.batch = 1;
    a.beta_re = *beta;
    return hcbk_scale_c(&a, stream) == HCBK_OK ? HCBLAS_STATUS_SUCCESS
                                               : HCBLAS_STATUS_EXECUTION_FAILED;
  }

  hcbk_pack_args pa;
  memset(&pa, 0, sizeof(pa));
  pa.src = A;
  pa.ld = lda;
  pa.k_contig = op_a != HCBK_OP_N; /* op(A) = A^T: element (m, k) at A[k + m*lda] */
  pa.rows = m;
  pa.kdim = k;
  pa.nplanes = nplanes;
  pa.ld_dst = kp;
  for (int i = 0; i < nplanes; ++i) pa.planes[i] = ds.scratch + i * a_bytes;
  hcbk_pack_args pb;
  memset(&pb, 0, sizeof(pb));
  pb.src = B;
  pb.ld = ldb;
  pb.k_contig = op_b == HCBK_OP_N; /* op(B) = B: element (k, n) at B[k + n*ldb] */
  pb.rows = n;
  pb.kdim = k;
  pb.nplanes = nplanes;
  pb.ld_dst = kp;
  unsigned char *bws = ds.scratch + nplanes * a_bytes;
  for (int i = 0; i < nplanes; ++i) pb.planes[i] = bws + i * b_bytes;
  if (hcbk_pack_split_bf16(&pa, stream) != HCBK_OK || hcbk_pack_split_bf16(&pb, stream) != HCBK_OK)
    return HCBLAS_STATUS_EXECUTION_FAILED;

  hcbk_split_gemm g;
  memset(&g, 0, sizeof(g));
  g.m = m;
  g.n = n;
  g.k = k;
  g.terms = terms;
  g.bn = 128;
  g.promote_kb = 1;
  g.pair = 0;
  for (int i = 0; i < nplanes; ++i) {
    g.a_planes[i] = pa.planes[i];
    g.b_planes[i] = pb.planes[i];
  }
  g.ld_a = kp;
  g.ld_b = kp;
  g.c = C;
  g.ldc = ldc;
  g.alpha = *alpha;
  g.beta = *beta;
  return hcbk_sgemm_split_tc(&g, ds.flag, stream) == HCBK_OK ? HCBLAS_STATUS_SUCCESS
                                                             : HCBLAS_STATUS_EXECUTION_FAILED;
}

extern "C" int hcblasSgemmSplitBF16NoAllocStatus(void *stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return -1;
  }
  DeviceScratch ds;
  if (!device_scratch(dev, &ds)) return -1;
  if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  int code = 0;
  if (cudaMemcpy(&code, ds.flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return code;
}
