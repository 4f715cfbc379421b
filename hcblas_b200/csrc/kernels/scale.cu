/*
 * scale.cu -- the alpha == 0 path: C := beta * C, or C := 0 when beta == 0
 * (C is then not read, as CBLAS specifies).
 *
 * Reference behaviour being replaced: gemm_alpha0_col / gemm_alpha0_row
 * (lib/src/blas/sgemm/sgemm_array_wrapper.cpp:157-293) launch one 256-thread
 * block per element with only thread 0 active, and first replace NaN/Inf in C
 * by 0.  Here the update is one coalesced grid-stride pass over the (column-
 * major canonical) C tile, and NaN/Inf are propagated per IEEE/CBLAS rather
 * than scrubbed.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hcbk.h"

namespace {

template <typename T> struct ScaleOps;
template <> struct ScaleOps<float> {
  using S = float;
  static __device__ float mul(S b, float c) { return b * c; }
  static __device__ float zero() { return 0.f; }
};
template <> struct ScaleOps<double> {
  using S = double;
  static __device__ double mul(S b, double c) { return b * c; }
  static __device__ double zero() { return 0.0; }
};
template <> struct ScaleOps<float2> {
  using S = float2;
  static __device__ float2 mul(S b, float2 c) {
    return make_float2(b.x * c.x - b.y * c.y, b.x * c.y + b.y * c.x);
  }
  static __device__ float2 zero() { return make_float2(0.f, 0.f); }
};
template <> struct ScaleOps<double2> {
  using S = double2;
  static __device__ double2 mul(S b, double2 c) {
    return make_double2(b.x * c.x - b.y * c.y, b.x * c.y + b.y * c.x);
  }
  static __device__ double2 zero() { return make_double2(0.0, 0.0); }
};
template <> struct ScaleOps<__half> {
  using S = float;
  static __device__ __half mul(S b, __half c) { return __float2half_rn(b * __half2float(c)); }
  static __device__ __half zero() { return __float2half_rn(0.f); }
};

template <typename T>
__global__ void scale_c_kernel(T *c, T *const *c_arr, int64_t c_off, int64_t sc, int64_t ldc,
                               int64_t m, int64_t n, int64_t batch,
                               typename ScaleOps<T>::S beta, int beta_nonzero) {
  const int64_t total = m * n;
  for (int64_t b = blockIdx.y; b < batch; b += gridDim.y) {
    T *C = (c_arr ? c_arr[b] : c) + c_off + b * sc;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
      const int64_t row = i % m, col = i / m;
      T *p = C + row + col * ldc;
      *p = beta_nonzero ? ScaleOps<T>::mul(beta, *p) : ScaleOps<T>::zero();
    }
  }
}

template <typename T>
int launch_scale(const hcbk_gemm_args *a, typename ScaleOps<T>::S beta, cudaStream_t st) {
  const int64_t total = a->m * a->n;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)hcbk_sm_count() * 8;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  dim3 grid((unsigned)blocks, (unsigned)(a->batch < 65535 ? a->batch : 65535));
  scale_c_kernel<T><<<grid, 256, 0, st>>>(static_cast<T *>(a->c),
                                           reinterpret_cast<T *const *>(a->c_array), a->c_off,
                                           a->stride_c, a->ldc, a->m, a->n, a->batch, beta,
                                           (a->beta_re != 0.0 || a->beta_im != 0.0));
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

}  // namespace

extern "C" int hcbk_scale_c(const hcbk_gemm_args *a, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->m <= 0 || a->n <= 0 || a->batch <= 0) return HCBK_OK;
  switch (a->dtype) {
    case HCBK_S: return launch_scale<float>(a, (float)a->beta_re, st);
    case HCBK_D: return launch_scale<double>(a, a->beta_re, st);
    case HCBK_C:
      return launch_scale<float2>(a, make_float2((float)a->beta_re, (float)a->beta_im), st);
    case HCBK_Z: return launch_scale<double2>(a, make_double2(a->beta_re, a->beta_im), st);
    case HCBK_H: return launch_scale<__half>(a, (float)a->beta_re, st);
    default: return HCBK_ERR_ARGS;
  }
}

extern "C" int hcbk_sm_count(void) {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (cached[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
      v = 148;
    cached[dev] = v;
  }
  return cached[dev];
}
