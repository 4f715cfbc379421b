/*
 * ozaki.cu -- operand preparation for the Ozaki-scheme DGEMM on INT8 tensor
 * cores (Ozaki, Ogita, Oishi & Rump, "Error-free transformations of matrix
 * multiplication by using fast routines of matrix multiplication and its
 * applications", Numer. Algorithms 59, 2012; INT8 variant after Ootomo, Ozaki
 * & Yokota, "DGEMM on integer matrix multiplication unit", IJHPCA 2024).
 *
 * For op(A) (rows m, K) and op(B) (columns n, K):
 *   1. e_m = exponent of max_k |A(m,k)| (frexp convention: max < 2^e_m), so
 *      every |A(m,k)| * 2^-e_m < 1; likewise f_n for the columns of B.
 *   2. y = A(m,k) * 2^-e_m; for i = 0..s-1: y *= 128, a_i = trunc(y),
 *      y -= a_i.  Each a_i is an integer in [-127, 127] and
 *          A(m,k) = 2^e_m * sum_i a_i 2^(-7(i+1)) + O(2^(e_m - 7s)),
 *      every step exact in binary64.
 *   3. The tensor cores form a_i . b_j exactly in INT32 and the epilogue adds
 *      2^(e_m + f_n - 7(i+j+2)) * (a_i . b_j) over i + j < s in binary64.
 * The slices are written K-major, int8, [rows][ld_dst], so the GEMM reads
 * 64-byte K rows whatever the source layout; MN-contiguous sources are
 * transposed through a 32x32 shared-memory tile.
 *
 * Non-finite inputs: a row/column containing Inf or NaN gets the exponent
 * HCBK_OZ_NONFINITE, its slices are zero and the epilogue returns NaN for
 * the outputs it touches.  An all-zero row gets exponent 0 and zero slices.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "hcbk.h"

namespace {

/* frexp-style exponent of |x| (x = f * 2^e, 0.5 <= f < 1); INT_MIN/2 for 0 */
__device__ __forceinline__ int exp_of(double x) {
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(x));
  const int biased = static_cast<int>((bits >> 52) & 0x7FF);
  if (biased == 0x7FF) return HCBK_OZ_NONFINITE;
  if (biased != 0) return biased - 1022;
  if ((bits & 0x000FFFFFFFFFFFFFull) == 0) return HCBK_OZ_ZERO;
  int e;
  frexp(x, &e);
  return e;
}

__device__ __forceinline__ int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

/* K-contiguous source: one warp per row */
__global__ void oz_exp_kcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                               int *exps) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    int e = HCBK_OZ_ZERO;
    const double *row = src + r * ld;
    for (int64_t k = lane; k < kdim; k += 32) e = max(e, exp_of(row[k]));
    e = warp_max(e);
    if (lane == 0) exps[r] = e;
  }
}

/* MN-contiguous source: threads along rows, K split over blockIdx.y; the
 * partial maxima meet in exps[] (pre-set to HCBK_OZ_ZERO) via atomicMax */
__global__ void oz_exp_rcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                               int64_t kchunk, int *exps) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  const int64_t k0 = (int64_t)blockIdx.y * kchunk;
  const int64_t k1 = (k0 + kchunk < kdim) ? k0 + kchunk : kdim;
  int e = HCBK_OZ_ZERO;
  for (int64_t k = k0; k < k1; ++k) e = max(e, exp_of(src[r + k * ld]));
  atomicMax(&exps[r], e);
}

__global__ void oz_fill(int *exps, int64_t n, int v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    exps[i] = v;
}

template <int S>
__device__ __forceinline__ void slice_value(double x, int e, int8_t (&a)[S]) {
  if (e == HCBK_OZ_NONFINITE || e == HCBK_OZ_ZERO) {
#pragma unroll
    for (int i = 0; i < S; ++i) a[i] = 0;
    return;
  }
  double y = ldexp(x, -e); /* |y| < 1, exact */
#pragma unroll
  for (int i = 0; i < S; ++i) {
    y *= 128.0;
    const double t = trunc(y);
    a[i] = static_cast<int8_t>(static_cast<int>(t));
    y -= t;
  }
}

/* K-contiguous source: 8 consecutive k per thread, 8-byte plane stores */
template <int S>
__global__ void oz_slice_kcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                                 const int *exps, int8_t *planes, int64_t plane_stride,
                                 int64_t ld_dst) {
  const int64_t kq = (kdim + 7) / 8;
  const int64_t total = rows * kq;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / kq;
    const int64_t k0 = (idx % kq) * 8;
    const int e = exps[r];
    int8_t out[S][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      int8_t a[S];
      const double x = (k0 + j < kdim) ? src[r * ld + k0 + j] : 0.0;
      slice_value<S>(x, e, a);
#pragma unroll
      for (int i = 0; i < S; ++i) out[i][j] = a[i];
    }
    for (int i = 0; i < S; ++i) {
      int8_t *d = planes + i * plane_stride + r * ld_dst + k0;
      if (k0 + 8 <= kdim && ((reinterpret_cast<uintptr_t>(d) & 7) == 0)) {
        uint64_t w = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) w |= static_cast<uint64_t>(static_cast<uint8_t>(out[i][j])) << (8 * j);
        *reinterpret_cast<uint64_t *>(d) = w;
      } else {
        for (int j = 0; j < 8; ++j)
          if (k0 + j < kdim) d[j] = out[i][j];
      }
    }
  }
}

/* MN-contiguous source: 32x32 tile through shared memory */
template <int S>
__global__ void oz_slice_rcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                                 const int *exps, int8_t *planes, int64_t plane_stride,
                                 int64_t ld_dst) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < rows && k < kdim) ? src[r + k * ld] : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 8 * i;
    const int64_t r = r0 + rl, k = k0 + tx;
    if (r < rows && k < kdim) {
      int8_t a[S];
      slice_value<S>(tile[tx][rl], exps[r], a);
#pragma unroll
      for (int p = 0; p < S; ++p) planes[p * plane_stride + r * ld_dst + k] = a[p];
    }
  }
}

template <int S>
int launch_slice(const hcbk_ozaki_prep *a, cudaStream_t st) {
  int8_t *planes = static_cast<int8_t *>(a->planes);
  if (a->k_contig) {
    const int64_t total = a->rows * ((a->kdim + 7) / 8);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    oz_slice_kcontig<S><<<(unsigned)blocks, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim,
                                                          a->exps, planes, a->plane_stride,
                                                          a->ld_dst);
  } else {
    const int64_t gx = (a->rows + 31) / 32, gy = (a->kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    oz_slice_rcontig<S><<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(
        a->src, a->ld, a->rows, a->kdim, a->exps, planes, a->plane_stride, a->ld_dst);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

}  // namespace

extern "C" int hcbk_ozaki_exponents(const hcbk_ozaki_prep *a, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->rows <= 0 || a->kdim <= 0) return HCBK_ERR_ARGS;
  if (a->k_contig) {
    int64_t blocks = (a->rows * 32 + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    oz_exp_kcontig<<<(unsigned)blocks, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, a->exps);
  } else {
    const int64_t gx = (a->rows + 255) / 256;
    /* enough K-splits to give every SM a few blocks */
    int64_t ky = ((int64_t)hcbk_sm_count() * 4 + gx - 1) / gx;
    if (ky > 1024) ky = 1024;
    int64_t kchunk = (a->kdim + ky - 1) / ky;
    if (kchunk < 64) kchunk = 64;
    ky = (a->kdim + kchunk - 1) / kchunk;
    oz_fill<<<(unsigned)((a->rows + 255) / 256), 256, 0, st>>>(a->exps, a->rows, HCBK_OZ_ZERO);
    oz_exp_rcontig<<<dim3((unsigned)gx, (unsigned)ky), 256, 0, st>>>(a->src, a->ld, a->rows,
                                                                     a->kdim, kchunk, a->exps);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_ozaki_slice(const hcbk_ozaki_prep *a, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->rows <= 0 || a->kdim <= 0) return HCBK_ERR_ARGS;
  switch (a->slices) {
    case 3: return launch_slice<3>(a, st);
    case 4: return launch_slice<4>(a, st);
    case 5: return launch_slice<5>(a, st);
    case 6: return launch_slice<6>(a, st);
    case 7: return launch_slice<7>(a, st);
    case 8: return launch_slice<8>(a, st);
    default: return HCBK_ERR_ARGS;
  }
}
