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
#include <cuda_fp16.h>
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

/* |x| as an ordered bit pattern: the maximum over a row of these is the
 * pattern of max |x| (Inf and NaN above every finite value), and exp_of is
 * monotone in |x|, so one exp_of per row replaces one per element */
__device__ __forceinline__ unsigned long long abs_bits(double x) {
  return static_cast<unsigned long long>(__double_as_longlong(x)) & 0x7FFFFFFFFFFFFFFFull;
}

__device__ __forceinline__ int exp_of_bits(unsigned long long b) {
  return exp_of(__longlong_as_double(static_cast<long long>(b)));
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

/* K-contiguous source: one warp per row; VEC = 2 reads 16-byte pairs
 * (row start 16-byte aligned, even kdim) */
template <int VEC, typename T = double>
__global__ void oz_exp_kcontig(const T *src, int64_t ld, int64_t rows, int64_t kdim,
                               int *exps) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    unsigned long long m = 0;
    const T *row = src + r * ld;
    if constexpr (VEC == 2) {
      const double2 *row2 = reinterpret_cast<const double2 *>(row);
      const int64_t k2 = kdim / 2;
      int64_t k = lane;
      for (; k + 96 < k2; k += 128) { /* four 16-byte loads in flight */
        double2 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = row2[k + 32 * u];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          m = max(m, abs_bits(v[u].x));
          m = max(m, abs_bits(v[u].y));
        }
      }
      for (; k < k2; k += 32) {
        const double2 v = row2[k];
        m = max(m, abs_bits(v.x));
        m = max(m, abs_bits(v.y));
      }
    } else {
      for (int64_t k = lane; k < kdim; k += 32) m = max(m, abs_bits(static_cast<double>(row[k])));
    }
    m = warp_max_u64(m);
    if (lane == 0) exps[r] = exp_of_bits(m);
  }
}

/* MN-contiguous source: threads along rows, K split over blockIdx.y; the
 * partial maxima meet in exps[] (pre-set to HCBK_OZ_ZERO) via atomicMax.
 * VEC = 2: each thread owns two adjacent rows and reads 16-byte pairs (even
 * rows and ld, 16-byte aligned source); eight loads in flight. */
template <int VEC, typename T = double>
__global__ void oz_exp_rcontig(const T *src, int64_t ld, int64_t rows, int64_t kdim,
                               int64_t kchunk, int *exps) {
  const int64_t r = VEC * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  if (r >= rows) return;
  const int64_t k0 = (int64_t)blockIdx.y * kchunk;
  const int64_t k1 = (k0 + kchunk < kdim) ? k0 + kchunk : kdim;
  if constexpr (VEC == 2) {
    unsigned long long m0 = 0, m1 = 0;
    const double2 *p = reinterpret_cast<const double2 *>(src + r);
    const int64_t step = ld / 2;
    int64_t k = k0;
    for (; k + 8 <= k1; k += 8) {
      double2 v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = p[(k + u) * step];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        m0 = max(m0, abs_bits(v[u].x));
        m1 = max(m1, abs_bits(v[u].y));
      }
    }
    for (; k < k1; ++k) {
      const double2 v = p[k * step];
      m0 = max(m0, abs_bits(v.x));
      m1 = max(m1, abs_bits(v.y));
    }
    atomicMax(&exps[r], exp_of_bits(m0));
    atomicMax(&exps[r + 1], exp_of_bits(m1));
  } else {
    unsigned long long m = 0;
    int64_t k = k0;
    for (; k + 4 <= k1; k += 4) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = static_cast<double>(src[r + (k + u) * ld]);
#pragma unroll
      for (int u = 0; u < 4; ++u) m = max(m, abs_bits(v[u]));
    }
    for (; k < k1; ++k) m = max(m, abs_bits(static_cast<double>(src[r + k * ld])));
    atomicMax(&exps[r], exp_of_bits(m));
  }
}

__global__ void oz_fill(int *exps, int64_t n, int v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    exps[i] = v;
}

/* slice storage: int8 with 7-bit slices (radix 128) or binary16 with 8-bit
 * slices (radix 256, integers <= 255 are exact in binary16) */
template <typename ST> struct SliceT;
template <> struct SliceT<int8_t> {
  static constexpr double RADIX = 128.0;
  static __device__ __forceinline__ int8_t make(int v) { return static_cast<int8_t>(v); }
};
template <> struct SliceT<__half> {
  static constexpr double RADIX = 256.0;
  static __device__ __forceinline__ __half make(int v) { return __int2half_rn(v); }
};

template <int S, typename ST>
__device__ __forceinline__ void slice_value(double x, int e, ST (&a)[S]) {
  if (e == HCBK_OZ_NONFINITE || e == HCBK_OZ_ZERO) {
#pragma unroll
    for (int i = 0; i < S; ++i) a[i] = SliceT<ST>::make(0);
    return;
  }
  double y = ldexp(x, -e); /* |y| < 1, exact */
#pragma unroll
  for (int i = 0; i < S; ++i) {
    y *= SliceT<ST>::RADIX;
    const double t = trunc(y);
    a[i] = SliceT<ST>::make(static_cast<int>(t));
    y -= t;
  }
}

/* K-contiguous source: 8 consecutive k per thread, one vector store of the
 * 8 slices per plane (8 bytes for int8, 16 bytes for binary16) */
template <int S, typename ST, typename T = double>
__global__ void oz_slice_kcontig(const T *src, int64_t ld, int64_t rows, int64_t kdim,
                                 const int *exps, char *planes, int64_t plane_stride,
                                 int64_t ld_dst) {
  struct alignas(8 * sizeof(ST)) Vec8 { ST v[8]; };
  const int64_t kq = (kdim + 7) / 8;
  const int64_t total = rows * kq;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / kq;
    const int64_t k0 = (idx % kq) * 8;
    const int e = exps[r];
    Vec8 out[S];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      ST a[S];
      const double x = (k0 + j < kdim) ? static_cast<double>(src[r * ld + k0 + j]) : 0.0;
      slice_value<S, ST>(x, e, a);
#pragma unroll
      for (int i = 0; i < S; ++i) out[i].v[j] = a[i];
    }
    for (int i = 0; i < S; ++i) {
      ST *d = reinterpret_cast<ST *>(planes + i * plane_stride) + r * ld_dst + k0;
      if (k0 + 8 <= kdim && ((reinterpret_cast<uintptr_t>(d) & (sizeof(Vec8) - 1)) == 0)) {
        *reinterpret_cast<Vec8 *>(d) = out[i];
      } else {
        for (int j = 0; j < 8; ++j)
          if (k0 + j < kdim) d[j] = out[i].v[j];
      }
    }
  }
}

/* MN-contiguous source: 32x32 tile through shared memory */
template <int S, typename ST, typename T = double>
__global__ void oz_slice_rcontig(const T *src, int64_t ld, int64_t rows, int64_t kdim,
                                 const int *exps, char *planes, int64_t plane_stride,
                                 int64_t ld_dst) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < rows && k < kdim) ? static_cast<double>(src[r + k * ld]) : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 8 * i;
    const int64_t r = r0 + rl, k = k0 + tx;
    if (r < rows && k < kdim) {
      ST a[S];
      slice_value<S, ST>(tile[tx][rl], exps[r], a);
#pragma unroll
      for (int p = 0; p < S; ++p)
        reinterpret_cast<ST *>(planes + p * plane_stride)[r * ld_dst + k] = a[p];
    }
  }
}

template <int S, typename ST, typename T>
int launch_slice_src(const hcbk_ozaki_prep *a, const T *src, cudaStream_t st) {
  char *planes = static_cast<char *>(a->planes);
  if (a->k_contig) {
    const int64_t total = a->rows * ((a->kdim + 7) / 8);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    oz_slice_kcontig<S, ST, T><<<(unsigned)blocks, 256, 0, st>>>(
        src, a->ld, a->rows, a->kdim, a->exps, planes, a->plane_stride, a->ld_dst);
  } else {
    const int64_t gx = (a->rows + 31) / 32, gy = (a->kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    oz_slice_rcontig<S, ST, T><<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(
        src, a->ld, a->rows, a->kdim, a->exps, planes, a->plane_stride, a->ld_dst);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

template <int S, typename ST>
int launch_slice(const hcbk_ozaki_prep *a, cudaStream_t st) {
  return a->src_f32 ? launch_slice_src<S, ST, float>(a, a->src_f32, st)
                    : launch_slice_src<S, ST, double>(a, a->src, st);
}

template <int S>
int launch_slice_any(const hcbk_ozaki_prep *a, cudaStream_t st) {
  return a->f16 ? launch_slice<S, __half>(a, st) : launch_slice<S, int8_t>(a, st);
}

/* ---------------------------------------------------------------------
 * Row scales with a norm constraint (the CRT path): x(r,k) becomes the
 * integer rint(x f_r 2^(53 - e_r)) with |x| f 2^(53-e) < 2^53 (e_r at least
 * the frexp exponent of the row maximum) and the row norm
 * ||x(r,:)|| f 2^(53-e) <= 2^nb.  The norm comes from one pass: a sum of squares scaled by
 * the running maximum exponent (taken 2^-40 larger to cover its rounding);
 * rows split over several blocks merge their partials in a fixed order, so
 * the result does not depend on timing.
 * --------------------------------------------------------------------- */

/* 2^e for -1022 <= e <= 1023, from its bit pattern */
__device__ __forceinline__ double pow2i(int e) {
  return __longlong_as_double((long long)(e + 1023) << 52);
}

/* Running sum of squares scaled by the running maximum exponent, in the
 * manner of the reference BLAS dnrm2: s = sum (x 2^-e)^2 with e the frexp
 * exponent of the largest |x| so far; a larger exponent rescales s.  Zeros
 * and non-finite values are skipped (the maximum flags the latter). */
struct NormAcc {
  int e;     /* -1100: nothing yet */
  double s;
  double sc; /* 2^-e, 0 when outside the normal range */
};

__device__ __forceinline__ void na_init(NormAcc &a) {
  a.e = -1100;
  a.s = 0.0;
  a.sc = 0.0;
}

__device__ __forceinline__ void na_add(NormAcc &a, double x) {
  const int be = (int)((static_cast<unsigned long long>(__double_as_longlong(x)) >> 52) & 0x7FF);
  if (be == 0x7FF || x == 0.0) return;
  const int e = be == 0 ? -1021 : be - 1022; /* subnormals: an upper bound */
  if (e > a.e) {
    const int d = 2 * (a.e - e); /* < 0 */
    a.s = d >= -1022 ? a.s * pow2i(d) : 0.0;
    a.e = e;
    a.sc = (e >= -1022 && e <= 1022) ? pow2i(-e) : 0.0;
  }
  const double y = a.sc != 0.0 ? x * a.sc : ldexp(x, -a.e);
  a.s = fma(y, y, a.s);
}

/* merge a partial (be, bs) into a */
__device__ __forceinline__ void na_merge(NormAcc &a, int be, double bs) {
  if (be <= -1100) return;
  if (be > a.e) {
    const int d = 2 * (a.e - be);
    a.s = (d >= -1022 ? a.s * pow2i(d) : 0.0) + bs;
    a.e = be;
  } else {
    const int d = 2 * (be - a.e);
    a.s += d >= -1022 ? bs * pow2i(d) : 0.0;
  }
}

/* The scale f 2^(53 - e) of a row from its maximum's frexp exponent emax
 * (HCBK_OZ_ZERO / HCBK_OZ_NONFINITE pass through with f = 1) and its running
 * sum (||x|| = 2^acc_e sqrt(s)): e >= emax keeps |x| f 2^(53-e) < 2^53, and
 * f in (1/2, 1] -- rounded down to 8 significant bits, so that products of
 * two of them are exact -- keeps ||x|| f 2^(53-e) <= 2^nb. */
__device__ __forceinline__ void row_scale(int emax, int acc_e, double s, int nb, int *e_out,
                                          double *f_out, double *inv_out) {
  if (emax == HCBK_OZ_NONFINITE || emax == HCBK_OZ_ZERO) {
    *e_out = emax;
    *f_out = 1.0;
    *inv_out = 1.0;
    return;
  }
  const double rt = sqrt(s * (1.0 + 0x1p-40)) * (1.0 + 0x1p-50); /* ||x|| <= 2^acc_e rt */
  int er;
  frexp(rt, &er); /* rt < 2^er */
  int e = acc_e + er + 52 - nb;
  if (e < emax) e = emax;
  double f = ldexp(1.0 / rt, nb - 53 + e - acc_e); /* 2^(nb - 53 + e) / ||x|| */
  if (f >= 1.0) {
    f = 1.0;
  } else {
    f = ldexp(floor(ldexp(f, 8) * (1.0 - 0x1p-50)), -8); /* 8 bits, rounded down */
  }
  *e_out = e;
  *f_out = f;
  *inv_out = 1.0 / f;
}

/* K-contiguous source: one warp per row, one pass (16-byte pairs when the
 * row allows) */
template <int VEC>
__global__ void crt_rowexp_kcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                                   int nb, int *exps, double *frac, double *inv,
                                   int64_t rows_per, int64_t bstride) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    /* rows of a batch: element r / rows_per, its row r % rows_per */
    const int64_t e = r / rows_per;
    const double *row = src + e * bstride + (r - e * rows_per) * ld;
    unsigned long long m = 0;
    NormAcc acc;
    na_init(acc);
    if (VEC == 2) {
      const double2 *row2 = reinterpret_cast<const double2 *>(row);
      const int64_t n2 = kdim / 2;
      int64_t k = lane;
      for (; k + 7 * 32 < n2; k += 8 * 32) { /* eight 16-byte loads in flight per lane */
        double2 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = row2[k + 32 * u];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          m = max(m, max(abs_bits(v[u].x), abs_bits(v[u].y)));
          na_add(acc, v[u].x);
          na_add(acc, v[u].y);
        }
      }
      for (; k < n2; k += 32) {
        const double2 v = row2[k];
        m = max(m, max(abs_bits(v.x), abs_bits(v.y)));
        na_add(acc, v.x);
        na_add(acc, v.y);
      }
    } else {
      int64_t k = lane;
      for (; k + 7 * 32 < kdim; k += 8 * 32) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = row[k + 32 * u];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          m = max(m, abs_bits(v[u]));
          na_add(acc, v[u]);
        }
      }
      for (; k < kdim; k += 32) {
        const double x = row[k];
        m = max(m, abs_bits(x));
        na_add(acc, x);
      }
    }
    const int emax = exp_of_bits(warp_max_u64(m));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int oe = __shfl_xor_sync(0xffffffffu, acc.e, o);
      const double os = __shfl_xor_sync(0xffffffffu, acc.s, o);
      na_merge(acc, oe, os);
    }
    if (lane == 0) row_scale(emax, acc.e, acc.s, nb, exps + r, frac + r, inv + r);
  }
}

/* MN-contiguous source: threads along rows (two adjacent rows by 16-byte
 * pairs when VEC = 2), K split over blockIdx.y; each (chunk, row) writes its
 * maximum's bit pattern and its running sum (exponent, sum) */
template <int VEC>
__global__ void crt_rowexp_rcontig(const double *src, int64_t ld, int64_t rows, int64_t kdim,
                                   int64_t kchunk, unsigned long long *pm, int *pe, double *ps,
                                   int64_t bstride) {
  const int64_t r = VEC * ((int64_t)blockIdx.x * blockDim.x + threadIdx.x);
  if (r >= rows) return;
  /* element blockIdx.z of a batch: its source, and its rows' partials after
   * those of the elements before it */
  src += (int64_t)blockIdx.z * bstride;
  const int64_t rbase = (int64_t)blockIdx.z * rows;
  const int64_t k0 = (int64_t)blockIdx.y * kchunk;
  const int64_t k1 = (k0 + kchunk < kdim) ? k0 + kchunk : kdim;
  unsigned long long m[VEC];
  NormAcc acc[VEC];
#pragma unroll
  for (int u = 0; u < VEC; ++u) {
    m[u] = 0;
    na_init(acc[u]);
  }
  if (VEC == 2) {
    const double2 *p = reinterpret_cast<const double2 *>(src + r);
    const int64_t step = ld / 2;
    int64_t k = k0;
    for (; k + 8 <= k1; k += 8) { /* eight 16-byte loads in flight per thread */
      double2 v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = p[(k + u) * step];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        m[0] = max(m[0], abs_bits(v[u].x));
        m[VEC - 1] = max(m[VEC - 1], abs_bits(v[u].y));
        na_add(acc[0], v[u].x);
        na_add(acc[VEC - 1], v[u].y);
      }
    }
    for (; k < k1; ++k) {
      const double2 v = p[k * step];
      m[0] = max(m[0], abs_bits(v.x));
      m[VEC - 1] = max(m[VEC - 1], abs_bits(v.y));
      na_add(acc[0], v.x);
      na_add(acc[VEC - 1], v.y);
    }
  } else {
    for (int64_t k = k0; k < k1; ++k) {
      const double x = src[r + k * ld];
      m[0] = max(m[0], abs_bits(x));
      na_add(acc[0], x);
    }
  }
#pragma unroll
  for (int u = 0; u < VEC; ++u) { /* partials stored [row][chunk] for the finish */
    const int64_t o = (rbase + r + u) * gridDim.y + blockIdx.y;
    pm[o] = m[u];
    pe[o] = acc[u].e;
    ps[o] = acc[u].s;
  }
}

/* one warp per row: lanes merge chunks lane, lane + 32, ... in order, then a
 * fixed butterfly merges the lanes -- the same sum every run */
__global__ void crt_rowexp_finish(const unsigned long long *pm, const int *pe, const double *ps,
                                  int64_t rows, int nchunks, int nb, int *exps, double *frac, double *inv) {
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nwarps) {
    unsigned long long m = 0;
    NormAcc acc;
    na_init(acc);
    for (int c = lane; c < nchunks; c += 32) {
      const int64_t o = r * nchunks + c;
      m = max(m, pm[o]);
      na_merge(acc, pe[o], ps[o]);
    }
    m = warp_max_u64(m);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const int oe = __shfl_xor_sync(0xffffffffu, acc.e, o);
      const double os = __shfl_xor_sync(0xffffffffu, acc.s, o);
      na_merge(acc, oe, os);
    }
    if (lane == 0) row_scale(exp_of_bits(m), acc.e, acc.s, nb, exps + r, frac + r, inv + r);
  }
}

/* int32 to binary64 without the conversion unit: the pattern
 * 0x43300000:(v + 2^31) is 2^52 + 2^31 + v */
__device__ __forceinline__ double i32_to_d(int v) {
  return __hiloint2double(0x43300000, v ^ (int)0x80000000) - 4503601774854144.0;
}

/* Ozaki-I slice-group combine: four consecutive rows of one column per
 * thread (16-byte loads of each group's int32 sums), groups added smallest
 * weight first, then the exponent scaling and alpha / beta in FP64. */
__global__ void __launch_bounds__(256) oz_groups_combine(const hcbk_ozaki_groups_combine_args a) {
  const int64_t rows4 = (a.m + 3) / 4;
  const int64_t total = rows4 * a.n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t col = idx / rows4, r0 = (idx - col * rows4) * 4;
    const bool whole = r0 + 4 <= a.m;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int d = a.slices - 1; d >= 0; --d) {
      const int32_t *src = a.d + d * a.d_plane + col * a.ldd + r0;
      int4 q = make_int4(0, 0, 0, 0);
      if (whole) {
        q = __ldcs(reinterpret_cast<const int4 *>(src)); /* read once: stream past L2 */
      } else {
        int t[4] = {0, 0, 0, 0};
        for (int u = 0; u < 4; ++u)
          if (r0 + u < a.m) t[u] = src[u];
        q = make_int4(t[0], t[1], t[2], t[3]);
      }
      const double w = __longlong_as_double((long long)(1023 - 7 * (d + 2)) << 52);
      v[0] = fma(i32_to_d(q.x), w, v[0]);
      v[1] = fma(i32_to_d(q.y), w, v[1]);
      v[2] = fma(i32_to_d(q.z), w, v[2]);
      v[3] = fma(i32_to_d(q.w), w, v[3]);
    }
    const int eb = a.exp_b[col];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (r0 + u >= a.m) break;
      const int ea = a.exp_a[r0 + u];
      double o;
      if (ea == HCBK_OZ_NONFINITE || eb == HCBK_OZ_NONFINITE) {
        o = __longlong_as_double(0x7ff8000000000000ll);
      } else if (ea == HCBK_OZ_ZERO || eb == HCBK_OZ_ZERO) {
        o = 0.0;
      } else {
        const int e = ea + eb;
        o = (e >= -1022 && e <= 1023) ? v[u] * __longlong_as_double((long long)(e + 1023) << 52)
                                      : ldexp(v[u], e);
      }
      o *= a.alpha;
      const int64_t ci = col * a.ldc + r0 + u;
      if (a.c_f32) {
        if (a.beta != 0.0) o = fma(a.beta, static_cast<double>(a.c_f32[ci]), o);
        a.c_f32[ci] = static_cast<float>(o);
      } else {
        if (a.beta != 0.0) o = fma(a.beta, a.c[ci], o);
        a.c[ci] = o;
      }
    }
  }
}

/* the K split of the MN-contiguous row-exponent pass */
static void rowexp_split(int64_t rows, int64_t kdim, int64_t *ky, int64_t *kchunk) {
  /* about four 256-thread blocks per SM in all: one wave */
  const int64_t gx = (rows + 511) / 512;
  int64_t y = ((int64_t)hcbk_sm_count() * 4 + gx - 1) / gx;
  if (y > 1024) y = 1024;
  int64_t kc = (kdim + y - 1) / y;
  kc = (kc + 7) & ~int64_t(7);
  if (kc < 32) kc = 32;
  *ky = (kdim + kc - 1) / kc;
  *kchunk = kc;
}

}  // namespace

extern "C" int hcbk_ozaki_exponents(const hcbk_ozaki_prep *a, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->rows <= 0 || a->kdim <= 0 || a->batch > 1) return HCBK_ERR_ARGS;
  if (a->src_f32) { /* FP32 source: element loads, widened in registers */
    if (a->k_contig) {
      int64_t blocks = (a->rows * 32 + 255) / 256;
      const int64_t cap = (int64_t)hcbk_sm_count() * 16;
      if (blocks > cap) blocks = cap;
      oz_exp_kcontig<1, float><<<(unsigned)blocks, 256, 0, st>>>(a->src_f32, a->ld, a->rows,
                                                                  a->kdim, a->exps);
    } else {
      const int64_t gx = (a->rows + 255) / 256;
      int64_t ky = ((int64_t)hcbk_sm_count() * 8 + gx - 1) / gx;
      if (ky > 1024) ky = 1024;
      int64_t kchunk = (a->kdim + ky - 1) / ky;
      if (kchunk < 32) kchunk = 32;
      ky = (a->kdim + kchunk - 1) / kchunk;
      if (ky > 65535) return HCBK_ERR_ARGS;
      oz_fill<<<(unsigned)((a->rows + 255) / 256), 256, 0, st>>>(a->exps, a->rows, HCBK_OZ_ZERO);
      oz_exp_rcontig<1, float><<<dim3((unsigned)gx, (unsigned)ky), 256, 0, st>>>(
          a->src_f32, a->ld, a->rows, a->kdim, kchunk, a->exps);
    }
    return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
  }
  const bool al16 = (reinterpret_cast<uintptr_t>(a->src) & 15) == 0 && (a->ld & 1) == 0;
  if (a->k_contig) {
    int64_t blocks = (a->rows * 32 + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    if (al16 && (a->kdim & 1) == 0)
      oz_exp_kcontig<2><<<(unsigned)blocks, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, a->exps);
    else
      oz_exp_kcontig<1><<<(unsigned)blocks, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, a->exps);
  } else {
    const int vec = (al16 && (a->rows & 1) == 0) ? 2 : 1;
    const int64_t gx = (a->rows / vec + 255) / 256;
    /* enough K-splits to give every SM several blocks */
    int64_t ky = ((int64_t)hcbk_sm_count() * 8 + gx - 1) / gx;
    if (ky > 1024) ky = 1024;
    int64_t kchunk = (a->kdim + ky - 1) / ky;
    if (kchunk < 32) kchunk = 32;
    ky = (a->kdim + kchunk - 1) / kchunk;
    if (ky > 65535) return HCBK_ERR_ARGS;
    oz_fill<<<(unsigned)((a->rows + 255) / 256), 256, 0, st>>>(a->exps, a->rows, HCBK_OZ_ZERO);
    const dim3 grid((unsigned)gx, (unsigned)ky);
    if (vec == 2)
      oz_exp_rcontig<2><<<grid, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, kchunk, a->exps);
    else
      oz_exp_rcontig<1><<<grid, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, kchunk, a->exps);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_ozaki_groups_combine(const hcbk_ozaki_groups_combine_args *a, void *stream) {
  if (a->m <= 0 || a->n <= 0 || a->slices < 1 || a->slices > 8 || a->ldd < a->m ||
      (a->ldd & 3) || (a->d_plane & 3) || (reinterpret_cast<uintptr_t>(a->d) & 15))
    return HCBK_ERR_ARGS;
  const int64_t total = (a->m + 3) / 4 * a->n;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)hcbk_sm_count() * 16;
  if (blocks > cap) blocks = cap;
  oz_groups_combine<<<(unsigned)blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(*a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_ozaki_slice(const hcbk_ozaki_prep *a, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->rows <= 0 || a->kdim <= 0 || a->batch > 1) return HCBK_ERR_ARGS;
  switch (a->slices) {
    case 3: return launch_slice_any<3>(a, st);
    case 4: return launch_slice_any<4>(a, st);
    case 5: return launch_slice_any<5>(a, st);
    case 6: return launch_slice_any<6>(a, st);
    case 7: return launch_slice_any<7>(a, st);
    case 8: return launch_slice_any<8>(a, st);
    default: return HCBK_ERR_ARGS;
  }
}

extern "C" int64_t hcbk_crt_row_exponents_workspace_batch(int64_t rows, int64_t kdim,
                                                           int k_contig, int64_t batch) {
  if (k_contig || rows <= 0 || kdim <= 0 || batch <= 0) return 0;
  int64_t ky, kc;
  rowexp_split(rows, kdim, &ky, &kc);
  return ky * rows * batch * (int64_t)(sizeof(unsigned long long) + sizeof(double) + sizeof(int)) +
         256;
}

extern "C" int64_t hcbk_crt_row_exponents_workspace(int64_t rows, int64_t kdim, int k_contig) {
  return hcbk_crt_row_exponents_workspace_batch(rows, kdim, k_contig, 1);
}

extern "C" int hcbk_crt_row_scales(const hcbk_ozaki_prep *a, int nb, int pair_rows, double *frac,
                                   double *inv, void *work, int64_t work_bytes, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->rows <= 0 || a->kdim <= 0 || !frac || !inv) return HCBK_ERR_ARGS;
  if (pair_rows && (a->k_contig || (a->rows & 1))) return HCBK_ERR_ARGS;
  /* a batch: every element's rows in turn (exps / frac / inv of element e
   * at + e * rows); one element when batch is 0 or 1 */
  const int64_t batch = a->batch > 1 ? a->batch : 1;
  const int64_t bstride = batch > 1 ? a->src_bstride : 0;
  if (batch > 65535 && !a->k_contig) return HCBK_ERR_ARGS;
  const int64_t all_rows = a->rows * batch;
  const bool al16 = (reinterpret_cast<uintptr_t>(a->src) & 15) == 0 && (a->ld & 1) == 0 &&
                    (bstride & 1) == 0;
  if (a->k_contig) {
    int64_t blocks = (all_rows * 32 + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    if (al16 && (a->kdim & 1) == 0)
      crt_rowexp_kcontig<2><<<(unsigned)blocks, 256, 0, st>>>(
          a->src, a->ld, all_rows, a->kdim, nb, a->exps, frac, inv, a->rows, bstride);
    else
      crt_rowexp_kcontig<1><<<(unsigned)blocks, 256, 0, st>>>(
          a->src, a->ld, all_rows, a->kdim, nb, a->exps, frac, inv, a->rows, bstride);
  } else {
    int64_t ky, kc;
    rowexp_split(a->rows, a->kdim, &ky, &kc);
    if (ky > 65535 || !work ||
        work_bytes < hcbk_crt_row_exponents_workspace_batch(a->rows, a->kdim, 0, batch))
      return HCBK_ERR_ARGS;
    unsigned long long *pm = static_cast<unsigned long long *>(work);
    double *ps = reinterpret_cast<double *>(pm + ky * all_rows);
    int *pe = reinterpret_cast<int *>(ps + ky * all_rows);
    const int vec = (al16 && (a->rows & 1) == 0) ? 2 : 1;
    const dim3 grid((unsigned)((a->rows / vec + 255) / 256), (unsigned)ky, (unsigned)batch);
    if (vec == 2)
      crt_rowexp_rcontig<2><<<grid, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, kc, pm, pe, ps,
                                                   bstride);
    else
      crt_rowexp_rcontig<1><<<grid, 256, 0, st>>>(a->src, a->ld, a->rows, a->kdim, kc, pm, pe, ps,
                                                   bstride);
    int64_t fb = (all_rows * 32 + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (fb > cap) fb = cap;
    /* partials sit [row][chunk], element after element: two consecutive
     * rows merged are one row of twice the chunks */
    const int g = pair_rows ? 2 : 1;
    crt_rowexp_finish<<<(unsigned)fb, 256, 0, st>>>(pm, pe, ps, all_rows / g, (int)ky * g, nb,
                                                     a->exps, frac, inv);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
