/*
 * pack.cu -- operand preparation for the emulated tensor-core paths.
 *
 * Split-BF16 (Henry, Tang & Heinecke, "Leveraging the bfloat16 artificial
 * intelligence datatype for higher-precision computations", ARITH 2019):
 * each f32 value x is written as an unevaluated sum of bf16 terms
 *     hi  = rn_bf16(x)
 *     mid = rn_bf16(x - hi)            (exact subtraction in f32)
 *     lo  = rn_bf16(x - hi - mid)
 * Two planes (hi, lo := mid) carry ~16 significant bits and feed the 3-product
 * scheme hi*hi + hi*lo + lo*hi; three planes carry the full 24 bits and feed
 * the 6-product scheme.  Non-finite hi keeps the special value in hi and
 * zeroes the lower terms.
 *
 * The planes are written K-major ([rows][ld_dst], K contiguous) whatever the
 * source layout, so the tensor-core kernel always reads 128-byte K rows; a
 * source whose rows are contiguous along M/N is transposed through a 32x32
 * shared-memory tile (coalesced on both sides).
 */
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "hcbk.h"
#include "split_bf16.cuh"

namespace {

/* K-contiguous sources of one or two operands in one launch: element
 * (r, k) of operand j at a[j].src[k + r*ld]; each thread splits 8
 * consecutive k of one row (two 16-byte loads where the source allows) and
 * writes 16 bytes to every plane where the planes' row pitch is a multiple of
 * 8 elements (the row's padding past K then receives zeros). */
struct PackPair {
  hcbk_pack_args a[2];
  int64_t kq[2];    /* 8-element groups per row */
  int64_t units0;   /* rows * kq of operand 0 */
  int64_t total;    /* all groups */
  int vec_src[2], vec_dst[2];
};

__global__ void pack_kcontig(const __grid_constant__ PackPair pp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pp.total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int which = i >= pp.units0 ? 1 : 0;
    const hcbk_pack_args &a = pp.a[which];
    const int64_t idx = i - (which ? pp.units0 : 0);
    const int64_t kq = pp.kq[which];
    const int64_t r = idx / kq;
    const int64_t k0 = (idx - r * kq) * 8;
    const float *s = a.src + r * a.ld + k0;
    float v[8];
    if (pp.vec_src[which] && k0 + 8 <= a.kdim) {
      const float4 f0 = *reinterpret_cast<const float4 *>(s);
      const float4 f1 = *reinterpret_cast<const float4 *>(s + 4);
      v[0] = f0.x; v[1] = f0.y; v[2] = f0.z; v[3] = f0.w;
      v[4] = f1.x; v[5] = f1.y; v[6] = f1.z; v[7] = f1.w;
    } else {
#pragma unroll
      for (int e = 0; e < 8; ++e) v[e] = (k0 + e < a.kdim) ? s[e] : 0.f;
    }
    uint32_t w[4][3];
#pragma unroll
    for (int j = 0; j < 4; ++j) split_terms2(v[2 * j], v[2 * j + 1], w[j]);
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      if (p >= a.nplanes) break;
      __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(a.planes[p]) + r * a.ld_dst + k0;
      if (pp.vec_dst[which]) {
        *reinterpret_cast<uint4 *>(d) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
      } else {
#pragma unroll
        for (int e = 0; e < 8; ++e)
          if (k0 + e < a.kdim)
            d[e] = __ushort_as_bfloat16(static_cast<unsigned short>(w[e >> 1][p] >> (16 * (e & 1))));
      }
    }
  }
}

/* source MN-contiguous: element (r, k) at src[r + k*ld]; 32x32 tiles */
__global__ void pack_rcontig(hcbk_pack_args a) {
  __shared__ float tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < a.rows && k < a.kdim) ? a.src[r + k * a.ld] : 0.f;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 8 * i;
    const int64_t r = r0 + rl, k = k0 + tx;
    if (r < a.rows && k < a.kdim) {
      __nv_bfloat16 t[3];
      split_terms(tile[tx][rl], t);
#pragma unroll
      for (int p = 0; p < 3; ++p)
        if (p < a.nplanes) static_cast<__nv_bfloat16 *>(a.planes[p])[r * a.ld_dst + k] = t[p];
    }
  }
}

/* complex source: parts 0 = real, 1 = imaginary (signed), 2 = their f32 sum */
__device__ __forceinline__ void cparts(float2 z, float im_sign, float (&v)[3]) {
  v[0] = z.x;
  v[1] = im_sign * z.y;
  v[2] = v[0] + v[1];
}

/* K-contiguous complex source: 4 k per thread */
__global__ void cpack_kcontig(hcbk_cpack_args a) {
  const int64_t kq = (a.kdim + 3) / 4;
  const int64_t total = a.rows * kq;
  const float im_sign = a.conj ? -1.f : 1.f;
  const float2 *src = static_cast<const float2 *>(a.src);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / kq;
    const int64_t k0 = (i % kq) * 4;
    float v[4][3];
#pragma unroll
    for (int e = 0; e < 4; ++e)
      cparts((k0 + e < a.kdim) ? src[r * a.ld + k0 + e] : make_float2(0.f, 0.f), im_sign, v[e]);
#pragma unroll
    for (int part = 0; part < 3; ++part) {
      __nv_bfloat16 t[4][3];
#pragma unroll
      for (int e = 0; e < 4; ++e) split_terms(v[e][part], t[e]);
      #pragma unroll
      for (int p = 0; p < 3; ++p) {
        if (p >= a.nplanes) break;
        __nv_bfloat16 *d = static_cast<__nv_bfloat16 *>(a.planes[part][p]) + r * a.ld_dst + k0;
#pragma unroll
        for (int e = 0; e < 4; ++e)
          if (k0 + e < a.kdim) d[e] = t[e][p];
      }
    }
  }
}

/* MN-contiguous complex source: 32x32 tiles */
__global__ void cpack_rcontig(hcbk_cpack_args a) {
  __shared__ float2 tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
  const float2 *src = static_cast<const float2 *>(a.src);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < a.rows && k < a.kdim) ? src[r + k * a.ld] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float im_sign = a.conj ? -1.f : 1.f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 8 * i;
    const int64_t r = r0 + rl, k = k0 + tx;
    if (r < a.rows && k < a.kdim) {
      float v[3];
      cparts(tile[tx][rl], im_sign, v);
#pragma unroll
      for (int part = 0; part < 3; ++part) {
        __nv_bfloat16 t[3];
        split_terms(v[part], t);
#pragma unroll
        for (int p = 0; p < 3; ++p)
          if (p < a.nplanes)
            static_cast<__nv_bfloat16 *>(a.planes[part][p])[r * a.ld_dst + k] = t[p];
      }
    }
  }
}

__global__ void c3m_combine_kernel(hcbk_c3m_combine_args a) {
  const bool bnz = a.beta_re != 0.f || a.beta_im != 0.f;
  float2 *C = static_cast<float2 *>(a.c);
  for (int64_t col = blockIdx.y; col < a.n; col += gridDim.y) {
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < a.m;
         row += (int64_t)gridDim.x * blockDim.x) {
      const int64_t t = row + col * a.ldt;
      const float t1 = a.t1[t], t2 = a.t2[t], t3 = a.t3[t];
      const float re = t1 - t2;
      const float im = (t3 - t1) - t2;
      float2 o;
      o.x = a.alpha_re * re - a.alpha_im * im;
      o.y = a.alpha_re * im + a.alpha_im * re;
      float2 *dst = C + row + col * a.ldc;
      if (bnz) {
        const float2 cv = *dst;
        o.x = fmaf(a.beta_re, cv.x, fmaf(-a.beta_im, cv.y, o.x));
        o.y = fmaf(a.beta_re, cv.y, fmaf(a.beta_im, cv.x, o.y));
      }
      *dst = o;
    }
  }
}

}  // namespace

extern "C" int hcbk_pack_split_bf16_complex(const hcbk_cpack_args *a, void *stream) {
  if (a->rows <= 0 || a->kdim <= 0 || a->nplanes < 1 || a->nplanes > 3) return HCBK_ERR_ARGS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->k_contig) {
    const int64_t total = a->rows * ((a->kdim + 3) / 4);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    cpack_kcontig<<<(unsigned)blocks, 256, 0, st>>>(*a);
  } else {
    const int64_t gx = (a->rows + 31) / 32, gy = (a->kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    cpack_rcontig<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(*a);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_c3m_combine(const hcbk_c3m_combine_args *a, void *stream) {
  if (a->m <= 0 || a->n <= 0) return HCBK_ERR_ARGS;
  int64_t gx = (a->m + 255) / 256;
  if (gx > 65535) gx = 65535;
  const int64_t gy = a->n < 65535 ? a->n : 65535;
  c3m_combine_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, 0,
                       static_cast<cudaStream_t>(stream)>>>(*a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

namespace {
bool pack_ok(const hcbk_pack_args *a) {
  return a->rows > 0 && a->kdim > 0 && a->nplanes >= 1 && a->nplanes <= 3 && a->ld_dst >= a->kdim;
}

/* one launch over the K-contiguous operands among a[0 .. n-1] */
int launch_kcontig(const hcbk_pack_args *const *a, int n, cudaStream_t st) {
  PackPair pp;
  memset(&pp, 0, sizeof(pp));
  int64_t total = 0;
  for (int j = 0; j < n; ++j) {
    pp.a[j] = *a[j];
    pp.kq[j] = (a[j]->kdim + 7) / 8;
    pp.vec_src[j] = (reinterpret_cast<uintptr_t>(a[j]->src) & 15) == 0 && (a[j]->ld & 3) == 0;
    int vd = (a[j]->ld_dst & 7) == 0;
    for (int p = 0; p < a[j]->nplanes; ++p)
      vd = vd && (reinterpret_cast<uintptr_t>(a[j]->planes[p]) & 15) == 0;
    pp.vec_dst[j] = vd;
    if (j == 0) pp.units0 = a[j]->rows * pp.kq[j];
    total += a[j]->rows * pp.kq[j];
  }
  pp.total = total;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)hcbk_sm_count() * 16;
  if (blocks > cap) blocks = cap;
  pack_kcontig<<<(unsigned)blocks, 256, 0, st>>>(pp);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

int launch_rcontig(const hcbk_pack_args *a, cudaStream_t st) {
  const int64_t gx = (a->rows + 31) / 32, gy = (a->kdim + 31) / 32;
  if (gy > 65535) return HCBK_ERR_ARGS;
  pack_rcontig<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(*a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
}  // namespace

extern "C" int hcbk_pack_split_bf16(const hcbk_pack_args *a, void *stream) {
  if (!pack_ok(a)) return HCBK_ERR_ARGS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->k_contig) return launch_kcontig(&a, 1, st);
  return launch_rcontig(a, st);
}

extern "C" int hcbk_pack_split_bf16_pair(const hcbk_pack_args *a, const hcbk_pack_args *b,
                                         void *stream) {
  if (!pack_ok(a) || !pack_ok(b)) return HCBK_ERR_ARGS;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->k_contig && b->k_contig) {
    const hcbk_pack_args *both[2] = {a, b};
    return launch_kcontig(both, 2, st);
  }
  int rc = a->k_contig ? launch_kcontig(&a, 1, st) : launch_rcontig(a, st);
  if (rc) return rc;
  return b->k_contig ? launch_kcontig(&b, 1, st) : launch_rcontig(b, st);
}
