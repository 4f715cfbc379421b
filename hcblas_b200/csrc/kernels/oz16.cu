/*
 * oz16.cu -- Ozaki-scheme DGEMM on the FP16 tensor-core path (tcgen05
 * kind::f16, FP32 accumulate in TMEM), sm_100a.
 *
 * Same scheme as the INT8 path (ozaki.cu / tc_gemm.cu), with 8-bit integer
 * slices stored as binary16:
 *   a_i, b_j in [-255, 255]  (exact in f16: 11-bit significand)
 *   a_i * b_j exact in f32 (< 2^16), and every f32 sum the tensor core forms
 *   here stays an integer below 2^24, hence exact: one TMEM accumulation
 *   covers one K-slab of 32 elements and one weight group d = i + j, at most
 *   (d+1) * 32 * 255^2 < 2^24 for d < 8.
 * After every (slab, group) the epilogue warps add 2^(-8(d+2)) * G_d into
 * FP64 registers, so the only roundings are these binary64 adds.  With s
 * slices the operands carry 8s bits (s = 7: 56 bits).
 *
 * Why this path exists: on the B200s this library is measured on,
 * tcgen05 kind::i8 sustains ~0.6 POPS in the same pipeline where kind::f16
 * sustains ~1.4 PFLOP/s, so f16 slice products finish ~2x sooner.
 *
 * CTA (192 threads, persistent, 1 per SM), tile 128 x 64:
 *   warp 0      TMA producer: per K-slab, the s A-planes and s B-planes
 *               (3-D tensor maps {K, rows, plane}, 64-byte swizzle)
 *   warp 1      TMEM owner + MMA issuer: per slab and group d, the d+1
 *               products a_i * b_(d-i) into one of two TMEM buffers
 *   warps 2..5  epilogue: warp w reads TMEM lane quadrant (w % 4), promotes
 *               the 64 columns of its lane into 64 FP64 accumulators, and
 *               finally writes alpha*2^(ea+eb)*acc + beta*C
 * Six warps keep at most two warps per SM sub-partition, which leaves the
 * epilogue threads the registers for 64 FP64 accumulators.
 * Every mbarrier wait is bounded (see tc_common.cuh).  No multicast.
 */
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hcbk.h"
#include "tc_common.cuh"

namespace hcbk {
namespace oz16 {

using namespace hcbk::tc;

constexpr int BM = 128, BN = 64;
constexpr int BKE = 32;   /* f16 elements per K-slab (64 bytes) */
constexpr int ROWB = 64;  /* bytes per tile row */
constexpr int UK = 16;    /* K per MMA */
constexpr uint32_t A_PLANE = BM * ROWB, B_PLANE = BN * ROWB;
constexpr int NTHREADS = 192;
constexpr int EPI_WARPS = 4;

struct Params {
  CUtensorMap ta;
  CUtensorMap tb;
  int m, n, k;
  int tiles_m, tiles_n;
  double *c;
  long long ldc;
  double alpha, beta;
  int beta_nonzero;
  const int *exp_a;
  const int *exp_b;
  int *err;
};

template <int S> struct Cfg {
  static constexpr uint32_t STAGE_BYTES = S * (A_PLANE + B_PLANE);
  static constexpr int STAGES = (STAGE_BYTES * 4 <= 200 * 1024) ? 4
                               : (STAGE_BYTES * 3 <= 216 * 1024) ? 3 : 2;
  static constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + 256 + 1024;
  static_assert(SMEM_BYTES <= 232448, "shared memory");
};

__device__ __forceinline__ double pow2_bits(int e) {
  return __longlong_as_double(static_cast<long long>(e + 1023) << 52);
}

template <int S>
__global__ void __launch_bounds__(NTHREADS, 1) oz16_kernel(const __grid_constant__ Params p) {
  using C = Cfg<S>;
  constexpr int STAGES = C::STAGES;
  constexpr int KSTEPS = BKE / UK; /* 2 */

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * C::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], EPI_WARPS);
    }
    mbar_fence_init();
  }
  if (warp == 0 && lane == 0) {
    tma_prefetch_desc(&p.ta);
    tma_prefetch_desc(&p.tb);
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 2 * BN);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  const int num_tiles = p.tiles_m * p.tiles_n;
  const int kblocks = (p.k + BKE - 1) / BKE;

  if (warp == 0) {
    /* ------------------------------------------------ TMA producer -- */
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int t = blockIdx.x; ok && t < num_tiles; t += gridDim.x) {
        const int tm = t % p.tiles_m, tn = t / p.tiles_m;
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], C::STAGE_BYTES);
          uint8_t *st = smem + s * C::STAGE_BYTES;
#pragma unroll
          for (int i = 0; i < S; ++i)
            tma_load_3d(st + i * A_PLANE, &p.ta, &full[s], kb * BKE, tm * BM, i);
#pragma unroll
          for (int j = 0; j < S; ++j)
            tma_load_3d(st + S * A_PLANE + j * B_PLANE, &p.tb, &full[s], kb * BKE, tn * BN, j);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
    }
  } else if (warp == 1) {
    /* ------------------------------------------------ MMA issuer -- */
    if (lane == 0) {
      const uint32_t idesc = make_idesc(1 /* f32 */, 0 /* f16 */, false, false, BM, BN);
      int s = 0;
      uint32_t ph = 0;
      uint32_t gi = 0; /* group counter: selects the TMEM buffer */
      bool ok = true;
      for (int t = blockIdx.x; ok && t < num_tiles; t += gridDim.x) {
        for (int kb = 0; ok && kb < kblocks; ++kb) {
          if (!mbar_wait(&full[s], ph, p.err, ERR_TIMEOUT_MMA_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sbase = smem_u32(smem + s * C::STAGE_BYTES);
#pragma unroll
          for (int d = 0; d < S; ++d, ++gi) {
            const uint32_t b = gi & 1u;
            if (!mbar_wait(&tempty[b], ((gi >> 1) & 1u) ^ 1u, p.err, ERR_TIMEOUT_MMA_TMEM)) {
              ok = false;
              break;
            }
            tc_fence_after();
#pragma unroll
            for (int i = 0; i <= d; ++i) {
#pragma unroll
              for (int kk = 0; kk < KSTEPS; ++kk) {
                const uint32_t aa = sbase + i * A_PLANE + kk * (UK * 2);
                const uint32_t ba = sbase + S * A_PLANE + (d - i) * B_PLANE + kk * (UK * 2);
                mma_f16(tmem_base + b * BN, smem_desc(aa, 16, 512, 4), smem_desc(ba, 16, 512, 4),
                        idesc, (i > 0 || kk > 0) ? 1u : 0u);
              }
            }
            mma_commit(&tfull[b]);
          }
          if (!ok) break;
          mma_commit(&empty[s]);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
    }
  } else {
    /* ------------------------------------------------ epilogue -- */
    const int q = warp & 3;
    uint32_t gi = 0;
    bool ok = true;
    for (int t = blockIdx.x; ok && t < num_tiles; t += gridDim.x) {
      const int tm = t % p.tiles_m, tn = t / p.tiles_m;
      double acc[64];
#pragma unroll
      for (int j = 0; j < 64; ++j) acc[j] = 0.0;
      for (int kb = 0; ok && kb < kblocks; ++kb) {
#pragma unroll
        for (int d = 0; d < S; ++d, ++gi) {
          const uint32_t b = gi & 1u;
          if (!mbar_wait(&tfull[b], (gi >> 1) & 1u, p.err, ERR_TIMEOUT_EPILOGUE)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t ta = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * BN;
          const double w = pow2_bits(-8 * (d + 2));
          uint32_t r[32];
          tmem_ld_32x32b_x32(ta, r);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[j] = fma((double)__uint_as_float(r[j]), w, acc[j]);
          tmem_ld_32x32b_x32(ta + 32, r);
          tmem_ld_wait();
#pragma unroll
          for (int j = 0; j < 32; ++j)
            acc[32 + j] = fma((double)__uint_as_float(r[j]), w, acc[32 + j]);
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&tempty[b]);
        }
      }
      if (!ok) break;
      /* C = alpha * 2^(ea + eb) * acc + beta * C */
      const int m = tm * BM + q * 32 + lane;
      if (m < p.m) {
        const int ea = p.exp_a[m];
        const int n0 = tn * BN;
        double *Cp = p.c + m;
#pragma unroll
        for (int c = 0; c < 64; c += 8) {
          const int nvalid = p.n - (n0 + c);
          if (nvalid <= 0) break;
          int eb[8];
          double cv[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) eb[j] = (j < nvalid) ? p.exp_b[n0 + c + j] : 0;
          if (p.beta_nonzero) {
#pragma unroll
            for (int j = 0; j < 8; ++j)
              cv[j] = (j < nvalid) ? Cp[(long long)(n0 + c + j) * p.ldc] : 0.0;
          }
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            if (j < nvalid) {
              const int e = ea + eb[j];
              double o;
              if (ea == HCBK_OZ_NONFINITE || eb[j] == HCBK_OZ_NONFINITE)
                o = __longlong_as_double(0x7ff8000000000000ll);
              else if (ea == HCBK_OZ_ZERO || eb[j] == HCBK_OZ_ZERO)
                o = 0.0;
              else if (e >= -1022 && e <= 1023)
                o = acc[c + j] * pow2_bits(e);
              else
                o = ldexp(acc[c + j], e);
              o *= p.alpha;
              if (p.beta_nonzero) o = fma(p.beta, cv[j], o);
              Cp[(long long)(n0 + c + j) * p.ldc] = o;
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, 2 * BN);
  }
}

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess && ptr)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    else
      cudaGetLastError();
  }
  return fn;
}

/* {K, rows, plane} f16 planes, row pitch ld elements, plane pitch pstride bytes */
static int make_map(CUtensorMap *map, const void *base, uint64_t kdim, uint64_t rows,
                    uint64_t planes, uint64_t ld, uint64_t pstride, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * 2) & 15) || (pstride & 15))
    return HCBK_ERR_ALIGN;
  cuuint64_t dims[3] = {kdim, rows, planes};
  cuuint64_t strides[2] = {ld * 2, pstride};
  cuuint32_t box[3] = {(cuuint32_t)BKE, box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, const_cast<void *>(base), dims,
                  strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HCBK_OK : HCBK_ERR_ALIGN;
}

template <int S>
static int launch(Params &p, void *stream) {
  auto kern = oz16_kernel<S>;
  static bool attr_set[64] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Cfg<S>::SMEM_BYTES) != cudaSuccess)
      return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  p.tiles_m = (p.m + BM - 1) / BM;
  p.tiles_n = (p.n + BN - 1) / BN;
  const int tiles = p.tiles_m * p.tiles_n;
  int grid = hcbk_sm_count();
  if (tiles < grid) grid = tiles;
  kern<<<grid, NTHREADS, Cfg<S>::SMEM_BYTES, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

}  // namespace oz16
}  // namespace hcbk

extern "C" int hcbk_ozaki16_gemm_tc(const hcbk_ozaki_gemm *g, int *err, void *stream) {
  using namespace hcbk::oz16;
  if (g->m > 0x7fffffff || g->n > 0x7fffffff || g->k > 0x7fffffff || g->k <= 0 || g->k0 != 0)
    return HCBK_ERR_ARGS;
  Params p;
  memset(&p, 0, sizeof(p));
  p.m = (int)g->m;
  p.n = (int)g->n;
  p.k = (int)g->k;
  int rc = make_map(&p.ta, g->a_planes, g->k, g->m, g->slices, g->ld_a, g->a_plane_stride, BM);
  if (rc) return rc;
  rc = make_map(&p.tb, g->b_planes, g->k, g->n, g->slices, g->ld_b, g->b_plane_stride, BN);
  if (rc) return rc;
  p.c = g->c;
  p.ldc = g->ldc;
  p.alpha = g->alpha;
  p.beta = g->beta;
  p.beta_nonzero = g->beta != 0.0;
  p.exp_a = g->exp_a;
  p.exp_b = g->exp_b;
  p.err = err;
  switch (g->slices) {
    case 3: return launch<3>(p, stream);
    case 4: return launch<4>(p, stream);
    case 5: return launch<5>(p, stream);
    case 6: return launch<6>(p, stream);
    case 7: return launch<7>(p, stream);
    default: return HCBK_ERR_ARGS;
  }
}
