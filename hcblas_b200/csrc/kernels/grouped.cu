/*
 * grouped.cu -- persistent grouped HGEMM on tcgen05: thousands of uneven
 * problems (each its own M, N, K, transposes, leading dimensions and
 * pointers) in ONE launch.
 *
 * The host writes a device-side problem table (hcbk_grouped_entry: TMA
 * tensor maps of op(A) and op(B), the C block, the shape) and the prefix
 * sums of every problem's 128 x 128 tile count.  Each CTA (one per SM,
 * 192 threads) walks the global tile sequence t = blockIdx.x,
 * blockIdx.x + gridDim.x, ...; every role finds the tile's problem by a
 * binary search over the prefix sums:
 *   warp 0      TMA producer: A and B K-slabs of the tile's problem, through
 *               that problem's tensor maps (read from global memory), into a
 *               6-stage SW128 ring
 *   warp 1      TMEM allocation; one lane issues tcgen05.mma with the
 *               problem's major-ness in the instruction descriptor
 *   warps 2..5  epilogue: TMEM -> alpha*acc + beta*C -> f16 C of the problem
 * Accumulators are double-buffered in TMEM, so a tile's epilogue overlaps the
 * next tile's MMAs, whichever problem it belongs to.  The host orders the
 * problems by decreasing work (longest-processing-time first) so that the
 * round-robin tile walk ends with the cheap tiles.  Every wait is bounded.
 * No cluster multicast is used.
 */
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include "hcbk.h"
#include "tc_common.cuh"

namespace hcbk {
namespace grouped {

using namespace hcbk::tc;

constexpr int BM = 128, BN = 128, BK = 64; /* BK f16 = one 128-byte swizzle atom */
constexpr int STAGES = 6;
constexpr uint32_t A_BYTES = BM * 128, B_BYTES = BN * 128;
constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES;
constexpr uint32_t SMEM_BYTES = STAGES * STAGE_BYTES + 256 + 1024;
constexpr uint32_t TMEM_COLS = 2 * BN;

struct Params {
  const hcbk_grouped_entry *table;
  const int32_t *tile_start;
  int count;
  int total_tiles;
  float alpha, beta;
  int beta_nonzero;
  int *err;
};

/* problem holding global tile t: the last g with tile_start[g] <= t */
__device__ __forceinline__ int find_problem(const int32_t *ts, int count, int t) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(ts + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct TileRef {
  const hcbk_grouped_entry *e;
  int tm, tn;
};

__device__ __forceinline__ TileRef tile_ref(const Params &p, int t) {
  const int g = find_problem(p.tile_start, p.count, t);
  const hcbk_grouped_entry *e = p.table + g;
  const int lt = t - __ldg(p.tile_start + g);
  const int tiles_m = __ldg(&e->tiles_m);
  return TileRef{e, lt % tiles_m, lt / tiles_m};
}

__global__ void __launch_bounds__(192, 1) grouped_hgemm_kernel(const __grid_constant__ Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
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
      mbar_init(&tempty[b], 4);
    }
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == 0) {
    /* ------------------------------------------------ TMA producer -- */
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
        const TileRef r = tile_ref(p, t);
        const CUtensorMap *ma = reinterpret_cast<const CUtensorMap *>(r.e->map_a);
        const CUtensorMap *mb = reinterpret_cast<const CUtensorMap *>(r.e->map_b);
        const int k = __ldg(&r.e->k);
        const int a_mn = __ldg(&r.e->a_mn), b_mn = __ldg(&r.e->b_mn);
        const int kblocks = (k + BK - 1) / BK;
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], STAGE_BYTES);
          uint8_t *st = smem + s * STAGE_BYTES;
          const int k0 = kb * BK;
          if (!a_mn) {
            tma_load_2d(st, ma, &full[s], k0, r.tm * BM);
          } else {
            tma_load_2d(st, ma, &full[s], r.tm * BM, k0);
            tma_load_2d(st + BK * 128, ma, &full[s], r.tm * BM + 64, k0);
          }
          uint8_t *sb = st + A_BYTES;
          if (!b_mn) {
            tma_load_2d(sb, mb, &full[s], k0, r.tn * BN);
          } else {
            tma_load_2d(sb, mb, &full[s], r.tn * BN, k0);
            tma_load_2d(sb + BK * 128, mb, &full[s], r.tn * BN + 64, k0);
          }
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
      int s = 0;
      uint32_t ph = 0;
      int ci = 0;
      bool ok = true;
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x, ++ci) {
        const TileRef r = tile_ref(p, t);
        const int k = __ldg(&r.e->k);
        const bool a_mn = __ldg(&r.e->a_mn) != 0, b_mn = __ldg(&r.e->b_mn) != 0;
        const int kblocks = (k + BK - 1) / BK;
        const uint32_t idesc = make_idesc(1, 0, a_mn, b_mn, BM, BN);
        const uint32_t a_lbo = a_mn ? BK * 128 : 16, b_lbo = b_mn ? BK * 128 : 16;
        const uint32_t a_kstep = a_mn ? 16 * 128 : 32, b_kstep = b_mn ? 16 * 128 : 32;
        const int b = ci & 1;
        const uint32_t tph = (ci >> 1) & 1;
        if (!mbar_wait(&tempty[b], tph ^ 1u, p.err, ERR_TIMEOUT_MMA_TMEM)) break;
        tc_fence_after();
        const uint32_t dbase = tmem_base + b * BN;
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&full[s], ph, p.err, ERR_TIMEOUT_MMA_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
          const uint32_t sb = sa + A_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint64_t ad = smem_desc(sa + kk * a_kstep, a_lbo, 1024, 2);
            const uint64_t bd = smem_desc(sb + kk * b_kstep, b_lbo, 1024, 2);
            mma_f16(dbase, ad, bd, idesc, (kb > 0 || kk > 0) ? 1u : 0u);
          }
          mma_commit(&empty[s]);
          if (++s == STAGES) {
            s = 0;
            ph ^= 1u;
          }
        }
        if (ok) mma_commit(&tfull[b]);
      }
    }
  } else {
    /* ------------------------------------------------ epilogue -- */
    const int q = warp & 3; /* TMEM lane quadrant */
    int ci = 0;
    for (int t = blockIdx.x; t < p.total_tiles; t += gridDim.x, ++ci) {
      const TileRef r = tile_ref(p, t);
      const int pm = __ldg(&r.e->m), pn = __ldg(&r.e->n);
      const long long ldc = __ldg(&r.e->ldc);
      __half *C = static_cast<__half *>(r.e->c);
      const int b = ci & 1;
      const uint32_t tph = (ci >> 1) & 1;
      if (!mbar_wait(&tfull[b], tph, p.err, ERR_TIMEOUT_EPILOGUE)) break;
      tc_fence_after();
      const int m = r.tm * BM + q * 32 + lane;
      const int n0 = r.tn * BN;
      const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * BN;
#pragma unroll 1
      for (int c = 0; c < BN; c += 32) {
        uint32_t v[32];
        tmem_ld_32x32b_x32(tbase + c, v);
        tmem_ld_wait();
        const int nvalid = pn - (n0 + c);
        if (m < pm && nvalid > 0) {
          __half *cp = C + (long long)m + (long long)(n0 + c) * ldc;
          float cv[32];
          if (p.beta_nonzero) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              cv[j] = (j < nvalid) ? __half2float(cp[(long long)j * ldc]) : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (j < nvalid) {
              float o = p.alpha * __uint_as_float(v[j]);
              if (p.beta_nonzero) o = fmaf(p.beta, cv[j], o);
              cp[(long long)j * ldc] = __float2half_rn(o);
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
    }
  }

  tc_fence_before();
  __syncwarp();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, TMEM_COLS);
  }
}

}  // namespace grouped
}  // namespace hcbk

extern "C" int hcbk_grouped_encode(hcbk_grouped_entry *e, int op_a, int op_b, int64_t m,
                                   int64_t n, int64_t k, const void *a, int64_t lda,
                                   const void *b, int64_t ldb, void *c, int64_t ldc) {
  if (m <= 0 || n <= 0 || k <= 0 || m > 0x7fffffff || n > 0x7fffffff || k > 0x7fffffff)
    return HCBK_ERR_ARGS;
  memset(e, 0, sizeof(*e));
  e->a_mn = op_a == HCBK_OP_N; /* op(A) = A: column-major M x K, M contiguous */
  e->b_mn = op_b != HCBK_OP_N; /* op(B) = B^T: N contiguous */
  int rc = e->a_mn ? hcbk_encode_tma_2d(e->map_a, 0, a, m, k, lda, 64, 64)
                   : hcbk_encode_tma_2d(e->map_a, 0, a, k, m, lda, 64, 128);
  if (rc) return rc;
  rc = e->b_mn ? hcbk_encode_tma_2d(e->map_b, 0, b, n, k, ldb, 64, 64)
               : hcbk_encode_tma_2d(e->map_b, 0, b, k, n, ldb, 64, 128);
  if (rc) return rc;
  e->c = c;
  e->ldc = ldc;
  e->m = (int32_t)m;
  e->n = (int32_t)n;
  e->k = (int32_t)k;
  e->tiles_m = (int32_t)((m + 127) / 128);
  return HCBK_OK;
}

extern "C" int hcbk_hgemm_grouped_tc(const hcbk_grouped_args *g, int *err, void *stream) {
  using namespace hcbk::grouped;
  if (g->count <= 0 || g->total_tiles <= 0) return HCBK_ERR_ARGS;
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(grouped_hgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SMEM_BYTES) != cudaSuccess)
      return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  Params p;
  p.table = g->table;
  p.tile_start = g->tile_start;
  p.count = g->count;
  p.total_tiles = g->total_tiles;
  p.alpha = g->alpha;
  p.beta = g->beta;
  p.beta_nonzero = g->beta != 0.0f;
  p.err = err;
  int grid = hcbk_sm_count();
  if (g->total_tiles < grid) grid = g->total_tiles;
  grouped_hgemm_kernel<<<grid, 192, SMEM_BYTES, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
