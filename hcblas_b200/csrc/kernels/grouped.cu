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
#include "split_bf16.cuh"
#include "tc_common.cuh"

namespace hcbk {
namespace grouped {

using namespace hcbk::tc;

constexpr int BM = 128, BN = 128, BK = 64; /* BK f16 = one 128-byte swizzle atom */
constexpr uint32_t A_BYTES = BM * 128, B_BYTES = BN * 128;
constexpr uint32_t STAGE_BYTES = A_BYTES + B_BYTES; /* stage slot sized for 128-wide tiles */
constexpr uint32_t OUT_BOX = 32 * 32 * 2;           /* one f16 32 x 32 C box */
constexpr uint32_t TMEM_COLS = 2 * BN;

/* Shared-memory layout of the grouped HGEMM for a ring of STG stages: the
 * stages, the epilogue's C boxes (4 warps x 2), the barriers.  MINB CTAs per
 * SM: one CTA with a 6-stage ring, or two with 3 stages each, whose tile
 * pipelines then hide each other's per-tile latencies. */
template <int STG, int MINB>
struct GCfg {
  static constexpr int STAGES = STG;
  static constexpr int NBOX = MINB == 1 ? 2 : 1; /* C boxes per epilogue warp */
  static constexpr uint32_t OUT_OFF = STG * STAGE_BYTES;
  static constexpr uint32_t BAR_OFF = OUT_OFF + 4 * NBOX * OUT_BOX;
  static constexpr uint32_t SMEM_BYTES = BAR_OFF + 256 + 1024;
  static_assert(SMEM_BYTES * MINB + 1024 * MINB <= 233472, "shared memory per SM");
  static_assert(TMEM_COLS * MINB <= 512, "TMEM per SM");
};

struct Params {
  const hcbk_grouped_entry *table;
  const int32_t *tile_start;
  const int4 *tile_desc; /* per tile: problem | flags << 24, tm, tn, k (host tables) */
  int count;
  int total_tiles;
  /* uniform batches (device-built tables): every problem has uniform_tiles
   * tiles of this shape; per-problem c_tma / skip come from the entries */
  int uniform_tiles, u_tiles_m, u_k, u_flags;
  float alpha, beta;
  int beta_nonzero;
  int device_maps; /* the table's maps were patched on the device: acquire them */
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
  int k;
  int flags; /* HCBK_GT_* */
};

/* One 16-byte load per tile (host tables) or arithmetic (uniform batches):
 * a binary search over the tile prefix sums costs a dozen dependent global
 * loads per tile and role, which dominated small tiles. */
__device__ __forceinline__ TileRef tile_ref(const Params &p, int t) {
  if (p.uniform_tiles > 0) {
    const int g = t / p.uniform_tiles, lt = t - g * p.uniform_tiles;
    const hcbk_grouped_entry *e = p.table + g;
    const int flags = p.u_flags | (__ldg(&e->c_tma) ? HCBK_GT_CTMA : 0) |
                      (__ldg(&e->skip) ? HCBK_GT_SKIP : 0);
    return TileRef{e, lt % p.u_tiles_m, lt / p.u_tiles_m, p.u_k, flags};
  }
  const int4 d = __ldg(p.tile_desc + t);
  return TileRef{p.table + (d.x & 0xffffff), d.y, d.z, d.w, (int)((unsigned)d.x >> 24)};
}

/* what the epilogue needs of a tile: its descriptor and the problem's C */
struct EpiRef {
  TileRef r;
  int m, n;
  long long ldc;
  void *c;
};

__device__ __forceinline__ EpiRef epi_ref(const Params &p, int t) {
  EpiRef x;
  x.r = tile_ref(p, t);
  x.m = __ldg(&x.r.e->m);
  x.n = __ldg(&x.r.e->n);
  x.ldc = __ldg(&x.r.e->ldc);
  x.c = x.r.e->c;
  return x;
}

/*
 * Per problem the tile is 128 x bn with bn = 64 or 128 (the entry's choice:
 * the width that pads N least), so narrow problems do not spend tensor work
 * on padding.  The epilogue stages each 32 x 32 block of C in shared memory
 * and writes it with one TMA tensor store through the problem's C map (C
 * read the same way when beta != 0); a C that TMA cannot address (base not
 * 16-byte aligned, ldc not a multiple of 8) is written by plain stores.  An
 * entry flagged `skip` (operands TMA cannot address, found by the
 * device-side table builder) is passed over by every role alike.
 */
template <int STG, int MINB>
__global__ void __launch_bounds__(192, MINB) grouped_hgemm_kernel(const __grid_constant__ Params p) {
  using Cfg = GCfg<STG, MINB>;
  constexpr int STAGES = Cfg::STAGES;
  constexpr int NBOX = Cfg::NBOX;
  constexpr uint32_t OUT_OFF = Cfg::OUT_OFF, BAR_OFF = Cfg::BAR_OFF;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + BAR_OFF);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint64_t *obar = tempty + 2; /* C loads: two per epilogue warp */
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(obar + 8);

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
    for (int b = 0; b < 8; ++b) mbar_init(&obar[b], 1);
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
      /* the next tile's descriptor is loaded while this tile's loads go out */
      TileRef nr = blockIdx.x < p.total_tiles ? tile_ref(p, blockIdx.x) : TileRef{};
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
        const TileRef r = nr;
        if (t + (int)gridDim.x < p.total_tiles) nr = tile_ref(p, t + gridDim.x);
        if (r.flags & HCBK_GT_SKIP) continue;
        const CUtensorMap *ma = reinterpret_cast<const CUtensorMap *>(r.e->map_a);
        const CUtensorMap *mb = reinterpret_cast<const CUtensorMap *>(r.e->map_b);
        if (p.device_maps) {
          tensormap_acquire(ma);
          tensormap_acquire(mb);
        }
        const int k = r.k;
        const int bn = (r.flags & HCBK_GT_BN64) ? 64 : 128;
        const int a_mn = r.flags & HCBK_GT_AMN, b_mn = r.flags & HCBK_GT_BMN;
        const int kblocks = (k + BK - 1) / BK;
        const uint32_t bytes = A_BYTES + (uint32_t)bn * 128u;
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], bytes);
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
            tma_load_2d(sb, mb, &full[s], k0, r.tn * bn); /* box {64, bn} */
          } else {
            for (int j = 0; j < bn; j += 64)
              tma_load_2d(sb + (j / 64) * (BK * 128), mb, &full[s], r.tn * bn + j, k0);
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
      int ci = 0; /* tiles computed by this CTA: selects the TMEM buffer */
      bool ok = true;
      TileRef nr = blockIdx.x < p.total_tiles ? tile_ref(p, blockIdx.x) : TileRef{};
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
        const TileRef r = nr;
        if (t + (int)gridDim.x < p.total_tiles) nr = tile_ref(p, t + gridDim.x);
        if (r.flags & HCBK_GT_SKIP) continue;
        const int k = r.k;
        const int bn = (r.flags & HCBK_GT_BN64) ? 64 : 128;
        const bool a_mn = (r.flags & HCBK_GT_AMN) != 0, b_mn = (r.flags & HCBK_GT_BMN) != 0;
        const int kblocks = (k + BK - 1) / BK;
        const uint32_t idesc = make_idesc(1, 0, a_mn, b_mn, BM, (uint32_t)bn);
        const uint32_t a_lbo = a_mn ? BK * 128 : 16, b_lbo = b_mn ? BK * 128 : 16;
        const uint32_t a_kstep = a_mn ? 16 * 128 : 32, b_kstep = b_mn ? 16 * 128 : 32;
        const int b = ci & 1;
        const uint32_t tph = (ci >> 1) & 1;
        ++ci;
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
    __half *boxes = reinterpret_cast<__half *>(smem + OUT_OFF) + q * NBOX * (32 * 32);
    uint64_t *wbar = obar + 2 * q;
    uint32_t lphase = 0; /* bit x: parity of box x's next C load */
    uint32_t pend = 0;   /* bit x: a C load into box x did not complete in time */
    int ci = 0;
    /* the next tile's descriptor and C geometry are loaded while this tile
     * waits for its accumulator */
    EpiRef nx = blockIdx.x < p.total_tiles ? epi_ref(p, blockIdx.x) : EpiRef{};
    for (int t = blockIdx.x; t < p.total_tiles; t += gridDim.x) {
      const EpiRef x0 = nx;
      if (t + (int)gridDim.x < p.total_tiles) nx = epi_ref(p, t + gridDim.x);
      const TileRef &r = x0.r;
      if (r.flags & HCBK_GT_SKIP) continue;
      const int pm = x0.m, pn = x0.n;
      const int bn = (r.flags & HCBK_GT_BN64) ? 64 : 128;
      const bool c_tma = (r.flags & HCBK_GT_CTMA) != 0;
      const CUtensorMap *mc = reinterpret_cast<const CUtensorMap *>(r.e->map_c);
      const long long ldc = x0.ldc;
      __half *C = static_cast<__half *>(x0.c);
      const int b = ci & 1;
      const uint32_t tph = (ci >> 1) & 1;
      ++ci;
      if (!mbar_wait(&tfull[b], tph, p.err, ERR_TIMEOUT_EPILOGUE)) break;
      tc_fence_after();
      if (c_tma && p.device_maps && lane == 0) tensormap_acquire(mc);
      const int m0 = r.tm * BM + q * 32;
      const int m = m0 + lane;
      const int n0 = r.tn * bn;
      const uint32_t tbase = tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * BN;
      bool wait_ok = true;
#pragma unroll 1
      for (int c = 0; c < bn; c += 32) {
        uint32_t v[32];
        tmem_ld_32x32b_x32(tbase + c, v);
        if (c_tma) {
          const int x = NBOX == 2 ? (c >> 5) & 1 : 0;
          __half *box = boxes + x * (32 * 32); /* column-major 32 x 32, as C */
          if (lane == 0) {
            /* the store issued from this box (NBOX groups ago) has read it */
            bulk_wait_read<NBOX - 1>();
            if (p.beta_nonzero) {
              mbar_expect_tx(&wbar[x], OUT_BOX);
              tma_load_2d(box, mc, &wbar[x], m0, n0 + c);
            }
          }
          __syncwarp();
          tmem_ld_wait();
          if (p.beta_nonzero) {
            /* the C box has landed (out-of-range parts read as zeros) */
            if (!__all_sync(0xffffffffu, mbar_wait(&wbar[x], (lphase >> x) & 1u, p.err,
                                                   ERR_TIMEOUT_EPILOGUE))) {
              pend |= 1u << x;
              wait_ok = false;
              break;
            }
            lphase ^= 1u << x;
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const float cv = __half2float(box[j * 32 + lane]);
              box[j * 32 + lane] = __float2half_rn(fmaf(p.beta, cv, p.alpha * __uint_as_float(v[j])));
            }
          } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              box[j * 32 + lane] = __float2half_rn(p.alpha * __uint_as_float(v[j]));
          }
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(mc, box, m0, n0 + c); /* rows >= m, columns >= n are dropped */
            bulk_commit();
          }
        } else {
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
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&tempty[b]);
      if (!wait_ok) break;
    }
    if (lane == 0) {
      /* a C load still in flight (only after a failed wait): a bounded time
       * to land before the CTA's shared memory is released */
      for (int x = 0; x < 2; ++x)
        if ((pend >> x) & 1u)
          for (int it = 0; it < (1 << 22) && !mbar_try_wait(&wbar[x], (lphase >> x) & 1u); ++it) {
          }
      bulk_wait_all(); /* this warp's tensor stores have completed */
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

/* Device-side table of a pointer-array batch (uniform problems): entry i is
 * the template with the global addresses of its A, B (and C) maps replaced
 * by a_arr[i] + a_off + i * a_stride (likewise B, C; byte offsets); an entry
 * whose A or B is not 16-byte aligned is flagged `skip` (the batch's
 * CUDA-core pass computes it), and one whose C is not is written by plain
 * stores.  tile_start[i] = i * tiles. */
struct PtrTableArgs {
  uint4 tmpl[sizeof(hcbk_grouped_entry) / 16]; /* the template entry's bytes */
  int tmpl_c_tma;
  hcbk_grouped_entry *table;
  int32_t *tile_start;
  int32_t *skip_out; /* per entry, for the CUDA-core pass (1 = compute there) */
  const void *const *a_arr;
  const void *const *b_arr;
  void *const *c_arr;
  int64_t a_off_bytes, b_off_bytes, c_off_bytes;
  int64_t a_stride_bytes, b_stride_bytes, c_stride_bytes;
  int count;
  int tiles;
};

__global__ void __launch_bounds__(128) grouped_ptr_table_kernel(const __grid_constant__ PtrTableArgs a) {
  /* one warp per entry: the lanes copy the template together, lane 0 then
   * patches the addresses */
  const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (i > a.count) return;
  if (lane == 0) a.tile_start[i] = i * a.tiles;
  if (i == a.count) return;
  hcbk_grouped_entry *e = a.table + i;
  uint4 *dst = reinterpret_cast<uint4 *>(e);
  for (int j = lane; j < (int)(sizeof(hcbk_grouped_entry) / 16); j += 32) dst[j] = a.tmpl[j];
  tensormap_release();
  __syncwarp(); /* the copies are ordered before lane 0's patches */
  if (lane != 0) return;
  const char *pa = static_cast<const char *>(a.a_arr[i]);
  const char *pb = static_cast<const char *>(a.b_arr[i]);
  char *pc = static_cast<char *>(a.c_arr[i]);
  pa = pa ? pa + a.a_off_bytes + (int64_t)i * a.a_stride_bytes : nullptr;
  pb = pb ? pb + a.b_off_bytes + (int64_t)i * a.b_stride_bytes : nullptr;
  pc = pc ? pc + a.c_off_bytes + (int64_t)i * a.c_stride_bytes : nullptr;
  const bool ok = pa && pb && pc && ((reinterpret_cast<uintptr_t>(pa) & 15) == 0) &&
                  ((reinterpret_cast<uintptr_t>(pb) & 15) == 0);
  const bool c_ok = ok && a.tmpl_c_tma && ((reinterpret_cast<uintptr_t>(pc) & 15) == 0);
  e->c = pc;
  e->skip = ok ? 0 : 1;
  e->c_tma = c_ok ? 1 : 0;
  a.skip_out[i] = ok ? 0 : 1;
  if (ok) {
    tensormap_replace_address(e->map_a, pa);
    tensormap_replace_address(e->map_b, pb);
    if (c_ok) tensormap_replace_address(e->map_c, pc);
  }
  tensormap_release();
}

/* ------------------------------------------------------------------------
 * Grouped split-BF16 SGEMM.  The host splits every problem's op(A) and op(B)
 * into K-major bf16 planes (grouped_pack_kernel, one launch for all
 * problems); each table entry then holds 3-D plane maps {K, rows, plane}.
 * The tile walk, roles and bounded waits are those of the HGEMM kernel
 * above; per 64-K slab the MMA warp issues the recipe's plane products into
 * NACC accumulators (RecipeBf16x3 / RecipeBf16x6), and the epilogue promotes
 * every slab's TMEM sums into f32 registers -- the tensor core's own f32
 * accumulation then never spans more than 64 K, which keeps the result's
 * error at or below plain FP32's -- and finally writes
 * alpha * acc + beta * C in f32.
 * ---------------------------------------------------------------------- */

template <class R, int ST>
struct SplitCfg {
  static constexpr int STAGES = ST;
  static constexpr uint32_t A_BYTES = BM * 128, B_BYTES = BN * 128;
  static constexpr uint32_t STAGE_BYTES = R::NA * A_BYTES + R::NB * B_BYTES;
  static constexpr uint32_t SMEM_BYTES = ST * STAGE_BYTES + 256 + 1024;
  static constexpr uint32_t ACC_COLS = R::NACC * BN;
  static constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;
  static_assert(SMEM_BYTES <= 232448, "shared memory");
  static_assert(TMEM_COLS <= 512, "TMEM");
};
using SplitCfg3 = SplitCfg<RecipeBf16x3, 3>;
using SplitCfg6 = SplitCfg<RecipeBf16x6, 2>;

template <class R, class Cfg>
__global__ void __launch_bounds__(192, 1) grouped_split_kernel(const __grid_constant__ Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  constexpr int S = Cfg::STAGES;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + S * Cfg::STAGE_BYTES);
  uint64_t *empty = full + S;
  uint64_t *tfull = empty + S;
  uint64_t *tempty = tfull + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
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
    tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
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
      TileRef nr = blockIdx.x < p.total_tiles ? tile_ref(p, blockIdx.x) : TileRef{};
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
        const TileRef r = nr;
        if (t + (int)gridDim.x < p.total_tiles) nr = tile_ref(p, t + gridDim.x);
        const CUtensorMap *ma = reinterpret_cast<const CUtensorMap *>(r.e->map_a);
        const CUtensorMap *mb = reinterpret_cast<const CUtensorMap *>(r.e->map_b);
        const int kblocks = (r.k + BK - 1) / BK;
        for (int kb = 0; kb < kblocks; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          mbar_expect_tx(&full[s], Cfg::STAGE_BYTES);
          uint8_t *st = smem + s * Cfg::STAGE_BYTES;
#pragma unroll
          for (int a = 0; a < R::NA; ++a)
            tma_load_3d(st + a * Cfg::A_BYTES, ma, &full[s], kb * BK, r.tm * BM, a);
#pragma unroll
          for (int b = 0; b < R::NB; ++b)
            tma_load_3d(st + R::NA * Cfg::A_BYTES + b * Cfg::B_BYTES, mb, &full[s], kb * BK,
                        r.tn * BN, b);
          if (++s == S) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
    }
  } else if (warp == 1) {
    /* ------------------------------------------------ MMA issuer -- */
    if (lane == 0) {
      const uint32_t idesc = make_idesc(1, 1, false, false, BM, BN); /* bf16 x bf16 -> f32 */
      int s = 0;
      uint32_t ph = 0;
      int ci = 0; /* 64-K slabs so far: selects the TMEM buffer */
      bool ok = true;
      TileRef nr = blockIdx.x < p.total_tiles ? tile_ref(p, blockIdx.x) : TileRef{};
      for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
        const TileRef r = nr;
        if (t + (int)gridDim.x < p.total_tiles) nr = tile_ref(p, t + gridDim.x);
        const int kblocks = (r.k + BK - 1) / BK;
        for (int kb = 0; ok && kb < kblocks; ++kb, ++ci) {
          const int b = ci & 1;
          if (!mbar_wait(&tempty[b], ((ci >> 1) & 1) ^ 1u, p.err, ERR_TIMEOUT_MMA_TMEM)) {
            ok = false;
            break;
          }
          tc_fence_after();
          if (!mbar_wait(&full[s], ph, p.err, ERR_TIMEOUT_MMA_FULL)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dbase = tmem_base + b * Cfg::ACC_COLS;
          const uint32_t sa = smem_u32(smem + s * Cfg::STAGE_BYTES);
          const uint32_t sb = sa + R::NA * Cfg::A_BYTES;
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
#pragma unroll
            for (int pi = 0; pi < R::NP; ++pi) {
              const uint64_t ad = smem_desc(sa + R::pa(pi) * Cfg::A_BYTES + kk * 32, 16, 1024, 2);
              const uint64_t bd = smem_desc(sb + R::pb(pi) * Cfg::B_BYTES + kk * 32, 16, 1024, 2);
              mma_f16(dbase + R::pacc(pi) * BN, ad, bd, idesc,
                      (kk > 0 || !R::first(pi)) ? 1u : 0u);
            }
          }
          mma_commit(&empty[s]);
          mma_commit(&tfull[b]);
          if (++s == S) {
            s = 0;
            ph ^= 1u;
          }
        }
      }
    }
  } else {
    /* ------------------------------------------------ epilogue -- */
    const int q = warp & 3; /* TMEM lane quadrant */
    int ci = 0;
    bool ok = true;
    EpiRef nx = blockIdx.x < p.total_tiles ? epi_ref(p, blockIdx.x) : EpiRef{};
    for (int t = blockIdx.x; ok && t < p.total_tiles; t += gridDim.x) {
      const EpiRef x0 = nx;
      if (t + (int)gridDim.x < p.total_tiles) nx = epi_ref(p, t + gridDim.x);
      const TileRef &r = x0.r;
      const int pm = x0.m, pn = x0.n;
      const int kblocks = (r.k + BK - 1) / BK;
      float acc[BN];
#pragma unroll
      for (int j = 0; j < BN; ++j) acc[j] = 0.f;
      for (int kb = 0; kb < kblocks; ++kb, ++ci) {
        const int b = ci & 1;
        if (!__all_sync(0xffffffffu,
                        mbar_wait(&tfull[b], (ci >> 1) & 1, p.err, ERR_TIMEOUT_EPILOGUE))) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tbase =
            tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * Cfg::ACC_COLS;
        /* this slab's products, correction accumulator first, added to acc
         * with IEEE round-to-nearest */
#pragma unroll
        for (int c = 0; c < BN; c += 32) {
          float part[32];
#pragma unroll
          for (int a = R::NACC - 1; a >= 0; --a) {
            uint32_t v[32];
            tmem_ld_32x32b_x32(tbase + a * BN + c, v);
            tmem_ld_wait();
#pragma unroll
            for (int j = 0; j < 32; ++j)
              part[j] = (a == R::NACC - 1) ? __uint_as_float(v[j]) : part[j] + __uint_as_float(v[j]);
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[c + j] += part[j];
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[b]);
      }
      if (!ok) break;
      const int m = r.tm * BM + q * 32 + lane;
      const int n0 = r.tn * BN;
      if (m < pm) {
        const long long ldc = x0.ldc;
        float *C = static_cast<float *>(x0.c) + (long long)m + (long long)n0 * ldc;
#pragma unroll
        for (int c = 0; c < BN; c += 32) {
          const int nvalid = pn - (n0 + c);
          if (nvalid <= 0) break;
          float *cp = C + (long long)c * ldc;
          float cv[32];
          if (p.beta_nonzero) {
#pragma unroll
            for (int j = 0; j < 32; ++j) cv[j] = (j < nvalid) ? cp[(long long)j * ldc] : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            if (j < nvalid) {
              float o = p.alpha * acc[c + j];
              if (p.beta_nonzero) o = fmaf(p.beta, cv[j], o);
              cp[(long long)j * ldc] = o;
            }
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncwarp();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
  }
}

/* One pack job's fields, read once per job (tiles of a job are consecutive). */
struct PackJob {
  const float *src;
  __nv_bfloat16 *planes;
  int64_t ld, pstride;
  int rows, kdim, ld_dst, tiles_r, k_contig;
};

__device__ __forceinline__ PackJob load_job(const hcbk_gpack_job *j) {
  PackJob o;
  o.src = j->src;
  o.planes = static_cast<__nv_bfloat16 *>(j->planes);
  o.ld = __ldg(&j->ld);
  o.pstride = __ldg(&j->plane_stride);
  o.rows = __ldg(&j->rows);
  o.kdim = __ldg(&j->kdim);
  o.ld_dst = __ldg(&j->ld_dst);
  o.tiles_r = __ldg(&j->tiles_r);
  o.k_contig = __ldg(&j->k_contig);
  return o;
}

/* this thread's eight source values of tile (r0, k0); the addresses step
 * by 8 rows (K-contiguous source) or 8 k (MN-contiguous) from one base */
__device__ __forceinline__ void pack_load(const PackJob &j, int r0, int k0, float (&v)[8]) {
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int64_t step = 8 * j.ld;
  if (j.k_contig) {
    const int ka = k0 + tx, kb = k0 + tx + 32;
    const bool oka = ka < j.kdim, okb = kb < j.kdim;
    const float *p = j.src + (int64_t)(r0 + ty) * j.ld;
#pragma unroll
    for (int q = 0; q < 4; ++q, p += step) {
      const bool rok = r0 + ty + 8 * q < j.rows;
      v[q] = (rok && oka) ? __ldg(p + ka) : 0.f;
      v[q + 4] = (rok && okb) ? __ldg(p + kb) : 0.f;
    }
  } else {
    const int r = r0 + tx;
    const bool rok = r < j.rows;
    const float *p = j.src + r + (int64_t)(k0 + ty) * j.ld;
#pragma unroll
    for (int i = 0; i < 8; ++i, p += step)
      v[i] = (rok && k0 + ty + 8 * i < j.kdim) ? __ldg(p) : 0.f;
  }
}

/* Split every job's f32 operand into nplanes K-major bf16 planes, one
 * 32 x 64 tile (rows x K) per iteration, read coalesced along whichever
 * dimension is contiguous in the source and written along K as bf16 pairs
 * (128 contiguous bytes per warp and plane).  Each block takes a contiguous
 * range of the tile sequence -- one binary search finds its first job, the
 * rest follow by stepping forward, and a job's fields are read once -- and
 * the next tile's loads are in flight while the current one is written. */
__global__ void __launch_bounds__(256) grouped_pack_kernel(const hcbk_gpack_job *jobs,
                                                           const int32_t *ts, int count,
                                                           int total, int nplanes) {
  __shared__ float tile[64][33]; /* [k][r] */
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
  const int t_begin = (int)((int64_t)total * blockIdx.x / gridDim.x);
  const int t_end = (int)((int64_t)total * (blockIdx.x + 1) / gridDim.x);
  if (t_begin >= t_end) return;
  int g = find_problem(ts, count, t_begin);
  int g_next = __ldg(ts + g + 1);
  PackJob nj = load_job(jobs + g);
  const int lt = t_begin - __ldg(ts + g); /* the one division: where the block starts */
  int nr0 = (lt % nj.tiles_r) * 32, nk0 = (lt / nj.tiles_r) * 64;
  float v[8];
  pack_load(nj, nr0, nk0, v);
  for (int t = t_begin; t < t_end; ++t) {
    const PackJob j = nj; /* the tile whose values are in v */
    const int r0 = nr0, k0 = nk0;
    __syncthreads(); /* the previous tile's reads of `tile` are done */
    if (j.k_contig) {
#pragma unroll
      for (int i = 0; i < 8; ++i) tile[tx + 32 * (i >> 2)][ty + 8 * (i & 3)] = v[i];
    } else {
#pragma unroll
      for (int i = 0; i < 8; ++i) tile[ty + 8 * i][tx] = v[i];
    }
    __syncthreads();
    if (t + 1 < t_end) { /* start the next tile's loads */
      if (t + 1 >= g_next) { /* the next job's first tile */
        while (t + 1 >= g_next) {
          ++g;
          g_next = __ldg(ts + g + 1);
        }
        nj = load_job(jobs + g);
        nr0 = 0;
        nk0 = 0;
      } else { /* the job's next tile: row tiles first, then K */
        nr0 += 32;
        if (nr0 >= nj.tiles_r * 32) {
          nr0 = 0;
          nk0 += 64;
        }
      }
      pack_load(nj, nr0, nk0, v);
    }
    /* this thread's row and 8 consecutive k: one 16-byte store per plane
     * (ld_dst is a multiple of 16 and every plane 1 KiB aligned); the row's
     * padding up to ld_dst is written too, as zeros, so that every sector is
     * written whole and L2 never fetches one to merge */
    {
      const int u = ty * 32 + tx;
      const int rl = u >> 3, kq = (u & 7) * 8;
      const int r = r0 + rl, k = k0 + kq;
      if (r < j.rows && k < j.ld_dst) {
        uint32_t w[4][3];
#pragma unroll
        for (int e = 0; e < 4; ++e)
          split_terms2(tile[kq + 2 * e][rl], tile[kq + 2 * e + 1][rl], w[e]);
        __nv_bfloat16 *d = j.planes + (int64_t)r * j.ld_dst + k;
#pragma unroll
        for (int pl = 0; pl < 3; ++pl) {
          if (pl >= nplanes) break;
          *reinterpret_cast<uint4 *>(d + pl * j.pstride) =
              make_uint4(w[0][pl], w[1][pl], w[2][pl], w[3][pl]);
        }
      }
    }
  }
}

/* Pointer-array batch on the grouped split-BF16 path: the plan's pack jobs
 * (2i: op(A) of problem i, 2i + 1: op(B)) and GEMM entries (i) take their
 * source and C pointers from the device-resident arrays, matrix i being
 * X[i] + x_off + i * x_stride (elements). */
__global__ void __launch_bounds__(128) grouped_split_patch_kernel(
    hcbk_gpack_job *jobs, hcbk_grouped_entry *table, const float *const *a_arr,
    const float *const *b_arr, float *const *c_arr, int64_t a_off, int64_t b_off, int64_t c_off,
    int64_t a_stride, int64_t b_stride, int64_t c_stride, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  jobs[2 * i].src = a_arr[i] + a_off + (int64_t)i * a_stride;
  jobs[2 * i + 1].src = b_arr[i] + b_off + (int64_t)i * b_stride;
  table[i].c = c_arr[i] + c_off + (int64_t)i * c_stride;
}

}  // namespace grouped
}  // namespace hcbk

extern "C" int hcbk_grouped_encode(hcbk_grouped_entry *e, int op_a, int op_b, int64_t m,
                                   int64_t n, int64_t k, const void *a, int64_t lda,
                                   const void *b, int64_t ldb, void *c, int64_t ldc) {
  if (m <= 0 || n <= 0 || k <= 0 || m > 0x7fffffff || n > 0x7fffffff || k > 0x7fffffff)
    return HCBK_ERR_ARGS;
  memset(e, 0, sizeof(*e));
  /* 64-wide tiles for problems no wider than 64 (half the tensor work of a
   * 128-wide tile for the same one tile); wider problems keep 128-wide tiles,
   * since more, narrower tiles re-read A once per tile column */
  e->bn = n <= 64 ? 64 : 128;
  e->a_mn = op_a == HCBK_OP_N; /* op(A) = A: column-major M x K, M contiguous */
  e->b_mn = op_b != HCBK_OP_N; /* op(B) = B^T: N contiguous */
  int rc = e->a_mn ? hcbk_encode_tma_2d(e->map_a, 0, a, m, k, lda, 64, 64)
                   : hcbk_encode_tma_2d(e->map_a, 0, a, k, m, lda, 64, 128);
  if (rc) return rc;
  rc = e->b_mn ? hcbk_encode_tma_2d(e->map_b, 0, b, n, k, ldb, 64, 64)
               : hcbk_encode_tma_2d(e->map_b, 0, b, k, n, ldb, 64, (uint32_t)e->bn);
  if (rc) return rc;
  /* C by tensor stores when TMA can address it */
  e->c_tma = hcbk_encode_out_2d(e->map_c, c, m, n, ldc) == HCBK_OK ? 1 : 0;
  e->c = c;
  e->ldc = ldc;
  e->m = (int32_t)m;
  e->n = (int32_t)n;
  e->k = (int32_t)k;
  e->tiles_m = (int32_t)((m + 127) / 128);
  return HCBK_OK;
}

extern "C" int hcbk_grouped_tiles(const hcbk_grouped_entry *e) {
  return e->tiles_m * (int)((e->n + e->bn - 1) / e->bn);
}

extern "C" int hcbk_grouped_tile_flags(const hcbk_grouped_entry *e) {
  return (e->bn == 64 ? HCBK_GT_BN64 : 0) | (e->a_mn ? HCBK_GT_AMN : 0) |
         (e->b_mn ? HCBK_GT_BMN : 0) | (e->c_tma ? HCBK_GT_CTMA : 0) |
         (e->skip ? HCBK_GT_SKIP : 0);
}

extern "C" void hcbk_grouped_fill_tiles(const hcbk_grouped_entry *e, int problem, int32_t *desc) {
  const int tiles = hcbk_grouped_tiles(e);
  const int flags = hcbk_grouped_tile_flags(e);
  for (int lt = 0; lt < tiles; ++lt) {
    int32_t *d = desc + 4 * lt;
    d[0] = (int32_t)((unsigned)problem | ((unsigned)flags << 24));
    d[1] = lt % e->tiles_m;
    d[2] = lt / e->tiles_m;
    d[3] = e->k;
  }
}

extern "C" int hcbk_grouped_ptr_table(const hcbk_grouped_entry *tmpl, hcbk_grouped_entry *table,
                                      int32_t *tile_start, int32_t *skip,
                                      const void *const *a_arr, const void *const *b_arr,
                                      void *const *c_arr, int64_t a_off_bytes,
                                      int64_t b_off_bytes, int64_t c_off_bytes,
                                      int64_t a_stride_bytes, int64_t b_stride_bytes,
                                      int64_t c_stride_bytes, int count, void *stream) {
  using namespace hcbk::grouped;
  if (count <= 0 || !a_arr || !b_arr || !c_arr ||
      (reinterpret_cast<uintptr_t>(table) & 127))
    return HCBK_ERR_ARGS;
  static_assert(sizeof(hcbk_grouped_entry) % 16 == 0, "entry size");
  PtrTableArgs a;
  memcpy(a.tmpl, tmpl, sizeof(hcbk_grouped_entry));
  a.tmpl_c_tma = tmpl->c_tma;
  a.table = table;
  a.tile_start = tile_start;
  a.skip_out = skip;
  a.a_arr = a_arr;
  a.b_arr = b_arr;
  a.c_arr = c_arr;
  a.a_off_bytes = a_off_bytes;
  a.b_off_bytes = b_off_bytes;
  a.c_off_bytes = c_off_bytes;
  a.a_stride_bytes = a_stride_bytes;
  a.b_stride_bytes = b_stride_bytes;
  a.c_stride_bytes = c_stride_bytes;
  a.count = count;
  a.tiles = hcbk_grouped_tiles(tmpl);
  const int threads = 128; /* four entries per block */
  const int blocks = (count + 1 + 3) / 4;
  grouped_ptr_table_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

namespace {
template <int STG, int MINB>
int launch_grouped_h(const hcbk_grouped_args *g, int *err, void *stream) {
  using namespace hcbk::grouped;
  using Cfg = GCfg<STG, MINB>;
  auto kern = grouped_hgemm_kernel<STG, MINB>;
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Cfg::SMEM_BYTES) != cudaSuccess)
      return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  Params p;
  p.table = g->table;
  p.tile_start = g->tile_start;
  p.tile_desc = reinterpret_cast<const int4 *>(g->tile_desc);
  p.count = g->count;
  p.total_tiles = g->total_tiles;
  p.uniform_tiles = g->uniform_tiles;
  p.u_tiles_m = g->u_tiles_m;
  p.u_k = g->u_k;
  p.u_flags = g->u_flags;
  p.alpha = g->alpha;
  p.beta = g->beta;
  p.beta_nonzero = g->beta != 0.0f;
  p.device_maps = g->device_maps;
  p.err = err;
  int grid = hcbk_sm_count() * MINB;
  if (g->total_tiles < grid) grid = g->total_tiles;
  kern<<<grid, 192, Cfg::SMEM_BYTES, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
}  // namespace

extern "C" int hcbk_hgemm_grouped_tc(const hcbk_grouped_args *g, int *err, void *stream) {
  if (g->count <= 0 || g->total_tiles <= 0) return HCBK_ERR_ARGS;
  if (g->ctas_per_sm == 2) return launch_grouped_h<3, 2>(g, err, stream);
  return launch_grouped_h<6, 1>(g, err, stream);
}

extern "C" int hcbk_grouped_pack(const hcbk_gpack_job *jobs, const int32_t *tile_start,
                                 int32_t count, int32_t total_tiles, int nplanes, void *stream) {
  using namespace hcbk::grouped;
  if (count <= 0 || total_tiles <= 0 || (nplanes != 2 && nplanes != 3)) return HCBK_ERR_ARGS;
  int grid = hcbk_sm_count() * 8;
  if (total_tiles < grid) grid = total_tiles;
  grouped_pack_kernel<<<grid, dim3(32, 8), 0, static_cast<cudaStream_t>(stream)>>>(
      jobs, tile_start, count, total_tiles, nplanes);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

namespace {
template <class R, class Cfg>
int launch_grouped_split(const hcbk_grouped_args *g, int *err, void *stream) {
  using namespace hcbk::grouped;
  auto kern = grouped_split_kernel<R, Cfg>;
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Cfg::SMEM_BYTES) != cudaSuccess)
      return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  Params p;
  p.table = g->table;
  p.tile_start = g->tile_start;
  p.tile_desc = reinterpret_cast<const int4 *>(g->tile_desc);
  p.count = g->count;
  p.total_tiles = g->total_tiles;
  p.uniform_tiles = 0;
  p.u_tiles_m = p.u_k = p.u_flags = 0;
  p.alpha = g->alpha;
  p.beta = g->beta;
  p.beta_nonzero = g->beta != 0.0f;
  p.device_maps = 0;
  p.err = err;
  int grid = hcbk_sm_count();
  if (g->total_tiles < grid) grid = g->total_tiles;
  kern<<<grid, 192, Cfg::SMEM_BYTES, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
}  // namespace

extern "C" int hcbk_sgemm_grouped_split_tc(const hcbk_grouped_args *g, int terms, int *err,
                                           void *stream) {
  using namespace hcbk::grouped;
  if (g->count <= 0 || g->total_tiles <= 0) return HCBK_ERR_ARGS;
  if (terms == 6) return launch_grouped_split<hcbk::tc::RecipeBf16x6, SplitCfg6>(g, err, stream);
  if (terms == 3) return launch_grouped_split<hcbk::tc::RecipeBf16x3, SplitCfg3>(g, err, stream);
  return HCBK_ERR_ARGS;
}

extern "C" int hcbk_grouped_split_patch(hcbk_gpack_job *jobs, hcbk_grouped_entry *table,
                                        const void *const *a_arr, const void *const *b_arr,
                                        void *const *c_arr, int64_t a_off, int64_t b_off,
                                        int64_t c_off, int64_t a_stride, int64_t b_stride,
                                        int64_t c_stride, int count, void *stream) {
  using namespace hcbk::grouped;
  if (count <= 0 || !a_arr || !b_arr || !c_arr) return HCBK_ERR_ARGS;
  const int threads = 128;
  grouped_split_patch_kernel<<<(count + threads - 1) / threads, threads, 0,
                               static_cast<cudaStream_t>(stream)>>>(
      jobs, table, reinterpret_cast<const float *const *>(a_arr),
      reinterpret_cast<const float *const *>(b_arr), reinterpret_cast<float *const *>(c_arr),
      a_off, b_off, c_off, a_stride, b_stride, c_stride, count);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
