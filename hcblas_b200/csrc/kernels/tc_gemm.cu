/*
 * tc_gemm.cu -- persistent tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
 *
 * One kernel family serves every tensor-core path of the library:
 *   HGEMM            f16 x f16 -> f32 accumulate in TMEM -> f16 C, operands
 *                    read straight from the caller's matrices by TMA (K-major
 *                    or MN-major: transposes live in the tensor maps and in
 *                    the descriptors' major bits, not in copy kernels);
 *   split-BF16 SGEMM f32 operands pre-split into bf16 planes (hi, lo[, lo2]);
 *                    3 (or 6) products per K-step into one f32 accumulator;
 *   (the "recipe" template describes which operand planes are multiplied
 *    into which accumulator, so emulated schemes reuse the same pipeline).
 *
 * CTA organisation (192 threads -- 320 with eight epilogue warps --, 1 CTA
 * per SM, persistent over output tiles):
 *   warp 0      TMA producer: one elected lane streams A/B K-slabs into a
 *               STAGES-deep shared-memory ring (full/empty mbarriers)
 *   warp 1      allocates TMEM; one lane issues tcgen05.mma for each K-slab
 *               and commits the slab back to the producer; accumulators are
 *               double-buffered in TMEM so the next tile's MMAs overlap the
 *               previous tile's epilogue
 *   warps 2..5  epilogue (2..9 with eight): tcgen05.ld (32 lanes x 32 columns) ->
 *               alpha*acc + beta*C in registers -> column-major C; each warp
 *               owns one 32-lane TMEM quadrant, so every store instruction
 *               writes 32 consecutive rows of one column (coalesced)
 * Tile: 128 x BN output, K-slab = 128 bytes of K per row (64 f16/bf16 or
 * 128 int8 elements), SWIZZLE_128B shared-memory layout shared by TMA and the
 * MMA descriptors.  No cluster multicast is used anywhere.
 */
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <type_traits>

#include "hcbk.h"
#include "tc_common.cuh"

namespace hcbk {
namespace tc {

constexpr int MAX_PLANES = 3;
constexpr int BM = 128;

struct TcParams {
  CUtensorMap ta[MAX_PLANES];
  CUtensorMap tb[MAX_PLANES];
  CUtensorMap tc; /* output map: int8 residue planes {rows, cols, plane} of the
                     modular epilogue, or f16 C {rows, cols} when out_tma is set */
  int m, n, k;
  int k0; /* first K coordinate (K split across launches) */
  int tiles_m, tiles_n;
  int a_mn, b_mn; /* operand is MN-major in global memory */
  void *c;
  long long ldc;
  float alpha, beta;
  int beta_nonzero;
  int out_tma; /* f16 epilogue: C read (beta != 0) and written by TMA via tc */
  int *err;
  /* failure-detection test: the producer arms the first stage's barrier
   * with its byte count but issues no load for it, so the MMA warp's wait
   * on that stage runs out (accepted only for one tile of one K block with
   * beta == 0, where nothing else is in flight) */
  int inject_skip_load;
  /* modular (CRT) epilogue: output plane i is reduced modulo
   * mod_tab[i % mod_period] (mod_period = moduli per GEMM; a batch of GEMMs
   * lays its elements' planes one after the other); planes of A, B (3-D
   * tensor maps) and C (c_plane_stride elements apart) are batched into one
   * launch */
  int nplanes;
  int mod_period;
  long long c_plane_stride;
  int mod_tab[HCBK_CRT_MAX_MODULI];
  float inv_mod_tab[HCBK_CRT_MAX_MODULI];
};

/* the modulus slot of a plane of a (batched) modular GEMM */
__device__ __forceinline__ int mod_slot(const TcParams &p, int plane) {
  return (p.mod_period <= 0 || plane < p.mod_period) ? plane : plane % p.mod_period;
}

/* ---------------------------------------------------------- recipes -- */

/* one plane pair per product: A plane PA[i] x B plane PB[i] -> accumulator
 * PACC[i]; FIRST[i] marks the first product written to its accumulator */
struct RecipeSingle {
  static constexpr int NA = 1, NB = 1, NP = 1, NACC = 1;
  static constexpr bool P3D = false; /* planes are separate 2-D tensor maps */
  __host__ __device__ static constexpr int pa(int) { return 0; }
  __host__ __device__ static constexpr int pb(int) { return 0; }
  __host__ __device__ static constexpr int pacc(int) { return 0; }
  __host__ __device__ static constexpr bool first(int i) { return i == 0; }
};
/* RecipeBf16x3 / RecipeBf16x6: tc_common.cuh (shared with the grouped kernel) */

/* ---------------------------------------------------------- epilogues -- */

__device__ __forceinline__ void store_out(float *p, float v) { *p = v; }
__device__ __forceinline__ void store_out(__half *p, float v) { *p = __float2half_rn(v); }
__device__ __forceinline__ float load_out(const float *p) { return *p; }
__device__ __forceinline__ float load_out(const __half *p) { return __half2float(*p); }

/* An epilogue warp's output staging: its two 32 x 32 boxes in shared memory,
 * the two mbarriers their C loads complete on, and the parity bit of each. */
struct OutStage {
  uint8_t *box;
  uint64_t *bar;
  uint32_t phase; /* bit x: parity of box x's next C load */
  uint32_t pend;  /* bit x: a C load into box x is in flight */
  int pre;        /* the current tile's first two C boxes are already loading */
};

/* f32 accumulator -> alpha*acc + beta*C in OutT (float or half) */
template <typename OutT> struct EpiAlphaBeta {
  static constexpr bool INPLACE = false;
  static constexpr bool PLANE_BATCH = false;
  /* output staging: per epilogue warp two 32 x 32 boxes of OutT in shared
   * memory (a kernel configuration whose stages leave no room for them runs
   * without: OutStage::box is then null and C is written by plain stores) */
  static constexpr uint32_t OUT_BOX_BYTES = 32 * 32 * sizeof(OutT);
  static constexpr uint32_t OUT_WARP_BYTES = 2 * OUT_BOX_BYTES;
  static constexpr uint32_t OUT_SMEM = 4 * OUT_WARP_BYTES;
  using AccT = float; /* register accumulator of the promoting path */

  /* One 32-column group c of this warp's 32 rows through box (c / 32) % 2:
   * values alpha * v (+ beta * C, C fetched by a TMA load that the previous
   * group started, or the tile's first group starts here) go to the box,
   * column-major as C, and leave by one TMA tensor store, which drops rows
   * >= m and columns >= n.  A box is rewritten only after the store issued
   * from it has read it.  load_v(r) fills r with the group's 32 f32 values
   * (bit patterns); it may start an asynchronous fetch that wait_v() ends. */
  /* Start the C loads of a tile's first two 32-column groups (beta != 0),
   * before the tile's accumulator is ready, so that they overlap its MMAs. */
  template <int BN>
  static __device__ __forceinline__ void prefetch_c(const TcParams &p, int m0, int n0,
                                                    OutStage &os) {
    if (!os.box || !p.out_tma || !p.beta_nonzero || os.pre) return;
    if ((threadIdx.x & 31) == 0) {
      bulk_wait_read<0>(); /* the previous tile's stores have read both boxes */
#pragma unroll
      for (int x = 0; x < 2; ++x)
        if (x * 32 < BN) {
          mbar_expect_tx(&os.bar[x], OUT_BOX_BYTES);
          tma_load_2d(os.box + x * OUT_BOX_BYTES, &p.tc, &os.bar[x], m0, n0 + 32 * x);
        }
    }
    os.pend |= BN > 32 ? 3u : 1u;
    os.pre = 1;
    __syncwarp();
  }

  template <int BN, class LoadV, class WaitV>
  static __device__ __forceinline__ void stage_group(const TcParams &p, int c, int m0, int n0,
                                                     OutStage &os, LoadV &&load_v,
                                                     WaitV &&wait_v) {
    const int lane = threadIdx.x & 31;
    const bool ld_c = p.beta_nonzero != 0;
    const int b = (c >> 5) & 1;
    OutT *box = reinterpret_cast<OutT *>(os.box + b * OUT_BOX_BYTES);
    uint32_t r[32];
    load_v(r);
    const bool load_first = ld_c && c == 0 && !os.pre;
    const bool load_next = ld_c && c + 32 < BN && !(os.pre && c == 0);
    if (lane == 0) {
      if (!ld_c) bulk_wait_read<1>(); /* the store from this box two groups ago */
      if (load_first) { /* the tile's first group was not prefetched */
        bulk_wait_read<0>();
        mbar_expect_tx(&os.bar[0], OUT_BOX_BYTES);
        tma_load_2d(os.box, &p.tc, &os.bar[0], m0, n0);
      }
      if (load_next) { /* the next group's C into the other box */
        bulk_wait_read<0>(); /* that box's store has read it */
        mbar_expect_tx(&os.bar[b ^ 1], OUT_BOX_BYTES);
        tma_load_2d(os.box + (b ^ 1) * OUT_BOX_BYTES, &p.tc, &os.bar[b ^ 1], m0, n0 + c + 32);
      }
    }
    if (load_first) os.pend |= 1u;
    if (load_next) os.pend |= 1u << (b ^ 1);
    __syncwarp();
    wait_v();
    if (ld_c) {
      mbar_wait(&os.bar[b], (os.phase >> b) & 1u, p.err, ERR_TIMEOUT_EPILOGUE);
      os.phase ^= 1u << b;
      os.pend &= ~(1u << b);
#pragma unroll
      for (int j = 0; j < 32; ++j)
        store_out(box + j * 32 + lane,
                  fmaf(p.beta, load_out(box + j * 32 + lane), p.alpha * __uint_as_float(r[j])));
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) store_out(box + j * 32 + lane, p.alpha * __uint_as_float(r[j]));
    }
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0) {
      tma_store_2d(&p.tc, box, m0, n0 + c);
      bulk_commit();
    }
  }

  /* the TMEM accumulator of one tile through the staged path */
  template <int BN>
  static __device__ __forceinline__ void run_tma(const TcParams &p, uint32_t tbase, int m0,
                                                 int n0, OutStage &os) {
#pragma unroll 1
    for (int c = 0; c < BN; c += 32)
      stage_group<BN>(
          p, c, m0, n0, os, [&](uint32_t(&r)[32]) { tmem_ld_32x32b_x32(tbase + c, r); },
          [] { tmem_ld_wait(); });
    os.pre = 0;
  }

  template <int BN, int NACC>
  static __device__ __forceinline__ void run(const TcParams &p, uint32_t tbase, int m, int n0,
                                             OutStage &os) {
    static_assert(NACC == 1, "several accumulators need the promoting epilogue");
    if (os.box && p.out_tma) {
      run_tma<BN>(p, tbase, m - (int)(threadIdx.x & 31), n0, os);
      return;
    }
    const bool row_ok = m < p.m;
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      uint32_t r[32];
      tmem_ld_32x32b_x32(tbase + c, r);
      tmem_ld_wait();
      if (row_ok) {
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
        store32(p, v, m, n0 + c);
      }
    }
  }

  /* Configurations without output staging read C with plain loads in the
   * tile's final store, one 32-column group at a time, each group a full
   * DRAM latency.  At the start of a tile (its MMAs still running) every
   * epilogue thread asks L2 for its row of the tile's C, so that those loads
   * hit L2 instead. */
  static constexpr bool L2_PREFETCH_C = true;
  template <int BN>
  static __device__ __forceinline__ void prefetch_c_l2(const TcParams &p, int m, int n0) {
    if (!p.beta_nonzero || m >= p.m) return;
    const OutT *C = static_cast<const OutT *>(p.c) + (long long)m + (long long)n0 * p.ldc;
    const int nvalid = p.n - n0 < BN ? p.n - n0 : BN;
#pragma unroll 4
    for (int j = 0; j < nvalid; ++j)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(C + (long long)j * p.ldc));
  }

  /* C[m, n0 .. n0+31] = alpha * v + beta * C: all C loads are issued before
   * the first store, so they overlap instead of serialising behind stores
   * that might alias them. */
  static __device__ __forceinline__ void store32(const TcParams &p, const float (&v)[32], int m,
                                                 int n0) {
    OutT *C = static_cast<OutT *>(p.c) + (long long)m + (long long)n0 * p.ldc;
    const int nvalid = p.n - n0;
    float cv[32];
    if (p.beta_nonzero) {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        cv[j] = (j < nvalid) ? load_out(C + (long long)j * p.ldc) : 0.f;
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      if (j < nvalid) {
        float o = p.alpha * v[j];
        if (p.beta_nonzero) o = fmaf(p.beta, cv[j], o);
        store_out(C + (long long)j * p.ldc, o);
      }
    }
  }

  /* acc[j] += sum over accumulators a (highest index first) of TMEM column
   * a*BN + j of this thread's lane, with IEEE round-to-nearest adds: the
   * promotion step of the chunked accumulation */
  template <int BN, int NACC>
  static __device__ __forceinline__ void accumulate(const TcParams &, uint32_t tbase,
                                                    float (&acc)[BN], int /* chunk */) {
#pragma unroll
    for (int c = 0; c < BN; c += 32) {
      float part[32];
#pragma unroll
      for (int a = NACC - 1; a >= 0; --a) {
        uint32_t r[32];
        tmem_ld_32x32b_x32(tbase + a * BN + c, r);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 32; ++j)
          part[j] = (a == NACC - 1) ? __uint_as_float(r[j]) : part[j] + __uint_as_float(r[j]);
      }
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[c + j] += part[j];
    }
  }

  template <int BN>
  static __device__ __forceinline__ void store_acc(const TcParams &p, const float (&acc)[BN],
                                                   int m, int n0, OutStage &os) {
    if (os.box && p.out_tma) { /* every lane takes part: rows >= m are dropped by the store */
      const int m0 = m - (int)(threadIdx.x & 31);
#pragma unroll
      for (int c = 0; c < BN; c += 32)
        stage_group<BN>(
            p, c, m0, n0, os,
            [&](uint32_t(&r)[32]) {
#pragma unroll
              for (int j = 0; j < 32; ++j) r[j] = __float_as_uint(acc[c + j]);
            },
            [] {});
      os.pre = 0;
      return;
    }
    if (m >= p.m) return;
#pragma unroll
    for (int c = 0; c < BN; c += 32) {
      if (n0 + c >= p.n) break;
      float v[32];
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = acc[c + j];
      store32(p, v, m, n0 + c);
    }
  }
};

/* Modular epilogue of the CRT scheme, reducing in place in TMEM.
 * With f16 residues |r| <= 127 (moduli <= 255) the tensor core's f32 sums
 * are exact integers while below 2^24: 1024 * 127^2 + 1.5 * 255 < 2^24.
 * The kernel therefore lets a TMEM accumulator grow over one 1024-element
 * K chunk, and the epilogue warps then reduce it modulo p where it lies
 * (tcgen05.ld -> q = rint(s / p) by the 1.5 * 2^23 rounding constant,
 * r = fma(-q, p, s), exact because r is a small integer -> tcgen05.st),
 * after which the MMAs keep accumulating on top of the reduced value.
 * Chunks alternate between the two TMEM buffers, so one buffer is reduced
 * while the tensor core fills the other; the last two chunks of a tile are
 * combined, reduced, and stored as symmetric int8 residues (C viewed as
 * the column-major int8 residue plane).  No register accumulator, no
 * float->int conversion before the final store. */
struct EpiModP {
  static constexpr bool INPLACE = true;
  static constexpr bool PLANE_BATCH = true; /* one tile walk over every modulus */
  static constexpr float RND = 12582912.0f; /* 1.5 * 2^23 */

  /* exact x mod p into (-p, p) for integral |x| < 2^24 */
  static __device__ __forceinline__ float mod_f(float x, float p, float inv_p) {
    const float q = fmaf(x, inv_p, RND) - RND;
    return fmaf(-q, p, x);
  }

  template <int BN, int NACC>
  static __device__ __forceinline__ void run(const TcParams &, uint32_t, int, int, OutStage &) {
    static_assert(NACC == 0, "the modular epilogue only runs on the in-place path");
  }

  /* reduce this warp's 32 lanes x BN columns of one buffer in place */
  template <int BN>
  static __device__ __forceinline__ void rmw(const TcParams &p, uint32_t tbase, int plane) {
    const int slot = mod_slot(p, plane);
    const float pf = static_cast<float>(p.mod_tab[slot]);
    const float inv = p.inv_mod_tab[slot];
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      uint32_t r[32];
      tmem_ld_32x32b_x32(tbase + c, r);
      tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < 32; ++j)
        r[j] = __float_as_uint(mod_f(__uint_as_float(r[j]), pf, inv));
      tmem_st_32x32b_x32(tbase + c, r);
    }
    tmem_st_wait();
  }

  /* output staging: per epilogue warp two 32 x 32 int8 boxes (1 KB each) */
  static constexpr uint32_t OUT_BOX_BYTES = 32 * 32; /* int8 residues */
  static constexpr uint32_t OUT_WARP_BYTES = 2 * OUT_BOX_BYTES;
  static constexpr uint32_t OUT_SMEM = 4 * OUT_WARP_BYTES;

  /* T[m0 + lane, n0 + c + j] = symmetric buffer mod p, for this warp's 32
   * rows: each 32-column group is written to one of the warp's two
   * shared-memory boxes (column-major int8, as the plane) and stored by one
   * TMA tensor store, which also drops rows >= m and columns >= n; a box is
   * rewritten only after the store issued from it two groups earlier has
   * read it.  `out` is this warp's OUT_WARP_BYTES of shared memory. */
  template <int BN>
  static __device__ __forceinline__ void final_store(const TcParams &p, uint32_t ta, uint8_t *out,
                                                     int m0, int n0, int plane) {
    const int lane = threadIdx.x & 31;
    const int slot = mod_slot(p, plane);
    const int mod = p.mod_tab[slot];
    const float pf = static_cast<float>(mod);
    const float inv = p.inv_mod_tab[slot];
    const float hp = static_cast<float>((mod - 1) >> 1);
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      int8_t *box = reinterpret_cast<int8_t *>(out + ((c >> 5) & 1) * OUT_BOX_BYTES);
      uint32_t ra[32];
      tmem_ld_32x32b_x32(ta + c, ra);
      if (lane == 0) bulk_wait_read<1>(); /* the store from this box two groups ago */
      __syncwarp();
      tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        /* an exact integer below 2^24 in magnitude, reduced to [-(p-1)/2, (p-1)/2] */
        float v = mod_f(__uint_as_float(ra[j]), pf, inv);
        if (v > hp) v -= pf;
        else if (v < -hp) v += pf;
        /* low 8 bits of the 1.5 * 2^23 + v pattern: v as int8 (|v| <= 127) */
        box[j * 32 + lane] = static_cast<int8_t>(__float_as_int(v + RND));
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        tma_store_3d(&p.tc, box, m0, n0 + c, plane);
        bulk_commit();
      }
    }
  }
};

/* Ozaki-I slice-group epilogue (concatenated-K mode, see CatK): the tile's
 * INT32 group sum D_d goes out unchanged, through per-warp shared-memory
 * boxes (32 x 32 int32, column-major) and TMA tensor stores into plane d of
 * the int32 output {rows, cols, group}; the FP64 weighting, exponent scaling
 * and alpha / beta happen in a separate element-wise pass. */
struct EpiI32Cat {
  static constexpr bool INPLACE = false;
  static constexpr bool PLANE_BATCH = true;
  static constexpr bool CAT_K = true;
  static constexpr uint32_t OUT_BOX_BYTES = 32 * 32 * 4;
  static constexpr uint32_t OUT_WARP_BYTES = 2 * OUT_BOX_BYTES;
  static constexpr uint32_t OUT_SMEM = 4 * OUT_WARP_BYTES;

  template <int BN>
  static __device__ __forceinline__ void prefetch_c(const TcParams &, int, int, OutStage &) {}

  template <int BN, int NACC>
  static __device__ __forceinline__ void run(const TcParams &, uint32_t, int, int, OutStage &) {
    static_assert(NACC == 0, "the slice-group epilogue stores through final_store");
  }

  /* `plane` is the walk's plane index; the group it holds is nplanes - 1 - plane */
  template <int BN>
  static __device__ __forceinline__ void final_store(const TcParams &p, uint32_t ta, uint8_t *out,
                                                     int m0, int n0, int plane) {
    const int lane = threadIdx.x & 31;
    const int d = p.nplanes - 1 - plane;
#pragma unroll 1
    for (int c = 0; c < BN; c += 32) {
      uint32_t *box = reinterpret_cast<uint32_t *>(out + ((c >> 5) & 1) * OUT_BOX_BYTES);
      uint32_t ra[32];
      tmem_ld_32x32b_x32(ta + c, ra);
      if (lane == 0) bulk_wait_read<1>(); /* the store from this box two groups ago */
      __syncwarp();
      tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < 32; ++j) box[j * 32 + lane] = ra[j];
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        tma_store_3d(&p.tc, box, m0, n0 + c, d);
        bulk_commit();
      }
    }
  }
};

/* Concatenated-K mode of an epilogue (CAT_K): the walk's plane index q
 * stands for the group d = nplanes - 1 - q (largest first) and the tile's K
 * loop runs over (d + 1) * kblocks slabs, slab j reading A plane j / kblocks
 * and B plane d - j / kblocks: D_d = sum_{i <= d} A_i B_(d-i)^T in one
 * accumulator. */
template <class E, class = void> struct CatK : std::false_type {};
/* epilogue warps (EPI_WARPS, default 4): with 8, two warps share each TMEM
 * lane quadrant and take half of the tile's columns each (plane-batched
 * TMA-store epilogues only) */
template <class E, class = void> struct EpiWarps {
  static constexpr int value = 4;
};
template <class E> struct EpiWarps<E, std::void_t<decltype(E::EPI_WARPS)>> {
  static constexpr int value = E::EPI_WARPS;
};
template <class E> struct CatK<E, std::void_t<decltype(E::CAT_K)>> : std::bool_constant<E::CAT_K> {};
/* epilogues whose final store reads C with plain loads and can ask L2 for
 * it ahead of time (L2_PREFETCH_C, default none) */
template <class E, class = void> struct EpiL2Prefetch : std::false_type {};
template <class E>
struct EpiL2Prefetch<E, std::void_t<decltype(E::L2_PREFETCH_C)>>
    : std::bool_constant<E::L2_PREFETCH_C> {};

/* Modular epilogue of the int8 path: the INT32 accumulator holds the
 * exact sum over all of K (|s| <= K 127^2 <= 2114125824 for K <= 131072),
 * reduced once per tile: s = hi 2^16 + lo with hi = (s + 2^15) >> 16 and
 * |lo| <= 2^15 gives y = hi (2^16 mod p) + lo, exact in int32 with
 * |y| <= 32259 * 127 + 2^15 < 2^22, so RND + y (RND = 1.5 * 2^23) is the f32
 * with bit pattern 0x4B400000 + y.  Since |y / p| < 25200 the f32 quotient
 * y * RN(1/p) is within 1.6e-3 of y / p, below the 1/(2p) >= 1.96e-3 that
 * separates y / p (p odd) from any half-integer: q = rint(y / p) exactly,
 * and RND + y - q p = RND + r with r already in [-(p-1)/2, (p-1)/2], whose
 * low 8 bits are r as an int8 (|r| <= 127).  Eight epilogue warps (two per TMEM lane
 * quadrant, half of the columns each) read TMEM 64 columns at a time (one
 * wait per 64) into two 32 x 32 int8 shared-memory boxes per warp, each
 * written by one TMA tensor store. */
struct EpiModPi8 {
  static constexpr bool INPLACE = false;
  static constexpr bool PLANE_BATCH = true;
  static constexpr float RND = 12582912.0f; /* 1.5 * 2^23 */
  static constexpr int EPI_WARPS = 8;
  static constexpr uint32_t OUT_BOX_BYTES = 32 * 32; /* int8 residues */
  static constexpr uint32_t OUT_WARP_BYTES = 2 * OUT_BOX_BYTES;
  static constexpr uint32_t OUT_SMEM = EPI_WARPS * OUT_WARP_BYTES;

  template <int BN>
  static __device__ __forceinline__ void prefetch_c(const TcParams &, int, int, OutStage &) {}

  template <int BN, int NACC>
  static __device__ __forceinline__ void run(const TcParams &, uint32_t, int, int, OutStage &) {
    static_assert(NACC == 0, "the modular epilogue stores through final_store");
  }

  /* the symmetric residue of s as an int8 (see above; |r| <= 127) */
  static __device__ __forceinline__ int8_t residue(uint32_t s, int c16, float pf, float inv) {
    const int sv = static_cast<int>(s);
    const int hi = (sv + 0x8000) >> 16;
    const int y = hi * c16 + (sv - hi * 65536);
    const float yr = __int_as_float(0x4B400000 + y); /* RND + y */
    const float q = fmaf(yr - RND, inv, RND) - RND;
    return static_cast<int8_t>(__float_as_int(fmaf(-q, pf, yr)));
  }

  template <int BN>
  static __device__ __forceinline__ void final_store(const TcParams &p, uint32_t ta, uint8_t *out,
                                                     int m0, int n0, int plane) {
    static_assert(BN % 64 == 0, "64 columns per TMEM wait");
    const int lane = threadIdx.x & 31;
    const int slot = mod_slot(p, plane);
    const int mod = p.mod_tab[slot];
    const float pf = static_cast<float>(mod);
    const float inv = p.inv_mod_tab[slot];
    int c16 = (1 << 16) % mod; /* 2^16 mod p, symmetric */
    if (c16 > (mod - 1) / 2) c16 -= mod;
#pragma unroll 1
    for (int c = 0; c < BN; c += 64) {
      int8_t *box = reinterpret_cast<int8_t *>(out);
      uint32_t ra[32], rb[32];
      tmem_ld_32x32b_x32(ta + c, ra);
      tmem_ld_32x32b_x32(ta + c + 32, rb);
      if (lane == 0) bulk_wait_read<0>(); /* the last two stores have read the boxes */
      __syncwarp();
      tmem_ld_wait();
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        box[j * 32 + lane] = residue(ra[j], c16, pf, inv);
        box[1024 + j * 32 + lane] = residue(rb[j], c16, pf, inv);
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) {
        tma_store_3d(&p.tc, box, m0, n0 + c, plane);
        bulk_commit();
        tma_store_3d(&p.tc, box + 1024, m0, n0 + c + 32, plane);
        bulk_commit();
      }
    }
  }
};


/* ------------------------------------------------------------- kernel -- */

/* per operand kind: K bytes per tile row (one swizzle atom), elements per
 * K-slab, K per MMA instruction, accumulator / operand formats, swizzle */
template <int KIND> struct KindTraits;
template <> struct KindTraits<0> { /* f16, 128-byte swizzle */
  static constexpr int ROWB = 128, BKE = 64, UK = 16, ESZ = 2;
  static constexpr uint32_t CFMT = 1, ABFMT = 0, LAYOUT = 2, SBO = 1024;
};
template <> struct KindTraits<1> { /* bf16, 128-byte swizzle */
  static constexpr int ROWB = 128, BKE = 64, UK = 16, ESZ = 2;
  static constexpr uint32_t CFMT = 1, ABFMT = 1, LAYOUT = 2, SBO = 1024;
};
template <> struct KindTraits<3> { /* s8 -> s32, 128-byte swizzle: 128 K per slab */
  static constexpr int ROWB = 128, BKE = 128, UK = 32, ESZ = 1;
  static constexpr uint32_t CFMT = 2, ABFMT = 1, LAYOUT = 2, SBO = 1024;
};

__host__ __device__ constexpr uint32_t tmem_cols_for(uint32_t c) {
  return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512;
}

/* NBUF: TMEM accumulator sets (2 = the epilogue of one tile/chunk overlaps
 * the MMAs of the next; 1 when the accumulators fill TMEM).
 * CG: CTAs per MMA (1, or 2 for a CTA pair computing a 256 x BN tile; each
 * CTA of a pair holds 128 rows of A and BN/2 rows of B per stage). */
template <int BN, int STAGES, class R, int KIND, int NBUF = 2, int CG = 1, uint32_t OUT = 0>
struct TcCfg {
  using KT = KindTraits<KIND>;
  static constexpr uint32_t A_PLANE = BM * KT::ROWB;
  static constexpr uint32_t B_ROWS = BN / CG;
  static constexpr uint32_t B_PLANE = B_ROWS * KT::ROWB;
  static constexpr uint32_t STAGE_BYTES = R::NA * A_PLANE + R::NB * B_PLANE;
  static constexpr uint32_t ACC_COLS = R::NACC * BN;
  static constexpr uint32_t TMEM_COLS = tmem_cols_for(NBUF * ACC_COLS);
  static constexpr uint32_t BAR_BYTES = 256;
  /* epilogue output staging (OUT bytes wanted) after the barriers,
   * 1024-aligned, when the stages leave room for it */
  static constexpr uint32_t OUT_OFF = STAGES * STAGE_BYTES + 1024;
  static constexpr uint32_t OUT_BYTES = OUT_OFF + OUT + 1024 <= 232448 ? OUT : 0;
  static constexpr uint32_t SMEM_BYTES =
      (OUT_BYTES ? OUT_OFF + OUT_BYTES : STAGES * STAGE_BYTES + BAR_BYTES) + 1024;
  static_assert(NBUF * ACC_COLS <= 512, "accumulators exceed TMEM");
  static_assert(BN % 64 == 0 && BN >= 64 && BN <= 256, "BN");
  static_assert(CG == 1 || (CG == 2 && !R::P3D && BN % 128 == 0), "CTA pair");
  static_assert(SMEM_BYTES <= 232448, "shared memory");
};

/*
 * PROMOTE_KB = 0: each tile accumulates over all of K in TMEM (double-
 *   buffered per tile) and the epilogue converts once.
 * PROMOTE_KB = n > 0: the tile's K range is cut into chunks of n K-slabs;
 *   every chunk starts a fresh TMEM accumulator (double-buffered per chunk)
 *   and the epilogue warps add it into an f32 register accumulator with
 *   IEEE round-to-nearest.  The tensor core's own f32 accumulation then
 *   spans only n*128 bytes of K, which bounds the error it adds; used by the
 *   split-BF16 paths, whose contract is "error no worse than FP32".
 */
/* The work sequence every role of a CTA walks, as (tile, chunk, slot)
 * items.  Normally a CTA's tiles come one after the other, chunk by chunk.
 * In the in-place modular mode its tiles go in pairs whose chunks alternate
 * -- (X,0) (Y,0) (X,1) (Y,1) ... -- with X in TMEM buffer 0 and Y in buffer 1,
 * so that while the epilogue reduces (or finally stores) one tile's buffer
 * the tensor core fills the other's; an unpaired last tile uses buffer 0. */
struct WorkItem {
  int t, c, slot;
};

__device__ __forceinline__ WorkItem work_item(int i, int tile0, int step, int ntiles_local,
                                              int nchunks, bool pairs) {
  if (pairs) {
    const int full = (ntiles_local >> 1) * 2 * nchunks;
    if (i < full) {
      const int pr = i / (2 * nchunks), r = i - pr * 2 * nchunks;
      const int slot = r & 1;
      return WorkItem{tile0 + (2 * pr + slot) * step, r >> 1, slot};
    }
    return WorkItem{tile0 + (ntiles_local - 1) * step, i - full, 0};
  }
  const int lt = i / nchunks;
  return WorkItem{tile0 + lt * step, i - lt * nchunks, 0};
}

/* Tile order within a plane: bands of TILE_GROUP tile rows, walked column
 * by column and down each column inside the band, so that the tiles running
 * at the same time (one per SM or SM pair) cover about TILE_GROUP row tiles
 * by (concurrent / TILE_GROUP) column tiles; their A and B panels then stay
 * in L2 where a column-major walk over all tile rows streams the whole of A
 * from DRAM once per wave. */
constexpr int TILE_GROUP = 8;
struct TileMN {
  int m, n;
};
__device__ __forceinline__ TileMN tile_mn(int t, int tiles_m, int tiles_n) {
  const int band = t / (TILE_GROUP * tiles_n);
  const int first = band * TILE_GROUP;
  const int rows = tiles_m - first < TILE_GROUP ? tiles_m - first : TILE_GROUP;
  const int r = t - band * TILE_GROUP * tiles_n;
  return TileMN{first + r % rows, r / rows};
}

template <int BN, int STAGES, class R, int KIND, class EPI, int PROMOTE_KB = 0, int NBUF = 2,
          int CG = 1>
__global__ void __launch_bounds__(64 + 32 * EpiWarps<EPI>::value, 1)
    tc_gemm_kernel(const __grid_constant__ TcParams p) {
  using Cfg = TcCfg<BN, STAGES, R, KIND, NBUF, CG, EPI::OUT_SMEM>;
  using KT = typename Cfg::KT;
  constexpr int BKE = KT::BKE;
  constexpr int ROWB = KT::ROWB;
  constexpr int KSTEPS = BKE / KT::UK;

  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = reinterpret_cast<uint8_t *>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * Cfg::STAGE_BYTES);
  uint64_t *empty = full + STAGES;
  uint64_t *tfull = empty + STAGES;
  uint64_t *tempty = tfull + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(tempty + 2);
  uint64_t *obar = tempty + 4; /* output staging: two C-load barriers per epilogue warp */
  constexpr int EW = EpiWarps<EPI>::value;
  static_assert(EW == 4 || (EW == 8 && EPI::PLANE_BATCH && !EPI::INPLACE && BN % 128 == 0),
                "eight epilogue warps: plane-batched TMA-store epilogues");

  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  /* CTA pair: rank 0 (the leader) issues the MMAs and owns the full and
   * TMEM-empty barriers both CTAs' producers and epilogues signal */
  const uint32_t rank = CG == 2 ? cluster_ctarank() : 0u;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], EW * CG);
    }
    if constexpr (Cfg::OUT_BYTES > 0)
      for (int b = 0; b < 2 * EW; ++b) mbar_init(&obar[b], 1);
    mbar_fence_init();
  }
  if (warp == 0 && lane == 0) {
    constexpr int NMA = R::P3D ? 1 : R::NA, NMB = R::P3D ? 1 : R::NB;
    for (int i = 0; i < NMA; ++i) tma_prefetch_desc(&p.ta[i]);
    for (int i = 0; i < NMB; ++i) tma_prefetch_desc(&p.tb[i]);
  }
  if (warp == 1) {
    if constexpr (CG == 2) {
      tmem_alloc_pair(tmem_slot, Cfg::TMEM_COLS);
      tmem_relinquish_pair();
    } else {
      tmem_alloc(tmem_slot, Cfg::TMEM_COLS);
      tmem_relinquish();
    }
  }
  tc_fence_before();
  __syncwarp();
  if constexpr (CG == 2)
    cluster_sync(); /* the peer's barriers are initialised before any signal */
  else
    __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  /* persistent loop over output tiles of (BM * CG) x BN, one per CTA group
   * (times the batched planes of a plane-batched epilogue) */
  const int tiles_per_plane = p.tiles_m * p.tiles_n;
  const int num_tiles = tiles_per_plane * (EPI::PLANE_BATCH ? p.nplanes : 1);
  const int tile0 = blockIdx.x / CG, tile_step = gridDim.x / CG;
  const int kblocks = (p.k + BKE - 1) / BKE;
  const int chunk_kb = PROMOTE_KB > 0 ? PROMOTE_KB : kblocks;
  const int nchunks = (kblocks + chunk_kb - 1) / chunk_kb;
  const int ntiles_local = tile0 < num_tiles ? (num_tiles - tile0 + tile_step - 1) / tile_step : 0;
  constexpr bool PAIRS = EPI::INPLACE && PROMOTE_KB > 0;
  const int nitems = ntiles_local * nchunks;

  if (warp == 0) {
    /* ------------------------------------------------ TMA producer -- */
    if (lane == 0) {
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int i = 0; ok && i < nitems; ++i) {
        const WorkItem w = work_item(i, tile0, tile_step, ntiles_local, nchunks, PAIRS);
        const int t = w.t;
        const int plane = EPI::PLANE_BATCH ? t / tiles_per_plane : 0;
        const int tt = t - plane * tiles_per_plane;
        const TileMN tc_ = tile_mn(tt, p.tiles_m, p.tiles_n);
        const int tm = tc_.m, tn = tc_.n;
        const int row0 = (tm * CG + (int)rank) * BM;               /* this CTA's A rows */
        const int col0 = tn * BN + (int)rank * (int)Cfg::B_ROWS;   /* this CTA's B rows */
        if constexpr (CatK<EPI>::value) {
          const int d = p.nplanes - 1 - plane;
          for (int j = 0; j < (d + 1) * kblocks; ++j) {
            const int ia = j / kblocks, kb = j - ia * kblocks;
            if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
              ok = false;
              break;
            }
            if (rank == 0) mbar_expect_tx(&full[s], CG * Cfg::STAGE_BYTES);
            uint8_t *st = smem + s * Cfg::STAGE_BYTES;
            const int k0 = p.k0 + kb * BKE;
            if constexpr (CG == 2) {
              tma_load_3d_pair(st, &p.ta[0], mapa_shared(&full[s], 0), k0, row0, ia);
              tma_load_3d_pair(st + Cfg::A_PLANE, &p.tb[0], mapa_shared(&full[s], 0), k0, col0,
                               d - ia);
            } else {
              tma_load_3d(st, &p.ta[0], &full[s], k0, row0, ia);
              tma_load_3d(st + Cfg::A_PLANE, &p.tb[0], &full[s], k0, col0, d - ia);
            }
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
          continue;
        }
        const int kb_end = (w.c + 1) * chunk_kb < kblocks ? (w.c + 1) * chunk_kb : kblocks;
        for (int kb = w.c * chunk_kb; kb < kb_end; ++kb) {
          if (!mbar_wait(&empty[s], ph ^ 1u, p.err, ERR_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          /* the leader's full barrier counts both CTAs' bytes */
          if (rank == 0) mbar_expect_tx(&full[s], CG * Cfg::STAGE_BYTES);
          if (p.inject_skip_load && i == 0 && kb == w.c * chunk_kb) {
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
            continue;
          }
          uint8_t *st = smem + s * Cfg::STAGE_BYTES;
          const int k0 = p.k0 + kb * BKE;
          auto load2d = [&](uint8_t *dst, const CUtensorMap *map, int c0, int c1) {
            if constexpr (EPI::PLANE_BATCH) { /* 3-D maps: {K, rows, plane} */
              if constexpr (CG == 2)
                tma_load_3d_pair(dst, map, mapa_shared(&full[s], 0), c0, c1, plane);
              else
                tma_load_3d(dst, map, &full[s], c0, c1, plane);
            } else if constexpr (CG == 2) {
              tma_load_2d_pair(dst, map, mapa_shared(&full[s], 0), c0, c1);
            } else {
              tma_load_2d(dst, map, &full[s], c0, c1);
            }
          };
#pragma unroll
          for (int a = 0; a < R::NA; ++a) {
            uint8_t *dst = st + a * Cfg::A_PLANE;
            if constexpr (R::P3D) {
              tma_load_3d(dst, &p.ta[0], &full[s], k0, row0, a);
            } else if (!p.a_mn) {
              load2d(dst, &p.ta[a], k0, row0);
            } else {
#pragma unroll
              for (int j = 0; j < BM / 64; ++j)
                load2d(dst + j * (BKE * ROWB), &p.ta[a], row0 + j * 64, k0);
            }
          }
#pragma unroll
          for (int b = 0; b < R::NB; ++b) {
            uint8_t *dst = st + R::NA * Cfg::A_PLANE + b * Cfg::B_PLANE;
            if constexpr (R::P3D) {
              tma_load_3d(dst, &p.tb[0], &full[s], k0, col0, b);
            } else if (!p.b_mn) {
              load2d(dst, &p.tb[b], k0, col0);
            } else {
#pragma unroll
              for (int j = 0; j < (int)Cfg::B_ROWS / 64; ++j)
                load2d(dst + j * (BKE * ROWB), &p.tb[b], col0 + j * 64, k0);
            }
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
    if (lane == 0 && rank == 0) {
      const uint32_t idesc =
          make_idesc(KT::CFMT, KT::ABFMT, p.a_mn != 0, p.b_mn != 0, BM * CG, BN);
      const uint32_t a_lbo = p.a_mn ? BKE * ROWB : 16, b_lbo = p.b_mn ? BKE * ROWB : 16;
      const uint32_t a_kstep = p.a_mn ? KT::UK * ROWB : KT::UK * KT::ESZ;
      const uint32_t b_kstep = p.b_mn ? KT::UK * ROWB : KT::UK * KT::ESZ;
      int s = 0;
      uint32_t ph = 0;
      int ci = 0; /* chunk counter (all tiles): selects the TMEM buffer */
      uint32_t uses = 0u; /* in-place mode: bit b = parity of buffer b's acquisitions */
      bool ok = true;
      for (int i = 0; ok && i < nitems; ++i, ++ci) {
        {
          const WorkItem w = work_item(i, tile0, tile_step, ntiles_local, nchunks, PAIRS);
          const int kc = w.c * chunk_kb;
          /* in-place mode: chunk c of a tile accumulates into its slot's
           * buffer on top of the epilogue's reduced value of chunk c - 1 */
          const int b = PAIRS ? w.slot : ci % NBUF;
          const uint32_t tph = PAIRS ? (uses >> b) & 1u : (ci / NBUF) & 1;
          if (PAIRS) uses ^= 1u << b;
          const bool fresh = !PAIRS || w.c == 0;
          if (!mbar_wait<CG == 2>(&tempty[b], tph ^ 1u, p.err, ERR_TIMEOUT_MMA_TMEM)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t dbase = tmem_base + b * Cfg::ACC_COLS;
          int kend = (kc + chunk_kb < kblocks) ? kc + chunk_kb : kblocks;
          if constexpr (CatK<EPI>::value)
            kend = (p.nplanes - (w.t / tiles_per_plane)) * kblocks; /* (d + 1) * kblocks */
          for (int kb = kc; kb < kend; ++kb) {
            if (!mbar_wait<CG == 2>(&full[s], ph, p.err, ERR_TIMEOUT_MMA_FULL)) {
              ok = false;
              break;
            }
            tc_fence_after();
            const uint32_t sbase = smem_u32(smem + s * Cfg::STAGE_BYTES);
#pragma unroll
            for (int kk = 0; kk < KSTEPS; ++kk) {
#pragma unroll
              for (int pi = 0; pi < R::NP; ++pi) {
                const uint32_t aa = sbase + R::pa(pi) * Cfg::A_PLANE + kk * a_kstep;
                const uint32_t ba =
                    sbase + R::NA * Cfg::A_PLANE + R::pb(pi) * Cfg::B_PLANE + kk * b_kstep;
                const uint64_t ad = smem_desc(aa, a_lbo, KT::SBO, KT::LAYOUT);
                const uint64_t bd = smem_desc(ba, b_lbo, KT::SBO, KT::LAYOUT);
                const uint32_t acc = (!fresh || kb > kc || kk > 0 || !R::first(pi)) ? 1u : 0u;
                if constexpr (KIND == 3 && CG == 1)
                  mma_i8(dbase + R::pacc(pi) * BN, ad, bd, idesc, acc);
                else if constexpr (KIND == 3)
                  mma_i8_pair(dbase + R::pacc(pi) * BN, ad, bd, idesc, acc);
                else if constexpr (CG == 2)
                  mma_f16_pair(dbase + R::pacc(pi) * BN, ad, bd, idesc, acc);
                else
                  mma_f16(dbase + R::pacc(pi) * BN, ad, bd, idesc, acc);
              }
            }
            if constexpr (CG == 2)
              mma_commit_pair(&empty[s], 0x3); /* frees the stage in both CTAs */
            else
              mma_commit(&empty[s]);
            if (++s == STAGES) {
              s = 0;
              ph ^= 1u;
            }
          }
          if (ok) {
            if constexpr (CG == 2)
              mma_commit_pair(&tfull[b], 0x3);
            else
              mma_commit(&tfull[b]);
          }
        }
      }
    }
  } else {
    /* ------------------------------------------------ epilogue -- */
    const int q = warp & 3;      /* TMEM lane quadrant of this warp */
    const int ew = warp - 2;     /* epilogue warp index */
    const int half = ew >> 2;    /* with eight warps: which half of the columns */
    int ci = 0;
    bool ok = true;
    OutStage ostage{Cfg::OUT_BYTES ? smem + Cfg::OUT_OFF + ew * EPI::OUT_WARP_BYTES : nullptr,
                    obar + 2 * ew, 0u, 0u, 0};
    static_assert(!EPI::INPLACE || Cfg::OUT_BYTES > 0, "the modular epilogue stores by TMA");
    static_assert(!EPI::PLANE_BATCH || Cfg::OUT_BYTES > 0, "plane-batched epilogues store by TMA");
    /* TMEM buffer released to the leader's MMA thread */
    auto release = [&](int b) {
      if (lane == 0) {
        if constexpr (CG == 2)
          mbar_arrive_cluster(mapa_shared(&tempty[b], 0));
        else
          mbar_arrive(&tempty[b]);
      }
    };
    uint32_t euses = 0u; /* in-place mode: bit b = parity of buffer b's acquisitions */
    if constexpr (PAIRS) {
      /* in-place modular mode: every chunk but a tile's last is reduced in
       * place and handed back; the last is reduced and stored from the same
       * buffer while the tensor core works on the pair's other tile */
      const uint32_t lane_off = static_cast<uint32_t>(q * 32) << 16;
      for (int i = 0; i < nitems; ++i) {
        const WorkItem w = work_item(i, tile0, tile_step, ntiles_local, nchunks, true);
        const int plane = EPI::PLANE_BATCH ? w.t / tiles_per_plane : 0;
        const int tt = w.t - plane * tiles_per_plane;
        const TileMN tc_ = tile_mn(tt, p.tiles_m, p.tiles_n);
        const int tm = tc_.m, tn = tc_.n;
        const int m = (tm * CG + (int)rank) * BM + q * 32 + lane;
        const int b = w.slot;
        const uint32_t tph = (euses >> b) & 1u;
        euses ^= 1u << b;
        if (!__all_sync(0xffffffffu, mbar_wait(&tfull[b], tph, p.err, ERR_TIMEOUT_EPILOGUE))) break;
        tc_fence_after();
        const uint32_t tb = tmem_base + lane_off + b * Cfg::ACC_COLS;
        if (w.c < nchunks - 1)
          EPI::template rmw<BN>(p, tb, plane);
        else
          EPI::template final_store<BN>(p, tb, ostage.box, m - lane, tn * BN, plane);
        tc_fence_before();
        __syncwarp();
        release(b);
      }
    } else {
    for (int t = tile0; ok && t < num_tiles; t += tile_step) {
      const int plane = EPI::PLANE_BATCH ? t / tiles_per_plane : 0;
      const int tt = t - plane * tiles_per_plane;
      const TileMN tc_ = tile_mn(tt, p.tiles_m, p.tiles_n);
      const int tm = tc_.m, tn = tc_.n;
      const int m = (tm * CG + (int)rank) * BM + q * 32 + lane;
      if constexpr (Cfg::OUT_BYTES > 0) EPI::template prefetch_c<BN>(p, m - lane, tn * BN, ostage);
      else if constexpr (EpiL2Prefetch<EPI>::value && !EPI::PLANE_BATCH)
        EPI::template prefetch_c_l2<BN>(p, m, tn * BN);
      if constexpr (PROMOTE_KB == 0) {
        const int b = ci % NBUF;
        const uint32_t tph = (ci / NBUF) & 1;
        ++ci;
        if (!__all_sync(0xffffffffu, mbar_wait(&tfull[b], tph, p.err, ERR_TIMEOUT_EPILOGUE))) break;
        tc_fence_after();
        const uint32_t tbase =
            tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * Cfg::ACC_COLS;
        if constexpr (EPI::PLANE_BATCH) {
          constexpr int COLS = BN / (EW / 4); /* this warp's columns */
          EPI::template final_store<COLS>(p, tbase + half * COLS, ostage.box, m - lane,
                                          tn * BN + half * COLS, plane);
        } else
          EPI::template run<BN, R::NACC>(p, tbase, m, tn * BN, ostage);
        tc_fence_before();
        __syncwarp();
        release(b);
      } else {
        typename EPI::AccT acc[BN];
#pragma unroll
        for (int j = 0; j < BN; ++j) acc[j] = 0;
        for (int kc = 0; kc < kblocks; kc += chunk_kb, ++ci) {
          const int b = ci % NBUF;
          const uint32_t tph = (ci / NBUF) & 1;
          if (!__all_sync(0xffffffffu, mbar_wait(&tfull[b], tph, p.err, ERR_TIMEOUT_EPILOGUE))) {
            ok = false;
            break;
          }
          tc_fence_after();
          EPI::template accumulate<BN, R::NACC>(
              p, tmem_base + (static_cast<uint32_t>(q * 32) << 16) + b * Cfg::ACC_COLS, acc,
              kc / chunk_kb);
          tc_fence_before();
          __syncwarp();
          release(b);
        }
        if (ok) EPI::template store_acc<BN>(p, acc, m, tn * BN, ostage);
      }
    }
    }
    if constexpr (Cfg::OUT_BYTES > 0) {
      if (lane == 0) {
        /* C loads still in flight (only after a failed wait): give them a
         * bounded time to land before the CTA's shared memory is released */
#pragma unroll
        for (int x = 0; x < 2; ++x)
          if ((ostage.pend >> x) & 1u)
            for (int it = 0; it < (1 << 22) && !mbar_try_wait(&ostage.bar[x], (ostage.phase >> x) & 1u);
                 ++it) {
            }
        bulk_wait_all(); /* this warp's last tensor stores have landed */
      }
    }
  }

  tc_fence_before();
  __syncwarp();
  if constexpr (CG == 2)
    cluster_sync(); /* neither CTA leaves while the pair still uses its memory */
  else
    __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    if constexpr (CG == 2)
      tmem_dealloc_pair(tmem_base, Cfg::TMEM_COLS);
    else
      tmem_dealloc(tmem_base, Cfg::TMEM_COLS);
  }
}

/* ------------------------------------------------------------- host -- */

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q);
    if (e == cudaSuccess && q == cudaDriverEntryPointSuccess && ptr) {
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    } else {
      cudaGetLastError();
      const char *env = getenv("HCBLAS_LOG");
      if (env && env[0] == '1')
        fprintf(stderr, "[hcblas] cuTensorMapEncodeTiled entry point unavailable (%d, %d)\n",
                (int)e, (int)q);
    }
  }
  return fn;
}

/* Tensor map over a 2-D operand with `inner` contiguous elements per line,
 * `outer` lines `ld` elements apart; box = {box_inner, box_outer}, 128-byte
 * swizzle, zero fill out of bounds. */
static int make_map(CUtensorMap *map, CUtensorMapDataType dt, int esz, const void *base,
                    uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_inner,
                    uint32_t box_outer) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * esz) & 15)) return HCBK_ERR_ALIGN;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {ld * esz};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    const char *e = getenv("HCBLAS_LOG");
    if (e && e[0] == '1')
      fprintf(stderr,
              "[hcblas] cuTensorMapEncodeTiled failed (%d): base=%p dims={%llu,%llu} "
              "stride=%llu box={%u,%u}\n",
              (int)r, base, (unsigned long long)inner, (unsigned long long)outer,
              (unsigned long long)(ld * esz), box_inner, box_outer);
    return HCBK_ERR_ALIGN;
  }
  return HCBK_OK;
}

template <int BN, int STAGES, class R, int KIND, class EPI, int PROMOTE_KB = 0, int NBUF = 2,
          int CG = 1>
static int launch_tc(TcParams &p, void *stream) {
  using Cfg = TcCfg<BN, STAGES, R, KIND, NBUF, CG, EPI::OUT_SMEM>;
  auto kern = tc_gemm_kernel<BN, STAGES, R, KIND, EPI, PROMOTE_KB, NBUF, CG>;
  static bool attr_set[64] = {false};
  static int pair_slots[64] = {0}; /* co-resident CTA pairs per device */
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  cudaLaunchConfig_t cfg;
  memset(&cfg, 0, sizeof(cfg));
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CG;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(64 + 32 * EpiWarps<EPI>::value, 1, 1);
  cfg.dynamicSmemBytes = Cfg::SMEM_BYTES;
  cfg.stream = static_cast<cudaStream_t>(stream);
  cfg.attrs = attr;
  cfg.numAttrs = CG == 2 ? 1 : 0;
  if (!attr_set[dev]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             Cfg::SMEM_BYTES) != cudaSuccess)
      return HCBK_ERR_LAUNCH;
    if (CG == 2) {
      /* SMs pair up within a GPC, so fewer than sm_count / 2 pairs may fit */
      int clusters = 0;
      cfg.gridDim = dim3(2 * (hcbk_sm_count() / 2), 1, 1);
      if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        return HCBK_ERR_LAUNCH;
      }
      pair_slots[dev] = clusters;
    }
    attr_set[dev] = true;
  }
  p.tiles_m = (p.m + BM * CG - 1) / (BM * CG);
  p.tiles_n = (p.n + BN - 1) / BN;
  const int tiles = p.tiles_m * p.tiles_n * (EPI::PLANE_BATCH ? p.nplanes : 1);
  int groups = CG == 2 ? pair_slots[dev] : hcbk_sm_count();
  if (tiles < groups) groups = tiles;
  cfg.gridDim = dim3((unsigned)(groups * CG), 1, 1);
  if (cudaLaunchKernelEx(&cfg, kern, p) != cudaSuccess) {
    cudaGetLastError();
    return HCBK_ERR_LAUNCH;
  }
  return HCBK_OK;
}

}  // namespace tc
}  // namespace hcbk

using namespace hcbk::tc;

/* 2-D f16/bf16 tensor map with 128-byte swizzle (see make_map). */
extern "C" int hcbk_encode_tma_2d(void *map, int bf16, const void *base, uint64_t inner,
                                  uint64_t outer, uint64_t ld, uint32_t box_inner,
                                  uint32_t box_outer) {
  return make_map(static_cast<CUtensorMap *>(map),
                  bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2,
                  base, inner, outer, ld, box_inner, box_outer);
}

/* 2-D map over a column-major C {rows, cols} of esz-byte elements, column
 * pitch ld elements; box {32, 32}, no swizzle.  HCBK_ERR_ALIGN when C is not
 * TMA-addressable (base not 16-byte aligned, pitch not a multiple of 16
 * bytes) or when a column is not a whole number of 16-byte chunks: measured
 * on B200, a tensor store whose box crosses the end of the rows writes the
 * rest of the 16-byte chunk holding the last row, which would overwrite the
 * leading-dimension padding below row `rows` (C outside the M x N window
 * must stay untouched). */
static int make_map_out(CUtensorMap *map, CUtensorMapDataType dt, uint32_t esz, void *base,
                        uint64_t rows, uint64_t cols, uint64_t ld) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * esz) & 15) || ((rows * esz) & 15) ||
      rows == 0 || cols == 0)
    return HCBK_ERR_ALIGN;
  cuuint64_t dims[2] = {rows, cols};
  cuuint64_t strides[1] = {ld * esz};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HCBK_OK : HCBK_ERR_ALIGN;
}

extern "C" int hcbk_encode_out_2d(void *map, void *base, uint64_t rows, uint64_t cols,
                                  uint64_t ld) {
  return make_map_out(static_cast<CUtensorMap *>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, base,
                      rows, cols, ld);
}

/* f16 operands straight from the caller's matrices (column-major canonical). */
static int hgemm_tc_impl(const hcbk_gemm_args *a, int bn, int pair, int *err, void *stream,
                         int inject_skip_load) {
  if (a->dtype != HCBK_H || a->batch != 1 || a->a_array || a->op_a == HCBK_OP_C ||
      a->op_b == HCBK_OP_C)
    return HCBK_ERR_ARGS;
  if (a->m > 0x7fffffff || a->n > 0x7fffffff || a->k > 0x7fffffff) return HCBK_ERR_ARGS;
  TcParams p;
  memset(&p, 0, sizeof(p));
  p.m = (int)a->m;
  p.n = (int)a->n;
  p.k = (int)a->k;
  const __half *A = static_cast<const __half *>(a->a) + a->a_off;
  const __half *B = static_cast<const __half *>(a->b) + a->b_off;
  /* op(A) = A: column-major M x K, M contiguous (MN-major);  op(A) = A^T: K contiguous */
  p.a_mn = (a->op_a == HCBK_OP_N);
  /* op(B) = B: K x N, K contiguous (K-major);  op(B) = B^T: N contiguous */
  p.b_mn = (a->op_b != HCBK_OP_N);
  const auto F16 = CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  int rc;
  if (p.a_mn)
    rc = make_map(&p.ta[0], F16, 2, A, a->m, a->k, a->lda, 64, 64);
  else
    rc = make_map(&p.ta[0], F16, 2, A, a->k, a->m, a->lda, 64, BM);
  if (rc) return rc;
  if ((bn != 128 && bn != 256) || (pair && bn != 256)) return HCBK_ERR_ARGS;
  const uint32_t bn_box = (uint32_t)(pair ? bn / 2 : bn); /* B rows per CTA */
  if (p.b_mn)
    rc = make_map(&p.tb[0], F16, 2, B, a->n, a->k, a->ldb, 64, 64);
  else
    rc = make_map(&p.tb[0], F16, 2, B, a->k, a->n, a->ldb, 64, bn_box);
  if (rc) return rc;
  p.c = static_cast<__half *>(a->c) + a->c_off;
  p.ldc = a->ldc;
  p.alpha = (float)a->alpha_re;
  p.beta = (float)a->beta_re;
  p.beta_nonzero = a->beta_re != 0.0;
  p.err = err;
  /* C tensor-map addressable: the epilogue stages 32 x 32 boxes in shared
   * memory, reading C (beta != 0) and writing it by TMA */
  p.out_tma =
      make_map_out(&p.tc, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, p.c, a->m, a->n, a->ldc) == HCBK_OK;
  using EH = EpiAlphaBeta<__half>;
  if (inject_skip_load) {
    /* one 128 x 128 tile of one 64-wide K block, beta == 0: the only load
     * the kernel would issue is the skipped one, the epilogue reads no C */
    if (a->m > BM || a->n > 128 || a->k > 64 || p.beta_nonzero || pair || bn != 128)
      return HCBK_ERR_ARGS;
    p.inject_skip_load = 1;
  }
  if (pair) return launch_tc<256, 6, RecipeSingle, 0, EH, 0, 2, 2>(p, stream);
  if (bn == 256) return launch_tc<256, 4, RecipeSingle, 0, EH>(p, stream);
  return launch_tc<128, 6, RecipeSingle, 0, EH>(p, stream);
}

extern "C" int hcbk_hgemm_tc(const hcbk_gemm_args *a, int bn, int pair, int *err, void *stream) {
  return hgemm_tc_impl(a, bn, pair, err, stream, 0);
}

extern "C" int hcbk_hgemm_tc_inject_timeout(const hcbk_gemm_args *a, int *err, void *stream) {
  return hgemm_tc_impl(a, 128, 0, err, stream, 1);
}

/* split-BF16 SGEMM on pre-split K-major planes:
 *   A planes: [M][lda_p] bf16 (K contiguous), B planes: [N][ldb_p] bf16. */
extern "C" int hcbk_sgemm_split_tc(const hcbk_split_gemm *g, int *err, void *stream) {
  TcParams p;
  memset(&p, 0, sizeof(p));
  if (g->m > 0x7fffffff || g->n > 0x7fffffff || g->k > 0x7fffffff) return HCBK_ERR_ARGS;
  p.m = (int)g->m;
  p.n = (int)g->n;
  p.k = (int)g->k;
  p.a_mn = 0;
  p.b_mn = 0;
  const auto BF16 = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  const int planes = g->terms == 6 ? 3 : 2;
  if (g->bn != 128) return HCBK_ERR_ARGS;
  const uint32_t bn_box = g->pair ? 64u : 128u; /* B rows per CTA */
  for (int i = 0; i < planes; ++i) {
    int rc = make_map(&p.ta[i], BF16, 2, g->a_planes[i], g->k, g->m, g->ld_a, 64, BM);
    if (rc) return rc;
    rc = make_map(&p.tb[i], BF16, 2, g->b_planes[i], g->k, g->n, g->ld_b, 64, bn_box);
    if (rc) return rc;
  }
  p.c = g->c;
  p.ldc = g->ldc;
  p.alpha = (float)g->alpha;
  p.beta = (float)g->beta;
  p.beta_nonzero = g->beta != 0.0;
  p.err = err;
  /* two accumulators per chunk, double-buffered: 2 x 2 x 128 TMEM columns */
  /* C tensor-map addressable: configurations with room stage the epilogue
   * through shared memory and TMA */
  p.out_tma = make_map_out(&p.tc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, p.c, g->m, g->n,
                           g->ldc) == HCBK_OK;
  using EF = EpiAlphaBeta<float>;
  if (g->pair) {
    if (g->terms == 6) {
      if (g->promote_kb == 4) return launch_tc<128, 3, RecipeBf16x6, 1, EF, 4, 2, 2>(p, stream);
      return launch_tc<128, 3, RecipeBf16x6, 1, EF, 1, 2, 2>(p, stream);
    }
    if (g->promote_kb == 4) return launch_tc<128, 4, RecipeBf16x3, 1, EF, 4, 2, 2>(p, stream);
    return launch_tc<128, 4, RecipeBf16x3, 1, EF, 1, 2, 2>(p, stream);
  }
  if (g->terms == 6) {
    if (g->promote_kb == 4) return launch_tc<128, 2, RecipeBf16x6, 1, EF, 4>(p, stream);
    return launch_tc<128, 2, RecipeBf16x6, 1, EF, 1>(p, stream);
  }
  if (g->promote_kb == 4) return launch_tc<128, 3, RecipeBf16x3, 1, EF, 4>(p, stream);
  return launch_tc<128, 3, RecipeBf16x3, 1, EF, 1>(p, stream);
}

extern "C" int64_t hcbk_ozaki_max_k(int slices) {
  if (slices < 1) return 0;
  /* |acc_d| <= slices * K * 127^2 must stay below 2^31 */
  const int64_t k = (int64_t)0x7fffffff / ((int64_t)slices * 127 * 127);
  return k & ~int64_t(127); /* whole 128-element K slabs of the int8 kernel */
}

/* 3-D map over `planes` f16 planes {K, rows, plane}: row pitch ld elements,
 * plane pitch pstride bytes; box {64, box_rows, 1}, 128-byte swizzle. */
static int make_map_planes(CUtensorMap *map, CUtensorMapDataType dt, const void *base,
                           uint64_t kdim, uint64_t rows, uint64_t planes, uint64_t ld,
                           uint64_t pstride, uint32_t box_rows, uint32_t esz = 2) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * esz) & 15) || (pstride & 15))
    return HCBK_ERR_ALIGN;
  cuuint64_t dims[3] = {kdim, rows, planes};
  cuuint64_t strides[2] = {ld * esz, pstride};
  cuuint32_t box[3] = {128 / esz, box_rows, 1}; /* one 128-byte swizzle row of K */
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, dt, 3, const_cast<void *>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HCBK_OK : HCBK_ERR_ALIGN;
}

static int make_map_planes_f16(CUtensorMap *map, const void *base, uint64_t kdim, uint64_t rows,
                               uint64_t planes, uint64_t ld, uint64_t pstride, uint32_t box_rows) {
  return make_map_planes(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, base, kdim, rows, planes, ld,
                         pstride, box_rows);
}

/* int8 residue planes: box {128, box_rows, 1} (one 128-byte swizzle row) */
static int make_map_planes_s8(CUtensorMap *map, const void *base, uint64_t kdim, uint64_t rows,
                              uint64_t planes, uint64_t ld, uint64_t pstride, uint32_t box_rows) {
  return make_map_planes(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, base, kdim, rows, planes, ld,
                         pstride, box_rows, 1);
}

extern "C" int hcbk_encode_tma_3d_planes(void *map, int bf16, const void *base, uint64_t kdim,
                                         uint64_t rows, uint64_t planes, uint64_t ld,
                                         uint64_t pstride, uint32_t box_rows) {
  return make_map_planes(static_cast<CUtensorMap *>(map),
                         bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                         base, kdim, rows, planes, ld, pstride, box_rows);
}

/* 3-D map over the int8 residue planes T {rows, cols, plane}: column pitch
 * ld bytes, plane pitch pstride bytes (multiples of 16); box {32, 32, 1}, no
 * swizzle (the modular epilogue's tensor stores). */
static int make_map_out_i8(CUtensorMap *map, void *base, uint64_t rows, uint64_t cols,
                           uint64_t planes, uint64_t ld, uint64_t pstride) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld & 15) || (pstride & 15))
    return HCBK_ERR_ALIGN;
  cuuint64_t dims[3] = {rows, cols, planes};
  cuuint64_t strides[2] = {ld, pstride};
  cuuint32_t box[3] = {32, 32, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HCBK_OK : HCBK_ERR_ALIGN;
}

/* 3-D map over the int32 slice-group sums D {rows, cols, group}: column
 * pitch ld elements, group pitch pstride elements; box {32, 32, 1}, no
 * swizzle (the slice-group epilogue's tensor stores). */
static int make_map_out_i32(CUtensorMap *map, void *base, uint64_t rows, uint64_t cols,
                            uint64_t planes, uint64_t ld, uint64_t pstride) {
  auto fn = encode_fn();
  if (!fn) return HCBK_ERR_DRIVER;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * 4) & 15) || ((pstride * 4) & 15))
    return HCBK_ERR_ALIGN;
  cuuint64_t dims[3] = {rows, cols, planes};
  cuuint64_t strides[2] = {ld * 4, pstride * 4};
  cuuint32_t box[3] = {32, 32, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_INT32, 3, base, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? HCBK_OK : HCBK_ERR_ALIGN;
}

extern "C" int hcbk_ozaki_groups_tc(const hcbk_ozaki_groups *g, int *err, void *stream) {
  if (g->m <= 0 || g->n <= 0 || g->k <= 0 || g->m > 0x7fffffff || g->n > 0x7fffffff ||
      g->k > hcbk_ozaki_max_k(g->slices) || g->k0 < 0 || g->k0 + g->k > 0x7fffffff ||
      g->slices < 1 || g->slices > 8 || (g->k0 & 127) || !g->d)
    return HCBK_ERR_ARGS;
  TcParams p;
  memset(&p, 0, sizeof(p));
  p.m = (int)g->m;
  p.n = (int)g->n;
  p.k = (int)g->k;
  p.k0 = (int)g->k0;
  const uint64_t kdim = (uint64_t)(g->k0 + g->k); /* zero fill beyond the range's end */
  int rc = make_map_planes_s8(&p.ta[0], g->a_planes, kdim, g->m, g->slices, g->ld_a,
                              g->a_plane_stride, BM);
  if (rc) return rc;
  rc = make_map_planes_s8(&p.tb[0], g->b_planes, kdim, g->n, g->slices, g->ld_b,
                          g->b_plane_stride, g->pair ? 128 : 256);
  if (rc) return rc;
  rc = make_map_out_i32(&p.tc, g->d, g->m, g->n, g->slices, g->ldd, g->d_plane);
  if (rc) return rc;
  p.nplanes = g->slices;
  p.err = err;
  if (g->pair) return launch_tc<256, 6, RecipeSingle, 3, EpiI32Cat, 0, 2, 2>(p, stream);
  return launch_tc<256, 4, RecipeSingle, 3, EpiI32Cat, 0, 2>(p, stream);
}

/* Every modulus of the CRT scheme in one launch: f16 residue planes
 * (K-major, |r| <= 127) read through 3-D tensor maps, tensor-core sums exact
 * over 1024-element K chunks (PROMOTE_KB = 16 slabs of 64:
 * 1024 * 127^2 + 383 < 2^24), reduced mod p in place in TMEM between chunks,
 * int8 residues out by TMA tensor stores (t 16-byte aligned, ldt and
 * t_plane_stride multiples of 16 bytes); the persistent tile walk spans all planes.  Tiles:
 * 256 x 256 over a CTA pair, or 128 x bn on one CTA. */
extern "C" int hcbk_crt_gemm_tc(const hcbk_crt_gemm *g, int *err, void *stream) {
  if (g->m > 0x7fffffff || g->n > 0x7fffffff || g->k > 0x7fffffff || g->k <= 0 ||
      g->nmod < 1 || g->nmod > HCBK_CRT_MAX_MODULI || !g->moduli ||
      (g->bn != 128 && g->bn != 256) || (g->pair && g->bn != 256))
    return HCBK_ERR_ARGS;
  for (int i = 0; i < g->nmod; ++i)
    if (g->moduli[i] < 3 || g->moduli[i] > 255 || (g->moduli[i] & 1) == 0) return HCBK_ERR_ARGS;
  if (g->i8 && g->k > HCBK_CRT_I8_MAX_K) return HCBK_ERR_ARGS;
  TcParams p;
  memset(&p, 0, sizeof(p));
  p.m = (int)g->m;
  p.n = (int)g->n;
  p.k = (int)g->k;
  /* a batch of GEMMs: element e's modulus-i planes are plane e * nmod + i
   * of A, B and T */
  const int64_t batch = g->batch > 1 ? g->batch : 1;
  const int64_t planes = batch * g->nmod;
  const int64_t tiles_m = (g->m + 127) / 128, tiles_n = (g->n + g->bn - 1) / g->bn;
  if (planes > 0x7fffffff || tiles_m * tiles_n * planes > 0x7fffffff) return HCBK_ERR_ARGS;
  auto planes_map = g->i8 ? make_map_planes_s8 : make_map_planes_f16;
  int rc = planes_map(&p.ta[0], g->a_planes, g->k, g->m, (int)planes, g->ld_a, g->a_plane_stride,
                      BM);
  if (rc) return rc;
  const uint32_t b_rows = g->pair ? g->bn / 2 : g->bn; /* B rows per CTA */
  rc = planes_map(&p.tb[0], g->b_planes, g->k, g->n, (int)planes, g->ld_b, g->b_plane_stride,
                  b_rows);
  if (rc) return rc;
  p.c = g->t;
  p.ldc = g->ldt;
  p.nplanes = (int)planes;
  p.mod_period = g->nmod;
  p.c_plane_stride = g->t_plane_stride;
  rc = make_map_out_i8(&p.tc, g->t, g->m, g->n, (int)planes, g->ldt, g->t_plane_stride);
  if (rc) return rc;
  for (int i = 0; i < g->nmod; ++i) {
    p.mod_tab[i] = g->moduli[i];
    p.inv_mod_tab[i] = 1.0f / (float)g->moduli[i];
  }
  p.err = err;
  if (g->i8) {
    if (g->pair) return launch_tc<256, 6, RecipeSingle, 3, EpiModPi8, 0, 2, 2>(p, stream);
    if (g->bn == 256) return launch_tc<256, 4, RecipeSingle, 3, EpiModPi8, 0, 2>(p, stream);
    return launch_tc<128, 6, RecipeSingle, 3, EpiModPi8, 0, 2>(p, stream);
  }
  if (g->pair) return launch_tc<256, 6, RecipeSingle, 0, EpiModP, 16, 2, 2>(p, stream);
  if (g->bn == 256) return launch_tc<256, 4, RecipeSingle, 0, EpiModP, 16, 2>(p, stream);
  return launch_tc<128, 6, RecipeSingle, 0, EpiModP, 16, 2>(p, stream);
}
