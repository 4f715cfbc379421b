/*
 * tc_common.cuh -- sm_100a building blocks written directly in PTX:
 * mbarriers with bounded waits, TMA tile loads (no cluster multicast),
 * tcgen05 MMA / TMEM allocation / TMEM loads, and the shared-memory matrix
 * and instruction descriptors of the 5th-generation tensor cores.
 *
 * Descriptor bit layouts follow the PTX ISA ("tcgen05 matrix descriptors",
 * "instruction descriptor"): they were cross-checked against the field
 * definitions in CUTLASS's cute/arch/mma_sm100_desc.hpp.
 *
 * Every wait on an mbarrier is bounded: after the wait limit of
 * %globaltimer time the wait records an error code in a device flag and
 * returns false, and the kernel unwinds (frees TMEM, exits) instead of
 * hanging the GPU.
 *
 * The flag is the first int of the device error block each tensor-core
 * kernel receives as `err` (16 bytes, 8-byte aligned): err[0] the error code
 * (0 = none), err[2..3] the wait limit in nanoseconds as one 64-bit value
 * (0 = HCBK_WAIT_TIMEOUT_NS).  The limit is read once per wait, when the
 * first try finds the phase incomplete.
 */
#ifndef HCBLAS_B200_TC_COMMON_CUH_
#define HCBLAS_B200_TC_COMMON_CUH_

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef HCBK_WAIT_TIMEOUT_NS
#define HCBK_WAIT_TIMEOUT_NS 2000000000ull /* 2 s */
#endif

namespace hcbk {
namespace tc {

/* error codes written to the device error flag */
enum : int {
  ERR_NONE = 0,
  ERR_TIMEOUT_PRODUCER = 1,
  ERR_TIMEOUT_MMA_FULL = 2,
  ERR_TIMEOUT_MMA_TMEM = 3,
  ERR_TIMEOUT_EPILOGUE = 4,
  ERR_TIMEOUT_COMBINE = 5,
  ERR_LAUNCH_SHAPE = 6, /* a kernel was launched with a block shape it does not support */
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

/* ------------------------------------------------------------ mbarrier -- */

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/* the same with cluster-scope acquire: for barriers that the peer CTA of
 * a pair arrives on */
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

/* Wait for the phase with the given parity to complete.  Bounded: returns
 * false (after recording `code` in *err) on timeout, or when another thread
 * has already recorded an error. */
template <bool CLUSTER = false>
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, int code) {
  auto try_once = [&]() {
    return CLUSTER ? mbar_try_wait_cluster(bar, parity) : mbar_try_wait(bar, parity);
  };
  if (try_once()) return true;
  const uint64_t t0 = globaltimer();
  const uint64_t set = *reinterpret_cast<volatile unsigned long long *>(err + 2);
  const uint64_t limit = set ? set : HCBK_WAIT_TIMEOUT_NS;
  uint32_t n = 0;
  while (true) {
    if (try_once()) return true;
    if ((++n & 1023u) == 0) {
      if (*reinterpret_cast<volatile int *>(err) != 0) return false;
      if (globaltimer() - t0 > limit) {
        atomicCAS(err, 0, code);
        return false;
      }
    }
  }
}

/* ------------------------------------------------- CTA pair (cluster) -- */

__device__ __forceinline__ uint32_t cluster_ctarank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

/* every thread of every CTA in the cluster; release/acquire ordering */
__device__ __forceinline__ void cluster_sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
               "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

/* shared::cluster address of the variable at `p` in CTA `rank` of the cluster */
__device__ __forceinline__ uint32_t mapa_shared(const void *p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
  return r;
}

/* arrive on an mbarrier given by its shared::cluster address (possibly in
 * the peer CTA) */
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t cluster_addr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
               : "memory");
}

/* ---------------------------------------------------------------- TMA -- */

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap *map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

/* 1-D bulk copy from global memory into this CTA's shared memory: both
 * addresses 16-byte aligned, `bytes` a multiple of 16; completion is
 * signalled on `bar` (complete_tx).  No multicast. */
__device__ __forceinline__ void bulk_load_1d(void *dst, const void *src, uint32_t bytes,
                                             uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_u32(dst)),
      "l"(static_cast<uint64_t>(__cvta_generic_to_global(src))), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

/* 2-D tiled bulk tensor load into this CTA's shared memory; completion is
 * signalled on `bar` (complete_tx).  No multicast. */
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int32_t c0, int32_t c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}

/* 3-D tiled bulk tensor load (coordinates innermost first).  No multicast. */
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar,
                                            int32_t c0, int32_t c1, int32_t c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

/* 2-D tiled load into this CTA's shared memory whose completion is counted
 * on the mbarrier at shared::cluster address `bar_cluster` -- the pair
 * leader's barrier (.cta_group::2 lets the barrier live in either CTA of the
 * pair).  No multicast. */
__device__ __forceinline__ void tma_load_2d_pair(void *dst, const CUtensorMap *map,
                                                 uint32_t bar_cluster, int32_t c0, int32_t c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(c0), "r"(c1)
      : "memory");
}

/* 3-D form of tma_load_2d_pair (coordinates innermost first).  No multicast. */
__device__ __forceinline__ void tma_load_3d_pair(void *dst, const CUtensorMap *map,
                                                 uint32_t bar_cluster, int32_t c0, int32_t c1,
                                                 int32_t c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar_cluster), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

/* 2-D tiled bulk tensor store from this CTA's shared memory (coordinates
 * innermost first); out-of-range parts of the box are not written. */
__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, const void *src, int32_t c0,
                                             int32_t c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(c0), "r"(c1)
      : "memory");
}

/* 3-D tiled bulk tensor store from this CTA's shared memory (coordinates
 * innermost first); out-of-range parts of the box are not written.  The
 * writing threads issue fence_proxy_async_smem() before the store. */
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *src, int32_t c0,
                                             int32_t c1, int32_t c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}

/* Tensor maps patched on the device (problem tables built by a kernel
 * from device-resident pointer arrays): the global address of a 128-byte
 * aligned map in global memory is replaced in place, the patching thread
 * releases its generic-proxy writes to the tensor-map proxy, and a kernel
 * that then loads or stores through the map acquires it first. */
__device__ __forceinline__ void tensormap_replace_address(void *map, const void *addr) {
  asm volatile("tensormap.replace.tile.global_address.global.b1024.b64 [%0], %1;" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "l"(reinterpret_cast<uint64_t>(addr))
               : "memory");
}

__device__ __forceinline__ void tensormap_release() {
  asm volatile("fence.proxy.tensormap::generic.release.gpu;" ::: "memory");
}

__device__ __forceinline__ void tensormap_acquire(const void *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

/* make this thread's generic-proxy shared-memory writes visible to the
 * async proxy (bulk / tensor copies) */
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

/* wait until at most N of this thread's committed bulk groups still read
 * their shared-memory source */
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

/* wait until all of this thread's committed bulk groups have completed */
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

/* ------------------------------------------------------------ tcgen05 -- */

/* TMEM allocation for a CTA pair: one warp (same warp index) in each CTA
 * of the pair issues it; both receive the same column range. */
__device__ __forceinline__ void tmem_alloc_pair(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish_pair() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc_pair(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

/* Pair MMA (issued by one thread of the leader CTA): M = 256 rows, rows
 * 0..127 of A from the leader's shared memory and 128..255 from the peer's
 * at the same offsets; B's N columns split in halves the same way; each
 * CTA's TMEM receives its 128 rows of D. */
__device__ __forceinline__ void mma_f16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                             uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

/* The pair MMA with 8-bit integer operands and an s32 accumulator. */
__device__ __forceinline__ void mma_i8_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

/* Arrive once on the mbarrier at this shared-memory offset in every CTA of
 * `cta_mask` when all prior pair MMAs of this thread have completed. */
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar, uint16_t cta_mask) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64"
      " [%0], %1;" ::"r"(smem_u32(bar)),
      "h"(cta_mask)
      : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

/* D[tmem] (+)= A[smem] * B[smem]; kind::f16 covers f16 and bf16 operands
 * with an f32 accumulator. */
__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

/* D[tmem] (+)= A[smem] * B[smem]; 8-bit integer operands, s32 accumulator. */
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

/* Arrive on `bar` once all previously issued tcgen05.mma of this thread
 * have completed. */
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}

/* 32 lanes x 32 consecutive 32-bit columns: thread i of the warp receives
 * lane (base + i), columns [col, col + 32). */
__device__ __forceinline__ void tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

/* 32 lanes x 32 consecutive 32-bit columns written from registers: thread
 * i of the warp writes lane (base + i), columns [col, col + 32). */
__device__ __forceinline__ void tmem_st_32x32b_x32(uint32_t taddr, const uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], "
      "{%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, "
      "%17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(
          taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]),
      "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]),
      "r"(r[29]), "r"(r[30]), "r"(r[31])
      : "memory");
}

__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

/* ------------------------------------------------------- descriptors -- */

/* Shared-memory matrix descriptor with sm_100 version bits (46-47 = 1) and a
 * swizzle layout (bits 61-63: 2 = 128B, 4 = 64B).  Offsets in bytes.
 *   K-major:  LBO unused (16), SBO = 8 rows x row bytes (1024 for 128B,
 *             512 for 64B swizzle)
 *   MN-major (128B): LBO = byte distance between 64-element MN blocks,
 *             SBO = 1024 (8 K-rows x 128 B) */
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo,
                                              uint32_t layout) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(layout & 7u) << 61;
  return d;
}

/* SWIZZLE_128B (layout 2) form used by the 16-bit paths.  (The int8 path
 * uses SWIZZLE_64B, layout 4: K-major rows of 64 bytes, SBO = 512.) */
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return smem_desc(saddr, lbo, sbo, 2);
}

/* Instruction descriptor (kind::f16 / kind::i8, dense).
 *   c_fmt: 1 = f32, 2 = s32 accumulator;  ab_fmt: f16 = 0, bf16 = 1 (kind::f16),
 *   u8 = 0, s8 = 1 (kind::i8);  a_mn/b_mn: operand is MN-major;
 *   neg_a: negate A (f16 kinds only). */
__host__ __device__ constexpr uint32_t make_idesc(uint32_t c_fmt, uint32_t ab_fmt, bool a_mn,
                                                  bool b_mn, uint32_t M, uint32_t N,
                                                  bool neg_a = false) {
  return (c_fmt << 4) | (ab_fmt << 7) | (ab_fmt << 10) | ((neg_a ? 1u : 0u) << 13) |
         ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) | ((N >> 3) << 17) |
         ((M >> 4) << 24);
}

/* ------------------------------------------------ split-BF16 recipes --
 * One plane pair per product: A plane pa(i) x B plane pb(i) -> accumulator
 * pacc(i); first(i) marks the first product written to its accumulator. */

/* bf16x3: lo*hi + hi*lo into accumulator 1, hi*hi into accumulator 0
 * (lo*lo dropped).  Keeping the correction terms (2^-8 smaller) apart from
 * the leading term keeps them from being truncated against it. */
struct RecipeBf16x3 {
  static constexpr int NA = 2, NB = 2, NP = 3, NACC = 2;
  static constexpr bool P3D = false;
  __host__ __device__ static constexpr int pa(int i) { return i == 0 ? 1 : 0; }
  __host__ __device__ static constexpr int pb(int i) { return i == 1 ? 1 : 0; }
  __host__ __device__ static constexpr int pacc(int i) { return i == 2 ? 0 : 1; }
  __host__ __device__ static constexpr bool first(int i) { return i == 0 || i == 2; }
};
/* bf16x6: three-way split, every product of total order <= 2; hi*hi into
 * accumulator 0, the five correction products into accumulator 1 */
struct RecipeBf16x6 {
  static constexpr int NA = 3, NB = 3, NP = 6, NACC = 2;
  static constexpr bool P3D = false;
  __host__ __device__ static constexpr int pa(int i) {
    return i == 0 ? 2 : i == 1 ? 1 : i == 2 ? 0 : i == 3 ? 1 : 0;
  }
  __host__ __device__ static constexpr int pb(int i) {
    return i == 0 ? 0 : i == 1 ? 1 : i == 2 ? 2 : i == 3 ? 0 : i == 4 ? 1 : 0;
  }
  __host__ __device__ static constexpr int pacc(int i) { return i == 5 ? 0 : 1; }
  __host__ __device__ static constexpr bool first(int i) { return i == 0 || i == 5; }
};

}  // namespace tc
}  // namespace hcbk

#endif /* HCBLAS_B200_TC_COMMON_CUH_ */
