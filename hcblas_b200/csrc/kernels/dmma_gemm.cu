/*
 * dmma_gemm.cu -- native FP64 DGEMM on the FP64 tensor path of sm_100a
 * (warp-level mma.sync .f64, m16n8k4), the plain DGEMM of this library
 * (reference: lib/src/blas/dgemm/dgemm_*kernels*.cpp, one HCC tile kernel per
 * layout and size bucket).
 *
 * Why the tensor path for FP64: B200's FP64 rate is the same on the CUDA
 * cores and through DMMA, but one m16n8k4 instruction does 512 multiply-adds
 * from 3 operand registers per lane where the CUDA-core form needs 16 DFMA
 * instructions and 32 register reads; the shared-memory traffic per flop
 * drops 4x, which leaves issue slots for loads and lets one CTA per SM keep
 * the FP64 pipe busy.
 *
 * Design: 128 x 128 CTA tiles, 256 threads = 8 warps as 2 (M) x 4 (N), each
 * warp a 64 x 32 block = 4 x 4 m16n8 accumulators (64 doubles per lane),
 * multiplied with m16n8k16 DMMAs (one instruction per 16 K where m16n8k4
 * needs four).  K advances in slabs of 32 through a 3-stage ring of
 * shared-memory stages filled by cp.async (16-byte copies where the operand
 * is 16-byte aligned with an even leading dimension, 8-byte copies
 * otherwise; zero fill outside the matrix): an MN-contiguous operand is
 * kept as [k][mn] (row pitch 132 doubles), a K-contiguous one as [mn][k]
 * (row pitch 36), so that each is copied along its contiguous dimension
 * and the 16 lanes of a half-warp reading a fragment hit 16 distinct bank
 * pairs in either layout.  Any shape, leading dimension, offset and
 * alignment runs here; batches (strided or pointer arrays) take
 * blockIdx.y.  Epilogue: alpha * acc + beta * C in registers, beta == 0
 * never reads C.
 *
 * Fragment layout of mma.sync.aligned.m16n8k4.row.col.f64 (PTX ISA, "matrix
 * fragments for mma.m16n8k4 .f64"): lane = 4 g + t; A (16 x 4, row):
 * a0 = A[g][t], a1 = A[g + 8][t]; B (4 x 8, col): b0 = B[t][g];
 * C (16 x 8): c0, c1 = C[g][2t], C[g][2t + 1]; c2, c3 = C[g + 8][2t],
 * C[g + 8][2t + 1].
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "hcbk.h"

namespace hcbk {
namespace {

constexpr int BM = 128, BN = 128, BK = 32;
constexpr int NT = 256;
constexpr int LDS = BM + 4; /* doubles per [k][mn] row: a half-warp's fragment loads hit 16 banks */
constexpr int LDK = BK + 4; /* doubles per [mn][k] row: the same for the K-contiguous layout */
/* doubles per operand and stage (the larger of the two layouts) */
constexpr int OPD = BK * LDS > BM * LDK ? BK * LDS : BM * LDK;
constexpr int DSTAGES = 3; /* cp.async ring depth */
constexpr int DNT = 256;        /* DGEMM: 8 warps as 2 (M) x 4 (N) */
constexpr int WM = 64, WN = 32; /* warp tile */
constexpr int MT = WM / 16, NTL = WN / 8; /* m16 x n8 accumulators per warp */

struct DmmaParams {
  int64_t m, n, k;
  const double *a;
  int64_t lda, sa, a_off;
  const double *b;
  int64_t ldb, sb, b_off;
  double *c;
  int64_t ldc, sc, c_off;
  const double *const *a_arr;
  const double *const *b_arr;
  double *const *c_arr;
  const int32_t *sel;
  int64_t batch;
  double alpha, beta;
  int beta_nonzero;
};

/* m16n8k16: a[2i] = A[g][t + 4i], a[2i + 1] = A[g + 8][t + 4i], b[i] = B[t + 4i][g]
 * (the m16n8k4 fragments of the four K quarters side by side; checked lane
 * by lane against a CPU product on B200) */
__device__ __forceinline__ void dmma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, "
      "{%4, %5, %6, %7, %8, %9, %10, %11}, {%12, %13, %14, %15}, {%0, %1, %2, %3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

struct alignas(16) D2 {
  double v[2];
};

/* shared-memory address of a generic pointer */
__device__ __forceinline__ uint32_t sptr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
/* asynchronous global -> shared copies; `bytes` of the source are read and
 * the rest of the destination is zero-filled (bytes = 0: nothing is read) */
__device__ __forceinline__ void cp_async16(void *dst, const void *src, int bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sptr(dst)), "l"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sptr(dst)), "l"(src),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

/* one operand's K slab of a stage: an MN-contiguous operand as [k][mn]
 * (pitch LDS), a K-contiguous one as [mn][k] (pitch LDK); either is copied
 * along its contiguous dimension, two doubles per copy (16-byte copies when
 * the operand allows, else two 8-byte ones), zero outside the matrix */
template <bool MN>
__device__ __forceinline__ void load_slab(double *dst, const double *X, int64_t ld, int64_t rows,
                                          int64_t K, int64_t r0, int64_t k0, bool vec, int tid) {
#pragma unroll
  for (int v = 0; v < (BM * BK) / (2 * DNT); ++v) {
    const int idx = tid + v * DNT;
    int64_t grow, gk;
    int off, nvalid;
    const double *src;
    if (MN) { /* 16 k rows of 64 pairs */
      const int mn = (idx % (BM / 2)) * 2, kk = idx / (BM / 2);
      grow = r0 + mn;
      gk = k0 + kk;
      src = X + grow + gk * ld;
      off = kk * LDS + mn;
      const int64_t left = rows - grow;
      nvalid = gk < K ? (left >= 2 ? 2 : left > 0 ? (int)left : 0) : 0;
    } else { /* 128 rows of 8 pairs */
      const int mn = idx / (BK / 2), kk = (idx % (BK / 2)) * 2;
      grow = r0 + mn;
      gk = k0 + kk;
      src = X + gk + grow * ld;
      off = mn * LDK + kk;
      const int64_t left = K - gk;
      nvalid = grow < rows ? (left >= 2 ? 2 : left > 0 ? (int)left : 0) : 0;
    }
    if (vec) {
      cp_async16(dst + off, nvalid ? src : X, nvalid * 8);
    } else {
      cp_async8(dst + off, nvalid >= 1 ? src : X, nvalid >= 1 ? 8 : 0);
      cp_async8(dst + off + 1, nvalid >= 2 ? src + 1 : X, nvalid >= 2 ? 8 : 0);
    }
  }
}

/*
 * OP_A / OP_B: 0 = N, 1 = T (column-major canonical; FP64 has no conjugate).
 *   op(A) MN-contiguous iff OP_A == N;  op(B) K-contiguous iff OP_B == N.
 * K slabs of 16 go through a DSTAGES-deep ring of shared-memory stages
 * filled by cp.async: while one slab is multiplied, the next DSTAGES - 1
 * are in flight, and one barrier per slab both publishes the landed slab
 * and frees the stage that the next copies overwrite.
 */
template <int OP_A, int OP_B>
__global__ void __launch_bounds__(DNT, 1) dmma_gemm_kernel(const DmmaParams p) {
  constexpr bool A_MN = (OP_A == HCBK_OP_N);
  constexpr bool B_MN = (OP_B != HCBK_OP_N);
  extern __shared__ __align__(16) double dmma_smem[];

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 1) * WM, wn = (warp >> 1) * WN;

  /* tile rasterisation: bands of 8 M-tiles for L2 reuse of B panels */
  const int64_t tiles_m = (p.m + BM - 1) / BM;
  const int64_t tiles_n = (p.n + BN - 1) / BN;
  const int64_t lin = blockIdx.x;
  constexpr int64_t BAND = 8;
  const int64_t per_band = BAND * tiles_n;
  const int64_t band = lin / per_band;
  const int64_t first_m = band * BAND;
  const int64_t band_h = (tiles_m - first_m) < BAND ? (tiles_m - first_m) : BAND;
  const int64_t in_band = lin - band * per_band;
  const int64_t m0 = (first_m + in_band % band_h) * BM;
  const int64_t n0 = (in_band / band_h) * BN;

  for (int64_t bidx = blockIdx.y; bidx < p.batch; bidx += gridDim.y) {
    if (p.sel && p.sel[bidx] == 0) continue; /* uniform across the block */
    const double *A = (p.a_arr ? p.a_arr[bidx] : p.a) + p.a_off + bidx * p.sa;
    const double *B = (p.b_arr ? p.b_arr[bidx] : p.b) + p.b_off + bidx * p.sb;
    double *C = (p.c_arr ? p.c_arr[bidx] : p.c) + p.c_off + bidx * p.sc;
    const bool vec_a = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) && ((p.lda & 1) == 0);
    const bool vec_b = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) && ((p.ldb & 1) == 0);
    const int64_t ktiles = (p.k + BK - 1) / BK;

    auto load_stage = [&](int slot, int64_t kt) {
      double *sa = dmma_smem + slot * 2 * OPD, *sb = sa + OPD;
      load_slab<A_MN>(sa, A, p.lda, p.m, p.k, m0, kt * BK, vec_a, tid);
      load_slab<B_MN>(sb, B, p.ldb, p.n, p.k, n0, kt * BK, vec_b, tid);
    };

    double acc[MT][NTL][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NTL; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

#pragma unroll
    for (int s = 0; s < DSTAGES - 1; ++s) {
      if (s < ktiles) load_stage(s, s);
      cp_async_commit();
    }
    for (int64_t kt = 0; kt < ktiles; ++kt) {
      cp_async_wait<DSTAGES - 2>(); /* this thread's copies of slab kt have landed */
      __syncthreads();              /* everyone's; and slab kt - 1 is no longer read */
      if (kt + DSTAGES - 1 < ktiles) load_stage((int)((kt + DSTAGES - 1) % DSTAGES), kt + DSTAGES - 1);
      cp_async_commit();
      const double *As = dmma_smem + (int)(kt % DSTAGES) * 2 * OPD, *Bs = As + OPD;
#pragma unroll
      for (int k16 = 0; k16 < BK; k16 += 16) {
        double af[MT][8];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          const int r = wm + 16 * i + g;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int kk = k16 + t + 4 * q;
            af[i][2 * q] = A_MN ? As[kk * LDS + r] : As[r * LDK + kk];
            af[i][2 * q + 1] = A_MN ? As[kk * LDS + r + 8] : As[(r + 8) * LDK + kk];
          }
        }
#pragma unroll
        for (int j = 0; j < NTL; ++j) {
          const int c = wn + 8 * j + g;
          double bf[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int kk = k16 + t + 4 * q;
            bf[q] = B_MN ? Bs[kk * LDS + c] : Bs[c * LDK + kk];
          }
#pragma unroll
          for (int i = 0; i < MT; ++i) dmma16(acc[i][j], af[i], bf);
        }
      }
    }
    cp_async_wait<0>(); /* only empty groups remain */

    /* epilogue: c0, c1 at (g, 2t), (g, 2t + 1); c2, c3 at row g + 8 */
    const bool rd = p.beta_nonzero != 0;
#pragma unroll
    for (int i = 0; i < MT; ++i) {
#pragma unroll
      for (int j = 0; j < NTL; ++j) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int64_t row = m0 + wm + 16 * i + g + (e >> 1) * 8;
          const int64_t col = n0 + wn + 8 * j + 2 * t + (e & 1);
          if (row < p.m && col < p.n) {
            double *dst = C + row + col * p.ldc;
            const double o = p.alpha * acc[i][j][e];
            *dst = rd ? fma(p.beta, *dst, o) : o;
          }
        }
      }
    }
    if (p.batch > 1) __syncthreads(); /* the stages are reused by the next entry */
  }
}

/*
 * Native ZGEMM on the same FP64 tensor path: the complex product is four
 * real products per fragment set, Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br
 * (the 4M form), on m16n8k16 DMMAs.  128 x 64 CTA tiles, 8 warps as 4 (M) x
 * 2 (N), warp tiles 32 x 32 = 2 x 4 m16n8 accumulator pairs.  K advances in
 * slabs of 16 complex elements through a 3-stage ring filled by cp.async,
 * one 16-byte copy per element (two 8-byte ones for an operand that is only
 * 8-byte aligned), complex values kept interleaved: an MN-contiguous operand
 * as [k][mn] (pitch ZBM + 2 or ZBN + 2 elements), a K-contiguous one as
 * [mn][k] (pitch 20), so that each quarter-warp's 16-byte fragment loads --
 * real and imaginary part together -- hit 8 distinct bank groups.
 * Conjugation is applied to the fragments.
 */
constexpr int ZBM = 128, ZBN = 64, ZBK = 16;
constexpr int ZSTAGES = 3;
constexpr int ZLDA = ZBM + 2, ZLDB = ZBN + 2; /* [k][mn] pitches (complex elements) */
constexpr int ZLDK = ZBK + 4;                 /* [mn][k] pitch */
constexpr int ZOPA = ZBK * ZLDA > ZBM * ZLDK ? ZBK * ZLDA : ZBM * ZLDK; /* per stage */
constexpr int ZOPB = ZBK * ZLDB > ZBN * ZLDK ? ZBK * ZLDB : ZBN * ZLDK;
constexpr int ZWM = 32, ZWN = 32, ZMT = ZWM / 16, ZNT = ZWN / 8;

struct ZmmaParams {
  int64_t m, n, k;
  const double2 *a;
  int64_t lda, sa, a_off;
  const double2 *b;
  int64_t ldb, sb, b_off;
  double2 *c;
  int64_t ldc, sc, c_off;
  const double2 *const *a_arr;
  const double2 *const *b_arr;
  double2 *const *c_arr;
  const int32_t *sel;
  int64_t batch;
  double2 alpha, beta;
  int beta_nonzero;
};

/* one operand's slab of complex elements into a stage (see load_slab) */
template <bool MN, int ROWS>
__device__ __forceinline__ void zload_slab(double2 *dst, const double2 *X, int64_t ld,
                                           int64_t rows, int64_t K, int64_t r0, int64_t k0,
                                           bool vec, int tid) {
  constexpr int PITCH_MN = ROWS + 2;
#pragma unroll
  for (int v = 0; v < (ROWS * ZBK) / NT; ++v) {
    const int idx = tid + v * NT;
    int mn, kk, off;
    if (MN) {
      mn = idx % ROWS;
      kk = idx / ROWS;
      off = kk * PITCH_MN + mn;
    } else {
      mn = idx / ZBK;
      kk = idx % ZBK;
      off = mn * ZLDK + kk;
    }
    const int64_t grow = r0 + mn, gk = k0 + kk;
    const bool ok = grow < rows && gk < K;
    const double2 *src = ok ? (MN ? X + grow + gk * ld : X + gk + grow * ld) : X;
    if (vec) {
      cp_async16(dst + off, src, ok ? 16 : 0);
    } else {
      const double *s = reinterpret_cast<const double *>(src);
      double *d = reinterpret_cast<double *>(dst + off);
      cp_async8(d, s, ok ? 8 : 0);
      cp_async8(d + 1, ok ? s + 1 : s, ok ? 8 : 0);
    }
  }
}

template <int OP_A, int OP_B>
__global__ void __launch_bounds__(NT, 1) zmma_gemm_kernel(const ZmmaParams p) {
  constexpr bool A_MN = (OP_A == HCBK_OP_N);
  constexpr bool B_MN = (OP_B != HCBK_OP_N);
  constexpr bool CJ_A = (OP_A == HCBK_OP_C);
  constexpr bool CJ_B = (OP_B == HCBK_OP_C);
  extern __shared__ __align__(16) double zmma_smem[];
  double2 *zs = reinterpret_cast<double2 *>(zmma_smem);

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp & 3) * ZWM, wn = (warp >> 2) * ZWN;

  const int64_t tiles_m = (p.m + ZBM - 1) / ZBM;
  const int64_t tiles_n = (p.n + ZBN - 1) / ZBN;
  const int64_t lin = blockIdx.x;
  constexpr int64_t BAND = 8;
  const int64_t per_band = BAND * tiles_n;
  const int64_t band = lin / per_band;
  const int64_t first_m = band * BAND;
  const int64_t band_h = (tiles_m - first_m) < BAND ? (tiles_m - first_m) : BAND;
  const int64_t in_band = lin - band * per_band;
  const int64_t m0 = (first_m + in_band % band_h) * ZBM;
  const int64_t n0 = (in_band / band_h) * ZBN;

  for (int64_t bidx = blockIdx.y; bidx < p.batch; bidx += gridDim.y) {
    if (p.sel && p.sel[bidx] == 0) continue; /* uniform across the block */
    const double2 *A = (p.a_arr ? p.a_arr[bidx] : p.a) + p.a_off + bidx * p.sa;
    const double2 *B = (p.b_arr ? p.b_arr[bidx] : p.b) + p.b_off + bidx * p.sb;
    double2 *C = (p.c_arr ? p.c_arr[bidx] : p.c) + p.c_off + bidx * p.sc;
    const bool vec_a = (reinterpret_cast<uintptr_t>(A) & 15) == 0;
    const bool vec_b = (reinterpret_cast<uintptr_t>(B) & 15) == 0;
    const int64_t ktiles = (p.k + ZBK - 1) / ZBK;

    auto load_stage = [&](int slot, int64_t kt) {
      double2 *sa = zs + slot * (ZOPA + ZOPB), *sb = sa + ZOPA;
      zload_slab<A_MN, ZBM>(sa, A, p.lda, p.m, p.k, m0, kt * ZBK, vec_a, tid);
      zload_slab<B_MN, ZBN>(sb, B, p.ldb, p.n, p.k, n0, kt * ZBK, vec_b, tid);
    };

    double cr[ZMT][ZNT][4], ci[ZMT][ZNT][4];
#pragma unroll
    for (int i = 0; i < ZMT; ++i)
#pragma unroll
      for (int j = 0; j < ZNT; ++j)
#pragma unroll
        for (int e = 0; e < 4; ++e) cr[i][j][e] = ci[i][j][e] = 0.0;

#pragma unroll
    for (int s = 0; s < ZSTAGES - 1; ++s) {
      if (s < ktiles) load_stage(s, s);
      cp_async_commit();
    }
    for (int64_t kt = 0; kt < ktiles; ++kt) {
      cp_async_wait<ZSTAGES - 2>();
      __syncthreads();
      if (kt + ZSTAGES - 1 < ktiles)
        load_stage((int)((kt + ZSTAGES - 1) % ZSTAGES), kt + ZSTAGES - 1);
      cp_async_commit();
      const double2 *As = zs + (int)(kt % ZSTAGES) * (ZOPA + ZOPB), *Bs = As + ZOPA;
#pragma unroll
      for (int i = 0; i < ZMT; ++i) {
        const int r = wm + 16 * i + g;
        /* real parts, and the imaginary parts both ways round: ai for the
         * imaginary accumulator, -ai for the real one */
        double ar[8], ai[8], nai[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int kk = t + 4 * q;
          const double2 x0 = A_MN ? As[kk * ZLDA + r] : As[r * ZLDK + kk];
          const double2 x1 = A_MN ? As[kk * ZLDA + r + 8] : As[(r + 8) * ZLDK + kk];
          ar[2 * q] = x0.x;
          ar[2 * q + 1] = x1.x;
          ai[2 * q] = CJ_A ? -x0.y : x0.y;
          ai[2 * q + 1] = CJ_A ? -x1.y : x1.y;
          nai[2 * q] = -ai[2 * q];
          nai[2 * q + 1] = -ai[2 * q + 1];
        }
#pragma unroll
        for (int j = 0; j < ZNT; ++j) {
          const int c = wn + 8 * j + g;
          double br[4], bi[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int kk = t + 4 * q;
            const double2 y = B_MN ? Bs[kk * ZLDB + c] : Bs[c * ZLDK + kk];
            br[q] = y.x;
            bi[q] = CJ_B ? -y.y : y.y;
          }
          dmma16(cr[i][j], ar, br);
          dmma16(cr[i][j], nai, bi);
          dmma16(ci[i][j], ar, bi);
          dmma16(ci[i][j], ai, br);
        }
      }
    }
    cp_async_wait<0>();

    const bool rd = p.beta_nonzero != 0;
#pragma unroll
    for (int i = 0; i < ZMT; ++i) {
#pragma unroll
      for (int j = 0; j < ZNT; ++j) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int64_t row = m0 + wm + 16 * i + g + (e >> 1) * 8;
          const int64_t col = n0 + wn + 8 * j + 2 * t + (e & 1);
          if (row < p.m && col < p.n) {
            double2 *dst = C + row + col * p.ldc;
            const double re = cr[i][j][e], im = ci[i][j][e];
            double2 o;
            o.x = p.alpha.x * re - p.alpha.y * im;
            o.y = p.alpha.x * im + p.alpha.y * re;
            if (rd) {
              const double2 cv = *dst;
              o.x += p.beta.x * cv.x - p.beta.y * cv.y;
              o.y += p.beta.x * cv.y + p.beta.y * cv.x;
            }
            *dst = o;
          }
        }
      }
    }
    if (p.batch > 1) __syncthreads(); /* the stages are reused by the next entry */
  }
}

}  // namespace
}  // namespace hcbk

using namespace hcbk;

extern "C" int hcbk_dgemm_dmma(const hcbk_gemm_args *a, void *stream) {
  if (a->dtype != HCBK_D || a->m <= 0 || a->n <= 0 || a->k <= 0 || a->batch <= 0 ||
      a->op_a == HCBK_OP_C || a->op_b == HCBK_OP_C)
    return HCBK_ERR_ARGS;
  DmmaParams p;
  p.m = a->m;
  p.n = a->n;
  p.k = a->k;
  p.a = static_cast<const double *>(a->a);
  p.lda = a->lda;
  p.sa = a->stride_a;
  p.a_off = a->a_off;
  p.b = static_cast<const double *>(a->b);
  p.ldb = a->ldb;
  p.sb = a->stride_b;
  p.b_off = a->b_off;
  p.c = static_cast<double *>(a->c);
  p.ldc = a->ldc;
  p.sc = a->stride_c;
  p.c_off = a->c_off;
  p.a_arr = reinterpret_cast<const double *const *>(a->a_array);
  p.b_arr = reinterpret_cast<const double *const *>(a->b_array);
  p.c_arr = reinterpret_cast<double *const *>(a->c_array);
  p.sel = a->batch_select;
  p.batch = a->batch;
  p.alpha = a->alpha_re;
  p.beta = a->beta_re;
  p.beta_nonzero = a->beta_re != 0.0;
  const int64_t tiles = ((a->m + BM - 1) / BM) * ((a->n + BN - 1) / BN);
  if (tiles > 0x7fffffffLL) return HCBK_ERR_ARGS;
  dim3 grid((unsigned)tiles, (unsigned)(a->batch < 65535 ? a->batch : 65535), 1);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  constexpr int smem = DSTAGES * 2 * OPD * (int)sizeof(double); /* the ring of A and B slabs */
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  auto kern = (a->op_a == HCBK_OP_N && a->op_b == HCBK_OP_N) ? dmma_gemm_kernel<0, 0>
              : (a->op_a == HCBK_OP_N)                        ? dmma_gemm_kernel<0, 1>
              : (a->op_b == HCBK_OP_N)                        ? dmma_gemm_kernel<1, 0>
                                                              : dmma_gemm_kernel<1, 1>;
  if (!attr_set[dev]) {
    for (auto k : {dmma_gemm_kernel<0, 0>, dmma_gemm_kernel<0, 1>, dmma_gemm_kernel<1, 0>,
                   dmma_gemm_kernel<1, 1>})
      if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
          cudaSuccess)
        return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  kern<<<grid, DNT, smem, st>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_zgemm_zmma(const hcbk_gemm_args *a, void *stream) {
  if (a->dtype != HCBK_Z || a->m <= 0 || a->n <= 0 || a->k <= 0 || a->batch <= 0)
    return HCBK_ERR_ARGS;
  ZmmaParams p;
  p.m = a->m;
  p.n = a->n;
  p.k = a->k;
  p.a = static_cast<const double2 *>(a->a);
  p.lda = a->lda;
  p.sa = a->stride_a;
  p.a_off = a->a_off;
  p.b = static_cast<const double2 *>(a->b);
  p.ldb = a->ldb;
  p.sb = a->stride_b;
  p.b_off = a->b_off;
  p.c = static_cast<double2 *>(a->c);
  p.ldc = a->ldc;
  p.sc = a->stride_c;
  p.c_off = a->c_off;
  p.a_arr = reinterpret_cast<const double2 *const *>(a->a_array);
  p.b_arr = reinterpret_cast<const double2 *const *>(a->b_array);
  p.c_arr = reinterpret_cast<double2 *const *>(a->c_array);
  p.sel = a->batch_select;
  p.batch = a->batch;
  p.alpha = make_double2(a->alpha_re, a->alpha_im);
  p.beta = make_double2(a->beta_re, a->beta_im);
  p.beta_nonzero = a->beta_re != 0.0 || a->beta_im != 0.0;
  const int64_t tiles = ((a->m + ZBM - 1) / ZBM) * ((a->n + ZBN - 1) / ZBN);
  if (tiles > 0x7fffffffLL) return HCBK_ERR_ARGS;
  dim3 grid((unsigned)tiles, (unsigned)(a->batch < 65535 ? a->batch : 65535), 1);
  constexpr int smem = ZSTAGES * (ZOPA + ZOPB) * (int)sizeof(double2); /* the ring */
  using K = void (*)(const ZmmaParams);
  static const K table[3][3] = {
      {zmma_gemm_kernel<0, 0>, zmma_gemm_kernel<0, 1>, zmma_gemm_kernel<0, 2>},
      {zmma_gemm_kernel<1, 0>, zmma_gemm_kernel<1, 1>, zmma_gemm_kernel<1, 2>},
      {zmma_gemm_kernel<2, 0>, zmma_gemm_kernel<2, 1>, zmma_gemm_kernel<2, 2>}};
  if (a->op_a < 0 || a->op_a > 2 || a->op_b < 0 || a->op_b > 2) return HCBK_ERR_ARGS;
  static bool attr_set[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HCBK_ERR_LAUNCH;
  if (!attr_set[dev]) {
    for (int x = 0; x < 3; ++x)
      for (int y = 0; y < 3; ++y)
        if (cudaFuncSetAttribute(table[x][y], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 smem) != cudaSuccess)
          return HCBK_ERR_LAUNCH;
    attr_set[dev] = true;
  }
  table[a->op_a][a->op_b]<<<grid, NT, smem, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
