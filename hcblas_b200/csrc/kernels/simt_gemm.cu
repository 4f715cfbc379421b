/*
 * simt_gemm.cu -- plain GEMM on the CUDA cores of sm_100a.
 *
 * Covers every case the reference's per-dtype HCC tile kernels cover
 * (lib/src/blas/{s,d,h,c,z}gemm/*kernels*.cpp: col-major NN/NT/TN/TT with
 * ld/offsets, pointer-array batches), in one templated kernel family:
 *
 *   S   binary32 FMA               (reference: sgemm_NN_kernels.cpp:26-136 ...)
 *   D   binary64 FMA               (dgemm_*kernels*.cpp)
 *   C   complex binary32, 4 real FMAs per complex MAC (cgemm_array_kernels.cpp)
 *   Z   complex binary64           (zgemm_*)
 *   H   binary16 storage, binary32 accumulation (the reference accumulates in
 *       half, hgemm_NN_kernels.cpp:40; this library deliberately does not)
 *
 * Design (B200):
 *   - 256 threads per CTA, a BM x BN output tile, K stepped by BK through two
 *     shared-memory buffers; the next K-slab is fetched into registers with
 *     128-bit loads while the current slab is multiplied (register
 *     prefetch -> one barrier per K-step).
 *   - Each operand is read along its contiguous dimension whatever op() is
 *     (MN-contiguous or K-contiguous) and written to shared memory as
 *     [k][mn], so the FMA loop is identical for all 9 op(A) x op(B) cases;
 *     conjugation is applied once, on the load.
 *   - Each thread owns TM x TN outputs split into 16-byte groups so that the
 *     shared-memory fragment reads are conflict-free 128-bit loads.
 *   - FP32 8 x 8 fragments run on the packed FMA (fma.rn.f32x2, two columns
 *     per instruction): the FMA pipe stays as busy with half the issue slots,
 *     which go to the fragment loads instead.
 *   - Epilogue: alpha * acc + beta * C in registers with 16-byte vector
 *     loads/stores of C when aligned; beta == 0 never reads C (CBLAS).
 *   - Out-of-range rows/columns/k are zero-filled on load, so ragged edges
 *     need no special kernel; misaligned operands fall back to scalar loads
 *     (decided per CTA from the actual pointer, so pointer-array batches with
 *     mixed alignment are handled).
 *   - Tiles are rasterised in bands of 8 M-tiles for L2 reuse of B panels.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "hcbk.h"

namespace hcbk {
namespace {

/* ---------------------------------------------------------------- types -- */

template <typename T> struct AccOf;
template <> struct AccOf<float> { using type = float; };
template <> struct AccOf<double> { using type = double; };
template <> struct AccOf<float2> { using type = float2; };
template <> struct AccOf<double2> { using type = double2; };
template <> struct AccOf<__half> { using type = float; };

template <typename A> __device__ __forceinline__ A zero_of();
template <> __device__ __forceinline__ float zero_of<float>() { return 0.f; }
template <> __device__ __forceinline__ double zero_of<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 zero_of<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 zero_of<double2>() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ float to_acc(float v, bool) { return v; }
__device__ __forceinline__ double to_acc(double v, bool) { return v; }
__device__ __forceinline__ float to_acc(__half v, bool) { return __half2float(v); }
__device__ __forceinline__ float2 to_acc(float2 v, bool cj) { return cj ? make_float2(v.x, -v.y) : v; }
__device__ __forceinline__ double2 to_acc(double2 v, bool cj) { return cj ? make_double2(v.x, -v.y) : v; }

/* c += a * b */
__device__ __forceinline__ void mac(float &c, float a, float b) { c = fmaf(a, b, c); }
__device__ __forceinline__ void mac(double &c, double a, double b) { c = fma(a, b, c); }
__device__ __forceinline__ void mac(float2 &c, float2 a, float2 b) {
  c.x = fmaf(a.x, b.x, c.x);
  c.x = fmaf(-a.y, b.y, c.x);
  c.y = fmaf(a.x, b.y, c.y);
  c.y = fmaf(a.y, b.x, c.y);
}
__device__ __forceinline__ void mac(double2 &c, double2 a, double2 b) {
  c.x = fma(a.x, b.x, c.x);
  c.x = fma(-a.y, b.y, c.x);
  c.y = fma(a.x, b.y, c.y);
  c.y = fma(a.y, b.x, c.y);
}

/* The FP32 outer-product step on the packed FMA: row i of the thread's
 * accumulators += a_i * (b_j, b_j+1) two columns per fma.rn.f32x2, each lane
 * rounded as the scalar FMA (the same results, half the FMA instructions). */
template <int TM, int TN>
__device__ __forceinline__ void outer_f32x2(float (&acc)[TM][TN], const float (&af)[TM],
                                            const float (&bf)[TN]) {
  static_assert(TN % 2 == 0, "column pairs");
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    uint64_t a2;
    asm("mov.b64 %0, {%1, %1};" : "=l"(a2) : "f"(af[i]));
#pragma unroll
    for (int j = 0; j < TN; j += 2) {
      uint64_t b2, c2;
      asm("mov.b64 %0, {%1, %2};" : "=l"(b2) : "f"(bf[j]), "f"(bf[j + 1]));
      asm("mov.b64 %0, {%1, %2};" : "=l"(c2) : "f"(acc[i][j]), "f"(acc[i][j + 1]));
      asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(c2) : "l"(a2), "l"(b2));
      asm("mov.b64 {%0, %1}, %2;" : "=f"(acc[i][j]), "=f"(acc[i][j + 1]) : "l"(c2));
    }
  }
}

/* alpha * acc + beta * c */
__device__ __forceinline__ float axpby(float al, float acc, float be, float c, bool rd) {
  return rd ? fmaf(be, c, al * acc) : al * acc;
}
__device__ __forceinline__ double axpby(double al, double acc, double be, double c, bool rd) {
  return rd ? fma(be, c, al * acc) : al * acc;
}
__device__ __forceinline__ float2 axpby(float2 al, float2 acc, float2 be, float2 c, bool rd) {
  float2 r;
  r.x = al.x * acc.x - al.y * acc.y;
  r.y = al.x * acc.y + al.y * acc.x;
  if (rd) {
    r.x += be.x * c.x - be.y * c.y;
    r.y += be.x * c.y + be.y * c.x;
  }
  return r;
}
__device__ __forceinline__ double2 axpby(double2 al, double2 acc, double2 be, double2 c, bool rd) {
  double2 r;
  r.x = al.x * acc.x - al.y * acc.y;
  r.y = al.x * acc.y + al.y * acc.x;
  if (rd) {
    r.x += be.x * c.x - be.y * c.y;
    r.y += be.x * c.y + be.y * c.x;
  }
  return r;
}

/* storage <-> compute for the C tile */
__device__ __forceinline__ float c_load(const float *p) { return *p; }
__device__ __forceinline__ double c_load(const double *p) { return *p; }
__device__ __forceinline__ float2 c_load(const float2 *p) { return *p; }
__device__ __forceinline__ double2 c_load(const double2 *p) { return *p; }
__device__ __forceinline__ float c_load(const __half *p) { return __half2float(*p); }
__device__ __forceinline__ void c_store(float *p, float v) { *p = v; }
__device__ __forceinline__ void c_store(double *p, double v) { *p = v; }
__device__ __forceinline__ void c_store(float2 *p, float2 v) { *p = v; }
__device__ __forceinline__ void c_store(double2 *p, double2 v) { *p = v; }
__device__ __forceinline__ void c_store(__half *p, float v) { *p = __float2half_rn(v); }

template <typename T> struct IsComplex { static constexpr bool value = false; };
template <> struct IsComplex<float2> { static constexpr bool value = true; };
template <> struct IsComplex<double2> { static constexpr bool value = true; };

template <typename A> struct HostScalar;
template <> struct HostScalar<float> {
  static float make(double re, double) { return (float)re; }
};
template <> struct HostScalar<double> {
  static double make(double re, double) { return re; }
};
template <> struct HostScalar<float2> {
  static float2 make(double re, double im) { return make_float2((float)re, (float)im); }
};
template <> struct HostScalar<double2> {
  static double2 make(double re, double im) { return make_double2(re, im); }
};

/* ----------------------------------------------------------- parameters -- */

template <typename T, typename Acc> struct SimtParams {
  int64_t m, n, k;
  const T *a;
  int64_t lda, sa, a_off;
  const T *b;
  int64_t ldb, sb, b_off;
  T *c;
  int64_t ldc, sc, c_off;
  const T *const *a_arr;
  const T *const *b_arr;
  T *const *c_arr;
  int64_t batch;
  const int32_t *sel; /* batch entries to compute (NULL: all) */
  Acc alpha, beta;
  int beta_nonzero;
};

/* 16-byte vector of VW storage elements */
template <typename T, int VW> struct alignas(16) Vec {
  T v[VW];
};

/* ---------------------------------------------------------------- kernel -- */

/* One output tile's problem: op(A) is m x k, op(B) is k x n, C m x n, all
 * column-major with their leading dimensions (pointers already offset). */
template <typename T> struct TileJob {
  int64_t m, n, k;
  const T *A;
  int64_t lda;
  const T *B;
  int64_t ldb;
  T *C;
  int64_t ldc;
};

/* the double-buffered K-slabs of both operands, as [k][mn] */
template <typename Acc, int BM, int BN, int BK> struct SimtSmem {
  static constexpr int PAD = 16 / (int)sizeof(Acc);
  Acc As[2][BK][BM + PAD];
  Acc Bs[2][BK][BN + PAD];
};

/*
 * One BM x BN tile of C = alpha op(A) op(B) + beta C at (m0, n0), computed by
 * the whole block.
 * OP_A / OP_B: 0 = N, 1 = T, 2 = C (column-major canonical).
 *   op(A) MN-contiguous iff OP_A == N;  op(B) K-contiguous iff OP_B == N.
 */
template <typename T, int BM, int BN, int BK, int TM, int TN, int OP_A, int OP_B>
__device__ __forceinline__ void simt_tile(const TileJob<T> &p, typename AccOf<T>::type alpha,
                                          typename AccOf<T>::type beta, bool rd, int64_t m0,
                                          int64_t n0,
                                          SimtSmem<typename AccOf<T>::type, BM, BN, BK> &sm) {
  using Acc = typename AccOf<T>::type;
  constexpr int NT = (BM / TM) * (BN / TN);
  constexpr int VW = 16 / (int)sizeof(T);              /* storage elems / 16 B */
  constexpr int GA = (TM * (int)sizeof(Acc)) / 16;       /* 16-byte groups along m */
  constexpr int GB = (TN * (int)sizeof(Acc)) / 16;
  constexpr int GSA = TM / GA;                           /* elems per group */
  constexpr int GSB = TN / GB;
  constexpr bool A_MN = (OP_A == HCBK_OP_N);
  constexpr bool B_MN = (OP_B != HCBK_OP_N);
  constexpr bool CJ_A = (OP_A == HCBK_OP_C);
  constexpr bool CJ_B = (OP_B == HCBK_OP_C);
  /* vectors per thread for each operand's K-slab */
  constexpr int VA = (BM * BK) / (VW * NT);
  constexpr int VB = (BN * BK) / (VW * NT);
  static_assert(VA * VW * NT == BM * BK, "A slab must split evenly");
  static_assert(VB * VW * NT == BN * BK, "B slab must split evenly");
  static_assert(GA >= 1 && GB >= 1 && GSA * GA == TM && GSB * GB == TN, "fragment groups");
  static_assert(BK % VW == 0 || (A_MN && B_MN), "K-contiguous loads need BK % VW == 0");
  auto &As = sm.As;
  auto &Bs = sm.Bs;

  const int tid = threadIdx.x;
  const int tx = tid % (BM / TM);
  const int ty = tid / (BM / TM);
  const T *A = p.A;
  const T *B = p.B;

  const bool vec_a = ((reinterpret_cast<uintptr_t>(A) & 15) == 0) &&
                     (((p.lda * (int64_t)sizeof(T)) & 15) == 0);
  const bool vec_b = ((reinterpret_cast<uintptr_t>(B) & 15) == 0) &&
                     (((p.ldb * (int64_t)sizeof(T)) & 15) == 0);

  Vec<T, VW> ra[VA];
  Vec<T, VW> rb[VB];

  /* Per-thread load positions inside a K-slab: vector v of A covers
   * (mn, kk) = (a_mn(v) .. + VW, a_kk(v)) for MN-contiguous A, or
   * (a_mn(v), a_kk(v) .. + VW) for K-contiguous A (likewise B).  The source
   * pointers advance by one slab per fetch; bounds are checked against the
   * tile's remaining rows and the slab's remaining K as 32-bit values. */
  auto a_mn = [&](int v) {
    const int idx = tid + v * NT;
    return A_MN ? (idx % (BM / VW)) * VW : idx / (BK / VW);
  };
  auto a_kk = [&](int v) {
    const int idx = tid + v * NT;
    return A_MN ? idx / (BM / VW) : (idx % (BK / VW)) * VW;
  };
  auto b_mn = [&](int v) {
    const int idx = tid + v * NT;
    return B_MN ? (idx % (BN / VW)) * VW : idx / (BK / VW);
  };
  auto b_kk = [&](int v) {
    const int idx = tid + v * NT;
    return B_MN ? idx / (BN / VW) : (idx % (BK / VW)) * VW;
  };
  const int rem_m = (int)((p.m - m0) < BM ? (p.m - m0) : BM);
  const int rem_n = (int)((p.n - n0) < BN ? (p.n - n0) : BN);
  const T *pa[VA];
  const T *pb[VB];
#pragma unroll
  for (int v = 0; v < VA; ++v)
    pa[v] = A_MN ? A + m0 + a_mn(v) + (int64_t)a_kk(v) * p.lda
                 : A + a_kk(v) + (m0 + a_mn(v)) * p.lda;
#pragma unroll
  for (int v = 0; v < VB; ++v)
    pb[v] = B_MN ? B + n0 + b_mn(v) + (int64_t)b_kk(v) * p.ldb
                 : B + b_kk(v) + (n0 + b_mn(v)) * p.ldb;
  const int64_t a_step = A_MN ? (int64_t)BK * p.lda : BK;
  const int64_t b_step = B_MN ? (int64_t)BK * p.ldb : BK;

  /* fetch the next K-slab (starting at k0) into registers, zero-filled */
  auto fetch_ptr = [&](int64_t k0) {
    const int rem_k = (int)((p.k - k0) < BK ? (p.k - k0) : BK);
#pragma unroll
    for (int v = 0; v < VA; ++v) {
      const T *src = pa[v];
      const int mn = a_mn(v), kk = a_kk(v);
      if (A_MN) {
        if (kk < rem_k && mn + VW <= rem_m && vec_a) {
          ra[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e) ra[v].v[e] = (kk < rem_k && mn + e < rem_m) ? src[e] : T();
        }
      } else {
        if (mn < rem_m && kk + VW <= rem_k && vec_a) {
          ra[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e) ra[v].v[e] = (mn < rem_m && kk + e < rem_k) ? src[e] : T();
        }
      }
      pa[v] += a_step;
    }
#pragma unroll
    for (int v = 0; v < VB; ++v) {
      const T *src = pb[v];
      const int mn = b_mn(v), kk = b_kk(v);
      if (B_MN) {
        if (kk < rem_k && mn + VW <= rem_n && vec_b) {
          rb[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e) rb[v].v[e] = (kk < rem_k && mn + e < rem_n) ? src[e] : T();
        }
      } else {
        if (mn < rem_n && kk + VW <= rem_k && vec_b) {
          rb[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e) rb[v].v[e] = (mn < rem_n && kk + e < rem_k) ? src[e] : T();
        }
      }
      pb[v] += b_step;
    }
  };

  /* the same K-slab fetch with positions recomputed from k0 (complex types:
   * measured faster than the advancing pointers at their 64 x 64 tiles) */
  auto fetch_idx = [&](int64_t k0) {
#pragma unroll
    for (int v = 0; v < VA; ++v) {
      const int idx = tid + v * NT;
      int64_t mn, kk;
      if (A_MN) {
        mn = m0 + (int64_t)(idx % (BM / VW)) * VW;
        kk = k0 + idx / (BM / VW);
      } else {
        mn = m0 + idx / (BK / VW);
        kk = k0 + (int64_t)(idx % (BK / VW)) * VW;
      }
      if (A_MN) {
        const T *src = A + mn + kk * p.lda;
        if (kk < p.k && mn + VW <= p.m && vec_a) {
          ra[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e)
            ra[v].v[e] = (kk < p.k && mn + e < p.m) ? src[e] : T();
        }
      } else {
        const T *src = A + kk + mn * p.lda;
        if (mn < p.m && kk + VW <= p.k && vec_a) {
          ra[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e)
            ra[v].v[e] = (mn < p.m && kk + e < p.k) ? src[e] : T();
        }
      }
    }
#pragma unroll
    for (int v = 0; v < VB; ++v) {
      const int idx = tid + v * NT;
      int64_t mn, kk;
      if (B_MN) {
        mn = n0 + (int64_t)(idx % (BN / VW)) * VW;
        kk = k0 + idx / (BN / VW);
      } else {
        mn = n0 + idx / (BK / VW);
        kk = k0 + (int64_t)(idx % (BK / VW)) * VW;
      }
      if (B_MN) {
        const T *src = B + mn + kk * p.ldb;
        if (kk < p.k && mn + VW <= p.n && vec_b) {
          rb[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e)
            rb[v].v[e] = (kk < p.k && mn + e < p.n) ? src[e] : T();
        }
      } else {
        const T *src = B + kk + mn * p.ldb;
        if (mn < p.n && kk + VW <= p.k && vec_b) {
          rb[v] = *reinterpret_cast<const Vec<T, VW> *>(src);
        } else {
#pragma unroll
          for (int e = 0; e < VW; ++e)
            rb[v].v[e] = (mn < p.n && kk + e < p.k) ? src[e] : T();
        }
      }
    }
  };

  auto fetch = [&](int64_t k0) {
    if constexpr (IsComplex<T>::value)
      fetch_idx(k0);
    else
      fetch_ptr(k0);
  };

  /* registers -> shared buffer s, as [k][mn] in the compute type */
  auto stash = [&](int s) {
#pragma unroll
    for (int v = 0; v < VA; ++v) {
      const int idx = tid + v * NT;
      if (A_MN) {
        const int mn = (idx % (BM / VW)) * VW;
        const int kk = idx / (BM / VW);
#pragma unroll
        for (int e = 0; e < VW; ++e) As[s][kk][mn + e] = to_acc(ra[v].v[e], CJ_A);
      } else {
        const int mn = idx / (BK / VW);
        const int kk = (idx % (BK / VW)) * VW;
#pragma unroll
        for (int e = 0; e < VW; ++e) As[s][kk + e][mn] = to_acc(ra[v].v[e], CJ_A);
      }
    }
#pragma unroll
    for (int v = 0; v < VB; ++v) {
      const int idx = tid + v * NT;
      if (B_MN) {
        const int mn = (idx % (BN / VW)) * VW;
        const int kk = idx / (BN / VW);
#pragma unroll
        for (int e = 0; e < VW; ++e) Bs[s][kk][mn + e] = to_acc(rb[v].v[e], CJ_B);
      } else {
        const int mn = idx / (BK / VW);
        const int kk = (idx % (BK / VW)) * VW;
#pragma unroll
        for (int e = 0; e < VW; ++e) Bs[s][kk + e][mn] = to_acc(rb[v].v[e], CJ_B);
      }
    }
  };

  Acc acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = zero_of<Acc>();

  const int64_t ktiles = (p.k + BK - 1) / BK;
  fetch(0);
  stash(0);
  __syncthreads();

  for (int64_t kt = 0; kt < ktiles; ++kt) {
    const int s = (int)(kt & 1);
    if (kt + 1 < ktiles) fetch((kt + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      Acc af[TM], bf[TN];
#pragma unroll
      for (int g = 0; g < GA; ++g) {
        const Acc *src = &As[s][kk][g * (BM / GA) + tx * GSA];
#pragma unroll
        for (int e = 0; e < GSA; ++e) af[g * GSA + e] = src[e];
      }
#pragma unroll
      for (int g = 0; g < GB; ++g) {
        const Acc *src = &Bs[s][kk][g * (BN / GB) + ty * GSB];
#pragma unroll
        for (int e = 0; e < GSB; ++e) bf[g * GSB + e] = src[e];
      }
      /* packed FMA for the 8 x 8 fragments; the 4 x 4 ones measured faster
       * with scalar FMAs (one broadcast move per two packed FMAs) */
      if constexpr (std::is_same<Acc, float>::value && TN >= 8 && TN % 2 == 0) {
        outer_f32x2<TM, TN>(acc, af, bf);
      } else {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) mac(acc[i][j], af[i], bf[j]);
      }
    }
    if (kt + 1 < ktiles) stash(s ^ 1);
    __syncthreads();
  }

  /* ---- epilogue: C = alpha * acc + beta * C ----
   * Each thread's GSA consecutive rows of a column are one contiguous run of
   * C (16 bytes in the compute type; the 16 lanes of a warp row cover 16 such
   * runs back to back), so a whole run is read and written as one vector
   * when it lies inside C and is aligned, element by element otherwise. */
  constexpr int RUN_BYTES = GSA * (int)sizeof(T);
  constexpr bool RUN_VEC = RUN_BYTES == 8 || RUN_BYTES == 16;
#pragma unroll
  for (int j = 0; j < TN; ++j) {
    const int64_t col = n0 + (j / GSB) * (BN / GB) + ty * GSB + (j % GSB);
    if (col >= p.n) continue;
#pragma unroll
    for (int g = 0; g < GA; ++g) {
      const int64_t row0 = m0 + g * (BM / GA) + tx * GSA;
      T *dst0 = p.C + row0 + col * p.ldc;
      if constexpr (RUN_VEC) {
        if (row0 + GSA <= p.m && (reinterpret_cast<uintptr_t>(dst0) & (RUN_BYTES - 1)) == 0) {
          struct alignas(RUN_BYTES) Run { T v[GSA]; };
          Run cr;
          if (rd) cr = *reinterpret_cast<const Run *>(dst0);
          Run out;
#pragma unroll
          for (int e = 0; e < GSA; ++e) {
            const Acc cv = rd ? c_load(&cr.v[e]) : zero_of<Acc>();
            c_store(&out.v[e], axpby(alpha, acc[g * GSA + e][j], beta, cv, rd));
          }
          *reinterpret_cast<Run *>(dst0) = out;
          continue;
        }
      }
#pragma unroll
      for (int e = 0; e < GSA; ++e) {
        if (row0 + e < p.m) {
          T *dst = dst0 + e;
          const Acc cv = rd ? c_load(dst) : zero_of<Acc>();
          c_store(dst, axpby(alpha, acc[g * GSA + e][j], beta, cv, rd));
        }
      }
    }
  }
}

template <typename T, int BM, int BN, int BK, int TM, int TN, int OP_A, int OP_B, int MINB>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), MINB)
simt_gemm_kernel(SimtParams<T, typename AccOf<T>::type> p) {
  using Acc = typename AccOf<T>::type;
  __shared__ __align__(16) SimtSmem<Acc, BM, BN, BK> sm;

  /* ---- tile rasterisation (bands of 8 M-tiles) ---- */
  const int64_t tiles_m = (p.m + BM - 1) / BM;
  const int64_t tiles_n = (p.n + BN - 1) / BN;
  const int64_t lin = blockIdx.x;
  constexpr int64_t BAND = 8;
  const int64_t per_band = BAND * tiles_n;
  const int64_t band = lin / per_band;
  const int64_t first_m = band * BAND;
  const int64_t band_h = (tiles_m - first_m) < BAND ? (tiles_m - first_m) : BAND;
  const int64_t in_band = lin - band * per_band;
  const int64_t tile_m = first_m + in_band % band_h;
  const int64_t tile_n = in_band / band_h;
  const int64_t m0 = tile_m * BM;
  const int64_t n0 = tile_n * BN;

  if (p.sel) {
    /* a selective pass (usually with nothing selected): the block's threads
     * read its entries' flags together and the block leaves when none is set */
    int any = 0;
    for (int64_t b = blockIdx.y + (int64_t)threadIdx.x * gridDim.y; b < p.batch;
         b += (int64_t)gridDim.y * blockDim.x)
      any |= p.sel[b];
    if (!__syncthreads_or(any)) return;
  }
  for (int64_t bidx = blockIdx.y; bidx < p.batch; bidx += gridDim.y) {
    if (p.sel && p.sel[bidx] == 0) continue; /* uniform across the block */
    TileJob<T> j;
    j.m = p.m;
    j.n = p.n;
    j.k = p.k;
    j.A = (p.a_arr ? p.a_arr[bidx] : p.a) + p.a_off + bidx * p.sa;
    j.B = (p.b_arr ? p.b_arr[bidx] : p.b) + p.b_off + bidx * p.sb;
    j.C = (p.c_arr ? p.c_arr[bidx] : p.c) + p.c_off + bidx * p.sc;
    j.lda = p.lda;
    j.ldb = p.ldb;
    j.ldc = p.ldc;
    simt_tile<T, BM, BN, BK, TM, TN, OP_A, OP_B>(j, p.alpha, p.beta, p.beta_nonzero != 0, m0, n0,
                                                 sm);
    if (p.batch > 1) __syncthreads(); /* shared buffers are reused by the next batch entry */
  }
}

/*
 * Persistent grouped GEMM on the CUDA cores: one launch walks the tiles of
 * every problem of a device-side problem table (each its own shape,
 * transposes, leading dimensions and pointers).  Global tile t belongs to the
 * last problem g with tile_start[g] <= t (binary search over the prefix sums
 * of the problems' tile counts); tiles are column-major within a problem.
 * The op(A) x op(B) combination of each problem selects the tile body, so
 * the per-combination code is the same as the single-problem kernel's.
 */
__device__ __forceinline__ int simt_find_problem(const int32_t *ts, int count, int t) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(ts + mid) <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
simt_grouped_kernel(const hcbk_simt_entry *table, const int32_t *tile_start, int count,
                    int total_tiles, typename AccOf<T>::type alpha,
                    typename AccOf<T>::type beta, int beta_nonzero) {
  using Acc = typename AccOf<T>::type;
  __shared__ __align__(16) SimtSmem<Acc, BM, BN, BK> sm;
  for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
    const int g = simt_find_problem(tile_start, count, t);
    const hcbk_simt_entry *e = table + g;
    const int lt = t - __ldg(tile_start + g);
    const int tiles_m = __ldg(&e->tiles_m);
    const int64_t m0 = (int64_t)(lt % tiles_m) * BM, n0 = (int64_t)(lt / tiles_m) * BN;
    TileJob<T> j;
    j.m = __ldg(&e->m);
    j.n = __ldg(&e->n);
    j.k = __ldg(&e->k);
    j.A = static_cast<const T *>(e->a);
    j.B = static_cast<const T *>(e->b);
    j.C = static_cast<T *>(e->c);
    j.lda = __ldg(&e->lda);
    j.ldb = __ldg(&e->ldb);
    j.ldc = __ldg(&e->ldc);
    const bool rd = beta_nonzero != 0;
    switch (__ldg(&e->op_a) * 3 + __ldg(&e->op_b)) {
#define HCBK_GT(OA, OB)                                                                    \
  case OA * 3 + OB:                                                                        \
    simt_tile<T, BM, BN, BK, TM, TN, OA, OB>(j, alpha, beta, rd, m0, n0, sm);              \
    break;
      HCBK_GT(0, 0) HCBK_GT(0, 1) HCBK_GT(1, 0) HCBK_GT(1, 1)
      default:
        if constexpr (IsComplex<T>::value) {
          switch (__ldg(&e->op_a) * 3 + __ldg(&e->op_b)) {
            HCBK_GT(0, 2) HCBK_GT(2, 0) HCBK_GT(2, 2) HCBK_GT(1, 2) HCBK_GT(2, 1)
            default: break;
          }
        }
        break;
#undef HCBK_GT
    }
    __syncthreads(); /* the shared buffers are reused by the next tile */
  }
}

/* ------------------------------------------------------------ launchers -- */

/* blocks of `kern` resident per SM (1 if the query fails) */
template <class K> static int resident_blocks(K kern, int threads) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return per_sm > 0 ? per_sm : 1;
}

/* MINB: CTAs per SM the register allocation must allow (2 for the FP32
 * 128 x 128 tile: sixteen warps per SM hide the global-load latency of each
 * K-slab better than eight) */
template <typename T, int BM, int BN, int BK, int TM, int TN, int MINB = 1>
int launch_cfg(const hcbk_gemm_args *a, cudaStream_t st) {
  using Acc = typename AccOf<T>::type;
  SimtParams<T, Acc> p;
  p.m = a->m; p.n = a->n; p.k = a->k;
  p.a = static_cast<const T *>(a->a); p.lda = a->lda; p.sa = a->stride_a; p.a_off = a->a_off;
  p.b = static_cast<const T *>(a->b); p.ldb = a->ldb; p.sb = a->stride_b; p.b_off = a->b_off;
  p.c = static_cast<T *>(a->c); p.ldc = a->ldc; p.sc = a->stride_c; p.c_off = a->c_off;
  p.a_arr = reinterpret_cast<const T *const *>(a->a_array);
  p.b_arr = reinterpret_cast<const T *const *>(a->b_array);
  p.c_arr = reinterpret_cast<T *const *>(a->c_array);
  p.batch = a->batch;
  p.sel = a->batch_select;
  p.alpha = HostScalar<Acc>::make(a->alpha_re, a->alpha_im);
  p.beta = HostScalar<Acc>::make(a->beta_re, a->beta_im);
  p.beta_nonzero = (a->beta_re != 0.0 || a->beta_im != 0.0);
  const int64_t tiles = ((a->m + BM - 1) / BM) * ((a->n + BN - 1) / BN);
  if (tiles > 0x7fffffffLL) return HCBK_ERR_ARGS;
  const int64_t gy = a->batch < 65535 ? a->batch : 65535;
  dim3 block((BM / TM) * (BN / TN));
  /* a selective pass runs as one wave of blocks, each scanning its share of
   * the flags at once (as many blocks as entries would queue in waves of
   * blocks that mostly find nothing to do) */
  auto grid_of = [&](int per_sm) {
    int64_t y = gy;
    if (a->batch_select) {
      const int64_t cap = ((int64_t)hcbk_sm_count() * per_sm + tiles - 1) / tiles;
      if (y > cap) y = cap;
    }
    return dim3((unsigned)tiles, (unsigned)y, 1);
  };
#define HCBK_SIMT_CASE(OA, OB)                                                    \
  if (a->op_a == OA && a->op_b == OB) {                                           \
    auto kern = simt_gemm_kernel<T, BM, BN, BK, TM, TN, OA, OB, MINB>;           \
    int per_sm = 1;                                                               \
    if (a->batch_select) {                                                        \
      static const int resident = resident_blocks(kern, (int)block.x);           \
      per_sm = resident;                                                          \
    }                                                                             \
    kern<<<grid_of(per_sm), block, 0, st>>>(p);                                   \
    return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;         \
  }
  HCBK_SIMT_CASE(0, 0) HCBK_SIMT_CASE(0, 1) HCBK_SIMT_CASE(1, 0) HCBK_SIMT_CASE(1, 1)
  /* conjugate transposes only exist for complex storage (the host maps
   * OP_C to OP_T for real types) */
  if constexpr (IsComplex<T>::value) {
    HCBK_SIMT_CASE(0, 2) HCBK_SIMT_CASE(2, 0) HCBK_SIMT_CASE(2, 2)
    HCBK_SIMT_CASE(1, 2) HCBK_SIMT_CASE(2, 1)
  }
#undef HCBK_SIMT_CASE
  return HCBK_ERR_ARGS;
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
int launch_grouped(const hcbk_simt_grouped_args *g, cudaStream_t st) {
  using Acc = typename AccOf<T>::type;
  auto kern = simt_grouped_kernel<T, BM, BN, BK, TM, TN>;
  constexpr int threads = (BM / TM) * (BN / TN);
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    return HCBK_ERR_LAUNCH;
  }
  int64_t grid = (int64_t)sms * (per_sm > 0 ? per_sm : 1);
  if (grid > g->total_tiles) grid = g->total_tiles;
  kern<<<(unsigned)grid, threads, 0, st>>>(
      g->table, g->tile_start, g->count, g->total_tiles,
      HostScalar<Acc>::make(g->alpha_re, g->alpha_im), HostScalar<Acc>::make(g->beta_re, g->beta_im),
      (g->beta_re != 0.0 || g->beta_im != 0.0) ? 1 : 0);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

}  // namespace
}  // namespace hcbk

using namespace hcbk;

extern "C" int hcbk_simt_grouped_tile(int dtype, int *bm, int *bn) {
  if (dtype < HCBK_S || dtype > HCBK_Z) return HCBK_ERR_ARGS;
  *bm = 64;
  *bn = 64;
  return HCBK_OK;
}

extern "C" int hcbk_gemm_simt_grouped(const hcbk_simt_grouped_args *g, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (g->count <= 0 || g->total_tiles <= 0) return HCBK_ERR_ARGS;
  switch (g->dtype) {
    case HCBK_S: return launch_grouped<float, 64, 64, 16, 4, 4>(g, st);
    case HCBK_D: return launch_grouped<double, 64, 64, 8, 4, 4>(g, st);
    case HCBK_C: return launch_grouped<float2, 64, 64, 8, 4, 4>(g, st);
    case HCBK_Z: return launch_grouped<double2, 64, 64, 8, 4, 4>(g, st);
    default: return HCBK_ERR_ARGS; /* f16 problems take the tensor-core grouped kernel */
  }
}

extern "C" int hcbk_gemm_simt(const hcbk_gemm_args *a, hcbk_simt_cfg cfg, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (a->m <= 0 || a->n <= 0 || a->k <= 0 || a->batch <= 0) return HCBK_ERR_ARGS;
  const bool small = cfg.variant == 1;
  switch (a->dtype) {
    case HCBK_S:
      return small ? launch_cfg<float, 64, 64, 16, 4, 4>(a, st)
                   : launch_cfg<float, 128, 128, 16, 8, 8, 2>(a, st);
    case HCBK_D:
      return small ? launch_cfg<double, 64, 64, 8, 4, 4>(a, st)
                   : launch_cfg<double, 128, 128, 8, 8, 8>(a, st);
    case HCBK_C:
      return launch_cfg<float2, 64, 64, 8, 4, 4>(a, st);
    case HCBK_Z:
      return launch_cfg<double2, 64, 64, 8, 4, 4>(a, st);
    case HCBK_H:
      return small ? launch_cfg<__half, 64, 64, 32, 4, 4>(a, st)
                   : launch_cfg<__half, 128, 128, 16, 8, 8>(a, st);
    default:
      return HCBK_ERR_ARGS;
  }
}
