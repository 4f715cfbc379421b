/*
 * crt.cu -- integer-modular (CRT) emulation of DGEMM, after Ozaki, Uchino &
 * Imamura, "Ozaki Scheme II: A GEMM-oriented emulation of floating-point
 * matrix multiplication using an integer modular technique" (2025).
 *
 *   1. Scale each row of op(A) / column of op(B) to integers:
 *        A'(m,k) = rint(A(m,k) * 2^(beta - e_m)),  |A'| <= 2^beta  (<= 2^53),
 *      with e_m the frexp exponent of max_k |A(m,k)|; likewise B'.
 *   2. For pairwise-coprime odd moduli p_1..p_n (<= 255), store the symmetric
 *      residues A' mod p_i, B' mod p_i (|r| <= 127) as binary16 planes --
 *      exact, and every f16 x f16 product is exact in f32.
 *   3. One tensor-core GEMM per modulus computes T_i = A'_i B'_i mod p_i
 *      exactly (tc_gemm.cu, EpiModP: f32 sums stay integers below 2^24 over
 *      1024-element K chunks and are reduced mod p_i in place in TMEM).
 *   4. This file's combine kernel rebuilds the exact integer product
 *      P' = A' B' (|P'| < (p_1...p_n)/2, guaranteed by the choice of n and
 *      beta) from (T_1..T_n) with the CRT formula P' = sum_i T_i w_i mod M
 *      (weights split into 40-bit chunks so every chunk sum is exact in
 *      binary64), evaluates it in double-double, and writes
 *        C = alpha * P' * 2^(e_m + f_n - 2 beta) + beta * C.
 * The only roundings are the scaling in step 1 (relative 2^-(beta+1) of the
 * row / column maximum) and the final conversion to binary64.
 *
 * Both element-wise kernels keep their modular arithmetic on the FMA pipes:
 * quotients are rounded with the 1.5 * 2^23 (f32) / 1.5 * 2^52 (f64)
 * constants, small integers move between int16 and f32 through the
 * exponent-bias trick, and the only conversion-unit instructions left are
 * one f64 -> f32 per 16-bit limb and one packed f32x2 -> f16x2 per two
 * residues.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hcbk.h"
#include "tc_common.cuh"

namespace {

constexpr float RND_F = 12582912.0f;             /* 1.5 * 2^23 */
constexpr double RND_D = 6755399441055744.0;     /* 1.5 * 2^52 */

/* exact x mod p into (-1.5p, 1.5p) for integral |x| < 2^23; the rounded
 * quotient may be one off, the remainder fma is exact either way */
__device__ __forceinline__ float mod_f(float x, float p, float inv_p) {
  const float q = fmaf(x, inv_p, RND_F) - RND_F;
  return fmaf(-q, p, x);
}

/* fold (-1.5p, 1.5p) into the symmetric range [-(p-1)/2, (p-1)/2] */
__device__ __forceinline__ float sym_f(float r, float p, float hp) {
  r = r > hp ? r - p : r;
  return r < -hp ? r + p : r;
}

/* small integer (|x| < 2^22) to f32 without the conversion unit */
__device__ __forceinline__ float small_int_to_f(int x) {
  return __int_as_float(0x4B400000 + x) - RND_F;
}

struct ModConst {
  float p, inv_p, hp;
  float c1, c2, c3; /* 2^14, 2^28, 2^42 mod p (symmetric) */
};

/* the same constants duplicated into (x, x) pairs for the packed f32x2
 * instructions, and -p for the remainder fma */
struct alignas(8) ModPair {
  float2 c1, c2, c3, inv_p, neg_p;
};

struct ResArgs {
  const double *src;
  int64_t ld;
  int64_t rows, kdim;
  const int *exps;
  const double *frac; /* optional: x * frac[r] is scaled */
  int beta;
  int nmod;
  ModPair mp[HCBK_CRT_MAX_MODULI];
  char *planes;
  int64_t plane_stride; /* bytes */
  int64_t ld_dst;       /* elements */
  /* strided batch: element e's source at src + e * src_bstride, its exps /
   * frac at + e * rows, its planes at planes + e * planes_bstride */
  int64_t batch, src_bstride, planes_bstride;
};

/* 14-bit limbs of the scaled integer y = rint(x 2^(beta - e)), |y| <= 2^53:
 * y = l3 2^42 + l2 2^28 + l1 2^14 + l0 with |l0..l2| <= 2^13 and
 * |l3| <= 2^11, all exact in f32 (0 for zero / non-finite rows) */
struct Limbs {
  float l0, l1, l2, l3;
};

/* rint(v) of |v| < 2^51 as a double whose low word is rint(v) as an int */
__device__ __forceinline__ double rnd_magic(double v) { return v + RND_D; }

/* x * 2^s without the library's general ldexp path when 2^s is a normal
 * number (a power-of-two scaling; an underflow only loses bits below 2^-1022,
 * which the rint that follows discards anyway) */
__device__ __forceinline__ double scale2(double x, int s) {
  return (s >= -1022 && s <= 1023) ? x * __longlong_as_double((long long)(s + 1023) << 52)
                                   : ldexp(x, s);
}

__device__ __forceinline__ Limbs limbs_of(double x, int e, int beta) {
  Limbs L{0.f, 0.f, 0.f, 0.f};
  if (e == HCBK_OZ_NONFINITE || e == HCBK_OZ_ZERO) return L;
  const double y = rint(scale2(x, beta - e));
  /* each limb's rounded quotient comes out of the magic-constant add with
   * the integer in the low word: no conversion-unit instructions */
  const double t3 = rnd_magic(y * 0x1p-42);
  double r = fma(-(t3 - RND_D), 0x1p42, y);
  const double t2 = rnd_magic(r * 0x1p-28);
  r = fma(-(t2 - RND_D), 0x1p28, r);
  const double t1 = rnd_magic(r * 0x1p-14);
  r = fma(-(t1 - RND_D), 0x1p14, r);
  const double t0 = rnd_magic(r);
  L.l0 = small_int_to_f(__double2loint(t0));
  L.l1 = small_int_to_f(__double2loint(t1));
  L.l2 = small_int_to_f(__double2loint(t2));
  L.l3 = small_int_to_f(__double2loint(t3));
  return L;
}

/* symmetric residue of the limb sum modulo one modulus.  |sum| <=
 * 2^13 (1 + 2 * 127) + 2^11 * 127 < 2^21.2, so |sum / p| < 14100 (p >= 167)
 * and the f32 quotient sum * RN(1/p) is off by < 8.5e-4 -- less than the
 * 0.5/p >= 0.00196 distance of any x/p (p odd) from a half-integer: the
 * rounded quotient is exact and the remainder already lies in
 * [-(p-1)/2, (p-1)/2]. */
__device__ __forceinline__ float residue(const Limbs &L, const ModConst &m) {
  float t = fmaf(L.l3, m.c3, L.l0);
  t = fmaf(L.l2, m.c2, t);
  t = fmaf(L.l1, m.c1, t);
  return mod_f(t, m.p, m.inv_p);
}

/* packed f32x2 arithmetic (two lanes per instruction, each rounded as the
 * scalar operation) */
__device__ __forceinline__ uint64_t pk2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ uint64_t pk2(float2 v) { return pk2(v.x, v.y); }
__device__ __forceinline__ float2 upk2(uint64_t r) {
  float2 v;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
  return v;
}
__device__ __forceinline__ uint64_t fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

/* limbs of two elements, lane-paired */
struct Limbs2 {
  uint64_t l0, l1, l2, l3;
};

__device__ __forceinline__ Limbs2 pair_limbs(const Limbs &a, const Limbs &b) {
  return Limbs2{pk2(a.l0, b.l0), pk2(a.l1, b.l1), pk2(a.l2, b.l2), pk2(a.l3, b.l3)};
}

/* x - rint(x / p) p for a pair of exact integers whose quotient rounds
 * exactly (the limb sums above, or |x| < 2^19) */
__device__ __forceinline__ uint64_t mod2(uint64_t t, const ModPair &m) {
  const uint64_t RND2 = pk2(RND_F, RND_F), NRND2 = pk2(-RND_F, -RND_F);
  const uint64_t q = add2(fma2(t, pk2(m.inv_p), RND2), NRND2);
  return fma2(q, pk2(m.neg_p), t);
}

/* residue() for two elements in six packed instructions */
__device__ __forceinline__ uint64_t residue2(const Limbs2 &L, const ModPair &m) {
  uint64_t t = fma2(L.l3, pk2(m.c3), L.l0);
  t = fma2(L.l2, pk2(m.c2), t);
  t = fma2(L.l1, pk2(m.c1), t);
  return mod2(t, m);
}

__device__ __forceinline__ __half2 to_h2(uint64_t r) {
  const float2 f = upk2(r);
  return __floats2half2_rn(f.x, f.y);
}

/* the residue pair converted to binary16 */
__device__ __forceinline__ __half2 residue2_h(const Limbs2 &L, const ModPair &m) {
  return to_h2(residue2(L, m));
}

/* a pair of small integers (|r| <= 127, f32x2) as two int8 in the low 16
 * bits: the low byte of the 1.5 * 2^23 + r pattern is r in two's complement */
__device__ __forceinline__ uint32_t to_s8x2(uint64_t r) {
  const float2 f = upk2(add2(r, pk2(RND_F, RND_F)));
  return __byte_perm(__float_as_uint(f.x), __float_as_uint(f.y), 0x0040);
}

/* the residue pair as two int8 */
__device__ __forceinline__ uint32_t residue2_s8(const Limbs2 &L, const ModPair &m) {
  return to_s8x2(residue2(L, m));
}

/* K-contiguous source: 8 consecutive k per thread, 16-byte (binary16) or
 * 8-byte (int8) plane stores */
/* grid-stride walk over the (row, chunk) cells of a rows x chunks grid, the
 * row and chunk kept by additions instead of a 64-bit division per step */
struct GridWalk {
  int64_t idx, r, c, dr, dc, chunks, stride;
  __device__ __forceinline__ explicit GridWalk(int64_t chunks_) {
    stride = (int64_t)gridDim.x * blockDim.x;
    idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    chunks = chunks_;
    r = idx / chunks;
    c = idx % chunks;
    dr = stride / chunks;
    dc = stride % chunks;
  }
  __device__ __forceinline__ void next() {
    idx += stride;
    r += dr;
    c += dc;
    if (c >= chunks) {
      c -= chunks;
      ++r;
    }
  }
};

template <bool I8>
__global__ void __launch_bounds__(256, 3) crt_res_kcontig(ResArgs a) {
  struct alignas(16) H8 { __half2 v[4]; };
  constexpr int ESZ = I8 ? 1 : 2;
  const int64_t kq = (a.kdim + 7) / 8;
  const int64_t total = a.rows * kq * a.batch; /* rows of every batch element in turn */
  for (GridWalk g(kq); g.idx < total; g.next()) {
    const int64_t b = g.r / a.rows, r = g.r - b * a.rows;
    const double *src = a.src + b * a.src_bstride;
    char *planes = a.planes + b * a.planes_bstride;
    const int64_t k0 = g.c * 8;
    const int e = a.exps[g.r];
    const double f = a.frac ? a.frac[g.r] : 1.0;
    Limbs2 L2[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const Limbs x0 = limbs_of(
          f * ((k0 + 2 * j < a.kdim) ? src[r * a.ld + k0 + 2 * j] : 0.0), e, a.beta);
      const Limbs x1 = limbs_of(
          f * ((k0 + 2 * j + 1 < a.kdim) ? src[r * a.ld + k0 + 2 * j + 1] : 0.0), e, a.beta);
      L2[j] = pair_limbs(x0, x1);
    }
#pragma unroll
    for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) { /* constant-bank operands, no indexed loads */
      if (i >= a.nmod) break;
      const ModPair m = a.mp[i];
      char *d = planes + i * a.plane_stride + (r * a.ld_dst + k0) * ESZ;
      const bool whole = k0 + 8 <= a.kdim && (reinterpret_cast<uintptr_t>(d) & (8 * ESZ - 1)) == 0;
      if constexpr (I8) {
        uint2 out;
        out.x = __byte_perm(residue2_s8(L2[0], m), residue2_s8(L2[1], m), 0x5410);
        out.y = __byte_perm(residue2_s8(L2[2], m), residue2_s8(L2[3], m), 0x5410);
        if (whole) {
          *reinterpret_cast<uint2 *>(d) = out;
        } else {
          const int8_t *h = reinterpret_cast<const int8_t *>(&out);
          for (int j = 0; j < 8; ++j)
            if (k0 + j < a.kdim) reinterpret_cast<int8_t *>(d)[j] = h[j];
        }
      } else {
        H8 out;
#pragma unroll
        for (int j = 0; j < 4; ++j) out.v[j] = residue2_h(L2[j], m);
        if (whole) {
          *reinterpret_cast<H8 *>(d) = out;
        } else {
          const __half *h = reinterpret_cast<const __half *>(&out);
          for (int j = 0; j < 8; ++j)
            if (k0 + j < a.kdim) reinterpret_cast<__half *>(d)[j] = h[j];
        }
      }
    }
  }
}

/* MN-contiguous source: a 32-row x KT tile (KT = 64 for int8 planes, 32 for
 * binary16) through shared memory; each thread then owns KT / 8 consecutive
 * k of one row (8-byte plane stores; eight threads write one row's 64
 * contiguous bytes), so each modulus's constants serve KT / 16 element pairs */
template <bool I8>
__global__ void __launch_bounds__(256) crt_res_rcontig(ResArgs a) {
  constexpr int ESZ = I8 ? 1 : 2;
  constexpr int KT = I8 ? 64 : 32, KPT = KT / 8, NP = KPT / 2;
  __shared__ double tile[KT][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * KT;
  const int64_t b = blockIdx.z; /* batch element */
  const double *src = a.src + b * a.src_bstride;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < KT / 8; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < a.rows && k < a.kdim) ? src[r + k * a.ld] : 0.0;
  }
  __syncthreads();
  const int t = ty * 32 + tx;
  const int rl = t >> 3, kq = (t & 7) * KPT;
  const int64_t r = r0 + rl, k = k0 + kq;
  if (r >= a.rows || k >= a.kdim) return;
  const int e = a.exps[b * a.rows + r];
  const double f = a.frac ? a.frac[b * a.rows + r] : 1.0;
  Limbs2 L2[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j)
    L2[j] = pair_limbs(limbs_of(f * tile[kq + 2 * j][rl], e, a.beta),
                       limbs_of(f * tile[kq + 2 * j + 1][rl], e, a.beta));
  const int64_t left = a.kdim - k;
  const int nk = left < KPT ? (int)left : KPT;
  char *d0 = a.planes + b * a.planes_bstride + (r * a.ld_dst + k) * (int64_t)ESZ;
  const bool vec = nk == KPT && (reinterpret_cast<uintptr_t>(d0) & 7) == 0 &&
                   (a.plane_stride & 7) == 0;
#pragma unroll
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) { /* constant-bank operands, no indexed loads */
    if (i >= a.nmod) break;
    const ModPair m = a.mp[i];
    uint2 w; /* KPT residues: 8 bytes either way */
    if constexpr (I8) {
      w.x = __byte_perm(residue2_s8(L2[0], m), residue2_s8(L2[1], m), 0x5410);
      w.y = __byte_perm(residue2_s8(L2[2], m), residue2_s8(L2[3], m), 0x5410);
    } else {
      __half2 v[2];
      v[0] = residue2_h(L2[0], m);
      v[1] = residue2_h(L2[1], m);
      w = *reinterpret_cast<const uint2 *>(v);
    }
    char *d = d0 + i * a.plane_stride;
    if (vec) {
      *reinterpret_cast<uint2 *>(d) = w;
    } else {
      const uint64_t wv = (static_cast<uint64_t>(w.y) << 32) | w.x;
      for (int j = 0; j < nk * ESZ; ++j) d[j] = static_cast<char>(wv >> (8 * j));
    }
  }
}

/* Reconstruction by the weighted residue sum (the CRT formula, as in Ozaki
 * scheme II):  with M = p_1...p_n, M_i = M / p_i and y_i = M_i^-1 mod p_i,
 *   P' = sum_i r_i w_i  mod M,   w_i = M_i y_i < M.
 * Each w_i is held as NC 40-bit chunks w_i = sum_k w_ik 2^(40k); with
 * |r_i| <= 127 and n <= 20 every chunk sum S_k = sum_i r_i w_ik is below
 * 20 * 127 * 2^40 < 2^52.4 and exact in binary64.  The quotient
 * q = rint(S / M) is below 2^12 and is exact from a binary64 estimate,
 * because |P'| <= M / (2 * 2^0.01) keeps S / M at least 0.003 away from a
 * half-integer (the count of moduli is chosen that way), far above the
 * estimate's 2^-39 error.  D_k = S_k - q M_k is exact (< 2^53), carries
 * normalise the chunks to |D_k| <= 2^39 below the top one, and the chunks are
 * summed in double-double. */
constexpr int CRT_CHUNK_BITS = 40;
constexpr int MAX_NC = 4; /* 20 moduli: M < 2^155 */

struct CombArgs {
  int64_t m, n;
  int nmod;
  int nc;
  float p[HCBK_CRT_MAX_MODULI];
  float inv_p[HCBK_CRT_MAX_MODULI];
  float hp[HCBK_CRT_MAX_MODULI];
  double w[HCBK_CRT_MAX_MODULI][MAX_NC]; /* 40-bit chunks of w_i, low first */
  double mk[MAX_NC];                     /* 40-bit chunks of M, low first */
  double inv_m;                          /* RN(1 / M) */
  const int8_t *res;
  int64_t res_plane; /* bytes between residue planes */
  int64_t ldr;
  const int *exp_a;
  const int *exp_b;
  const double *inv_a, *inv_b; /* optional reciprocals of the row fractions */
  int shift;
  double *c;
  int64_t ldc;
  double alpha, beta;
  int beta_nonzero;
  int *err; /* device error flag (pipeline wait timed out) */
  /* strided batch: element e's residue planes at res + e * res_bstride,
   * exp_a / inv_a at + e * m, exp_b / inv_b at + e * n, C at c + e * c_bstride */
  int64_t batch, res_bstride, c_bstride;
};

/* small integer to binary64 without the conversion unit: the bit pattern
 * 0x43300000:(r + 2^31) is 2^52 + 2^31 + r */
__device__ __forceinline__ double small_int_to_d(int r) {
  return __hiloint2double(0x43300000, r ^ (int)0x80000000) - 4503601774854144.0;
}

/* byte u of four int8 residues whose sign bits were flipped (each byte
 * r + 128, 0..255) as the binary64 value r: the byte, zero-extended by one
 * byte permute, under the exponent of 2^52 gives 2^52 + 128 + r */
__device__ __forceinline__ double biased_byte_to_d(uint32_t qb, int u) {
  return __hiloint2double(0x43300000, (int)__byte_perm(qb, 0u, 0x4440u + (uint32_t)u)) -
         4503599627370624.0;
}

template <int NC>
struct CrtAcc {
  double S[NC];

  __device__ __forceinline__ CrtAcc() {
#pragma unroll
    for (int k = 0; k < NC; ++k) S[k] = 0.0;
  }

  /* add residue r (|r| <= 127) with weight chunks w */
  __device__ __forceinline__ void add(const double *w, int r) {
    const double rd = small_int_to_d(r);
#pragma unroll
    for (int k = 0; k < NC; ++k) S[k] = fma(rd, w[k], S[k]);
  }

  /* P' * 2^(ea + eb - shift) */
  __device__ __forceinline__ double finish(const CombArgs &a, int ea, int eb) const {
    if (ea == HCBK_OZ_NONFINITE || eb == HCBK_OZ_NONFINITE)
      return __longlong_as_double(0x7ff8000000000000ll);
    if (ea == HCBK_OZ_ZERO || eb == HCBK_OZ_ZERO) return 0.0;
    constexpr double CH = 1099511627776.0;     /* 2^40 */
    constexpr double INV_CH = 1.0 / 1099511627776.0;
    double s = S[NC - 1];
#pragma unroll
    for (int k = NC - 2; k >= 0; --k) s = fma(s, CH, S[k]);
    const double q = fma(s, a.inv_m, RND_D) - RND_D;
    double D[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) D[k] = fma(-q, a.mk[k], S[k]);
#pragma unroll
    for (int k = 0; k < NC - 1; ++k) {
      const double cy = fma(D[k], INV_CH, RND_D) - RND_D;
      D[k] = fma(-cy, CH, D[k]);
      D[k + 1] += cy;
    }
    /* Horner from the low chunk: with |D_k| <= 2^39 below the top chunk the
     * partial sums stay below half the top chunk's unit, so the rounded
     * result is within 1.5 ulp of P' */
    double x = D[0];
    double w = CH;
#pragma unroll
    for (int k = 1; k < NC; ++k) {
      x = fma(D[k], w, x);
      w *= CH;
    }
    const int e = ea + eb - a.shift;
    return (e >= -1022 && e <= 1023) ? x * __longlong_as_double((long long)(e + 1023) << 52)
                                     : ldexp(x, e);
  }
};

/* real combine: 256 consumer threads x 4 consecutive rows (one 4-byte
 * load of four int8 residues per modulus); 3 stages of nmod KB */
constexpr int CMB_THREADS = 256, CMB_RPT = 4, CMB_ROWS = CMB_THREADS * CMB_RPT;
constexpr int CMB_STAGES = 3;
/* complex combine: 256 consumer threads x 2 rows (two accumulators a
 * row); 3 stages of 1.5 nmod KB */
constexpr int ZCMB_THREADS = 256, ZCMB_RPT = 2, ZCMB_ROWS = ZCMB_THREADS * ZCMB_RPT;
constexpr int ZCMB_STAGES = 3;
static_assert(ZCMB_RPT == 2, "the complex combine loads two rows' residues as one 2-byte word");


/* Walk over a block's tiles first, first + stride, ... of a grid of
 * row_tiles x columns tiles (column-major tile order), keeping the tile's
 * row tile and column by additions: no 64-bit division per tile.  Also
 * tracks the ring stage and its phase.  Row tiles and the stride are below
 * 2^31; the walk ends once the column reaches the column count. */
template <int STAGES>
struct TileWalk {
  int64_t col, dcol;
  int rt, drt, row_tiles, s;
  uint32_t ph;
  __device__ __forceinline__ TileWalk(int first, int stride, int row_tiles_)
      : col(first / row_tiles_), dcol(stride / row_tiles_), rt(first % row_tiles_),
        drt(stride % row_tiles_), row_tiles(row_tiles_), s(0), ph(0) {}
  __device__ __forceinline__ void next() {
    rt += drt;
    col += dcol;
    if (rt >= row_tiles) {
      rt -= row_tiles;
      ++col;
    }
    if (++s == STAGES) {
      s = 0;
      ph ^= 1u;
    }
  }
};

/* Producer of a warp-specialised combine (one thread): tile j of this block
 * (ROWS rows of one column, every residue plane; the columns of a batch's
 * elements one after the other, ncols in all) goes to stage j % STAGES by
 * 1-D bulk copies once the consumers have released the stage's previous
 * tile; before returning it lets the last copies land (immediately when the
 * consumers took them; bounded when a wait failed), so that no copy writes
 * shared memory after the block has left. */
template <int STAGES, int ROWS>
__device__ __forceinline__ void ws_produce(const int8_t *res, int64_t res_plane, int64_t ldr,
                                           int nplanes, int64_t row_tiles, int64_t ncols,
                                           int64_t cols_per, int64_t res_bstride,
                                           int8_t *buf, uint64_t *full, uint64_t *empty,
                                           int *err) {
  using namespace hcbk::tc;
  const size_t stage_elems = (size_t)nplanes * ROWS;
  int64_t j = 0;
  TileWalk<STAGES> w((int)blockIdx.x, (int)gridDim.x, (int)row_tiles);
  for (; w.col < ncols; w.next(), ++j) {
    const int s = w.s;
    /* the stage's previous tile was taken in the phase before this one */
    if (j >= STAGES && !mbar_wait(&empty[s], w.ph ^ 1u, err, ERR_TIMEOUT_COMBINE)) break;
    const int64_t r0 = w.rt * ROWS;
    const int64_t rows = ldr - r0 < ROWS ? ldr - r0 : ROWS;
    const uint32_t bytes = (uint32_t)rows; /* ldr, r0 multiples of 16 */
    mbar_expect_tx(&full[s], bytes * (uint32_t)nplanes);
    /* column w.col of the batch: element e's column c */
    const int64_t e = w.col / cols_per, c = w.col - e * cols_per;
    const int8_t *src = res + e * res_bstride + c * ldr + r0;
    int8_t *dst = buf + s * stage_elems;
    for (int p = 0; p < nplanes; ++p)
      bulk_load_1d(dst + p * ROWS, src + p * res_plane, bytes, &full[s]);
  }
  for (int64_t k = (j > STAGES ? j - STAGES : 0); k < j; ++k) {
    const int s = (int)(k % STAGES);
    const uint32_t ph = (uint32_t)(k / STAGES) & 1u;
    for (int it = 0; it < (1 << 22) && !mbar_try_wait(&full[s], ph); ++it) {
    }
  }
}

/* Real combine, warp-specialised: warps 0-7 reconstruct 512-row tiles (two
 * consecutive rows per thread, one 2-byte load of an int8 residue pair per
 * modulus), warp 8's lane 0 keeps CMB_STAGES tiles of residues in flight by
 * 1-D bulk copies.  Per stage a `full` barrier (transaction bytes) and an
 * `empty` barrier (one arrival per consumer warp) replace block-wide
 * barriers, so consumer warps run up to CMB_STAGES - 1 tiles apart.  The
 * modulus loop is unrolled over the maximum count, so every weight chunk is
 * a constant-bank operand of its FMA.  Requires the row pitch and plane
 * stride to be multiples of 16 bytes. */
constexpr int CMB_CONSUMERS = CMB_THREADS / 32;
constexpr int CMB_BLOCK = CMB_THREADS + 32;

template <int NC>
__global__ void __launch_bounds__(CMB_BLOCK, 4) crt_combine_kernel(const __grid_constant__ CombArgs a) {
  using namespace hcbk::tc;
  extern __shared__ __align__(128) unsigned char cmb_smem[];
  __shared__ __align__(8) uint64_t full[CMB_STAGES], empty[CMB_STAGES];
  if (blockDim.x != CMB_BLOCK) { /* the tile covers CMB_ROWS rows only at this shape */
    if (threadIdx.x == 0) atomicCAS(a.err, 0, (int)ERR_LAUNCH_SHAPE);
    return;
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nmod = a.nmod;
  int8_t *buf = reinterpret_cast<int8_t *>(cmb_smem);
  const int64_t row_tiles = (a.m + CMB_ROWS - 1) / CMB_ROWS;
  const int64_t first = blockIdx.x, stride = gridDim.x;
  const size_t stage_elems = (size_t)nmod * CMB_ROWS;
  if (tid == 0) {
    for (int s = 0; s < CMB_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], CMB_CONSUMERS);
    }
    mbar_fence_init();
  }
  __syncthreads();

  if (warp == CMB_CONSUMERS) { /* producer */
    if (lane == 0)
      ws_produce<CMB_STAGES, CMB_ROWS>(a.res, a.res_plane, a.ldr, nmod, row_tiles,
                                       a.n * a.batch, a.n, a.res_bstride, buf, full, empty,
                                       a.err);
    return;
  }

  /* ------------------------------------------------ consumers -- */
  const int64_t ncols = a.n * a.batch; /* the columns of every batch element in turn */
  for (TileWalk<CMB_STAGES> w((int)first, (int)stride, (int)row_tiles); w.col < ncols; w.next()) {
    const int s = w.s;
    if (!__all_sync(0xffffffffu, mbar_wait(&full[s], w.ph, a.err, ERR_TIMEOUT_COMBINE))) break;
    const int8_t *R = buf + s * stage_elems;
    const int64_t be = w.col / a.n; /* batch element */
    const int64_t row = w.rt * CMB_ROWS + CMB_RPT * tid, col = w.col - be * a.n;
    if (row < a.m) {
      CrtAcc<NC> acc[CMB_RPT];
#pragma unroll
      for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) { /* constant-bank weights */
        if (i >= nmod) break;
        /* the four rows' residues of this modulus, sign bits flipped */
        const uint32_t q =
            *reinterpret_cast<const uint32_t *>(R + i * CMB_ROWS + CMB_RPT * tid) ^ 0x80808080u;
#pragma unroll
        for (int u = 0; u < CMB_RPT; ++u) {
          const double r = biased_byte_to_d(q, u);
#pragma unroll
          for (int k = 0; k < NC; ++k) acc[u].S[k] = fma(r, a.w[i][k], acc[u].S[k]);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]); /* the stage's residues are in registers */
      const int eb = a.exp_b[be * a.n + col];
      const double ib = a.inv_b ? a.inv_b[be * a.n + col] : 1.0;
      double *dst = a.c + be * a.c_bstride + row + col * a.ldc;
      const int64_t ra = be * a.m + row;
#pragma unroll
      for (int u = 0; u < CMB_RPT; ++u) {
        if (row + u >= a.m) break;
        double v = acc[u].finish(a, a.exp_a[ra + u], eb);
        if (a.inv_a) v *= a.inv_a[ra + u] * ib;
        double o = a.alpha * v;
        if (a.beta_nonzero) o = fma(a.beta, dst[u], o);
        dst[u] = o;
      }
    } else {
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
}

/* modular inverse by the extended Euclidean algorithm */
static long long inv_mod_ll(long long a, long long m) {
  long long t = 0, nt = 1, r = m, nr = ((a % m) + m) % m;
  while (nr != 0) {
    const long long qq = r / nr;
    long long tmp = t - qq * nt;
    t = nt;
    nt = tmp;
    tmp = r - qq * nr;
    r = nr;
    nr = tmp;
  }
  if (t < 0) t += m;
  return t;
}

/* symmetric representative of 2^bits modulo p */
static float pow2_mod_sym(int bits, int p) {
  long long v = 1;
  for (int i = 0; i < bits; ++i) v = (v * 2) % p;
  if (v > (p - 1) / 2) v -= p;
  return (float)v;
}

static void fill_mod_consts(ModConst (&mc)[HCBK_CRT_MAX_MODULI]) {
  const int *M = hcbk_crt_moduli(nullptr);
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) {
    ModConst &m = mc[i];
    m.p = (float)M[i];
    m.inv_p = 1.0f / (float)M[i];
    m.hp = (float)((M[i] - 1) / 2);
    m.c1 = pow2_mod_sym(14, M[i]);
    m.c2 = pow2_mod_sym(28, M[i]);
    m.c3 = pow2_mod_sym(42, M[i]);
  }
}

/* unsigned multi-word integer, 32-bit words, low first */
struct BigU {
  uint32_t w[8];
  int len;
};

static void big_set(BigU &b, uint32_t v) {
  for (int i = 0; i < 8; ++i) b.w[i] = 0;
  b.w[0] = v;
  b.len = 1;
}

static void big_mul_small(BigU &b, uint32_t s) {
  uint64_t carry = 0;
  for (int i = 0; i < b.len; ++i) {
    const uint64_t t = (uint64_t)b.w[i] * s + carry;
    b.w[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) b.w[b.len++] = (uint32_t)carry;
}

/* b /= d, returns b mod d */
static uint32_t big_div_small(BigU &b, uint32_t d) {
  uint64_t rem = 0;
  for (int i = b.len - 1; i >= 0; --i) {
    const uint64_t cur = (rem << 32) | b.w[i];
    b.w[i] = (uint32_t)(cur / d);
    rem = cur % d;
  }
  while (b.len > 1 && b.w[b.len - 1] == 0) --b.len;
  return (uint32_t)rem;
}

static int big_bits(const BigU &b) {
  int top = b.len - 1;
  while (top > 0 && b.w[top] == 0) --top;
  int bits = 32 * top;
  for (uint32_t v = b.w[top]; v; v >>= 1) ++bits;
  return bits;
}

/* bits [lo, lo + n) as a double (exact for n <= 53) */
static double big_bits_at(const BigU &b, int lo, int n) {
  double v = 0.0;
  for (int j = n - 1; j >= 0; --j) {
    const int bit = lo + j;
    const int word = bit / 32;
    const uint32_t set = word < b.len ? (b.w[word] >> (bit % 32)) & 1u : 0u;
    v = v * 2.0 + (double)set;
  }
  return v;
}

static double big_to_double(const BigU &b) {
  double v = 0.0;
  for (int i = b.len - 1; i >= 0; --i) v = v * 4294967296.0 + (double)b.w[i];
  return v;
}

static void fill_mod_pairs(ModPair (&mp)[HCBK_CRT_MAX_MODULI]) {
  ModConst mc[HCBK_CRT_MAX_MODULI];
  fill_mod_consts(mc);
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) {
    mp[i].c1 = make_float2(mc[i].c1, mc[i].c1);
    mp[i].c2 = make_float2(mc[i].c2, mc[i].c2);
    mp[i].c3 = make_float2(mc[i].c3, mc[i].c3);
    mp[i].inv_p = make_float2(mc[i].inv_p, mc[i].inv_p);
    mp[i].neg_p = make_float2(-mc[i].p, -mc[i].p);
  }
}

/* moduli and the weights, chunks and reciprocal of the reconstruction */
static void fill_comb_moduli(CombArgs &a, int nmod) {
  const int *P = hcbk_crt_moduli(nullptr);
  a.nmod = nmod;
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) {
    a.p[i] = (float)P[i];
    a.inv_p[i] = 1.0f / (float)P[i];
    a.hp[i] = (float)((P[i] - 1) / 2);
    for (int k = 0; k < MAX_NC; ++k) a.w[i][k] = 0.0;
  }
  BigU M;
  big_set(M, 1);
  for (int i = 0; i < nmod; ++i) big_mul_small(M, (uint32_t)P[i]);
  const int bits = big_bits(M);
  a.nc = (bits + CRT_CHUNK_BITS - 1) / CRT_CHUNK_BITS;
  for (int k = 0; k < MAX_NC; ++k)
    a.mk[k] = k < a.nc ? big_bits_at(M, CRT_CHUNK_BITS * k, CRT_CHUNK_BITS) : 0.0;
  a.inv_m = 1.0 / big_to_double(M);
  for (int i = 0; i < nmod; ++i) {
    BigU Mi = M;
    big_div_small(Mi, (uint32_t)P[i]); /* exact: M_i = M / p_i */
    BigU t = Mi;
    const uint32_t mi_mod = big_div_small(t, (uint32_t)P[i]);
    const uint32_t y = (uint32_t)inv_mod_ll(mi_mod, P[i]);
    big_mul_small(Mi, y); /* w_i = M_i y_i < M */
    for (int k = 0; k < a.nc; ++k)
      a.w[i][k] = big_bits_at(Mi, CRT_CHUNK_BITS * k, CRT_CHUNK_BITS);
  }
}

/* ------------------------------------------------ complex (ZGEMM) path --
 * 3M (Karatsuba) in modular arithmetic, where it is exact:
 *   T1 = Ar Br, T2 = Ai Bi, T3 = (Ar + Ai)(Br + Bi)   (mod p, one GEMM each)
 *   Re = T1 - T2,  Im = T3 - T1 - T2                  (mod p, then the CRT sum)
 * Real and imaginary parts of a row share one exponent (the larger), so
 * Ar' + Ai' is the residue sum of one scaled integer pair. */

struct ZResArgs {
  const double2 *src;
  int64_t ld;
  int64_t rows, kdim;
  const int *exps;
  int exp_pair;    /* exponent of row r = max(exps[2r], exps[2r+1]) */
  const double *frac; /* optional row fractions: z * frac[r] is scaled */
  float im_sign;   /* -1 for a conjugate-transposed operand */
  int beta;
  int nmod;
  ModConst mc[HCBK_CRT_MAX_MODULI];
  ModPair mp[HCBK_CRT_MAX_MODULI];
  char *planes;          /* plane (set, i) at planes + (set * nmod + i) * plane_stride */
  int64_t plane_stride;  /* bytes; sets: 0 = real, 1 = imaginary, 2 = sum */
  int64_t ld_dst;        /* elements */
};

__device__ __forceinline__ int row_exp(const int *exps, int pair, int64_t r) {
  return pair ? max(exps[2 * r], exps[2 * r + 1]) : exps[r];
}

struct ZRes3 {
  float re, im, sum;
};

__device__ __forceinline__ ZRes3 zresidue(const Limbs &lr, const Limbs &li, const ModConst &m,
                                          float im_sign) {
  ZRes3 o;
  o.re = residue(lr, m);
  o.im = im_sign * residue(li, m);
  o.sum = mod_f(o.re + o.im, m.p, m.inv_p); /* |re + im| <= 254: exact quotient */
  return o;
}

/* K-contiguous complex source: 4 consecutive k per thread (40 limb
 * registers), residues of element pairs by packed f32x2 arithmetic with the
 * moduli constants as constant-bank operands, 8-byte (binary16) or 4-byte
 * (int8) stores per plane */
/* moduli loop of the complex residue kernels: constants staged in shared
 * memory and the loop unrolled ZRES_UNROLL deep, which keeps the kernel's
 * code within the instruction cache (fully unrolled over 20 moduli with three
 * plane sets it was not, and warps stalled on instruction fetch) */
constexpr int ZRES_UNROLL = 2;

template <bool I8>
__global__ void __launch_bounds__(256, 3) zcrt_res_kcontig(ZResArgs a) {
  constexpr int ESZ = I8 ? 1 : 2;
  __shared__ ModPair smp[HCBK_CRT_MAX_MODULI];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) smp[i] = a.mp[i];
  }
  __syncthreads();
  const int64_t kq = (a.kdim + 3) / 4;
  const int64_t total = a.rows * kq;
  for (GridWalk g(kq); g.idx < total; g.next()) {
    const int64_t r = g.r;
    const int64_t k0 = g.c * 4;
    const int e = row_exp(a.exps, a.exp_pair, r);
    const double f = a.frac ? a.frac[r] : 1.0;
    Limbs2 lr[2], li[2]; /* element pairs (0, 1), (2, 3); im carries the conj sign */
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double2 z0 =
          (k0 + 2 * j < a.kdim) ? a.src[r * a.ld + k0 + 2 * j] : make_double2(0.0, 0.0);
      const double2 z1 =
          (k0 + 2 * j + 1 < a.kdim) ? a.src[r * a.ld + k0 + 2 * j + 1] : make_double2(0.0, 0.0);
      lr[j] = pair_limbs(limbs_of(f * z0.x, e, a.beta), limbs_of(f * z1.x, e, a.beta));
      li[j] = pair_limbs(limbs_of(a.im_sign * (f * z0.y), e, a.beta),
                         limbs_of(a.im_sign * (f * z1.y), e, a.beta));
    }
    const int64_t left = a.kdim - k0;
    const int nk = left < 4 ? (int)left : 4;
    char *d0 = a.planes + (r * a.ld_dst + k0) * (int64_t)ESZ;
    const bool vec = nk == 4 && (reinterpret_cast<uintptr_t>(d0) & (4 * ESZ - 1)) == 0 &&
                     (a.plane_stride & (4 * ESZ - 1)) == 0;
#pragma unroll ZRES_UNROLL
    for (int i = 0; i < a.nmod; ++i) {
      const ModPair m = smp[i];
      if constexpr (I8) {
        uint32_t w[3][2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const uint64_t re = residue2(lr[j], m), im = residue2(li[j], m);
          w[0][j] = to_s8x2(re);
          w[1][j] = to_s8x2(im);
          w[2][j] = to_s8x2(mod2(add2(re, im), m));
        }
#pragma unroll
        for (int set = 0; set < 3; ++set) {
          const uint32_t v = __byte_perm(w[set][0], w[set][1], 0x5410);
          int8_t *d = reinterpret_cast<int8_t *>(d0 + (set * a.nmod + i) * a.plane_stride);
          if (vec) {
            *reinterpret_cast<uint32_t *>(d) = v;
          } else {
            for (int j = 0; j < nk; ++j) d[j] = (int8_t)(v >> (8 * j));
          }
        }
        continue;
      }
      __half2 o[3][2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const uint64_t re = residue2(lr[j], m), im = residue2(li[j], m);
        o[0][j] = to_h2(re);
        o[1][j] = to_h2(im);
        o[2][j] = to_h2(mod2(add2(re, im), m)); /* |re + im| <= 254: exact quotient */
      }
#pragma unroll
      for (int set = 0; set < 3; ++set) {
        __half *d = reinterpret_cast<__half *>(d0 + (set * a.nmod + i) * a.plane_stride);
        if (vec) {
          *reinterpret_cast<uint2 *>(d) = *reinterpret_cast<const uint2 *>(o[set]);
        } else {
          const __half h[4] = {__low2half(o[set][0]), __high2half(o[set][0]),
                               __low2half(o[set][1]), __high2half(o[set][1])};
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (j < nk) d[j] = h[j];
        }
      }
    }
  }
}

/* MN-contiguous complex source: 32x32 tile through shared memory; two
 * consecutive k per thread (binary16 or int8 planes) */
template <bool I8>
__global__ void zcrt_res_rcontig(ZResArgs a) {
  constexpr int ESZ = I8 ? 1 : 2;
  __shared__ double2 tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < a.rows && k < a.kdim) ? a.src[r + k * a.ld] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  const int kp = (ty * 32 + tx) & 15, rl0 = (ty * 32 + tx) >> 4;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int rl = rl0 + 16 * h;
    const int64_t r = r0 + rl, k = k0 + 2 * kp;
    if (r >= a.rows || k >= a.kdim) continue;
    const int e = row_exp(a.exps, a.exp_pair, r);
    const double f = a.frac ? a.frac[r] : 1.0;
    const double2 z0 = tile[2 * kp][rl], z1 = tile[2 * kp + 1][rl];
    const Limbs r0l = limbs_of(f * z0.x, e, a.beta), i0l = limbs_of(f * z0.y, e, a.beta);
    const Limbs r1l = limbs_of(f * z1.x, e, a.beta), i1l = limbs_of(f * z1.y, e, a.beta);
    const bool two = k + 1 < a.kdim;
    const bool vec = two && (a.plane_stride & (2 * ESZ - 1)) == 0 &&
                     (reinterpret_cast<uintptr_t>(a.planes + (r * a.ld_dst + k) * ESZ) &
                      (2 * ESZ - 1)) == 0;
#pragma unroll
    for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) { /* constant-bank operands, no indexed loads */
      if (i >= a.nmod) break;
      const ModConst m = a.mc[i];
      const ZRes3 x0 = zresidue(r0l, i0l, m, a.im_sign);
      const ZRes3 x1 = zresidue(r1l, i1l, m, a.im_sign);
      if constexpr (I8) {
        const uint32_t w[3] = {to_s8x2(pk2(x0.re, x1.re)), to_s8x2(pk2(x0.im, x1.im)),
                               to_s8x2(pk2(x0.sum, x1.sum))};
#pragma unroll
        for (int set = 0; set < 3; ++set) {
          int8_t *d = reinterpret_cast<int8_t *>(a.planes + (set * a.nmod + i) * a.plane_stride) +
                      r * a.ld_dst + k;
          if (vec) {
            *reinterpret_cast<uint16_t *>(d) = (uint16_t)w[set];
          } else {
            d[0] = (int8_t)w[set];
            if (two) d[1] = (int8_t)(w[set] >> 8);
          }
        }
        continue;
      }
      const __half2 v[3] = {__floats2half2_rn(x0.re, x1.re), __floats2half2_rn(x0.im, x1.im),
                            __floats2half2_rn(x0.sum, x1.sum)};
#pragma unroll
      for (int set = 0; set < 3; ++set) {
        __half *d = reinterpret_cast<__half *>(a.planes + (set * a.nmod + i) * a.plane_stride) +
                    r * a.ld_dst + k;
        if (vec) {
          *reinterpret_cast<__half2 *>(d) = v[set];
        } else {
          d[0] = __low2half(v[set]);
          if (two) d[1] = __high2half(v[set]);
        }
      }
    }
  }
}

struct ZCombArgs {
  CombArgs g;  /* moduli, reconstruction constants, residues (3 sets of nmod planes) */
  int exp_a_pair, exp_b_pair;
  double2 *c;
  int64_t ldc;
  double2 alpha, beta;
};

/* f32 holding a small integer (|x| < 2^22) to binary64 without the
 * conversion unit: x + 1.5 * 2^23 has the bit pattern 0x4B400000 + x, which
 * under the exponent of 2^52 gives 2^52 + 0x4B400000 + x */
__device__ __forceinline__ double small_f_to_d(float x) {
  return __hiloint2double(0x43300000, __float_as_int(x + RND_F)) - 4503600889856000.0;
}

/* byte u of two int8 residues whose sign bits were flipped (r + 128) as the
 * f32 value 1.5 * 2^23 + 128 + r: the byte under the bit pattern of 1.5 * 2^23 */
__device__ __forceinline__ float biased_byte_to_f(uint32_t qb, int u) {
  return __int_as_float((int)__byte_perm(qb, 0x4B400000u, 0x7650u + (uint32_t)u));
}

/* residues stream through the two accumulators, one modulus at a time: the
 * weighted-sum reconstruction keeps no per-modulus state.  Warp-specialised
 * like the real combine: warps 0-7 reconstruct 256-row tiles (one row per
 * thread), warp 8's lane 0 keeps the residues of ZCMB_STAGES tiles in flight. */
constexpr int ZCMB_CONSUMERS = ZCMB_THREADS / 32;
constexpr int ZCMB_BLOCK = ZCMB_THREADS + 32;

template <int NC>
__global__ void __launch_bounds__(ZCMB_BLOCK, 3) zcrt_combine_kernel(const __grid_constant__ ZCombArgs a) {
  using namespace hcbk::tc;
  extern __shared__ __align__(128) unsigned char cmb_smem[];
  __shared__ __align__(8) uint64_t full[ZCMB_STAGES], empty[ZCMB_STAGES];
  if (blockDim.x != ZCMB_BLOCK) { /* the tile covers ZCMB_ROWS rows only at this shape */
    if (threadIdx.x == 0) atomicCAS(a.g.err, 0, (int)ERR_LAUNCH_SHAPE);
    return;
  }
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nmod = a.g.nmod;
  int8_t *buf = reinterpret_cast<int8_t *>(cmb_smem);
  const int64_t row_tiles = (a.g.m + ZCMB_ROWS - 1) / ZCMB_ROWS;
  const size_t stage_elems = (size_t)3 * nmod * ZCMB_ROWS;
  if (tid == 0) {
    for (int s = 0; s < ZCMB_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], ZCMB_CONSUMERS);
    }
    mbar_fence_init();
  }
  __syncthreads();
  if (warp == ZCMB_CONSUMERS) { /* producer */
    if (lane == 0)
      ws_produce<ZCMB_STAGES, ZCMB_ROWS>(a.g.res, a.g.res_plane, a.g.ldr, 3 * nmod, row_tiles,
                                         a.g.n, a.g.n, 0, buf, full, empty, a.g.err);
    return;
  }
  for (TileWalk<ZCMB_STAGES> w((int)blockIdx.x, (int)gridDim.x, (int)row_tiles); w.col < a.g.n;
       w.next()) {
    const int s = w.s;
    if (!__all_sync(0xffffffffu, mbar_wait(&full[s], w.ph, a.g.err, ERR_TIMEOUT_COMBINE))) break;
    const int8_t *R = buf + s * stage_elems;
    /* two consecutive rows per thread: twice the independent FMA chains */
    const int64_t row = w.rt * ZCMB_ROWS + ZCMB_RPT * tid, col = w.col;
    CrtAcc<NC> acc_re[ZCMB_RPT], acc_im[ZCMB_RPT];
    if (row < a.g.m) {
#pragma unroll
      for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) { /* constant-bank weights and moduli */
        if (i >= nmod) break;
        const float p = a.g.p[i], ip = a.g.inv_p[i], hp = a.g.hp[i];
        /* the two rows' residues of each plane in one 2-byte load, sign bits
         * flipped; as f32 each is c = B + r with B = 1.5 * 2^23 + 128, so
         * differences of two are exact without removing B */
        const int o = ZCMB_RPT * tid;
        const uint32_t q1 = *reinterpret_cast<const uint16_t *>(R + i * ZCMB_ROWS + o) ^ 0x8080u;
        const uint32_t q2 =
            *reinterpret_cast<const uint16_t *>(R + (nmod + i) * ZCMB_ROWS + o) ^ 0x8080u;
        const uint32_t q3 =
            *reinterpret_cast<const uint16_t *>(R + (2 * nmod + i) * ZCMB_ROWS + o) ^ 0x8080u;
#pragma unroll
        for (int u = 0; u < ZCMB_RPT; ++u) {
          const float c1 = biased_byte_to_f(q1, u), c2 = biased_byte_to_f(q2, u);
          const float c3 = biased_byte_to_f(q3, u);
          const float t2 = c2 - (RND_F + 128.0f);             /* r2 */
          const double re = small_f_to_d(sym_f(mod_f(c1 - c2, p, ip), p, hp));
          const double im = small_f_to_d(sym_f(mod_f((c3 - c1) - t2, p, ip), p, hp));
#pragma unroll
          for (int k = 0; k < NC; ++k) {
            acc_re[u].S[k] = fma(re, a.g.w[i][k], acc_re[u].S[k]);
            acc_im[u].S[k] = fma(im, a.g.w[i][k], acc_im[u].S[k]);
          }
        }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]); /* the stage's residues are in registers */
    const int eb = row_exp(a.g.exp_b, a.exp_b_pair, col);
#pragma unroll
    for (int u = 0; u < ZCMB_RPT; ++u) {
      const int64_t r = row + u;
      if (r >= a.g.m) break;
      const int ea = row_exp(a.g.exp_a, a.exp_a_pair, r);
      double re = acc_re[u].finish(a.g, ea, eb);
      double im = acc_im[u].finish(a.g, ea, eb);
      if (a.g.inv_a) {
        const double sc = a.g.inv_a[r] * a.g.inv_b[col];
        re *= sc;
        im *= sc;
      }
      double2 *dst = a.c + r + col * a.ldc;
      double2 o;
      o.x = a.alpha.x * re - a.alpha.y * im;
      o.y = a.alpha.x * im + a.alpha.y * re;
      if (a.g.beta_nonzero) {
        const double2 cv = *dst;
        o.x = fma(a.beta.x, cv.x, fma(-a.beta.y, cv.y, o.x));
        o.y = fma(a.beta.x, cv.y, fma(a.beta.y, cv.x, o.y));
      }
      *dst = o;
    }
  }
}

/* persistent grid for a combine kernel: as many blocks as fit, at most one
 * per tile; opts in to the dynamic shared memory it needs */
template <class K>
static int combine_grid(K kernel, int threads, size_t smem, int64_t ntiles, int64_t *grid) {
  /* static shared memory counts against the same 48 KB default, so opt in
   * well below it */
  if (smem > 32 * 1024 &&
      cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return HCBK_ERR_LAUNCH;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
          cudaSuccess ||
      per_sm < 1)
    return HCBK_ERR_LAUNCH;
  const int64_t cap = (int64_t)hcbk_sm_count() * per_sm;
  *grid = ntiles < cap ? ntiles : cap;
  return HCBK_OK;
}

}  // namespace

extern "C" const int *hcbk_crt_moduli(int *count) {
  /* pairwise coprime, odd, <= 255 (symmetric residues fit |r| <= 127):
   * 255 = 3*5*17, 253 = 11*23, 247 = 13*19, 217 = 7*31, the rest prime */
  static const int M[HCBK_CRT_MAX_MODULI] = {255, 253, 251, 247, 241, 239, 233,
                                             229, 227, 223, 217, 211, 199, 197,
                                             193, 191, 181, 179, 173, 167};
  if (count) *count = HCBK_CRT_MAX_MODULI;
  return M;
}

extern "C" int hcbk_crt_residues(const hcbk_crt_prep *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->rows <= 0 || in->kdim <= 0 || in->nmod < 1 || in->nmod > HCBK_CRT_MAX_MODULI ||
      in->beta_bits < 1 || in->beta_bits > 53)
    return HCBK_ERR_ARGS;
  ResArgs a;
  a.src = in->src;
  a.ld = in->ld;
  a.rows = in->rows;
  a.kdim = in->kdim;
  a.exps = in->exps;
  a.frac = in->frac;
  a.beta = in->beta_bits;
  a.nmod = in->nmod;
  fill_mod_pairs(a.mp);
  a.planes = static_cast<char *>(in->planes);
  a.plane_stride = in->plane_stride;
  a.ld_dst = in->ld_dst;
  a.batch = in->batch > 1 ? in->batch : 1;
  a.src_bstride = a.batch > 1 ? in->src_bstride : 0;
  a.planes_bstride = a.batch > 1 ? in->planes_bstride : 0;
  if (in->k_contig) {
    const int64_t total = a.rows * ((a.kdim + 7) / 8) * a.batch;
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    if (in->i8)
      crt_res_kcontig<true><<<(unsigned)blocks, 256, 0, st>>>(a);
    else
      crt_res_kcontig<false><<<(unsigned)blocks, 256, 0, st>>>(a);
  } else {
    const int64_t kt = in->i8 ? 64 : 32; /* k per tile (crt_res_rcontig's KT) */
    const int64_t gx = (a.rows + 31) / 32, gy = (a.kdim + kt - 1) / kt;
    if (gy > 65535 || a.batch > 65535) return HCBK_ERR_ARGS;
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)a.batch);
    if (in->i8)
      crt_res_rcontig<true><<<grid, dim3(32, 8), 0, st>>>(a);
    else
      crt_res_rcontig<false><<<grid, dim3(32, 8), 0, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_crt_combine(const hcbk_crt_combine_args *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->m <= 0 || in->n <= 0 || in->nmod < 2 || in->nmod > HCBK_CRT_MAX_MODULI ||
      in->ldr < in->m || (in->ldr & 7) || (in->res_plane & 7) ||
      (reinterpret_cast<uintptr_t>(in->res) & 15) || !in->err)
    return HCBK_ERR_ARGS;
  CombArgs a;
  a.m = in->m;
  a.n = in->n;
  fill_comb_moduli(a, in->nmod);
  a.res = in->res;
  a.res_plane = in->res_plane;
  a.ldr = in->ldr;
  a.exp_a = in->exp_a;
  a.exp_b = in->exp_b;
  a.inv_a = in->inv_a;
  a.inv_b = in->inv_b;
  a.shift = in->shift;
  a.c = in->c;
  a.ldc = in->ldc;
  a.alpha = in->alpha;
  a.beta = in->beta;
  a.beta_nonzero = in->beta != 0.0;
  a.err = in->err;
  a.batch = in->batch > 1 ? in->batch : 1;
  a.res_bstride = a.batch > 1 ? in->res_bstride : 0;
  a.c_bstride = a.batch > 1 ? in->c_bstride : 0;
  if (a.res_bstride & 15) return HCBK_ERR_ARGS; /* bulk copies start on 16 bytes */
  const int64_t ntiles = (a.m + CMB_ROWS - 1) / CMB_ROWS * a.n * a.batch;
  if (ntiles > 0x7fffffff) return HCBK_ERR_ARGS;
  const size_t smem = (size_t)CMB_STAGES * a.nmod * CMB_ROWS * sizeof(int8_t);
  int64_t grid = 0;
  int rc;
  switch (a.nc) {
    case 1: rc = combine_grid(crt_combine_kernel<1>, CMB_BLOCK, smem, ntiles, &grid); break;
    case 2: rc = combine_grid(crt_combine_kernel<2>, CMB_BLOCK, smem, ntiles, &grid); break;
    case 3: rc = combine_grid(crt_combine_kernel<3>, CMB_BLOCK, smem, ntiles, &grid); break;
    default: rc = combine_grid(crt_combine_kernel<4>, CMB_BLOCK, smem, ntiles, &grid); break;
  }
  if (rc != HCBK_OK) return rc;
  switch (a.nc) {
    case 1: crt_combine_kernel<1><<<(unsigned)grid, CMB_BLOCK, smem, st>>>(a); break;
    case 2: crt_combine_kernel<2><<<(unsigned)grid, CMB_BLOCK, smem, st>>>(a); break;
    case 3: crt_combine_kernel<3><<<(unsigned)grid, CMB_BLOCK, smem, st>>>(a); break;
    default: crt_combine_kernel<4><<<(unsigned)grid, CMB_BLOCK, smem, st>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_zcrt_residues(const hcbk_zcrt_prep *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->rows <= 0 || in->kdim <= 0 || in->nmod < 1 || in->nmod > HCBK_CRT_MAX_MODULI ||
      in->beta_bits < 1 || in->beta_bits > 53)
    return HCBK_ERR_ARGS;
  ZResArgs a;
  a.src = static_cast<const double2 *>(in->src);
  a.ld = in->ld;
  a.rows = in->rows;
  a.kdim = in->kdim;
  a.exps = in->exps;
  a.exp_pair = in->exp_pair;
  a.frac = in->frac;
  a.im_sign = in->conj ? -1.0f : 1.0f;
  a.beta = in->beta_bits;
  a.nmod = in->nmod;
  fill_mod_consts(a.mc);
  fill_mod_pairs(a.mp);
  a.planes = static_cast<char *>(in->planes);
  a.plane_stride = in->plane_stride;
  a.ld_dst = in->ld_dst;
  if (in->k_contig) {
    const int64_t total = a.rows * ((a.kdim + 3) / 4);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 12;
    if (blocks > cap) blocks = cap;
    if (in->i8)
      zcrt_res_kcontig<true><<<(unsigned)blocks, 256, 0, st>>>(a);
    else
      zcrt_res_kcontig<false><<<(unsigned)blocks, 256, 0, st>>>(a);
  } else {
    const int64_t gx = (a.rows + 31) / 32, gy = (a.kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    if (in->i8)
      zcrt_res_rcontig<true><<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(a);
    else
      zcrt_res_rcontig<false><<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_zcrt_combine(const hcbk_zcrt_combine_args *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->m <= 0 || in->n <= 0 || in->nmod < 2 || in->nmod > HCBK_CRT_MAX_MODULI ||
      in->ldr < in->m || (in->ldr & 7) || (in->res_plane & 7) ||
      (reinterpret_cast<uintptr_t>(in->res) & 15) || !in->err)
    return HCBK_ERR_ARGS;
  ZCombArgs a;
  a.g.m = in->m;
  a.g.n = in->n;
  fill_comb_moduli(a.g, in->nmod);
  a.g.res = in->res;
  a.g.res_plane = in->res_plane;
  a.g.ldr = in->ldr;
  a.g.exp_a = in->exp_a;
  a.g.exp_b = in->exp_b;
  a.g.inv_a = in->inv_a;
  a.g.inv_b = in->inv_b;
  a.g.shift = in->shift;
  a.g.c = nullptr;
  a.g.ldc = 0;
  a.g.alpha = 0.0;
  a.g.beta = 0.0;
  a.g.beta_nonzero = in->beta_re != 0.0 || in->beta_im != 0.0;
  a.g.err = in->err;
  a.g.batch = 1; /* the complex combine takes one GEMM */
  a.g.res_bstride = a.g.c_bstride = 0;
  a.exp_a_pair = in->exp_a_pair;
  a.exp_b_pair = in->exp_b_pair;
  a.c = static_cast<double2 *>(in->c);
  a.ldc = in->ldc;
  a.alpha = make_double2(in->alpha_re, in->alpha_im);
  a.beta = make_double2(in->beta_re, in->beta_im);
  const int64_t ntiles = (a.g.m + ZCMB_ROWS - 1) / ZCMB_ROWS * a.g.n;
  const size_t smem = (size_t)ZCMB_STAGES * 3 * a.g.nmod * ZCMB_ROWS * sizeof(int8_t);
  int64_t grid = 0;
  int rc;
  switch (a.g.nc) {
    case 1: rc = combine_grid(zcrt_combine_kernel<1>, ZCMB_BLOCK, smem, ntiles, &grid); break;
    case 2: rc = combine_grid(zcrt_combine_kernel<2>, ZCMB_BLOCK, smem, ntiles, &grid); break;
    case 3: rc = combine_grid(zcrt_combine_kernel<3>, ZCMB_BLOCK, smem, ntiles, &grid); break;
    default: rc = combine_grid(zcrt_combine_kernel<4>, ZCMB_BLOCK, smem, ntiles, &grid); break;
  }
  if (rc != HCBK_OK) return rc;
  switch (a.g.nc) {
    case 1: zcrt_combine_kernel<1><<<(unsigned)grid, ZCMB_BLOCK, smem, st>>>(a); break;
    case 2: zcrt_combine_kernel<2><<<(unsigned)grid, ZCMB_BLOCK, smem, st>>>(a); break;
    case 3: zcrt_combine_kernel<3><<<(unsigned)grid, ZCMB_BLOCK, smem, st>>>(a); break;
    default: zcrt_combine_kernel<4><<<(unsigned)grid, ZCMB_BLOCK, smem, st>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
