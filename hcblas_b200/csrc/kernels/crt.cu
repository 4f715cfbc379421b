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
 *      beta) from (T_1..T_n) with Garner's mixed-radix algorithm, evaluates
 *      it in double-double, and writes
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

/* the same in binary64 for integral |y| < 2^51 */
__device__ __forceinline__ double sym_mod_d(double y, double q, double inv_q, double hq) {
  const double t = fma(y, inv_q, RND_D) - RND_D;
  double r = fma(-t, q, y);
  r = r > hq ? r - q : r;
  return r < -hq ? r + q : r;
}

/* small integer (|x| < 2^22) to f32 without the conversion unit */
__device__ __forceinline__ float small_int_to_f(int x) {
  return __int_as_float(0x4B400000 + x) - RND_F;
}

struct ModConst {
  float p, inv_p, hp;
  float c1, c2, c3, c4; /* 2^11, 2^22, 2^33, 2^44 mod p (symmetric) */
};

struct ResArgs {
  const double *src;
  int64_t ld;
  int64_t rows, kdim;
  const int *exps;
  int beta;
  int nmod;
  ModConst mc[HCBK_CRT_MAX_MODULI];
  char *planes;
  int64_t plane_stride; /* bytes */
  int64_t ld_dst;       /* elements */
};

/* 11-bit limbs of the scaled integer y = rint(x 2^(beta - e)), |y| <= 2^53:
 * y = l4 2^44 + l3 2^33 + l2 2^22 + l1 2^11 + l0 with |l0..l3| <= 2^10 and
 * |l4| <= 2^9, all exact in f32 (0 for zero / non-finite rows) */
struct Limbs {
  float l0, l1, l2, l3, l4;
};

__device__ __forceinline__ Limbs limbs_of(double x, int e, int beta) {
  Limbs L{0.f, 0.f, 0.f, 0.f, 0.f};
  if (e == HCBK_OZ_NONFINITE || e == HCBK_OZ_ZERO) return L;
  const double y = rint(ldexp(x, beta - e));
  const double h4 = rint(y * 0x1p-44);
  double r = fma(-h4, 0x1p44, y);
  const double h3 = rint(r * 0x1p-33);
  r = fma(-h3, 0x1p33, r);
  const double h2 = rint(r * 0x1p-22);
  r = fma(-h2, 0x1p22, r);
  const double h1 = rint(r * 0x1p-11);
  r = fma(-h1, 0x1p11, r);
  L.l0 = static_cast<float>(r);
  L.l1 = static_cast<float>(h1);
  L.l2 = static_cast<float>(h2);
  L.l3 = static_cast<float>(h3);
  L.l4 = static_cast<float>(h4);
  return L;
}

/* symmetric residue of the limb sum modulo one modulus.  |sum| <=
 * 2^10 (1 + 4 * 127) < 2^19, so |sum / p| < 3200 and the f32 quotient
 * sum * RN(1/p) is off by < 2e-4 -- less than the 0.5/p >= 0.002 distance of
 * any x/p (p odd) from a half-integer: the rounded quotient is exact and the
 * remainder already lies in [-(p-1)/2, (p-1)/2]. */
__device__ __forceinline__ float residue(const Limbs &L, const ModConst &m) {
  float t = fmaf(L.l4, m.c4, L.l0);
  t = fmaf(L.l3, m.c3, t);
  t = fmaf(L.l2, m.c2, t);
  t = fmaf(L.l1, m.c1, t);
  return mod_f(t, m.p, m.inv_p);
}

/* K-contiguous source: 8 consecutive k per thread, 16-byte plane stores */
__global__ void crt_res_kcontig(ResArgs a) {
  struct alignas(16) H8 { __half2 v[4]; };
  const int64_t kq = (a.kdim + 7) / 8;
  const int64_t total = a.rows * kq;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / kq;
    const int64_t k0 = (idx % kq) * 8;
    const int e = a.exps[r];
    Limbs L[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      L[j] = limbs_of((k0 + j < a.kdim) ? a.src[r * a.ld + k0 + j] : 0.0, e, a.beta);
    for (int i = 0; i < a.nmod; ++i) {
      const ModConst m = a.mc[i];
      H8 out;
#pragma unroll
      for (int j = 0; j < 4; ++j)
        out.v[j] = __floats2half2_rn(residue(L[2 * j], m), residue(L[2 * j + 1], m));
      __half *d = reinterpret_cast<__half *>(a.planes + i * a.plane_stride) + r * a.ld_dst + k0;
      if (k0 + 8 <= a.kdim && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
        *reinterpret_cast<H8 *>(d) = out;
      } else {
        const __half *h = reinterpret_cast<const __half *>(&out);
        for (int j = 0; j < 8; ++j)
          if (k0 + j < a.kdim) d[j] = h[j];
      }
    }
  }
}

/* MN-contiguous source: 32x32 tile through shared memory, each thread then
 * owns two consecutive k of one row (32-bit plane stores) */
__global__ void crt_res_rcontig(ResArgs a) {
  __shared__ double tile[32][33];
  const int64_t r0 = (int64_t)blockIdx.x * 32;
  const int64_t k0 = (int64_t)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y; /* 32 x 8 */
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int kl = ty + 8 * i;
    const int64_t r = r0 + tx, k = k0 + kl;
    tile[kl][tx] = (r < a.rows && k < a.kdim) ? a.src[r + k * a.ld] : 0.0;
  }
  __syncthreads();
  /* 256 threads = 16 k-pairs x 16 rows, twice */
  const int kp = (ty * 32 + tx) & 15, rl0 = (ty * 32 + tx) >> 4;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int rl = rl0 + 16 * h;
    const int64_t r = r0 + rl, k = k0 + 2 * kp;
    if (r >= a.rows || k >= a.kdim) continue;
    const int e = a.exps[r];
    const Limbs L0 = limbs_of(tile[2 * kp][rl], e, a.beta);
    const Limbs L1 = limbs_of(tile[2 * kp + 1][rl], e, a.beta);
    const bool two = k + 1 < a.kdim;
    for (int i = 0; i < a.nmod; ++i) {
      const ModConst m = a.mc[i];
      const __half2 v = __floats2half2_rn(residue(L0, m), residue(L1, m));
      __half *d = reinterpret_cast<__half *>(a.planes + i * a.plane_stride) + r * a.ld_dst + k;
      if (two && (reinterpret_cast<uintptr_t>(d) & 3) == 0) {
        *reinterpret_cast<__half2 *>(d) = v;
      } else {
        d[0] = __low2half(v);
        if (two) d[1] = __high2half(v);
      }
    }
  }
}

/* residues merge in groups of GROUP moduli: q_j = p_3j p_3j+1 p_3j+2 < 2^24 */
constexpr int GROUP = 3;
constexpr int MAX_Q = (HCBK_CRT_MAX_MODULI + GROUP - 1) / GROUP;

struct CombArgs {
  int64_t m, n;
  int nmod;
  float p[HCBK_CRT_MAX_MODULI];
  float inv_p[HCBK_CRT_MAX_MODULI];
  float hp[HCBK_CRT_MAX_MODULI];
  /* minv[i] = (p_g0 ... p_(i-1))^-1 mod p_i over the moduli of i's group
   * before i (0 for a group's first modulus); gsize[j] = moduli in group j */
  float minv[HCBK_CRT_MAX_MODULI];
  int nq;
  int gsize[MAX_Q];
  double q[MAX_Q];
  double inv_q[MAX_Q];
  double hq[MAX_Q];
  /* qinv[i][j] = q_j^-1 mod q_i (j < i) */
  double qinv[MAX_Q][MAX_Q];
  const int16_t *res;
  int64_t res_plane; /* elements between residue planes */
  int64_t ldr;
  const int *exp_a;
  const int *exp_b;
  int shift;
  double *c;
  int64_t ldc;
  double alpha, beta;
  int beta_nonzero;
};

/* P' * 2^(ea + eb - shift) for one output element from its n residues
 * (already in f32), Garner over groups of three moduli */
template <class Res>
__device__ __forceinline__ double crt_value(const CombArgs &a, const Res &t, int ea, int eb) {
  if (ea == HCBK_OZ_NONFINITE || eb == HCBK_OZ_NONFINITE)
    return __longlong_as_double(0x7ff8000000000000ll);
  if (ea == HCBK_OZ_ZERO || eb == HCBK_OZ_ZERO) return 0.0;
  /* 1. merge each group in f32: with x the symmetric residue modulo
   *    Q = p_g0...p_(i-1), x += Q * (((r_i - x) mod p_i) Q^-1 mod p_i) is the
   *    symmetric residue modulo Q p_i (Q < 2^16, |x| < 2^23: exact) */
  double v[MAX_Q];
#pragma unroll
  for (int j = 0; j < MAX_Q; ++j) {
    if (j >= a.nq) break;
    const int i0 = GROUP * j;
    float x = t[i0];
    float qq = a.p[i0];
#pragma unroll
    for (int g = 1; g < GROUP; ++g) {
      if (g >= a.gsize[j]) break;
      const int i = i0 + g;
      const float d0 = mod_f(t[i] - x, a.p[i], a.inv_p[i]);
      /* |d0 * minv| < 1.5 * 255 * 254 < 2^17: exact quotient, symmetric result */
      const float d = mod_f(d0 * a.minv[i], a.p[i], a.inv_p[i]);
      x = fmaf(qq, d, x);
      qq *= a.p[i];
    }
    /* 2. Garner over the q_j (< 2^24): (x - v_j) qinv < 2^48, exact */
    double xd = static_cast<double>(x);
#pragma unroll
    for (int l = 0; l < MAX_Q; ++l) {
      if (l >= j) break;
      xd = sym_mod_d((xd - v[l]) * a.qinv[j][l], a.q[j], a.inv_q[j], a.hq[j]);
    }
    v[j] = xd;
  }
  /* 3. P' = v_0 + q_0 (v_1 + q_1 (v_2 + ...)), in double-double */
  double hi = 0.0, lo = 0.0;
#pragma unroll
  for (int i = MAX_Q - 1; i >= 0; --i) {
    if (i >= a.nq) continue;
    const double p = a.q[i];
    const double ph = hi * p;
    const double pl = fma(hi, p, -ph); /* exact product error */
    const double s = ph + v[i];
    const double bb = s - ph;
    const double err = (ph - (s - bb)) + (v[i] - bb);
    lo = fma(lo, p, pl + err);
    hi = s + lo;
    lo = lo - (hi - s);
  }
  const double x = hi + lo;
  const int e = ea + eb - a.shift;
  return (e >= -1022 && e <= 1023) ? x * __longlong_as_double((long long)(e + 1023) << 52)
                                   : ldexp(x, e);
}

/* one element per thread, consecutive threads on consecutive rows of one
 * column (coalesced residue loads and C stores); grid.y strides columns */
__global__ void __launch_bounds__(256) crt_combine_kernel(CombArgs a) {
  for (int64_t col = blockIdx.y; col < a.n; col += gridDim.y) {
    const int eb = a.exp_b[col];
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < a.m;
         row += (int64_t)gridDim.x * blockDim.x) {
      const int16_t *tp = a.res + row + col * a.ldr;
      float t[HCBK_CRT_MAX_MODULI];
#pragma unroll
      for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i)
        t[i] = i < a.nmod ? small_int_to_f(tp[i * a.res_plane]) : 0.f;
      double *dst = a.c + row + col * a.ldc;
      double o = a.alpha * crt_value(a, t, a.exp_a[row], eb);
      if (a.beta_nonzero) o = fma(a.beta, *dst, o);
      *dst = o;
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
    m.c1 = pow2_mod_sym(11, M[i]);
    m.c2 = pow2_mod_sym(22, M[i]);
    m.c3 = pow2_mod_sym(33, M[i]);
    m.c4 = pow2_mod_sym(44, M[i]);
  }
}

/* moduli, group constants and Garner inverses of the combine */
static void fill_comb_moduli(CombArgs &a, int nmod) {
  const int *M = hcbk_crt_moduli(nullptr);
  a.nmod = nmod;
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) {
    a.p[i] = (float)M[i];
    a.inv_p[i] = 1.0f / (float)M[i];
    a.hp[i] = (float)((M[i] - 1) / 2);
    a.minv[i] = 0.f;
  }
  a.nq = (nmod + GROUP - 1) / GROUP;
  long long q[MAX_Q];
  for (int j = 0; j < MAX_Q; ++j) a.gsize[j] = 0;
  for (int j = 0; j < a.nq; ++j) {
    const int i0 = GROUP * j;
    const int gs = nmod - i0 < GROUP ? nmod - i0 : GROUP;
    a.gsize[j] = gs;
    long long qq = M[i0];
    for (int g = 1; g < gs; ++g) {
      a.minv[i0 + g] = (float)inv_mod_ll(qq, M[i0 + g]);
      qq *= M[i0 + g];
    }
    q[j] = qq;
    a.q[j] = (double)q[j];
    a.inv_q[j] = 1.0 / (double)q[j];
    a.hq[j] = (double)((q[j] - 1) / 2);
  }
  for (int i = 0; i < MAX_Q; ++i)
    for (int j = 0; j < MAX_Q; ++j)
      a.qinv[i][j] = (i < a.nq && j < i) ? (double)inv_mod_ll(q[j], q[i]) : 0.0;
}

/* ------------------------------------------------ complex (ZGEMM) path --
 * 3M (Karatsuba) in modular arithmetic, where it is exact:
 *   T1 = Ar Br, T2 = Ai Bi, T3 = (Ar + Ai)(Br + Bi)   (mod p, one GEMM each)
 *   Re = T1 - T2,  Im = T3 - T1 - T2                  (mod p, then Garner)
 * Real and imaginary parts of a row share one exponent (the larger), so
 * Ar' + Ai' is the residue sum of one scaled integer pair. */

struct ZResArgs {
  const double2 *src;
  int64_t ld;
  int64_t rows, kdim;
  const int *exps;
  int exp_pair;    /* exponent of row r = max(exps[2r], exps[2r+1]) */
  float im_sign;   /* -1 for a conjugate-transposed operand */
  int beta;
  int nmod;
  ModConst mc[HCBK_CRT_MAX_MODULI];
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

/* K-contiguous complex source: 8 consecutive k per thread, 16-byte stores */
__global__ void zcrt_res_kcontig(ZResArgs a) {
  struct alignas(16) H8 { __half2 v[4]; };
  const int64_t kq = (a.kdim + 7) / 8;
  const int64_t total = a.rows * kq;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / kq;
    const int64_t k0 = (idx % kq) * 8;
    const int e = row_exp(a.exps, a.exp_pair, r);
    Limbs lr[8], li[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const double2 z = (k0 + j < a.kdim) ? a.src[r * a.ld + k0 + j] : make_double2(0.0, 0.0);
      lr[j] = limbs_of(z.x, e, a.beta);
      li[j] = limbs_of(z.y, e, a.beta);
    }
    for (int i = 0; i < a.nmod; ++i) {
      const ModConst m = a.mc[i];
      H8 o[3];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const ZRes3 x0 = zresidue(lr[2 * j], li[2 * j], m, a.im_sign);
        const ZRes3 x1 = zresidue(lr[2 * j + 1], li[2 * j + 1], m, a.im_sign);
        o[0].v[j] = __floats2half2_rn(x0.re, x1.re);
        o[1].v[j] = __floats2half2_rn(x0.im, x1.im);
        o[2].v[j] = __floats2half2_rn(x0.sum, x1.sum);
      }
#pragma unroll
      for (int set = 0; set < 3; ++set) {
        __half *d = reinterpret_cast<__half *>(a.planes + (set * a.nmod + i) * a.plane_stride) +
                    r * a.ld_dst + k0;
        if (k0 + 8 <= a.kdim && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
          *reinterpret_cast<H8 *>(d) = o[set];
        } else {
          const __half *h = reinterpret_cast<const __half *>(&o[set]);
          for (int j = 0; j < 8; ++j)
            if (k0 + j < a.kdim) d[j] = h[j];
        }
      }
    }
  }
}

/* MN-contiguous complex source: 32x32 tile through shared memory */
__global__ void zcrt_res_rcontig(ZResArgs a) {
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
    const double2 z0 = tile[2 * kp][rl], z1 = tile[2 * kp + 1][rl];
    const Limbs r0l = limbs_of(z0.x, e, a.beta), i0l = limbs_of(z0.y, e, a.beta);
    const Limbs r1l = limbs_of(z1.x, e, a.beta), i1l = limbs_of(z1.y, e, a.beta);
    const bool two = k + 1 < a.kdim;
    for (int i = 0; i < a.nmod; ++i) {
      const ModConst m = a.mc[i];
      const ZRes3 x0 = zresidue(r0l, i0l, m, a.im_sign);
      const ZRes3 x1 = zresidue(r1l, i1l, m, a.im_sign);
      const __half2 v[3] = {__floats2half2_rn(x0.re, x1.re), __floats2half2_rn(x0.im, x1.im),
                            __floats2half2_rn(x0.sum, x1.sum)};
#pragma unroll
      for (int set = 0; set < 3; ++set) {
        __half *d = reinterpret_cast<__half *>(a.planes + (set * a.nmod + i) * a.plane_stride) +
                    r * a.ld_dst + k;
        if (two && (reinterpret_cast<uintptr_t>(d) & 3) == 0) {
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
  CombArgs g;  /* moduli, Garner constants, residues (3 sets of nmod planes) */
  int exp_a_pair, exp_b_pair;
  double2 *c;
  int64_t ldc;
  double2 alpha, beta;
};

/* residues of one element kept in shared memory, [modulus][thread]: the
 * complex combine holds two sets, which in registers would cut occupancy */
struct SmemRes {
  const float *base;
  __device__ __forceinline__ float operator[](int i) const { return base[i * 256]; }
};

__global__ void __launch_bounds__(256) zcrt_combine_kernel(ZCombArgs a) {
  __shared__ float sres[2][HCBK_CRT_MAX_MODULI][256];
  const int nmod = a.g.nmod;
  const int tid = threadIdx.x;
  for (int64_t col = blockIdx.y; col < a.g.n; col += gridDim.y) {
    const int eb = row_exp(a.g.exp_b, a.exp_b_pair, col);
    for (int64_t row = (int64_t)blockIdx.x * blockDim.x + tid; row < a.g.m;
         row += (int64_t)gridDim.x * blockDim.x) {
      const int ea = row_exp(a.g.exp_a, a.exp_a_pair, row);
      const int16_t *tp = a.g.res + row + col * a.g.ldr;
#pragma unroll 4
      for (int i = 0; i < nmod; ++i) {
        const float t1 = small_int_to_f(tp[(int64_t)i * a.g.res_plane]);
        const float t2 = small_int_to_f(tp[(int64_t)(nmod + i) * a.g.res_plane]);
        const float t3 = small_int_to_f(tp[(int64_t)(2 * nmod + i) * a.g.res_plane]);
        sres[0][i][tid] = sym_f(mod_f(t1 - t2, a.g.p[i], a.g.inv_p[i]), a.g.p[i], a.g.hp[i]);
        sres[1][i][tid] = sym_f(mod_f(t3 - t1 - t2, a.g.p[i], a.g.inv_p[i]), a.g.p[i], a.g.hp[i]);
      }
      const double re = crt_value(a.g, SmemRes{&sres[0][0][tid]}, ea, eb);
      const double im = crt_value(a.g, SmemRes{&sres[1][0][tid]}, ea, eb);
      double2 *dst = a.c + row + col * a.ldc;
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
  a.beta = in->beta_bits;
  a.nmod = in->nmod;
  fill_mod_consts(a.mc);
  a.planes = static_cast<char *>(in->planes);
  a.plane_stride = in->plane_stride;
  a.ld_dst = in->ld_dst;
  if (in->k_contig) {
    const int64_t total = a.rows * ((a.kdim + 7) / 8);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    crt_res_kcontig<<<(unsigned)blocks, 256, 0, st>>>(a);
  } else {
    const int64_t gx = (a.rows + 31) / 32, gy = (a.kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    crt_res_rcontig<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_crt_combine(const hcbk_crt_combine_args *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->m <= 0 || in->n <= 0 || in->nmod < 2 || in->nmod > HCBK_CRT_MAX_MODULI ||
      (in->ldr & 1) || (in->res_plane & 1) || (reinterpret_cast<uintptr_t>(in->res) & 3))
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
  a.shift = in->shift;
  a.c = in->c;
  a.ldc = in->ldc;
  a.alpha = in->alpha;
  a.beta = in->beta;
  a.beta_nonzero = in->beta != 0.0;
  int64_t gx = (a.m + 255) / 256;
  if (gx > 65535) gx = 65535;
  const int64_t gy = a.n < 65535 ? a.n : 65535;
  crt_combine_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, 0, st>>>(a);
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
  a.im_sign = in->conj ? -1.0f : 1.0f;
  a.beta = in->beta_bits;
  a.nmod = in->nmod;
  fill_mod_consts(a.mc);
  a.planes = static_cast<char *>(in->planes);
  a.plane_stride = in->plane_stride;
  a.ld_dst = in->ld_dst;
  if (in->k_contig) {
    const int64_t total = a.rows * ((a.kdim + 7) / 8);
    int64_t blocks = (total + 255) / 256;
    const int64_t cap = (int64_t)hcbk_sm_count() * 16;
    if (blocks > cap) blocks = cap;
    zcrt_res_kcontig<<<(unsigned)blocks, 256, 0, st>>>(a);
  } else {
    const int64_t gx = (a.rows + 31) / 32, gy = (a.kdim + 31) / 32;
    if (gy > 65535) return HCBK_ERR_ARGS;
    zcrt_res_rcontig<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}

extern "C" int hcbk_zcrt_combine(const hcbk_zcrt_combine_args *in, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (in->m <= 0 || in->n <= 0 || in->nmod < 2 || in->nmod > HCBK_CRT_MAX_MODULI)
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
  a.g.shift = in->shift;
  a.g.c = nullptr;
  a.g.ldc = 0;
  a.g.alpha = 0.0;
  a.g.beta = 0.0;
  a.g.beta_nonzero = in->beta_re != 0.0 || in->beta_im != 0.0;
  a.exp_a_pair = in->exp_a_pair;
  a.exp_b_pair = in->exp_b_pair;
  a.c = static_cast<double2 *>(in->c);
  a.ldc = in->ldc;
  a.alpha = make_double2(in->alpha_re, in->alpha_im);
  a.beta = make_double2(in->beta_re, in->beta_im);
  int64_t gx = (a.g.m + 255) / 256;
  if (gx > 65535) gx = 65535;
  const int64_t gy = a.g.n < 65535 ? a.g.n : 65535;
  zcrt_combine_kernel<<<dim3((unsigned)gx, (unsigned)gy), 256, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
