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
 *      1024-element K chunks, then are reduced mod p_i with exact FP32 FMAs).
 *   4. This file's combine kernel rebuilds the exact integer product
 *      P' = A' B' (|P'| < (p_1...p_n)/2, guaranteed by the choice of n and
 *      beta) from (T_1..T_n) with Garner's mixed-radix algorithm, evaluates
 *      it in double-double, and writes
 *        C = alpha * P' * 2^(e_m + f_n - 2 beta) + beta * C.
 * The only roundings are the scaling in step 1 (relative 2^-(beta+1) of the
 * row / column maximum) and the final conversion to binary64.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "hcbk.h"

namespace {

/* symmetric residue of an integer-valued double |y| <= 2^53 modulo p:
 * q = rint(y / p) is within one of the true quotient (|y/p| error < 0.01),
 * and fma(-q, p, y) is exact because its exact value is a small integer. */
__device__ __forceinline__ int sym_mod_d(double y, double p, double inv_p, int hp) {
  const double q = rint(y * inv_p);
  int r = static_cast<int>(fma(-q, p, y));
  const int pi = static_cast<int>(p);
  if (r > hp) r -= pi;
  else if (r < -hp) r += pi;
  return r;
}

struct ResArgs {
  const double *src;
  int64_t ld;
  int64_t rows, kdim;
  const int *exps;
  int beta;
  int nmod;
  double p[HCBK_CRT_MAX_MODULI];
  double inv_p[HCBK_CRT_MAX_MODULI];
  char *planes;
  int64_t plane_stride; /* bytes */
  int64_t ld_dst;       /* elements */
};

/* scaled integer of one element (0 for zero / non-finite rows) */
__device__ __forceinline__ double scaled_int(double x, int e, int beta) {
  if (e == HCBK_OZ_NONFINITE || e == HCBK_OZ_ZERO) return 0.0;
  return rint(ldexp(x, beta - e));
}

/* K-contiguous source: 8 consecutive k per thread, 16-byte plane stores */
__global__ void crt_res_kcontig(ResArgs a) {
  struct alignas(16) H8 { __half v[8]; };
  const int64_t kq = (a.kdim + 7) / 8;
  const int64_t total = a.rows * kq;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = idx / kq;
    const int64_t k0 = (idx % kq) * 8;
    const int e = a.exps[r];
    double y[8];
#pragma unroll
    for (int j = 0; j < 8; ++j)
      y[j] = (k0 + j < a.kdim) ? scaled_int(a.src[r * a.ld + k0 + j], e, a.beta) : 0.0;
    for (int i = 0; i < a.nmod; ++i) {
      const double p = a.p[i], ip = a.inv_p[i];
      const int hp = (static_cast<int>(p) - 1) / 2;
      H8 out;
#pragma unroll
      for (int j = 0; j < 8; ++j) out.v[j] = __int2half_rn(sym_mod_d(y[j], p, ip, hp));
      __half *d = reinterpret_cast<__half *>(a.planes + i * a.plane_stride) + r * a.ld_dst + k0;
      if (k0 + 8 <= a.kdim && (reinterpret_cast<uintptr_t>(d) & 15) == 0) {
        *reinterpret_cast<H8 *>(d) = out;
      } else {
        for (int j = 0; j < 8; ++j)
          if (k0 + j < a.kdim) d[j] = out.v[j];
      }
    }
  }
}

/* MN-contiguous source: 32x32 tile through shared memory */
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
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int rl = ty + 8 * i;
    const int64_t r = r0 + rl, k = k0 + tx;
    if (r < a.rows && k < a.kdim) {
      const double y = scaled_int(tile[tx][rl], a.exps[r], a.beta);
      for (int m = 0; m < a.nmod; ++m) {
        const int hp = (static_cast<int>(a.p[m]) - 1) / 2;
        reinterpret_cast<__half *>(a.planes + m * a.plane_stride)[r * a.ld_dst + k] =
            __int2half_rn(sym_mod_d(y, a.p[m], a.inv_p[m], hp));
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
  int p[HCBK_CRT_MAX_MODULI];
  float inv_pf[HCBK_CRT_MAX_MODULI];
  /* minv[i] = (p_g0 ... p_(i-1))^-1 mod p_i over the moduli of i's group
   * before i (0 for a group's first modulus); gsize[j] = moduli in group j */
  int minv[HCBK_CRT_MAX_MODULI];
  int nq;
  int gsize[MAX_Q];
  double q[MAX_Q];
  double inv_q[MAX_Q];
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

/* symmetric residue of |v| < 2^22 modulo p (float reciprocal, one fix-up) */
__device__ __forceinline__ int sym_mod_i(int v, int p, float inv_p) {
  const int q = __float2int_rn(static_cast<float>(v) * inv_p);
  int r = v - q * p;
  const int hp = (p - 1) >> 1;
  if (r > hp) r -= p;
  else if (r < -hp) r += p;
  return r;
}

__global__ void crt_combine_kernel(CombArgs a) {
  const int64_t total = a.m * a.n;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = idx % a.m, col = idx / a.m;
    const int ea = a.exp_a[row], eb = a.exp_b[col];
    double out;
    if (ea == HCBK_OZ_NONFINITE || eb == HCBK_OZ_NONFINITE) {
      out = __longlong_as_double(0x7ff8000000000000ll);
    } else if (ea == HCBK_OZ_ZERO || eb == HCBK_OZ_ZERO) {
      out = 0.0;
    } else {
      const int16_t *t = a.res + row + col * a.ldr;
      /* 1. merge each group: with x the symmetric residue modulo
       *    Q = p_g0...p_(i-1), x += Q * ((r_i - x) Q^-1 mod p_i) is the
       *    symmetric residue modulo Q p_i (Q < 2^16, |x| < 2^15: every int
       *    product stays below 2^23) */
      double u[MAX_Q];
#pragma unroll
      for (int j = 0; j < MAX_Q; ++j) {
        if (j >= a.nq) break;
        const int i0 = GROUP * j;
        int x = t[i0 * a.res_plane];
        int qq = a.p[i0];
#pragma unroll
        for (int g = 1; g < GROUP; ++g) {
          if (g >= a.gsize[j]) break;
          const int i = i0 + g;
          const int r = t[i * a.res_plane];
          const int d = sym_mod_i(sym_mod_i(r - x, a.p[i], a.inv_pf[i]) * a.minv[i], a.p[i],
                                  a.inv_pf[i]);
          x += qq * d;
          qq *= a.p[i];
        }
        u[j] = static_cast<double>(x);
      }
      /* 2. Garner over the q_j (< 2^24): (x - v_j) * qinv < 2^48 is exact in
       *    binary64 and sym_mod_d reduces it exactly */
      double v[MAX_Q];
#pragma unroll
      for (int i = 0; i < MAX_Q; ++i) {
        if (i >= a.nq) break;
        double x = u[i];
        const int hq = (static_cast<int>(a.q[i]) - 1) / 2;
#pragma unroll
        for (int j = 0; j < MAX_Q; ++j) {
          if (j >= i) break;
          x = static_cast<double>(sym_mod_d((x - v[j]) * a.qinv[i][j], a.q[i], a.inv_q[i], hq));
        }
        v[i] = x;
      }
      /* 3. P' = v_0 + q_0 (v_1 + q_1 (v_2 + ...)), in double-double */
      double hi = 0.0, lo = 0.0;
#pragma unroll
      for (int i = MAX_Q - 1; i >= 0; --i) {
        if (i >= a.nq) continue;
        const double p = a.q[i];
        const double ph = hi * p;
        const double pl = fma(hi, p, -ph); /* exact product error */
        double s = ph + v[i];
        double bb = s - ph;
        double err = (ph - (s - bb)) + (v[i] - bb);
        lo = lo * p + pl + err;
        hi = s + lo;
        lo = lo - (hi - s);
      }
      const double x = hi + lo;
      const int e = ea + eb - a.shift;
      out = (e >= -1022 && e <= 1023) ? x * __longlong_as_double((long long)(e + 1023) << 52)
                                      : ldexp(x, e);
    }
    double *dst = a.c + row + col * a.ldc;
    out *= a.alpha;
    if (a.beta_nonzero) out = fma(a.beta, *dst, out);
    *dst = out;
  }
}

static void fill_moduli(int nmod, const int *moduli, double *p, double *inv_p) {
  for (int i = 0; i < nmod; ++i) {
    p[i] = moduli[i];
    inv_p[i] = 1.0 / moduli[i];
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
  fill_moduli(in->nmod, hcbk_crt_moduli(nullptr), a.p, a.inv_p);
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
  if (in->m <= 0 || in->n <= 0 || in->nmod < 2 || in->nmod > HCBK_CRT_MAX_MODULI)
    return HCBK_ERR_ARGS;
  CombArgs a;
  a.m = in->m;
  a.n = in->n;
  a.nmod = in->nmod;
  const int *M = hcbk_crt_moduli(nullptr);
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) {
    a.p[i] = M[i];
    a.inv_pf[i] = 1.0f / (float)M[i];
  }
  a.nq = (in->nmod + GROUP - 1) / GROUP;
  long long q[MAX_Q];
  for (int j = 0; j < MAX_Q; ++j) a.gsize[j] = 0;
  for (int i = 0; i < HCBK_CRT_MAX_MODULI; ++i) a.minv[i] = 0;
  for (int j = 0; j < a.nq; ++j) {
    const int i0 = GROUP * j;
    const int gs = in->nmod - i0 < GROUP ? in->nmod - i0 : GROUP;
    a.gsize[j] = gs;
    long long qq = M[i0];
    for (int g = 1; g < gs; ++g) {
      a.minv[i0 + g] = (int)inv_mod_ll(qq, M[i0 + g]);
      qq *= M[i0 + g];
    }
    q[j] = qq;
    a.q[j] = (double)q[j];
    a.inv_q[j] = 1.0 / (double)q[j];
  }
  for (int i = 0; i < MAX_Q; ++i)
    for (int j = 0; j < MAX_Q; ++j)
      a.qinv[i][j] = (i < a.nq && j < i) ? (double)inv_mod_ll(q[j], q[i]) : 0.0;
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
  const int64_t total = a.m * a.n;
  int64_t blocks = (total + 255) / 256;
  const int64_t cap = (int64_t)hcbk_sm_count() * 32;
  if (blocks > cap) blocks = cap;
  crt_combine_kernel<<<(unsigned)blocks, 256, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? HCBK_OK : HCBK_ERR_LAUNCH;
}
