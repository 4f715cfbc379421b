/*
 * gemm_oracle.c -- CPU oracle for the GEMM hot path.  TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this file's shared object, and only as the checker.  The product library
 * (hcblas_b200/libhcblas.so) never links or calls it.
 *
 * What it restates.  hcBLAS checks every GEMM against host CBLAS
 * (test/unit/hcblas_sgemm.cpp:28 `#include <cblas.h>`, linked with -lblas at
 * test/unit/CMakeLists.txt:30; calls such as cblas_sgemm(CblasColMajor, ...)
 * at test/unit/hcblas_sgemm.cpp:252).  CBLAS is a third-party dependency that
 * is not vendored and carries no version pin; its published algorithm is the
 * netlib reference BLAS xGEMM (dgemm.f / zgemm.f):
 *
 *     C := alpha * op(A) * op(B) + beta * C,
 *     op(X) = X, X^T or X^H (conjugate transpose, complex only),
 *     beta == 0  =>  C is not read (it is overwritten),
 *     row-major via the CBLAS identity  C^T = op(B)^T op(A)^T.
 *
 * This file evaluates that definition directly, with more precision than the
 * library under test:
 *   - S, C, H (binary32 / complex binary32 / binary16 inputs): every product
 *     of two inputs is exact in binary64, and the K-term sums are carried in
 *     binary64 ("FP64 oracle").
 *   - D, Z (binary64 inputs): products are split exactly with fma() and the
 *     sums are carried in double-double (Dekker / Knuth TwoSum, TwoProd via
 *     FMA), i.e. ~106 significant bits ("double-double oracle").
 * It writes C rounded to the storage type (what a CBLAS call would leave in
 * C) and, optionally, the high-precision result in binary64 (hi part) so that
 * normwise errors can be measured against it.
 *
 * Addressing follows the hcBLAS class API (include/hcblaslib.h:215-231 of the
 * reference): element offsets aOffset/bOffset/cOffset are added to the base
 * pointers, leading dimensions are in elements, order RowMajor=0/ColMajor=1
 * (lib/include/hcblaslib.h:47).  Unlike hcBLAS (lib/src/hcblas.cpp:1346, which
 * maps OP_C to a plain transpose), conjugate transpose really conjugates: that
 * is CBLAS's definition and the one this library implements.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).  The
 * -ffp-contract=off flag matters: the TwoSum error terms must not be fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { ORC_S = 0, ORC_D = 1, ORC_C = 2, ORC_Z = 3, ORC_H = 4 };
enum { ORC_ROW = 0, ORC_COL = 1 };
enum { ORC_N = 0, ORC_T = 1, ORC_CONJ = 2 };

/* ---------------- IEEE binary16 <-> binary64 (from the IEEE 754 format) ---- */

double oracle_half_to_double(uint16_t h) {
  int sign = (h >> 15) & 1;
  int exp = (h >> 10) & 0x1f;
  int man = h & 0x3ff;
  double v;
  if (exp == 0) {
    v = ldexp((double)man, -24); /* subnormal: man * 2^-24 */
  } else if (exp == 31) {
    v = man ? NAN : INFINITY;
  } else {
    v = ldexp((double)(man | 0x400), exp - 25);
  }
  return sign ? -v : v;
}

/* Round a binary64 value to the nearest binary16 (ties to even). */
uint16_t oracle_double_to_half(double x) {
  uint16_t sign = signbit(x) ? 0x8000 : 0;
  double a = fabs(x);
  if (isnan(x)) return 0x7e00;
  if (a == 0.0) return sign;
  /* Largest finite half is 65504; values >= 65520 round to infinity. */
  if (a >= 65520.0) return sign | 0x7c00;
  int e;
  frexp(a, &e); /* a = f * 2^e, f in [0.5, 1) */
  int unbiased = e - 1; /* a in [2^unbiased, 2^(unbiased+1)) */
  double q; /* quantum (spacing) of half at this magnitude */
  if (unbiased < -14) q = ldexp(1.0, -24); /* subnormal range */
  else q = ldexp(1.0, unbiased - 10);
  double r = a / q; /* exact: power-of-two scaling */
  double fl = floor(r);
  double diff = r - fl;
  double n;
  if (diff > 0.5) n = fl + 1.0;
  else if (diff < 0.5) n = fl;
  else n = (fmod(fl, 2.0) == 0.0) ? fl : fl + 1.0;
  double v = n * q;
  if (v >= 65520.0) return sign | 0x7c00;
  /* Re-encode v exactly. */
  if (v < ldexp(1.0, -14)) {
    return sign | (uint16_t)(v / ldexp(1.0, -24));
  }
  int e2;
  double f2 = frexp(v, &e2);
  int E = e2 - 1 + 15;
  uint16_t man = (uint16_t)((f2 * 2.0 - 1.0) * 1024.0);
  if (E >= 31) return sign | 0x7c00;
  return sign | (uint16_t)(E << 10) | man;
}

/* ---------------- double-double arithmetic ------------------------------- */

typedef struct { double hi, lo; } dd_t;

static inline dd_t two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double err = (a - (s - bb)) + (b - bb);
  dd_t r = {s, err};
  return r;
}

static inline dd_t quick_two_sum(double a, double b) {
  double s = a + b;
  double err = b - (s - a);
  dd_t r = {s, err};
  return r;
}

static inline dd_t dd_add(dd_t x, dd_t y) {
  dd_t s = two_sum(x.hi, y.hi);
  dd_t t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}

/* exact product a*b as a double-double (TwoProd with FMA) */
static inline dd_t two_prod(double a, double b) {
  double p = a * b;
  double e = fma(a, b, -p);
  dd_t r = {p, e};
  return r;
}

static inline dd_t dd_mul(dd_t x, dd_t y) {
  dd_t p = two_prod(x.hi, y.hi);
  p.lo += x.hi * y.lo + x.lo * y.hi;
  return quick_two_sum(p.hi, p.lo);
}

static inline dd_t dd_from(double a) {
  dd_t r = {a, 0.0};
  return r;
}

/* ---------------- element access ------------------------------------------ */

/* Read element (i, j) of a stored matrix X (not yet op'ed) as (re, im). */
static inline void load_elem(int dtype, int order, const void *X, int64_t off,
                             int64_t ld, int64_t i, int64_t j, double *re,
                             double *im) {
  int64_t idx = (order == ORC_COL) ? off + i + j * ld : off + i * ld + j;
  *re = 0.0;
  *im = 0.0;
  switch (dtype) {
    case ORC_S: *re = ((const float *)X)[idx]; *im = 0; break;
    case ORC_D: *re = ((const double *)X)[idx]; *im = 0; break;
    case ORC_C:
      *re = ((const float *)X)[2 * idx];
      *im = ((const float *)X)[2 * idx + 1];
      break;
    case ORC_Z:
      *re = ((const double *)X)[2 * idx];
      *im = ((const double *)X)[2 * idx + 1];
      break;
    case ORC_H:
      *re = oracle_half_to_double(((const uint16_t *)X)[idx]);
      *im = 0;
      break;
  }
}

static inline void store_elem(int dtype, int order, void *X, int64_t off,
                              int64_t ld, int64_t i, int64_t j, double re,
                              double im) {
  int64_t idx = (order == ORC_COL) ? off + i + j * ld : off + i * ld + j;
  switch (dtype) {
    case ORC_S: ((float *)X)[idx] = (float)re; break;
    case ORC_D: ((double *)X)[idx] = re; break;
    case ORC_C:
      ((float *)X)[2 * idx] = (float)re;
      ((float *)X)[2 * idx + 1] = (float)im;
      break;
    case ORC_Z:
      ((double *)X)[2 * idx] = re;
      ((double *)X)[2 * idx + 1] = im;
      break;
    case ORC_H: ((uint16_t *)X)[idx] = oracle_double_to_half(re); break;
  }
}

/*
 * Materialise op(X) as a dense column-major binary64 matrix of R x S
 * (re and im planes), where op(X)(r, s) = X(r, s), X(s, r) or conj(X(s, r)).
 */
static void materialise_op(int dtype, int order, int trans, const void *X,
                           int64_t off, int64_t ld, int64_t R, int64_t S,
                           double *re, double *im) {
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < S; ++s) {
    for (int64_t r = 0; r < R; ++r) {
      double a, b;
      if (trans == ORC_N) load_elem(dtype, order, X, off, ld, r, s, &a, &b);
      else load_elem(dtype, order, X, off, ld, s, r, &a, &b);
      if (trans == ORC_CONJ) b = -b;
      re[r + s * R] = a;
      im[r + s * R] = b;
    }
  }
}

static int is_complex(int dtype) { return dtype == ORC_C || dtype == ORC_Z; }
static int is_wide(int dtype) { return dtype == ORC_D || dtype == ORC_Z; }

/*
 * oracle_gemm: C := alpha*op(A)*op(B) + beta*C with CBLAS semantics.
 *
 *   dtype     ORC_S/D/C/Z/H
 *   order     0 = RowMajor, 1 = ColMajor (hcblasOrder values)
 *   transa/b  0 = N, 1 = T, 2 = C (conjugate transpose)
 *   alpha,beta  {re, im} in binary64 (im ignored for real types)
 *   A,B,C     base pointers; *_off element offsets; ld* leading dimensions
 *   ref_out   optional (may be NULL): the high-precision result, as binary64
 *             (hi part) in a dense column-major M x N array; complex types
 *             store interleaved {re, im} pairs.
 *   nthreads  OpenMP threads (<= 0: library default)
 *
 * Returns 0, or -1 on a bad argument.
 */
int oracle_gemm(int dtype, int order, int transa, int transb, int64_t M,
                int64_t N, int64_t K, const double *alpha, const void *A,
                int64_t a_off, int64_t lda, const void *B, int64_t b_off,
                int64_t ldb, const double *beta, void *C, int64_t c_off,
                int64_t ldc, double *ref_out, int nthreads) {
  if (M < 0 || N < 0 || K < 0) return -1;
  if (dtype < ORC_S || dtype > ORC_H) return -1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const int cplx = is_complex(dtype);
  const int wide = is_wide(dtype);
  const double ar = alpha[0], ai = cplx ? alpha[1] : 0.0;
  const double br = beta[0], bi = cplx ? beta[1] : 0.0;
  const int beta_zero = (br == 0.0 && bi == 0.0);
  /* netlib xGEMM: alpha == 0 -> C := beta*C without referencing A or B */
  const int alpha_zero = (ar == 0.0 && ai == 0.0);
  const int64_t Keff = alpha_zero ? 0 : K;

  double *opA_re = (double *)malloc(sizeof(double) * (size_t)(M * K + 1));
  double *opA_im = (double *)malloc(sizeof(double) * (size_t)(M * K + 1));
  double *opB_re = (double *)malloc(sizeof(double) * (size_t)(K * N + 1));
  double *opB_im = (double *)malloc(sizeof(double) * (size_t)(K * N + 1));
  if (!opA_re || !opA_im || !opB_re || !opB_im) {
    free(opA_re); free(opA_im); free(opB_re); free(opB_im);
    return -1;
  }
  /* op(A) is M x K, op(B) is K x N.  Transpose op(A) once more so that the
   * inner loop walks both operands contiguously: At[k + m*K] = op(A)(m, k). */
  double *At_re = (double *)malloc(sizeof(double) * (size_t)(M * K + 1));
  double *At_im = (double *)malloc(sizeof(double) * (size_t)(M * K + 1));
  materialise_op(dtype, order, transa, A, a_off, lda, M, K, opA_re, opA_im);
  materialise_op(dtype, order, transb, B, b_off, ldb, K, N, opB_re, opB_im);
#pragma omp parallel for schedule(static)
  for (int64_t m = 0; m < M; ++m)
    for (int64_t k = 0; k < K; ++k) {
      At_re[k + m * K] = opA_re[m + k * M];
      At_im[k + m * K] = opA_im[m + k * M];
    }
  free(opA_re);
  free(opA_im);

#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int64_t n = 0; n < N; ++n) {
    for (int64_t m = 0; m < M; ++m) {
      const double *ar_row = At_re + m * K, *ai_row = At_im + m * K;
      const double *br_col = opB_re + n * K, *bi_col = opB_im + n * K;
      double out_re, out_im, hp_re, hp_im;
      if (wide) {
        dd_t sr = dd_from(0.0), si = dd_from(0.0);
        for (int64_t k = 0; k < Keff; ++k) {
          sr = dd_add(sr, two_prod(ar_row[k], br_col[k]));
          if (cplx) {
            sr = dd_add(sr, two_prod(-ai_row[k], bi_col[k]));
            si = dd_add(si, two_prod(ar_row[k], bi_col[k]));
            si = dd_add(si, two_prod(ai_row[k], br_col[k]));
          }
        }
        /* alpha * acc (complex multiply in double-double) */
        dd_t rr = dd_add(dd_mul(dd_from(ar), sr),
                         dd_mul(dd_from(-ai), si));
        dd_t ri = dd_add(dd_mul(dd_from(ar), si), dd_mul(dd_from(ai), sr));
        if (!beta_zero) {
          double cr, ci;
          load_elem(dtype, order, C, c_off, ldc, m, n, &cr, &ci);
          rr = dd_add(rr, dd_add(two_prod(br, cr), two_prod(-bi, ci)));
          ri = dd_add(ri, dd_add(two_prod(br, ci), two_prod(bi, cr)));
        }
        hp_re = rr.hi + rr.lo;
        hp_im = ri.hi + ri.lo;
      } else {
        double sr = 0.0, si = 0.0;
        for (int64_t k = 0; k < Keff; ++k) {
          sr += ar_row[k] * br_col[k];
          if (cplx) {
            sr -= ai_row[k] * bi_col[k];
            si += ar_row[k] * bi_col[k] + ai_row[k] * br_col[k];
          }
        }
        double rr = ar * sr - ai * si;
        double ri = ar * si + ai * sr;
        if (!beta_zero) {
          double cr, ci;
          load_elem(dtype, order, C, c_off, ldc, m, n, &cr, &ci);
          rr += br * cr - bi * ci;
          ri += br * ci + bi * cr;
        }
        hp_re = rr;
        hp_im = ri;
      }
      out_re = hp_re;
      out_im = hp_im;
      if (ref_out) {
        if (cplx) {
          ref_out[2 * (m + n * M)] = hp_re;
          ref_out[2 * (m + n * M) + 1] = hp_im;
        } else {
          ref_out[m + n * M] = hp_re;
        }
      }
      /* C is written after every thread has read its own element only, so
       * the in-place update is race-free: element (m, n) is read and written
       * by one iteration. */
      store_elem(dtype, order, C, c_off, ldc, m, n, out_re, out_im);
    }
  }
  free(At_re);
  free(At_im);
  free(opB_re);
  free(opB_im);
  return 0;
}

/*
 * Input recipes of the reference tests, drawn from glibc rand_r:
 *   oracle_rand_r_u02: static_cast<float>(rand_r(&seed)) /
 *                      static_cast<float>(RAND_MAX / 2.0f)
 *                      (test/unit/hcblas_sgemm.cpp:222-243)
 *   oracle_rand_r_mod: rand_r(&seed) % mod  (test/unit/hcblas_dgemm.cpp:228-236)
 * The seed is updated in place so consecutive calls continue one stream.
 */
int rand_r(unsigned int *seedp);
void oracle_rand_r_u02(unsigned int *seed, int64_t n, float *out) {
  const float denom = (float)(2147483647 / 2.0f);
  for (int64_t i = 0; i < n; ++i) out[i] = (float)rand_r(seed) / denom;
}
void oracle_rand_r_mod(unsigned int *seed, int64_t n, int mod, double *out) {
  for (int64_t i = 0; i < n; ++i) out[i] = (double)(rand_r(seed) % mod);
}

/*
 * The hcBLAS test metric sgemmCompareL2fe (test/include/helper_functions.h:
 * 10-53): ||ref - data||_2 / ||ref||_2 over a flat array, evaluated here in
 * binary64.  Returns -1 when ||ref|| is ~0 (the reference returns false).
 */
double oracle_compare_l2fe(const double *ref, const double *data, int64_t len) {
  double err = 0.0, nrm = 0.0;
  for (int64_t i = 0; i < len; ++i) {
    double d = ref[i] - data[i];
    err += d * d;
    nrm += ref[i] * ref[i];
  }
  if (fabs(nrm) < 1e-7) return -1.0;
  return sqrt(err) / sqrt(nrm);
}
