/*
 * hcbk.h -- the thin C-ABI shim between the C++ host library (handle,
 * argument checks, dispatch, autotuner) and the sm_100a CUDA kernels.
 *
 * Everything crossing this boundary is plain C: POD structs, raw device
 * pointers, int64 sizes and a cudaStream_t passed as void*.  The host side is
 * compiled by g++, the kernel side by nvcc; neither includes the other's
 * headers.  All problems arrive here already in column-major canonical form
 * (the host rewrites row-major C = op(A) op(B) as column-major
 * C^T = op(B)^T op(A)^T), so every kernel implements column-major only.
 */
#ifndef HCBLAS_B200_HCBK_H_
#define HCBLAS_B200_HCBK_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* storage types */
enum hcbk_dtype { HCBK_S = 0, HCBK_D = 1, HCBK_C = 2, HCBK_Z = 3, HCBK_H = 4 };
/* operand transforms: op(X) = X, X^T, X^H */
enum hcbk_op { HCBK_OP_N = 0, HCBK_OP_T = 1, HCBK_OP_C = 2 };

/* return codes of every hcbk_* launcher */
enum hcbk_status {
  HCBK_OK = 0,
  HCBK_ERR_ARGS = 1,      /* unsupported argument combination */
  HCBK_ERR_LAUNCH = 2,    /* cudaGetLastError() reported a failure */
  HCBK_ERR_ALIGN = 3,     /* operands not aligned for the requested path */
  HCBK_ERR_NOMEM = 4,     /* workspace too small */
  HCBK_ERR_DRIVER = 5     /* driver entry point (tensor maps) unavailable */
};

/*
 * One GEMM problem (or a batch of identically-shaped ones), column-major:
 *   C_b := alpha * op(A_b) * op(B_b) + beta * C_b,   b = 0 .. batch-1
 * with
 *   X_b = (x_array ? x_array[b] : x) + x_off + b * stride_x   (elements).
 * op(A) is m x k, op(B) is k x n, C is m x n.  alpha/beta are given in
 * binary64 {re, im}; the kernels cast them to the compute type.
 */
typedef struct hcbk_gemm_args {
  int dtype;
  int op_a, op_b;
  int64_t m, n, k;
  const void *a;
  int64_t lda, stride_a, a_off;
  const void *b;
  int64_t ldb, stride_b, b_off;
  void *c;
  int64_t ldc, stride_c, c_off;
  const void *const *a_array; /* device-resident pointer arrays or NULL */
  const void *const *b_array;
  void *const *c_array;
  int64_t batch;
  /* device flags or NULL: batch entry i is computed only where
   * batch_select[i] != 0 (the CUDA-core pass of a batch whose tensor-core
   * pass skipped entries it could not address) */
  const int32_t *batch_select;
  double alpha_re, alpha_im;
  double beta_re, beta_im;
} hcbk_gemm_args;

/* SIMT tile-shape choice (index into the per-dtype config table). */
typedef struct hcbk_simt_cfg {
  int variant; /* 0 = large tile, 1 = small tile */
} hcbk_simt_cfg;

/* Plain paths on CUDA cores: FP32 / FP64 / complex FMA, FP16 with FP32
 * accumulation.  Any op, ld, offset, alignment, batch. */
int hcbk_gemm_simt(const hcbk_gemm_args *args, hcbk_simt_cfg cfg, void *stream);

/* Native FP64 GEMM on the FP64 tensor path (mma.sync .f64 m16n8k4, 128 x 128
 * CTA tiles).  Any ld, offset, alignment, batch (strided or pointer arrays,
 * batch_select honoured); HCBK_ERR_ARGS for other dtypes. */
int hcbk_dgemm_dmma(const hcbk_gemm_args *args, void *stream);

/* Native complex FP64 GEMM on the same path: Re += Ar Br - Ai Bi,
 * Im += Ar Bi + Ai Br as four real DMMA products (128 x 64 CTA tiles); any
 * op (N, T, C), ld, offset, alignment, batch; HCBK_ERR_ARGS for other dtypes. */
int hcbk_zgemm_zmma(const hcbk_gemm_args *args, void *stream);

/* C := beta * C (beta == 0 writes zeros without reading C): the alpha == 0
 * path.  Any dtype, ld, offset, batch. */
int hcbk_scale_c(const hcbk_gemm_args *args, void *stream);

/* Number of SMs of the current device (cached per device). */
int hcbk_sm_count(void);

/* Issue-rate probe of one arithmetic pipe (peak.cu): kind 0 = FP32 FMA
 * (f32x2), 1 = FP64 FMA, 2 = FP64 mma.sync m16n8k4; iters per chain, 0 for
 * the default.  Writes TFLOP/s. */
int hcbk_peak_probe(int kind, int iters, double *tflops);

/* ------------------------------------------------ tensor-core paths -- */

/* HGEMM on tcgen05: f16 operands read by TMA directly from the caller's
 * matrices (any N/T combination), f32 accumulation in TMEM, f16 C.
 * Requirements (else HCBK_ERR_ALIGN / HCBK_ERR_ARGS and the caller falls
 * back to hcbk_gemm_simt): batch == 1, base pointers (after offsets) 16-byte
 * aligned, lda/ldb multiples of 8 elements.  `bn` = 128 or 256.
 * `pair` = 1 runs CTA pairs (tcgen05 cta_group::2, 256 x bn tiles, bn = 256
 * only), 0 single CTAs (128 x bn tiles).
 * `err` is a device int that receives a nonzero code if a pipeline wait
 * times out (the kernel then exits instead of hanging). */
int hcbk_hgemm_tc(const hcbk_gemm_args *args, int bn, int pair, int *err, void *stream);
/* Failure-detection test of the bounded pipeline waits: the HGEMM kernel on
 * one 128 x 128 tile of one K block (beta == 0) whose producer arms the
 * stage barrier without issuing its load, so that the MMA warp's wait runs
 * out after the wait limit in err[2..3]; nothing asynchronous is in flight
 * when the kernel unwinds.  HCBK_ERR_ARGS for any other shape. */
int hcbk_hgemm_tc_inject_timeout(const hcbk_gemm_args *args, int *err, void *stream);

/* Split-BF16 SGEMM: operands already split into bf16 planes, K-major:
 * a_planes[t] is M rows x ld_a elements (row m holds op(A)(m, 0..K-1)),
 * b_planes[t] is N rows x ld_b elements (row n holds op(B)(0..K-1, n)).
 * terms = 3 (planes hi, lo) or 6 (planes hi, mid, lo). */
typedef struct hcbk_split_gemm {
  int64_t m, n, k;
  int terms;
  int bn;         /* 128 */
  int promote_kb; /* K-slabs (64 elements) per TMEM chunk: 1 or 4 */
  int pair;       /* 1: CTA pairs, 256 x bn tiles */
  const void *a_planes[3];
  const void *b_planes[3];
  int64_t ld_a, ld_b;
  float *c;
  int64_t ldc;
  double alpha, beta;
} hcbk_split_gemm;
int hcbk_sgemm_split_tc(const hcbk_split_gemm *g, int *err, void *stream);

/* Split an f32 operand into bf16 planes in K-major layout.
 *   src element (r, k) = src[k + r*ld] if k_contig else src[r + k*ld]
 *   planes[t][r*ld_dst + k], t < nplanes (2: hi/lo, 3: hi/mid/lo)
 * r < rows, k < kdim. */
typedef struct hcbk_pack_args {
  const float *src;
  int64_t ld;
  int k_contig;
  int64_t rows, kdim;
  void *planes[3];
  int nplanes;
  int64_t ld_dst;
} hcbk_pack_args;
int hcbk_pack_split_bf16(const hcbk_pack_args *a, void *stream);
/* both operands of a split-BF16 GEMM: one launch when both are K-contiguous,
 * else one per operand */
int hcbk_pack_split_bf16_pair(const hcbk_pack_args *a, const hcbk_pack_args *b, void *stream);

/* CGEMM 3M on the split-BF16 path: split one complex f32 operand (float2
 * storage, `ld` in complex elements; element (r, k) at src[k + r*ld] if
 * k_contig else src[r + k*ld]) into bf16 planes of three parts -- real,
 * imaginary (negated when conj), and their f32 sum -- planes[part][t] at
 * [r*ld_dst + k]. */
typedef struct hcbk_cpack_args {
  const void *src;
  int64_t ld;
  int k_contig;
  int conj;
  int64_t rows, kdim;
  void *planes[3][3];
  int nplanes;
  int64_t ld_dst;
} hcbk_cpack_args;
int hcbk_pack_split_bf16_complex(const hcbk_cpack_args *a, void *stream);

/* C := alpha * ((T1 - T2) + i (T3 - T1 - T2)) + beta * C for f32 partial
 * products T1 = Ar Br, T2 = Ai Bi, T3 = (Ar+Ai)(Br+Bi) (m x n, leading
 * dimension ldt) and a float2 C. */
typedef struct hcbk_c3m_combine_args {
  const float *t1, *t2, *t3;
  int64_t ldt;
  int64_t m, n;
  void *c;
  int64_t ldc;
  float alpha_re, alpha_im, beta_re, beta_im;
} hcbk_c3m_combine_args;
int hcbk_c3m_combine(const hcbk_c3m_combine_args *a, void *stream);

/* ------------------------------------------------------- Ozaki DGEMM -- */

/* exponent markers of the Ozaki scaling */
#define HCBK_OZ_ZERO (-2000000)     /* all-zero row / column */
#define HCBK_OZ_NONFINITE 2000000   /* row / column holds Inf or NaN */

/* One operand of the Ozaki scheme, viewed as `rows` x `kdim`:
 *   element (r, k) = src[k + r*ld] if k_contig else src[r + k*ld].
 * hcbk_ozaki_exponents writes exps[r] (frexp exponent of max_k |x(r,k)|);
 * hcbk_ozaki_slice then writes `slices` int8 planes, plane i at
 * planes + i*plane_stride, element (r, k) at [r*ld_dst + k]. */
typedef struct hcbk_ozaki_prep {
  const double *src;
  int64_t ld;
  int k_contig;
  int64_t rows, kdim;
  int *exps;
  int slices;
  void *planes;
  int64_t plane_stride; /* bytes between planes */
  int64_t ld_dst;       /* elements between rows */
  int f16;              /* 0: int8 slices of 7 bits; 1: binary16 slices of 8 bits */
  const float *src_f32; /* exponents and slices only: an FP32 source instead of src */
  /* hcbk_crt_row_scales only: a strided batch of operands (0 or 1: one);
   * element e's source at src + e * src_bstride, its exps / frac / inv at
   * + e * rows (the other functions take one operand) */
  int64_t batch, src_bstride;
} hcbk_ozaki_prep;
int hcbk_ozaki_exponents(const hcbk_ozaki_prep *a, void *stream);

/* CRT row scales: x(r,k) is to become rint(x f_r 2^(53 - e_r)), e_r in
 * a->exps and f_r in frac[r] (1/2 <= f <= 1, 8 significant bits; inv[r] =
 * RN(1 / f_r)), with |x| f 2^(53-e) < 2^53 and row norm
 * ||x(r,:)|| f 2^(53-e) <= 2^nb.  MN-contiguous operands need `work` of
 * hcbk_crt_row_exponents_workspace bytes (partial sums per K chunk).
 * pair_rows (MN-contiguous only, even rows): rows 2r and 2r+1 share one
 * scale (the real and imaginary rows of a complex operand's real view);
 * exps / frac / inv then hold rows / 2 entries. */
int64_t hcbk_crt_row_exponents_workspace(int64_t rows, int64_t kdim, int k_contig);
/* the same for a batch of `batch` operands of rows x kdim */
int64_t hcbk_crt_row_exponents_workspace_batch(int64_t rows, int64_t kdim, int k_contig,
                                               int64_t batch);
int hcbk_crt_row_scales(const hcbk_ozaki_prep *a, int nb, int pair_rows, double *frac,
                        double *inv, void *work, int64_t work_bytes, void *stream);
int hcbk_ozaki_slice(const hcbk_ozaki_prep *a, void *stream);

/* Slice-product GEMM operands over K range [k0, k0 + k): a_planes M rows,
 * b_planes N rows, K-major with row pitch ld and plane pitch plane_stride
 * (bytes); C column-major FP64:
 *   C := alpha * 2^(ea_m + eb_n) * sum_{i+j<s} w^(i+j+2) a_i . b_j + beta * C
 * (used by the f16 path, w = 2^-8). */
typedef struct hcbk_ozaki_gemm {
  int64_t m, n, k, k0;
  int slices;
  const void *a_planes;
  const void *b_planes;
  int64_t ld_a, ld_b;
  int64_t a_plane_stride, b_plane_stride;
  const int *exp_a;
  const int *exp_b;
  double *c;
  int64_t ldc;
  double alpha, beta;
} hcbk_ozaki_gemm;
/* INT8 Ozaki-I slice groups on the int8 tensor cores: for every group
 * d = 0 .. slices-1 one INT32 GEMM over the concatenated K of its slice pairs,
 *   D_d = sum_{i <= d} a_i . b_(d-i)   (K range [k0, k0 + k)),
 * exact while slices * k * 127^2 < 2^31 (k <= hcbk_ozaki_max_k, a multiple
 * of 128 unless it ends the operand); every group in one persistent launch,
 * largest first.  Slice planes int8, K-major, row pitch ld_a / ld_b bytes and
 * plane pitches multiples of 16; D_d column-major int32 at d + d*d_plane
 * with leading dimension ldd (ldd, d_plane multiples of 4 elements, d
 * 16-byte aligned).  Tiles 256 x 256 over CTA pairs (pair = 1) or 128 x 256. */
typedef struct hcbk_ozaki_groups {
  int64_t m, n, k, k0;
  int slices;
  const void *a_planes;
  const void *b_planes;
  int64_t ld_a, ld_b;
  int64_t a_plane_stride, b_plane_stride;
  int32_t *d;
  int64_t ldd, d_plane;
  int pair;
} hcbk_ozaki_groups;
int hcbk_ozaki_groups_tc(const hcbk_ozaki_groups *g, int *err, void *stream);
/* C := alpha * 2^(exp_a[m] + exp_b[n]) * sum_d 2^(-7(d+2)) D_d + beta * C,
 * the groups summed in binary64 smallest weight first (FP64 element-wise). */
typedef struct hcbk_ozaki_groups_combine_args {
  int64_t m, n;
  int slices;
  const int32_t *d;
  int64_t ldd, d_plane;
  const int *exp_a;
  const int *exp_b;
  double *c;
  float *c_f32; /* when set, C is FP32 (c unused): the FP64 result rounded once */
  int64_t ldc;
  double alpha, beta;
} hcbk_ozaki_groups_combine_args;

int hcbk_ozaki_groups_combine(const hcbk_ozaki_groups_combine_args *a, void *stream);
/* The product on the f16 tensor path: binary16 planes holding 8-bit
 * integer slices (ld_a / ld_b in elements), weights 2^(-8(i+j+2)); any K
 * (k0 must be 0), slices 3..7. */
int hcbk_ozaki16_gemm_tc(const hcbk_ozaki_gemm *g, int *err, void *stream);
/* largest K per launch for s slices (INT32 exactness), multiple of 128 */
int64_t hcbk_ozaki_max_k(int slices);

/* ----------------------------------------- CRT (Ozaki scheme II) DGEMM -- */

#define HCBK_CRT_MAX_MODULI 20

/* The library's moduli (pairwise coprime, odd, <= 255), largest first. */
const int *hcbk_crt_moduli(int *count);

/* Residues of the scaled integer operand: for row r (exponent exps[r], from
 * hcbk_ozaki_exponents) A'(r,k) = rint(x(r,k) * 2^(beta_bits - exps[r])) and
 * plane i holds the symmetric residue A' mod moduli[i] (|r| <= 127) as
 * binary16, or as int8 when i8 is set, at [r*ld_dst + k] (planes
 * plane_stride bytes apart). */
typedef struct hcbk_crt_prep {
  const double *src;
  int64_t ld;
  int k_contig;
  int64_t rows, kdim;
  const int *exps;
  const double *frac; /* optional row fractions f_r: x * f_r is what gets scaled */
  int beta_bits;
  int nmod;
  void *planes;
  int64_t plane_stride; /* bytes */
  int64_t ld_dst;       /* elements */
  int i8;               /* 1: int8 planes (hcbk_crt_gemm's i8 path), 0: binary16 */
  /* a strided batch of operands (batch 0 or 1: one): element e's source at
   * src + e * src_bstride, its exps / frac at + e * rows, its nmod planes at
   * planes + e * planes_bstride bytes */
  int64_t batch, src_bstride, planes_bstride;
} hcbk_crt_prep;
int hcbk_crt_residues(const hcbk_crt_prep *a, void *stream);

/* All moduli in one launch: plane i of T = A_res_i * B_res_i mod moduli[i]
 * on the tensor cores, written as symmetric int16 residues (column-major
 * M x N, leading dimension ldt, planes t_plane_stride elements apart).
 * Residue planes: M (resp. N) rows x ld_a (ld_b) elements, K contiguous,
 * planes a_plane_stride (b_plane_stride) bytes apart; f16 elements
 * (kind::f16, sums reduced mod p every 1024 K), or int8 when i8 is set
 * (kind::i8, INT32 sums exact over the whole K, which must then be at most
 * HCBK_CRT_I8_MAX_K). */
#define HCBK_CRT_I8_MAX_K 131072 /* 131072 * 127^2 < 2^31 */
typedef struct hcbk_crt_gemm {
  int64_t m, n, k;
  const void *a_planes;
  const void *b_planes;
  int64_t ld_a, ld_b;
  int64_t a_plane_stride, b_plane_stride; /* bytes, multiples of 16 */
  int nmod;
  const int *moduli; /* host array of nmod moduli */
  int8_t *t;                        /* residues of C, 16-byte aligned */
  int64_t ldt, t_plane_stride;      /* bytes, multiples of 16 */
  int bn;   /* tile columns: 128 or 256 */
  int pair; /* 1: CTA pairs, 256 x 256 tiles (bn = 256) */
  int i8;   /* 1: int8 residue planes on kind::i8 */
  int64_t batch; /* GEMMs in the launch (0 or 1: one); element e's modulus-i
                    planes are plane e * nmod + i of A, B and T */
} hcbk_crt_gemm;
int hcbk_crt_gemm_tc(const hcbk_crt_gemm *g, int *err, void *stream);

/* CRT reconstruction of P' from the int8 residue planes (|r| <= 127) and
 * the epilogue C = alpha * P' * 2^(exp_a[m] + exp_b[n] - shift) + beta * C.
 * Residues are read by 1-D bulk copies: res 16-byte aligned, ldr >= m and
 * res_plane multiples of 16. */
typedef struct hcbk_crt_combine_args {
  int64_t m, n;
  int nmod;
  const int8_t *res;
  int64_t res_plane; /* bytes between planes, multiple of 16 */
  int64_t ldr;       /* >= m, multiple of 16 */
  const int *exp_a;
  const int *exp_b;
  const double *inv_a, *inv_b; /* optional reciprocals of the row fractions
                                  (hcbk_crt_row_scales): the result is multiplied
                                  by inv_a[m] * inv_b[n] */
  int shift; /* 2 * beta_bits */
  double *c;
  int64_t ldc;
  double alpha, beta;
  int *err; /* device error flag: set when the pipeline's wait times out */
  /* a strided batch (batch 0 or 1: one): element e's residue planes at
   * res + e * res_bstride bytes, its exp_a / inv_a at + e * m, exp_b / inv_b
   * at + e * n, its C at c + e * c_bstride */
  int64_t batch, res_bstride, c_bstride;
} hcbk_crt_combine_args;
int hcbk_crt_combine(const hcbk_crt_combine_args *a, void *stream);

/* ZGEMM on the CRT path (3M in modular arithmetic).  Residues of one complex
 * operand (double2 storage, `ld` in complex elements; element (r, k) at
 * src[k + r*ld] if k_contig else src[r + k*ld]): three plane sets of nmod
 * planes -- real, imaginary (negated when conj), and their sum mod p --
 * plane (set, i) at planes + (set*nmod + i)*plane_stride.  Row exponents come
 * from hcbk_ozaki_exponents on the real view; exp_pair = 1 when that view
 * split each complex row into two real rows (exponent = their max). */
typedef struct hcbk_zcrt_prep {
  const void *src;
  int64_t ld;
  int k_contig;
  int conj;
  int64_t rows, kdim;
  const int *exps;
  int exp_pair;
  const double *frac; /* optional row fractions (exp_pair 0): z * f_r is what gets scaled */
  int beta_bits;
  int nmod;
  void *planes;
  int64_t plane_stride; /* bytes */
  int64_t ld_dst;       /* elements */
  int i8;               /* 1: int8 planes (hcbk_crt_gemm's i8 path), 0: binary16 */
} hcbk_zcrt_prep;
int hcbk_zcrt_residues(const hcbk_zcrt_prep *a, void *stream);

/* Complex combine: res holds 3 sets of nmod int8 planes (T1 = Ar Br,
 * T2 = Ai Bi, T3 = (Ar+Ai)(Br+Bi) mod p_i); writes
 * C = alpha * ((T1 - T2) + i (T3 - T1 - T2)) 2^(e_m + f_n - shift) + beta * C
 * into the double2 matrix c. */
typedef struct hcbk_zcrt_combine_args {
  int64_t m, n;
  int nmod;
  const int8_t *res;
  int64_t res_plane; /* bytes between planes, multiple of 16 */
  int64_t ldr;       /* >= m, multiple of 16 */
  const int *exp_a;
  const int *exp_b;
  int exp_a_pair, exp_b_pair;
  const double *inv_a, *inv_b; /* optional reciprocals of the row fractions */
  int shift;
  void *c;
  int64_t ldc;
  double alpha_re, alpha_im, beta_re, beta_im;
  int *err; /* device error flag: set when the pipeline's wait times out */
} hcbk_zcrt_combine_args;
int hcbk_zcrt_combine(const hcbk_zcrt_combine_args *a, void *stream);

/* ------------------------------------------------------ GEMV and GER -- */

/* y := alpha * op(A) x + beta * y for column-major A (m x n, lda),
 * op = A (trans = 0: x has n, y has m entries) or A^T (trans = 1: x has m,
 * y has n); positive increments; beta == 0 means y is not read.  Partial
 * sums of at most max_splits slices go to `workspace` (see
 * hcbk_gemv_workspace_elems, elements of the dtype). */
typedef struct hcbk_gemv_args {
  int dtype; /* HCBK_S or HCBK_D */
  int trans;
  int64_t m, n;
  const void *a;
  int64_t lda;
  const void *x;
  int64_t incx;
  void *y;
  int64_t incy;
  double alpha, beta;
  void *workspace;
  int max_splits;
} hcbk_gemv_args;
int hcbk_gemv(const hcbk_gemv_args *g, void *stream);
int64_t hcbk_gemv_workspace_elems(int64_t m, int64_t n, int trans, int max_splits);

/* A := alpha * x y^T + A, column-major m x n; x, y point at their logical
 * first elements (increments may be negative, not zero). */
typedef struct hcbk_ger_args {
  int dtype; /* HCBK_S or HCBK_D */
  int64_t m, n;
  double alpha;
  const void *x;
  int64_t incx;
  const void *y;
  int64_t incy;
  void *a;
  int64_t lda;
} hcbk_ger_args;
int hcbk_ger(const hcbk_ger_args *g, void *stream);

/* ----------------------------------------------- grouped (uneven) GEMM -- */

/* One problem of a grouped HGEMM, as the persistent kernel reads it from
 * device memory: TMA tensor maps of op(A) and op(B) (encoded on the host by
 * hcbk_grouped_encode), the C block and the problem shape.  128-byte maps,
 * 64-byte aligned entries. */
typedef struct alignas(128) hcbk_grouped_entry {
  unsigned char map_a[128];
  unsigned char map_b[128];
  unsigned char map_c[128]; /* f16 C {m, n}, box 32 x 32 (valid when c_tma) */
  void *c;
  int64_t ldc;
  int32_t m, n, k;
  int32_t a_mn, b_mn; /* operand is MN-major in memory */
  int32_t tiles_m;
  int32_t bn;    /* tile columns of this problem: 64 or 128 */
  int32_t c_tma; /* C is written (and read) by TMA through map_c */
  int32_t skip;  /* set by the device-side table builder: computed elsewhere */
} hcbk_grouped_entry;

/* 2-D tensor map (128 bytes at `map`, 64-byte aligned) over 16-bit data
 * (bf16 != 0: bf16, else f16): `inner` contiguous elements per line, `outer`
 * lines `ld` elements apart, box {box_inner, box_outer}, 128-byte swizzle,
 * zero fill out of bounds. */
int hcbk_encode_tma_2d(void *map, int bf16, const void *base, uint64_t inner, uint64_t outer,
                       uint64_t ld, uint32_t box_inner, uint32_t box_outer);

/* Fill one table entry for column-major f16 C(m x n) = op(A) op(B):
 * op_a/op_b HCBK_OP_N or HCBK_OP_T.  HCBK_ERR_ALIGN when a base address is
 * not 16-byte aligned or lda/ldb is not a multiple of 8 (TMA rules). */
int hcbk_grouped_encode(hcbk_grouped_entry *e, int op_a, int op_b, int64_t m, int64_t n,
                        int64_t k, const void *a, int64_t lda, const void *b, int64_t ldb,
                        void *c, int64_t ldc);

/* 2-D map over a column-major f16 C {rows, cols} with column pitch ld
 * elements, box {32, 32}, no swizzle (the grouped epilogue's tensor stores);
 * HCBK_ERR_ALIGN when TMA cannot address C. */
int hcbk_encode_out_2d(void *map, void *base, uint64_t rows, uint64_t cols, uint64_t ld);

/* tiles of an encoded problem: tiles_m * ceil(n / bn) */
int hcbk_grouped_tiles(const hcbk_grouped_entry *e);

/* Per-tile descriptors of the grouped kernels (host tables): four int32 per
 * tile {problem | flags << 24, tile row, tile column, k}; problem < 2^24. */
enum {
  HCBK_GT_BN64 = 1, /* 64-wide tiles */
  HCBK_GT_AMN = 2,  /* op(A) MN-major */
  HCBK_GT_BMN = 4,  /* op(B) MN-major */
  HCBK_GT_CTMA = 8, /* C through tensor stores */
  HCBK_GT_SKIP = 16 /* not computed by the grouped kernel */
};
int hcbk_grouped_tile_flags(const hcbk_grouped_entry *e);
/* the descriptors of every tile of problem `problem` (entry e) into desc */
void hcbk_grouped_fill_tiles(const hcbk_grouped_entry *e, int problem, int32_t *desc);

/* Device-side table of a uniform pointer-array batch: entry i is *tmpl with
 * the addresses of its maps replaced by a_arr[i] + a_off_bytes +
 * i * a_stride_bytes etc. (on the
 * GPU, by tensormap.replace), skip[i] = 1 where A or B is not 16-byte
 * aligned, tile_start[i] = i * tiles (count + 1 entries).  table must be
 * 128-byte aligned. */
int hcbk_grouped_ptr_table(const hcbk_grouped_entry *tmpl, hcbk_grouped_entry *table,
                           int32_t *tile_start, int32_t *skip, const void *const *a_arr,
                           const void *const *b_arr, void *const *c_arr, int64_t a_off_bytes,
                           int64_t b_off_bytes, int64_t c_off_bytes, int64_t a_stride_bytes,
                           int64_t b_stride_bytes, int64_t c_stride_bytes, int count,
                           void *stream);

/* Persistent grouped HGEMM: 128 x bn tiles (bn per problem) of every problem,
 * enumerated by tile_start[] (count + 1 ascending prefix sums of each
 * problem's tile count), C = alpha * op(A) op(B) + beta * C with f32
 * accumulation. */
typedef struct hcbk_grouped_args {
  const hcbk_grouped_entry *table; /* device */
  const int32_t *tile_start;        /* device, count + 1 entries */
  int32_t count;
  int32_t total_tiles;
  float alpha, beta;
  int32_t device_maps; /* the table's maps were patched on the device */
  const int32_t *tile_desc; /* device, 4 int32 per tile (host tables), or NULL with: */
  int32_t uniform_tiles;    /* > 0: every problem has this many tiles, of shape: */
  int32_t u_tiles_m, u_k, u_flags;
  int32_t ctas_per_sm; /* f16 kernel: 1 (6-stage ring) or 2 (3 stages each) */
} hcbk_grouped_args;
int hcbk_hgemm_grouped_tc(const hcbk_grouped_args *g, int *err, void *stream);

/* ---------------------------------------------- grouped SIMT GEMM -- */

/* One problem of the persistent grouped GEMM on the CUDA cores (any dtype):
 * column-major C(m x n) = alpha op(A) op(B) + beta C, op_a/op_b HCBK_OP_*,
 * pointers already offset, tiles_m = ceil(m / bm) of the dtype's tile. */
typedef struct hcbk_simt_entry {
  const void *a;
  const void *b;
  void *c;
  int64_t lda, ldb, ldc;
  int32_t m, n, k;
  int32_t op_a, op_b;
  int32_t tiles_m;
} hcbk_simt_entry;

typedef struct hcbk_simt_grouped_args {
  int dtype;
  const hcbk_simt_entry *table; /* device */
  const int32_t *tile_start;    /* device, count + 1 ascending prefix sums */
  int32_t count;
  int32_t total_tiles;
  double alpha_re, alpha_im, beta_re, beta_im;
} hcbk_simt_grouped_args;

/* the tile (bm x bn) the grouped kernel uses for a dtype */
int hcbk_simt_grouped_tile(int dtype, int *bm, int *bn);
int hcbk_gemm_simt_grouped(const hcbk_simt_grouped_args *g, void *stream);

/* ------------------------------------------ grouped split-BF16 SGEMM -- */

/* One operand of one grouped problem to split into bf16 planes:
 * element (r, k) of the f32 source at src[k + r*ld] if k_contig else
 * src[r + k*ld]; plane t at planes + t * plane_stride (elements), K-major
 * [r * ld_dst + k] with ld_dst a multiple of 16 (the padding k >= kdim is
 * written as zeros); the job's tiles are ceil(rows / 32) x ceil(kdim / 64). */
typedef struct hcbk_gpack_job {
  const float *src;
  int64_t ld;
  void *planes;
  int64_t plane_stride;
  int32_t k_contig;
  int32_t rows, kdim, ld_dst;
  int32_t tiles_r;
  int32_t pad_;
} hcbk_gpack_job;

/* Pointer-array batches on the grouped split-BF16 path: job 2i / 2i + 1 and
 * entry i take a_arr[i] + a_off + i * a_stride (f32 elements; B, C alike)
 * as their source / C pointers, on the device. */
int hcbk_grouped_split_patch(hcbk_gpack_job *jobs, hcbk_grouped_entry *table,
                             const void *const *a_arr, const void *const *b_arr,
                             void *const *c_arr, int64_t a_off, int64_t b_off, int64_t c_off,
                             int64_t a_stride, int64_t b_stride, int64_t c_stride, int count,
                             void *stream);

/* Split every job's operand in one launch: 32 x 64 tiles enumerated by
 * tile_start[] (count + 1 ascending prefix sums, device). */
int hcbk_grouped_pack(const hcbk_gpack_job *jobs, const int32_t *tile_start, int32_t count,
                      int32_t total_tiles, int nplanes, void *stream);

/* 3-D tensor map (128 bytes at `map`) over `planes` 16-bit K-major planes
 * {kdim, rows, plane}: row pitch ld elements, plane pitch pstride bytes;
 * box {64, box_rows, 1}, 128-byte swizzle, zero fill beyond kdim and rows. */
int hcbk_encode_tma_3d_planes(void *map, int bf16, const void *base, uint64_t kdim,
                              uint64_t rows, uint64_t planes, uint64_t ld, uint64_t pstride,
                              uint32_t box_rows);

/* Persistent grouped split-BF16 SGEMM over a table whose map_a / map_b are
 * 3-D plane maps (hcbk_encode_tma_3d_planes) of the split operands and whose
 * C is f32: C = alpha * op(A) op(B) + beta * C with the products of `terms`
 * (3 or 6) and the TMEM sums promoted into f32 registers every 64 K. */
int hcbk_sgemm_grouped_split_tc(const hcbk_grouped_args *g, int terms, int *err, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HCBLAS_B200_HCBK_H_ */
