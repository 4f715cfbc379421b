/*
 * dispatch.cpp -- path selection for a canonical column-major GEMM.
 *
 * Replaces the reference's hand-written size-bucket dispatchers
 * (e.g. lib/src/blas/sgemm/sgemm_array_kernels.cpp:3291-3490, thresholds such
 * as `M % 128 == 0 && ... && M <= 6700`) with:
 *   math mode (native / emulated) -> storage type -> alignment -> tile shape
 *   from the SM count and the problem's tile count.
 * Tensor-core paths fall back to the SIMT kernels when an operand is not
 * TMA-addressable (16-byte base and stride alignment).
 */
#include "dispatch.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../kernels/hcbk.h"

namespace hcblas_b200 {

namespace {

int64_t tiles_of(int64_t m, int64_t n, int64_t bm, int64_t bn) {
  return ((m + bm - 1) / bm) * ((n + bn - 1) / bn);
}

bool aligned16(const void *p, int64_t off, int esz) {
  return ((reinterpret_cast<uintptr_t>(p) + (uintptr_t)(off * esz)) & 15) == 0;
}

int simt(HcblasB200State *st, const hcbk_gemm_args *a, void *stream, const char **path) {
  if (a->dtype == HCBK_D && st->dgemm_dmma) {
    /* native FP64 on the DMMA path (mma.sync .f64) */
    *path = "dmma.d.128x128";
    int rc = timed_launch(st, stream, *path, [&] { return hcbk_dgemm_dmma(a, stream); });
    if (rc != HCBK_ERR_ARGS) return rc;
  }
  if (a->dtype == HCBK_Z && st->dgemm_dmma) {
    /* native complex FP64: four real DMMA products per fragment set */
    *path = "dmma.z.128x64";
    int rc = timed_launch(st, stream, *path, [&] { return hcbk_zgemm_zmma(a, stream); });
    if (rc != HCBK_ERR_ARGS) return rc;
  }
  const int sms = hcbk_sm_count();
  const int64_t big = (a->dtype == HCBK_C || a->dtype == HCBK_Z) ? 64 : 128;
  hcbk_simt_cfg cfg;
  cfg.variant = (tiles_of(a->m, a->n, big, big) * a->batch >= sms) ? 0 : 1;
  const bool zero_beta = a->beta_re == 0.0 && a->beta_im == 0.0;
  if (st->autotune) {
    /* beta == 0: the candidates write C, which the final launch rewrites;
     * otherwise they write a scratch matrix of C's shape */
    TuneTarget tt(a, stream);
    if (zero_beta || tt.usable())
      cfg.variant = tune_choice(st, stream, tune_key("simt", a), 2, [&](int i) {
        const hcbk_gemm_args *t = zero_beta ? a : tt.args();
        if (!t) return (int)HCBK_ERR_NOMEM;
        hcbk_simt_cfg c;
        c.variant = i;
        return hcbk_gemm_simt(t, c, stream);
      }, cfg.variant);
  }
  static const char *names[5][2] = {
      {"simt.s.128x128", "simt.s.64x64"}, {"simt.d.128x128", "simt.d.64x64"},
      {"simt.c.64x64", "simt.c.64x64"},   {"simt.z.64x64", "simt.z.64x64"},
      {"simt.h.128x128", "simt.h.64x64"}};
  *path = names[a->dtype][cfg.variant];
  return timed_launch(st, stream, *path, [&] { return hcbk_gemm_simt(a, cfg, stream); });
}

/* CTA pairs (256-row tiles) once the problem has enough of them to fill
 * every SM pair; tc_pair = 2 forces them, 0 disables them.  Auto mode is
 * used by the 256 x 256 pair tiles (HGEMM, CRT); the split-BF16 paths, whose
 * register accumulators cap them at 256 x 128 pair tiles, measured no
 * faster with pairs and take them only when forced. */
bool use_pair(const HcblasB200State *st, int64_t m, int64_t n, int64_t bn) {
  if (st->tc_pair == 0) return false;
  if (st->tc_pair == 2) return true;
  return tiles_of(m, n, 256, bn) >= hcbk_sm_count() / 2;
}

/* HGEMM on tcgen05 with operands read in place by TMA. */
int hgemm_tc(HcblasB200State *st, const hcbk_gemm_args *a, void *stream, const char **path) {
  if (a->batch != 1 || a->a_array) return HCBK_ERR_ARGS;
  if (!aligned16(a->a, a->a_off, 2) || !aligned16(a->b, a->b_off, 2) || (a->lda & 7) ||
      (a->ldb & 7))
    return HCBK_ERR_ALIGN;
  int *err = device_error_flag(st);
  if (!err) return HCBK_ERR_NOMEM;
  if (st->inject_timeout) { /* failure-detection test: one call, then disarmed */
    st->inject_timeout = 0;
    *path = "tc.h.128x128.inject_timeout";
    const int rc = timed_launch(st, stream, *path,
                                [&] { return hcbk_hgemm_tc_inject_timeout(a, err, stream); });
    /* a shape the injection does not accept fails the call (no fallback) */
    return rc == HCBK_ERR_ARGS || rc == HCBK_ERR_ALIGN ? HCBK_ERR_LAUNCH : rc;
  }
  int pair = use_pair(st, a->m, a->n, 256) ? 1 : 0;
  int bn = pair || tiles_of(a->m, a->n, 128, 256) >= hcbk_sm_count() ? 256 : 128;
  if (st->autotune && st->tc_pair == 1) {
    /* candidates: 128x128, 128x256, 256x256 over a CTA pair; with beta != 0
     * they write a scratch matrix of C's shape */
    static const int cbn[3] = {128, 256, 256}, cpair[3] = {0, 0, 1};
    TuneTarget tt(a, stream);
    const int c = tune_choice(st, stream, tune_key("hgemm_tc", a), 3, [&](int i) {
      const hcbk_gemm_args *t = tt.args();
      if (!t) return (int)HCBK_ERR_NOMEM;
      return hcbk_hgemm_tc(t, cbn[i], cpair[i], err, stream);
    }, pair ? 2 : bn == 256 ? 1 : 0);
    bn = cbn[c];
    pair = cpair[c];
  }
  *path = pair ? "tc.h.256x256.pair" : bn == 256 ? "tc.h.128x256" : "tc.h.128x128";
  return timed_launch(st, stream, *path,
                      [&] { return hcbk_hgemm_tc(a, bn, pair, err, stream); });
}

/* Split-BF16 SGEMM: split both operands into bf16 planes (K-major), then one
 * tensor-core GEMM over the 3 or 6 plane products. */
int sgemm_split(HcblasB200State *st, const hcbk_gemm_args *a, int terms, void *stream,
                const char **path) {
  if (a->batch != 1 || a->a_array) return HCBK_ERR_ARGS;
  const int nplanes = terms == 6 ? 3 : 2;
  const int64_t kp = (a->k + 7) & ~int64_t(7); /* 16-byte row pitch */
  const size_t a_plane = (size_t)a->m * kp * 2, b_plane = (size_t)a->n * kp * 2;
  const size_t a_bytes = (a_plane + 1023) & ~size_t(1023);
  const size_t b_bytes = (b_plane + 1023) & ~size_t(1023);
  char *ws = static_cast<char *>(ensure_workspace(st, nplanes * (a_bytes + b_bytes), stream));
  int *err = device_error_flag(st);
  if (!ws || !err) return HCBK_ERR_NOMEM;

  hcbk_pack_args pa;
  pa.src = static_cast<const float *>(a->a) + a->a_off;
  pa.ld = a->lda;
  pa.k_contig = a->op_a != HCBK_OP_N; /* op(A) = A^T: element (m, k) at A[k + m*lda] */
  pa.rows = a->m;
  pa.kdim = a->k;
  pa.nplanes = nplanes;
  pa.ld_dst = kp;
  for (int i = 0; i < 3; ++i) pa.planes[i] = i < nplanes ? ws + i * a_bytes : nullptr;
  hcbk_pack_args pb;
  pb.src = static_cast<const float *>(a->b) + a->b_off;
  pb.ld = a->ldb;
  pb.k_contig = a->op_b == HCBK_OP_N; /* op(B) = B: element (k, n) at B[k + n*ldb] */
  pb.rows = a->n;
  pb.kdim = a->k;
  pb.nplanes = nplanes;
  pb.ld_dst = kp;
  char *bws = ws + nplanes * a_bytes;
  for (int i = 0; i < 3; ++i) pb.planes[i] = i < nplanes ? bws + i * b_bytes : nullptr;

  /* both operands in one launch when both are K-contiguous */
  int rc = timed_launch(st, stream, "pack.split_bf16",
                        [&] { return hcbk_pack_split_bf16_pair(&pa, &pb, stream); },
                        pa.k_contig && pb.k_contig ? 1 : 2);
  if (rc) return rc;

  hcbk_split_gemm g;
  g.m = a->m;
  g.n = a->n;
  g.k = a->k;
  g.terms = terms;
  g.bn = 128;
  g.promote_kb = st->split_promote_kb;
  g.pair = st->tc_pair == 2 ? 1 : 0;
  for (int i = 0; i < 3; ++i) {
    g.a_planes[i] = pa.planes[i];
    g.b_planes[i] = pb.planes[i];
  }
  g.ld_a = kp;
  g.ld_b = kp;
  g.c = static_cast<float *>(a->c) + a->c_off;
  g.ldc = a->ldc;
  g.alpha = a->alpha_re;
  g.beta = a->beta_re;
  if (st->autotune && st->tc_pair == 1) {
    /* 128 x 128 tiles or 256 x 128 over a CTA pair: the same sums in the
     * same order, so the choice never changes a result (the promotion
     * interval, which does, stays the knob's) */
    TuneTarget tt(a, stream);
    g.pair = tune_choice(st, stream, tune_key(terms == 6 ? "split6" : "split3", a), 2, [&](int i) {
      const hcbk_gemm_args *t = tt.args();
      if (!t) return (int)HCBK_ERR_NOMEM;
      hcbk_split_gemm gi = g;
      gi.pair = i;
      gi.c = static_cast<float *>(t->c) + t->c_off;
      return hcbk_sgemm_split_tc(&gi, err, stream);
    }, 0);
  }
  static const char *names[2][2][2] = {
      {{"tc.split_bf16x3.128x128.p1", "tc.split_bf16x3.128x128.p4"},
       {"tc.split_bf16x3.256x128.pair.p1", "tc.split_bf16x3.256x128.pair.p4"}},
      {{"tc.split_bf16x6.128x128.p1", "tc.split_bf16x6.128x128.p4"},
       {"tc.split_bf16x6.256x128.pair.p1", "tc.split_bf16x6.256x128.pair.p4"}}};
  *path = names[terms == 6][g.pair][g.promote_kb == 4];
  return timed_launch(st, stream, *path, [&] { return hcbk_sgemm_split_tc(&g, err, stream); });
}

/* CGEMM 3M on the split-BF16 path: T1 = Ar Br, T2 = Ai Bi,
 * T3 = (Ar+Ai)(Br+Bi), each one split-BF16 tensor-core GEMM into an f32
 * workspace matrix, then C = alpha ((T1 - T2) + i (T3 - T1 - T2)) + beta C.
 * Three real products instead of four; conj-transposed operands carry
 * negated imaginary planes. */
int cgemm_split3m(HcblasB200State *st, const hcbk_gemm_args *a, int terms, void *stream,
                  const char **path) {
  if (a->batch != 1 || a->a_array) return HCBK_ERR_ARGS;
  const int nplanes = terms == 6 ? 3 : 2;
  const int64_t kp = (a->k + 7) & ~int64_t(7);
  auto up1k = [](size_t v) { return (v + 1023) & ~size_t(1023); };
  const size_t a_plane = up1k((size_t)a->m * kp * 2), b_plane = up1k((size_t)a->n * kp * 2);
  const size_t t_bytes = up1k((size_t)a->m * a->n * 4);
  const size_t total = 3 * nplanes * (a_plane + b_plane) + 3 * t_bytes;
  char *ws = static_cast<char *>(ensure_workspace(st, total, stream));
  int *err = device_error_flag(st);
  if (!ws || !err) return HCBK_ERR_NOMEM;
  char *pa_base = ws, *pb_base = ws + 3 * nplanes * a_plane;
  float *T = reinterpret_cast<float *>(pb_base + 3 * nplanes * b_plane);
  const int64_t t_elems = (int64_t)(t_bytes / 4);

  hcbk_cpack_args pa;
  std::memset(&pa, 0, sizeof(pa));
  pa.src = static_cast<const char *>(a->a) + 8 * a->a_off;
  pa.ld = a->lda;
  pa.k_contig = a->op_a != HCBK_OP_N;
  pa.conj = a->op_a == HCBK_OP_C;
  pa.rows = a->m;
  pa.kdim = a->k;
  pa.nplanes = nplanes;
  pa.ld_dst = kp;
  for (int part = 0; part < 3; ++part)
    for (int t = 0; t < nplanes; ++t) pa.planes[part][t] = pa_base + (part * nplanes + t) * a_plane;
  hcbk_cpack_args pb;
  std::memset(&pb, 0, sizeof(pb));
  pb.src = static_cast<const char *>(a->b) + 8 * a->b_off;
  pb.ld = a->ldb;
  pb.k_contig = a->op_b == HCBK_OP_N;
  pb.conj = a->op_b == HCBK_OP_C;
  pb.rows = a->n;
  pb.kdim = a->k;
  pb.nplanes = nplanes;
  pb.ld_dst = kp;
  for (int part = 0; part < 3; ++part)
    for (int t = 0; t < nplanes; ++t) pb.planes[part][t] = pb_base + (part * nplanes + t) * b_plane;
  int rc = timed_launch(st, stream, "pack.split_bf16_complex",
                        [&] { return hcbk_pack_split_bf16_complex(&pa, stream); });
  if (!rc)
    rc = timed_launch(st, stream, "pack.split_bf16_complex",
                      [&] { return hcbk_pack_split_bf16_complex(&pb, stream); });
  if (rc) return rc;

  static const char *names[2][2] = {{"tc.split_bf16x3.128x128.p1", "tc.split_bf16x3.128x128.p4"},
                                    {"tc.split_bf16x6.128x128.p1", "tc.split_bf16x6.128x128.p4"}};
  for (int part = 0; part < 3 && !rc; ++part) {
    hcbk_split_gemm g;
    std::memset(&g, 0, sizeof(g));
    g.m = a->m;
    g.n = a->n;
    g.k = a->k;
    g.terms = terms;
    g.bn = 128;
    g.promote_kb = st->split_promote_kb;
    g.pair = st->tc_pair == 2 ? 1 : 0;
    for (int t = 0; t < nplanes; ++t) {
      g.a_planes[t] = pa.planes[part][t];
      g.b_planes[t] = pb.planes[part][t];
    }
    g.ld_a = kp;
    g.ld_b = kp;
    g.c = T + part * t_elems;
    g.ldc = a->m;
    g.alpha = 1.0;
    g.beta = 0.0;
    rc = timed_launch(st, stream, names[terms == 6][g.promote_kb == 4],
                      [&] { return hcbk_sgemm_split_tc(&g, err, stream); });
  }
  if (rc) return rc;
  hcbk_c3m_combine_args cb;
  cb.t1 = T;
  cb.t2 = T + t_elems;
  cb.t3 = T + 2 * t_elems;
  cb.ldt = a->m;
  cb.m = a->m;
  cb.n = a->n;
  cb.c = static_cast<char *>(a->c) + 8 * a->c_off;
  cb.ldc = a->ldc;
  cb.alpha_re = (float)a->alpha_re;
  cb.alpha_im = (float)a->alpha_im;
  cb.beta_re = (float)a->beta_re;
  cb.beta_im = (float)a->beta_im;
  *path = terms == 6 ? "tc.csplit3m_bf16x6" : "tc.csplit3m_bf16x3";
  return timed_launch(st, stream, "split.c3m_combine", [&] { return hcbk_c3m_combine(&cb, stream); });
}

/* Ozaki-scheme DGEMM (Ozaki-I): per-row / per-column exponents, `s` slices
 * per operand.  INT8 slices: the slice products of each weight group summed
 * exactly in INT32 on the int8 tensor cores (K split so that every group sum
 * stays exact), then an FP64 element-wise weighting pass; 8-bit slices in
 * binary16: f16 tensor cores with per-slab FP64 promotion. */
int dgemm_ozaki(HcblasB200State *st, const hcbk_gemm_args *a_in, int s, bool f16, void *stream,
                const char **path) {
  if (a_in->batch != 1 || a_in->a_array) return HCBK_ERR_ARGS;
  if (s < 3 || s > (f16 ? 7 : 8)) return HCBK_ERR_ARGS;
  /* SGEMM on the INT8 path: the exponent and slicing passes read the FP32
   * operands directly (widened in registers, exact); the group combine rounds
   * the FP64 result once into the FP32 C */
  const bool f32 = a_in->dtype == HCBK_S;
  if (f32 && f16) return HCBK_ERR_ARGS;
  const hcbk_gemm_args *a = a_in;
  const int esz = f16 ? 2 : 1;
  const int64_t kp = (a->k + 15) & ~int64_t(15); /* 16-byte row pitch for either slice type */
  auto up1k = [](size_t v) { return (v + 1023) & ~size_t(1023); };
  const size_t a_pl = up1k((size_t)a->m * kp * esz), b_pl = up1k((size_t)a->n * kp * esz);
  const size_t ea_bytes = up1k(sizeof(int) * a->m), eb_bytes = up1k(sizeof(int) * a->n);
  /* int8 path: the s slice-group INT32 sums of C, column-major */
  const int64_t ldd = (a->m + 3) & ~int64_t(3);
  const size_t d_bytes = f16 ? 0 : up1k((size_t)s * ldd * a->n * sizeof(int32_t));
  const size_t total = ea_bytes + eb_bytes + s * (a_pl + b_pl) + d_bytes;
  char *ws = static_cast<char *>(ensure_workspace(st, total, stream));
  int *err = device_error_flag(st);
  if (!ws || !err) return HCBK_ERR_NOMEM;

  int *exp_a = reinterpret_cast<int *>(ws);
  int *exp_b = reinterpret_cast<int *>(ws + ea_bytes);
  char *pa_base = ws + ea_bytes + eb_bytes;
  char *pb_base = pa_base + s * a_pl;
  int32_t *dsum = reinterpret_cast<int32_t *>(pb_base + s * b_pl);

  hcbk_ozaki_prep pa{};
  pa.src = f32 ? nullptr : static_cast<const double *>(a->a) + a->a_off;
  pa.src_f32 = f32 ? static_cast<const float *>(a->a) + a->a_off : nullptr;
  pa.ld = a->lda;
  pa.k_contig = a->op_a != HCBK_OP_N;
  pa.rows = a->m;
  pa.kdim = a->k;
  pa.exps = exp_a;
  pa.slices = s;
  pa.planes = pa_base;
  pa.plane_stride = (int64_t)a_pl;
  pa.ld_dst = kp;
  pa.f16 = f16 ? 1 : 0;
  hcbk_ozaki_prep pb{};
  pb.src = f32 ? nullptr : static_cast<const double *>(a->b) + a->b_off;
  pb.src_f32 = f32 ? static_cast<const float *>(a->b) + a->b_off : nullptr;
  pb.ld = a->ldb;
  pb.k_contig = a->op_b == HCBK_OP_N;
  pb.rows = a->n;
  pb.kdim = a->k;
  pb.exps = exp_b;
  pb.slices = s;
  pb.planes = pb_base;
  pb.plane_stride = (int64_t)b_pl;
  pb.ld_dst = kp;
  pb.f16 = f16 ? 1 : 0;

  int rc = timed_launch(st, stream, "ozaki.exponents", [&] { return hcbk_ozaki_exponents(&pa, stream); }, pa.k_contig ? 1 : 2);
  if (!rc) rc = timed_launch(st, stream, "ozaki.exponents", [&] { return hcbk_ozaki_exponents(&pb, stream); }, pb.k_contig ? 1 : 2);
  if (!rc) rc = timed_launch(st, stream, "ozaki.slice", [&] { return hcbk_ozaki_slice(&pa, stream); });
  if (!rc) rc = timed_launch(st, stream, "ozaki.slice", [&] { return hcbk_ozaki_slice(&pb, stream); });
  if (rc) return rc;

  static const char *names[9] = {"", "", "", "tc.ozaki_i8_s3", "tc.ozaki_i8_s4", "tc.ozaki_i8_s5",
                                  "tc.ozaki_i8_s6", "tc.ozaki_i8_s7", "tc.ozaki_i8_s8"};
  static const char *names16[8] = {"", "", "", "tc.ozaki_f16_s3", "tc.ozaki_f16_s4",
                                    "tc.ozaki_f16_s5", "tc.ozaki_f16_s6", "tc.ozaki_f16_s7"};
  static const char *names32[9] = {"", "", "", "tc.sozaki_i8_s3", "tc.sozaki_i8_s4",
                                   "tc.sozaki_i8_s5", "tc.sozaki_i8_s6", "tc.sozaki_i8_s7",
                                   "tc.sozaki_i8_s8"};
  *path = f16 ? names16[s] : f32 ? names32[s] : names[s];
  if (!f16) {
    /* one launch of every slice group per K range (INT32 exactness bounds
     * the range), then the FP64 weighting, scaling and alpha / beta */
    const int64_t kmax = hcbk_ozaki_max_k(s);
    hcbk_ozaki_groups g;
    g.m = a->m;
    g.n = a->n;
    g.slices = s;
    g.a_planes = pa_base;
    g.b_planes = pb_base;
    g.ld_a = kp;
    g.ld_b = kp;
    g.a_plane_stride = (int64_t)a_pl;
    g.b_plane_stride = (int64_t)b_pl;
    g.d = dsum;
    g.ldd = ldd;
    g.d_plane = ldd * a->n;
    g.pair = st->tc_pair == 2 ||
             (st->tc_pair == 1 && tiles_of(a->m, a->n, 256, 256) * s >= hcbk_sm_count() / 2);
    if (st->autotune && st->tc_pair == 1) {
      /* the slice products land in workspace planes: re-running is harmless */
      g.k0 = 0;
      g.k = a->k < kmax ? a->k : kmax;
      g.pair = tune_choice(st, stream, tune_key(f32 ? "sozaki_groups" : "ozaki_groups", a), 2,
                           [&](int i) {
                             hcbk_ozaki_groups gi = g;
                             gi.pair = i;
                             return hcbk_ozaki_groups_tc(&gi, err, stream);
                           },
                           g.pair);
    }
    hcbk_ozaki_groups_combine_args cb;
    cb.m = a->m;
    cb.n = a->n;
    cb.slices = s;
    cb.d = dsum;
    cb.ldd = ldd;
    cb.d_plane = ldd * a->n;
    cb.exp_a = exp_a;
    cb.exp_b = exp_b;
    cb.c = f32 ? nullptr : static_cast<double *>(a->c) + a->c_off;
    cb.c_f32 = f32 ? static_cast<float *>(a->c) + a->c_off : nullptr;
    cb.ldc = a->ldc;
    cb.alpha = a->alpha_re;
    for (int64_t k0 = 0; k0 < a->k; k0 += kmax) {
      g.k0 = k0;
      g.k = (a->k - k0 < kmax) ? a->k - k0 : kmax;
      cb.beta = (k0 == 0) ? a->beta_re : 1.0;
      rc = timed_launch(st, stream, *path, [&] { return hcbk_ozaki_groups_tc(&g, err, stream); });
      if (!rc)
        rc = timed_launch(st, stream, "ozaki.groups_combine",
                          [&] { return hcbk_ozaki_groups_combine(&cb, stream); });
      if (rc) return rc;
    }
    return HCBK_OK;
  }
  const int64_t kmax = a->k; /* the f16 kernel promotes per K-slab and takes any K */
  hcbk_ozaki_gemm g;
  g.m = a->m;
  g.n = a->n;
  g.slices = s;
  g.a_planes = pa_base;
  g.b_planes = pb_base;
  g.ld_a = kp;
  g.ld_b = kp;
  g.a_plane_stride = (int64_t)a_pl;
  g.b_plane_stride = (int64_t)b_pl;
  g.exp_a = exp_a;
  g.exp_b = exp_b;
  g.c = static_cast<double *>(a->c) + a->c_off;
  g.ldc = a->ldc;
  g.alpha = a->alpha_re;
  for (int64_t k0 = 0; k0 < a->k; k0 += kmax) {
    g.k0 = k0;
    g.k = (a->k - k0 < kmax) ? a->k - k0 : kmax;
    g.beta = (k0 == 0) ? a->beta_re : 1.0;
    rc = timed_launch(st, stream, *path, [&] { return hcbk_ozaki16_gemm_tc(&g, err, stream); });
    if (rc) return rc;
  }
  return HCBK_OK;
}

/* CRT (Ozaki scheme II) DGEMM: exponents, residue planes of the scaled
 * integer operands, one modular tensor-core GEMM launch over every modulus,
 * CRT reconstruction (weighted residue sum mod M) with the alpha/beta
 * epilogue.  A strided batch runs as one pass of each kernel over `nb`
 * elements starting at element e0 (element e's planes after element e-1's;
 * its modulus-i GEMM is plane e * nmod + i of the modular GEMM). */
static int dgemm_crt_elements(HcblasB200State *st, const hcbk_gemm_args *a, int nmod, int shift,
                              bool norm, int64_t e0, int64_t nb, void *stream,
                              const char **path) {
  const int beta_bits = 53;
  const int *mods = hcbk_crt_moduli(nullptr);
  /* int8 residues on kind::i8 (INT32 sums exact over all of K) unless K is
   * too long for them or the knob asks for the binary16 path */
  const bool i8 = st->crt_i8 && a->k <= HCBK_CRT_I8_MAX_K;
  const int esz = i8 ? 1 : 2;
  const int64_t kp = (a->k + 15) & ~int64_t(15); /* 16-byte row pitch for both element sizes */
  auto up1k = [](size_t v) { return (v + 1023) & ~size_t(1023); };
  const size_t a_pl = up1k((size_t)a->m * kp * esz), b_pl = up1k((size_t)a->n * kp * esz);
  /* int8 residues of C: 16-byte columns for the tensor stores and the
   * combine's bulk copies */
  const int64_t ldt = (a->m + 15) & ~int64_t(15);
  const size_t t_pl = up1k((size_t)ldt * a->n);
  const size_t ea_bytes = up1k(sizeof(int) * a->m * nb), eb_bytes = up1k(sizeof(int) * a->n * nb);
  const bool a_k = a->op_a != HCBK_OP_N, b_k = a->op_b == HCBK_OP_N;
  /* per row: the fraction and its reciprocal */
  const size_t fa_bytes = norm ? up1k(2 * sizeof(double) * a->m * nb) : 0;
  const size_t fb_bytes = norm ? up1k(2 * sizeof(double) * a->n * nb) : 0;
  const size_t wa_bytes =
      norm ? up1k((size_t)hcbk_crt_row_exponents_workspace_batch(a->m, a->k, a_k, nb)) : 0;
  const size_t wb_bytes =
      norm ? up1k((size_t)hcbk_crt_row_exponents_workspace_batch(a->n, a->k, b_k, nb)) : 0;
  const size_t total = ea_bytes + eb_bytes + fa_bytes + fb_bytes + wa_bytes + wb_bytes +
                       (size_t)nb * nmod * (a_pl + b_pl + t_pl);
  char *ws = static_cast<char *>(ensure_workspace(st, total, stream));
  int *err = device_error_flag(st);
  if (!ws || !err) return HCBK_ERR_NOMEM;
  int *exp_a = reinterpret_cast<int *>(ws);
  int *exp_b = reinterpret_cast<int *>(ws + ea_bytes);
  double *frac_a = norm ? reinterpret_cast<double *>(ws + ea_bytes + eb_bytes) : nullptr;
  double *frac_b = norm ? reinterpret_cast<double *>(ws + ea_bytes + eb_bytes + fa_bytes) : nullptr;
  double *inv_a = norm ? frac_a + a->m * nb : nullptr;
  double *inv_b = norm ? frac_b + a->n * nb : nullptr;
  char *wa = ws + ea_bytes + eb_bytes + fa_bytes + fb_bytes, *wb = wa + wa_bytes;
  char *pa_base = wb + wb_bytes;
  char *pb_base = pa_base + nb * nmod * a_pl;
  char *t_base = pb_base + nb * nmod * b_pl;

  hcbk_ozaki_prep ea;
  std::memset(&ea, 0, sizeof(ea));
  ea.src = static_cast<const double *>(a->a) + a->a_off + e0 * a->stride_a;
  ea.ld = a->lda;
  ea.k_contig = a->op_a != HCBK_OP_N;
  ea.rows = a->m;
  ea.kdim = a->k;
  ea.exps = exp_a;
  ea.batch = nb;
  ea.src_bstride = a->stride_a;
  hcbk_ozaki_prep eb = ea;
  eb.src = static_cast<const double *>(a->b) + a->b_off + e0 * a->stride_b;
  eb.ld = a->ldb;
  eb.k_contig = a->op_b == HCBK_OP_N;
  eb.rows = a->n;
  eb.exps = exp_b;
  eb.src_bstride = a->stride_b;
  /* row exponents: the row maximum's; when the moduli are too few for the
   * worst case, exponent and 8-bit fraction from the row norm instead */
  auto exps = [&](const hcbk_ozaki_prep &p, double *frac, double *inv, char *w, size_t wbytes,
                  void *s) {
    return timed_launch(st, s, "ozaki.exponents", [&] {
      return norm ? hcbk_crt_row_scales(&p, 53 - shift, 0, frac, inv, w, (int64_t)wbytes, s)
                  : hcbk_ozaki_exponents(&p, s);
    }, p.k_contig ? 1 : 2);
  };

  hcbk_crt_prep ra{};
  ra.src = ea.src;
  ra.ld = ea.ld;
  ra.k_contig = ea.k_contig;
  ra.rows = a->m;
  ra.kdim = a->k;
  ra.exps = exp_a;
  ra.frac = frac_a;
  ra.beta_bits = beta_bits;
  ra.nmod = nmod;
  ra.planes = pa_base;
  ra.plane_stride = (int64_t)a_pl;
  ra.ld_dst = kp;
  ra.i8 = i8 ? 1 : 0;
  ra.batch = nb;
  ra.src_bstride = a->stride_a;
  ra.planes_bstride = (int64_t)(nmod * a_pl);
  hcbk_crt_prep rb = ra;
  rb.src = eb.src;
  rb.ld = eb.ld;
  rb.k_contig = eb.k_contig;
  rb.rows = a->n;
  rb.exps = exp_b;
  rb.frac = frac_b;
  rb.planes = pb_base;
  rb.plane_stride = (int64_t)b_pl;
  rb.src_bstride = a->stride_b;
  rb.planes_bstride = (int64_t)(nmod * b_pl);
  /* the two operands' passes are independent: op(B)'s go to the handle's
   * second stream, so that its memory-bound row-scale pass overlaps op(A)'s
   * and the residue passes fill each other's tails */
  void *aux = aux_fork(st, stream);
  void *sb = aux ? aux : stream;
  int rc = exps(ea, frac_a, inv_a, wa, wa_bytes, stream);
  int rcb = exps(eb, frac_b, inv_b, wb, wb_bytes, sb);
  if (!rc) rc = timed_launch(st, stream, "crt.residues", [&] { return hcbk_crt_residues(&ra, stream); });
  if (!rcb) rcb = timed_launch(st, sb, "crt.residues", [&] { return hcbk_crt_residues(&rb, sb); });
  if (aux) {
    const int rcj = aux_join(st, stream);
    if (!rcb) rcb = rcj;
  }
  if (!rc) rc = rcb;
  if (rc) return rc;

  /* every modulus of every element in one persistent launch: the tile walk
   * covers nb * nmod planes, so the tile-count thresholds count all of them */
  const int64_t planes = nmod * nb;
  /* 256-row CTA-pair and 256-column tiles only where the GEMM is larger than
   * the 128-row / 128-column tile (a batch of small GEMMs would otherwise pad
   * every plane's tile) */
  int pair = st->tc_pair == 2 ||
             (st->tc_pair == 1 && a->m > 128 && a->n > 128 &&
              tiles_of(a->m, a->n, 256, 256) * planes >= hcbk_sm_count() / 2);
  int bn = pair || (a->n > 128 && tiles_of(a->m, a->n, 128, 256) * planes >= hcbk_sm_count())
               ? 256 : 128;
  hcbk_crt_gemm g{};
  g.m = a->m;
  g.n = a->n;
  g.k = a->k;
  g.a_planes = pa_base;
  g.b_planes = pb_base;
  g.ld_a = kp;
  g.ld_b = kp;
  g.a_plane_stride = (int64_t)a_pl;
  g.b_plane_stride = (int64_t)b_pl;
  g.nmod = nmod;
  g.moduli = mods;
  g.t = reinterpret_cast<int8_t *>(t_base);
  g.ldt = ldt;
  g.t_plane_stride = (int64_t)t_pl;
  g.pair = pair;
  g.bn = bn;
  g.i8 = i8 ? 1 : 0;
  g.batch = nb;
  if (st->autotune && st->tc_pair == 1) {
    /* every candidate writes the same exact residues: tuning in place is safe */
    static const int cbn[3] = {128, 256, 256}, cpair[3] = {0, 0, 1};
    const int c = tune_choice(st, stream, tune_key("crt_modgemm", a), 3, [&](int i) {
      hcbk_crt_gemm gi = g;
      gi.bn = cbn[i];
      gi.pair = cpair[i];
      return hcbk_crt_gemm_tc(&gi, err, stream);
    }, pair ? 2 : bn == 256 ? 1 : 0);
    g.bn = cbn[c];
    g.pair = cpair[c];
  }
  rc = timed_launch(st, stream, "tc.crt_modgemm", [&] { return hcbk_crt_gemm_tc(&g, err, stream); });
  if (rc) return rc;

  hcbk_crt_combine_args cb{};
  cb.m = a->m;
  cb.n = a->n;
  cb.nmod = nmod;
  cb.res = reinterpret_cast<const int8_t *>(t_base);
  cb.res_plane = (int64_t)t_pl;
  cb.ldr = ldt;
  cb.exp_a = exp_a;
  cb.exp_b = exp_b;
  cb.inv_a = inv_a;
  cb.inv_b = inv_b;
  cb.shift = 2 * beta_bits;
  cb.c = static_cast<double *>(a->c) + a->c_off + e0 * a->stride_c;
  cb.ldc = a->ldc;
  cb.alpha = a->alpha_re;
  cb.beta = a->beta_re;
  cb.err = err;
  cb.batch = nb;
  cb.res_bstride = (int64_t)(nmod * t_pl);
  cb.c_bstride = a->stride_c;
  static const char *names[2][HCBK_CRT_MAX_MODULI + 1] = {
      {"", "", "", "", "", "", "", "", "tc.crt_m8", "tc.crt_m9", "tc.crt_m10", "tc.crt_m11",
       "tc.crt_m12", "tc.crt_m13", "tc.crt_m14", "tc.crt_m15", "tc.crt_m16", "tc.crt_m17",
       "tc.crt_m18", "tc.crt_m19", "tc.crt_m20"},
      {"", "", "", "", "", "", "", "", "tc.crt_m8.batched", "tc.crt_m9.batched",
       "tc.crt_m10.batched", "tc.crt_m11.batched", "tc.crt_m12.batched", "tc.crt_m13.batched",
       "tc.crt_m14.batched", "tc.crt_m15.batched", "tc.crt_m16.batched", "tc.crt_m17.batched",
       "tc.crt_m18.batched", "tc.crt_m19.batched", "tc.crt_m20.batched"}};
  *path = names[a->batch > 1 ? 1 : 0][nmod];
  return timed_launch(st, stream, "crt.combine", [&] { return hcbk_crt_combine(&cb, stream); });
}

/* Workspace bytes per element of a CRT DGEMM (planes, exponents, scales and
 * partial sums), to size the element chunks of a batch. */
static size_t crt_bytes_per_element(const hcbk_gemm_args *a, int nmod, bool norm, bool i8) {
  const int64_t kp = (a->k + 15) & ~int64_t(15);
  const int64_t ldt = (a->m + 15) & ~int64_t(15);
  const int esz = i8 ? 1 : 2;
  auto up1k = [](size_t v) { return (v + 1023) & ~size_t(1023); };
  size_t b = (size_t)nmod * (up1k((size_t)a->m * kp * esz) + up1k((size_t)a->n * kp * esz) +
                             up1k((size_t)ldt * a->n));
  b += sizeof(int) * (size_t)(a->m + a->n);
  if (norm) {
    b += 2 * sizeof(double) * (size_t)(a->m + a->n);
    b += (size_t)hcbk_crt_row_exponents_workspace(a->m, a->k, a->op_a != HCBK_OP_N) +
         (size_t)hcbk_crt_row_exponents_workspace(a->n, a->k, a->op_b == HCBK_OP_N);
  }
  return b;
}

int dgemm_crt(HcblasB200State *st, const hcbk_gemm_args *a, int want, void *stream,
              const char **path) {
  if (a->a_array || a->batch < 1) return HCBK_ERR_ARGS;
  int nmod = 0, shift = 0;
  bool norm = false;
  if (!crt_plan_rows(a->k, want, &nmod, &shift, &norm)) return HCBK_ERR_ARGS;
  if (a->batch == 1) return dgemm_crt_elements(st, a, nmod, shift, norm, 0, 1, stream, path);
  /* a strided batch: the full-width plan's row exponents take one operand
   * at a time (declined here: the caller runs element by element) */
  if (!norm) return HCBK_ERR_ARGS;
  /* elements per pass: the workspace of a pass stays within 2 GiB (or the
   * handle's limit) and the grids' batch dimension within 65535 */
  const bool i8 = st->crt_i8 && a->k <= HCBK_CRT_I8_MAX_K;
  const size_t per = crt_bytes_per_element(a, nmod, norm, i8) + 8192;
  size_t budget = (size_t)2 << 30;
  if (st->workspace_limit && st->workspace_limit < budget) budget = st->workspace_limit;
  int64_t chunk = (int64_t)(budget / per);
  if (chunk < 1) chunk = 1;
  if (chunk > 65535) chunk = 65535;
  for (int64_t e0 = 0; e0 < a->batch; e0 += chunk) {
    const int64_t nb = a->batch - e0 < chunk ? a->batch - e0 : chunk;
    const int rc = dgemm_crt_elements(st, a, nmod, shift, norm, e0, nb, stream, path);
    /* after the first pass, C of earlier elements is written: no fallback */
    if (rc) return e0 > 0 && (rc == HCBK_ERR_ARGS || rc == HCBK_ERR_ALIGN) ? HCBK_ERR_LAUNCH : rc;
  }
  return HCBK_OK;
}

/* ZGEMM on the CRT path: 3M in modular arithmetic (exact), so one complex
 * product costs three modular GEMMs per modulus.  Real and imaginary parts
 * of a row share the row's scale.  The plan is the real one over the 2K
 * reals of a complex row (crt_plan_rows(2K)): with full width every row is
 * scaled to its largest part; with fewer moduli each complex row's norm is
 * kept below 2^nb, which bounds |Re P'| and |Im P'| (both at most
 * sum_k |a'_k||b'_k| <= ||a'|| ||b'||). */
int zgemm_crt(HcblasB200State *st, const hcbk_gemm_args *a, int want, void *stream,
              const char **path) {
  if (a->batch != 1 || a->a_array) return HCBK_ERR_ARGS;
  int nmod = 0, shift = 0;
  bool norm = false;
  if (!crt_plan_rows(2 * a->k, want, &nmod, &shift, &norm)) return HCBK_ERR_ARGS;
  const int beta_bits = 53;
  const int *mods = hcbk_crt_moduli(nullptr);
  const bool i8 = st->crt_i8 && a->k <= HCBK_CRT_I8_MAX_K; /* as in dgemm_crt */
  const int esz = i8 ? 1 : 2;
  const int64_t kp = (a->k + 15) & ~int64_t(15); /* 16-byte row pitch for both element sizes */
  auto up1k = [](size_t v) { return (v + 1023) & ~size_t(1023); };
  const size_t a_pl = up1k((size_t)a->m * kp * esz), b_pl = up1k((size_t)a->n * kp * esz);
  /* int8 residues of C: 16-byte columns for the tensor stores and the
   * combine's bulk copies */
  const int64_t ldt = (a->m + 15) & ~int64_t(15);
  const size_t t_pl = up1k((size_t)ldt * a->n);
  /* the real view of an MN-contiguous operand has two real rows per row */
  const bool a_k = a->op_a != HCBK_OP_N, b_k = a->op_b == HCBK_OP_N;
  const size_t ea_bytes = up1k(sizeof(int) * a->m * 2), eb_bytes = up1k(sizeof(int) * a->n * 2);
  /* norm scaling: per complex row the fraction and its reciprocal, and the
   * row-norm pass's partials over the real view */
  const size_t fa_bytes = norm ? up1k(2 * sizeof(double) * a->m) : 0;
  const size_t fb_bytes = norm ? up1k(2 * sizeof(double) * a->n) : 0;
  const size_t wa_bytes =
      norm ? up1k((size_t)hcbk_crt_row_exponents_workspace(a_k ? a->m : 2 * a->m,
                                                           a_k ? 2 * a->k : a->k, a_k))
           : 0;
  const size_t wb_bytes =
      norm ? up1k((size_t)hcbk_crt_row_exponents_workspace(b_k ? a->n : 2 * a->n,
                                                           b_k ? 2 * a->k : a->k, b_k))
           : 0;
  const size_t total = ea_bytes + eb_bytes + fa_bytes + fb_bytes + wa_bytes + wb_bytes +
                       3 * (size_t)nmod * (a_pl + b_pl + t_pl);
  char *ws = static_cast<char *>(ensure_workspace(st, total, stream));
  int *err = device_error_flag(st);
  if (!ws || !err) return HCBK_ERR_NOMEM;
  int *exp_a = reinterpret_cast<int *>(ws);
  int *exp_b = reinterpret_cast<int *>(ws + ea_bytes);
  double *frac_a = norm ? reinterpret_cast<double *>(ws + ea_bytes + eb_bytes) : nullptr;
  double *frac_b = norm ? reinterpret_cast<double *>(ws + ea_bytes + eb_bytes + fa_bytes) : nullptr;
  double *inv_a = norm ? frac_a + a->m : nullptr;
  double *inv_b = norm ? frac_b + a->n : nullptr;
  char *wa = ws + ea_bytes + eb_bytes + fa_bytes + fb_bytes, *wb = wa + wa_bytes;
  ws = wb + wb_bytes; /* the planes follow */
  char *pa_base = ws;
  char *pb_base = pa_base + 3 * nmod * a_pl;
  char *t_base = pb_base + 3 * nmod * b_pl;
  const double *A = reinterpret_cast<const double *>(a->a) + 2 * a->a_off;
  const double *B = reinterpret_cast<const double *>(a->b) + 2 * a->b_off;

  /* exponents on the real views: K-contiguous rows hold 2K reals; an
   * MN-contiguous operand becomes 2 x rows real rows of K */
  hcbk_ozaki_prep ea;
  std::memset(&ea, 0, sizeof(ea));
  ea.src = A;
  ea.ld = 2 * a->lda;
  ea.k_contig = a_k;
  ea.rows = a_k ? a->m : 2 * a->m;
  ea.kdim = a_k ? 2 * a->k : a->k;
  ea.exps = exp_a;
  hcbk_ozaki_prep eb = ea;
  eb.src = B;
  eb.ld = 2 * a->ldb;
  eb.k_contig = b_k;
  eb.rows = b_k ? a->n : 2 * a->n;
  eb.kdim = b_k ? 2 * a->k : a->k;
  eb.exps = exp_b;
  auto exps = [&](const hcbk_ozaki_prep &p, double *frac, double *inv, char *w, size_t wbytes,
                  void *s) {
    return timed_launch(st, s, "ozaki.exponents", [&] {
      return norm ? hcbk_crt_row_scales(&p, 53 - shift, p.k_contig ? 0 : 1, frac, inv, w,
                                        (int64_t)wbytes, s)
                  : hcbk_ozaki_exponents(&p, s);
    }, p.k_contig ? 1 : 2);
  };

  hcbk_zcrt_prep ra;
  std::memset(&ra, 0, sizeof(ra));
  ra.src = static_cast<const char *>(a->a) + 16 * a->a_off;
  ra.ld = a->lda;
  ra.k_contig = a_k;
  ra.conj = a->op_a == HCBK_OP_C;
  ra.rows = a->m;
  ra.kdim = a->k;
  ra.exps = exp_a;
  ra.exp_pair = norm ? 0 : !a_k; /* norm scales are per complex row already */
  ra.frac = frac_a;
  ra.beta_bits = beta_bits;
  ra.nmod = nmod;
  ra.planes = pa_base;
  ra.plane_stride = (int64_t)a_pl;
  ra.ld_dst = kp;
  ra.i8 = i8 ? 1 : 0;
  hcbk_zcrt_prep rb = ra;
  rb.src = static_cast<const char *>(a->b) + 16 * a->b_off;
  rb.ld = a->ldb;
  rb.k_contig = b_k;
  rb.conj = a->op_b == HCBK_OP_C;
  rb.rows = a->n;
  rb.exps = exp_b;
  rb.exp_pair = norm ? 0 : !b_k;
  rb.frac = frac_b;
  rb.planes = pb_base;
  rb.plane_stride = (int64_t)b_pl;
  /* op(B)'s passes on the handle's second stream, as in dgemm_crt */
  void *aux = aux_fork(st, stream);
  void *sb = aux ? aux : stream;
  int rc = exps(ea, frac_a, inv_a, wa, wa_bytes, stream);
  int rcb = exps(eb, frac_b, inv_b, wb, wb_bytes, sb);
  if (!rc) rc = timed_launch(st, stream, "crt.zresidues", [&] { return hcbk_zcrt_residues(&ra, stream); });
  if (!rcb) rcb = timed_launch(st, sb, "crt.zresidues", [&] { return hcbk_zcrt_residues(&rb, sb); });
  if (aux) {
    const int rcj = aux_join(st, stream);
    if (!rcb) rcb = rcj;
  }
  if (!rc) rc = rcb;
  if (rc) return rc;

  const int pair = st->tc_pair == 2 ||
                   (st->tc_pair == 1 && tiles_of(a->m, a->n, 256, 256) * nmod >= hcbk_sm_count() / 2);
  const int bn = pair || tiles_of(a->m, a->n, 128, 256) * nmod >= hcbk_sm_count() ? 256 : 128;
  /* one launch per 3M product (all moduli in each) */
  for (int set = 0; set < 3 && !rc; ++set) {
    hcbk_crt_gemm g{};
    g.m = a->m;
    g.n = a->n;
    g.k = a->k;
    g.a_planes = pa_base + set * nmod * a_pl;
    g.b_planes = pb_base + set * nmod * b_pl;
    g.ld_a = kp;
    g.ld_b = kp;
    g.a_plane_stride = (int64_t)a_pl;
    g.b_plane_stride = (int64_t)b_pl;
    g.nmod = nmod;
    g.moduli = mods;
    g.t = reinterpret_cast<int8_t *>(t_base + set * nmod * t_pl);
    g.ldt = ldt;
    g.t_plane_stride = (int64_t)t_pl;
    g.pair = pair;
    g.bn = bn;
    g.i8 = i8 ? 1 : 0;
    rc = timed_launch(st, stream, "tc.crt_modgemm", [&] { return hcbk_crt_gemm_tc(&g, err, stream); });
  }
  if (rc) return rc;

  hcbk_zcrt_combine_args cb;
  cb.m = a->m;
  cb.n = a->n;
  cb.nmod = nmod;
  cb.res = reinterpret_cast<const int8_t *>(t_base);
  cb.res_plane = (int64_t)t_pl;
  cb.ldr = ldt;
  cb.exp_a = exp_a;
  cb.exp_b = exp_b;
  cb.exp_a_pair = norm ? 0 : !a_k;
  cb.exp_b_pair = norm ? 0 : !b_k;
  cb.inv_a = inv_a;
  cb.inv_b = inv_b;
  cb.shift = 2 * beta_bits;
  cb.c = static_cast<char *>(a->c) + 16 * a->c_off;
  cb.ldc = a->ldc;
  cb.alpha_re = a->alpha_re;
  cb.alpha_im = a->alpha_im;
  cb.beta_re = a->beta_re;
  cb.beta_im = a->beta_im;
  cb.err = err;
  static const char *names[HCBK_CRT_MAX_MODULI + 1] = {
      "", "", "", "", "", "", "", "", "tc.zcrt3m_m8", "tc.zcrt3m_m9", "tc.zcrt3m_m10",
      "tc.zcrt3m_m11", "tc.zcrt3m_m12", "tc.zcrt3m_m13", "tc.zcrt3m_m14", "tc.zcrt3m_m15",
      "tc.zcrt3m_m16", "tc.zcrt3m_m17", "tc.zcrt3m_m18", "tc.zcrt3m_m19", "tc.zcrt3m_m20"};
  *path = names[nmod];
  return timed_launch(st, stream, "crt.zcombine", [&] { return hcbk_zcrt_combine(&cb, stream); });
}

}  // namespace

/* CRT plan of the real (DGEMM) path.  Operands are scaled to integers of
 * up to 53 bits, x' = rint(x 2^(53 - e_r)) per row/column.  Two bounds keep
 * |P'| = |sum_k a'_k b'_k| below M / (2 * 2^0.01): K 2^106 when the moduli
 * are that wide (then e_r is the frexp exponent of the row maximum), else
 * ||a'||_2 ||b'||_2 <= (2^nb + sqrt(K) / 2)^2 with the row exponents raised
 * so that every row norm is below 2^nb (Cauchy-Schwarz): rows that are not
 * dominated by one entry then keep about log2(max |x| sqrt(K) / ||x||_2)
 * more bits than scaling for the worst case K 2^(2 beta) allows.
 * want = 0 picks the fewest moduli with the first bound (full binary64
 * width whatever the data); want = n uses n moduli. */
bool crt_plan_rows(int64_t k, int want, int *nmod, int *shift, bool *norm) {
  int count = 0;
  const int *mods = hcbk_crt_moduli(&count);
  const double lk = std::ceil(std::log2((double)(k > 1 ? k : 2)));
  /* rint of the rounded product x f: at most 3/4 of a unit per element */
  const double rnd_norm = 0.75 * std::sqrt((double)k);
  double cum = 0.0;
  for (int i = 0; i < count; ++i) {
    cum += std::log2((double)mods[i]);
    const int n = i + 1;
    const bool full = cum >= 2.0 * 53 + 1.0 + lk + 0.01;
    if ((want == 0 && full) || want == n || (want == 0 && n == count)) {
      *nmod = n;
      *norm = !full;
      *shift = 0;
      if (full) return true;
      int nb = (int)std::floor((cum - 1.02) / 2.0);
      while (nb > 0 && 2.0 * std::log2(std::ldexp(1.0, nb) + rnd_norm) + 0.01 >= cum - 1.0) --nb;
      if (nb < 8) return false;
      *shift = 53 - nb;
      return true;
    }
  }
  return false;
}


/* Strided-batched HGEMM as a special case of the grouped kernel: one table
 * entry per batch element.  Declined (HCBK_ERR_ALIGN) unless every element
 * is TMA-addressable, so that the batch never splits across paths. */
int hgemm_strided_grouped(HcblasB200State *st, const hcbk_gemm_args *a, void *stream,
                          const char **path) {
  if (a->a_array || a->batch < 2 || a->batch > 0x7fffffff || a->m > 0x7fffffff ||
      a->n > 0x7fffffff || a->k > 0x7fffffff || a->lda > 0x7fffffff || a->ldb > 0x7fffffff ||
      a->ldc > 0x7fffffff)
    return HCBK_ERR_ARGS;
  if ((a->lda & 7) || (a->ldb & 7) || (a->stride_a & 7) || (a->stride_b & 7) ||
      !aligned16(a->a, a->a_off, 2) || !aligned16(a->b, a->b_off, 2))
    return HCBK_ERR_ALIGN;
  const uint16_t *A = static_cast<const uint16_t *>(a->a) + a->a_off; /* f16 storage */
  const uint16_t *B = static_cast<const uint16_t *>(a->b) + a->b_off;
  uint16_t *C = static_cast<uint16_t *>(a->c) + a->c_off;
  /* the batch in a few words: a repeated call finds its table without
   * spelling out every element */
  int dev = 0;
  cudaGetDevice(&dev);
  const int64_t ck[] = {a->op_a, a->op_b, a->m, a->n, a->k, a->lda, a->ldb, a->ldc,
                        a->stride_a, a->stride_b, a->stride_c, a->batch,
                        (int64_t)reinterpret_cast<uintptr_t>(A),
                        (int64_t)reinterpret_cast<uintptr_t>(B),
                        (int64_t)reinterpret_cast<uintptr_t>(C), st->grouped_c_tma, dev};
  const std::vector<unsigned char> compact(reinterpret_cast<const unsigned char *>(ck),
                                           reinterpret_cast<const unsigned char *>(ck) + sizeof(ck));
  if (a->alpha_re != 0.0 && grouped_hgemm_compact_match(st, compact)) {
    const int rc = grouped_hgemm(st, stream, ColMajor, (int)a->batch, nullptr,
                                 (float)a->alpha_re, (float)a->beta_re, &compact);
    *path = st->last_path;
    return rc;
  }
  std::vector<hcblasGemmProblem> probs((size_t)a->batch);
  for (int64_t i = 0; i < a->batch; ++i) {
    hcblasGemmProblem &p = probs[(size_t)i];
    p.transa = a->op_a == HCBK_OP_N ? HCBLAS_OP_N : HCBLAS_OP_T;
    p.transb = a->op_b == HCBK_OP_N ? HCBLAS_OP_N : HCBLAS_OP_T;
    p.m = (int)a->m;
    p.n = (int)a->n;
    p.k = (int)a->k;
    p.A = A + i * a->stride_a;
    p.lda = (int)a->lda;
    p.B = B + i * a->stride_b;
    p.ldb = (int)a->ldb;
    p.C = C + i * a->stride_c;
    p.ldc = (int)a->ldc;
  }
  int rc = grouped_hgemm(st, stream, ColMajor, (int)a->batch, probs.data(), (float)a->alpha_re,
                         (float)a->beta_re, &compact);
  *path = st->last_path;
  return rc;
}

/* Pointer-array HGEMM batch on the grouped tensor-core kernel: a kernel
 * builds the problem table on the device (the template entry's tensor maps
 * with their global addresses replaced from the device-resident pointer
 * arrays), the grouped kernel walks every problem's tiles, and a CUDA-core
 * pass computes the entries whose A or B TMA cannot address (flagged by the
 * builder; that pass launches whether or not any is flagged, since the host
 * cannot see the flags without waiting). */
int hgemm_ptr_grouped(HcblasB200State *st, const hcbk_gemm_args *a, void *stream,
                      const char **path) {
  if (!a->a_array || a->batch < 1 || a->batch > (1 << 24) || a->m > 0x7fffffff ||
      a->n > 0x7fffffff || a->k > 0x7fffffff || a->op_a == HCBK_OP_C || a->op_b == HCBK_OP_C)
    return HCBK_ERR_ARGS;
  if ((a->lda & 7) || (a->ldb & 7)) return HCBK_ERR_ALIGN; /* TMA strides: 16 bytes */
  HcblasGroupedPlan &gp = st->grouped_ptr;
  const int count = (int)a->batch;
  const size_t ent_bytes = sizeof(hcbk_grouped_entry) * (size_t)count;
  const size_t ts_off = (ent_bytes + 255) & ~size_t(255);
  const size_t skip_off = (ts_off + sizeof(int32_t) * ((size_t)count + 1) + 255) & ~size_t(255);
  const size_t bytes = skip_off + sizeof(int32_t) * (size_t)count;
  if (!grouped_ensure_table(gp, bytes, stream)) return HCBK_ERR_NOMEM;
  char *tb = static_cast<char *>(gp.table);
  /* the template: this batch's shape and strides, with the table itself as
   * a stand-in base address (replaced for every entry on the device); kept
   * for the next call of the same shape */
  const int64_t tkey[] = {a->op_a, a->op_b, a->m, a->n, a->k, a->lda, a->ldb, a->ldc,
                          st->grouped_c_tma, (int64_t)reinterpret_cast<uintptr_t>(tb)};
  hcbk_grouped_entry tmpl;
  if (gp.key.size() == sizeof(tkey) + sizeof(tmpl) &&
      std::memcmp(gp.key.data(), tkey, sizeof(tkey)) == 0) {
    std::memcpy(&tmpl, gp.key.data() + sizeof(tkey), sizeof(tmpl));
  } else {
    gp.key.clear();
    const int rc = hcbk_grouped_encode(&tmpl, a->op_a, a->op_b, a->m, a->n, a->k, tb, a->lda,
                                       tb, a->ldb, tb, a->ldc);
    if (rc) return rc;
    if (!st->grouped_c_tma) tmpl.c_tma = 0; /* direct stores */
    gp.key.resize(sizeof(tkey) + sizeof(tmpl));
    std::memcpy(gp.key.data(), tkey, sizeof(tkey));
    std::memcpy(gp.key.data() + sizeof(tkey), &tmpl, sizeof(tmpl));
  }
  int rc = HCBK_OK;
  int *err = device_error_flag(st);
  if (!err) return HCBK_ERR_NOMEM;
  auto *table = reinterpret_cast<hcbk_grouped_entry *>(tb);
  auto *ts = reinterpret_cast<int32_t *>(tb + ts_off);
  auto *skip = reinterpret_cast<int32_t *>(tb + skip_off);
  rc = timed_launch(st, stream, "tc.h.grouped.table", [&] {
    return hcbk_grouped_ptr_table(&tmpl, table, ts, skip, a->a_array, a->b_array, a->c_array,
                                  a->a_off * 2, a->b_off * 2, a->c_off * 2, a->stride_a * 2,
                                  a->stride_b * 2, a->stride_c * 2, count, stream);
  });
  if (rc) return rc;
  hcbk_grouped_args g;
  g.table = table;
  g.tile_start = ts;
  g.count = count;
  g.total_tiles = hcbk_grouped_tiles(&tmpl) * count;
  g.alpha = (float)a->alpha_re;
  g.beta = (float)a->beta_re;
  g.device_maps = 1;
  g.tile_desc = nullptr; /* uniform problems: tiles found by arithmetic */
  g.uniform_tiles = hcbk_grouped_tiles(&tmpl);
  g.u_tiles_m = tmpl.tiles_m;
  g.u_k = tmpl.k;
  g.u_flags = hcbk_grouped_tile_flags(&tmpl) & (HCBK_GT_BN64 | HCBK_GT_AMN | HCBK_GT_BMN);
  g.ctas_per_sm = st->grouped_ctas;
  if ((int64_t)hcbk_grouped_tiles(&tmpl) * count > 0x7fffffff) return HCBK_ERR_ARGS;
  rc = timed_launch(st, stream, "tc.h.grouped.ptr",
                    [&] { return hcbk_hgemm_grouped_tc(&g, err, stream); });
  if (rc) return rc;
  /* the entries the table builder flagged, on the CUDA cores */
  hcbk_gemm_args f = *a;
  f.batch_select = skip;
  hcbk_simt_cfg cfg;
  cfg.variant = 1;
  rc = timed_launch(st, stream, "simt.h.flagged", [&] { return hcbk_gemm_simt(&f, cfg, stream); });
  if (rc) return rc;
  *path = "tc.h.grouped.ptr";
  return HCBK_OK;
}

/* split-BF16 SGEMM batch (strided or pointer-array) on the grouped
 * tensor-core path: one pack launch and one GEMM launch for the batch */
int sgemm_split_batched(HcblasB200State *st, const hcbk_gemm_args *a, int terms, void *stream,
                        const char **path) {
  if (a->batch < 2 || a->batch > 0x7fffffff || a->m > 0x7fffffff || a->n > 0x7fffffff ||
      a->k > 0x7fffffff || a->lda > 0x7fffffff || a->ldb > 0x7fffffff || a->ldc > 0x7fffffff)
    return HCBK_ERR_ARGS;
  std::vector<hcblasGemmProblem> probs((size_t)a->batch);
  const bool ptr = a->a_array != nullptr;
  const float *A = static_cast<const float *>(a->a) + a->a_off;
  const float *B = static_cast<const float *>(a->b) + a->b_off;
  float *C = static_cast<float *>(a->c) + a->c_off;
  for (int64_t i = 0; i < a->batch; ++i) {
    hcblasGemmProblem &p = probs[(size_t)i];
    p.transa = a->op_a == HCBK_OP_N ? HCBLAS_OP_N : HCBLAS_OP_T;
    p.transb = a->op_b == HCBK_OP_N ? HCBLAS_OP_N : HCBLAS_OP_T;
    p.m = (int)a->m;
    p.n = (int)a->n;
    p.k = (int)a->k;
    p.lda = (int)a->lda;
    p.ldb = (int)a->ldb;
    p.ldc = (int)a->ldc;
    if (ptr) { /* placeholders: the device arrays supply the pointers */
      p.A = p.B = p.C = reinterpret_cast<void *>(uintptr_t(256));
    } else {
      p.A = A + i * a->stride_a;
      p.B = B + i * a->stride_b;
      p.C = C + i * a->stride_c;
    }
  }
  PtrBatch pb;
  if (ptr) {
    pb.a = a->a_array;
    pb.b = a->b_array;
    pb.c = a->c_array;
    pb.a_off = a->a_off;
    pb.b_off = a->b_off;
    pb.c_off = a->c_off;
    pb.sa = a->stride_a;
    pb.sb = a->stride_b;
    pb.sc = a->stride_c;
  }
  const int rc = grouped_sgemm_split(st, stream, ColMajor, (int)a->batch, probs.data(),
                                     (float)a->alpha_re, (float)a->beta_re, terms,
                                     ptr ? &pb : nullptr);
  *path = st->last_path;
  return rc;
}

/* Does the handle's math mode give this dtype an emulated path? */
bool emulated_mode(const HcblasB200State *st, int dtype) {
  switch (st->math_mode) {
    case 1: return dtype == HCBK_S || dtype == HCBK_C;  /* split-BF16 */
    case 2: return dtype == HCBK_D || dtype == HCBK_S;  /* Ozaki-I int8 */
    case 3: return dtype == HCBK_D;                     /* Ozaki-I binary16 */
    case 4: return dtype == HCBK_D || dtype == HCBK_Z;  /* CRT */
    default: return false;
  }
}

int dispatch_gemm(HcblasB200State *st, const hcbk_gemm_args *a, void *stream, const char **path) {
  if (a->dtype == HCBK_S && st->math_mode == 1 /* HCBLAS_MATH_SPLIT_BF16 */ && a->batch > 1) {
    /* strided and pointer-array batches: the grouped split-BF16 kernel */
    const int terms = plan_emulation(1, st->math_param, st->accuracy_bits, HCBK_S, a->k, nullptr);
    int rc = sgemm_split_batched(st, a, terms, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] split-bf16 batch path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_H && a->a_array) {
    int rc = hgemm_ptr_grouped(st, a, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] pointer-array hgemm grouped path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_D && st->math_mode == 4 /* HCBLAS_MATH_OZAKI_CRT */ && a->batch > 1 &&
      !a->a_array) {
    /* strided CRT DGEMM batch: each pass of the CRT pipeline over a chunk of
     * elements (the norm-scaled plans; the full-width plan runs per element) */
    const int want = plan_emulation(4, st->math_param, st->accuracy_bits, HCBK_D, a->k, nullptr);
    int rc = dgemm_crt(st, a, want, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] batched crt path declined (%d)\n", rc);
  }
  if (a->batch > 1 && !a->a_array && emulated_mode(st, a->dtype)) {
    /* strided batch under an emulated math mode: one emulated call per
     * element, in order on the stream (they share the workspace) */
    for (int64_t i = 0; i < a->batch; ++i) {
      hcbk_gemm_args e = *a;
      e.batch = 1;
      e.a_off = a->a_off + i * a->stride_a;
      e.b_off = a->b_off + i * a->stride_b;
      e.c_off = a->c_off + i * a->stride_c;
      e.stride_a = e.stride_b = e.stride_c = 0;
      const int rc = dispatch_gemm(st, &e, stream, path);
      if (rc) return rc;
    }
    return HCBK_OK;
  }
  if (a->dtype == HCBK_H && a->batch > 1 && !a->a_array) {
    int rc = hgemm_strided_grouped(st, a, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] strided hgemm grouped path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_H && a->batch == 1 && !a->a_array) {
    int rc = hgemm_tc(st, a, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] hgemm tensor-core path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_S && st->math_mode == 1 /* HCBLAS_MATH_SPLIT_BF16 */ && a->batch == 1 &&
      !a->a_array) {
    const int terms = plan_emulation(1, st->math_param, st->accuracy_bits, HCBK_S, a->k, nullptr);
    int rc = sgemm_split(st, a, terms, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] split-bf16 path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_C && st->math_mode == 1 /* HCBLAS_MATH_SPLIT_BF16 */ && a->batch == 1 &&
      !a->a_array) {
    const int terms = plan_emulation(1, st->math_param, st->accuracy_bits, HCBK_C, a->k, nullptr);
    int rc = cgemm_split3m(st, a, terms, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] complex split-bf16 path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_S && st->math_mode == 2 /* HCBLAS_MATH_OZAKI_INT8 */ && a->batch == 1 &&
      !a->a_array) {
    /* 4 slices (28 bits) unless a count or an accuracy target is set */
    const int s = plan_emulation(2, st->math_param, st->accuracy_bits, HCBK_S, a->k, nullptr);
    int rc = dgemm_ozaki(st, a, s, false, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] sgemm ozaki path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_D && (st->math_mode == 2 || st->math_mode == 3) && a->batch == 1 &&
      !a->a_array) {
    /* 2: HCBLAS_MATH_OZAKI_INT8, 3: HCBLAS_MATH_OZAKI_F16 */
    const bool f16 = st->math_mode == 3;
    const int s = st->math_param > 0 || st->accuracy_bits != 0
                      ? plan_emulation(st->math_mode, st->math_param, st->accuracy_bits, HCBK_D,
                                       a->k, nullptr)
                      : (f16 ? 7 : st->ozaki_default_slices);
    int rc = dgemm_ozaki(st, a, s, f16, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] ozaki path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_D && st->math_mode == 4 /* HCBLAS_MATH_OZAKI_CRT */ && a->batch == 1 &&
      !a->a_array) {
    const int want = plan_emulation(4, st->math_param, st->accuracy_bits, HCBK_D, a->k, nullptr);
    int rc = dgemm_crt(st, a, want, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] crt path declined (%d)\n", rc);
  }
  if (a->dtype == HCBK_Z && st->math_mode == 4 /* HCBLAS_MATH_OZAKI_CRT */ && a->batch == 1 &&
      !a->a_array) {
    const int want = plan_emulation(4, st->math_param, st->accuracy_bits, HCBK_Z, a->k, nullptr);
    int rc = zgemm_crt(st, a, want, stream, path);
    if (rc != HCBK_ERR_ALIGN && rc != HCBK_ERR_ARGS) return rc;
    if (log_enabled()) std::fprintf(stderr, "[hcblas] complex crt path declined (%d)\n", rc);
  }
  return simt(st, a, stream, path);
}

}  // namespace hcblas_b200
