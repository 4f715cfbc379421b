/*
 * dispatch.cpp -- path selection for a canonical column-major GEMM.
 *
 * Replaces the reference's hand-written size-bucket dispatchers
 * (e.g. lib/src/blas/sgemm/sgemm_array_kernels.cpp:3291-3490, thresholds such
 * as `M % 128 == 0 && ... && M <= 6700`) with: math mode (native / emulated)
 * -> storage type -> alignment -> tile shape from the SM count and the
 * problem's tile count.
 */
#include "dispatch.h"

#include "../kernels/hcbk.h"

namespace hcblas_b200 {

int dispatch_gemm(HcblasB200State *st, const hcbk_gemm_args *a, void *stream, const char **path) {
  const int sms = hcbk_sm_count();
  /* large tiles when they fill the machine at least once; else small tiles */
  int64_t big_tile = (a->dtype == HCBK_C || a->dtype == HCBK_Z) ? 64 : 128;
  const int64_t tiles = ((a->m + big_tile - 1) / big_tile) * ((a->n + big_tile - 1) / big_tile) *
                        a->batch;
  hcbk_simt_cfg cfg;
  cfg.variant = (tiles >= sms) ? 0 : 1;
  static const char *names[5][2] = {
      {"simt.s.128x128", "simt.s.64x64"},   {"simt.d.128x128", "simt.d.64x64"},
      {"simt.c.64x64", "simt.c.64x64"},     {"simt.z.64x64", "simt.z.64x64"},
      {"simt.h.128x128", "simt.h.64x64"}};
  *path = names[a->dtype][cfg.variant];
  return timed_launch(st, stream, *path, [&] { return hcbk_gemm_simt(a, cfg, stream); });
}

}  // namespace hcblas_b200
