/*
 * dispatch.h -- internal interface between the API layer (gemm.cpp) and the
 * path selection (dispatch.cpp).  Internal header.
 */
#ifndef HCBLAS_B200_DISPATCH_H_
#define HCBLAS_B200_DISPATCH_H_

#include <stdint.h>

#include <functional>
#include <string>

#include "../../../include/hcblas.h"
#include "../../../include/hcblaslib.h"
#include "../kernels/hcbk.h"
#include "state.h"

namespace hcblas_b200 {

/* One GEMM call as the API layer sees it (before canonicalisation). */
struct GemmCall {
  int dtype;            /* HCBK_S .. HCBK_H */
  hcblasOrder order;
  int op_a, op_b;       /* HCBK_OP_* */
  int64_t m, n, k;
  double alpha_re, alpha_im, beta_re, beta_im;
  const void *a;
  int64_t lda, a_off, stride_a;
  const void *const *a_arr;
  const void *b;
  int64_t ldb, b_off, stride_b;
  const void *const *b_arr;
  void *c;
  int64_t ldc, c_off, stride_c;
  void *const *c_arr;
  int64_t batch;
};

int op_from_char(hcblasTranspose t);
hcblasTranspose char_from_op(hcblasOperation_t op);
hcblasStatus run_gemm(Hcblaslibrary *h, const hc::accelerator_view &view, GemmCall g);

/* Choose and launch the kernel path for a canonical (column-major, alpha != 0)
 * problem.  Returns an HCBK_* code; *path names the path taken. */
int dispatch_gemm(HcblasB200State *st, const hcbk_gemm_args *a, void *stream, const char **path);

/* Autotuner (tune.cpp): the size-bucket key of a call for a kernel family,
 * and the fastest of `ncand` candidates -- run(i) launches candidate i and
 * returns an HCBK_* code -- measured once per key while the handle's
 * "autotune" knob is on (else `fallback`). */
std::string tune_key(const char *family, const hcbk_gemm_args *a);
/* the same key for a family whose bucket is described by `shape` */
std::string tune_key_shape(const char *family, const char *shape);
int tune_choice(HcblasB200State *st, void *stream, const std::string &key, int ncand,
                const std::function<int(int)> &run, int fallback);

/* Output of the candidates while a call whose C must not be rewritten
 * (beta != 0) is tuned: the call's arguments with C moved to a scratch
 * matrix of the same shape, leading dimension and 256-byte phase, allocated
 * stream-ordered on first use (only when the bucket is actually tuned) and
 * released by the destructor.  For beta == 0 the candidates write C itself,
 * which the final launch overwrites.  Single problems only (batch 1, no
 * pointer arrays); args() is nullptr when the scratch cannot be had. */
class TuneTarget {
 public:
  TuneTarget(const hcbk_gemm_args *a, void *stream);
  ~TuneTarget();
  TuneTarget(const TuneTarget &) = delete;
  TuneTarget &operator=(const TuneTarget &) = delete;
  const hcbk_gemm_args *args();
  /* whether tuning is offered for this call at all */
  bool usable() const { return usable_; }

 private:
  hcbk_gemm_args t_;
  const hcbk_gemm_args *a_;
  void *stream_;
  void *scratch_ = nullptr;
  bool usable_ = false, failed_ = false;
};

/* CRT plan of a real row of length k (dispatch.cpp): the moduli count, the
 * shift below 53 bits of the norm-scaled integers and whether rows are
 * norm-scaled; want = 0 picks the fewest moduli that keep every row at its
 * full 53 bits, want = n uses n moduli.  false when n moduli are too few. */
bool crt_plan_rows(int64_t k, int want, int *nmod, int *shift, bool *norm);

/* The emulated modes' planner (plan.cpp): the count (terms, slices or
 * moduli) a call of `dtype` with inner dimension k uses under math mode
 * `mode` -- `param` when it is > 0, else the smallest count whose model
 * error reaches `bits` (-1: the format's native precision), else (bits == 0)
 * the mode's default; 0 when the mode does not apply to the dtype.
 * *model_bits (optional) receives the count's model accuracy in bits. */
int plan_emulation(int mode, int param, int bits, int dtype, int64_t k, double *model_bits);
double emulation_model_bits(int mode, int dtype, int64_t k, int count);

/* Grouped HGEMM over `count` problems (grouped.cpp): builds or reuses the
 * handle's device problem table and runs the persistent kernel.  `compact`
 * (optional) is a short key that determines every problem (a strided batch's
 * shape, strides and base addresses): when it matches the one the table was
 * built for, the table is reused without looking at `probs`, which may then
 * be null (alpha != 0 only). */
int grouped_hgemm(HcblasB200State *st, void *stream, hcblasOrder order, int count,
                  const hcblasGemmProblem *probs, float alpha, float beta,
                  const std::vector<unsigned char> *compact = nullptr);

/* whether `compact` is the short key of the handle's current grouped HGEMM
 * table (the caller may then pass no problems) */
bool grouped_hgemm_compact_match(HcblasB200State *st, const std::vector<unsigned char> &compact);

/* Grouped GEMM of S/D/C/Z problems on the CUDA cores (one persistent
 * launch); scalars as real and imaginary parts. */
int grouped_simt(HcblasB200State *st, void *stream, int dtype, hcblasOrder order, int count,
                 const hcblasGemmProblem *probs, double alpha_re, double alpha_im,
                 double beta_re, double beta_im);

/* Device-resident pointer arrays of a uniform batch: matrix i of X is
 * x[i] + x_off + i * x_stride (elements). */
struct PtrBatch {
  const void *const *a;
  const void *const *b;
  void *const *c;
  int64_t a_off, b_off, c_off;
  int64_t sa, sb, sc;
};

/* Grouped FP32 GEMM on the split-BF16 tensor-core path (terms 3 or 6).
 * With `ptrs`, the problems' A, B, C pointers are placeholders and the
 * operands come from the device-resident arrays (patched on the device). */
int grouped_sgemm_split(HcblasB200State *st, void *stream, hcblasOrder order, int count,
                        const hcblasGemmProblem *probs, float alpha, float beta, int terms,
                        const PtrBatch *ptrs = nullptr);

/* Shared helpers of the grouped paths (grouped.cpp): a plan's device table
 * of at least `bytes` (grown after the stream's queued work) */
bool grouped_ensure_table(HcblasGroupedPlan &gp, size_t bytes, void *stream);

}  // namespace hcblas_b200

#endif /* HCBLAS_B200_DISPATCH_H_ */
