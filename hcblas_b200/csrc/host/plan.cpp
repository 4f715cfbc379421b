/*
 * plan.cpp -- the emulated math modes' count (CRT moduli, Ozaki slices,
 * split-BF16 terms) chosen from a requested accuracy.
 *
 * Accuracy is stated in bits against one model for every mode: for an
 * output element c_ij = a_i . b_j (a_i a row of op(A), b_j a column of
 * op(B), length K), the root-mean-square error the scheme adds is at most
 *     2^-bits * ||a_i||_2 * ||b_j||_2 .
 * A length-K dot product accumulated in a binary floating-point format with
 * a `bits`-bit significand (unit roundoff u = 2^-bits) by FMA, with
 * independent rounding errors, has RMS error u/sqrt(3) * sqrt(sum of the
 * squared partial sums), about 0.41 u ||a|| ||b|| -- the same form -- so
 * "53 bits" asks for native FP64 accuracy and "24 bits" for native FP32.
 *
 * Per scheme (the "model bits" of a count):
 *   CRT (Ozaki scheme II), D and Z: with the moduli wide enough for rows
 *     scaled to their maximum (crt_plan_rows' full plan) the scaled integers
 *     are exact: no representation error (model bits = +inf).  Otherwise
 *     every row is scaled so that its norm is 2^nb (to an 8-bit fraction)
 *     and rounded to integers: per element an error of at most 1/2 unit, so
 *     sum_k da_k b'_k / (s_a s_b) has RMS ||b|| / (s_a sqrt(12)) and both
 *     operands together 0.41 * 2^-nb ||a|| ||b||: model bits = nb.  This
 *     does not depend on the data (the row-norm scaling absorbs it) nor on K.
 *     Z is planned over the 2K reals of a complex row.
 *   Ozaki-I, int8 slices of 7 bits (s slices) or binary16 slices of 8 bits:
 *     each row is scaled by its maximum's exponent e (2^e <= 2 max|a| <=
 *     2 ||a||).  Truncation of the operands below the s-th slice adds RMS
 *     2 / sqrt(3) 2^-bs ||a|| ||b|| per operand; the slice products that
 *     the triangular scheme drops (i + j = s + 2, s - 1 of them) add
 *     sqrt(K) / 3 * 4 * 2^-bs ||a|| ||b|| each.  Together
 *         model bits = b s - log2(1.33 sqrt(K (s - 1)) + 1.63),
 *     a worst case over the data (rows whose maximum is close to their norm
 *     and whose other entries fill the lower slices); rows of comparable
 *     entries do several bits better.
 *   split-BF16 (S, C): 3 products keep hi x hi, hi x lo and lo x hi of a
 *     two-term split (16 significant bits per operand): 15 bits; 6 products
 *     of a three-term split fall below FP32's own accumulation error: 24.
 * The planner returns the smallest count whose model bits reach the target,
 * else the largest count of the mode (its model bits then fall short).
 */
#include <cmath>
#include <limits>

#include "dispatch.h"

namespace hcblas_b200 {

namespace {

double ozaki_model_bits(int slice_bits, int s, int64_t k) {
  const double kk = (double)(k > 1 ? k : 1);
  const double drop = s > 1 ? 1.33 * std::sqrt(kk * (s - 1)) : 0.0;
  return slice_bits * s - std::log2(drop + 1.63);
}

/* native precision of a dtype's format, in bits */
int native_bits(int dtype) { return (dtype == HCBK_D || dtype == HCBK_Z) ? 53 : 24; }

}  // namespace

double emulation_model_bits(int mode, int dtype, int64_t k, int count) {
  switch (mode) {
    case 1: /* split-BF16 */
      return count == 6 ? 24.0 : 15.0;
    case 2: /* Ozaki-I int8 */
      return ozaki_model_bits(7, count, k);
    case 3: /* Ozaki-I binary16 slices */
      return ozaki_model_bits(8, count, k);
    case 4: { /* CRT */
      int nmod = 0, shift = 0;
      bool norm = false;
      const int64_t kr = dtype == HCBK_Z ? 2 * k : k;
      if (!crt_plan_rows(kr, count, &nmod, &shift, &norm)) return 0.0;
      return norm ? (double)(53 - shift) : std::numeric_limits<double>::infinity();
    }
    default:
      return 0.0;
  }
}

int plan_emulation(int mode, int param, int bits, int dtype, int64_t k, double *model_bits) {
  int lo = 0, hi = 0, legacy = 0;
  const int candidates_split[2] = {3, 6};
  switch (mode) {
    case 1:
      if (dtype != HCBK_S && dtype != HCBK_C) return 0;
      legacy = 3;
      break;
    case 2:
      if (dtype != HCBK_D && dtype != HCBK_S) return 0;
      lo = 3, hi = 8, legacy = dtype == HCBK_S ? 4 : 7;
      break;
    case 3:
      if (dtype != HCBK_D) return 0;
      lo = 3, hi = 7, legacy = 7;
      break;
    case 4: {
      if (dtype != HCBK_D && dtype != HCBK_Z) return 0;
      lo = 8, hi = HCBK_CRT_MAX_MODULI;
      /* the legacy default: the fewest moduli of the full plan */
      int nmod = 0, shift = 0;
      bool norm = false;
      if (!crt_plan_rows(dtype == HCBK_Z ? 2 * k : k, 0, &nmod, &shift, &norm)) return 0;
      legacy = nmod;
      break;
    }
    default:
      return 0;
  }
  int count = legacy;
  if (param > 0) {
    count = param;
  } else if (bits != 0) {
    const int want = bits < 0 ? native_bits(dtype) : bits;
    if (mode == 1) {
      count = 6;
      for (int c : candidates_split)
        if (emulation_model_bits(mode, dtype, k, c) >= want) {
          count = c;
          break;
        }
    } else {
      count = hi;
      for (int c = lo; c <= hi; ++c) {
        const double mb = emulation_model_bits(mode, dtype, k, c);
        if (mb >= want) {
          count = c;
          break;
        }
      }
      if (mode == 4 && count > legacy) count = legacy; /* the full plan is exact */
    }
  }
  if (model_bits) *model_bits = emulation_model_bits(mode, dtype, k, count);
  return count;
}

}  // namespace hcblas_b200

extern "C" hcblasStatus_t hcblasPlanEmulation(int mode, int param, int bits, int dtype,
                                              long long k, int *count, double *model_bits) {
  if (count == nullptr || k < 1 || dtype < 0 || dtype > 3 || bits < -1 || bits > 64)
    return HCBLAS_STATUS_INVALID_VALUE;
  /* public dtype numbering 0 = S, 1 = D, 2 = C, 3 = Z is the internal one */
  const int c = hcblas_b200::plan_emulation(mode, param, bits, dtype, (int64_t)k, model_bits);
  *count = c;
  return c > 0 ? HCBLAS_STATUS_SUCCESS : HCBLAS_STATUS_INVALID_VALUE;
}

extern "C" hcblasStatus_t hcblasSetAccuracyTarget(hcblasHandle_t handle, int bits) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (bits < -1 || bits > 64) return HCBLAS_STATUS_INVALID_VALUE;
  handle->impl->accuracy_bits = bits;
  return HCBLAS_STATUS_SUCCESS;
}

extern "C" hcblasStatus_t hcblasGetAccuracyTarget(hcblasHandle_t handle, int *bits) {
  if (handle == nullptr || !handle->initialized || !handle->impl)
    return HCBLAS_STATUS_NOT_INITIALIZED;
  if (bits) *bits = handle->impl->accuracy_bits;
  return HCBLAS_STATUS_SUCCESS;
}
