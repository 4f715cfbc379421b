/*
 * split_bf16.cuh -- the split of an f32 value into bf16 terms (Henry, Tang &
 * Heinecke, ARITH 2019), shared by the plane-packing kernels and the fused
 * grouped kernel:
 *     hi  = rn_bf16(x)
 *     mid = rn_bf16(x - hi)            (exact subtraction in f32)
 *     lo  = rn_bf16(x - hi - mid)
 * A non-finite hi keeps the special value (NaN as the canonical 0x7FFF) and
 * zeroes the lower terms.
 *
 * The rounding to bf16 is done on the bit pattern with integer arithmetic
 * (round to nearest, ties to even: add 0x7FFF plus the lowest kept bit,
 * clear the low half), which is exactly the IEEE conversion for every
 * non-NaN f32 -- subnormals and the overflow to infinity included -- and
 * runs on the integer pipes instead of the conversion unit, whose 16
 * results per clock per SM would otherwise bound every split kernel.  The
 * terms come out as f32 bit patterns whose high halves are the bf16 values
 * and whose low halves are zero, i.e. as the f32 values they stand for.
 */
#ifndef HCBLAS_B200_SPLIT_BF16_CUH_
#define HCBLAS_B200_SPLIT_BF16_CUH_

#include <cuda_bf16.h>
#include <stdint.h>

/* bf16(x) rounded to nearest even, as the f32 bit pattern of its value
 * (x not NaN) */
__device__ __forceinline__ uint32_t rn_bf16_bits(uint32_t u) {
  return (u + 0x7FFFu + ((u >> 16) & 1u)) & 0xFFFF0000u;
}

/* the three terms of x as f32 bit patterns (bf16 in the high halves) */
__device__ __forceinline__ void split_terms_bits(float x, uint32_t (&t)[3]) {
  const uint32_t u = __float_as_uint(x);
  if ((u & 0x7FFFFFFFu) > 0x7F800000u) { /* NaN */
    t[0] = 0x7FFF0000u;
    t[1] = t[2] = 0u;
    return;
  }
  const uint32_t h = rn_bf16_bits(u);
  t[0] = h;
  if ((h & 0x7F800000u) == 0x7F800000u) { /* infinite (x or its rounding) */
    t[1] = t[2] = 0u;
    return;
  }
  const float r1 = x - __uint_as_float(h);
  const uint32_t m = rn_bf16_bits(__float_as_uint(r1));
  t[1] = m;
  t[2] = rn_bf16_bits(__float_as_uint(r1 - __uint_as_float(m)));
}

__device__ __forceinline__ void split_terms(float x, __nv_bfloat16 (&t)[3]) {
  uint32_t b[3];
  split_terms_bits(x, b);
#pragma unroll
  for (int i = 0; i < 3; ++i) t[i] = __ushort_as_bfloat16(static_cast<unsigned short>(b[i] >> 16));
}

/* the bf16 terms of two values as bf16x2 words (first value in the low half) */
__device__ __forceinline__ void split_terms2(float x0, float x1, uint32_t (&w)[3]) {
  uint32_t a[3], b[3];
  split_terms_bits(x0, a);
  split_terms_bits(x1, b);
#pragma unroll
  for (int i = 0; i < 3; ++i) w[i] = __byte_perm(a[i], b[i], 0x7632);
}

#endif /* HCBLAS_B200_SPLIT_BF16_CUH_ */
