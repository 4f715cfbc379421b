/*
 * split_bf16.cuh -- the split of an f32 value into bf16 terms (Henry, Tang &
 * Heinecke, ARITH 2019), shared by the plane-packing kernels:
 *     hi  = rn_bf16(x)
 *     mid = rn_bf16(x - hi)            (exact subtraction in f32)
 *     lo  = rn_bf16(x - hi - mid)
 * A non-finite hi keeps the special value (NaN as the canonical 0x7FFF) and
 * zeroes the lower terms.
 *
 * split_terms_bits rounds to bf16 on the bit pattern with integer arithmetic
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

/* packed f32x2 arithmetic, each lane rounded to nearest even */
__device__ __forceinline__ uint64_t sp_pk2(float a, float b) {
  uint64_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ uint64_t sp_fma2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ uint64_t sp_add2(uint64_t a, uint64_t b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}

/* exponent field in [27, 236]: 2^-100 <= |x| < 2^110 */
__device__ __forceinline__ bool veltkamp_range(uint32_t u) {
  return ((u >> 23) & 0xFFu) - 27u <= 209u;
}

/* head of two values to 8 significant bits by Veltkamp's splitting with
 * sigma = 2^16 + 1 (Dekker, "A floating-point technique for extending the
 * available precision", 1971): g = sigma x, h = g + (x - g).  In
 * round-to-nearest-even f32 arithmetic and inside veltkamp_range (no
 * overflow of sigma x, no subnormal residuals) h is the round-to-nearest-
 * even bf16 value of x, ties included, and x - h is exact. */
__device__ __forceinline__ uint64_t veltkamp8(uint64_t x) {
  const uint64_t S = sp_pk2(65537.0f, 65537.0f), NZ = sp_pk2(-0.0f, -0.0f);
  const uint64_t M1 = sp_pk2(-1.0f, -1.0f);
  const uint64_t g = sp_fma2(x, S, NZ);
  return sp_add2(g, sp_fma2(g, M1, x));
}

/* the bf16 terms of two values as bf16x2 words (first value in the low
 * half).  Where both values lie in veltkamp_range the terms come from
 * Veltkamp splits on the packed f32x2 pipe (hi, the head of x; mid, the
 * head of x - hi; lo = x - hi - mid, exact and already a bf16 value) --
 * the same bits as split_terms_bits, in about half the instructions; zeros,
 * very small or very large values and non-finite ones take split_terms_bits. */
__device__ __forceinline__ void split_terms2(float x0, float x1, uint32_t (&w)[3]) {
  if (veltkamp_range(__float_as_uint(x0)) && veltkamp_range(__float_as_uint(x1))) {
    const uint64_t M1 = sp_pk2(-1.0f, -1.0f);
    const uint64_t x = sp_pk2(x0, x1);
    const uint64_t h = veltkamp8(x);
    const uint64_t r1 = sp_fma2(h, M1, x);
    const uint64_t m = veltkamp8(r1);
    const uint64_t l = sp_fma2(m, M1, r1);
    w[0] = __byte_perm(static_cast<uint32_t>(h), static_cast<uint32_t>(h >> 32), 0x7632);
    w[1] = __byte_perm(static_cast<uint32_t>(m), static_cast<uint32_t>(m >> 32), 0x7632);
    w[2] = __byte_perm(static_cast<uint32_t>(l), static_cast<uint32_t>(l >> 32), 0x7632);
    return;
  }
  uint32_t a[3], b[3];
  split_terms_bits(x0, a);
  split_terms_bits(x1, b);
#pragma unroll
  for (int i = 0; i < 3; ++i) w[i] = __byte_perm(a[i], b[i], 0x7632);
}

#endif /* HCBLAS_B200_SPLIT_BF16_CUH_ */
