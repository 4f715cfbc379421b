/*
 * split_bf16.cuh -- the split of an f32 value into bf16 terms (Henry, Tang &
 * Heinecke, ARITH 2019), shared by the plane-packing kernels:
 *     hi  = rn_bf16(x)
 *     mid = rn_bf16(x - hi)            (exact subtraction in f32)
 *     lo  = rn_bf16(x - hi - mid)
 * A non-finite hi keeps the special value and zeroes the lower terms.
 */
#ifndef HCBLAS_B200_SPLIT_BF16_CUH_
#define HCBLAS_B200_SPLIT_BF16_CUH_

#include <cuda_bf16.h>

__device__ __forceinline__ void split_terms(float x, __nv_bfloat16 (&t)[3]) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  const float hf = __bfloat162float(h);
  t[0] = h;
  if (!isfinite(hf)) {
    t[1] = __float2bfloat16_rn(0.f);
    t[2] = t[1];
    return;
  }
  const float r1 = x - hf;
  const __nv_bfloat16 m = __float2bfloat16_rn(r1);
  t[1] = m;
  t[2] = __float2bfloat16_rn(r1 - __bfloat162float(m));
}

#endif /* HCBLAS_B200_SPLIT_BF16_CUH_ */
