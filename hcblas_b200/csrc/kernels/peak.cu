/*
 * Issue-rate probes of the arithmetic pipes that the native GEMM kernels run
 * on, so that their rates can be stated as fractions of what this GPU
 * delivers rather than of a data-sheet figure:
 *
 *   kind 0  FP32 FMA pipe, packed fma.rn.f32x2 (2 x 2 flops per lane)
 *   kind 1  FP64 pipe, fma.rn.f64
 *   kind 2  FP64 tensor path, mma.sync.aligned.m16n8k4 .f64 (1024 flops per
 *           warp instruction)
 *
 * Each thread (warp, for kind 2) runs independent accumulation chains that
 * are long enough to keep the pipe busy, on a grid of as many 256-thread
 * blocks as are resident at once.  The operands are runtime values and every chain's
 * result is stored, so nothing folds away.  The probe times one launch after
 * a warm-up launch with CUDA events on its own stream and reports TFLOP/s.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include "hcbk.h"

namespace {

constexpr int PEAK_THREADS = 256;
constexpr int F32_CHAINS = 8;  /* f32x2 pairs per thread */
constexpr int F64_CHAINS = 8;
constexpr int DMMA_CHAINS = 4; /* accumulator fragments per warp */

__device__ __forceinline__ uint64_t fma_f32x2(uint64_t a, uint64_t b, uint64_t c) {
  uint64_t d;
  asm volatile("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

__global__ void __launch_bounds__(PEAK_THREADS) peak_f32(uint64_t x, uint64_t y, int iters,
                                                         uint64_t *out) {
  uint64_t acc[F32_CHAINS];
#pragma unroll
  for (int j = 0; j < F32_CHAINS; ++j) acc[j] = x + (uint64_t)(threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < F32_CHAINS; ++j) acc[j] = fma_f32x2(acc[j], x, y);
  }
  uint64_t s = 0;
#pragma unroll
  for (int j = 0; j < F32_CHAINS; ++j) s ^= acc[j];
  out[blockIdx.x * PEAK_THREADS + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PEAK_THREADS) peak_f64(double x, double y, int iters,
                                                         double *out) {
  double acc[F64_CHAINS];
#pragma unroll
  for (int j = 0; j < F64_CHAINS; ++j) acc[j] = x * (double)(threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < F64_CHAINS; ++j) acc[j] = fma(acc[j], x, y);
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < F64_CHAINS; ++j) s += acc[j];
  out[blockIdx.x * PEAK_THREADS + threadIdx.x] = s;
}

__global__ void __launch_bounds__(PEAK_THREADS) peak_dmma(double x, double y, int iters,
                                                          double *out) {
  double c[DMMA_CHAINS][4];
#pragma unroll
  for (int j = 0; j < DMMA_CHAINS; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) c[j][q] = 0.0;
  const double a0 = x * (double)(threadIdx.x & 31), a1 = y, b0 = x + y;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < DMMA_CHAINS; ++j)
      asm volatile(
          "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5}, "
          "{%6}, {%0, %1, %2, %3};"
          : "+d"(c[j][0]), "+d"(c[j][1]), "+d"(c[j][2]), "+d"(c[j][3])
          : "d"(a0), "d"(a1), "d"(b0));
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < DMMA_CHAINS; ++j) s += c[j][0] + c[j][1] + c[j][2] + c[j][3];
  out[blockIdx.x * PEAK_THREADS + threadIdx.x] = s;
}

}  // namespace

/* kind: 0 FP32 FMA (f32x2), 1 FP64 FMA, 2 FP64 mma.sync; iters per chain
 * (0 = a default of about 10 ms of work).  Writes the achieved TFLOP/s and
 * returns HCBK_OK, or an error code (device memory, launch). */
extern "C" int hcbk_peak_probe(int kind, int iters, double *tflops) {
  if (kind < 0 || kind > 2 || iters < 0 || !tflops) return HCBK_ERR_ARGS;
  if (iters == 0) iters = kind == 0 ? 200000 : (kind == 1 ? 100000 : 20000);
  int per_sm = 0;
  const void *fn = kind == 0 ? (const void *)peak_f32
                             : (kind == 1 ? (const void *)peak_f64 : (const void *)peak_dmma);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, PEAK_THREADS, 0) != cudaSuccess ||
      per_sm < 1)
    return HCBK_ERR_LAUNCH;
  const int blocks = hcbk_sm_count() * per_sm;
  const size_t out_bytes = (size_t)blocks * PEAK_THREADS * 8;
  cudaStream_t st = nullptr;
  void *out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = HCBK_ERR_LAUNCH;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return rc;
  if (cudaMalloc(&out, out_bytes) != cudaSuccess) {
    cudaStreamDestroy(st);
    return HCBK_ERR_NOMEM;
  }
  if (cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess) {
    float ms = 0.f;
    bool ok = true;
    for (int rep = 0; rep < 2 && ok; ++rep) { /* warm-up, then the timed launch */
      ok = cudaEventRecord(e0, st) == cudaSuccess;
      if (kind == 0) {
        const uint64_t x = 0x3f8000003f800000ull, y = 0x3380000033800000ull; /* 1, 2^-24 */
        peak_f32<<<blocks, PEAK_THREADS, 0, st>>>(x, y, iters, static_cast<uint64_t *>(out));
      } else if (kind == 1) {
        peak_f64<<<blocks, PEAK_THREADS, 0, st>>>(1.0, 0x1p-53, iters, static_cast<double *>(out));
      } else {
        peak_dmma<<<blocks, PEAK_THREADS, 0, st>>>(1.0, 0x1p-53, iters, static_cast<double *>(out));
      }
      ok = ok && cudaGetLastError() == cudaSuccess && cudaEventRecord(e1, st) == cudaSuccess &&
           cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
    }
    if (ok && ms > 0.f) {
      const double threads = (double)blocks * PEAK_THREADS;
      double flop;
      if (kind == 0)
        flop = threads * iters * F32_CHAINS * 4.0;
      else if (kind == 1)
        flop = threads * iters * F64_CHAINS * 2.0;
      else
        flop = threads / 32.0 * iters * DMMA_CHAINS * (16.0 * 8.0 * 4.0 * 2.0);
      *tflops = flop / (ms * 1e-3) / 1e12;
      rc = HCBK_OK;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(out);
  cudaStreamDestroy(st);
  return rc;
}
