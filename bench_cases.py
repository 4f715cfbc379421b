"""Named single-GEMM workloads for profiling the library's kernels (a
harness beside bench.py, not part of the library package).

    python bench_cases.py <case> [<case> ...]
    python bench_cases.py --list

Each case allocates its operands on cuda:0 (seeded, synthetic), makes one
warm-up call, then one more call of the same GEMM through the public C ABI,
and synchronises: under a profiler, skip the warm-up call's launches (`-s`)
and capture the second call's.  Sizes keep every case to a few GB of device
memory and inputs larger than the 126 MB L2 where the workload allows.
"""
from __future__ import annotations

import ctypes
import sys

import numpy as np

import hcblas_b200 as hb

N_, T_, C_ = hb.HCBLAS_OP_N, hb.HCBLAS_OP_T, hb.HCBLAS_OP_C


def _dev(h, x):
    return hb.DeviceArray(h, x)


def _real(h, dtype, op_a, op_b, m, n, k, mode=0, param=0, seed=0, beta=0.0):
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if op_a == N_ else (k, m)
    br, bc = (k, n) if op_b == N_ else (n, k)
    A = rng.standard_normal(ar * ac).astype(dtype)
    B = rng.standard_normal(br * bc).astype(dtype)
    C = (rng.standard_normal(m * n) if beta else np.zeros(m * n)).astype(dtype)
    dA, dB, dC = _dev(h, A), _dev(h, B), _dev(h, C)
    L = hb.lib()
    f = {np.float16: L.hcblasHgemm, np.float32: L.hcblasSgemm, np.float64: L.hcblasDgemm}[dtype]
    one, bb = hb.scalar_bytes(np.dtype(dtype), 1.0), hb.scalar_bytes(np.dtype(dtype), beta)
    hb.hcblasSetMathMode(h, mode, param)

    def call():
        assert f(h, op_a, op_b, m, n, k, one.ctypes.data, dA.ptr, ar, dB.ptr, br,
                 bb.ctypes.data, dC.ptr, m) == 0
    return call, (dA, dB, dC)


def _complex(h, dtype, op_a, op_b, m, n, k, mode=0, param=0, seed=4):
    rng = np.random.default_rng(seed)
    ar, ac = (m, k) if op_a == N_ else (k, m)
    br, bc = (k, n) if op_b == N_ else (n, k)
    A = (rng.standard_normal(ar * ac) + 1j * rng.standard_normal(ar * ac)).astype(dtype)
    B = (rng.standard_normal(br * bc) + 1j * rng.standard_normal(br * bc)).astype(dtype)
    C = np.zeros(m * n, dtype=dtype)
    dA, dB, dC = _dev(h, A), _dev(h, B), _dev(h, C)
    L = hb.lib()
    f = L.hcblasCgemm if dtype == np.complex64 else L.hcblasZgemm
    al = hb.scalar_bytes(np.dtype(dtype), 1 + 0.5j)
    be = hb.scalar_bytes(np.dtype(dtype), 0.5 - 0.25j)
    hb.hcblasSetMathMode(h, mode, param)

    def call():
        assert f(h, op_a, op_b, m, n, k, al.ctypes.data, dA.ptr, ar, dB.ptr, br, be.ctypes.data,
                 dC.ptr, m) == 0
    return call, (dA, dB, dC)


def _grouped(h, count=4096, seed=3, dtype=np.float16, pad_c=False):
    """Uneven grouped GEMM: M, N, K log-uniform integers in [16, 1024], mixed
    N/T; f16 (hcblasHgemmGrouped, the leading dimensions of A and B padded to
    8 elements for TMA; C's too when pad_c) or f32 (hcblasSgemmGrouped on the
    split-BF16 path, unpadded)."""
    rng = np.random.default_rng(seed)
    lu = lambda: int(np.exp(rng.uniform(np.log(16), np.log(1025))))
    probs, keep = [], []
    esz = np.dtype(dtype).itemsize
    for _ in range(count):
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        m, n, k = lu(), lu(), lu()
        r8 = (lambda v: -(-v // 8) * 8) if esz == 2 else (lambda v: v)
        lda, ldb = r8(m if ta == 0 else k), r8(k if tb == 0 else n)
        A = rng.uniform(-1, 1, lda * (k if ta == 0 else m)).astype(dtype)
        B = rng.uniform(-1, 1, ldb * (n if tb == 0 else k)).astype(dtype)
        dA, dB = _dev(h, A), _dev(h, B)
        ldc = r8(m) if pad_c else m
        dC = hb.DeviceArray(h, nbytes=esz * ldc * n, dtype=dtype)
        keep += [dA, dB, dC]
        probs.append(hb.GemmProblem(ta, tb, m, n, k, dA.ptr, lda, dB.ptr, ldb, dC.ptr, ldc))
    arr = (hb.GemmProblem * count)(*probs)
    if esz == 2:
        one = np.array([1.0], np.float16).view(np.uint16)
        zero = np.array([0.0], np.float16).view(np.uint16)
        fn = hb.lib().hcblasHgemmGrouped
    else:
        one, zero = np.array([1.0], np.float32), np.array([0.0], np.float32)
        fn = hb.lib().hcblasSgemmGrouped

    def call():
        assert fn(h, count, ctypes.cast(arr, ctypes.c_void_p), one.ctypes.data,
                  zero.ctypes.data) == 0
    return call, (keep, arr)


def _strided(h, batch=512, n=128, seed=5):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, n * n * batch).astype(np.float16)
    B = rng.uniform(-1, 1, n * n * batch).astype(np.float16)
    dA, dB = _dev(h, A), _dev(h, B)
    dC = hb.DeviceArray(h, nbytes=2 * n * n * batch, dtype=np.float16)

    def call():
        assert hb.gemm_strided_batched(h, 0, 0, n, n, n, 1.0, dA, n, n * n, dB, n, n * n, 0.0,
                                       dC, n, n * n, batch) == 0
    return call, (dA, dB, dC)


def _ptr_batch(h, batch=512, n=128, seed=5):
    """The strided case's batch through hcblasHgemmBatched (device-resident
    pointer arrays): table build, grouped launch, selective CUDA-core pass."""
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, n * n * batch).astype(np.float16)
    B = rng.uniform(-1, 1, n * n * batch).astype(np.float16)
    dA, dB = _dev(h, A), _dev(h, B)
    dC = hb.DeviceArray(h, nbytes=2 * n * n * batch, dtype=np.float16)
    ptrs = [_dev(h, np.array([d.ptr + 2 * i * n * n for i in range(batch)], dtype=np.uint64))
            for d in (dA, dB, dC)]

    def call():
        assert hb.gemm_batched(h, 0, 0, n, n, n, 1.0, ptrs[0].ptr, n, ptrs[1].ptr, n, 0.0,
                               ptrs[2].ptr, n, batch, np.float16) == 0
    return call, (dA, dB, dC, ptrs)


def _gemv(h, dtype, trans, m, n, seed=6):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, m * n).astype(dtype)
    x = rng.uniform(-1, 1, n if trans == 0 else m).astype(dtype)
    y = np.zeros(m if trans == 0 else n, dtype=dtype)
    dA, dx, dy = _dev(h, A), _dev(h, x), _dev(h, y)

    def call():
        assert hb.gemv(h, trans, m, n, 1.0, dA, m, dx, 1, 0.0, dy, 1) == 0
    return call, (dA, dx, dy)


def _ger(h, dtype, m, n, seed=7):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, m * n).astype(dtype)
    x = rng.uniform(-1, 1, m).astype(dtype)
    y = rng.uniform(-1, 1, n).astype(dtype)
    dA, dx, dy = _dev(h, A), _dev(h, x), _dev(h, y)

    def call():
        assert hb.ger(h, m, n, 0.5, dx, 1, dy, 1, dA, m) == 0
    return call, (dA, dx, dy)


def _cublas_int8(h, n=8192, reps=20):
    """Reference rate of the int8 tensor cores: cuBLASLt's int8 GEMM
    (torch._int_mm, s8 x s8 -> s32, n^3, uniform s8 data), timed with CUDA
    events over `reps` back-to-back calls; prints TOPS.  Library code, not
    part of this library's paths."""
    import torch
    g = torch.Generator(device="cuda").manual_seed(11)
    a = torch.randint(-127, 128, (n, n), device="cuda", dtype=torch.int8, generator=g)
    b = torch.randint(-127, 128, (n, n), device="cuda", dtype=torch.int8, generator=g)
    bt = b.t().contiguous().t()

    def call():
        for _ in range(3):
            torch._int_mm(a, bt)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            torch._int_mm(a, bt)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        print(f"cublas int8 {n}^3: {ms:.4f} ms -> {2 * n ** 3 / ms / 1e9:.1f} TOPS", flush=True)
    return call, (a, bt)


CASES = {
    "hgemm_nt_8192": lambda h: _real(h, np.float16, N_, T_, 8192, 8192, 8192),
    "hgemm_nt_8192_beta05": lambda h: _real(h, np.float16, N_, T_, 8192, 8192, 8192, beta=0.5),
    "sgemm_split6_tn_8192x8192x256_beta1": lambda h: _real(h, np.float32, T_, N_, 8192, 8192, 256,
                                                           1, 6, beta=1.0),
    "sgemm_plain_tn_8192x8192x256_beta1": lambda h: _real(h, np.float32, T_, N_, 8192, 8192, 256,
                                                          beta=1.0),
    "sgemm_plain_tn_4096": lambda h: _real(h, np.float32, T_, N_, 4096, 4096, 4096),
    "sgemm_split6_tn_4096": lambda h: _real(h, np.float32, T_, N_, 4096, 4096, 4096, 1, 6),
    "sgemm_split3_tn_4096": lambda h: _real(h, np.float32, T_, N_, 4096, 4096, 4096, 1, 3),
    "dgemm_native_nt_4096": lambda h: _real(h, np.float64, N_, T_, 4096, 4096, 4096),
    "dgemm_crt15_nt_4096": lambda h: _real(h, np.float64, N_, T_, 4096, 4096, 4096, 4, 15),
    "dgemm_crt14_nt_4096": lambda h: _real(h, np.float64, N_, T_, 4096, 4096, 4096, 4, 14),
    "dgemm_ozaki_i8_s6_nt_4096": lambda h: _real(h, np.float64, N_, T_, 4096, 4096, 4096, 2, 6),
    "sgemm_ozaki_i8_s4_tn_4096_beta1": lambda h: _real(h, np.float32, T_, N_, 4096, 4096, 4096,
                                                       2, 4, beta=1.0),
    "cublas_int8_8192": _cublas_int8,
    "cgemm_plain_cn_2048": lambda h: _complex(h, np.complex64, C_, N_, 2048, 2048, 2048),
    "cgemm_split3m_cn_2048": lambda h: _complex(h, np.complex64, C_, N_, 2048, 2048, 2048, 1, 6),
    "zgemm_native_cn_2048": lambda h: _complex(h, np.complex128, C_, N_, 2048, 2048, 2048),
    "zgemm_crt3m_cn_2048": lambda h: _complex(h, np.complex128, C_, N_, 2048, 2048, 2048, 4, 0),
    "hgemm_grouped_4096": _grouped,
    "hgemm_grouped_4096_ldc8": lambda h: _grouped(h, pad_c=True),
    "sgemm_grouped_4096": lambda h: _grouped(h, dtype=np.float32),
    "hgemm_strided_512x128": _strided,
    "hgemm_ptr_512x128": _ptr_batch,
    "sgemv_n_16384": lambda h: _gemv(h, np.float32, 0, 16384, 16384),
    "sgemv_t_16384": lambda h: _gemv(h, np.float32, 1, 16384, 16384),
    "dgemv_n_16384": lambda h: _gemv(h, np.float64, 0, 16384, 16384),
    "dgemv_t_16384": lambda h: _gemv(h, np.float64, 1, 16384, 16384),
    "sger_16384": lambda h: _ger(h, np.float32, 16384, 16384),
    "dger_16384": lambda h: _ger(h, np.float64, 16384, 16384),
}


def main(argv):
    if not argv or argv[0] == "--list":
        print("\n".join(CASES))
        return 0
    import torch
    torch.cuda.set_device(0)
    s, h = hb.hcblasCreate(0)
    assert s == 0
    for name in argv:
        call, keep = CASES[name](h)
        call()  # warm-up (and plan / workspace set-up)
        torch.cuda.synchronize()
        call()  # the call to profile
        torch.cuda.synchronize()
        assert hb.device_error(h) == 0, name
        print(f"{name}: path {hb.hcblasGetLastPath(h)}", flush=True)
        del keep
    hb.hcblasDestroy(h)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
