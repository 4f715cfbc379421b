"""Generate the golden GEMM fixtures under tests/golden/ (run on a CPU; no GPU).

The reference (hcBLAS) holds no stored output vectors: its tests rebuild
inputs from glibc ``rand_r`` seeds and compare against host CBLAS at run time.
This script reproduces those recipes and freezes the answers:

* ``int_chain_{s,d,c,z}.npz`` -- the integer-valued recipes of
  test/unit/hcblas_dgemm.cpp:201-353 (A = rand_r % 100, B = % 15, C = % 25,
  M=189, N=9, K=19, global_seed = 100; complex parts % 10/20/15/25/18/28 as in
  test/unit/hcblas_cgemm.cpp:268-302).  As in those tests, one C buffer is
  updated by a chain of calls (col/row-major x NN/NT/TN/TT, then alpha = 0 and
  alpha = beta = 0); complex chains also take the conjugate-transpose cases.
  The expected C after every step is computed here in exact integer
  arithmetic (Python ints), independently of both the oracle and CBLAS, and
  checked against OpenBLAS's CBLAS.
* ``float_cases.npz`` -- seeded Gaussian inputs at 21x17x13 for every dtype,
  order, transpose (incl. conjugate), with element offsets and padded leading
  dimensions, alpha/beta generic and beta = 0 over a NaN-filled C (CBLAS does
  not read C when beta = 0); expected outputs from OpenBLAS 0.3.30's CBLAS.
* ``sgemm_recipe.npz`` -- the U[0,2) SGEMM recipe of
  test/unit/hcblas_sgemm.cpp:222-243 with alpha/beta drawn as at :966-969, at
  the vvsmall (4) and vsmall (48) shape classes of test/unit/test_constants.h,
  column-major NN; expected output from OpenBLAS; pass bound 1e-5 (:260-261).
* ``capi_ones.npz`` -- the C-API all-ones case of
  test/unit-api/test-blas.cpp:1851-1937 (123x78x23, alpha = beta = 2).

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import cblas_ref  # noqa: E402
from oracle.oracle import RandR, srand_rand  # noqa: E402

ROW, COL = 0, 1
N_, T_, C_ = 0, 1, 2


def exact_gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc):
    """Exact CBLAS-semantics GEMM on Python ints / Gaussian integers."""
    def get(X, ld, i, j):
        return X[i + j * ld] if order == COL else X[i * ld + j]

    def opget(X, ld, trans, r, s):
        v = get(X, ld, r, s) if trans == N_ else get(X, ld, s, r)
        if trans == C_:
            v = v.conjugate()
        return v

    out = list(C)
    for n in range(N):
        for m in range(M):
            acc = 0
            for k in range(K):
                acc += opget(A, lda, ta, m, k) * opget(B, ldb, tb, k, n)
            idx = m + n * ldc if order == COL else m * ldc + n
            val = alpha * acc
            if beta != 0:
                val += beta * C[idx]
            out[idx] = val
    return out


class GaussInt:
    """Minimal exact Gaussian integer for the complex chains."""

    __slots__ = ("re", "im")

    def __init__(self, re, im=0):
        self.re, self.im = int(re), int(im)

    def __add__(self, o):
        o = o if isinstance(o, GaussInt) else GaussInt(o)
        return GaussInt(self.re + o.re, self.im + o.im)

    __radd__ = __add__

    def __mul__(self, o):
        o = o if isinstance(o, GaussInt) else GaussInt(o)
        return GaussInt(self.re * o.re - self.im * o.im, self.re * o.im + self.im * o.re)

    __rmul__ = __mul__

    def conjugate(self):
        return GaussInt(self.re, -self.im)

    def __ne__(self, o):
        o = o if isinstance(o, GaussInt) else GaussInt(o)
        return self.re != o.re or self.im != o.im


def chain_steps(M, N, K, cplx):
    steps = []
    combos = [(N_, N_), (N_, T_), (T_, N_), (T_, T_)]
    if cplx:
        combos += [(C_, N_), (N_, C_), (C_, C_), (C_, T_)]
    for ta, tb in combos:
        steps.append((COL, ta, tb, M if ta == N_ else K, K if tb == N_ else N, M))
        steps.append((ROW, ta, tb, K if ta == N_ else M, N if tb == N_ else K, N))
    return steps


def make_int_chain(kind):
    M, N, K = 189, 9, 19
    rr = RandR(100)
    cplx = kind in ("c", "z")
    if cplx:
        # test/unit/hcblas_cgemm.cpp:268-290: re/im drawn alternately per element
        def draw(n, m1, m2):
            out = []
            for _ in range(n):
                re = rr.next() % m1
                im = rr.next() % m2
                out.append(GaussInt(re, im))
            return out
        A = draw(M * K, 10, 20)
        B = draw(K * N, 15, 25)
        C = draw(M * N, 18, 28)
        one = GaussInt(1, 1)  # cAlpha = cBeta = 1 + 1i
    else:
        A = [rr.next() % 100 for _ in range(M * K)]
        B = [rr.next() % 15 for _ in range(K * N)]
        C = [rr.next() % 25 for _ in range(M * N)]
        one = 1
    steps = chain_steps(M, N, K, cplx)
    records = []  # (order, ta, tb, lda, ldb, ldc, alpha_re, alpha_im, beta_re, beta_im)
    states = []
    cur = C
    for (order, ta, tb, lda, ldb, ldc) in steps:
        cur = exact_gemm(order, ta, tb, M, N, K, one, A, lda, B, ldb, one, cur, ldc)
        a = (1, 1) if cplx else (1, 0)
        records.append((order, ta, tb, lda, ldb, ldc, a[0], a[1], a[0], a[1]))
        states.append(list(cur))
    # alpha = 0, then alpha = beta = 0 (test/unit/hcblas_dgemm.cpp:293-353)
    zero = GaussInt(0) if cplx else 0
    for beta in (one, zero):
        cur = exact_gemm(COL, N_, T_, M, N, K, zero, A, M, B, N, beta, cur, M)
        b = ((1, 1) if cplx else (1, 0)) if beta != zero else (0, 0)
        records.append((COL, N_, T_, M, N, M, 0, 0, b[0], b[1]))
        states.append(list(cur))

    def to_np(vals):
        if cplx:
            return np.array([complex(v.re, v.im) for v in vals], dtype=np.complex128)
        return np.array(vals, dtype=np.float64)

    npdt = {"s": np.float32, "d": np.float64, "c": np.complex64, "z": np.complex128}[kind]
    A_np, B_np, C_np = to_np(A), to_np(B), to_np(C)
    S_np = np.stack([to_np(s) for s in states])
    assert np.max(np.abs(S_np)) < 2 ** 24, "chain left the exactly-representable range"
    # Cross-check against a real CBLAS (OpenBLAS): must match exactly.
    a_c = A_np.astype(npdt)
    b_c = B_np.astype(npdt)
    c_c = C_np.astype(npdt)
    for rec, st in zip(records, S_np):
        order, ta, tb, lda, ldb, ldc, ar, ai, br, bi = rec
        al = complex(ar, ai) if cplx else float(ar)
        be = complex(br, bi) if cplx else float(br)
        cblas_ref.gemm(order, ta, tb, M, N, K, al, a_c, lda, b_c, ldb, be, c_c, ldc)
        assert np.array_equal(c_c.astype(st.dtype), st), f"OpenBLAS disagrees at step {rec}"
    np.savez_compressed(
        os.path.join(HERE, f"int_chain_{kind}.npz"),
        M=M, N=N, K=K, A=A_np.astype(npdt), B=B_np.astype(npdt), C=C_np.astype(npdt),
        steps=np.array(records, dtype=np.int64), states=S_np.astype(npdt))
    return len(records)


def make_float_cases():
    rng = np.random.default_rng(20240)
    M, N, K = 21, 17, 13
    out = {}
    idx = 0
    meta = []
    for kind, dt in (("s", np.float32), ("d", np.float64), ("c", np.complex64), ("z", np.complex128)):
        cplx = kind in ("c", "z")
        transes = (N_, T_, C_) if cplx else (N_, T_)
        for order in (COL, ROW):
            for ta in transes:
                for tb in transes:
                    for beta_zero in (False, True):
                        ar_, ac_ = (M, K) if ta == N_ else (K, M)
                        br_, bc_ = (K, N) if tb == N_ else (N, K)
                        pad = 2
                        lda = (ar_ if order == COL else ac_) + pad
                        ldb = (br_ if order == COL else bc_) + pad
                        ldc = (M if order == COL else N) + pad
                        a_off, b_off, c_off = 3, 5, 7
                        na = a_off + lda * (ac_ if order == COL else ar_)
                        nb = b_off + ldb * (bc_ if order == COL else br_)
                        nc = c_off + ldc * (N if order == COL else M)

                        def rnd(n):
                            v = rng.standard_normal(n)
                            if cplx:
                                v = v + 1j * rng.standard_normal(n)
                            return v.astype(dt)
                        A, B, C = rnd(na), rnd(nb), rnd(nc)
                        if beta_zero:
                            C[:] = np.nan
                            beta = 0.0
                        else:
                            beta = (0.5 - 0.75j) if cplx else 0.5
                        alpha = (1.5 + 0.25j) if cplx else 1.5
                        Cout = C.copy()
                        cblas_ref.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, Cout, ldc,
                                       a_off, b_off, c_off)
                        key = f"c{idx:03d}"
                        out[key + "_A"], out[key + "_B"], out[key + "_C"], out[key + "_out"] = A, B, C, Cout
                        meta.append((idx, "sdcz".index(kind), order, ta, tb, M, N, K, lda, ldb, ldc,
                                     a_off, b_off, c_off))
                        out[key + "_alpha"] = np.array([complex(alpha)])
                        out[key + "_beta"] = np.array([complex(beta)])
                        idx += 1
    out["meta"] = np.array(meta, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "float_cases.npz"), **out)
    return idx


def make_sgemm_recipe():
    # test/unit/test_constants.h: srand(1); rand() % range + base
    vvsmall = srand_rand(1) % 10 + 1
    vsmall = srand_rand(1) % 89 + 11
    rr = RandR(100)
    out = {}
    shapes = []
    RAND_MAX = RandR.RAND_MAX
    for i, s in enumerate((vvsmall, vsmall)):
        M = N = K = int(s)
        alpha = np.float32(np.float32(rr.next()) / np.float32(RAND_MAX * 1.172))
        beta = np.float32(np.float32(rr.next()) / np.float32(RAND_MAX * 3.414))
        A = rr.uniform02(M * K)
        B = rr.uniform02(K * N)
        C = rr.uniform02(M * N)
        Cout = C.copy()
        cblas_ref.gemm(COL, N_, N_, M, N, K, float(alpha), A, M, B, K, float(beta), Cout, M)
        out[f"s{i}_A"], out[f"s{i}_B"], out[f"s{i}_C"], out[f"s{i}_out"] = A, B, C, Cout
        out[f"s{i}_ab"] = np.array([alpha, beta], dtype=np.float32)
        shapes.append(M)
    out["shapes"] = np.array(shapes)
    out["tolerance"] = np.array(1.0e-5)
    np.savez_compressed(os.path.join(HERE, "sgemm_recipe.npz"), **out)
    return shapes


def make_capi_ones():
    M, N, K = 123, 78, 23
    A = np.ones(M * K, np.float32)
    B = np.ones(K * N, np.float32)
    C = np.ones(M * N, np.float32)
    Cout = C.copy()
    cblas_ref.gemm(COL, N_, N_, M, N, K, 2.0, A, M, B, K, 2.0, Cout, M)
    assert np.all(Cout == 2 * K + 2)
    np.savez_compressed(os.path.join(HERE, "capi_ones.npz"), M=M, N=N, K=K, A=A, B=B, C=C, out=Cout)


if __name__ == "__main__":
    cblas_ref.set_threads(1)
    for kind in "sdcz":
        print("int_chain", kind, make_int_chain(kind), "steps")
    print("float_cases", make_float_cases())
    print("sgemm_recipe shapes", make_sgemm_recipe())
    make_capi_ones()
    print("capi_ones done")
