"""GPU parity of the Ozaki-scheme DGEMM (INT8 slices on tcgen05 kind::i8, and
8-bit slices in binary16 on tcgen05 kind::f16) against the double-double
oracle.

Bound (a-priori, per element).  With e_m, f_n the row/column exponents
(|A(m,k)| < 2^e_m, |B(k,n)| < 2^f_n), s slices of b bits (b = 7 for INT8,
b = 8 for f16):
  representation: |A - A_s| < 2^(e_m - b s), same for B     -> 2 * 2^(-b s)
  dropped products a_i b_j with i + j >= s                  -> (s+1) * 2^(-b s)
  binary64 additions of the group sums (n_add of them, each
  on a partial sum below K 2^(e_m + f_n))                   -> n_add * u
so |C - C_s| <= |alpha| K 2^(e_m + f_n) ((s+3) 2^(-b s) + n_add u) + 2u|beta C|.
The test uses the Frobenius norm of that elementwise bound.
"""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O
from tests.test_gemm_gpu import make_case, op_dense, TCH

pytestmark = pytest.mark.gpu

MODES = {"i8": (hb.HCBLAS_MATH_OZAKI_INT8, 7), "f16": (hb.HCBLAS_MATH_OZAKI_F16, 8)}
U = 2.0 ** -53


def ozaki_bound(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, s, ref, kind="i8", beta=0.0, C=None,
                ldc=None):
    bits = MODES[kind][1]
    Ad = op_dense(A, order, ta, M, K, lda, 0)
    Bd = op_dense(B, order, tb, K, N, ldb, 0)
    ea = np.frexp(np.max(np.abs(Ad), axis=1))[1].astype(np.float64)
    eb = np.frexp(np.max(np.abs(Bd), axis=0))[1].astype(np.float64)
    scale = np.exp2(ea[:, None] + eb[None, :])
    n_add = (-(-K // 32)) * s + 2 if kind == "f16" else s + 2
    elem = abs(alpha) * K * scale * ((s + 3) * 2.0 ** (-bits * s) + n_add * U)
    out = np.linalg.norm(elem) + 4 * U * np.linalg.norm(ref)
    if beta and C is not None:
        out += 2 * U * abs(beta) * np.linalg.norm(O.view_c(C, order, M, N, ldc))
    return out


def run_ozaki(handle, kind, s, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc):
    assert hb.hcblasSetMathMode(handle, MODES[kind][0], s) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta,
                         dC, ldc)
        assert rc == 0
        assert hb.device_error(handle) == 0
        path = hb.hcblasGetLastPath(handle)
        return dC.download(), path
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


CASES = [(O.COL, 0, 1, 300, 200, 500), (O.COL, 1, 0, 129, 77, 64), (O.ROW, 0, 0, 256, 256, 1000),
         (O.COL, 1, 1, 1000, 130, 257)]


@pytest.mark.parametrize("kind,s", [("i8", 3), ("i8", 5), ("i8", 7), ("i8", 8), ("f16", 3),
                                    ("f16", 4), ("f16", 5), ("f16", 6), ("f16", 7)])
def test_ozaki_slices_vs_dd_oracle(handle, kind, s):
    rng = np.random.default_rng(500 + s)
    for order, ta, tb, M, N, K in CASES:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        alpha, beta = 1.5, -0.25
        got, path = run_ozaki(handle, kind, s, order, ta, tb, M, N, K, alpha, beta, A, lda, B,
                              ldb, C, ldc)
        assert path == f"tc.ozaki_{kind}_s{s}", path
        _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        gv = O.view_c(got, order, M, N, ldc)
        err = np.linalg.norm(gv - ref)
        bound = ozaki_bound(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, s, ref, kind, beta, C,
                            ldc)
        assert err <= bound, (kind, s, order, ta, tb, M, N, K, err, bound)


@pytest.mark.parametrize("kind", ["i8", "f16"])
def test_ozaki_hard_exponent_range(handle, kind):
    """Entries N(0,1) * 2^e, e ~ U{-20..20} per row of A and per column of B."""
    rng = np.random.default_rng(1)
    M = N = K = 512
    A = (rng.standard_normal((M, K)) * np.exp2(rng.integers(-20, 21, M))[:, None])
    B = (rng.standard_normal((K, N)) * np.exp2(rng.integers(-20, 21, N))[None, :])
    Af = np.asfortranarray(A).reshape(-1, order="F")
    Bf = np.asfortranarray(B).reshape(-1, order="F")
    C = np.zeros(M * N)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, Af, M, Bf, K, 0.0, C, M)
    errs = {}
    for s in (5, 6, 7):
        got, _ = run_ozaki(handle, kind, s, O.COL, 0, 0, M, N, K, 1.0, 0.0, Af, M, Bf, K, C, M)
        gv = O.view_c(got, O.COL, M, N, M)
        errs[s] = O.normwise_rel_error(gv, ref)
        bound = ozaki_bound(O.COL, 0, 0, M, N, K, 1.0, Af, M, Bf, K, s, ref, kind)
        assert np.linalg.norm(gv - ref) <= bound
    print(f"ozaki {kind} hard-range normwise errors:", errs)
    assert errs[7] < errs[6] < errs[5]


@pytest.mark.parametrize("kind", ["i8", "f16"])
def test_ozaki_special_rows(handle, kind):
    rng = np.random.default_rng(4)
    M, N, K = 64, 48, 80
    A = rng.standard_normal(M * K)
    B = rng.standard_normal(K * N)
    A[3 + np.arange(K) * M] = 0.0       # row 3 of A all zero
    A[5 + 7 * M] = np.nan               # row 5 holds a NaN
    C = np.ones(M * N)
    got, _ = run_ozaki(handle, kind, 7, O.COL, 0, 0, M, N, K, 1.0, 0.5, A, M, B, K, C, M)
    gv = O.view_c(got, O.COL, M, N, M)
    assert np.all(np.isnan(gv[5, :]))
    assert np.all(gv[3, :] == 0.5)
    ok = np.ones(M, bool)
    ok[5] = False
    A0 = np.nan_to_num(A)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, 0.5, C, M)
    bound = ozaki_bound(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, 7, ref, kind, 0.5, C, M)
    assert np.linalg.norm(gv[ok] - ref[ok]) <= bound


def test_ozaki_i8_pair_matches_single_cta(handle):
    """The INT8 slice-group sums are exact, so the CTA-pair and single-CTA
    launches give bit-identical results."""
    rng = np.random.default_rng(41)
    for order, ta, tb, M, N, K in CASES + [(O.COL, 0, 1, 600, 520, 300)]:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        outs = []
        for pair in (0, 2):
            assert hb.set_tuning(handle, "tc_pair", pair) == 0
            try:
                outs.append(run_ozaki(handle, "i8", 6, order, ta, tb, M, N, K, 1.5, -0.25, A, lda,
                                      B, ldb, C, ldc)[0])
            finally:
                hb.set_tuning(handle, "tc_pair", 1)
        assert np.array_equal(outs[0], outs[1]), (order, ta, tb, M, N, K)


@pytest.mark.parametrize("kind", ["i8", "f16"])
def test_ozaki_long_k(handle, kind):
    """K beyond one INT8 launch's INT32-exact range (16640 for s = 8) is split
    into launches of whole 128-element slabs; the f16 kernel promotes per
    slab and runs it in one."""
    rng = np.random.default_rng(6)
    M, N, K = 40, 36, 17000
    s = 8 if kind == "i8" else 7
    A, lda, B, ldb, C, ldc = make_case(rng, "d", O.COL, 1, 0, M, N, K)
    got, path = run_ozaki(handle, kind, s, O.COL, 1, 0, M, N, K, 1.0, 1.0, A, lda, B, ldb, C, ldc)
    _, ref = O.gemm(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, 1.0, C, ldc)
    err = np.linalg.norm(O.view_c(got, O.COL, M, N, ldc) - ref)
    assert err <= ozaki_bound(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, s, ref, kind, 1.0, C, ldc)


CRT_MODULI = [255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181,
              179, 173, 167]
# K over 3 and 5 1024-element chunks (the in-place modular reduction
# alternates TMEM buffers, so odd chunk counts matter)
CRT_CASES = CASES + [(O.COL, 0, 1, 160, 96, 2500), (O.ROW, 1, 0, 300, 260, 4100)]


def crt_plan_rows(K, want=0):
    """Moduli count and norm shift of the real (DGEMM) CRT path, as the
    library chooses them: integers of up to 53 bits; when the moduli are too
    few for the worst case K 2^106, every row is scaled so that its norm
    stays below 2^(53 - shift) (Cauchy-Schwarz on the integer products; the
    per-element rounding adds at most 3/4 sqrt(K))."""
    lk = np.ceil(np.log2(max(K, 2)))
    hr = 0.75 * np.sqrt(K)
    cum = 0.0
    for i, p in enumerate(CRT_MODULI):
        cum += np.log2(p)
        n = i + 1
        full = cum >= 2 * 53 + 1 + lk + 0.01
        if (want == 0 and full) or want == n or (want == 0 and n == len(CRT_MODULI)):
            if full:
                return n, None
            nb = int(np.floor((cum - 1.02) / 2))
            while nb > 0 and 2 * np.log2(2.0 ** nb + hr) + 0.01 >= cum - 1:
                nb -= 1
            return n, 53 - nb
    raise AssertionError("no plan")


def row_deltas(X, shift):
    """Upper bounds of the per-element rounding error of the rows of X (2-D)
    as the library scales them.  Full width: x' = rint(x 2^(53 - e)), e the
    row maximum's frexp exponent, error 2^(e - 54).  Norm scaling: x' =
    rint(fl(x f) 2^(53 - e)) with f in [1/2, 1] rounded down to 8 bits and
    the scale f 2^-e the smaller of 2^-e_max and 2^(nb - 53) / ||x||, so the
    error is at most 3/4 2^-53 max(2^e_max, ||x|| 2^(53 - nb)) (1 + 2^-6)."""
    mx = np.max(np.abs(X), axis=1)
    e = np.frexp(mx)[1].astype(np.float64)
    if shift is None:
        return np.where(mx > 0, np.exp2(e - 54), 0.0)
    nb = 53 - shift
    nrm = np.linalg.norm(X, axis=1)
    inv_scale = np.maximum(np.exp2(e), nrm * 2.0 ** (53 - nb)) * (1 + 2.0 ** -6)
    return np.where(mx > 0, 0.75 * 2.0 ** -53 * inv_scale, 0.0)


def crt_bound_rows(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, shift, ref, beta=0.0, C=None,
                   ldc=None):
    """|alpha| (da_m sum_k |b_kn| + db_n sum_k |a_mk| + K da_m db_n) with the
    per-element rounding bounds da, db of the scaled rows, plus 10u|C| (and
    2u|beta C|) for the reconstruction and epilogue roundings: P' to binary64
    within 1.5 ulp (3u), the reciprocals of the row fractions and their
    product with the result (4u), alpha and the beta fma (2u)."""
    Ad = op_dense(A, order, ta, M, K, lda, 0)
    Bd = op_dense(B, order, tb, K, N, ldb, 0)
    da = row_deltas(Ad, shift)
    db = row_deltas(Bd.T, shift)
    elem = abs(alpha) * (da[:, None] * np.sum(np.abs(Bd), axis=0)[None, :] +
                         np.sum(np.abs(Ad), axis=1)[:, None] * db[None, :] +
                         K * da[:, None] * db[None, :])
    out = np.linalg.norm(elem) + 10 * U * np.linalg.norm(ref)
    if beta and C is not None:
        out += 2 * U * abs(beta) * np.linalg.norm(O.view_c(C, order, M, N, ldc))
    return out


def run_crt(handle, want, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C, ldc):
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, want) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb, beta,
                         dC, ldc)
        assert rc == 0
        assert hb.device_error(handle) == 0
        return dC.download(), hb.hcblasGetLastPath(handle)
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)


@pytest.mark.parametrize("want", [0, 10, 12, 14, 16, 18, 20])
def test_crt_vs_dd_oracle(handle, want):
    rng = np.random.default_rng(900 + want)
    for order, ta, tb, M, N, K in CRT_CASES:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        alpha, beta = 1.5, -0.25
        nmod, shift = crt_plan_rows(K, want)
        got, path = run_crt(handle, want, order, ta, tb, M, N, K, alpha, beta, A, lda, B, ldb, C,
                            ldc)
        assert path == f"tc.crt_m{nmod}", path
        _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        err = np.linalg.norm(O.view_c(got, order, M, N, ldc) - ref)
        bound = crt_bound_rows(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, shift, ref, beta, C,
                               ldc)
        assert err <= bound, (want, nmod, shift, order, ta, tb, M, N, K, err, bound)


def test_crt_pair_matches_single_cta(handle):
    """The CRT residue GEMMs are exact, so CTA-pair and single-CTA kernels
    must give bit-identical results."""
    rng = np.random.default_rng(31)
    for order, ta, tb, M, N, K in CRT_CASES:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        outs = []
        for pair in (0, 2):
            assert hb.set_tuning(handle, "tc_pair", pair) == 0
            try:
                outs.append(run_crt(handle, 0, order, ta, tb, M, N, K, 1.5, -0.25, A, lda, B, ldb,
                                    C, ldc)[0])
            finally:
                hb.set_tuning(handle, "tc_pair", 1)
        assert np.array_equal(outs[0], outs[1]), (order, ta, tb, M, N, K)


@pytest.mark.parametrize("want", [0, 14])
def test_crt_i8_matches_f16(handle, want):
    """The int8 (kind::i8, INT32 sums over all of K) and binary16 (kind::f16,
    sums reduced mod p every 1024 K) modular GEMMs both produce the exact
    residues, so the two paths must give bit-identical results."""
    rng = np.random.default_rng(77 + want)
    for order, ta, tb, M, N, K in CRT_CASES + [(O.COL, 1, 0, 130, 70, 129)]:
        A, lda, B, ldb, C, ldc = make_case(rng, "d", order, ta, tb, M, N, K)
        outs = []
        for i8 in (1, 0):
            assert hb.set_tuning(handle, "crt_i8", i8) == 0
            try:
                outs.append(run_crt(handle, want, order, ta, tb, M, N, K, 1.5, -0.25, A, lda, B,
                                    ldb, C, ldc)[0])
            finally:
                hb.set_tuning(handle, "crt_i8", 1)
        assert np.array_equal(outs[0], outs[1]), (want, order, ta, tb, M, N, K)


def test_crt_k_beyond_int8_range(handle):
    """K above 131072 (the INT32-exact range of the int8 modular GEMM) falls
    back to the binary16 residue path, which reduces every 1024 K: the result
    equals the forced binary16 path bit for bit and meets the bound."""
    rng = np.random.default_rng(91)
    M, N, K = 40, 36, 131072 + 200
    A, lda, B, ldb, C, ldc = make_case(rng, "d", O.COL, 1, 0, M, N, K)
    got, path = run_crt(handle, 14, O.COL, 1, 0, M, N, K, 1.0, 0.5, A, lda, B, ldb, C, ldc)
    assert path == "tc.crt_m14", path
    assert hb.set_tuning(handle, "crt_i8", 0) == 0
    try:
        forced, _ = run_crt(handle, 14, O.COL, 1, 0, M, N, K, 1.0, 0.5, A, lda, B, ldb, C, ldc)
    finally:
        hb.set_tuning(handle, "crt_i8", 1)
    assert np.array_equal(got, forced)
    _, ref = O.gemm(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, 0.5, C, ldc)
    _, shift = crt_plan_rows(K, 14)
    err = np.linalg.norm(O.view_c(got, O.COL, M, N, ldc) - ref)
    assert err <= crt_bound_rows(O.COL, 1, 0, M, N, K, 1.0, A, lda, B, ldb, shift, ref, 0.5, C,
                                 ldc)


def test_crt_special_and_hard_range(handle):
    rng = np.random.default_rng(12)
    M, N, K = 96, 80, 700
    A = rng.standard_normal(M * K) * np.exp2(rng.integers(-20, 21, M))[np.arange(M * K) % M]
    B = rng.standard_normal(K * N) * np.exp2(rng.integers(-20, 21, N))[np.arange(K * N) // K]
    A[4 + np.arange(K) * M] = 0.0  # zero row
    A[9 + 3 * M] = np.inf          # non-finite row
    C = np.ones(M * N)
    got, _ = run_crt(handle, 0, O.COL, 0, 0, M, N, K, 1.0, 0.5, A, M, B, K, C, M)
    gv = O.view_c(got, O.COL, M, N, M)
    assert np.all(np.isnan(gv[9, :]))
    assert np.all(gv[4, :] == 0.5)
    ok = np.ones(M, bool)
    ok[9] = False
    A0 = np.where(np.isfinite(A), A, 0.0)
    _, ref = O.gemm(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, 0.5, C, M)
    _, shift = crt_plan_rows(K)
    bound = crt_bound_rows(O.COL, 0, 0, M, N, K, 1.0, A0, M, B, K, shift, ref, 0.5, C, M)
    assert np.linalg.norm(gv[ok] - ref[ok]) <= bound


def test_ozaki_vs_native_accuracy(handle):
    """Config of the headline: col-major N/T, N(0,1); errors of native FP64
    and of the Ozaki paths against the double-double oracle."""
    rng = np.random.default_rng(1)
    M = N = K = 1024
    A = rng.standard_normal(M * K)
    B = rng.standard_normal(N * K)
    C = np.zeros(M * N)
    _, ref = O.gemm(O.COL, 0, 1, M, N, K, 1.0, A, M, B, N, 0.0, C, M)
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.lib_gemm(handle, O.COL, "n", "t", M, N, K, 1.0, dA, M, dB, N, 0.0, dC, M) == 0
    errs = {"native": O.normwise_rel_error(O.view_c(dC.download(), O.COL, M, N, M), ref)}
    for kind, s in (("i8", 6), ("i8", 7), ("i8", 8), ("f16", 6), ("f16", 7)):
        got, _ = run_ozaki(handle, kind, s, O.COL, 0, 1, M, N, K, 1.0, 0.0, A, M, B, N, C, M)
        errs[f"{kind}_s{s}"] = O.normwise_rel_error(O.view_c(got, O.COL, M, N, M), ref)
    for want in (0, 14, 15):
        got, path = run_crt(handle, want, O.COL, 0, 1, M, N, K, 1.0, 0.0, A, M, B, N, C, M)
        errs[path] = O.normwise_rel_error(O.view_c(got, O.COL, M, N, M), ref)
    print("native vs ozaki normwise errors:", errs)
    assert errs["i8_s8"] <= errs["native"] * 4
    assert errs["f16_s7"] <= errs["native"] * 4
    nmod, _ = crt_plan_rows(K)
    assert errs[f"tc.crt_m{nmod}"] <= errs["native"]


# ---------------------------------------------------------------- ZGEMM --
# 3M in modular arithmetic: Re = Ar Br - Ai Bi and Im = (Ar+Ai)(Br+Bi) - Ar Br
# - Ai Bi are exact integers of 2K products; the only errors are the scaling
# of each complex row to integers (real and imaginary parts share the row's
# scale, planned like a real row of 2K entries) and the final roundings, so
# with the per-part rounding bounds d of row_deltas over the row's 2K reals
# (|complex error| <= sqrt(2) d) per element
#   |dC| <= |alpha| (sqrt2 da_m sum_k |b_kn| + sqrt2 db_n sum_k |a_mk| + 2K da db)
#           + 10u|C| + 4u|beta C|.

def zcrt_bound_rows(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, shift, ref, beta, C, ldc):
    Ad = op_dense(A, order, ta, M, K, lda, 0)
    Bd = op_dense(B, order, tb, K, N, ldb, 0)
    da = row_deltas(np.concatenate([Ad.real, Ad.imag], axis=1), shift)
    db = row_deltas(np.concatenate([Bd.T.real, Bd.T.imag], axis=1), shift)
    r2 = np.sqrt(2.0)
    elem = abs(alpha) * (r2 * da[:, None] * np.sum(np.abs(Bd), axis=0)[None, :] +
                         r2 * np.sum(np.abs(Ad), axis=1)[:, None] * db[None, :] +
                         2 * K * da[:, None] * db[None, :])
    out = np.linalg.norm(elem) + 10 * U * np.linalg.norm(ref)
    if beta:
        out += 4 * U * abs(beta) * np.linalg.norm(O.view_c(C, order, M, N, ldc))
    return out


ZCASES = [(O.COL, 2, 0, 200, 150, 300), (O.COL, 0, 0, 129, 77, 64), (O.ROW, 1, 2, 256, 100, 1000),
          (O.COL, 2, 1, 90, 260, 2100), (O.ROW, 0, 0, 64, 64, 33)]


@pytest.mark.parametrize("want", [0, 12, 14, 16])
def test_zgemm_crt_vs_dd_oracle(handle, want):
    rng = np.random.default_rng(700 + want)
    for order, ta, tb, M, N, K in ZCASES:
        A, lda, B, ldb, C, ldc = make_case(rng, "z", order, ta, tb, M, N, K)
        alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
        nmod, bb = crt_plan_rows(2 * K, want)
        assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, want) == 0
        try:
            dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
            rc = hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb,
                             beta, dC, ldc)
            assert rc == 0
            assert hb.device_error(handle) == 0
            path = hb.hcblasGetLastPath(handle)
            got = dC.download()
        finally:
            hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
        assert path == f"tc.zcrt3m_m{nmod}", path
        _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
        err = np.linalg.norm(O.view_c(got, order, M, N, ldc) - ref)
        bound = zcrt_bound_rows(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, bb, ref, beta, C,
                                ldc)
        assert err <= bound, (want, nmod, bb, order, ta, tb, M, N, K, err, bound)


def test_zgemm_crt_i8_matches_f16(handle):
    """Complex CRT: int8 and binary16 residue planes give the same exact
    modular products, hence bit-identical results."""
    rng = np.random.default_rng(707)
    for order, ta, tb, M, N, K in ZCASES:
        A, lda, B, ldb, C, ldc = make_case(rng, "z", order, ta, tb, M, N, K)
        alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
        outs = []
        for i8 in (1, 0):
            assert hb.set_tuning(handle, "crt_i8", i8) == 0
            assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 0) == 0
            try:
                dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
                assert hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB,
                                   ldb, beta, dC, ldc) == 0
                assert hb.device_error(handle) == 0
                outs.append(dC.download())
            finally:
                hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
                hb.set_tuning(handle, "crt_i8", 1)
        assert np.array_equal(outs[0], outs[1]), (order, ta, tb, M, N, K)


@pytest.mark.parametrize("kind,order,ta,tb,M,N,K", [("d", O.COL, 0, 1, 1001, 3000, 40),
                                                    ("d", O.ROW, 1, 0, 700, 2600, 24),
                                                    ("z", O.COL, 2, 0, 520, 1500, 24)])
def test_crt_combine_many_tiles_per_block(handle, kind, order, ta, tb, M, N, K):
    """Thousands of output tiles: every combine block walks several tiles, so
    each stage of its shared-memory ring is refilled (and the last row tile is
    partial)."""
    rng = np.random.default_rng(31 + M)
    A, lda, B, ldb, C, ldc = make_case(rng, kind, order, ta, tb, M, N, K)
    alpha, beta = ((1.5, -0.25) if kind == "d" else ((1 + 0.5j), (0.5 - 0.25j)))
    if kind == "d":
        nmod, bb = crt_plan_rows(K, 0)
    else:
        nmod, bb = crt_plan_rows(2 * K, 0)
    assert hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_OZAKI_CRT, 0) == 0
    try:
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        assert hb.lib_gemm(handle, order, TCH[ta], TCH[tb], M, N, K, alpha, dA, lda, dB, ldb,
                           beta, dC, ldc) == 0
        assert hb.device_error(handle) == 0
        got = dC.download()
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    _, ref = O.gemm(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc)
    err = np.linalg.norm(O.view_c(got, order, M, N, ldc) - ref)
    bound_fn = crt_bound_rows if kind == "d" else zcrt_bound_rows
    bound = bound_fn(order, ta, tb, M, N, K, alpha, A, lda, B, ldb, bb, ref, beta, C, ldc)
    assert err <= bound, (kind, nmod, bb, err, bound)


def test_zgemm_crt_vs_native_accuracy(handle):
    """Complex config (conj-transposed A, N(0,1) parts): the CRT ZGEMM at full
    width is no less accurate than the native FP64 kernel."""
    rng = np.random.default_rng(4)
    M = N = K = 512
    A = (rng.standard_normal(M * K) + 1j * rng.standard_normal(M * K))
    B = (rng.standard_normal(K * N) + 1j * rng.standard_normal(K * N))
    C = (rng.standard_normal(M * N) + 1j * rng.standard_normal(M * N))
    alpha, beta = (1 + 0.5j), (0.5 - 0.25j)
    _, ref = O.gemm(O.COL, 2, 0, M, N, K, alpha, A, K, B, K, beta, C, M)
    errs = {}
    for mode in (hb.HCBLAS_MATH_NATIVE, hb.HCBLAS_MATH_OZAKI_CRT):
        hb.hcblasSetMathMode(handle, mode, 0)
        dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
        assert hb.lib_gemm(handle, O.COL, "c", "n", M, N, K, alpha, dA, K, dB, K, beta, dC, M) == 0
        errs[hb.hcblasGetLastPath(handle)] = O.normwise_rel_error(
            O.view_c(dC.download(), O.COL, M, N, M), ref)
    hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    print("zgemm native vs crt:", errs)
    native = [v for k, v in errs.items() if k.startswith(("simt", "dmma"))][0]
    crt = [v for k, v in errs.items() if k.startswith("tc.zcrt")][0]
    assert crt <= native


@pytest.mark.parametrize("kind,mode,param,prefix", [("d", hb.HCBLAS_MATH_OZAKI_CRT, 0, "tc.crt_m"),
                                                    ("z", hb.HCBLAS_MATH_OZAKI_CRT, 0, "tc.zcrt3m_m"),
                                                    ("s", hb.HCBLAS_MATH_SPLIT_BF16, 6, "tc.s.grouped_split_bf16x6"),
                                                    ("c", hb.HCBLAS_MATH_SPLIT_BF16, 6, "tc.csplit3m_bf16x6")])
def test_strided_batch_uses_emulated_mode(handle, kind, mode, param, prefix):
    """A strided batch under an emulated math mode runs every element on the
    emulated path (element-wise bound of that path, checked against the
    oracle per element)."""
    from tests.test_gemm_gpu import NP, rand_op
    rng = np.random.default_rng(61)
    M, N, K, batch = 96, 80, 200, 4
    sA, sB, sC = M * K + 8, K * N + 8, M * N + 8
    A, B, C = (rand_op(rng, kind, n * batch) for n in (sA, sB, sC))
    dA, dB, dC = (hb.DeviceArray(handle, X) for X in (A, B, C))
    assert hb.hcblasSetMathMode(handle, mode, param) == 0
    try:
        alpha = (1 + 0.5j) if kind in "cz" else 1.5
        s = hb.gemm_strided_batched(handle, 0, 0, M, N, K, alpha, dA, M, sA, dB, K, sB, 0.0, dC,
                                    M, sC, batch)
        assert s == hb.HCBLAS_STATUS_SUCCESS
        assert hb.device_error(handle) == 0
        assert hb.hcblasGetLastPath(handle).startswith(prefix), hb.hcblasGetLastPath(handle)
    finally:
        hb.hcblasSetMathMode(handle, hb.HCBLAS_MATH_NATIVE, 0)
    got = dC.download()
    tol = {"d": 1e-15, "z": 1e-15, "s": 2e-6, "c": 2e-6}[kind]
    for i in range(batch):
        _, ref = O.gemm(O.COL, 0, 0, M, N, K, alpha, A[i * sA:(i + 1) * sA], M,
                        B[i * sB:(i + 1) * sB], K, 0.0, C[i * sC:(i + 1) * sC], M)
        gv = O.view_c(got[i * sC:(i + 1) * sC], O.COL, M, N, M)
        assert O.normwise_rel_error(gv, ref) < tol, i
