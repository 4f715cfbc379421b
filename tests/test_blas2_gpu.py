"""GEMV and GER (hcblas{S,D}gemv[Batched], hcblas{S,D}ger[Batched]) against
the CPU oracle, as the GEMM special cases they are (GEMV = GEMM with one
column, GER = GEMM with K = 1, beta = 1).  Tolerance: the GEMM normwise bound
gamma_{K+2} || |alpha||op(A)||x| + |beta||y| || (K = inner length; 1 for GER)."""
import numpy as np
import pytest

import hcblas_b200 as hb
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NP = {"s": np.float32, "d": np.float64}
U = {"s": 2.0 ** -24, "d": 2.0 ** -53}


def gam(kind, K):
    u = U[kind]
    return (K + 2) * u / (1 - (K + 2) * u)


def strided(v, n, inc):
    return v[: (n - 1) * inc + 1: inc] if n > 0 else v[:0]


@pytest.mark.parametrize("kind", "sd")
@pytest.mark.parametrize("trans", [0, 1])
@pytest.mark.parametrize("pad", [0, 5])  # pad 0 with m % 4 == 0: the 16-byte vector kernels
@pytest.mark.parametrize("m,n,incx,incy", [(300, 200, 1, 1), (257, 513, 3, 2), (1, 5000, 1, 1),
                                           (70000, 3, 1, 4), (5000, 1, 2, 1), (4100, 4100, 1, 1),
                                           (8192, 96, 1, 1)])
def test_gemv_vs_oracle(handle, kind, trans, pad, m, n, incx, incy):
    rng = np.random.default_rng(m + 7 * n + trans + pad)
    dt = NP[kind]
    lda = m + pad
    A = rng.uniform(-1, 1, lda * n).astype(dt)
    lx, ly = (n, m) if trans == 0 else (m, n)
    x = rng.uniform(-1, 1, (lx - 1) * incx + 1).astype(dt)
    y = rng.uniform(-1, 1, (ly - 1) * incy + 1).astype(dt)
    alpha, beta = 1.25, -0.5
    dA, dx, dy = (hb.DeviceArray(handle, v) for v in (A, x, y))
    assert hb.gemv(handle, trans, m, n, alpha, dA, lda, dx, incx, beta, dy, incy) == 0
    got = strided(dy.download(), ly, incy).astype(np.float64)
    xc = np.ascontiguousarray(strided(x, lx, incx))
    yc = np.ascontiguousarray(strided(y, ly, incy))
    _, ref = O.gemm(O.COL, trans, 0, ly, 1, lx, alpha, A, lda, xc, lx, beta, yc, ly)
    Ad = np.abs(A.reshape(n, lda)[:, :m].T.astype(np.float64))
    opA = Ad if trans == 0 else Ad.T
    bound = gam(kind, lx) * np.linalg.norm(abs(alpha) * opA @ np.abs(xc) + abs(beta) * np.abs(yc))
    assert np.linalg.norm(got - ref[:, 0]) <= bound
    # untouched gaps between strided elements of y
    if incy > 1:
        full = dy.download()
        mask = np.ones(full.size, bool)
        mask[::incy] = False
        assert np.array_equal(full[mask], y[mask])


@pytest.mark.parametrize("kind", "sd")
def test_gemv_special_scalars(handle, kind):
    rng = np.random.default_rng(5)
    dt = NP[kind]
    m, n = 129, 77
    A = rng.uniform(-1, 1, m * n).astype(dt)
    x = rng.uniform(-1, 1, n).astype(dt)
    y = np.full(m, np.nan, dtype=dt)  # beta == 0: y is not read
    dA, dx, dy = (hb.DeviceArray(handle, v) for v in (A, x, y))
    assert hb.gemv(handle, 0, m, n, 1.0, dA, m, dx, 1, 0.0, dy, 1) == 0
    assert np.all(np.isfinite(dy.download()))
    y2 = rng.uniform(-1, 1, m).astype(dt)
    dy.upload(y2)
    A[3] = np.nan  # alpha == 0: A and x are not read
    dA.upload(A)
    assert hb.gemv(handle, 0, m, n, 0.0, dA, m, dx, 1, 2.0, dy, 1) == 0
    assert np.array_equal(dy.download(), (2 * y2.astype(np.float64)).astype(dt))


@pytest.mark.parametrize("kind", "sd")
def test_gemv_batched_reference_offsets(handle, kind):
    """Batch b reads A at b*m*n, x at b*len(x), y at b*len(y) (the
    reference's implicit offsets)."""
    rng = np.random.default_rng(9)
    dt = NP[kind]
    m, n, batch = 90, 60, 4
    for trans in (0, 1):
        lx, ly = (n, m) if trans == 0 else (m, n)
        A = rng.uniform(-1, 1, m * n * batch).astype(dt)
        x = rng.uniform(-1, 1, lx * batch).astype(dt)
        y = rng.uniform(-1, 1, ly * batch).astype(dt)
        dA, dx, dy = (hb.DeviceArray(handle, v) for v in (A, x, y))
        assert hb.gemv(handle, trans, m, n, 0.5, dA, m, dx, 1, 1.5, dy, 1, batch=batch) == 0
        got = dy.download().astype(np.float64)
        for b in range(batch):
            _, ref = O.gemm(O.COL, trans, 0, ly, 1, lx, 0.5, A[b * m * n:(b + 1) * m * n], m,
                            x[b * lx:(b + 1) * lx], lx, 1.5, y[b * ly:(b + 1) * ly], ly)
            assert np.allclose(got[b * ly:(b + 1) * ly], ref[:, 0], rtol=0,
                               atol=50 * gam(kind, lx) * (lx + ly))


@pytest.mark.parametrize("kind", "sd")
@pytest.mark.parametrize("m,pad", [(333, 3), (336, 4)])  # (336, 4): the 16-byte vector kernel
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 3), (-1, 2), (3, -2)])
def test_ger_vs_oracle(handle, kind, m, pad, incx, incy):
    rng = np.random.default_rng(20 + incx * 3 + incy + m)
    dt = NP[kind]
    n = 210
    lda = m + pad
    A = rng.uniform(-1, 1, lda * n).astype(dt)
    x = rng.uniform(-1, 1, (m - 1) * abs(incx) + 1).astype(dt)
    y = rng.uniform(-1, 1, (n - 1) * abs(incy) + 1).astype(dt)
    dA, dx, dy = (hb.DeviceArray(handle, v) for v in (A, x, y))
    assert hb.ger(handle, m, n, 0.75, dx, incx, dy, incy, dA, lda) == 0
    # BLAS order: element i of a negatively strided vector is v[(len-1-i)*|inc|]
    xl = strided(x, m, abs(incx))[:: (1 if incx > 0 else -1)]
    yl = strided(y, n, abs(incy))[:: (1 if incy > 0 else -1)]
    _, ref = O.gemm(O.COL, 0, 1, m, n, 1, 0.75, np.ascontiguousarray(xl), m,
                    np.ascontiguousarray(yl), n, 1.0, A, lda)
    got = O.view_c(dA.download(), O.COL, m, n, lda).astype(np.float64)
    mag = 0.75 * np.abs(np.outer(xl, yl)) + np.abs(O.view_c(A, O.COL, m, n, lda))
    assert np.linalg.norm(got - ref) <= gam(kind, 1) * np.linalg.norm(mag)
    pad = dA.download().reshape(n, lda)[:, m:]
    assert np.array_equal(pad, A.reshape(n, lda)[:, m:])


@pytest.mark.parametrize("kind", "sd")
def test_ger_batched_and_alpha_zero(handle, kind):
    rng = np.random.default_rng(30)
    dt = NP[kind]
    m, n, batch = 64, 48, 3
    A = rng.uniform(-1, 1, m * n * batch).astype(dt)
    x = rng.uniform(-1, 1, m * batch).astype(dt)
    y = rng.uniform(-1, 1, n * batch).astype(dt)
    dA, dx, dy = (hb.DeviceArray(handle, v) for v in (A, x, y))
    assert hb.ger(handle, m, n, 0.0, dx, 1, dy, 1, dA, m, batch=batch) == 0
    assert np.array_equal(dA.download(), A)
    assert hb.ger(handle, m, n, 2.0, dx, 1, dy, 1, dA, m, batch=batch) == 0
    got = dA.download().astype(np.float64)
    for b in range(batch):
        Ab = A[b * m * n:(b + 1) * m * n].astype(np.float64).reshape(n, m).T
        want = Ab + 2.0 * np.outer(x[b * m:(b + 1) * m], y[b * n:(b + 1) * n])
        gv = got[b * m * n:(b + 1) * m * n].reshape(n, m).T
        assert np.allclose(gv, want, rtol=0, atol=8 * U[kind])


def test_blas2_status_rules(handle):
    d = hb.DeviceArray(handle, np.zeros(64, np.float32))
    assert hb.gemv(handle, 0, -1, 4, 1.0, d, 4, d, 1, 0.0, d, 1) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert hb.gemv(handle, 0, 4, 4, 1.0, d, 4, d, 0, 0.0, d, 1) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert hb.gemv(handle, 0, 0, 4, 1.0, d, 4, d, 1, 0.0, d, 1) == hb.HCBLAS_STATUS_EXECUTION_FAILED
    assert hb.gemv(handle, 0, 4, 4, 1.0, d, 4, d, -1, 0.0, d, 1) == \
        hb.HCBLAS_STATUS_EXECUTION_FAILED
    assert hb.ger(handle, 4, -2, 1.0, d, 1, d, 1, d, 4) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert hb.ger(handle, 4, 4, 1.0, d, 1, d, 0, d, 4) == hb.HCBLAS_STATUS_INVALID_VALUE
    assert hb.ger(handle, 4, 0, 1.0, d, 1, d, 1, d, 4) == hb.HCBLAS_STATUS_EXECUTION_FAILED
