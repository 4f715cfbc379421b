"""The emulated modes' planner (hcblasPlanEmulation), without a GPU.

The planner chooses the count (CRT moduli, Ozaki slices, split-BF16 terms)
from a requested accuracy in bits; its model is restated here independently
from the CRT plan (the moduli's bit widths and the norm-scaling headroom) and
the Ozaki-I worst-case formula, and the counts it returns are checked to be
the smallest whose model reaches the target.
"""
import math

import numpy as np
import pytest

import hcblas_b200 as hb

CRT, OZ8, OZ16, SPLIT = (hb.HCBLAS_MATH_OZAKI_CRT, hb.HCBLAS_MATH_OZAKI_INT8,
                         hb.HCBLAS_MATH_OZAKI_F16, hb.HCBLAS_MATH_SPLIT_BF16)
MODULI = [255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193, 191, 181,
          179, 173, 167]


def crt_model_bits(k, n):
    """nb of the norm-scaled plan with n moduli (inf for the full plan):
    prod p >= 2 * 2^0.01 * (2^nb + 3/4 sqrt(k))^2, full when
    prod p >= 2^(2*53+1) * 2^ceil(log2 k) * 2^0.01."""
    cum = sum(math.log2(p) for p in MODULI[:n])
    lk = math.ceil(math.log2(max(k, 2)))
    if cum >= 2 * 53 + 1 + lk + 0.01:
        return math.inf
    nb = math.floor((cum - 1.02) / 2)
    while nb > 0 and 2 * math.log2(2.0 ** nb + 0.75 * math.sqrt(k)) + 0.01 >= cum - 1.0:
        nb -= 1
    return nb if nb >= 8 else 0


def ozaki_model_bits(b, s, k):
    return b * s - math.log2(1.33 * math.sqrt(k * (s - 1)) + 1.63)


@pytest.mark.parametrize("k", [64, 1000, 4096, 8192, 65536])
def test_crt_native_target_is_14_moduli(k):
    s, count, mb = hb.plan_emulation(CRT, 0, hb.HCBLAS_ACCURACY_NATIVE, "d", k)
    assert s == 0 and count == 14 and mb == crt_model_bits(k, 14) >= 53
    s, count, _ = hb.plan_emulation(CRT, 0, 53, "d", k)
    assert count == 14
    s, count, _ = hb.plan_emulation(CRT, 0, hb.HCBLAS_ACCURACY_NATIVE, "z", k // 2 or 1)
    assert count == 14  # complex rows are planned over 2K reals


@pytest.mark.parametrize("k", [256, 4096, 8192])
@pytest.mark.parametrize("bits", [30, 40, 45, 50, 53])
def test_crt_count_is_smallest_reaching_target(k, bits):
    s, count, mb = hb.plan_emulation(CRT, 0, bits, "d", k)
    assert s == 0
    assert crt_model_bits(k, count) >= bits and mb == crt_model_bits(k, count)
    assert count == 8 or crt_model_bits(k, count - 1) < bits


def test_crt_default_keeps_full_width():
    """Accuracy target 0 (the default) keeps the legacy plan: the fewest
    moduli whose product covers rows scaled to their maximum (exact
    integers, model bits infinite)."""
    for k, want in ((1024, 15), (4096, 16), (8192, 16)):
        s, count, mb = hb.plan_emulation(CRT, 0, 0, "d", k)
        assert count == want and math.isinf(mb)
    # an explicit count wins over any target
    assert hb.plan_emulation(CRT, 12, 53, "d", 4096)[1] == 12


@pytest.mark.parametrize("k", [256, 4096, 8192])
def test_ozaki_counts(k):
    for bits in (20, 30, 40, 45):
        s, count, mb = hb.plan_emulation(OZ8, 0, bits, "d", k)
        assert abs(mb - ozaki_model_bits(7, count, k)) < 1e-9
        if count < 8:
            assert mb >= bits
        if count > 3:
            assert ozaki_model_bits(7, count - 1, k) < bits
    # native FP64 is out of reach of 7-bit slices in the worst case: the
    # largest count, with its model bits reported below the target
    s, count, mb = hb.plan_emulation(OZ8, 0, -1, "d", k)
    assert count == 8 and mb < 53
    # S defaults to 4 slices; its native target (24 bits) takes 5
    assert hb.plan_emulation(OZ8, 0, 0, "s", k)[1] == 4
    assert hb.plan_emulation(OZ8, 0, -1, "s", k)[1] == 5
    s, count, mb = hb.plan_emulation(OZ16, 0, 40, "d", k)
    assert abs(mb - ozaki_model_bits(8, count, k)) < 1e-9


def test_split_terms():
    for dt in "sc":
        assert hb.plan_emulation(SPLIT, 0, 0, dt, 4096)[1:] == (3, 15.0)
        assert hb.plan_emulation(SPLIT, 0, 15, dt, 4096)[1] == 3
        assert hb.plan_emulation(SPLIT, 0, -1, dt, 4096)[1:] == (6, 24.0)
        assert hb.plan_emulation(SPLIT, 6, 0, dt, 4096)[1] == 6


def test_status_rules():
    bad = hb.HCBLAS_STATUS_INVALID_VALUE
    assert hb.plan_emulation(CRT, 0, -1, "s", 4096)[0] == bad   # CRT does not emulate S
    assert hb.plan_emulation(SPLIT, 0, -1, "d", 4096)[0] == bad
    assert hb.plan_emulation(hb.HCBLAS_MATH_NATIVE, 0, -1, "d", 4096)[0] == bad
    assert hb.plan_emulation(CRT, 0, -2, "d", 4096)[0] == bad
    assert hb.plan_emulation(CRT, 0, 65, "d", 4096)[0] == bad
    assert hb.plan_emulation(CRT, 0, 53, "d", 0)[0] == bad
    assert hb.hcblasSetAccuracyTarget(None, 53) == hb.HCBLAS_STATUS_NOT_INITIALIZED
