"""The issue-rate probes behind the native kernels' fractions (hcbk_peak_probe):
each reports a rate within a wide band around the B200's nominal figures
(FP32 ~75, FP64 ~37 TFLOP/s), so a probe that stopped doing its work, or one
folded away by the compiler, is caught."""
import pytest

import hcblas_b200 as hb

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,lo,hi", [(0, 20.0, 200.0), (1, 8.0, 100.0), (2, 8.0, 100.0)])
def test_peak_probe_rates(kind, lo, hi):
    v = hb.peak_probe(kind, 5000)
    assert v is not None and lo < v < hi, (kind, v)


def test_peak_probe_rejects_bad_kind():
    assert hb.peak_probe(7) is None
