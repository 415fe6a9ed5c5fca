"""The register-resident rate probes behind the rooflines: the butterfly
rate of the NTT-bound stages (opir_measure_butterfly_rate) and the
recombination rate of a byte-sliced tensor-core product's epilogue
(opir_measure_recombine_rate). Positive, repeatable, ordered as their work
is (64-bit butterflies slower than 32-bit ones; seven shift classes slower
than five), and unknown arguments refused."""
import ctypes as C

import pytest

from onionpirv2_b200 import _lib as L
from onionpirv2_b200.server import measure_butterfly_rate, measure_recombine_rate

pytestmark = pytest.mark.gpu


def test_butterfly_rate_is_plausible():
    k1 = [measure_butterfly_rate("CONFIG_N2048_K1_COMP") for _ in range(2)]
    c4 = measure_butterfly_rate("CONFIG_N4096_K2_MP")
    for r in k1 + [c4]:
        assert 1e11 < r < 1e14           # butterflies per second on one GPU
    assert abs(k1[0] - k1[1]) / k1[0] < 0.2
    assert c4 < k1[0]


def test_butterfly_rate_rejects_unknown_config():
    out = C.c_double()
    assert L.load().opir_measure_butterfly_rate(7, 0, C.byref(out)) != 0


def test_recombine_rate_is_plausible():
    r7 = [measure_recombine_rate(7) for _ in range(2)]
    r5 = measure_recombine_rate(5)
    for r in r7 + [r5]:
        assert 1e10 < r < 1e14           # outputs per second on one GPU
    assert abs(r7[0] - r7[1]) / r7[0] < 0.2
    assert r5 > r7[0]


def test_recombine_rate_rejects_other_class_counts():
    out = C.c_double()
    for classes in (0, 6, 8):
        assert L.load().opir_measure_recombine_rate(classes, 0, C.byref(out)) != 0
