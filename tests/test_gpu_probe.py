"""The butterfly-rate probe behind the NTT stages' roofline
(opir_measure_butterfly_rate): positive, repeatable, and the 64-bit
two-limb butterfly slower than the 32-bit residue one."""
import pytest

from onionpirv2_b200.server import measure_butterfly_rate

pytestmark = pytest.mark.gpu


def test_butterfly_rate_is_plausible():
    k1 = [measure_butterfly_rate("CONFIG_N2048_K1_COMP") for _ in range(2)]
    c4 = measure_butterfly_rate("CONFIG_N4096_K2_MP")
    for r in k1 + [c4]:
        assert 1e11 < r < 1e14           # butterflies per second on one GPU
    assert abs(k1[0] - k1[1]) / k1[0] < 0.2
    assert c4 < k1[0]


def test_butterfly_rate_rejects_unknown_config():
    import ctypes as C
    from onionpirv2_b200 import _lib as L
    out = C.c_double()
    assert L.load().opir_measure_butterfly_rate(7, 0, C.byref(out)) != 0
