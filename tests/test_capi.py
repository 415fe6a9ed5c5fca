"""C-ABI library: loads, exports every declared symbol, derives the
reference's parameters and serializes responses -- all host-only calls."""
import ctypes as C

import numpy as np
import pytest

from onionpirv2_b200 import _lib as L
from onionpirv2_b200 import PirParams, save_response
from oracle import oracle as O
from tests import golden_cases as G


def test_library_exports_every_header_symbol():
    lib = C.CDLL(L.LIB_PATH)
    syms = L.header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert L.load().opir_version().startswith(b"onionpir_b200")


@pytest.mark.parametrize("case", G.cases(), ids=lambda c: c["name"])
def test_params_match_reference_layouts(case):
    p = PirParams(case["target_num_pt"], case["expansion_height"], case["fst_dim_pow2"])
    for k in ("num_pt", "fst_dim_sz", "num_dims", "other_dim_sz", "q", "q1", "q2", "w1", "w2", "small_q"):
        assert getattr(p, k) == case[k], k
    assert p.plain_mod == case["t"]
    o = O.params(case["target_num_pt"], case["expansion_height"], case["fst_dim_pow2"])
    assert p.w_crt == o.w_crt and p.q1_inv_mod_q2 == o.q1_inv_mod_q2
    assert (p.base_log2, p.base_log2_key, p.base_log2_ks) == (o.base_ep, o.base_key, o.base_ks)
    assert p.response_bytes() == case["resp_bytes"]


def test_invalid_layouts_raise_like_the_reference():
    with pytest.raises(ValueError):
        PirParams(0, 0)          # pir.cpp:101-103
    with pytest.raises(ValueError):
        PirParams(100, 12)       # pir.cpp:105-111 (beyond log2 N)


def test_save_response_matches_oracle_codec():
    p = PirParams(16384, 9)
    o = O.params(16384, 9)
    rng = np.random.default_rng(3)
    for _ in range(5):
        r = rng.integers(0, p.small_q, (2, p.N), dtype=np.uint64)
        assert save_response(p, r) == O.serialize(o, r)
    c = G.case("c1_16384_h9")
    assert len(save_response(p, np.zeros((2, p.N), np.uint64))) == c["resp_bytes"]
