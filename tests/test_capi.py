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


C4 = "CONFIG_N4096_K2_MP"


@pytest.mark.parametrize("case", G.cases_c4(), ids=lambda c: c["name"])
def test_c4_params_match_reference_layouts(case):
    p = PirParams(case["target_num_pt"], case["expansion_height"], case["fst_dim_pow2"], config=C4)
    assert (p.poly_degree, p.num_limbs, p.q) == (4096, 2, 0)
    assert p.get_rns_mods() == case["q_limbs"]
    for k in ("num_pt", "fst_dim_sz", "num_dims", "other_dim_sz", "small_q"):
        assert getattr(p, k) == case[k], k
    assert p.plain_mod == case["t"]
    assert (p.base_log2, p.base_log2_key) == (case["base_log2"], case["base_log2_key"])
    o = O.c4_params(case["target_num_pt"], case["expansion_height"], case["fst_dim_pow2"])
    assert (p.w1, p.w2, p.q1_inv_mod_q2) == (o.w[0], o.w[1], o.q0_inv_mod_q1)
    assert (p.base_log2_ks, p.l_ep, p.l_key, p.l_ks) == (o.base_ks, o.l_ep, o.l_key, o.l_ks)
    assert p.response_bytes() == case["resp_bytes"] == 51200
    assert p.ct_shape == (2, 2, 4096)
    assert p.with_layout(64, 6).config == C4


def test_c4_invalid_layouts_and_configs():
    with pytest.raises(ValueError):
        PirParams(0, 0, config=C4)
    with pytest.raises(ValueError):
        PirParams(100, 13, config=C4)   # beyond log2 N = 12
    with pytest.raises(ValueError):
        PirParams(100, 5, config="CONFIG_N8192")
    lay, out = L.Layout(100, 5, 1), L.Params()
    assert L.load().opir_params_init_config(7, C.byref(lay), C.byref(out)) == 1


def test_c4_save_response_matches_oracle_codec():
    p = PirParams(2048, 7, config=C4)
    o = O.c4_params(2048, 7)
    rng = np.random.default_rng(5)
    for _ in range(3):
        r = rng.integers(0, p.small_q, (2, p.N), dtype=np.uint64)
        assert save_response(p, r) == O.c4_serialize(o, r)


def test_c4_memory_plan_counts_the_two_limb_buffers():
    from onionpirv2_b200.server import plan_memory
    p = PirParams(1 << 20, 11, config=C4)
    m = plan_memory(p)
    # NTT-form database: 2 limbs x N levels x 2^20 plaintexts x 8 bytes
    assert m["database_bytes"] >= 2 * 4096 * (1 << 20) * 8
    # BV keys (11 levels x 8 rows) + RGSW (16 rows): 4N u64 per row and as
    # many Shoup companions
    assert m["client_key_bytes"] == (11 * 8 + 16) * 8 * 4096 * 8
    assert m["scratch_bytes_per_query"] > 2 * 1024 * 4 * 4096 * 8
