"""The CONFIG_N2048_K2_MP oracle (the two-limb routines of
oracle/opir_oracle_c4.c at N = 2048 with 29-bit limbs) against the reference
itself: golden_k2mp.json was produced by the unmodified reference sources
built with CONFIG_N2048_K2_MP (tests/golden/make_golden.py --k2mp). The
seeded client must reproduce the reference client's keys and query, and the
server restatement every public stage, the response and its 22-bit
serialization; the client must decrypt the requested plaintext."""
import hashlib

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G

CASES = [c["name"] for c in G.cases_set("k2mp")]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_k2mp_oracle_matches_reference(name):
    c = G.case_set("k2mp", name)
    p = O.k2mp_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    assert [p.q[0], p.q[1]] == c["q_limbs"]
    assert (p.t, p.small_q, p.fst_dim_sz, p.num_dims, p.other_dim_sz) == (
        c["t"], c["small_q"], c["fst_dim_sz"], c["num_dims"], c["other_dim_sz"])
    assert (p.base_ep, p.base_key) == (c["base_log2"], c["base_log2_key"])
    cl = O.C4Client(p, c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    q = cl.query(c["index"])
    assert sha(bv) == c["sha256_bv_keys_u64"]
    assert sha(gsw) == c["sha256_gsw_key_u64"]
    assert sha(q) == c["sha256_query_u64"]
    s = O.C4Server(p)
    s.load_seeded(c["target_num_pt"], c["db_seed"])
    s.set_keys(bv, gsw)
    exp = s.expand(q)
    assert sha(exp) == c["sha256_stage_expand"]
    sel = s.complete_selectors(exp)
    assert sha(sel) == c["sha256_stage_selectors"]
    mid = s.first_dim(exp)
    assert sha(mid) == c["sha256_stage_first_dim"]
    assert sha(s.other_dim(mid, sel)) == c["sha256_stage_other_dim"]
    resp = s.make_query(q)
    assert sha(resp) == c["sha256_response_u64"]
    assert O.c4_serialize(p, resp) == G.stream(c)
    want = (O.c4_db_plaintext(c["db_seed"], c["index"], p) if c["index"] < c["target_num_pt"]
            else np.zeros(p.N, np.uint64))
    assert np.array_equal(cl.decrypt(resp), want)
