"""The CPU oracle (oracle/opir_oracle.c) against the reference's own outputs.

The fixtures were produced by the reference server and client code itself
(tests/golden/make_golden.py); the oracle must reproduce the client material
(query, BV keys, RGSW key) and the response bit for bit, and the response
must decrypt to the requested plaintext.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G

FAST = [c["name"] for c in G.cases() if c["num_pt"] <= 20000]
FULL = [c["name"] for c in G.cases() if c["num_pt"] > 20000]


def _run(name):
    c = G.case(name)
    p = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    for k in ("num_pt", "fst_dim_sz", "num_dims", "other_dim_sz", "q", "q1", "q2", "w1", "w2", "t", "small_q"):
        assert getattr(p, k) == c[k], k
    cl = O.Client(p, c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    q = cl.query(c["index"])
    assert G.sha256(q) == c["sha256_query_u64"]
    assert G.sha256(gsw) == c["sha256_gsw_key_u64"]
    if p.expansion_height:
        assert G.sha256(bv) == c["sha256_bv_keys_u64"]
    s = O.Server(p)
    s.load_seeded(c["target_num_pt"], c["db_seed"])
    s.set_keys(bv, gsw)
    r = s.make_query(q)
    assert G.sha256(r) == c["sha256_response_u64"]
    assert O.serialize(p, r) == G.stream(c)
    want = O.db_plaintext(c["db_seed"], c["index"], p) if c["index"] < c["target_num_pt"] else np.zeros(p.N)
    assert np.array_equal(cl.decrypt(r), want)


@pytest.mark.parametrize("name", FAST)
def test_oracle_matches_reference(name):
    _run(name)


@pytest.mark.slow
@pytest.mark.parametrize("name", FULL)
def test_oracle_matches_reference_full_size(name):
    _run(name)
