"""The oracle's tree query (oracle_client_tree_query, restating
src/tree_query.cpp:142-196 with the seeded client) against the reference's
own make_tree_query digests in golden_tree.json and golden_tree_c4.json
(made by the reference's tree layer under each parameter set,
tests/golden/make_golden.py --tree [--c4]). Host-only."""
import hashlib

import numpy as np
import pytest

from onionpirv2_b200 import PirParams
from onionpirv2_b200 import tree as T
from oracle import oracle as O
from tests import golden_cases as G

CASES = G.cases_tree()


@pytest.mark.parametrize("c", CASES, ids=lambda c: c["name"])
def test_tree_query_matches_reference(c):
    scheme = PirParams()
    tree = T.make_tree_pir_params_for_scheme(c["L"], c["a"], scheme)
    assert (tree.N0, tree.b, tree.r, tree.h_q, tree.w) == (c["N0"], c["b"], c["r"], c["h_q"], c["w"])
    coords = T.client_index(c["leaf"], tree)
    assert coords.alpha == c["alpha"]
    cl = O.Client(O.params(scheme.target_num_pt, scheme.expansion_height), c["client_seed"])
    cl.bv_keys(), cl.gsw_key()
    q = cl.tree_query(tree.N0, tree.h_q, coords.alpha, coords.beta_bits_le, coords.gamma_bits_le)
    assert hashlib.sha256(q.tobytes()).hexdigest() == c["sha256_query_u64"]


C4_CASES = G.cases_tree_c4()


@pytest.mark.parametrize("c", C4_CASES, ids=lambda c: c["name"])
def test_c4_tree_query_matches_reference(c):
    scheme = PirParams(config="CONFIG_N4096_K2_MP")
    tree = T.make_tree_pir_params_for_scheme(c["L"], c["a"], scheme)
    assert (tree.N0, tree.b, tree.r, tree.h_q, tree.w) == (c["N0"], c["b"], c["r"], c["h_q"], c["w"])
    coords = T.client_index(c["leaf"], tree)
    assert coords.alpha == c["alpha"]
    cl = O.C4Client(O.c4_params(scheme.target_num_pt, scheme.expansion_height), c["client_seed"])
    q = cl.tree_query(tree.N0, tree.h_q, coords.alpha, coords.beta_bits_le, coords.gamma_bits_le)
    assert hashlib.sha256(q.tobytes()).hexdigest() == c["sha256_query_u64"]
