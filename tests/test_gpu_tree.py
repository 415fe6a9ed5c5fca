"""GPU tree PIR select_level (opir_tree_select_level) against the
reference's tree layer: for each case of golden_tree.json the oracle client's
tree query (pinned to the reference's by test_oracle_golden_tree.py) is
unpacked on a query-shape server (expand_query + complete_selectors), every
level of the synthetic tree is built as a device-resident level database,
and each level's selected ciphertext must equal the reference's
select_level output bit for bit and decrypt to its packed plaintext D_l[p_l]
(the reference's own Milestone-2 gate)."""
import functools
import hashlib

import numpy as np
import pytest

from onionpirv2_b200 import PirParams, PirServer
from onionpirv2_b200 import tree as T
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

CASES = G.cases_tree()


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@functools.lru_cache(maxsize=None)
def tree_levels(L, a):
    scheme = PirParams()
    tree = T.make_tree_pir_params_for_scheme(L, a, scheme)
    src = lambda level, idx: T.synthetic_tree_node_value(level, idx, scheme.plain_mod)
    pts = [T.pack_tree_level(level, tree, src) for level in range(L + 1)]
    levels = [T.TreeLevel(scheme, tree, level, pts[level]) for level in range(L + 1)]
    return scheme, tree, pts, levels


@pytest.mark.parametrize("c", CASES, ids=lambda c: c["name"])
def test_select_level_matches_reference(c):
    scheme, tree, pts, levels = tree_levels(c["L"], c["a"])
    cl = O.Client(O.params(scheme.target_num_pt, scheme.expansion_height), c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    coords = T.client_index(c["leaf"], tree)
    q = cl.tree_query(tree.N0, tree.h_q, coords.alpha, coords.beta_bits_le, coords.gamma_bits_le)
    qparams = T.tree_query_expansion_params(tree, scheme)
    with PirServer(qparams) as srv:
        srv.set_client_keys(1, bv[: qparams.expansion_height], gsw)
        alpha, beta, gamma = T.unpack_tree_query(srv, scheme, tree, 1, q)
    assert sha(alpha) == c["sha256_alpha_u64"]
    assert sha(beta) == c["sha256_beta_selectors_u64"]
    assert gamma.shape[0] == tree.r
    for level in range(tree.L + 1):
        out = levels[level].select_level(alpha, beta)
        assert sha(out) == c["sha256_levels_u64"][level], level
        _, p_l, _ = T.level_oracle(c["leaf"], level, tree)
        assert np.array_equal(cl.decrypt_q(out), pts[level][p_l]), level


def test_views_refuse_out_of_scope_calls():
    scheme, tree, pts, levels = tree_levels(13, 2)
    qparams = T.tree_query_expansion_params(tree, scheme)
    with PirServer(qparams) as srv:
        with pytest.raises(ValueError):
            srv.load_data_seeded(8, 1)           # no database behind a query shape
        with pytest.raises(ValueError):
            srv.make_query(1, np.zeros((2, scheme.N), np.uint64))
    lvl = levels[tree.L]
    with pytest.raises(ValueError):
        lvl.select_level(np.zeros((tree.N0 + 1, 2, scheme.N), np.uint64), None)
    bad = np.zeros((tree.N0, 2, scheme.N), np.uint64)
    bad[0, 0, 0] = scheme.q
    with pytest.raises(ValueError):
        lvl.select_level(bad, np.zeros((max(tree.b, 1), 12, 2, scheme.N), np.uint64))


@functools.lru_cache(maxsize=None)
def whole_tree(L, a):
    scheme, tree, pts, _ = tree_levels(L, a)
    return T.Tree(scheme, tree, pts)


@pytest.mark.parametrize("c", CASES, ids=lambda c: c["name"])
def test_device_resident_tree_matches_reference(c):
    """opir_tree_query: the whole path in one call, levels on their own
    streams, equal to the reference's select_level at every level."""
    scheme, tree, pts, _ = tree_levels(c["L"], c["a"])
    t = whole_tree(c["L"], c["a"])
    cl = O.Client(O.params(scheme.target_num_pt, scheme.expansion_height), c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    t.set_client_keys(c["client_seed"], bv, gsw)
    coords = T.client_index(c["leaf"], tree)
    q = cl.tree_query(tree.N0, tree.h_q, coords.alpha, coords.beta_bits_le, coords.gamma_bits_le)
    for _ in range(2):     # a repeated query gives the same answer
        out = t.query(c["client_seed"], q)
        for level in range(tree.L + 1):
            assert sha(out[level]) == c["sha256_levels_u64"][level], level


# ---------------------------------------------------------- CONFIG_N4096_K2_MP
C4 = "CONFIG_N4096_K2_MP"
C4_CASES = G.cases_tree_c4()


@functools.lru_cache(maxsize=None)
def tree_levels_c4(L, a):
    scheme = PirParams(config=C4)
    tree = T.make_tree_pir_params_for_scheme(L, a, scheme)
    src = lambda level, idx: T.synthetic_tree_node_value(level, idx, scheme.plain_mod)
    pts = [T.pack_tree_level(level, tree, src) for level in range(L + 1)]
    levels = [T.TreeLevel(scheme, tree, level, pts[level]) for level in range(L + 1)]
    return scheme, tree, pts, levels


def c4_client_query(c, scheme, tree):
    cl = O.C4Client(O.c4_params(scheme.target_num_pt, scheme.expansion_height), c["client_seed"])
    coords = T.client_index(c["leaf"], tree)
    q = cl.tree_query(tree.N0, tree.h_q, coords.alpha, coords.beta_bits_le, coords.gamma_bits_le)
    return cl, q


@pytest.mark.parametrize("c", C4_CASES, ids=lambda c: c["name"])
def test_c4_select_level_matches_reference(c):
    """The two-limb tree layer: unpack on a query-shape server and every
    level's select_level, bit for bit the reference built under
    CONFIG_N4096_K2_MP (which checked that every level decrypts)."""
    scheme, tree, pts, levels = tree_levels_c4(c["L"], c["a"])
    cl, q = c4_client_query(c, scheme, tree)
    qparams = T.tree_query_expansion_params(tree, scheme)
    with PirServer(qparams) as srv:
        srv.set_client_keys(1, cl.bv_keys()[: qparams.expansion_height], cl.gsw_key())
        alpha, beta, gamma = T.unpack_tree_query(srv, scheme, tree, 1, q)
    assert sha(alpha) == c["sha256_alpha_u64"]
    assert sha(beta) == c["sha256_beta_selectors_u64"]
    for level in range(tree.L + 1):
        out = levels[level].select_level(alpha, beta)
        assert sha(out) == c["sha256_levels_u64"][level], level


@functools.lru_cache(maxsize=None)
def whole_tree_c4(L, a):
    scheme, tree, pts, _ = tree_levels_c4(L, a)
    return T.Tree(scheme, tree, pts)


@pytest.mark.parametrize("c", C4_CASES, ids=lambda c: c["name"])
def test_c4_device_resident_tree_matches_reference(c):
    scheme, tree, pts, _ = tree_levels_c4(c["L"], c["a"])
    t = whole_tree_c4(c["L"], c["a"])
    cl, q = c4_client_query(c, scheme, tree)
    t.set_client_keys(c["client_seed"], cl.bv_keys(), cl.gsw_key())
    for _ in range(2):
        out = t.query(c["client_seed"], q)
        assert out.shape == (tree.L + 1,) + scheme.ct_shape
        for level in range(tree.L + 1):
            assert sha(out[level]) == c["sha256_levels_u64"][level], level
