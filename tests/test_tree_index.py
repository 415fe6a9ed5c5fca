"""Tree PIR index math (the library's C++ restatement of src/tree_index.cpp
and src/tree_query.cpp:42-68, through the C ABI), checked the way the
reference's own src/tests/test_tree_index.cpp checks it: every (leaf, level)
pair of its sanity configurations against a direct tree walk, the plan
boundaries, the hard validation gates and the scheme binding. Host-only."""
import pytest

from onionpirv2_b200 import PirParams
from onionpirv2_b200 import tree as T

MODS = [577]


def exhaust(params):
    plans = T.build_level_plans(params)
    assert len(plans) == params.L + 1
    for leaf in range(params.N):
        c = T.client_index(leaf, params)
        gamma = leaf // params.P
        beta = (leaf % params.P) % params.B
        assert sum(bit << u for u, bit in enumerate(c.beta_bits_le)) == beta
        assert sum(bit << v for v, bit in enumerate(c.gamma_bits_le)) == gamma
        assert gamma * params.P + c.alpha * params.B + beta == leaf
        for level in range(params.L + 1):
            node, p_l, gamma_l = T.level_oracle(leaf, level, params)
            plan = plans[level]
            assert node == leaf >> (params.L - level)
            assert node == gamma_l * plan.R + p_l          # invariant 1
            assert p_l < plan.R
            if level >= params.r:
                assert gamma_l == gamma
                assert T.level_record_position_from_coordinates(c.alpha, beta, level,
                                                                params) == p_l
            else:
                assert p_l == 0 and gamma_l == gamma >> (params.r - level)


def check_plans(params):
    for level, plan in enumerate(T.build_level_plans(params)):
        assert plan.level == level
        assert plan.R == (1 << (level - params.r) if level >= params.r else 1)
        if plan.R == 1:
            assert plan.select_case == T.SINGLE and plan.coarsen_count == params.a
            assert plan.beta_count == 0 and plan.beta_begin == params.b
        elif plan.R < params.N0:
            assert plan.select_case == T.COARSENED_ALPHA
            assert plan.coarsen_count == params.a - (level - params.r)
            assert plan.beta_count == 0 and plan.beta_begin == params.b
        else:
            assert plan.select_case == T.ALPHA_BETA
            assert plan.beta_begin == params.L - level
            assert plan.beta_count == level - params.r - params.a
            assert plan.beta_begin + plan.beta_count == params.b
        if level >= params.r:
            assert (plan.gamma_begin, plan.gamma_count) == (0, params.r)
        else:
            assert (plan.gamma_begin, plan.gamma_count) == (params.r - level, level)
        assert plan.projection_depth == min(level, params.r)


@pytest.mark.parametrize("shape", [(6, 1, 8), (7, 1, 8), (8, 2, 16), (5, 2, 8)])
def test_sanity_configurations(shape):
    L, a, n = shape
    p = T.make_tree_pir_params(L, a, n, 1, 1, 17, MODS)
    exhaust(p)
    check_plans(p)


@pytest.mark.parametrize("args", [
    (4, 2, 8, 1, 1, 17, MODS),                 # L below r + a
    (6, 0, 8, 1, 1, 17, MODS),                 # N0 = 1
    (6, 1, 6, 1, 1, 17, MODS),                 # non-power-of-two ring
    (0, 1, 8, 1, 1, 17, MODS),                 # zero height
    (6, 64, 8, 1, 1, 17, MODS),                # first dimension out of range
    (6, 1, 8, 4, 4, 17, MODS),                 # W above the ring degree
    (19, 3, 2048, 1 << 60, 1 << 60, 17, MODS), # wrapping packed width
    (6, 1, 8, 1, 1, 16, MODS),                 # even plaintext modulus
    (6, 1, 8, 1, 1, 17, [578]),                # even RNS modulus
])
def test_validation_gates(args):
    with pytest.raises(ValueError):
        T.make_tree_pir_params(*args)


def test_out_of_range_leaf():
    with pytest.raises(ValueError):
        T.client_index(64, T.make_tree_pir_params(6, 1, 8, 1, 1, 17, MODS))


def test_scheme_binding():
    scheme = PirParams()
    bound = T.make_tree_pir_params_for_scheme(16, 3, scheme)
    assert bound.n == scheme.N and bound.r == 11
    assert bound.ell_beta == bound.ell_gamma == scheme.l_ep
    assert (bound.N0, bound.B, bound.b) == (8, 4, 2)
    assert (bound.w, bound.W, bound.h_q) == (86, 128, 7)      # L_EP = 6 anchor
    with pytest.raises(ValueError):   # h_q beyond the scheme's session keys
        T.make_tree_pir_params_for_scheme(bound.r + 10, 10, scheme)
    exhaust(T.make_tree_pir_params(13, 1, 2048, scheme.l_ep, scheme.l_ep, scheme.plain_mod,
                                   [scheme.q]))
    qp = T.tree_query_expansion_params(bound, scheme)
    assert (qp.fst_dim_sz, qp.num_dims, qp.expansion_height, qp.num_pt) == (8, 14, 7, 8)
    assert qp.view == 1


def test_query_shape_gates():
    scheme = PirParams()
    qp = scheme.with_query_shape(8, 2, 7)
    assert (qp.fst_dim_sz, qp.num_dims, qp.other_dim_sz, qp.num_pt) == (8, 3, 1, 8)
    for bad in ((8, 2, 12), (0, 1, 7), (256, 0, 7), (8, 21, 7)):
        with pytest.raises(ValueError):
            scheme.with_query_shape(*bad)


def test_synthetic_node_source_and_packing():
    p = T.make_tree_pir_params(6, 1, 8, 1, 1, 17, MODS)
    assert all(0 <= T.synthetic_tree_node_value(l, i, 17) < 17 for l in range(7) for i in range(8))
    src = lambda level, idx: 1000 * level + idx
    lvl5 = T.pack_tree_level(5, p, src)            # R = 4 plaintexts, 32 nodes
    assert lvl5.shape == (4, 8)
    for pp in range(4):
        for u in range(8):
            assert lvl5[pp, u] == (5000 + pp + 4 * u) % 17
    lvl1 = T.pack_tree_level(1, p, src)            # R = 1, 2 nodes then zeros
    assert list(lvl1[0]) == [1000 % 17, 1001 % 17, 0, 0, 0, 0, 0, 0]
