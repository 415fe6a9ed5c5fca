"""Known-answer tests the reference's own test suite holds, restated against
the CPU oracle: tests/test_hexl_ntt.cpp, tests/test_utils.cpp,
tests/test_runtime_layout.cpp, tests/test_bv_keyswitch.cpp:10-57,
tests/test_fst_dim.cpp:11-93 (paths relative to the reference's src/)."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O

L = O.lib()
P = O.params(16384, 9)


def test_mt19937_64_standard_value():
    # 10000th output of std::mt19937_64 with the default seed 5489.
    assert L.oracle_mt_test(5489, 9999) == 9981545732273789042


def test_constants_of_config_n2048_k1_comp():
    assert (P.q1, P.q2, P.q) == (536813569, 536752129, 288135826036838401)
    assert P.t == 4099 and P.small_q == 4169729 and P.small_q_width == 22
    assert (P.base_ep, P.base_key, P.base_ks) == (10, 6, 8)
    assert P.w_crt % P.q1 == P.w1 and P.w_crt % P.q2 == P.w2


def test_ntt_poly_product_kat():
    # test_hexl_ntt.cpp:41-58: (1+2x+3x^2)(4+5x) = 4+13x+22x^2+15x^3
    N, q, root = P.N, P.q, P.w_crt
    a = np.zeros(N, np.uint64); b = np.zeros(N, np.uint64)
    a[:3] = [1, 2, 3]; b[:2] = [4, 5]
    L.oracle_ntt_fwd(O.ptr(a), N, q, root); L.oracle_ntt_fwd(O.ptr(b), N, q, root)
    c = np.array([(int(x) * int(y)) % q for x, y in zip(a, b)], dtype=np.uint64)
    L.oracle_ntt_inv(O.ptr(c), N, q, root)
    assert list(c[:5]) == [4, 13, 22, 15, 0] and not c[5:].any()


def test_ntt_round_trip_and_negacyclic_wrap():
    rng = np.random.default_rng(42)
    N = P.N
    for q, root in ((P.q, P.w_crt), (P.q1, P.w1), (P.small_q, L.oracle_min_primitive_root(2 * N, P.small_q))):
        x = rng.integers(0, q, N, dtype=np.uint64)
        y = x.copy()
        L.oracle_ntt_fwd(O.ptr(y), N, q, root); L.oracle_ntt_inv(O.ptr(y), N, q, root)
        assert np.array_equal(x, y)
    # x^(N-1) * x = -1
    a = np.zeros(N, np.uint64); b = np.zeros(N, np.uint64); a[N - 1] = 1; b[1] = 1
    q, root = P.q1, P.w1
    L.oracle_ntt_fwd(O.ptr(a), N, q, root); L.oracle_ntt_fwd(O.ptr(b), N, q, root)
    c = np.array([(int(u) * int(v)) % q for u, v in zip(a, b)], dtype=np.uint64)
    L.oracle_ntt_inv(O.ptr(c), N, q, root)
    assert c[0] == q - 1 and not c[1:].any()


def test_primes_kat():
    # test_utils.cpp:11-45
    for p in (2, 3, 5, 7, 11, 13, 97, 1000003, 1152921504606748673, 1152921504606830593,
              36028797018820609, (1 << 61) - 1):
        assert L.oracle_is_prime(p)
    for c in (0, 1, 4, 6, 9, 15, 21, 25, 49, 1000000, 1152921504606748673 - 2, 1 << 61,
              (1 << 60) + 1, 3215031751):
        assert not L.oracle_is_prime(c)
    assert L.oracle_generate_prime(13) == 4099


def test_runtime_layout_kat():
    # test_runtime_layout.cpp:9-33
    flat = O.params(349526, 10)
    assert (flat.fst_dim_sz, flat.num_dims, flat.num_pt) == (512, 11, 349696)
    single = O.params(1, 0)
    assert (single.num_pt, single.num_dims, single.expansion_height) == (1, 1, 0)
    fst, dims = C.c_uint64(), C.c_uint64()
    assert L.oracle_calc_db_shape(43, 6, 5, 0, C.byref(fst), C.byref(dims)) == 0
    assert (fst.value, dims.value) == (26, 2)
    with pytest.raises(ValueError):
        O.params(0, 0)


def test_baseline_layouts():
    c1 = O.params(16384, 9)
    assert (c1.fst_dim_sz, c1.num_dims, c1.num_pt) == (256, 7, 16384)
    c2 = O.params(262144, 10)
    assert (c2.fst_dim_sz, c2.num_dims, c2.num_pt) == (512, 10, 262144)


def test_signed_decompose_reconstructs():
    # test_bv_keyswitch.cpp:10-57 with the keyswitch base (2^8, 8 digits)
    rng = np.random.default_rng(42)
    q, base, nd = P.q, P.base_ks, P.l_ks
    out = np.zeros(nd, np.uint64)
    vals = list(rng.integers(0, q, 2000, dtype=np.uint64)) + [0, 1, q - 1, q // 2, q // 2 + 1]
    for v in vals:
        L.oracle_signed_decompose(int(v), base, q, O.ptr(out), nd)
        rec = sum(int(d) * pow(2, base * i, q) for i, d in enumerate(out)) % q
        assert rec == int(v)
        mags = [min(int(d), q - int(d)) for d in out]
        assert max(mags) <= 1 << (base - 1)


def test_first_dim_kernel_against_naive_mod():
    # test_fst_dim.cpp:11-40 (diag n = 512, q = q1) and :46-93 shape
    rng = np.random.default_rng(0x51A1A5)
    for m, n, levels, q in ((1, 512, 1, P.q1), (4, 1024, 3, P.q2)):
        A = rng.integers(0, q, m * n * levels, dtype=np.uint64).astype(np.uint32)
        B = rng.integers(0, q, n * 2 * levels, dtype=np.uint64).astype(np.uint32)
        out = np.zeros(m * 2 * levels, np.uint64)
        L.oracle_level_mat_mat_32(O.ptr(A, C.c_uint32), O.ptr(B, C.c_uint32), O.ptr(out), m, n, levels, q)
        A3 = A.reshape(levels, m, n).astype(object); B3 = B.reshape(levels, n, 2).astype(object)
        ref = np.array([(A3[l] @ B3[l]) % q for l in range(levels)]).reshape(-1).astype(np.uint64)
        assert np.array_equal(out, ref)


def test_rescale_edges():
    q, sq = P.q, P.small_q
    for a in (0, 1, q // 2 - 1, q // 2, q // 2 + 1, q - 1):
        v = a - q if a >= q // 2 else a
        num = v * sq
        half = q // 2
        r = (num + half) // q if v >= 0 else -((-num + half) // q)
        assert L.oracle_rescale(a, q, sq) == r % sq
