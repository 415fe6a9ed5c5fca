"""Host-only checks of what the GPU client tests feed the kernels: the
oracle client's coefficient-form secret and the error it draws for a query
(oracle_client_secret / oracle_client_query_parts and their two-limb forms)
reproduce its own query, c0 = -(a s + e) mod q_k away from the packed
plaintext's positions (client.cpp:107-225), with the negacyclic product
computed here in exact integers. Also the C ABI's create-time argument
checks, which run before any device call."""
import numpy as np
import pytest

from onionpirv2_b200 import PirParams
from onionpirv2_b200.client import PirClient
from oracle import oracle as O

C4 = "CONFIG_N4096_K2_MP"


def negacyclic_ternary(a: np.ndarray, s: np.ndarray, q: int) -> np.ndarray:
    """(a * s) mod q in Z_q[X]/(X^N + 1) for ternary s, exact (31-bit parts)."""
    N = a.size
    lo = (a & np.uint64(0x7FFFFFFF)).astype(np.int64)
    hi = (a >> np.uint64(31)).astype(np.int64)
    ext_lo = np.concatenate([-lo, lo])
    ext_hi = np.concatenate([-hi, hi])
    acc_lo = np.zeros(N, np.int64)
    acc_hi = np.zeros(N, np.int64)
    idx = np.arange(N)
    for j in np.nonzero(s)[0]:
        sel = N + idx - j
        acc_lo += int(s[j]) * ext_lo[sel]
        acc_hi += int(s[j]) * ext_hi[sel]
    return np.array([((int(h) << 31) + int(l)) % q for h, l in zip(acc_hi, acc_lo)],
                    dtype=object)


def test_k1_secret_and_error_reproduce_the_query():
    sch = PirParams()
    p = O.params(16384, 9)
    rng = np.random.default_rng(3)
    a = rng.integers(0, p.q, p.N, dtype=np.uint64)
    idx = 16383
    want = O.Client(p, 41).query_with_a(idx, a)
    cl = O.Client(p, 41)
    q, e = cl.query_parts(idx, a)
    assert np.array_equal(q, want)
    s = cl.secret()
    assert set(np.unique(s)) <= {-1, 0, 1} and s.shape == (sch.N,)
    prod = negacyclic_ternary(a, s, p.q)
    c0 = np.array([(-(int(x) + int(y))) % p.q for x, y in zip(prod, e)], dtype=object)
    diff = np.nonzero(c0 != q[0].astype(object))[0]
    # the one-hot plus the set selector bits' gadget rows
    assert 1 <= diff.size <= 1 + (p.num_dims - 1) * p.l_ep
    assert np.array_equal(q[1], a)


def test_c4_secret_and_error_reproduce_the_query():
    p = O.c4_params(16384, 9)
    rng = np.random.default_rng(4)
    a = np.stack([rng.integers(0, int(qk), p.N, dtype=np.uint64) for qk in p.q[:2]])
    idx = 12345
    cl = O.C4Client(p, 43)
    q, e = cl.query_parts(idx, a)
    s = cl.secret()
    assert set(np.unique(s)) <= {-1, 0, 1}
    for k in range(2):
        qk = int(p.q[k])
        prod = negacyclic_ternary(a[k], s, qk)
        c0 = np.array([(-(int(x) + int(y))) % qk for x, y in zip(prod, e)], dtype=object)
        diff = np.nonzero(c0 != q[0][k].astype(object))[0]
        assert 1 <= diff.size <= 1 + (p.num_dims - 1) * p.l_ep
        assert np.array_equal(q[1][k], a[k])


def test_create_rejects_bad_arguments_before_any_device_call():
    p = PirParams(16384, 9)
    with pytest.raises(ValueError):
        PirClient(p, np.full(p.N, 2, np.int8))
    with pytest.raises(ValueError):
        PirClient(p, np.zeros(p.N - 1, np.int8))
    shaped = PirParams().with_query_shape(8, 2, 7)
    with pytest.raises(ValueError):
        PirClient(shaped, np.zeros(p.N, np.int8))


def _ntt(poly, q, root):
    a = np.ascontiguousarray(np.array([int(v) % q for v in poly], dtype=np.uint64))
    O.lib().oracle_ntt_fwd(O.ptr(a), a.size, q, root)
    return a


def _sigma(s, k):
    N = s.size
    out = np.zeros(N, np.int8)
    for j in range(N):
        d = (j * k) % (2 * N)
        if d < N:
            out[d] = s[j]
        else:
            out[d - N] = -s[j]
    return out


def _row(a, e, s, msg, scale, half, esign, q):
    """(c0, c1) coefficient form: c0 = -(a s) + esign e + [half=0] scale msg,
    c1 = a + [half=1] scale msg (mod q)."""
    prod = negacyclic_ternary(a, s, q)
    m = [scale * int(x) for x in msg]
    c0 = [(-int(prod[i]) + esign * int(e[i]) + (m[i] if half == 0 else 0)) % q
          for i in range(a.size)]
    c1 = [(int(a[i]) + (m[i] if half == 1 else 0)) % q for i in range(a.size)]
    return c0, c1


@pytest.mark.parametrize("config", ["k1", "c4"])
def test_keygen_randomness_reproduces_the_keys(config):
    """The session keys are, row by row, coefficient-form ciphertexts built
    from the captured (a, e) and then NTT'd per limb -- the computation the
    GPU key generation performs (sampled rows)."""
    if config == "k1":
        p = O.params(16384, 9)
        cl = O.Client(p, 12, keygen_parts=True)
        mods, roots = [int(p.q)], [int(p.w_crt)]
        base_ks, base_key = p.base_ks, p.base_key
    else:
        p = O.c4_params(16384, 9)
        cl = O.C4Client(p, 12, keygen_parts=True)
        mods, roots = [int(x) for x in p.q[:2]], [int(x) for x in p.w[:2]]
        base_ks, base_key = p.base_ks, p.base_key
    s = cl.secret()
    kg = cl.keygen
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    h, N = p.expansion_height, p.N
    for i in (0, h - 1):
        sig = _sigma(s, (N >> i) + 1)
        for r in (0, p.l_ks - 1):
            for k, (q, root) in enumerate(zip(mods, roots)):
                a = kg["bv_a"][i, r] if config == "k1" else kg["bv_a"][i, r, k]
                c0, c1 = _row(a, kg["bv_e"][i, r], s, sig, pow(2, r * base_ks, q), 0, 1, q)
                got = bv[i, r] if config == "k1" else bv[i, r, :, k]
                assert np.array_equal(_ntt(c0, q, root), got[0])
                assert np.array_equal(_ntt(c1, q, root), got[1])
    for row in (0, p.l_key - 1, p.l_key, 2 * p.l_key - 1):
        half, r = divmod(row, p.l_key)
        for k, (q, root) in enumerate(zip(mods, roots)):
            a = kg["gsw_a"][row] if config == "k1" else kg["gsw_a"][row, k]
            scale = pow(2, base_key * (p.l_key - 1 - r), q)
            c0, c1 = _row(a, kg["gsw_e"][row], s, s, scale, half, -1, q)
            got = gsw[row] if config == "k1" else gsw[row, :, k]
            assert np.array_equal(_ntt(c0, q, root), got[0])
            assert np.array_equal(_ntt(c1, q, root), got[1])
