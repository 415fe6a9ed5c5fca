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
