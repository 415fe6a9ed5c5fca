"""The NTT-domain identities behind the last expansion level's NTT-form
children (k_expand_level_ntt, k4_expand_level_ntt, k1p_expand_level_ntt),
checked on the CPU against the oracle's forward NTT, which the reference
goldens pin (its order is the reference's bit-reversed one):

  * slot i holds the value at psi^e_i with e_i = 2 brev(i) + 1;
  * sigma_g (X -> X^g) is the slot gather f^[i] <- f^[j], e_j = e_i g mod 2N;
  * multiplication by X^-k scales slot i by psi^(-k e_i).

For every parameter set's moduli and ring degree, with the galois elements
g = N / 2^d + 1 and shifts k = 2^d of every expansion level d."""
import numpy as np
import pytest

from oracle import oracle as O


def _brev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2)


def _ntt(f, N, q, psi):
    a = np.array(f, dtype=np.uint64)
    O.lib().oracle_ntt_fwd(O.ptr(a), N, q, psi)
    return [int(v) for v in a]


def _sigma(f, g, N, q):
    """Coefficient form: sigma_g(f) = f(X^g) in Z_q[X]/(X^N + 1)."""
    out = [0] * N
    for m, c in enumerate(f):
        e = (m * g) % (2 * N)
        if e < N:
            out[e] = (out[e] + c) % q
        else:
            out[e - N] = (out[e - N] - c) % q
    return out


def _shift(f, k, N, q):
    """Coefficient form: f X^-k (negacyclic)."""
    out = [0] * N
    for m, c in enumerate(f):
        e = m - k
        if e >= 0:
            out[e] = c
        else:
            out[e + N] = (-c) % q
    return out


def _sets():
    p = O.params(16384, 9)
    c4 = O.c4_params(2048, 7)
    k1 = O.k1p_params(16384, 9)
    return [
        ("k1_comp q1", p.N, p.q1, p.w1),
        ("k1_comp q2", p.N, p.q2, p.w2),
        ("CONFIG_N4096_K2_MP limb 0", c4.N, c4.q[0], c4.w[0]),
        ("CONFIG_N4096_K2_MP limb 1", c4.N, c4.q[1], c4.w[1]),
        ("CONFIG_N2048_K1", k1.N, k1.q, k1.w_crt),  # the one prime's root
    ]


@pytest.mark.parametrize("name,N,q,psi", _sets())
def test_slot_exponents_sigma_gather_and_shift(name, N, q, psi):
    bits = N.bit_length() - 1
    rng = np.random.default_rng(N + q % 1000)
    # slot exponents: the NTT of f = X puts psi^e_i in slot i
    x = [0] * N
    x[1] = 1
    e = [2 * _brev(i, bits) + 1 for i in range(N)]
    assert _ntt(x, N, q, psi) == [pow(psi, ei, q) for ei in e]
    f = [int(v) for v in rng.integers(0, q, N, dtype=np.uint64)]
    F = _ntt(f, N, q, psi)
    for d in (0, 1, bits - 2, bits - 1):
        g, k = N // (1 << d) + 1, 1 << d
        S = _ntt(_sigma(f, g, N, q), N, q, psi)
        gathered = [F[_brev(((ei * g) % (2 * N)) >> 1, bits)] for ei in e]
        assert S == gathered, (name, d)
        R = _ntt(_shift(f, k, N, q), N, q, psi)
        assert R == [Fi * pow(psi, (-k * ei) % (2 * N), q) % q for Fi, ei in zip(F, e)], (name, d)
