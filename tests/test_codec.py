"""Seed-compressed wire codec (onionpirv2_b200.codec, opir_query_* /
opir_keys_* / opir_prf_expand), host-only: the library's ChaCha20 keystream
against the `cryptography` package's, the uniform expansion's range and
determinism, encode/decode round trips for both parameter sets (queries and
full key bundles), the wire sizes the reference's communication model
predicts, and the rejections of tampered input."""
import numpy as np
import pytest

from onionpirv2_b200 import PirParams
from onionpirv2_b200 import codec

C4 = "CONFIG_N4096_K2_MP"
SEED = bytes(range(32))


def chacha_words(seed, domain, index, count):
    algorithms = pytest.importorskip("cryptography.hazmat.primitives.ciphers.algorithms")
    from cryptography.hazmat.primitives.ciphers import Cipher
    nonce = (0).to_bytes(4, "little") + domain.to_bytes(4, "little") + index.to_bytes(8, "little")
    enc = Cipher(algorithms.ChaCha20(seed, nonce), mode=None).encryptor()
    return np.frombuffer(enc.update(b"\0" * (8 * count)), dtype="<u8")


@pytest.mark.parametrize("config", ["CONFIG_N2048_K1_COMP", C4])
def test_expand_is_chacha20_rejection_sampling(config):
    p = PirParams(43690 if config != C4 else 2048, 10 if config != C4 else 7, config=config)
    mods = [int(m) for m in p.get_rns_mods()]
    for domain, index in ((1, 0), (2, 37), (3, 5)):
        got = codec.prf_expand(p, SEED, domain, index).reshape(len(mods), -1)
        words = chacha_words(SEED, domain, index, 3 * got.size)
        want, w = [], iter(words)
        for q in mods:
            mask = (1 << int(q - 1).bit_length()) - 1
            row = []
            while len(row) < p.N:
                v = int(next(w)) & mask
                if v < q:
                    row.append(v)
            want.append(row)
        assert np.array_equal(got, np.array(want, dtype=np.uint64))
        assert all((got[k] < mods[k]).all() for k in range(len(mods)))
    a, b = codec.prf_expand(p, SEED, 1, 0), codec.prf_expand(p, SEED, 1, 1)
    assert not np.array_equal(a, b)


def _query(p, rng):
    mods = np.array(p.get_rns_mods(), dtype=np.uint64).reshape(-1, 1)
    c0 = rng.integers(0, np.iinfo(np.uint64).max, p.ct_shape[1:], dtype=np.uint64, endpoint=True)
    c0 = c0 % (mods if c0.ndim == 2 else mods[0])
    return np.stack([c0, codec.prf_expand(p, SEED, codec.PRF_QUERY, 0)])


@pytest.mark.parametrize("config,size", [("CONFIG_N2048_K1_COMP", 14884), (C4, 4 + 32 + 2 * 4096 * 60 // 8)])
def test_query_round_trip(config, size):
    p = PirParams(43690 if config != C4 else 2048, 10 if config != C4 else 7, config=config)
    rng = np.random.default_rng(3)
    q = _query(p, rng)
    data = codec.encode_query(p, SEED, q)
    assert len(data) == size == codec.query_wire_bytes(p)
    assert np.array_equal(codec.decode_query(p, data), q)
    bad = q.copy()
    bad[1].flat[7] ^= 1                     # c1 no longer Expand(seed)
    with pytest.raises(ValueError):
        codec.encode_query(p, SEED, bad)
    with pytest.raises(ValueError):
        codec.decode_query(p, data[:-1])
    with pytest.raises(ValueError):
        codec.decode_query(p, b"XPQ1" + data[4:])


@pytest.mark.parametrize("config", ["CONFIG_N2048_K1_COMP", C4])
def test_key_bundle_round_trip(config):
    p = PirParams(43690 if config != C4 else 2048, 10 if config != C4 else 7, config=config)
    rng = np.random.default_rng(4)
    mods = np.array(p.get_rns_mods(), dtype=np.uint64)
    poly = p.ct_shape[1:]

    def uniform():
        v = rng.integers(0, np.iinfo(np.uint64).max, poly, dtype=np.uint64, endpoint=True)
        return v % (mods.reshape(-1, 1) if len(poly) == 2 else mods[0])

    h = p.expansion_height
    bv = np.zeros((h, p.l_ks, 2) + poly, dtype=np.uint64)
    for i in range(h):
        for j in range(p.l_ks):
            bv[i, j, 0] = uniform()
            bv[i, j, 1] = codec.prf_expand(p, SEED, codec.PRF_BV_KEY, i * p.l_ks + j)
    g = np.zeros((2 * p.l_key, 2) + poly, dtype=np.uint64)
    for r in range(2 * p.l_key):
        g[r, 0] = uniform()
        g[r, 1] = codec.prf_expand(p, SEED, codec.PRF_GSW_KEY, r)
    data = codec.encode_keys(p, SEED, bv, g)
    assert len(data) == codec.keys_wire_bytes(p)
    bv2, ks, g2 = codec.decode_keys(p, data)
    assert np.array_equal(bv2, bv) and np.array_equal(g2, g)
    assert list(ks) == [(p.N >> i) + 1 for i in range(h)]
    g[3, 1].flat[0] ^= 1
    with pytest.raises(ValueError):
        codec.encode_keys(p, SEED, bv, g)


def test_wire_sizes_match_the_reference_model():
    p = PirParams()   # get_BFV_size(true) = 32 + 58 N / 8; keys = h L_KS + 2 L_KEY rows
    assert codec.query_wire_bytes(p) == 4 + 32 + 58 * p.N // 8
    rows = p.expansion_height * p.l_ks + 2 * p.l_key
    assert codec.keys_wire_bytes(p) == 4 + 32 + rows * 58 * p.N // 8
