"""GPU client batch operations (opir_client_*, the reference's
PirClient::fast_generate_query, client.cpp:107-225, and decrypt_mod_q,
client.cpp:364-410) against the oracle client, bit for bit: queries packed on
the GPU from the oracle's own uniform c1 and error equal the oracle's queries;
responses decrypted on the GPU equal the oracle's plaintexts and max noise;
and a GPU-packed query answered by the GPU server decrypts on the GPU to the
database plaintext. Every case runs three times: as the launcher picks
(auto: tensor-core decryption for single-modulus batches of 32 or more, the
window kernel for other batches that fill the GPU), with the tensor-core form
off (OPIR_CLIENT_TC=0) and with the index-list kernel forced
(OPIR_CLIENT_WINDOW=0); batch sizes cover every outputs-per-thread width each
CUDA-core kernel uses (list: 1, 2, 4, 8; window: 4, 8) and full and partial
column tiles of the tensor-core scan (33, 80, 150, 300)."""
import numpy as np
import pytest

from onionpirv2_b200 import OutOfRange, PirParams, PirServer
from onionpirv2_b200.client import PirClient
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["auto", "window", "list"])
def kernel(request, monkeypatch):
    monkeypatch.delenv("OPIR_CLIENT_WINDOW", raising=False)
    monkeypatch.delenv("OPIR_CLIENT_TC", raising=False)
    if request.param == "window":
        monkeypatch.setenv("OPIR_CLIENT_TC", "0")
    elif request.param == "list":
        monkeypatch.setenv("OPIR_CLIENT_WINDOW", "0")
    return request.param

C4 = "CONFIG_N4096_K2_MP"


def _indices(num_pt, rng, n):
    fixed = [0, num_pt - 1, num_pt // 2]
    return (fixed + [int(x) for x in rng.integers(0, num_pt, max(n - 3, 0))])[:n]


def _uniform(rng, mods, n, N):
    return np.stack([np.stack([rng.integers(0, int(q), N, dtype=np.uint64) for q in mods])
                     for _ in range(n)])


@pytest.mark.parametrize("n", [1, 80, 150, 300])
def test_k1_queries_match_oracle(n, kernel):
    target, h = 43690, 10
    gp, op = PirParams(target, h), O.params(target, h)
    rng = np.random.default_rng(1000 + n)
    idx = _indices(op.num_pt, rng, n)
    a = _uniform(rng, [op.q], n, op.N)[:, 0]
    cl = O.Client(op, 91)
    parts = [cl.query_parts(x, a[i]) for i, x in enumerate(idx)]
    gc = PirClient(gp, cl.secret())
    got = gc.fast_generate_query_batch(idx, a, np.stack([e for _, e in parts]))
    assert got.shape == (n, 2, op.N)
    assert np.array_equal(got, np.stack([q for q, _ in parts]))


@pytest.mark.parametrize("n", [1, 40, 75, 200])
def test_c4_queries_match_oracle(n, kernel):
    target, h = 16384, 9
    gp, op = PirParams(target, h, config=C4), O.c4_params(target, h)
    rng = np.random.default_rng(2000 + n)
    idx = _indices(op.num_pt, rng, n)
    a = _uniform(rng, op.q[:2], n, op.N)
    cl = O.C4Client(op, 93)
    parts = [cl.query_parts(x, a[i]) for i, x in enumerate(idx)]
    gc = PirClient(gp, cl.secret())
    got = gc.fast_generate_query_batch(idx, a, np.stack([e for _, e in parts]))
    assert got.shape == (n, 2, 2, op.N)
    assert np.array_equal(got, np.stack([q for q, _ in parts]))


def test_k1_error_of_any_size_enters_linearly(kernel):
    """c0 is -(a s + e) mod q for any int64 error, not only Gaussian ones:
    the difference of two packings is -(e' - e) mod q everywhere."""
    target, h = 16384, 9
    gp, op = PirParams(target, h), O.params(target, h)
    rng = np.random.default_rng(7)
    n = 160  # wide enough for the window kernel
    a = _uniform(rng, [op.q], n, op.N)[:, 0]
    cl = O.Client(op, 5)
    gc = PirClient(gp, cl.secret())
    e = np.stack([cl.query_parts(3, a[i])[1] for i in range(n)])
    big = rng.integers(-(1 << 62), 1 << 62, size=(n, op.N), dtype=np.int64)
    big[0, :4] = [np.iinfo(np.int64).min, np.iinfo(np.int64).max, -1, 0]
    q1 = gc.fast_generate_query_batch([3] * n, a, e)
    q2 = gc.fast_generate_query_batch([3] * n, a, big)
    q = int(op.q)
    for i in (0, n - 1):
        for j in range(op.N):
            assert (int(q2[i, 0, j]) - int(q1[i, 0, j])) % q == (-(int(big[i, j]) - int(e[i, j]))) % q
    assert np.array_equal(q1[:, 1], q2[:, 1])


@pytest.mark.parametrize("config,n", [("k1", 1), ("k1", 33), ("k1", 80), ("k1", 150), ("k1", 300),
                                      ("c4", 1), ("c4", 40), ("c4", 75), ("c4", 200)])
def test_decrypt_matches_oracle(config, n, kernel):
    if config == "k1":
        gp, op = PirParams(16384, 9), O.params(16384, 9)
        cl = O.Client(op, 17)
    else:
        gp, op = PirParams(16384, 9, config=C4), O.c4_params(16384, 9)
        cl = O.C4Client(op, 19)
    rng = np.random.default_rng(n)
    resp = rng.integers(0, int(op.small_q), size=(n, 2, op.N), dtype=np.uint64)
    resp[0, :, :3] = int(op.small_q) - 1
    gc = PirClient(gp, cl.secret())
    pt, noise = gc.decrypt_mod_q_batch(resp, with_noise=True)
    for i in range(n):
        want, want_noise = cl.decrypt_noise(resp[i])
        assert np.array_equal(pt[i], want)
        assert int(noise[i]) == want_noise


@pytest.mark.parametrize("config", ["k1", "c4"])
def test_gpu_query_answer_decrypt_round_trip(config, kernel):
    target, h, db_seed = 16384, 9, 23
    if config == "k1":
        gp, op = PirParams(target, h), O.params(target, h)
        cl = O.Client(op, 29)
        mods = [op.q]
        plain = lambda i: O.db_plaintext(db_seed, i, op).astype(np.uint64)  # noqa: E731
    else:
        gp, op = PirParams(target, h, config=C4), O.c4_params(target, h)
        cl = O.C4Client(op, 31)
        mods = op.q[:2]
        plain = lambda i: O.c4_db_plaintext(db_seed, i, op)  # noqa: E731
    rng = np.random.default_rng(5)
    idx = [0, 77, target - 1, 9000]
    a = _uniform(rng, mods, len(idx), op.N).reshape((len(idx),) + gp.ct_shape[1:])
    e = np.stack([cl.query_parts(i, a[k])[1] for k, i in enumerate(idx)])
    gc = PirClient(gp, cl.secret())
    queries = gc.fast_generate_query_batch(idx, a, e)
    srv = PirServer(gp)
    srv.load_data_seeded(target, db_seed)
    srv.set_client_keys(3, cl.bv_keys(), cl.gsw_key())
    resp = srv.make_query_batch([3] * len(idx), queries)
    pt, noise = gc.decrypt_mod_q_batch(resp, with_noise=True)
    for k, i in enumerate(idx):
        assert np.array_equal(pt[k], plain(i))
        assert np.array_equal(pt[k], cl.decrypt(resp[k]))
    assert int(noise.max()) < int(op.small_q) // (2 * int(op.t))


def test_out_of_range_index():
    gp, op = PirParams(16384, 9), O.params(16384, 9)
    gc = PirClient(gp, O.Client(op, 1).secret())
    a = np.zeros((1, op.N), np.uint64)
    e = np.zeros((1, op.N), np.int64)
    with pytest.raises(OutOfRange):
        gc.fast_generate_query_batch([op.num_pt], a, e)
    # the handle stays usable
    assert gc.fast_generate_query_batch([0], a, e).shape == (1, 2, op.N)


@pytest.mark.parametrize("config,target,h", [("k1", 16384, 9), ("k1", 43690, 10),
                                             ("c4", 16384, 9)])
def test_session_keys_match_oracle(config, target, h):
    """create_session_keys on the GPU from the randomness the oracle client's
    key generation drew equals its BV and RGSW keys bit for bit, and the
    GPU server answers with them like with the oracle's keys."""
    if config == "k1":
        gp, op = PirParams(target, h), O.params(target, h)
        cl = O.Client(op, 61, keygen_parts=True)
    else:
        gp, op = PirParams(target, h, config=C4), O.c4_params(target, h)
        cl = O.C4Client(op, 61, keygen_parts=True)
    kg = cl.keygen
    gc = PirClient(gp, cl.secret())
    bv, gsw = gc.create_session_keys(kg["bv_a"], kg["bv_e"], kg["gsw_a"], kg["gsw_e"])
    assert np.array_equal(bv, cl.bv_keys())
    assert np.array_equal(gsw, cl.gsw_key())
    idx = 1234
    srv = PirServer(gp)
    srv.load_data_seeded(target, 3)
    srv.set_client_keys(1, bv, gsw)
    resp = srv.make_query(1, cl.query(idx))
    want = (O.db_plaintext(3, idx, op).astype(np.uint64) if config == "k1"
            else O.c4_db_plaintext(3, idx, op))
    assert np.array_equal(gc.decrypt_mod_q(resp), want)


@pytest.mark.parametrize("config,n", [("k1", 64), ("c4", 40)])
def test_whole_client_pipeline_on_the_gpu(config, n):
    """Session keys, queries and decryption all on the GPU around the GPU
    server: every plaintext comes back."""
    target, h, db_seed = 16384, 9, 41
    if config == "k1":
        gp, op = PirParams(target, h), O.params(target, h)
        cl = O.Client(op, 71, keygen_parts=True)
        mods = [op.q]
        plain = lambda i: O.db_plaintext(db_seed, i, op).astype(np.uint64)  # noqa: E731
    else:
        gp, op = PirParams(target, h, config=C4), O.c4_params(target, h)
        cl = O.C4Client(op, 71, keygen_parts=True)
        mods = op.q[:2]
        plain = lambda i: O.c4_db_plaintext(db_seed, i, op)  # noqa: E731
    gc = PirClient(gp, cl.secret())
    bv, gsw = gc.create_session_keys(**cl.keygen)
    srv = PirServer(gp)
    srv.load_data_seeded(target, db_seed)
    srv.set_client_keys(9, bv, gsw)
    rng = np.random.default_rng(13)
    idx = [int(x) for x in rng.integers(0, target, n)]
    a = _uniform(rng, mods, n, op.N).reshape((n,) + gp.ct_shape[1:])
    e = np.rint(rng.normal(0.0, 3.2, (n, op.N))).astype(np.int64)
    resp = srv.make_query_batch([9] * n, gc.fast_generate_query_batch(idx, a, e))
    pt = gc.decrypt_mod_q_batch(resp)
    for k, i in enumerate(idx):
        assert np.array_equal(pt[k], plain(i))


@pytest.mark.parametrize("config", ["k1", "c4"])
def test_tree_queries_match_oracle(config):
    """make_tree_query on the GPU equals the oracle client's for the same c1
    and error, over the golden tree cases' coordinates and random leaves."""
    from onionpirv2_b200 import tree as T
    from tests import golden_cases as G
    if config == "k1":
        scheme, cases = PirParams(), G.cases_tree()
        op = O.params(scheme.target_num_pt, scheme.expansion_height)
        cl = O.Client(op, 55)
        mods = [op.q]
    else:
        scheme, cases = PirParams(config=C4), G.cases_tree_c4()
        op = O.c4_params(scheme.target_num_pt, scheme.expansion_height)
        cl = O.C4Client(op, 55)
        mods = op.q[:2]
    gc = PirClient(scheme, cl.secret())
    rng = np.random.default_rng(3)
    for c in cases[:4]:
        tree = T.make_tree_pir_params_for_scheme(c["L"], c["a"], scheme)
        leaves = [c["leaf"]] + [int(x) for x in rng.integers(0, 1 << c["L"], 5)]
        coords = [T.client_index(leaf, tree) for leaf in leaves]
        bits = np.array([list(k.beta_bits_le) + list(k.gamma_bits_le) for k in coords],
                        dtype=np.uint8)
        a = _uniform(rng, mods, len(leaves), op.N).reshape((len(leaves),) + scheme.ct_shape[1:])
        parts = [cl.tree_query_parts(tree.N0, tree.h_q, k.alpha, k.beta_bits_le,
                                     k.gamma_bits_le, a[i]) for i, k in enumerate(coords)]
        got = gc.make_tree_queries(tree, [k.alpha for k in coords], bits, a,
                                   np.stack([e for _, e in parts]))
        assert np.array_equal(got, np.stack([q for q, _ in parts])), c["name"]
