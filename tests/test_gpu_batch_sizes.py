"""GPU parity at the batch sizes the benchmark runs, on small layouts.

The first-dimension scans change form with the batch: the two-limb scan
(CONFIG_N4096_K2_MP) uses 16-column tiles up to 8 queries, then 32-column
tiles, with the two column tiles of a row tile run by neighbouring CTAs in
lock step at 17-32 queries and three or more unpaired tiles above 32; the
k1_comp scan uses one 64-column tile up to 32 queries and several above
(four at 128). Each batch mixes the reference's golden client (its response
must equal the reference's digest) with other clients' queries, each of
which must equal the CPU oracle server's answer for that client
(server.cpp:895-947 per query) and decrypt to the requested plaintext.
Integer work: every comparison is bit-exact."""
import functools

import numpy as np
import pytest

from onionpirv2_b200 import PirParams, PirServer
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

C4 = "CONFIG_N4096_K2_MP"


@functools.lru_cache(maxsize=None)
def c4_pool(name="c4_2048_h7", clients=4, per_client=16):
    """The golden client plus `clients - 1` other clients, `per_client`
    random indices each, with the oracle's answers (one oracle server per
    client, since the oracle holds one client's keys)."""
    c = G.case_c4(name)
    op = O.c4_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    ref = O.C4Server(op)
    ref.load_seeded(c["target_num_pt"], c["db_seed"])
    rng = np.random.default_rng(2024)
    cls = [O.C4Client(op, c["client_seed"])] + [O.C4Client(op, 300 + j) for j in range(clients - 1)]
    items = []   # (client number, index, query, oracle answer)
    for k, cl in enumerate(cls):
        ref.set_keys(cl.bv_keys(), cl.gsw_key())
        for i in rng.integers(0, op.num_pt, per_client):
            q = cl.query(int(i))
            items.append((k, int(i), q, ref.make_query(q)))
    # the golden query is the first one a fresh golden client draws
    golden_q = O.C4Client(op, c["client_seed"]).query(c["index"])
    return c, op, cls, items, golden_q


@functools.lru_cache(maxsize=None)
def c4_server(name="c4_2048_h7"):
    c, op, cls, items, golden_q = c4_pool(name)
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"], config=C4)
    srv = PirServer(gp)
    srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
    for k, cl in enumerate(cls):
        srv.set_client_keys(k, cl.bv_keys(), cl.gsw_key())
    return srv


def _interleave(items, batch, shift):
    """`batch - 1` pool items, clients interleaved, starting at `shift`."""
    order = sorted(range(len(items)), key=lambda j: (j % 16, j // 16))
    return [items[order[(shift + j) % len(order)]] for j in range(batch - 1)]


@pytest.mark.parametrize("batch", [17, 24, 32, 33, 64])
def test_c4_benchmarked_batch_sizes(batch):
    c, op, cls, items, golden_q = c4_pool()
    srv = c4_server()
    chosen = _interleave(items, batch, batch)
    at = batch // 2   # the golden query in the middle of the batch
    ids = [k for k, _, _, _ in chosen]
    qs = [q for _, _, q, _ in chosen]
    ids.insert(at, 0)
    qs.insert(at, golden_q)
    out = srv.make_query_batch(ids, np.stack(qs))
    assert G.sha256(out[at]) == c["sha256_response_u64"]
    j = 0
    for pos in range(batch):
        if pos == at:
            continue
        k, idx, q, want = chosen[j]
        j += 1
        assert np.array_equal(out[pos], want), (batch, pos)
        assert np.array_equal(cls[k].decrypt(out[pos]), O.c4_db_plaintext(c["db_seed"], idx, op))


@functools.lru_cache(maxsize=None)
def k1_pool(name="small_1000_h7", clients=4, per_client=32):
    c = G.case(name)
    op = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    ref = O.Server(op)
    ref.load_seeded(c["target_num_pt"], c["db_seed"])
    rng = np.random.default_rng(4048)
    cls = [O.Client(op, c["client_seed"])] + [O.Client(op, 500 + j) for j in range(clients - 1)]
    items = []
    for k, cl in enumerate(cls):
        ref.set_keys(cl.bv_keys(), cl.gsw_key())
        for i in rng.integers(0, op.num_pt, per_client):
            q = cl.query(int(i))
            items.append((k, int(i), q, ref.make_query(q)))
    return c, op, cls, items, O.Client(op, c["client_seed"]).query(c["index"])


@pytest.mark.parametrize("tiling", [None, "64,64,4", "64,128,2"])
@pytest.mark.parametrize("batch", [64, 128])
def test_k1_benchmarked_batch_sizes(batch, tiling, monkeypatch):
    """Two and four 64-column tiles of the tensor-core scan (the default
    tiling and the ones the autotuner picks on the 2^18 layout)."""
    c, op, cls, items, golden_q = k1_pool()
    if tiling:
        monkeypatch.setenv("OPIR_SCAN_TILE", tiling)
    chosen = [items[(batch + 5 * j) % len(items)] for j in range(batch - 1)]
    at = batch - 1   # the golden query in the last column tile
    ids = [k for k, _, _, _ in chosen] + [0]
    qs = np.stack([q for _, _, q, _ in chosen] + [golden_q])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    with PirServer(gp) as srv:
        srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
        for k, cl in enumerate(cls):
            srv.set_client_keys(k, cl.bv_keys(), cl.gsw_key())
        t = srv.scan_tile(batch)
        assert t["ntile"] == 64
        out = srv.make_query_batch(ids, qs)
    assert G.sha256(out[at]) == c["sha256_response_u64"]
    for pos, (k, idx, q, want) in enumerate(chosen):
        assert np.array_equal(out[pos], want), (batch, pos)
        # indices past the logical count are padding rows of zeros
        pt = (O.db_plaintext(c["db_seed"], idx, op).astype(np.uint64) if idx < c["target_num_pt"]
              else np.zeros(op.N, np.uint64))
        assert np.array_equal(cls[k].decrypt(out[pos]), pt)


@pytest.mark.parametrize("name", ["c1_16384_h9", "c4_ragged_43_h5"])
def test_scan_wait_timeout_is_reported_and_the_handle_recovers(name, monkeypatch):
    """Every wait of the tensor-core scans is bounded. With the limit set to
    a few dozen cycles a wait runs out (a TMA load alone takes longer): the
    kernel records the error, drains its own copies and MMAs, frees its
    tensor memory and returns, and the call raises RuntimeError. With the
    default limit restored, the same handle answers bit-exact again."""
    c4 = name.startswith("c4_")
    c = G.case_c4(name) if c4 else G.case(name)
    if c4:
        op = O.c4_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
        cl = O.C4Client(op, c["client_seed"])
        gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"], config=C4)
    else:
        op = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
        cl = O.Client(op, c["client_seed"])
        gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
        monkeypatch.setenv("OPIR_SCAN", "tc")
    q = cl.query(c["index"])
    with PirServer(gp) as srv:
        srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
        srv.set_client_keys(7, cl.bv_keys(), cl.gsw_key())
        assert G.sha256(srv.make_query(7, q)) == c["sha256_response_u64"]
        srv.set_scan_wait_limit(32)
        for _ in range(2):   # eager, then a captured pipeline
            with pytest.raises(RuntimeError, match="timed out"):
                srv.make_query(7, q)
        with pytest.raises(RuntimeError, match="timed out"):
            srv.make_query_batch([7, 7, 7], np.stack([q, q, q]))
        srv.set_scan_wait_limit(0)
        for _ in range(3):   # eager, captured, replayed
            assert G.sha256(srv.make_query(7, q)) == c["sha256_response_u64"]
        out = srv.make_query_batch([7, 7, 7], np.stack([q, q, q]))
        for r in out:
            assert G.sha256(r) == c["sha256_response_u64"]
