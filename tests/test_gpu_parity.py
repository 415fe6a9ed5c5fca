"""GPU parity: the CUDA path through the C ABI against the CPU oracle and the
reference-generated goldens. Integer work, so every comparison is bit-exact.

Stage tests mirror the reference's public PirServer methods
(expand_query, complete_selectors, evaluate_first_dim, evaluate_other_dim);
end-to-end tests compare make_query responses (u64 arrays and the 22-bit
serialized stream) with the golden responses the reference itself produced,
and check that the client decrypts the requested plaintext.
"""
import functools

import numpy as np
import pytest

from onionpirv2_b200 import OutOfRange, PirParams, PirServer, save_response
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

SMALL = [c["name"] for c in G.cases() if c["num_pt"] <= 20000]
LARGE = [c["name"] for c in G.cases() if c["num_pt"] > 20000]


@functools.lru_cache(maxsize=None)
def setup(name):
    c = G.case(name)
    op = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    cl = O.Client(op, c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    q = cl.query(c["index"])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    srv = PirServer(gp)
    srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
    srv.set_client_keys(7, bv, gsw)
    return c, op, cl, bv, gsw, q, gp, srv


@functools.lru_cache(maxsize=None)
def oracle_server(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    s = O.Server(op)
    s.load_seeded(c["target_num_pt"], c["db_seed"])
    s.set_keys(bv, gsw)
    return s


def _check_response(c, cl, op, resp):
    assert G.sha256(resp) == c["sha256_response_u64"]
    assert save_response(PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"]),
                         resp) == G.stream(c)
    want = (O.db_plaintext(c["db_seed"], c["index"], op) if c["index"] < c["target_num_pt"]
            else np.zeros(op.N, np.uint16))
    assert np.array_equal(cl.decrypt(resp), want.astype(np.uint64))


@pytest.mark.parametrize("name", SMALL)
def test_expand_query_matches_oracle(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    got = srv.expand_query(7, q)
    want = oracle_server(name).expand(q)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", SMALL)
def test_complete_selectors_matches_oracle(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    exp = oracle_server(name).expand(q)
    got = srv.complete_selectors(7, exp)
    want = oracle_server(name).complete_selectors(exp)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", SMALL)
def test_first_dim_matches_oracle(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    exp = oracle_server(name).expand(q)
    got = srv.evaluate_first_dim(exp)
    want = oracle_server(name).first_dim(exp)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", SMALL)
def test_other_dim_matches_oracle(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    os_ = oracle_server(name)
    exp = os_.expand(q)
    sel = os_.complete_selectors(exp)
    mid = os_.first_dim(exp)
    got = srv.evaluate_other_dim(mid, sel)
    want = os_.other_dim(mid, sel)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", SMALL + LARGE)
def test_make_query_matches_reference_golden(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    _check_response(c, cl, op, srv.make_query(7, q))


def test_batch_equals_single_queries():
    name = "c1_16384_h9"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    rng = np.random.default_rng(5)
    clients, queries, idxs = [], [], []
    for i in range(5):
        k = O.Client(op, 1000 + i)
        srv.set_client_keys(100 + i, k.bv_keys(), k.gsw_key())
        idx = int(rng.integers(0, op.num_pt))
        clients.append(k); idxs.append(idx); queries.append(k.query(idx))
    ids = [100 + i for i in range(5)]
    batch = srv.make_query_batch(ids, np.stack(queries))
    for i in range(5):
        single = srv.make_query(ids[i], queries[i])
        assert np.array_equal(batch[i], single)
        assert np.array_equal(clients[i].decrypt(batch[i]),
                              O.db_plaintext(c["db_seed"], idxs[i], op).astype(np.uint64))
    # the batch mixes in the golden client and still matches the golden
    mixed = srv.make_query_batch([ids[0], 7, ids[1]], np.stack([queries[0], q, queries[1]]))
    _check_response(c, cl, op, mixed[1])


def test_load_paths_agree():
    name = "small_1000_h7"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    pts = np.stack([O.db_plaintext(c["db_seed"], i, op) for i in range(c["target_num_pt"])])
    for src in (pts, pts.astype(np.uint64), lambda i: pts[i]):
        s2 = PirServer(gp)
        s2.load_data(c["target_num_pt"], src)
        s2.set_client_keys(7, bv, gsw)
        _check_response(c, cl, op, s2.make_query(7, q))
        s2.close()


def test_errors_follow_the_reference():
    name = "ragged_43_h5"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    with pytest.raises(OutOfRange):
        srv.make_query(12345, q)                      # map::at on an unknown client
    bad = np.stack([O.db_plaintext(1, i, op) for i in range(c["target_num_pt"])]).astype(np.uint64)
    bad[3, 17] = op.t
    s2 = PirServer(gp)
    with pytest.raises(ValueError):                   # server.cpp:134-137
        s2.load_data(c["target_num_pt"], bad)
    with pytest.raises(ValueError):                   # server.cpp:85-88
        s2.load_data_seeded(op.num_pt + 1, 1)
    with pytest.raises(ValueError):                   # fewer keys than the height
        s2.set_client_keys(1, bv[:1], gsw)
    with pytest.raises(OutOfRange):                   # BvGaloisKeys::get
        s2.set_client_keys(1, bv, gsw, galois_ks=[3] * bv.shape[0])
    s2.close()
    # the handle stays usable after errors
    _check_response(c, cl, op, srv.make_query(7, q))


@pytest.mark.parametrize("mode", ["tc", "cuda"])
@pytest.mark.parametrize("name", SMALL + LARGE)
def test_both_scan_kernels_match_golden(name, mode, monkeypatch):
    """Force the tensor-core (tcgen05) or the CUDA-core first-dimension scan."""
    c, op, cl, bv, gsw, q, gp, _ = setup(name)
    monkeypatch.setenv("OPIR_SCAN", mode)
    with PirServer(gp) as srv:
        srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
        srv.set_client_keys(7, bv, gsw)
        _check_response(c, cl, op, srv.make_query(7, q))


@pytest.mark.parametrize("mode,batch", [("tc", 40), ("cuda", 9), ("tc", 3), ("tc", 16),
                                        ("tc", 32), ("tc", 12)])
def test_batched_scan_kernels(mode, batch, monkeypatch):
    """Every tensor-core tile width (16, 32, 64 columns; 80 columns = two
    tiles of 64) and a CUDA-core batch over several column tiles (18 > 16),
    against the single-query answers."""
    name = "small_1000_h7"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    rng = np.random.default_rng(batch)
    idx = [int(i) for i in rng.integers(0, c["target_num_pt"], batch)]
    monkeypatch.setenv("OPIR_SCAN", mode)
    with PirServer(gp) as s2:
        s2.load_data_seeded(c["target_num_pt"], c["db_seed"])
        s2.set_client_keys(7, bv, gsw)
        queries = np.stack([cl.query(i) for i in idx])
        out = s2.make_query_batch([7] * batch, queries)
    for i in range(batch):
        assert np.array_equal(out[i], srv.make_query(7, queries[i]))
        assert np.array_equal(cl.decrypt(out[i]),
                              O.db_plaintext(c["db_seed"], idx[i], op).astype(np.uint64))


TILINGS = [(16, 128, 2), (16, 128, 3), (32, 128, 2), (64, 128, 2), (16, 64, 6), (32, 64, 5),
           (64, 64, 4), (64, 64, 3)]


@pytest.mark.parametrize("tiling", TILINGS, ids=lambda t: "x".join(map(str, t)))
def test_every_scan_tiling_matches(tiling, monkeypatch):
    """Each tensor-core tiling the autotuner may pick (query columns per tile,
    K bytes per stage with its swizzle, pipeline depth), on a batch that
    spans two column tiles of 16 and on the single query, against the
    reference golden and the single-query answers."""
    name = "c1_16384_h9"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    monkeypatch.setenv("OPIR_SCAN_TILE", ",".join(map(str, tiling)))
    rng = np.random.default_rng(sum(tiling))
    idx = [int(i) for i in rng.integers(0, c["target_num_pt"], 11)]
    queries = np.stack([q] + [cl.query(i) for i in idx])
    with PirServer(gp) as s2:
        s2.load_data_seeded(c["target_num_pt"], c["db_seed"])
        s2.set_client_keys(7, bv, gsw)
        assert s2.scan_tile(12) == dict(zip(("ntile", "kt", "stages"), tiling))
        _check_response(c, cl, op, s2.make_query(7, q))
        out = s2.make_query_batch([7] * len(queries), queries)
    _check_response(c, cl, op, out[0])
    for i in range(len(idx)):
        assert np.array_equal(cl.decrypt(out[i + 1]),
                              O.db_plaintext(c["db_seed"], idx[i], op).astype(np.uint64))


def test_autotune_keeps_results():
    name = "c1_16384_h9"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    with PirServer(gp) as s2:
        s2.load_data_seeded(c["target_num_pt"], c["db_seed"])
        s2.set_client_keys(7, bv, gsw)
        s2.autotune(8)
        for n in (1, 2, 5, 8):
            t = s2.scan_tile(n)
            assert t["ntile"] in (16, 32, 64) and t["kt"] in (64, 128) and t["stages"] >= 2
            sp = s2.level_splits(n)
            assert all(w in (1, 2, 4, 8) for w in sp["expand"][:gp.expansion_height])
            assert all(w in (1, 2, 4) for w in sp["mux"][:gp.num_dims - 1])
        _check_response(c, cl, op, s2.make_query(7, q))
        out = s2.make_query_batch([7] * 5, np.stack([q] * 5))
        for i in range(5):
            _check_response(c, cl, op, out[i])


def test_graph_replays_match_eager_launches(monkeypatch):
    """The per-batch-size CUDA graph (eager on first use, captured on the
    second, replayed afterwards, with and without stage timing) gives the
    same responses and replays the same kernels as eager launches."""
    from onionpirv2_b200.server import launch_count
    name = "c1_16384_h9"
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    rng = np.random.default_rng(9)
    clients = [O.Client(op, 3000 + i) for i in range(3)]
    monkeypatch.setenv("OPIR_GRAPHS", "0")
    eager = PirServer(gp)
    monkeypatch.delenv("OPIR_GRAPHS")
    graphed = PirServer(gp)
    for s2 in (eager, graphed):
        s2.load_data_seeded(c["target_num_pt"], c["db_seed"])
        for i, k in enumerate(clients):
            s2.set_client_keys(i, k.bv_keys(), k.gsw_key())
    counts = {}
    for rnd in range(5):
        if rnd == 3:
            eager.set_stage_timing(True)
            graphed.set_stage_timing(True)
        idx = [int(i) for i in rng.integers(0, op.num_pt, 3)]
        qs = np.stack([clients[i].query(idx[i]) for i in range(3)])
        for tag, s2 in (("eager", eager), ("graph", graphed)):
            l0 = launch_count()
            out = s2.make_query_batch([0, 1, 2], qs)
            counts.setdefault(tag, []).append(launch_count() - l0)
            if tag == "eager":
                want = out
            else:
                assert np.array_equal(out, want), rnd
        for i in range(3):
            assert np.array_equal(clients[i].decrypt(want[i]),
                                  O.db_plaintext(c["db_seed"], idx[i], op).astype(np.uint64))
    assert counts["graph"] == counts["eager"]
    st = graphed.stage_times()
    assert st["calls"] == 2 and st["Core"] > 0 and st["Expand"] > 0
    eager.close()
    graphed.close()


def test_stream_priority_leaves_results_unchanged():
    """opir_server_set_priority moves the work to another stream; the
    responses stay the reference's."""
    c, op, cl, bv, gsw, q, gp, srv = setup("c1_16384_h9")
    for prio in (-1, 0, -100):
        srv.set_priority(prio)
        _check_response(c, cl, op, srv.make_query(7, q))


@pytest.mark.parametrize("name", SMALL + LARGE[:1])
def test_ntt_form_leaves_match_coefficient_leaves(name, monkeypatch):
    """The make_query pipeline's last expansion level writes the
    first-dimension leaves in NTT form (sigma and X^-k applied in the NTT
    domain); with OPIR_NTT_LEAVES=0 every leaf stays in coefficient form and
    the first dimension runs its own forward NTT. Both give the golden
    response, single and batched (eager, captured, replayed)."""
    c, op, cl, bv, gsw, q, gp, _ = setup(name)
    qs = np.stack([q, q, q])
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("OPIR_NTT_LEAVES", flag)
        with PirServer(gp) as srv:
            srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
            srv.set_client_keys(7, bv, gsw)
            for _ in range(3):
                r = srv.make_query(7, q)
                _check_response(c, cl, op, r)
            out[flag] = [srv.make_query_batch([7, 7, 7], qs) for _ in range(3)]
    for a, b in zip(out["1"], out["0"]):
        for ra, rb in zip(a, b):
            assert np.array_equal(ra, rb)
            assert G.sha256(ra) == c["sha256_response_u64"]
