"""GPU parity for CONFIG_N2048_K1, the reference's default parameter set (N =
2048, one 60-bit NTT prime, signed single-modulus gadgets): the CUDA path
through the C ABI against the golden digests the reference itself produced
when built with that configuration (tests/golden/golden_k1p.json), stage by
stage, and against the CPU oracle (single-prime form) for batches of clients
the goldens do not cover. The set runs on its own 64-bit kernels
(opir_k1p_kernels.cu) and the 64-bit-limb tensor-core scan. Integer work:
every comparison is bit-exact."""
import functools

import numpy as np
import pytest

from onionpirv2_b200 import OutOfRange, PirParams, PirServer, save_response
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

K1P = "CONFIG_N2048_K1"
CASES = [c["name"] for c in G.cases_set("k1p")]


@functools.lru_cache(maxsize=None)
def setup(name):
    c = G.case_set("k1p", name)
    op = O.k1p_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    cl = O.Client(op, c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    q = cl.query(c["index"])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"], config=K1P)
    srv = PirServer(gp)
    srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
    srv.set_client_keys(7, bv, gsw)
    return c, op, cl, bv, gsw, q, gp, srv


def _plaintext(c, op):
    if c["index"] < c["target_num_pt"]:
        return O.db_plaintext(c["db_seed"], c["index"], op).astype(np.uint64)
    return np.zeros(op.N, np.uint64)


@pytest.mark.parametrize("name", CASES)
def test_k1p_stages_match_reference(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    exp = srv.expand_query(7, q)
    assert G.sha256(exp) == c["sha256_stage_expand"]
    sel = srv.complete_selectors(7, exp)
    assert G.sha256(np.ascontiguousarray(sel)) == c["sha256_stage_selectors"]
    mid = srv.evaluate_first_dim(exp)
    assert G.sha256(mid) == c["sha256_stage_first_dim"]
    fin = srv.evaluate_other_dim(mid, sel)
    assert G.sha256(fin) == c["sha256_stage_other_dim"]


@pytest.mark.parametrize("name", CASES)
def test_k1p_make_query_matches_reference(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    resp = srv.make_query(7, q)
    assert G.sha256(resp) == c["sha256_response_u64"]
    assert save_response(gp, resp) == G.stream(c)
    assert np.array_equal(cl.decrypt(resp), _plaintext(c, op))


def test_k1p_batch_of_clients_matches_oracle():
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_1000_h7")
    rng = np.random.default_rng(11)
    clients, queries, ids, idxs = [], [], [], []
    for j in range(3):
        k = O.Client(op, 100 + j)
        srv.set_client_keys(50 + j, k.bv_keys(), k.gsw_key())
        idx = int(rng.integers(0, op.num_pt))
        clients.append(k)
        queries.append(k.query(idx))
        ids.append(50 + j)
        idxs.append(idx)
    # the golden client in the middle of the batch
    clients.insert(1, cl)
    queries.insert(1, q)
    ids.insert(1, 7)
    idxs.insert(1, c["index"])
    out = srv.make_query_batch(ids, np.stack(queries))
    assert G.sha256(out[1]) == c["sha256_response_u64"]
    ref = O.Server(op)
    ref.load_seeded(c["target_num_pt"], c["db_seed"])
    for j, k in enumerate(clients):
        ref.set_keys(k.bv_keys(), k.gsw_key())
        assert np.array_equal(out[j], ref.make_query(queries[j])), j
        assert np.array_equal(k.decrypt(out[j]), O.db_plaintext(c["db_seed"], idxs[j], op).astype(np.uint64))
        assert np.array_equal(out[j], srv.make_query(ids[j], queries[j]))


def test_k1p_device_batch_matches_host_batch():
    torch = pytest.importorskip("torch")
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_ragged_43_h5")
    qs = np.stack([q, q])
    want = srv.make_query_batch([7, 7], qs)
    stream = torch.cuda.Stream()   # a real stream: the call orders itself after it
    with torch.cuda.stream(stream):
        dq = torch.from_numpy(qs.view(np.int64)).cuda()
        dr = torch.zeros((2, 2, op.N), dtype=torch.int64, device="cuda")
        srv.make_query_batch_device([7, 7], dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
        got = dr.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, want)


def test_k1p_load_paths_agree():
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_ragged_43_h5")
    pts = np.stack([O.db_plaintext(c["db_seed"], i, op).astype(np.uint64) for i in range(c["target_num_pt"])])
    with PirServer(gp) as s2:
        s2.load_data(c["target_num_pt"], pts)
        s2.set_client_keys(7, bv, gsw)
        assert G.sha256(s2.make_query(7, q)) == c["sha256_response_u64"]
        s2.load_data(c["target_num_pt"], lambda i: pts[i])
        assert G.sha256(s2.make_query(7, q)) == c["sha256_response_u64"]


def test_k1p_errors_follow_the_reference():
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_ragged_43_h5")
    with pytest.raises(OutOfRange):
        srv.make_query(12345, q)
    bad = q.copy()
    bad[1, 3] = op.q                # not reduced mod q
    with pytest.raises(ValueError):
        srv.make_query(7, bad)
    with pytest.raises(ValueError):
        srv.make_query(7, q[:1])    # one polynomial only
    pts = np.zeros((2, op.N), np.uint64)
    pts[1, 5] = op.t
    with PirServer(gp) as s2:
        with pytest.raises(ValueError):
            s2.load_data(2, pts)
        with pytest.raises(RuntimeError):
            s2.make_query(7, q)     # before load_data
    with pytest.raises(ValueError):
        srv.set_client_keys(9, bv[:0], gsw, galois_ks=[])   # fewer keys than the height
    with pytest.raises(OutOfRange):                          # BvGaloisKeys::get
        srv.set_client_keys(9, bv, gsw, galois_ks=[3] * bv.shape[0])
    assert np.array_equal(srv.make_query(7, q), srv.make_query(7, q))


@pytest.mark.parametrize("batch", [3, 17, 40])
def test_k1p_batches_through_every_scan_tile_width(batch):
    """Batches of 3, 17 and 40 queries (one 16-column tile, two paired
    32-column tiles and three unpaired ones of the 64-bit-limb tensor-core
    scan) with the golden client inside: each answer
    equals the oracle's for its client and decrypts to its plaintext."""
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_1000_h7")
    ref = O.Server(op)
    ref.load_seeded(c["target_num_pt"], c["db_seed"])
    others = [O.Client(op, 700 + j) for j in range(2)]
    for j, k in enumerate(others):
        srv.set_client_keys(60 + j, k.bv_keys(), k.gsw_key())
    rng = np.random.default_rng(batch)
    ids, qs, idxs, owners = [], [], [], []
    for i in range(batch):
        if i == batch // 2:
            ids.append(7); qs.append(q); idxs.append(c["index"]); owners.append(cl)
            continue
        k = others[i % 2]
        idx = int(rng.integers(0, op.num_pt))
        ids.append(60 + i % 2); qs.append(k.query(idx)); idxs.append(idx); owners.append(k)
    out = srv.make_query_batch(ids, np.stack(qs))
    assert G.sha256(out[batch // 2]) == c["sha256_response_u64"]
    for i in range(batch):
        ref.set_keys(owners[i].bv_keys(), owners[i].gsw_key())
        assert np.array_equal(out[i], ref.make_query(qs[i])), i
        assert np.array_equal(owners[i].decrypt(out[i]), _plaintext_at(c, op, idxs[i]))


def _plaintext_at(c, op, idx):
    if idx < c["target_num_pt"]:
        return O.db_plaintext(c["db_seed"], idx, op).astype(np.uint64)
    return np.zeros(op.N, np.uint64)


def test_k1p_graph_replays_match_eager_launches(monkeypatch):
    """The two-limb pipeline captured as a CUDA graph (eager on first use,
    captured on the second, replayed after, also under stage timing) gives
    the eager responses and replays the same kernels."""
    from onionpirv2_b200.server import launch_count
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_1000_h7")
    monkeypatch.setenv("OPIR_GRAPHS", "0")
    eager = PirServer(gp)
    monkeypatch.delenv("OPIR_GRAPHS")
    graphed = PirServer(gp)
    clients = [cl, O.Client(op, 4242)]
    for s2 in (eager, graphed):
        s2.load_data_seeded(c["target_num_pt"], c["db_seed"])
        for i, k in enumerate(clients):
            s2.set_client_keys(i, k.bv_keys(), k.gsw_key())
    rng = np.random.default_rng(3)
    counts = {"eager": [], "graph": []}
    for rnd in range(5):
        if rnd == 3:
            eager.set_stage_timing(True)
            graphed.set_stage_timing(True)
        idx = [int(i) for i in rng.integers(0, op.num_pt, 2)]
        qs = np.stack([clients[i].query(idx[i]) for i in range(2)])
        l0 = launch_count()
        want = eager.make_query_batch([0, 1], qs)
        counts["eager"].append(launch_count() - l0)
        l0 = launch_count()
        got = graphed.make_query_batch([0, 1], qs)
        counts["graph"].append(launch_count() - l0)
        assert np.array_equal(got, want), rnd
        for i in range(2):
            assert np.array_equal(clients[i].decrypt(got[i]),
                                  O.db_plaintext(c["db_seed"], idx[i], op).astype(np.uint64))
    assert counts["graph"] == counts["eager"]
    st = graphed.stage_times()
    assert st["calls"] == 2 and st["Core"] > 0 and st["Other dim"] > 0
    eager.close()
    graphed.close()


def test_k1p_ext_prod_mux_matches_oracle():
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_1000_h7")
    exp = srv.expand_query(7, q)
    sel = srv.complete_selectors(7, exp)
    mid = srv.evaluate_first_dim(exp)
    for a, b, s in ((0, 1, 0), (3, 2, 1)):
        got = srv.ext_prod_mux(mid[a], mid[b], sel[s])
        assert np.array_equal(got, O.ext_prod_mux(op, mid[a], mid[b], sel[s]))


def test_k1p_stream_priority_leaves_results_unchanged():
    c, op, cl, bv, gsw, q, gp, srv = setup("k1p_1000_h7")
    srv.set_priority(-1)
    resp = srv.make_query(7, q)
    assert G.sha256(resp) == c["sha256_response_u64"]
    srv.set_priority(0)


@pytest.mark.parametrize("name", CASES)
def test_k1p_ntt_form_leaves_match_coefficient_leaves(name, monkeypatch):
    """make_query's last expansion level writes the first-dimension leaves
    in NTT form (sigma and X^-k in the NTT domain); OPIR_NTT_LEAVES=0 keeps
    every leaf in coefficient form and runs k1p_fst_ntt. Both give the
    golden response, single and batched (1 and 2 CTAs per SM), eager and
    replayed."""
    c, op, cl, bv, gsw, q, gp, _ = setup(name)
    qs = np.stack([q] * 40)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("OPIR_NTT_LEAVES", flag)
        with PirServer(gp) as srv:
            srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
            srv.set_client_keys(7, bv, gsw)
            for _ in range(3):
                r = srv.make_query(7, q)
                assert G.sha256(r) == c["sha256_response_u64"]
            out[flag] = [srv.make_query_batch([7] * 40, qs) for _ in range(2)]
    for a, b in zip(out["1"], out["0"]):
        for ra, rb in zip(a, b):
            assert np.array_equal(ra, rb)
            assert G.sha256(ra) == c["sha256_response_u64"]
    assert np.array_equal(cl.decrypt(out["1"][0][0]), _plaintext(c, op))
