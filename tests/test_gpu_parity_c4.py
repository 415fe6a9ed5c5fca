"""GPU parity for CONFIG_N4096_K2_MP (N = 4096, two 60-bit RNS limbs): the
CUDA path through the C ABI against the golden digests the reference itself
produced when built with that configuration (tests/golden/golden_c4.json),
stage by stage, and against the two-limb CPU oracle for batches of clients
the goldens do not cover. Integer work: every comparison is bit-exact."""
import functools

import numpy as np
import pytest

from onionpirv2_b200 import OutOfRange, PirParams, PirServer, save_response
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

C4 = "CONFIG_N4096_K2_MP"
CASES = [c["name"] for c in G.cases_c4()]


@functools.lru_cache(maxsize=None)
def setup(name):
    c = G.case_c4(name)
    op = O.c4_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    cl = O.C4Client(op, c["client_seed"])
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    q = cl.query(c["index"])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"], config=C4)
    srv = PirServer(gp)
    srv.load_data_seeded(c["target_num_pt"], c["db_seed"])
    srv.set_client_keys(7, bv, gsw)
    return c, op, cl, bv, gsw, q, gp, srv


def _plaintext(c, op):
    if c["index"] < c["target_num_pt"]:
        return O.c4_db_plaintext(c["db_seed"], c["index"], op)
    return np.zeros(op.N, np.uint64)


@pytest.mark.parametrize("name", CASES)
def test_c4_stages_match_reference(name):
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
def test_c4_make_query_matches_reference(name):
    c, op, cl, bv, gsw, q, gp, srv = setup(name)
    resp = srv.make_query(7, q)
    assert G.sha256(resp) == c["sha256_response_u64"]
    assert save_response(gp, resp) == G.stream(c)
    assert np.array_equal(cl.decrypt(resp), _plaintext(c, op))


def test_c4_batch_of_clients_matches_oracle():
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_2048_h7")
    rng = np.random.default_rng(11)
    clients, queries, ids, idxs = [], [], [], []
    for j in range(3):
        k = O.C4Client(op, 100 + j)
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
    ref = O.C4Server(op)
    ref.load_seeded(c["target_num_pt"], c["db_seed"])
    for j, k in enumerate(clients):
        ref.set_keys(k.bv_keys(), k.gsw_key())
        assert np.array_equal(out[j], ref.make_query(queries[j])), j
        assert np.array_equal(k.decrypt(out[j]), O.c4_db_plaintext(c["db_seed"], idxs[j], op))
        assert np.array_equal(out[j], srv.make_query(ids[j], queries[j]))


def test_c4_device_batch_matches_host_batch():
    torch = pytest.importorskip("torch")
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_ragged_43_h5")
    qs = np.stack([q, q])
    want = srv.make_query_batch([7, 7], qs)
    stream = torch.cuda.Stream()   # a real stream: the call orders itself after it
    with torch.cuda.stream(stream):
        dq = torch.from_numpy(qs.view(np.int64)).cuda()
        dr = torch.zeros((2, 2, op.N), dtype=torch.int64, device="cuda")
        srv.make_query_batch_device([7, 7], dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
        got = dr.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, want)


def test_c4_load_paths_agree():
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_ragged_43_h5")
    pts = np.stack([O.c4_db_plaintext(c["db_seed"], i, op) for i in range(c["target_num_pt"])])
    with PirServer(gp) as s2:
        s2.load_data(c["target_num_pt"], pts)
        s2.set_client_keys(7, bv, gsw)
        assert G.sha256(s2.make_query(7, q)) == c["sha256_response_u64"]
        s2.load_data(c["target_num_pt"], lambda i: pts[i])
        assert G.sha256(s2.make_query(7, q)) == c["sha256_response_u64"]


def test_c4_errors_follow_the_reference():
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_ragged_43_h5")
    with pytest.raises(OutOfRange):
        srv.make_query(12345, q)
    bad = q.copy()
    bad[1, 1, 3] = op.q[1]          # not reduced mod limb 1
    with pytest.raises(ValueError):
        srv.make_query(7, bad)
    with pytest.raises(ValueError):
        srv.make_query(7, q[:, 0])  # a one-limb ciphertext
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


def test_c4_full_size_batch_decrypts():
    """The benchmark layout itself (2^20 plaintexts, 64 GiB in NTT form, first
    dimension 1024 x 10 binary dimensions), beyond what the reference can run:
    genuine clients' queries, batched with repeats, must decrypt to the
    requested plaintexts, and a batch answer must equal the lone answer."""
    target, height = 1 << 20, 11
    op = O.c4_params(target, height)
    gp = PirParams(target, height, config=C4)
    assert (gp.fst_dim_sz, gp.num_dims, gp.other_dim_sz) == (1024, 11, 1024)
    seed = 424242
    clients = [O.C4Client(op, 9000 + j) for j in range(3)]
    rng = np.random.default_rng(77)
    idxs = [0, target - 1] + [int(i) for i in rng.integers(0, target, 2)]
    with PirServer(gp) as srv:
        srv.load_data_seeded(target, seed)
        for j, cl in enumerate(clients):
            srv.set_client_keys(j, cl.bv_keys(), cl.gsw_key())
        owner = [0, 1, 2, 0]
        queries = np.stack([clients[o].query(i) for o, i in zip(owner, idxs)])
        out = srv.make_query_batch(owner, queries)
        for k, (o, i) in enumerate(zip(owner, idxs)):
            assert np.array_equal(clients[o].decrypt(out[k]), O.c4_db_plaintext(seed, i, op)), i
        assert np.array_equal(out[1], srv.make_query(owner[1], queries[1]))


def test_c4_graph_replays_match_eager_launches(monkeypatch):
    """The two-limb pipeline captured as a CUDA graph (eager on first use,
    captured on the second, replayed after, also under stage timing) gives
    the eager responses and replays the same kernels."""
    from onionpirv2_b200.server import launch_count
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_2048_h7")
    monkeypatch.setenv("OPIR_GRAPHS", "0")
    eager = PirServer(gp)
    monkeypatch.delenv("OPIR_GRAPHS")
    graphed = PirServer(gp)
    clients = [cl, O.C4Client(op, 4242)]
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
                                  O.c4_db_plaintext(c["db_seed"], idx[i], op))
    assert counts["graph"] == counts["eager"]
    st = graphed.stage_times()
    assert st["calls"] == 2 and st["Core"] > 0 and st["Other dim"] > 0
    eager.close()
    graphed.close()


def test_c4_ext_prod_mux_matches_oracle():
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_2048_h7")
    exp = srv.expand_query(7, q)
    sel = srv.complete_selectors(7, exp)
    mid = srv.evaluate_first_dim(exp)
    for a, b, s in ((0, 1, 0), (3, 2, 1)):
        got = srv.ext_prod_mux(mid[a], mid[b], sel[s])
        assert np.array_equal(got, O.ext_prod_mux(op, mid[a], mid[b], sel[s]))


def test_c4_stream_priority_leaves_results_unchanged():
    c, op, cl, bv, gsw, q, gp, srv = setup("c4_2048_h7")
    srv.set_priority(-1)
    resp = srv.make_query(7, q)
    assert G.sha256(resp) == c["sha256_response_u64"]
    srv.set_priority(0)


@pytest.mark.parametrize("name", CASES)
def test_c4_ntt_form_leaves_match_coefficient_leaves(name, monkeypatch):
    """make_query's last expansion level writes the first-dimension leaves
    in NTT form (sigma and X^-k in the NTT domain); OPIR_NTT_LEAVES=0 keeps
    every leaf in coefficient form and runs k4_fst_ntt. Both give the
    golden response, single and batched, eager and replayed."""
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
                assert G.sha256(r) == c["sha256_response_u64"]
            out[flag] = [srv.make_query_batch([7, 7, 7], qs) for _ in range(3)]
    for a, b in zip(out["1"], out["0"]):
        for ra, rb in zip(a, b):
            assert np.array_equal(ra, rb)
            assert G.sha256(ra) == c["sha256_response_u64"]
    assert np.array_equal(cl.decrypt(out["1"][0][0]), _plaintext(c, op))
