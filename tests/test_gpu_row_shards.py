"""GPU parity of row shards (one database split by candidate rows over G
shards, opir_server_create_row_shard): every shard's partial ciphertext
against the oracle's restatement of the reference's MUX tree
(src/server.cpp:599-649) cut at level h - log2 G, and the combined
responses against the reference-generated goldens. The G shards run one
after another on one GPU (no kernel waits on another shard); the
multi-process gather is covered on CPU in test_row_shards.py."""
import functools

import numpy as np
import pytest
import torch

from onionpirv2_b200 import PirParams, PirServer, RowShardServer, save_response
from onionpirv2_b200.server import _ptr
from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

C4 = "CONFIG_N4096_K2_MP"


def shard_counts(p, limit=None):
    """Every valid shard count (1 .. 2^(h-1)), or those of `limit`."""
    h = p.num_dims - 1
    out, g = [], 1
    while g <= 1 << (h - 1):
        out.append(g)
        g *= 2
    return [g for g in out if g in limit] if limit else out


def run_shards(gp, G_, load, keys, ids, queries):
    """The G shards of gp answer the batch; returns (partials, responses)."""
    shards = [RowShardServer(gp, g, G_) for g in range(G_)]
    for s in shards:
        load(s)
        for cid, (bv, gsw) in keys.items():
            s.set_client_keys(cid, bv, gsw)
    partials = np.stack([s.make_query_shard_batch(ids, queries) for s in shards])
    resp = shards[G_ - 1].combine_shards(ids, partials)
    for s in shards:
        s.close()
    return partials, resp


@functools.lru_cache(maxsize=None)
def golden_setup(name):
    c = G.case(name)
    op = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    cl = O.Client(op, c["client_seed"])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    return c, op, cl, gp, cl.query(c["index"])


def _check_golden(c, cl, op, gp, resp):
    assert G.sha256(resp) == c["sha256_response_u64"]
    assert save_response(gp, resp) == G.stream(c)
    want = (O.db_plaintext(c["db_seed"], c["index"], op) if c["index"] < c["target_num_pt"]
            else np.zeros(op.N, np.uint16))
    assert np.array_equal(cl.decrypt(resp), want.astype(np.uint64))


@pytest.mark.parametrize("name,limit", [
    ("c1_16384_h9", None), ("ragged_43_h5_pad", None), ("small_1000_h7", None),
    ("flat_349526_h10", (1, 4, 64)), ("c2_262144_h10", (2, 32))])
def test_sharded_response_matches_reference(name, limit):
    c, op, cl, gp, q = golden_setup(name)
    keys = {7: (cl.bv_keys(), cl.gsw_key())}
    for G_ in shard_counts(gp, limit):
        _, resp = run_shards(gp, G_, lambda s: s.load_data_seeded(c["target_num_pt"], c["db_seed"]),
                             keys, [7], q[None])
        _check_golden(c, cl, op, gp, resp[0])


def test_partials_match_oracle_tree():
    """Each shard's partial = the reference tree's level-(h - log2 G)
    position g, for a batch of two clients."""
    c, op, cl, gp, q = golden_setup("c1_16384_h9")
    srv = O.Server(op)
    srv.load_seeded(c["target_num_pt"], c["db_seed"])
    clients = [O.Client(op, 300 + j) for j in range(2)]
    idxs = [123, 16383]
    queries = np.stack([k.query(i) for k, i in zip(clients, idxs)])
    stages = []
    for k, qq in zip(clients, queries):
        srv.set_keys(k.bv_keys(), k.gsw_key())
        e = srv.expand(qq)
        stages.append((srv.complete_selectors(e), srv.first_dim(e), srv.make_query(qq)))
    keys = {10 + j: (k.bv_keys(), k.gsw_key()) for j, k in enumerate(clients)}
    for G_ in (1, 2, 8, 32):
        partials, resp = run_shards(gp, G_, lambda s: s.load_data_seeded(c["target_num_pt"],
                                                                          c["db_seed"]),
                                    keys, [10, 11], queries)
        for j, (sel, mid, full) in enumerate(stages):
            want_parts, _ = O.sharded_other_dim(op, mid, sel, G_)
            assert np.array_equal(partials[:, j], want_parts), (G_, j)
            assert np.array_equal(resp[j], full)
            assert np.array_equal(clients[j].decrypt(resp[j]),
                                  O.db_plaintext(c["db_seed"], idxs[j], op).astype(np.uint64))


def test_device_entry_points_match_host():
    c, op, cl, gp, q = golden_setup("c1_16384_h9")
    G_ = 4
    shards = [RowShardServer(gp, g, G_) for g in range(G_)]
    bv, gsw = cl.bv_keys(), cl.gsw_key()
    queries = np.stack([q, q])
    ids = [7, 8]
    for s in shards:
        s.load_data_seeded(c["target_num_pt"], c["db_seed"])
        for cid in ids:
            s.set_client_keys(cid, bv, gsw)
    dev = torch.device("cuda", 0)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        d_q = torch.from_numpy(queries.view(np.int64)).to(dev)
        d_parts = torch.empty((G_, 2) + gp.ct_shape, dtype=torch.int64, device=dev)
        for g, s in enumerate(shards):
            s.make_query_shard_batch_device(ids, d_q.data_ptr(), d_parts[g].data_ptr(),
                                            st.cuda_stream)
        d_resp = torch.empty((2, 2, gp.N), dtype=torch.int64, device=dev)
        shards[0].combine_shards_device(ids, d_parts.data_ptr(), d_resp.data_ptr(), st.cuda_stream)
    st.synchronize()
    resp = d_resp.cpu().numpy().view(np.uint64)
    for j in range(2):
        _check_golden(c, cl, op, gp, resp[j])
    for s in shards:
        s.close()


def test_shard_loads_from_array_and_source():
    name = "ragged_43_h5"
    c, op, cl, gp, q = golden_setup(name)
    rng = np.random.default_rng(5)
    db = rng.integers(0, op.t, size=(c["target_num_pt"], op.N), dtype=np.uint64)
    whole = PirServer(gp)
    whole.load_data(c["target_num_pt"], db)
    whole.set_client_keys(7, cl.bv_keys(), cl.gsw_key())
    want = whole.make_query(7, q)
    keys = {7: (cl.bv_keys(), cl.gsw_key())}
    asked = []

    def source(i):
        asked.append(i)
        return db[i]

    for load in (lambda s: s.load_data(c["target_num_pt"], db),
                 lambda s: s.load_data(c["target_num_pt"], db.astype(np.uint16)),
                 lambda s: s.load_data(c["target_num_pt"], source)):
        _, resp = run_shards(gp, 2, load, keys, [7], q[None])
        assert np.array_equal(resp[0], want)
    # the source is asked for each shard's plaintexts only, in increasing order
    assert sorted(asked) == list(range(c["target_num_pt"]))
    assert np.array_equal(cl.decrypt(want), db[42])


def test_shard_view_refusals():
    c, op, cl, gp, q = golden_setup("c1_16384_h9")
    s = RowShardServer(gp, 0, 2)
    s.load_data_seeded(c["target_num_pt"], c["db_seed"])
    s.set_client_keys(7, cl.bv_keys(), cl.gsw_key())
    with pytest.raises(ValueError):
        s.make_query(7, q)
    with pytest.raises(ValueError):   # no batch yet
        s.combine_shards([7], np.zeros((2, 1) + gp.ct_shape, np.uint64))
    part = s.make_query_shard_batch([7], q[None])
    with pytest.raises(ValueError):   # not the ids of the last batch
        s.combine_shards([8], np.stack([part, part]))
    whole = PirServer(gp)
    ids = np.array([7], np.uint64)
    out = np.zeros((1,) + gp.ct_shape, np.uint64)
    with pytest.raises(ValueError):   # a whole layout has no shard calls
        whole._check(whole._lib.opir_server_make_query_shard_batch(
            whole._h, 1, _ptr(ids), _ptr(np.ascontiguousarray(q)), _ptr(out)))
    with pytest.raises(ValueError):
        RowShardServer(gp, 2, 2)
    with pytest.raises(ValueError):
        RowShardServer(gp.with_query_shape(8, 2, 7), 0, 2)


@functools.lru_cache(maxsize=None)
def c4_setup(name):
    c = G.case_c4(name)
    op = O.c4_params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
    cl = O.C4Client(op, c["client_seed"])
    gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"], config=C4)
    return c, op, cl, gp, cl.query(c["index"])


@pytest.mark.parametrize("name", ["c4_2048_h7", "c4_ragged_43_h5", "c4_tight_100_h6"])
def test_c4_sharded_matches_reference(name):
    c, op, cl, gp, q = c4_setup(name)
    keys = {7: (cl.bv_keys(), cl.gsw_key())}
    for G_ in shard_counts(gp):
        partials, resp = run_shards(gp, G_, lambda s: s.load_data_seeded(c["target_num_pt"],
                                                                          c["db_seed"]),
                                    keys, [7], q[None])
        assert partials.shape == (G_, 1) + gp.ct_shape
        assert G.sha256(resp[0]) == c["sha256_response_u64"]
        assert save_response(gp, resp[0]) == G.stream(c)


def test_c4_partials_match_oracle_tree():
    c, op, cl, gp, q = c4_setup("c4_2048_h7")
    srv = O.C4Server(op)
    srv.load_seeded(c["target_num_pt"], c["db_seed"])
    srv.set_keys(cl.bv_keys(), cl.gsw_key())
    e = srv.expand(q)
    sel, mid = srv.complete_selectors(e), srv.first_dim(e)
    keys = {7: (cl.bv_keys(), cl.gsw_key())}
    for G_ in (2, 4):
        partials, _ = run_shards(gp, G_, lambda s: s.load_data_seeded(c["target_num_pt"],
                                                                       c["db_seed"]),
                                 keys, [7], q[None])
        want, _ = O.sharded_other_dim(op, mid, sel, G_)
        assert np.array_equal(partials[:, 0], want)
