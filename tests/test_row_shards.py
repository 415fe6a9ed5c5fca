"""Row shards (one database across GPUs), host side: the library's row
partition (opir_row_shard_rows) against the oracle's restatement, the
oracle's sharded MUX tree against the reference's evaluate_other_dim
(src/server.cpp:599-649), and the two-rank orchestration in
onionpirv2_b200/sharded.py over gloo with an oracle-computed shard engine."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from onionpirv2_b200 import PirParams, row_shard_rows
from oracle import oracle as O

LAYOUTS = [(16384, 9, True), (349526, 10, True), (1000, 7, True), (43, 5, True), (5000, 8, False)]


@pytest.mark.parametrize("layout", LAYOUTS)
def test_partition_matches_oracle(layout):
    p = PirParams(*layout)
    h = p.num_dims - 1
    G = 1
    while G <= 1 << (h - 1):
        seen = []
        for g in range(G):
            rows, tree_h = row_shard_rows(p, g, G)
            assert list(rows) == O.shard_rows(p.other_dim_sz, p.num_dims, g, G)
            assert tree_h == h - (G.bit_length() - 1)
            # a shard is itself a layout of height tree_h
            assert (1 << (tree_h - 1)) <= len(rows) <= (1 << tree_h)
            seen += list(rows)
        assert sorted(seen) == list(range(p.other_dim_sz))
        G *= 2
    for bad in ((0, G), (0, 3), (0, 0), (G // 2, G // 2)):
        with pytest.raises(ValueError):
            row_shard_rows(p, *bad)


def test_c4_partition():
    p = PirParams(1 << 14, 9, config="CONFIG_N4096_K2_MP")
    rows, tree_h = row_shard_rows(p, 1, 4)
    assert tree_h == p.num_dims - 1 - 2
    assert list(rows) == O.shard_rows(p.other_dim_sz, p.num_dims, 1, 4)


def _oracle_stages(layout, seed_db=7, seed_client=11, idx=5):
    p = O.params(*layout)
    srv = O.Server(p)
    srv.load_seeded(layout[0], seed_db)
    cl = O.Client(p, seed_client)
    srv.set_keys(cl.bv_keys(), cl.gsw_key())
    q = cl.query(idx)
    e = srv.expand(q)
    return p, srv, srv.complete_selectors(e), srv.first_dim(e)


@pytest.mark.parametrize("layout", [(16384, 9, True), (43, 5, True)])
def test_oracle_sharded_tree_equals_full(layout):
    p, srv, sel, mid = _oracle_stages(layout)
    full = srv.other_dim(mid, sel)
    G = 1
    while G <= 1 << (p.num_dims - 2):
        parts, res = O.sharded_other_dim(p, mid, sel, G)
        assert parts.shape[0] == G
        assert np.array_equal(res, full), G
        G *= 2


class OracleShardEngine:
    """One rank's shard computed by the oracle (checker only)."""

    def __init__(self, layout, shard, num_shards, seed_db):
        self.p = O.params(*layout)
        self.layout = layout
        self.shard, self.num_shards = shard, num_shards
        self.srv = O.Server(self.p)
        self.keys = {}
        self.sel = {}
        self.seed_db = seed_db

    def load_data_seeded(self, logical, seed):
        self.srv.load_seeded(logical, seed)

    def set_client_keys(self, cid, bv, gsw):
        self.keys[cid] = (bv, gsw)

    def make_query_shard_batch(self, ids, queries):
        p = self.p
        h = p.num_dims - 1
        k = self.num_shards.bit_length() - 1
        rows = O.shard_rows(p.other_dim_sz, p.num_dims, self.shard, self.num_shards)
        out = []
        for cid, q in zip(ids, queries):
            self.srv.set_keys(*self.keys[cid])
            e = self.srv.expand(q)
            sel = self.srv.complete_selectors(e)
            mid = self.srv.first_dim(e)
            self.sel[cid] = sel
            out.append(O.mux_levels(p, mid[rows], sel, h - k, 0, h - k)[0])
        return np.stack(out)

    def combine_shards(self, ids, stacked):
        p = self.p
        h = p.num_dims - 1
        k = self.num_shards.bit_length() - 1
        resp = []
        for i, cid in enumerate(ids):
            ct = O.mux_levels(p, stacked[:, i], self.sel[cid], h, h - k, h)[0].copy()
            O.lib().oracle_mod_switch(O.C.byref(p), O.ptr(ct))
            resp.append(ct)
        return np.stack(resp)


LAYOUT = (16384, 9, True)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from onionpirv2_b200.sharded import ShardedServer
        engine = OracleShardEngine(LAYOUT, rank, world, 7)
        srv = ShardedServer(PirParams(LAYOUT[0], LAYOUT[1]), engine=engine)
        srv.load_data_seeded(LAYOUT[0], 7)
        p = engine.p
        clients = {cid: O.Client(p, 100 + cid) for cid in (3, 9)}
        for cid, cl in clients.items():
            srv.set_client_keys(cid, cl.bv_keys(), cl.gsw_key())
        idxs = [5, 16000]
        queries = np.stack([clients[c].query(i) for c, i in zip((3, 9), idxs)])
        resp = srv.make_query_batch([3, 9], queries)
        if rank == 0:
            full = O.Server(p)
            full.load_seeded(LAYOUT[0], 7)
            ok = []
            for j, (cid, i) in enumerate(zip((3, 9), idxs)):
                full.set_keys(clients[cid].bv_keys(), clients[cid].gsw_key())
                want = full.make_query(queries[j])
                dec = clients[cid].decrypt(resp[j])
                ok.append(bool(np.array_equal(resp[j], want)) and
                          bool(np.array_equal(dec, O.db_plaintext(7, i, p).astype(np.uint64))))
            out["ok"] = ok
        else:
            out["other"] = resp is None
    finally:
        dist.destroy_process_group()


def test_sharded_server_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = 29700 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    assert out["ok"] == [True, True]
    assert out["other"] is True
