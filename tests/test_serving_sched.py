"""Host-side tests of the continuous-batching request loop (no GPU).

The device lane is replaced by a fake whose batches "finish" after a fixed
delay and whose answer is a fixed function of (client, query), so routing,
batch formation, overlap across databases, HBM admission and error paths are
checked on the CPU. The GPU form of the same loop is in test_gpu_serving.py.
"""
import threading
import time

import numpy as np
import pytest

from onionpirv2_b200 import PirParams, plan_memory
from onionpirv2_b200.serving import ServingEngine

N = 2048


class FakeLane:
    def __init__(self, params, max_batch, depth, seed, plaintexts, delay=0.004):
        self.max_batch = max_batch
        self.delay = delay
        self.launched = [None] * depth
        self.out = [None] * depth
        self.keys = set()
        self.closed = False

    def set_client_keys(self, cid, bv, gsw):
        self.keys.add(cid)

    def launch(self, slot, client_ids, queries):
        assert len(client_ids) <= self.max_batch
        if any(c not in self.keys for c in client_ids):
            raise IndexError("unknown client id")
        self.out[slot] = np.stack([q ^ np.uint64(c) for c, q in zip(client_ids, queries)])
        self.launched[slot] = time.perf_counter()

    def done(self, slot):
        return time.perf_counter() - self.launched[slot] >= self.delay

    def results(self, slot, n):
        return self.out[slot][:n].copy()

    def close(self):
        self.closed = True


def make_engine(budget=1 << 40, depth=2, delay=0.004):
    return ServingEngine(hbm_budget_bytes=budget, depth=depth,
                         lane_factory=lambda p, mb, d, s, pts: FakeLane(p, mb, d, s, pts, delay))


def query(rng):
    return rng.integers(0, 1 << 57, size=(2, N), dtype=np.uint64)


SMALL = PirParams(1000, 7)
MID = PirParams(16384, 9)


def test_memory_plan_matches_layout():
    p = PirParams(262144, 10)
    plan = plan_memory(p)
    # byte-plane database: 2 residues x N levels x 4 byte planes x 512 x 512
    assert plan["database_bytes"] == 2 * N * 4 * 512 * 512 + 16 * N * 4 + 4
    # 10 BV keys x 8 rows x (b, a) + 20 RGSW rows x (c0, c1), residue pairs of u32
    assert plan["client_key_bytes"] == (10 * 8 * 2 * N + 20 * 2 * N) * 2 * 4
    assert plan["scratch_bytes_per_query"] > 0
    small = plan_memory(SMALL)
    assert small["database_bytes"] < plan["database_bytes"]
    assert small["scratch_bytes_per_query"] < plan["scratch_bytes_per_query"]


def test_every_request_gets_its_own_answer_across_databases():
    eng = make_engine()
    eng.add_database("a", SMALL, max_batch=8)
    eng.add_database("b", MID, max_batch=4)
    for c in range(6):
        eng.register_client("a", c, None, None)
        eng.register_client("b", 100 + c, None, None)
    eng.start()
    rng = np.random.default_rng(1)
    subs = []
    for i in range(200):
        name, cid = ("a", i % 6) if i % 3 else ("b", 100 + i % 6)
        q = query(rng)
        subs.append((q, cid, eng.submit(name, cid, q)))
        if i % 17 == 0:
            time.sleep(0.002)
    eng.drain(timeout=60)
    for q, cid, f in subs:
        assert np.array_equal(f.result(timeout=1), q ^ np.uint64(cid))
    st = eng.stats()
    assert st["completed"] == 200
    assert st["databases"]["a"]["completed"] + st["databases"]["b"]["completed"] == 200
    assert all(n <= 8 for nm, n, _, _ in eng.batch_log if nm == "a")
    assert all(n <= 4 for nm, n, _, _ in eng.batch_log if nm == "b")
    eng.close()


def test_requests_arriving_during_a_batch_join_the_next_batches():
    eng = make_engine(depth=2, delay=0.05)
    eng.add_database("a", SMALL, max_batch=16, min_fill=4)
    eng.register_client("a", 1, None, None)
    eng.start()
    rng = np.random.default_rng(2)
    first = eng.submit("a", 1, query(rng))
    time.sleep(0.01)                         # first batch (1 query) is on the "device"
    rest = [eng.submit("a", 1, query(rng)) for _ in range(12)]
    eng.drain(timeout=30)
    first.result(timeout=1)
    [f.result(timeout=1) for f in rest]
    sizes = [n for _, n, _, _ in eng.batch_log]
    assert sizes[0] == 1
    assert sum(sizes) == 13 and len(sizes) <= 3 and max(sizes[1:]) > 1
    # a second batch was enqueued while the first was still running
    (_, _, l0, d0), (_, _, l1, _d1) = eng.batch_log[0], eng.batch_log[1]
    assert l1 < d0
    eng.close()


def test_databases_overlap_on_the_device():
    eng = make_engine(depth=1, delay=0.03)
    eng.add_database("a", SMALL, max_batch=4)
    eng.add_database("b", SMALL, max_batch=4)
    eng.register_client("a", 1, None, None)
    eng.register_client("b", 1, None, None)
    eng.start()
    rng = np.random.default_rng(3)
    fs = [eng.submit(n, 1, query(rng)) for n in ("a", "b")]
    eng.drain(timeout=30)
    [f.result(timeout=1) for f in fs]
    la = [x for x in eng.batch_log if x[0] == "a"][0]
    lb = [x for x in eng.batch_log if x[0] == "b"][0]
    assert la[2] < lb[3] and lb[2] < la[3]   # the two batches' lifetimes intersect
    eng.close()


def test_hbm_budget_admission():
    need_small = ServingEngine(hbm_budget_bytes=1 << 40, depth=2,
                               lane_factory=lambda *a: FakeLane(*a)).database_bytes(SMALL, 8)
    key = plan_memory(SMALL)["client_key_bytes"]
    eng = make_engine(budget=need_small + 2 * key)
    with pytest.raises(MemoryError):
        eng.add_database("big", MID, max_batch=8)
    assert eng.reserved == 0
    eng.add_database("a", SMALL, max_batch=8)
    eng.register_client("a", 1, None, None)
    eng.register_client("a", 1, None, None)  # re-registering reserves nothing new
    eng.register_client("a", 2, None, None)
    with pytest.raises(MemoryError):
        eng.register_client("a", 3, None, None)
    assert eng.reserved == need_small + 2 * key
    eng.close()


def test_errors_are_per_request():
    eng = make_engine()
    eng.add_database("a", SMALL, max_batch=4)
    eng.register_client("a", 1, None, None)
    rng = np.random.default_rng(4)
    assert isinstance(eng.submit("a", 1, query(rng)).exception(timeout=1), RuntimeError)  # not started
    eng.start()
    assert isinstance(eng.submit("zz", 1, query(rng)).exception(timeout=1), KeyError)
    assert isinstance(eng.submit("a", 9, query(rng)).exception(timeout=1), IndexError)
    assert isinstance(eng.submit("a", 1, np.zeros(5, np.uint64)).exception(timeout=1), ValueError)
    ok = eng.submit("a", 1, query(rng))
    eng.drain(timeout=10)
    assert ok.exception(timeout=1) is None
    eng.close()


def test_concurrent_submitters():
    eng = make_engine(delay=0.002)
    eng.add_database("a", SMALL, max_batch=32)
    for c in range(4):
        eng.register_client("a", c, None, None)
    eng.start()
    results = {}

    def worker(c):
        rng = np.random.default_rng(10 + c)
        out = []
        for _ in range(50):
            q = query(rng)
            out.append((q, eng.submit("a", c, q)))
        results[c] = out

    ts = [threading.Thread(target=worker, args=(c,)) for c in range(4)]
    [t.start() for t in ts]
    [t.join() for t in ts]
    eng.drain(timeout=60)
    for c, out in results.items():
        for q, f in out:
            assert np.array_equal(f.result(timeout=1), q ^ np.uint64(c))
    assert eng.stats()["completed"] == 200
    eng.close()
