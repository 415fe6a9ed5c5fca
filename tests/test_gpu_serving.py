"""GPU test of the continuous-batching request loop.

Three device-resident databases of different layouts receive seeded Poisson
arrivals from several clients each (plus an initial burst so that batches
form). Every response is checked bit for bit against the same query answered
alone, and decrypted by its client to the requested plaintext; the golden
query of the reference-generated cases is mixed in and must still match the
reference's response.
"""
import threading
import time

import numpy as np
import pytest

from oracle import oracle as O
from tests import golden_cases as G

pytestmark = pytest.mark.gpu

LAYOUTS = {"small_1000_h7": 4, "c1_16384_h9": 3, "ragged_43_h5": 2}  # case -> clients


def test_mixed_arrivals_match_single_queries():
    from onionpirv2_b200 import PirParams
    from onionpirv2_b200.serving import ServingEngine

    eng = ServingEngine(depth=2)
    clients = {}
    for name, k in LAYOUTS.items():
        c = G.case(name)
        gp = PirParams(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
        eng.add_database(name, gp, max_batch=8, seed=c["db_seed"], min_fill=2)
        op = O.params(c["target_num_pt"], c["expansion_height"], c["fst_dim_pow2"])
        cls = [O.Client(op, c["client_seed"])] + [O.Client(op, 500 + j) for j in range(1, k)]
        for j, cl in enumerate(cls):
            eng.register_client(name, j, cl.bv_keys(), cl.gsw_key())
        clients[name] = (c, op, cls)

    rng = np.random.default_rng(11)
    plan = []                      # (t_offset, name, client, index)
    names = list(LAYOUTS)
    t = 0.0
    for i in range(60):
        t += 0 if i < 12 else rng.exponential(1 / 400)
        name = names[int(rng.choice(3, p=[0.6, 0.3, 0.1]))]
        c, op, cls = clients[name]
        j = int(rng.integers(0, len(cls)))
        plan.append((t, name, j, int(rng.integers(0, c["target_num_pt"]))))
    for name in names:             # the golden query of each case, in the mix
        c, op, cls = clients[name]
        plan.append((plan[-1][0] + 0.001, name, 0, c["index"]))
    queries = [clients[n][2][j].query(idx) for _, n, j, idx in plan[:-3]]
    for _, name, _, idx in plan[-3:]:  # first query of a fresh client: the golden one
        c, op, _ = clients[name]
        fresh = O.Client(op, c["client_seed"])
        fresh.bv_keys(), fresh.gsw_key()
        queries.append(fresh.query(idx))

    futures = [None] * len(plan)
    eng.start()

    def submitter():
        t0 = time.perf_counter()
        for k, (off, name, j, _idx) in enumerate(plan):
            while time.perf_counter() - t0 < off:
                time.sleep(0.0002)
            futures[k] = eng.submit(name, j, queries[k])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    eng.drain(timeout=300)
    got = [f.result(timeout=10) for f in futures]
    eng.stop()

    sizes = [n for _, n, _, _ in eng.batch_log]
    assert max(sizes) > 1, "no batch formed"
    for k, (_, name, j, idx) in enumerate(plan):
        c, op, cls = clients[name]
        alone = eng.dbs[name].lane.server.make_query(j, queries[k])
        assert np.array_equal(got[k], alone), (name, j, idx)
        want = (O.db_plaintext(c["db_seed"], idx, op) if idx < c["target_num_pt"]
                else np.zeros(op.N, np.uint16))
        assert np.array_equal(cls[j].decrypt(got[k]), want.astype(np.uint64))
    for k in range(len(plan) - 3, len(plan)):
        name = plan[k][1]
        assert G.sha256(got[k]) == clients[name][0]["sha256_response_u64"]
    st = eng.stats()
    assert st["completed"] == len(plan)
    assert st["p99_ms"] >= st["p50_ms"] > 0
    eng.close()


def test_admission_refuses_over_budget_before_allocating():
    import torch
    from onionpirv2_b200 import PirParams
    from onionpirv2_b200.serving import ServingEngine

    gp = PirParams(16384, 9)
    eng = ServingEngine(hbm_budget_bytes=64 << 20)   # below the 256 MiB database
    before = torch.cuda.mem_get_info()[0]
    with pytest.raises(MemoryError):
        eng.add_database("c1", gp, max_batch=8, seed=1)
    assert eng.reserved == 0 and not eng.dbs
    assert torch.cuda.mem_get_info()[0] >= before - (8 << 20)
    eng.close()


def test_two_parameter_sets_share_one_engine():
    """A CONFIG_N2048_K1_COMP and a CONFIG_N4096_K2_MP database served side
    by side: every response equals the query answered alone and decrypts to
    the requested plaintext; the two-limb golden query matches the reference."""
    from onionpirv2_b200 import PirParams
    from onionpirv2_b200.serving import ServingEngine

    eng = ServingEngine(depth=2)
    c1 = G.case("c1_16384_h9")
    op1 = O.params(c1["target_num_pt"], c1["expansion_height"], c1["fst_dim_pow2"])
    eng.add_database("k1", PirParams(c1["target_num_pt"], c1["expansion_height"]), max_batch=8,
                     seed=c1["db_seed"], min_fill=2)
    c4 = G.case_c4("c4_2048_h7")
    op4 = O.c4_params(c4["target_num_pt"], c4["expansion_height"], c4["fst_dim_pow2"])
    eng.add_database("c4", PirParams(c4["target_num_pt"], c4["expansion_height"],
                                     config="CONFIG_N4096_K2_MP"),
                     max_batch=4, seed=c4["db_seed"], min_fill=2)
    k1_clients = [O.Client(op1, 700 + j) for j in range(2)]
    c4_clients = [O.C4Client(op4, c4["client_seed"])] + [O.C4Client(op4, 800 + j) for j in range(2)]
    for j, cl in enumerate(k1_clients):
        eng.register_client("k1", j, cl.bv_keys(), cl.gsw_key())
    for j, cl in enumerate(c4_clients):
        eng.register_client("c4", j, cl.bv_keys(), cl.gsw_key())

    rng = np.random.default_rng(23)
    jobs = []   # (db, client index, plaintext index, query)
    jobs.append(("c4", 0, c4["index"], c4_clients[0].query(c4["index"])))  # the golden query
    for i in range(24):
        if i % 2:
            j, idx = int(rng.integers(0, 2)), int(rng.integers(0, op1.num_pt))
            jobs.append(("k1", j, idx, k1_clients[j].query(idx)))
        else:
            j, idx = int(rng.integers(1, 3)), int(rng.integers(0, op4.num_pt))
            jobs.append(("c4", j, idx, c4_clients[j].query(idx)))
    eng.start()
    futures = [eng.submit(db, j, q) for db, j, _, q in jobs]
    eng.drain(timeout=300)
    got = [f.result(timeout=10) for f in futures]
    eng.stop()
    assert G.sha256(got[0]) == c4["sha256_response_u64"]
    for k, (db, j, idx, q) in enumerate(jobs):
        alone = eng.dbs[db].lane.server.make_query(j, q)
        assert np.array_equal(got[k], alone), (db, j, idx)
        if db == "k1":
            want = O.db_plaintext(c1["db_seed"], idx, op1).astype(np.uint64)
            assert np.array_equal(k1_clients[j].decrypt(got[k]), want)
        else:
            want = O.c4_db_plaintext(c4["db_seed"], idx, op4)
            assert np.array_equal(c4_clients[j].decrypt(got[k]), want)
    assert max(n for _, n, _, _ in eng.batch_log) > 1
    eng.close()
