"""Continuous-batching request loop over several device-resident databases.

Requests (database, client, query) arrive at any time from any thread. A
scheduler thread keeps one queue per database. Each database owns a lane: its
server handle (database, client keys and scratch arena in HBM), a CUDA stream
and `depth` sets of pinned-host / device query and response buffers. Whenever
a lane has a free slot the scheduler forms a batch from what has arrived for
that database (up to its batch limit) and enqueues it at once: upload, the
library's batched make_query (one first-dimension scan for the whole batch),
download, and an event. Lanes of different databases run concurrently on
their own streams, and a second batch of the same database is enqueued behind
the running one when enough requests are waiting, so the device does not
idle between batches. Completed batches resolve their requests' futures as
soon as their event fires; requests that arrive meanwhile join the next batch.

Admission is by HBM budget, from the library's own memory plan
(opir_plan_memory): a database is admitted with its database bytes, its
scratch arena for max_batch queries (reserved up front, so no query ever
waits on the CUDA allocator) and the lane buffers; a client with its key
bytes. Anything that does not fit is refused with MemoryError before any
device allocation. Latency is measured per request from submission to the
response landing in host memory; stats() reports p50/p99 and queries/s.

This module is host-side orchestration; every arithmetic step runs in the
library's kernels.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass

import numpy as np

from .server import PirParams, PirServer, plan_memory


@dataclass
class _Request:
    client_id: int
    query: np.ndarray
    future: Future
    t_submit: float


class CudaLane:
    """Device side of one database: server handle, stream, `depth` buffer sets."""

    def __init__(self, params: PirParams, max_batch: int, depth: int, device: int,
                 seed: int | None, plaintexts):
        import torch
        self.torch = torch
        dev = torch.device("cuda", device)
        self.server = PirServer(params, device=device)
        if plaintexts is not None:
            self.server.load_data(len(plaintexts), plaintexts)
        else:
            self.server.load_data_seeded(params.target_num_pt, 0 if seed is None else seed)
        self.server.reserve(max_batch)
        self.stream = torch.cuda.Stream(dev)
        qshape = (max_batch,) + params.ct_shape      # (2, N) or (2, K, N)
        rshape = (max_batch, 2, params.N)            # responses mod small_q
        self.d_q = [torch.empty(qshape, dtype=torch.int64, device=dev) for _ in range(depth)]
        self.d_r = [torch.empty(rshape, dtype=torch.int64, device=dev) for _ in range(depth)]
        self.h_q = [torch.empty(qshape, dtype=torch.int64).pin_memory() for _ in range(depth)]
        self.h_r = [torch.empty(rshape, dtype=torch.int64).pin_memory() for _ in range(depth)]
        self.events = [None] * depth

    @staticmethod
    def buffer_bytes(params: PirParams, max_batch: int, depth: int) -> int:
        per_query = (int(np.prod(params.ct_shape)) + 2 * params.N) * 8
        return depth * max_batch * per_query

    def set_client_keys(self, client_id, bv_keys, gsw_key):
        self.server.set_client_keys(client_id, bv_keys, gsw_key)

    def set_priority(self, priority: int):
        """CUDA stream priority of this database's copies and kernels."""
        torch = self.torch
        self.stream.synchronize()
        self.stream = torch.cuda.Stream(self.stream.device, priority=priority)
        self.server.set_priority(priority)

    def launch(self, slot: int, client_ids, queries: list) -> None:
        torch = self.torch
        n = len(client_ids)
        hq = self.h_q[slot].numpy().view(np.uint64)
        for i, q in enumerate(queries):
            hq[i] = q
        with torch.cuda.stream(self.stream):
            self.d_q[slot][:n].copy_(self.h_q[slot][:n], non_blocking=True)
            self.server.make_query_batch_device(client_ids, self.d_q[slot].data_ptr(),
                                                self.d_r[slot].data_ptr(), self.stream.cuda_stream)
            self.h_r[slot][:n].copy_(self.d_r[slot][:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        self.events[slot] = ev

    def done(self, slot: int) -> bool:
        return self.events[slot].query()

    def results(self, slot: int, n: int) -> np.ndarray:
        self.events[slot] = None
        return self.h_r[slot].numpy().view(np.uint64)[:n].copy()

    def close(self):
        self.stream.synchronize()
        self.server.close()


@dataclass
class _Batch:
    slot: int
    requests: list
    t_launch: float


class _Database:
    def __init__(self, name, params, lane, max_batch, depth, min_fill):
        self.name = name
        self.params = params
        self.lane = lane
        self.max_batch = max_batch
        self.min_fill = min_fill
        self.free_slots = list(range(depth))
        self.inflight: collections.deque[_Batch] = collections.deque()
        self.queue: collections.deque[_Request] = collections.deque()
        self.clients: set = set()


class ServingEngine:
    """Continuous batching across several databases on one GPU.

    depth    : batches a database may have enqueued on the device at once.
    min_fill : a database that already has a batch on the device enqueues the
               next one only once this many requests wait (default: a quarter
               of its batch limit); with nothing on the device it launches at
               once, whatever the queue length.
    """

    def __init__(self, device: int = 0, hbm_budget_bytes: int | None = None, depth: int = 2,
                 lane_factory=None):
        self.device = device
        self.depth = depth
        self._lane_factory = lane_factory or (
            lambda params, max_batch, depth, seed, plaintexts:
            CudaLane(params, max_batch, depth, device, seed, plaintexts))
        if hbm_budget_bytes is None:
            import torch
            free, _total = torch.cuda.mem_get_info(torch.device("cuda", device))
            hbm_budget_bytes = int(free * 0.9)
        self.budget = int(hbm_budget_bytes)
        self.reserved = 0
        self.dbs: dict[str, _Database] = {}
        self._incoming: collections.deque = collections.deque()
        self._cv = threading.Condition()          # guards _incoming and _running
        self._handle_lock = threading.Lock()      # serialises calls on server handles
        self._running = False
        self._thread = None
        self._error = None
        self.latencies_ms: dict[str, list] = collections.defaultdict(list)
        self.batch_log: list[tuple[str, int, float, float]] = []  # name, n, launch, done
        self.completed = 0
        self.t_first = None
        self.t_last = None

    # ------------------------------------------------------------ admission
    def _reserve(self, nbytes: int, what: str):
        if self.reserved + nbytes > self.budget:
            raise MemoryError(f"HBM budget refuses {what}: needs {nbytes} B, "
                              f"{self.budget - self.reserved} B of {self.budget} B left")
        self.reserved += nbytes

    def database_bytes(self, params: PirParams, max_batch: int) -> int:
        plan = plan_memory(params)
        return (plan["database_bytes"] + plan["scratch_bytes_fixed"]
                + max_batch * plan["scratch_bytes_per_query"]
                + CudaLane.buffer_bytes(params, max_batch, self.depth))

    def add_database(self, name: str, params: PirParams, max_batch: int = 32,
                     seed: int | None = None, plaintexts=None, min_fill: int | None = None,
                     priority: int | None = None):
        """Admit a database (seeded synthetic or the given plaintexts) that
        answers batches of up to max_batch queries. `priority` (CUDA stream
        priority, lower = first) lets a database with cheap queries overtake
        the long batches of an expensive one on the GPU."""
        if name in self.dbs:
            raise ValueError(f"database {name} exists")
        self._reserve(self.database_bytes(params, max_batch), f"database {name}")
        try:
            lane = self._lane_factory(params, max_batch, self.depth, seed, plaintexts)
        except BaseException:
            self.reserved -= self.database_bytes(params, max_batch)
            raise
        if priority is not None and hasattr(lane, "set_priority"):
            lane.set_priority(priority)
        mf = max(1, max_batch // 4) if min_fill is None else max(1, min_fill)
        self.dbs[name] = _Database(name, params, lane, max_batch, self.depth, mf)

    def register_client(self, name: str, client_id: int, bv_keys: np.ndarray,
                        gsw_key: np.ndarray):
        """Per-client key state on the device for one database (replaces the
        keys of a known client id without a new reservation)."""
        db = self.dbs[name]
        new = client_id not in db.clients
        if new:
            self._reserve(plan_memory(db.params)["client_key_bytes"], f"keys of client {client_id}")
        try:
            with self._handle_lock:  # key upload and batch launches share the handle
                db.lane.set_client_keys(client_id, bv_keys, gsw_key)
        except BaseException:
            if new:
                self.reserved -= plan_memory(db.params)["client_key_bytes"]
            raise
        db.clients.add(client_id)

    # ------------------------------------------------------------ requests
    def submit(self, name: str, client_id: int, query: np.ndarray) -> Future:
        fut: Future = Future()
        db = self.dbs.get(name)
        if db is None:
            fut.set_exception(KeyError(f"unknown database {name}"))
            return fut
        if client_id not in db.clients:
            fut.set_exception(IndexError(f"unknown client id {client_id}"))
            return fut
        q = np.ascontiguousarray(query, dtype=np.uint64)
        if q.shape != db.params.ct_shape:
            fut.set_exception(ValueError(f"query must be {db.params.ct_shape}"))
            return fut
        req = _Request(client_id, q, fut, time.perf_counter())
        with self._cv:
            if not self._running:
                fut.set_exception(RuntimeError("serving engine is not running"))
                return fut
            self._incoming.append((db, req))
            self._cv.notify()
        return fut

    def start(self):
        with self._cv:
            self._running = True
        self._thread = threading.Thread(target=self._loop, name="opir-serving", daemon=True)
        self._thread.start()

    def drain(self, timeout: float = 600.0):
        """Wait until every submitted request has been answered."""
        end = time.monotonic() + timeout
        while True:
            with self._cv:
                busy = bool(self._incoming) or any(d.queue or d.inflight for d in self.dbs.values())
            if not busy or self._error is not None:
                break
            if time.monotonic() > end:
                raise TimeoutError("serving engine did not drain")
            time.sleep(0.0005)
        if self._error is not None:
            raise self._error

    def stop(self):
        with self._cv:
            self._running = False
            self._cv.notify()
        if self._thread is not None:
            self._thread.join()
            self._thread = None

    def close(self):
        self.stop()
        for d in self.dbs.values():
            d.lane.close()
        self.dbs.clear()

    # ------------------------------------------------------------ scheduler
    def _launch(self, db: _Database):
        n = min(len(db.queue), db.max_batch)
        reqs = [db.queue.popleft() for _ in range(n)]
        slot = db.free_slots.pop()
        try:
            db.lane.launch(slot, [r.client_id for r in reqs], [r.query for r in reqs])
        except Exception as e:  # e.g. keys removed meanwhile: fail this batch only
            db.free_slots.append(slot)
            for r in reqs:
                r.future.set_exception(e)
            return
        db.inflight.append(_Batch(slot, reqs, time.perf_counter()))

    def _complete(self, db: _Database):
        b = db.inflight.popleft()
        out = db.lane.results(b.slot, len(b.requests))
        db.free_slots.append(b.slot)
        now = time.perf_counter()
        lat = self.latencies_ms[db.name]
        for i, r in enumerate(b.requests):
            lat.append((now - r.t_submit) * 1e3)
            r.future.set_result(out[i])
        self.completed += len(b.requests)
        self.t_last = now
        self.batch_log.append((db.name, len(b.requests), b.t_launch, now))

    def _step(self) -> bool:
        progressed = False
        for db in self.dbs.values():
            while db.inflight and db.lane.done(db.inflight[0].slot):
                self._complete(db)
                progressed = True
            while db.queue and db.free_slots and (
                    not db.inflight or len(db.queue) >= db.min_fill):
                self._launch(db)
                progressed = True
        return progressed

    def _loop(self):
        try:
            while True:
                with self._cv:
                    while self._incoming:
                        db, req = self._incoming.popleft()
                        db.queue.append(req)
                        if self.t_first is None:
                            self.t_first = req.t_submit
                    running = self._running
                with self._handle_lock:
                    progressed = self._step()
                idle = not any(d.inflight or d.queue for d in self.dbs.values())
                if not running and idle:
                    return
                if not progressed:
                    with self._cv:
                        if not self._incoming and self._running:
                            # nothing to launch: sleep until a request arrives,
                            # or poll the in-flight events again shortly
                            self._cv.wait(timeout=None if idle else 0.0001)
        except BaseException as e:  # surface scheduler failures to waiters
            self._error = e
            for d in self.dbs.values():
                for b in d.inflight:
                    for r in b.requests:
                        if not r.future.done():
                            r.future.set_exception(e)
                for r in d.queue:
                    if not r.future.done():
                        r.future.set_exception(e)

    # ------------------------------------------------------------ metrics
    def reset_stats(self):
        """Forget latencies and batches recorded so far (between load levels)."""
        self.latencies_ms = collections.defaultdict(list)
        self.batch_log = []
        self.completed = 0
        self.t_first = None
        self.t_last = None

    def stats(self) -> dict:
        def pct(v, p):
            return float(np.percentile(np.asarray(v), p)) if v else 0.0
        every = [x for v in self.latencies_ms.values() for x in v]
        span = (self.t_last - self.t_first) if self.t_first and self.t_last else 0.0
        per_db = {}
        for name in self.dbs:
            sizes = [n for nm, n, _, _ in self.batch_log if nm == name]
            per_db[name] = {"completed": len(self.latencies_ms[name]),
                            "p50_ms": pct(self.latencies_ms[name], 50),
                            "p99_ms": pct(self.latencies_ms[name], 99),
                            "batches": len(sizes),
                            "mean_batch": float(np.mean(sizes)) if sizes else 0.0}
        return {"completed": self.completed,
                "qps": self.completed / span if span > 0 else 0.0,
                "p50_ms": pct(every, 50), "p99_ms": pct(every, 99),
                "hbm_reserved_bytes": self.reserved, "hbm_budget_bytes": self.budget,
                "databases": per_db}
