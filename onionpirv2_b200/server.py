"""Python mirror of the reference's PirParams / PirServer interface over the
C ABI (include/onionpir_b200.h).

Names, argument meaning and error behaviour follow the reference
(src/includes/pir.h, src/includes/server.h): invalid layouts and inputs raise
ValueError (std::invalid_argument), unknown clients raise KeyError-compatible
IndexError subclass OutOfRange (std::out_of_range), device failures raise
RuntimeError. Ciphertexts are numpy uint64 arrays shaped (2, N) = (c0, c1)
under CONFIG_N2048_K1_COMP and CONFIG_N2048_K1 and (2, 2, N) = (poly, RNS
limb, coefficient) under CONFIG_N2048_K2_MP and CONFIG_N4096_K2_MP; responses
are (2, N) mod small_q under all four.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Iterable, Sequence

import numpy as np

from . import _lib as L

OPIR_OK = 0
OPIR_ERR_INVALID_ARGUMENT = 1
OPIR_ERR_OUT_OF_RANGE = 2
OPIR_ERR_RUNTIME = 3
OPIR_ERR_CUDA = 4
OPIR_ERR_NO_MEMORY = 5
OPIR_ERR_OVERFLOW = 6


class OutOfRange(IndexError, KeyError):
    """std::out_of_range in the reference (unknown client, missing key)."""


class DeviceError(RuntimeError):
    """CUDA failure reported by the library."""


def _raise(code: int, msg: str):
    if code == OPIR_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    if code == OPIR_ERR_OUT_OF_RANGE:
        raise OutOfRange(msg)
    if code == OPIR_ERR_OVERFLOW:
        raise OverflowError(msg)
    if code == OPIR_ERR_NO_MEMORY:
        raise MemoryError(msg)
    if code == OPIR_ERR_CUDA:
        raise DeviceError(msg)
    raise RuntimeError(msg)


def _ptr(a: np.ndarray, t=C.c_uint64):
    return a.ctypes.data_as(C.POINTER(t))


CONFIGS = {"CONFIG_N2048_K1_COMP": 0, "CONFIG_N4096_K2_MP": 1, "CONFIG_N2048_K2_MP": 2,
           "CONFIG_N2048_K1": 3}


class PirParams:
    """PirParams().with_layout({target_num_pt, expansion_height, fst_dim_pow2})
    under one ACTIVE_CONFIG (includes/database_constants.h:31-40):
    "CONFIG_N2048_K1_COMP" (default), "CONFIG_N2048_K1" (the reference's own
    default: one 60-bit prime), "CONFIG_N2048_K2_MP" or "CONFIG_N4096_K2_MP"."""

    def __init__(self, target_num_pt: int = 43690, expansion_height: int = 10,
                 fst_dim_pow2: bool = True, config: str = "CONFIG_N2048_K1_COMP"):
        if config not in CONFIGS:
            raise ValueError(f"unknown parameter set {config!r}")
        self.config = config
        self._layout = L.Layout(target_num_pt, expansion_height, 1 if fst_dim_pow2 else 0)
        self._p = L.Params()
        rc = L.load().opir_params_init_config(CONFIGS[config], C.byref(self._layout),
                                              C.byref(self._p))
        if rc != OPIR_OK:
            _raise(rc, f"invalid layout {target_num_pt}/{expansion_height}/{fst_dim_pow2}")

    def with_layout(self, target_num_pt: int, expansion_height: int,
                    fst_dim_pow2: bool = True) -> "PirParams":
        return PirParams(target_num_pt, expansion_height, fst_dim_pow2, self.config)

    @classmethod
    def _wrap(cls, raw: "L.Params", config: str) -> "PirParams":
        p = cls.__new__(cls)
        p.config = config
        p._layout = None
        p._p = raw
        return p

    def with_query_shape(self, fst_dim_sz: int, num_selector_bits: int,
                         expansion_height: int) -> "PirParams":
        """PirParams::with_query_shape (src/pir.cpp:136-166): a view with no
        database behind it, for servers that only expand queries and complete
        selectors."""
        shape = L.QueryShape(fst_dim_sz, num_selector_bits, expansion_height)
        raw = L.Params()
        rc = L.load().opir_params_query_shape(C.byref(self._p), C.byref(shape), C.byref(raw))
        if rc != OPIR_OK:
            _raise(rc, "query shape does not fit this scheme")
        return PirParams._wrap(raw, self.config)

    def __getattr__(self, name):
        p = self.__dict__.get("_p")
        if p is not None and name in dict(L.Params._fields_):
            return getattr(p, name)
        raise AttributeError(name)

    # getters named as in includes/pir.h
    def get_num_pt(self): return self._p.num_pt
    def get_fst_dim_sz(self): return self._p.fst_dim_sz
    def get_other_dim_sz(self): return self._p.other_dim_sz
    def get_num_dims(self): return self._p.num_dims
    def get_expan_height(self): return self._p.expansion_height
    def get_plain_mod(self): return self._p.plain_mod
    def get_small_q(self): return self._p.small_q
    def get_rns_mods(self):
        return [self._p.q] if self._p.num_limbs == 1 else [self._p.q1, self._p.q2]
    def get_poly_degree(self): return self._p.poly_degree
    def get_l(self): return self._p.l_ep
    def get_l_key(self): return self._p.l_key
    def get_target_num_pt(self): return self._p.target_num_pt

    @property
    def N(self) -> int:
        return self._p.poly_degree

    @property
    def ct_shape(self) -> tuple:
        """Shape of one ciphertext: (2, N), or (2, K, N) with RNS limbs."""
        N = self._p.poly_degree
        return (2, N) if self._p.num_limbs == 1 else (2, self._p.num_limbs, N)

    @property
    def useful(self) -> int:
        return self._p.fst_dim_sz + self._p.l_ep * (self._p.num_dims - 1)

    def response_bytes(self) -> int:
        return int(L.load().opir_response_bytes(C.byref(self._p)))

    def as_dict(self) -> dict:
        return {f: getattr(self._p, f) for f, _ in L.Params._fields_ if f != "view"}


class PirServer:
    """Device-resident OnionPIRv2 server (PirServer, includes/server.h:15-172)."""

    def __init__(self, params: PirParams, device: int = 0):
        self.params = params
        self._lib = L.load()
        h = C.c_void_p()
        rc = self._lib.opir_server_create(C.byref(params._p), device, C.byref(h))
        if rc != OPIR_OK:
            _raise(rc, f"opir_server_create failed (status {rc})")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.opir_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc: int):
        if rc != OPIR_OK:
            msg = self._lib.opir_server_last_error(self._h)
            _raise(rc, msg.decode() if msg else f"status {rc}")

    # ---- database
    def load_data(self, logical_num_pt: int,
                  source: Callable[[int], Sequence[int]] | np.ndarray):
        """load_data(logical_num_pt, source): source is either an array
        (logical_num_pt, N) of coefficients < t or a callable index -> N
        coefficients (the reference's PlaintextSource)."""
        N = self.params.N
        if isinstance(source, np.ndarray):
            arr = np.ascontiguousarray(source)
            if arr.shape != (logical_num_pt, N):
                raise ValueError("Plaintext source returned the wrong coefficient count")
            if arr.dtype == np.uint16:
                self._check(self._lib.opir_server_load_db_u16(self._h, logical_num_pt, _ptr(arr, C.c_uint16)))
            else:
                a64 = np.ascontiguousarray(arr, dtype=np.uint64)
                self._check(self._lib.opir_server_load_db(self._h, logical_num_pt, _ptr(a64)))
            return
        err: list[BaseException] = []

        def cb(_user, idx, out):
            try:
                vals = np.asarray(source(int(idx)), dtype=np.uint64)
                if vals.shape != (N,):
                    raise ValueError("Plaintext source returned the wrong coefficient count")
                C.memmove(out, vals.ctypes.data, N * 8)
                return 0
            except BaseException as e:  # propagate after the C call returns
                err.append(e)
                return 1

        cfun = L.SOURCE_CB(cb)
        rc = self._lib.opir_server_load_db_source(self._h, logical_num_pt, cfun, None)
        if err:
            raise err[0]
        self._check(rc)

    def load_data_seeded(self, logical_num_pt: int, seed: int):
        self._check(self._lib.opir_server_load_db_seeded(self._h, logical_num_pt, seed))

    # ---- keys
    def set_client_keys(self, client_id: int, bv_keys: np.ndarray, gsw_key: np.ndarray,
                        galois_ks: Iterable[int] | None = None, key_form: str = "ntt"):
        """set_client_bv_galois_key + set_client_gsw_key. bv_keys: (n_keys, L_KS,
        2, N) NTT form [b, a]; galois_ks defaults to (N >> i) + 1. key_form
        "coeff": every row polynomial in coefficient form instead (keys from a
        producer with another NTT convention); the server NTTs them itself."""
        if key_form not in ("ntt", "coeff"):
            raise ValueError("key_form is 'ntt' or 'coeff'")
        N = self.params.N
        bv = np.ascontiguousarray(bv_keys, dtype=np.uint64)
        n_keys = bv.shape[0] if bv.size else 0
        if galois_ks is None:
            galois_ks = [(N >> i) + 1 for i in range(n_keys)]
        gk = np.ascontiguousarray(np.asarray(list(galois_ks), dtype=np.uint32))
        if gk.size == 0:
            gk = np.zeros(1, dtype=np.uint32)
        if bv.size == 0:
            bv = np.zeros(1, dtype=np.uint64)
        g = np.ascontiguousarray(gsw_key, dtype=np.uint64)
        self._check(self._lib.opir_server_set_client_keys_ex(
            self._h, client_id, _ptr(bv), _ptr(gk, C.c_uint32), n_keys, _ptr(g),
            0 if key_form == "ntt" else 1))

    def remove_client(self, client_id: int):
        self._check(self._lib.opir_server_remove_client(self._h, client_id))

    # ---- query path
    def make_query(self, client_id: int, query: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(query, dtype=np.uint64)
        if q.shape != self.params.ct_shape:
            raise ValueError(f"query must be {self.params.ct_shape}")
        out = np.zeros((2, self.params.N), dtype=np.uint64)
        self._check(self._lib.opir_server_make_query(self._h, client_id, _ptr(q), _ptr(out)))
        return out

    def make_query_batch(self, client_ids: Sequence[int], queries: np.ndarray,
                         out: np.ndarray | None = None) -> np.ndarray:
        """n queries in one pass; `out` (n, 2, N) uint64 may be supplied (e.g.
        pinned host memory)."""
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        n = ids.size
        if q.shape != (n,) + self.params.ct_shape:
            raise ValueError(f"queries must be (n,) + {self.params.ct_shape}")
        shape = (n, 2, self.params.N)
        if out is None:
            out = np.zeros(shape, dtype=np.uint64)
        elif out.shape != shape or out.dtype != np.uint64 or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a contiguous (n, 2, N) uint64 array")
        self._check(self._lib.opir_server_make_query_batch(self._h, n, _ptr(ids), _ptr(q), _ptr(out)))
        return out

    def make_query_batch_device(self, client_ids: Sequence[int], d_queries: int,
                                d_responses: int, stream: int = 0):
        """Enqueue on device pointers (ints), e.g. torch tensors' data_ptr()."""
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        self._check(self._lib.opir_server_make_query_batch_device(
            self._h, ids.size, _ptr(ids), C.c_void_p(d_queries), C.c_void_p(d_responses),
            C.c_void_p(stream) if stream else None))

    def reserve(self, max_batch: int):
        """Size the device scratch arena for batches of up to max_batch now, so
        that later calls of that size allocate no device memory."""
        self._check(self._lib.opir_server_reserve(self._h, int(max_batch)))

    def set_priority(self, priority: int):
        """Run the handle's work on a stream of this CUDA priority (lower =
        scheduled first); results are unchanged."""
        self._check(self._lib.opir_server_set_priority(self._h, int(priority)))

    def level_splits(self, n: int) -> dict:
        """Cluster widths a batch of n uses per expansion and MUX level
        (0 = the default rule, else the autotuned width)."""
        e = (C.c_uint8 * 16)()
        m = (C.c_uint8 * 32)()
        self._check(self._lib.opir_server_level_splits(self._h, int(n), e, m))
        return {"expand": list(e), "mux": list(m)}

    def set_scan_wait_limit(self, cycles: int):
        """Limit (SM clock cycles) of each wait inside the tensor-core scan;
        0 restores the default of about one second. A wait that runs out
        makes the call raise RuntimeError, and the handle stays usable."""
        self._check(self._lib.opir_server_set_scan_wait_limit(self._h, int(cycles)))

    def autotune(self, max_batch: int):
        """Time the tensor-core scan's tilings on this database for batches
        up to max_batch and keep the fastest per batch-size bucket."""
        self._check(self._lib.opir_server_autotune(self._h, int(max_batch)))

    def scan_tile(self, n: int) -> dict:
        """Tiling of the first-dimension scan for a batch of n queries."""
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        self._check(self._lib.opir_server_scan_tile(self._h, int(n), C.byref(a), C.byref(b),
                                                    C.byref(c)))
        return {"ntile": a.value, "kt": b.value, "stages": c.value}

    def set_stage_timing(self, enabled: bool):
        self._check(self._lib.opir_server_set_stage_timing(self._h, 1 if enabled else 0))

    def stage_times(self) -> dict:
        """Average per-stage device ms since set_stage_timing(True); "Core" is
        the first-dimension scan kernel alone."""
        buf = (C.c_float * 6)()
        calls = C.c_uint32()
        self._check(self._lib.opir_server_stage_times(self._h, buf, C.byref(calls)))
        names = ["Expand", "Convert", "First dim", "Other dim", "Modulus switching", "Core"]
        out = dict(zip(names, [float(x) for x in buf]))
        out["calls"] = calls.value
        return out

    # ---- individual stages (public PirServer methods)
    def expand_query(self, client_id: int, query: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(query, dtype=np.uint64)
        if q.shape != self.params.ct_shape:
            raise ValueError(f"query must be {self.params.ct_shape}")
        out = np.zeros((self.params.useful,) + self.params.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_expand_query(self._h, client_id, _ptr(q), _ptr(out)))
        return out

    def complete_selectors(self, client_id: int, expanded: np.ndarray) -> np.ndarray:
        p = self.params
        e = np.ascontiguousarray(expanded, dtype=np.uint64)
        if e.shape != (p.useful,) + p.ct_shape:
            raise ValueError(f"expanded must be ({p.useful},) + {p.ct_shape}")
        out = np.zeros((max(p.num_dims - 1, 1), 2 * p.l_ep) + p.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_complete_selectors(self._h, client_id, _ptr(e), _ptr(out)))
        return out[: p.num_dims - 1]

    def evaluate_first_dim(self, fst_query: np.ndarray) -> np.ndarray:
        p = self.params
        f = np.ascontiguousarray(fst_query[: p.fst_dim_sz], dtype=np.uint64)
        if f.shape != (p.fst_dim_sz,) + p.ct_shape:
            raise ValueError(f"fst_query must hold ({p.fst_dim_sz},) + {p.ct_shape}")
        out = np.zeros((p.other_dim_sz,) + p.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_evaluate_first_dim(self._h, _ptr(f), _ptr(out)))
        return out

    def evaluate_other_dim(self, mid: np.ndarray, selectors: np.ndarray) -> np.ndarray:
        p = self.params
        m = np.ascontiguousarray(mid, dtype=np.uint64)
        if m.shape != (p.other_dim_sz,) + p.ct_shape:
            raise ValueError(f"mid must be ({p.other_dim_sz},) + {p.ct_shape}")
        s = np.ascontiguousarray(selectors, dtype=np.uint64)
        if s.size == 0:
            s = np.zeros(1, dtype=np.uint64)
        out = np.zeros(p.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_evaluate_other_dim(self._h, _ptr(m), _ptr(s), _ptr(out)))
        return out

    def ext_prod_mux(self, x: np.ndarray, y: np.ndarray, selector: np.ndarray) -> np.ndarray:
        """x + b (y - x) for the RGSW selector bit b (ext_prod_mux); y is
        left unchanged. selector: (2 L_EP,) + ct_shape rows, NTT form."""
        p = self.params
        xx = np.ascontiguousarray(x, dtype=np.uint64)
        yy = np.ascontiguousarray(y, dtype=np.uint64)
        ss = np.ascontiguousarray(selector, dtype=np.uint64)
        if xx.shape != p.ct_shape or yy.shape != p.ct_shape:
            raise ValueError(f"x and y must be {p.ct_shape}")
        if ss.shape != (2 * p.l_ep,) + p.ct_shape:
            raise ValueError(f"selector must be ({2 * p.l_ep},) + {p.ct_shape}")
        out = np.zeros(p.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_ext_prod_mux(self._h, _ptr(xx), _ptr(yy), _ptr(ss),
                                                       _ptr(out)))
        return out

    def save_resp_to_stream(self, response: np.ndarray) -> bytes:
        return save_response(self.params, response)


def row_shard_rows(params: PirParams, shard: int, num_shards: int) -> tuple[np.ndarray, int]:
    """Database rows of shard `shard` of `num_shards` in storage order, and
    the MUX levels the shard answers (opir_row_shard_rows)."""
    lib = L.load()
    n = C.c_uint64()
    th = C.c_uint32()
    rc = lib.opir_row_shard_rows(C.byref(params._p), shard, num_shards, None, C.byref(n), C.byref(th))
    if rc != OPIR_OK:
        _raise(rc, f"invalid row shard {shard} of {num_shards} for this layout")
    rows = np.zeros(max(n.value, 1), dtype=np.uint32)
    rc = lib.opir_row_shard_rows(C.byref(params._p), shard, num_shards, _ptr(rows, C.c_uint32),
                                 C.byref(n), C.byref(th))
    if rc != OPIR_OK:
        _raise(rc, "opir_row_shard_rows failed")
    return rows[: n.value], int(th.value)


class RowShardServer(PirServer):
    """One GPU's rows of a database split by candidate rows across
    `num_shards` GPUs (opir_server_create_row_shard). Loads take the whole
    database's arguments; make_query_shard_batch returns each query's partial
    ciphertext (shape params.ct_shape, mod q); combine_shards, on any shard
    whose last batch had the same client ids, finishes the queries from all
    shards' partials and returns make_query's responses."""

    def __init__(self, params: PirParams, shard: int, num_shards: int, device: int = 0):
        self.params = params
        self.shard, self.num_shards = int(shard), int(num_shards)
        self._lib = L.load()
        h = C.c_void_p()
        rc = self._lib.opir_server_create_row_shard(C.byref(params._p), self.shard,
                                                    self.num_shards, device, C.byref(h))
        if rc != OPIR_OK:
            _raise(rc, f"opir_server_create_row_shard failed (status {rc})")
        self._h = h

    def make_query_shard_batch(self, client_ids: Sequence[int], queries: np.ndarray) -> np.ndarray:
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        q = np.ascontiguousarray(queries, dtype=np.uint64)
        n = ids.size
        if q.shape != (n,) + self.params.ct_shape:
            raise ValueError(f"queries must be (n,) + {self.params.ct_shape}")
        out = np.zeros((n,) + self.params.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_server_make_query_shard_batch(self._h, n, _ptr(ids), _ptr(q),
                                                                 _ptr(out)))
        return out

    def make_query_shard_batch_device(self, client_ids: Sequence[int], d_queries: int,
                                      d_partials: int, stream: int = 0):
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        self._check(self._lib.opir_server_make_query_shard_batch_device(
            self._h, ids.size, _ptr(ids), C.c_void_p(d_queries), C.c_void_p(d_partials),
            C.c_void_p(stream) if stream else None))

    def combine_shards(self, client_ids: Sequence[int], partials: np.ndarray) -> np.ndarray:
        """partials: (num_shards, n) + ct_shape, shard g's batch at [g]."""
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        n = ids.size
        pa = np.ascontiguousarray(partials, dtype=np.uint64)
        if pa.shape != (self.num_shards, n) + self.params.ct_shape:
            raise ValueError(f"partials must be ({self.num_shards}, {n}) + {self.params.ct_shape}")
        out = np.zeros((n, 2, self.params.N), dtype=np.uint64)
        self._check(self._lib.opir_server_combine_shards(self._h, n, _ptr(ids), _ptr(pa), _ptr(out)))
        return out

    def combine_shards_device(self, client_ids: Sequence[int], d_partials: int,
                              d_responses: int, stream: int = 0):
        ids = np.ascontiguousarray(np.asarray(client_ids, dtype=np.uint64))
        self._check(self._lib.opir_server_combine_shards_device(
            self._h, ids.size, _ptr(ids), C.c_void_p(d_partials), C.c_void_p(d_responses),
            C.c_void_p(stream) if stream else None))


def plan_memory(params: PirParams) -> dict:
    """Device bytes a server of these parameters requests: database, one
    client's keys, and scratch = fixed + batch * per_query."""
    plan = L.MemoryPlan()
    rc = L.load().opir_plan_memory(C.byref(params._p), C.byref(plan))
    if rc != OPIR_OK:
        _raise(rc, "opir_plan_memory failed")
    return {f: int(getattr(plan, f)) for f, _ in L.MemoryPlan._fields_}


def measure_butterfly_rate(config: str = "CONFIG_N2048_K1_COMP", device: int = 0) -> float:
    """NTT butterflies per second the device retires with register-resident
    operands (opir_measure_butterfly_rate): the NTT-bound stages' peak."""
    out = C.c_double()
    rc = L.load().opir_measure_butterfly_rate(CONFIGS[config], device, C.byref(out))
    if rc != OPIR_OK:
        _raise(rc, "opir_measure_butterfly_rate failed")
    return float(out.value)


def measure_recombine_rate(classes: int = 7, device: int = 0) -> float:
    """Outputs per second the device finishes for an int8 tensor-core product
    of byte-sliced 29-bit residues: `classes` shift-class sums recombined and
    reduced mod q, register-resident (opir_measure_recombine_rate)."""
    out = C.c_double()
    rc = L.load().opir_measure_recombine_rate(classes, device, C.byref(out))
    if rc != OPIR_OK:
        _raise(rc, "opir_measure_recombine_rate failed")
    return float(out.value)


def launch_count() -> int:
    """Kernel launches issued by the library in this process."""
    return int(L.load().opir_launch_count())


def save_response(params: PirParams, response: np.ndarray) -> bytes:
    """PirServer::save_resp_to_stream (server.cpp:950-1009)."""
    r = np.ascontiguousarray(response, dtype=np.uint64)
    cap = params.response_bytes()
    buf = np.zeros(cap, dtype=np.uint8)
    n = L.load().opir_save_response(C.byref(params._p), _ptr(r), _ptr(buf, C.c_uint8), cap)
    return buf[:n].tobytes()
