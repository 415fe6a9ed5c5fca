"""Python mirror of the reference's full-binary-tree PIR layer over the C ABI
(src/includes/tree_index.h, tree_query.h, tree_select.h).

The index math (tree parameters, level plans, the query-shape view) runs in
the library's C++ host code; `select_level` runs on the GPU as one
first-dimension contraction over the N0 alpha ciphertexts plus the MSB-first
beta fold (opir_tree_select_level). Client-side helpers that the reference
keeps next to them (client_index, the synthetic node source, pack_tree_level)
are plain index arithmetic and are restated here for callers and tests.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from . import _lib as L
from .server import OPIR_OK, PirParams, PirServer, _ptr, _raise

SINGLE, COARSENED_ALPHA, ALPHA_BETA = 0, 1, 2


class TreePirParams:
    """TreePirParams (includes/tree_index.h:23-55) bound to a scheme."""

    def __init__(self, raw: "L.TreeParams", scheme: PirParams):
        self._t = raw
        self.scheme = scheme

    def __getattr__(self, name):
        t = self.__dict__.get("_t")
        if t is not None and name in dict(L.TreeParams._fields_):
            return getattr(t, name)
        raise AttributeError(name)


@dataclass
class LevelPlan:
    """LevelPlan (includes/tree_index.h:76-92)."""
    level: int
    R: int
    select_case: int
    coarsen_count: int
    beta_begin: int
    beta_count: int
    gamma_begin: int
    gamma_count: int
    projection_depth: int


@dataclass
class ClientCoordinates:
    alpha: int
    beta_bits_le: list
    gamma_bits_le: list


def make_tree_pir_params(L_: int, a: int, n: int, ell_beta: int, ell_gamma: int, t: int,
                         rns_moduli: Sequence[int]) -> TreePirParams:
    """make_tree_pir_params (src/tree_index.cpp:47-92): pure index math for
    any ring shape (no scheme bound; unusable for ciphertext calls)."""
    raw = L.TreeParams()
    mods = np.ascontiguousarray(np.asarray(list(rns_moduli) or [1], dtype=np.uint64))
    rc = L.load().opir_tree_params_make(L_, a, n, ell_beta, ell_gamma, t, _ptr(mods),
                                        len(list(rns_moduli)), C.byref(raw))
    if rc != OPIR_OK:
        _raise(rc, f"invalid tree shape L={L_} a={a} n={n}")
    return TreePirParams(raw, None)


def make_tree_pir_params_for_scheme(L_: int, a: int, scheme: PirParams) -> TreePirParams:
    """src/tree_query.cpp:42-62; invalid shapes raise ValueError."""
    raw = L.TreeParams()
    rc = L.load().opir_tree_params_init(L_, a, C.byref(scheme._p), C.byref(raw))
    if rc != OPIR_OK:
        _raise(rc, f"invalid tree shape L={L_} a={a}")
    return TreePirParams(raw, scheme)


def build_level_plans(tree: TreePirParams) -> list[LevelPlan]:
    """src/tree_index.cpp:177-225."""
    arr = (L.TreeLevelPlan * (tree.L + 1))()
    rc = L.load().opir_tree_level_plans(C.byref(tree._t), arr)
    if rc != OPIR_OK:
        _raise(rc, "build_level_plans failed")
    return [LevelPlan(p.level, p.R, p.select_case, p.coarsen_count, p.beta_begin, p.beta_count,
                      p.gamma_begin, p.gamma_count, p.projection_depth) for p in arr]


def tree_query_expansion_params(tree: TreePirParams, scheme: PirParams) -> PirParams:
    """src/tree_query.cpp:64-68: the query-shape view {N0, b + r, h_q}."""
    raw = L.Params()
    rc = L.load().opir_tree_query_params(C.byref(tree._t), C.byref(scheme._p), C.byref(raw))
    if rc != OPIR_OK:
        _raise(rc, "tree query shape does not fit the scheme")
    return PirParams._wrap(raw, scheme.config)


def client_index(leaf: int, tree: TreePirParams) -> ClientCoordinates:
    """Algorithm 1 ClientIndex (src/tree_index.cpp:152-175)."""
    if leaf >= tree.N:
        raise ValueError("client_index leaf is out of range")
    gamma, p = divmod(leaf, tree.P)
    alpha, beta = divmod(p, tree.B)
    return ClientCoordinates(alpha, [(beta >> u) & 1 for u in range(tree.b)],
                             [(gamma >> v) & 1 for v in range(tree.r)])


def level_record_position_from_coordinates(alpha: int, beta: int, level: int,
                                           tree: TreePirParams) -> int:
    """Invariant 2 (src/tree_index.cpp:250-262)."""
    if level < tree.r or level > tree.L:
        raise ValueError("record position formula is defined for levels in [r, L]")
    s = tree.L - level
    if s <= tree.b:
        return alpha * (1 << (tree.b - s)) + (beta >> s)
    return alpha >> (s - tree.b)


def level_oracle(leaf: int, level: int, tree: TreePirParams) -> tuple[int, int, int]:
    """build_level_oracle_for_test (src/tree_index.cpp:227-248): (node
    index, packed plaintext index, record position) of leaf's ancestor."""
    if leaf >= tree.N or level > tree.L:
        raise ValueError("level oracle out of range")
    node = leaf >> (tree.L - level)
    gamma, p = divmod(leaf, tree.P)
    if level >= tree.r:
        return node, p >> (tree.L - level), gamma
    return node, 0, gamma >> (tree.r - level)


_M64 = (1 << 64) - 1


def _splitmix64_once(v: int) -> int:
    v = (v + 0x9E3779B97F4A7C15) & _M64
    v = ((v ^ (v >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    v = ((v ^ (v >> 27)) * 0x94D049BB133111EB) & _M64
    return v ^ (v >> 31)


def synthetic_tree_node_value(level: int, index: int, t: int) -> int:
    """src/tree_select.cpp:44-53 (benchmark/test node source)."""
    if t == 0:
        raise ValueError("synthetic node values need a modulus")
    mixed = _splitmix64_once(0x74726565506972 ^ ((level * 0xD6E8FEB86659FD93) & _M64)
                             ^ ((index * 0xA5A3564E27F8862F) & _M64))
    return mixed % t


def pack_tree_level(level: int, tree: TreePirParams,
                    source: Callable[[int, int], int]) -> np.ndarray:
    """pack_tree_level (src/tree_select.cpp:55-75): R_l x n plaintexts with
    D_l[p][u] = M[l][p + u R_l] below 2^l, zero elsewhere."""
    if level > tree.L:
        raise ValueError("level is out of range")
    R = 1 << (level - tree.r) if level >= tree.r else 1
    out = np.zeros((R, tree.n), dtype=np.uint64)
    count = 1 << level
    for p in range(R):
        for u in range(tree.n):
            node = p + u * R
            if node >= count:
                break
            out[p, u] = source(level, node) % tree.t
    return out


def unpack_tree_query(server: PirServer, scheme: PirParams, tree: TreePirParams,
                      client_id: int, query: np.ndarray):
    """QueryUnpack (src/tree_query.cpp:198-240) on a server built on
    tree_query_expansion_params: (alpha ciphertexts, beta selectors, gamma
    selectors)."""
    view = server.params
    if (view.fst_dim_sz != tree.N0 or view.num_dims != 1 + tree.b + tree.r
            or view.expansion_height != tree.h_q):
        raise ValueError("unpack_tree_query server was not built on this tree's query shape")
    expanded = server.expand_query(client_id, query)
    if expanded.shape[0] != tree.w:
        raise RuntimeError("unpack_tree_query expansion returned an unexpected leaf count")
    selectors = server.complete_selectors(client_id, expanded)
    return expanded[: tree.N0], selectors[: tree.b], selectors[tree.b:]


class TreeLevel:
    """A device-resident tree level (opir_tree_level_create) answering
    select_level (src/tree_select.cpp:203-238) for expanded tree queries."""

    def __init__(self, scheme: PirParams, tree: TreePirParams, level: int,
                 plaintexts: np.ndarray, device: int = 0):
        self.scheme, self.tree, self.level = scheme, tree, level
        self._lib = L.load()
        pts = np.ascontiguousarray(plaintexts, dtype=np.uint64)
        R = 1 << (level - tree.r) if level >= tree.r else 1
        if pts.shape != (R, tree.n):
            raise ValueError(f"level {level} needs {R} x {tree.n} plaintext coefficients")
        h = C.c_void_p()
        rc = self._lib.opir_tree_level_create(C.byref(scheme._p), C.byref(tree._t), level,
                                              _ptr(pts), device, C.byref(h))
        if rc != OPIR_OK:
            _raise(rc, f"opir_tree_level_create failed (status {rc})")
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

    def select_level(self, alpha: np.ndarray, beta_selectors: np.ndarray | None) -> np.ndarray:
        """alpha: N0 ciphertexts; beta_selectors: the b RGSW selectors of
        unpack_tree_query (None or empty when the level folds no beta bit)."""
        shape = self.scheme.ct_shape
        a = np.ascontiguousarray(alpha, dtype=np.uint64)
        if a.shape != (self.tree.N0,) + shape:
            raise ValueError(f"alpha must be ({self.tree.N0},) + {shape}")
        bsel = None
        if beta_selectors is not None and np.asarray(beta_selectors).size:
            bsel = np.ascontiguousarray(beta_selectors, dtype=np.uint64)
        out = np.zeros(shape, dtype=np.uint64)
        rc = self._lib.opir_tree_select_level(self._h, _ptr(a),
                                              _ptr(bsel) if bsel is not None else None,
                                              _ptr(out))
        if rc != OPIR_OK:
            msg = self._lib.opir_server_last_error(self._h)
            _raise(rc, msg.decode() if msg else f"status {rc}")
        return out


class Tree:
    """A whole device-resident tree (opir_tree_create): unpack + select_level
    at every level per query with no host round trip between stages, the
    levels running on their own streams (either parameter set)."""

    def __init__(self, scheme: PirParams, tree: TreePirParams, level_plaintexts, device: int = 0):
        self.scheme, self.tree = scheme, tree
        self._lib = L.load()
        self._pts = []
        for level, pts in enumerate(level_plaintexts):
            a = np.ascontiguousarray(pts, dtype=np.uint64)
            R = 1 << (level - tree.r) if level >= tree.r else 1
            if a.shape != (R, tree.n):
                raise ValueError(f"level {level} needs {R} x {tree.n} plaintext coefficients")
            self._pts.append(a)
        if len(self._pts) != tree.L + 1:
            raise ValueError(f"a tree of height {tree.L} has {tree.L + 1} levels")
        arr = (L.u64p * len(self._pts))(*[_ptr(a) for a in self._pts])
        h = C.c_void_p()
        rc = self._lib.opir_tree_create(C.byref(scheme._p), C.byref(tree._t), arr, device,
                                        C.byref(h))
        if rc != OPIR_OK:
            _raise(rc, f"opir_tree_create failed (status {rc})")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.opir_tree_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int):
        if rc != OPIR_OK:
            msg = self._lib.opir_tree_last_error(self._h)
            _raise(rc, msg.decode() if msg else f"status {rc}")

    def set_client_keys(self, client_id: int, bv_keys: np.ndarray, gsw_key: np.ndarray):
        bv = np.ascontiguousarray(bv_keys[: self.tree.h_q], dtype=np.uint64)
        n_keys = bv.shape[0]
        gk = np.ascontiguousarray([(self.tree.n >> i) + 1 for i in range(n_keys)], dtype=np.uint32)
        g = np.ascontiguousarray(gsw_key, dtype=np.uint64)
        self._check(self._lib.opir_tree_set_client_keys(self._h, client_id, _ptr(bv),
                                                        _ptr(gk, C.c_uint32), n_keys, _ptr(g)))

    def query(self, client_id: int, query: np.ndarray) -> np.ndarray:
        """(L + 1) selected ciphertexts, level order."""
        q = np.ascontiguousarray(query, dtype=np.uint64)
        if q.shape != self.scheme.ct_shape:
            raise ValueError(f"query must be {self.scheme.ct_shape}")
        out = np.zeros((self.tree.L + 1,) + self.scheme.ct_shape, dtype=np.uint64)
        self._check(self._lib.opir_tree_query(self._h, client_id, _ptr(q), _ptr(out)))
        return out
