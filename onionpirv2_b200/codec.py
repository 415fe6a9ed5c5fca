"""Seed-compressed wire format of queries and client keys (the C ABI's
opir_query_* / opir_keys_* / opir_prf_expand, include/onionpir_b200.h).

The reference ships no serializer; its communication model
(includes/pir.h:115-139) counts a 32-byte seed for every uniformly random
polynomial. Here that seed expands with ChaCha20 (RFC 8439) into the query's
c1, the `a` of every BV key row and the c1 of every RGSW row, and the other
polynomial of each ciphertext is bit-packed at the modulus width.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .server import OPIR_OK, PirParams, _ptr, _raise

SEED_BYTES = 32
PRF_QUERY, PRF_BV_KEY, PRF_GSW_KEY = 1, 2, 3


def _seed(seed: bytes) -> np.ndarray:
    if len(seed) != SEED_BYTES:
        raise ValueError(f"a seed is {SEED_BYTES} bytes")
    return np.frombuffer(bytes(seed), dtype=np.uint8).copy()


def prf_expand(params: PirParams, seed: bytes, domain: int, index: int) -> np.ndarray:
    """Expand(seed, domain, index): one polynomial, shape ct_shape[1:]."""
    out = np.zeros(params.ct_shape[1:], dtype=np.uint64)
    rc = L.load().opir_prf_expand(C.byref(params._p), _ptr(_seed(seed), C.c_uint8), domain, index,
                                  _ptr(out))
    if rc != OPIR_OK:
        _raise(rc, "opir_prf_expand failed")
    return out


def query_wire_bytes(params: PirParams) -> int:
    return int(L.load().opir_query_wire_bytes(C.byref(params._p)))


def keys_wire_bytes(params: PirParams) -> int:
    return int(L.load().opir_keys_wire_bytes(C.byref(params._p)))


def encode_query(params: PirParams, seed: bytes, query: np.ndarray) -> bytes:
    q = np.ascontiguousarray(query, dtype=np.uint64)
    if q.shape != params.ct_shape:
        raise ValueError(f"query must be {params.ct_shape}")
    out = np.zeros(query_wire_bytes(params), dtype=np.uint8)
    rc = L.load().opir_query_encode(C.byref(params._p), _ptr(_seed(seed), C.c_uint8), _ptr(q),
                                    _ptr(out, C.c_uint8), out.size)
    if rc != OPIR_OK:
        _raise(rc, "query encoding failed (is c1 Expand(seed)?)")
    return out.tobytes()


def decode_query(params: PirParams, data: bytes) -> np.ndarray:
    buf = np.frombuffer(bytes(data), dtype=np.uint8).copy()
    out = np.zeros(params.ct_shape, dtype=np.uint64)
    rc = L.load().opir_query_decode(C.byref(params._p), _ptr(buf, C.c_uint8), buf.size, _ptr(out))
    if rc != OPIR_OK:
        _raise(rc, "not an encoded query of this parameter set")
    return out


def encode_keys(params: PirParams, seed: bytes, bv_keys: np.ndarray, gsw_key: np.ndarray) -> bytes:
    """bv_keys: (h, L_KS) + ct_shape as [b, a]; gsw_key: (2 L_KEY,) + ct_shape."""
    bv = np.ascontiguousarray(bv_keys, dtype=np.uint64)
    g = np.ascontiguousarray(gsw_key, dtype=np.uint64)
    if bv.size == 0:
        bv = np.zeros(1, dtype=np.uint64)
    out = np.zeros(keys_wire_bytes(params), dtype=np.uint8)
    rc = L.load().opir_keys_encode(C.byref(params._p), _ptr(_seed(seed), C.c_uint8), _ptr(bv),
                                   _ptr(g), _ptr(out, C.c_uint8), out.size)
    if rc != OPIR_OK:
        _raise(rc, "key encoding failed (are the uniform parts Expand(seed)?)")
    return out.tobytes()


def decode_keys(params: PirParams, data: bytes):
    """(bv_keys, galois_ks, gsw_key) ready for PirServer.set_client_keys."""
    h = params.expansion_height
    buf = np.frombuffer(bytes(data), dtype=np.uint8).copy()
    bv = np.zeros((max(h, 1), params.l_ks) + params.ct_shape, dtype=np.uint64)
    ks = np.zeros(max(h, 1), dtype=np.uint32)
    g = np.zeros((2 * params.l_key,) + params.ct_shape, dtype=np.uint64)
    rc = L.load().opir_keys_decode(C.byref(params._p), _ptr(buf, C.c_uint8), buf.size, _ptr(bv),
                                   _ptr(ks, C.c_uint32), _ptr(g))
    if rc != OPIR_OK:
        _raise(rc, "not an encoded key bundle of this parameter set")
    return bv[:h], ks[:h], g
