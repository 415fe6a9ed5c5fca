"""GPU batch operations of the reference's PirClient (src/client.cpp) for
one client's secret: query packing (fast_generate_query, :107-225),
response decryption (decrypt_mod_q, :364-410) and the session keys
(create_session_keys, :40-45), over the C ABI's opir_client_* calls
(include/onionpir_b200.h).

The randomness of a query (the uniform c1 `a` and the error `e`) is an input:
the reference draws it from its own generators, the codec expands `a` from a
seed (codec.prf_expand), and a caller may sample `e` however it likes; the
same holds for the uniform parts and errors of the session keys.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L
from .server import OPIR_OK, PirParams, _ptr, _raise


class PirClient:
    """One client's ternary secret, resident on one GPU."""

    def __init__(self, params: PirParams, secret: np.ndarray, device: int = 0):
        s = np.ascontiguousarray(secret, dtype=np.int8)
        if s.shape != (params.N,):
            raise ValueError(f"secret must be ({params.N},) int8 in {{-1, 0, 1}}")
        self.params = params
        self.device = device
        self._lib = L.load()
        h = C.c_void_p()
        rc = self._lib.opir_client_create(C.byref(params._p), _ptr(s, C.c_int8), device,
                                          C.byref(h))
        if rc != OPIR_OK:
            _raise(rc, "client creation failed")
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.opir_client_destroy(h)
            self._h = None

    def _check(self, rc: int):
        if rc != OPIR_OK:
            _raise(rc, self._lib.opir_client_last_error(self._h).decode())

    @property
    def query_shape(self) -> tuple:
        return self.params.ct_shape

    # ---- device-pointer form ------------------------------------------------
    def generate_queries_device(self, pt_idx: Sequence[int], d_a: int, d_e: int, d_queries: int,
                                stream: int = 0):
        """Enqueue on device pointers (ints), e.g. torch tensors' data_ptr()."""
        idx = np.ascontiguousarray(np.asarray(pt_idx, dtype=np.uint64))
        self._check(self._lib.opir_client_generate_queries_device(
            self._h, idx.size, _ptr(idx), C.c_void_p(d_a), C.c_void_p(d_e),
            C.c_void_p(d_queries), C.c_void_p(stream) if stream else None))

    def decrypt_device(self, n: int, d_responses: int, d_plaintexts: int, d_max_noise: int = 0,
                       stream: int = 0):
        self._check(self._lib.opir_client_decrypt_device(
            self._h, int(n), C.c_void_p(d_responses), C.c_void_p(d_plaintexts),
            C.c_void_p(d_max_noise) if d_max_noise else None,
            C.c_void_p(stream) if stream else None))

    def keygen_device(self, d_bv_a: int, d_bv_e: int, d_gsw_a: int, d_gsw_e: int,
                      d_bv_keys: int, d_gsw_key: int, stream: int = 0):
        p = lambda v: C.c_void_p(v) if v else None  # noqa: E731
        self._check(self._lib.opir_client_keygen_device(
            self._h, p(d_bv_a), p(d_bv_e), p(d_gsw_a), p(d_gsw_e), p(d_bv_keys), p(d_gsw_key),
            p(stream)))

    # ---- host form (the C ABI's host-buffer calls) ---------------------------
    def create_session_keys(self, bv_a: np.ndarray, bv_e: np.ndarray, gsw_a: np.ndarray,
                            gsw_e: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """The BV keys (h, L_KS) + ct_shape and the RGSW key (2 L_KEY,) +
        ct_shape from the uniform parts (coefficient form, limb-major per
        row) and errors the reference's generators would draw."""
        P = self.params
        h, lks, lkey, N = P.expansion_height, P.l_ks, P.l_key, P.N
        cs = P.ct_shape
        ba = np.ascontiguousarray(bv_a, dtype=np.uint64).reshape((h * lks,) + cs[1:]) if h else None
        be = np.ascontiguousarray(bv_e, dtype=np.int64).reshape(h * lks, N) if h else None
        ga = np.ascontiguousarray(gsw_a, dtype=np.uint64).reshape((2 * lkey,) + cs[1:])
        ge = np.ascontiguousarray(gsw_e, dtype=np.int64).reshape(2 * lkey, N)
        bv = np.zeros((h, lks) + cs, np.uint64)
        gsw = np.zeros((2 * lkey,) + cs, np.uint64)
        self._check(self._lib.opir_client_keygen(
            self._h, _ptr(ba) if h else None, _ptr(be, C.c_int64) if h else None, _ptr(ga),
            _ptr(ge, C.c_int64), _ptr(bv) if h else None, _ptr(gsw)))
        return bv, gsw

    def fast_generate_query_batch(self, pt_idx: Sequence[int], a: np.ndarray,
                                  e: np.ndarray) -> np.ndarray:
        """Queries for pt_idx with c1 = a[i] and error e[i]: (n,) + ct_shape."""
        idx = np.ascontiguousarray(np.asarray(pt_idx, dtype=np.uint64).reshape(-1))
        n = idx.size
        cs = self.params.ct_shape
        a = np.ascontiguousarray(a, dtype=np.uint64).reshape((n,) + cs[1:])
        e = np.ascontiguousarray(e, dtype=np.int64).reshape(n, self.params.N)
        out = np.zeros((n,) + cs, np.uint64)
        self._check(self._lib.opir_client_generate_queries(
            self._h, n, _ptr(idx), _ptr(a), _ptr(e, C.c_int64), _ptr(out)))
        return out

    def fast_generate_query(self, pt_idx: int, a: np.ndarray, e: np.ndarray) -> np.ndarray:
        return self.fast_generate_query_batch([pt_idx], a[None], e[None])[0]

    def decrypt_mod_q_batch(self, responses: np.ndarray, with_noise: bool = False):
        """Plaintexts (n, N) of responses (n, 2, N); with_noise adds each
        response's max noise."""
        N = self.params.N
        r = np.ascontiguousarray(responses, dtype=np.uint64)
        n = r.shape[0]
        r = r.reshape(n, 2, N)
        pt = np.zeros((n, N), np.uint64)
        noise = np.zeros(n, np.uint64) if with_noise else None
        self._check(self._lib.opir_client_decrypt(
            self._h, n, _ptr(r), _ptr(pt), _ptr(noise) if with_noise else None))
        return (pt, noise) if with_noise else pt

    def decrypt_mod_q(self, response: np.ndarray) -> np.ndarray:
        return self.decrypt_mod_q_batch(np.asarray(response)[None])[0]

    def make_tree_queries(self, tree, alpha: Sequence[int], bits: np.ndarray, a: np.ndarray,
                          e: np.ndarray) -> np.ndarray:
        """make_tree_query (tree_query.cpp:142-196) for n client coordinates:
        alpha (n,), bits (n, b + r) beta then gamma bits, a (n,) + ct_shape[1:]
        uniform c1, e (n, N) errors; returns (n,) + ct_shape."""
        al = np.ascontiguousarray(np.asarray(alpha, dtype=np.uint64).reshape(-1))
        n = al.size
        bt = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8).reshape(n, -1))
        groups = bt.shape[1]
        if groups == 0:
            bt = np.zeros((n, 1), np.uint8)
        cs = self.params.ct_shape
        aa = np.ascontiguousarray(a, dtype=np.uint64).reshape((n,) + cs[1:])
        ee = np.ascontiguousarray(e, dtype=np.int64).reshape(n, self.params.N)
        out = np.zeros((n,) + cs, np.uint64)
        self._check(self._lib.opir_client_generate_tree_queries(
            self._h, C.byref(tree._t), n, _ptr(al), _ptr(bt, C.c_uint8), groups, _ptr(aa),
            _ptr(ee, C.c_int64), _ptr(out)))
        return out
