"""ctypes view of the CPU oracle (libopir_oracle.so). TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg import
this module, and only as the checker. The library restates the reference
server path in plain C (oracle/opir_oracle.c for CONFIG_N2048_K1_COMP,
oracle/opir_oracle_c4.c for CONFIG_N4096_K2_MP); see those files for the
file:line map into the reference.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libopir_oracle.so")
_u64p = C.POINTER(C.c_uint64)


class Params(C.Structure):
    _fields_ = [
        ("N", C.c_uint32),
        ("q", C.c_uint64), ("q1", C.c_uint64), ("q2", C.c_uint64),
        ("w1", C.c_uint64), ("w2", C.c_uint64), ("w_crt", C.c_uint64),
        ("q1_inv_mod_q2", C.c_uint64),
        ("t", C.c_uint64), ("small_q", C.c_uint64),
        ("small_q_width", C.c_uint32), ("ct_mod_width", C.c_uint32),
        ("l_ep", C.c_uint32), ("l_key", C.c_uint32), ("l_ks", C.c_uint32),
        ("base_ep", C.c_uint32), ("base_key", C.c_uint32), ("base_ks", C.c_uint32),
        ("target_num_pt", C.c_uint64), ("num_pt", C.c_uint64),
        ("fst_dim_sz", C.c_uint64), ("other_dim_sz", C.c_uint64),
        ("num_dims", C.c_uint32), ("expansion_height", C.c_uint32),
        ("fst_dim_pow2", C.c_uint32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}

    @property
    def useful(self) -> int:
        return self.fst_dim_sz + self.l_ep * (self.num_dims - 1)


class C4Params(C.Structure):
    """CONFIG_N4096_K2_MP parameters (two 60-bit limbs, N = 4096)."""
    _fields_ = [
        ("N", C.c_uint32), ("K", C.c_uint32),
        ("q", C.c_uint64 * 2), ("w", C.c_uint64 * 2),
        ("q0_inv_mod_q1", C.c_uint64), ("r64_mod_q", C.c_uint64 * 2),
        ("t", C.c_uint64), ("small_q", C.c_uint64),
        ("small_q_width", C.c_uint32), ("ct_mod_width", C.c_uint32),
        ("l_ep", C.c_uint32), ("l_key", C.c_uint32), ("l_ks", C.c_uint32),
        ("base_ep", C.c_uint32), ("base_key", C.c_uint32), ("base_ks", C.c_uint32),
        ("target_num_pt", C.c_uint64), ("num_pt", C.c_uint64),
        ("fst_dim_sz", C.c_uint64), ("other_dim_sz", C.c_uint64),
        ("num_dims", C.c_uint32), ("expansion_height", C.c_uint32),
        ("fst_dim_pow2", C.c_uint32),
    ]

    @property
    def useful(self) -> int:
        return self.fst_dim_sz + self.l_ep * (self.num_dims - 1)


def build() -> str:
    """Compile libopir_oracle.so (the C restatement) if it is missing."""
    if not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "libopir_oracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        L.oracle_params_init.argtypes = [C.c_uint64, C.c_uint32, C.c_int, C.POINTER(Params)]
        L.oracle_k1p_params_init.argtypes = [C.c_uint64, C.c_uint32, C.c_int, C.POINTER(Params)]
        L.oracle_client_new.argtypes = [C.POINTER(Params), C.c_uint64]
        L.oracle_client_new.restype = C.c_void_p
        L.oracle_client_new_keygen_parts.argtypes = [C.POINTER(Params), C.c_uint64, _u64p,
                                                     C.POINTER(C.c_int64), _u64p,
                                                     C.POINTER(C.c_int64)]
        L.oracle_client_new_keygen_parts.restype = C.c_void_p
        L.oracle_client_free.argtypes = [C.c_void_p]
        L.oracle_client_bv_keys.argtypes = [C.c_void_p, _u64p]
        L.oracle_client_gsw_key.argtypes = [C.c_void_p, _u64p]
        L.oracle_client_query.argtypes = [C.c_void_p, C.c_uint64, _u64p]
        L.oracle_client_query_with_a.argtypes = [C.c_void_p, C.c_uint64, _u64p, _u64p]
        L.oracle_client_decrypt.argtypes = [C.c_void_p, _u64p, _u64p]
        L.oracle_client_decrypt_noise.argtypes = [C.c_void_p, _u64p, _u64p, _u64p]
        L.oracle_client_query_parts.argtypes = [C.c_void_p, C.c_uint64, _u64p, _u64p,
                                                C.POINTER(C.c_int64)]
        L.oracle_client_secret.argtypes = [C.c_void_p, C.POINTER(C.c_int8)]
        L.oracle_client_tree_query.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint64,
                                               C.POINTER(C.c_uint8), C.c_uint32, _u64p]
        L.oracle_client_decrypt_q.argtypes = [C.c_void_p, _u64p, _u64p]
        L.oracle_client_tree_query_parts.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32,
                                                     C.c_uint64, C.POINTER(C.c_uint8),
                                                     C.c_uint32, _u64p, _u64p,
                                                     C.POINTER(C.c_int64)]
        L.oracle_server_new.argtypes = [C.POINTER(Params)]
        L.oracle_server_new.restype = C.c_void_p
        L.oracle_server_free.argtypes = [C.c_void_p]
        L.oracle_server_load_seeded.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.oracle_server_load.argtypes = [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint16)]
        L.oracle_server_set_keys.argtypes = [C.c_void_p, _u64p, _u64p]
        for f in ("oracle_server_expand", "oracle_server_complete_selectors",
                  "oracle_server_first_dim", "oracle_server_make_query"):
            getattr(L, f).argtypes = [C.c_void_p, _u64p, _u64p]
        L.oracle_server_other_dim.argtypes = [C.c_void_p, _u64p, _u64p, _u64p]
        L.oracle_ext_prod_mux.argtypes = [C.POINTER(Params), _u64p, _u64p, _u64p, _u64p]
        L.oracle_mod_switch.argtypes = [C.POINTER(Params), _u64p]
        L.oracle_serialize.argtypes = [C.POINTER(Params), _u64p, C.POINTER(C.c_uint8)]
        L.oracle_serialize.restype = C.c_size_t
        L.oracle_ntt_fwd.argtypes = [_u64p, C.c_uint32, C.c_uint64, C.c_uint64]
        L.oracle_ntt_inv.argtypes = [_u64p, C.c_uint32, C.c_uint64, C.c_uint64]
        L.oracle_min_primitive_root.argtypes = [C.c_uint64, C.c_uint64]
        L.oracle_min_primitive_root.restype = C.c_uint64
        L.oracle_generate_prime.argtypes = [C.c_uint32]
        L.oracle_generate_prime.restype = C.c_uint64
        L.oracle_is_prime.argtypes = [C.c_uint64]
        L.oracle_calc_db_shape.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32, C.c_int,
                                           _u64p, _u64p]
        L.oracle_rescale.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.oracle_rescale.restype = C.c_uint64
        L.oracle_signed_decompose.argtypes = [C.c_uint64, C.c_uint32, C.c_uint64, _u64p, C.c_uint32]
        L.oracle_mt_test.argtypes = [C.c_uint64, C.c_uint64]
        L.oracle_mt_test.restype = C.c_uint64
        L.oracle_db_coeff.argtypes = [C.c_uint64] * 5
        L.oracle_db_coeff.restype = C.c_uint64
        L.oracle_db_plaintext.argtypes = [C.c_uint64, C.c_uint64, C.POINTER(Params),
                                          C.POINTER(C.c_uint16)]
        L.oracle_level_mat_mat_32.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                              _u64p, C.c_uint64, C.c_uint64, C.c_uint64,
                                              C.c_uint64]
        L.oracle_external_product.argtypes = [C.POINTER(Params), _u64p, C.c_uint32, C.c_uint32,
                                              _u64p, _u64p]
        L.oracle_bv_apply_galois.argtypes = [C.POINTER(Params), _u64p, C.c_uint32, _u64p]
        P4 = C.POINTER(C4Params)
        L.oracle_c4_params_init.argtypes = [C.c_uint64, C.c_uint32, C.c_int, P4]
        L.oracle_k2mp_params_init.argtypes = [C.c_uint64, C.c_uint32, C.c_int, P4]
        L.oracle_c4_db_plaintext.argtypes = [C.c_uint64, C.c_uint64, P4, _u64p]
        L.oracle_c4_client_new.argtypes = [P4, C.c_uint64]
        L.oracle_c4_client_new.restype = C.c_void_p
        L.oracle_c4_client_new_keygen_parts.argtypes = [C.POINTER(C4Params), C.c_uint64, _u64p,
                                                        C.POINTER(C.c_int64), _u64p,
                                                        C.POINTER(C.c_int64)]
        L.oracle_c4_client_new_keygen_parts.restype = C.c_void_p
        L.oracle_c4_client_free.argtypes = [C.c_void_p]
        L.oracle_c4_client_bv_keys.argtypes = [C.c_void_p, _u64p]
        L.oracle_c4_client_gsw_key.argtypes = [C.c_void_p, _u64p]
        L.oracle_c4_client_query.argtypes = [C.c_void_p, C.c_uint64, _u64p]
        L.oracle_c4_client_decrypt.argtypes = [C.c_void_p, _u64p, _u64p]
        L.oracle_c4_client_decrypt_noise.argtypes = [C.c_void_p, _u64p, _u64p, _u64p]
        L.oracle_c4_client_query_parts.argtypes = [C.c_void_p, C.c_uint64, _u64p, _u64p,
                                                   C.POINTER(C.c_int64)]
        L.oracle_c4_client_secret.argtypes = [C.c_void_p, C.POINTER(C.c_int8)]
        L.oracle_c4_client_tree_query.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32,
                                                  C.c_uint64, C.POINTER(C.c_uint8), C.c_uint32,
                                                  _u64p]
        L.oracle_c4_client_tree_query_parts.argtypes = [C.c_void_p, C.c_uint64, C.c_uint32,
                                                        C.c_uint64, C.POINTER(C.c_uint8),
                                                        C.c_uint32, _u64p, _u64p,
                                                        C.POINTER(C.c_int64)]
        L.oracle_c4_server_new.argtypes = [P4]
        L.oracle_c4_server_new.restype = C.c_void_p
        L.oracle_c4_server_free.argtypes = [C.c_void_p]
        L.oracle_c4_server_load_seeded.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64]
        L.oracle_c4_server_set_keys.argtypes = [C.c_void_p, _u64p, _u64p]
        for f in ("oracle_c4_server_expand", "oracle_c4_server_complete_selectors",
                  "oracle_c4_server_first_dim", "oracle_c4_server_make_query"):
            getattr(L, f).argtypes = [C.c_void_p, _u64p, _u64p]
        L.oracle_c4_server_other_dim.argtypes = [C.c_void_p, _u64p, _u64p, _u64p]
        L.oracle_c4_ext_prod_mux.argtypes = [P4, _u64p, _u64p, _u64p, _u64p]
        L.oracle_c4_mod_switch.argtypes = [P4, _u64p, _u64p]
        L.oracle_c4_serialize.argtypes = [P4, _u64p, C.POINTER(C.c_uint8)]
        L.oracle_c4_serialize.restype = C.c_size_t
        _lib = L
    return _lib


def ptr(a: np.ndarray, ctype=C.c_uint64):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


def params(target: int, height: int, pow2: bool = True) -> Params:
    p = Params()
    rc = lib().oracle_params_init(target, height, 1 if pow2 else 0, C.byref(p))
    if rc != 0:
        raise ValueError(f"invalid layout target={target} height={height}")
    return p


def k1p_params(target: int, height: int, pow2: bool = True) -> Params:
    """CONFIG_N2048_K1 (the reference's default): one 60-bit NTT prime
    (q1 = q2 = 0 in the struct); the Client/Server classes and functions take
    these parameters too."""
    p = Params()
    rc = lib().oracle_k1p_params_init(target, height, 1 if pow2 else 0, C.byref(p))
    if rc != 0:
        raise ValueError(f"invalid layout target={target} height={height}")
    return p


def db_plaintext(seed: int, pt: int, p: Params) -> np.ndarray:
    out = np.empty(p.N, dtype=np.uint16)
    lib().oracle_db_plaintext(seed, pt, C.byref(p), ptr(out, C.c_uint16))
    return out


class Client:
    """Seeded client: the reference client with seeded generators."""

    def __init__(self, p: Params, seed: int, keygen_parts: bool = False):
        """keygen_parts keeps the randomness key generation drew in
        self.keygen: bv_a / bv_e (h, L_KS, N), gsw_a / gsw_e (2 L_KEY, N)."""
        self.p = p
        if keygen_parts:
            h = max(p.expansion_height, 0)
            k = {"bv_a": np.zeros((h, p.l_ks, p.N), np.uint64),
                 "bv_e": np.zeros((h, p.l_ks, p.N), np.int64),
                 "gsw_a": np.zeros((2 * p.l_key, p.N), np.uint64),
                 "gsw_e": np.zeros((2 * p.l_key, p.N), np.int64)}
            bv_a = k["bv_a"] if h else np.zeros(1, np.uint64)
            bv_e = k["bv_e"] if h else np.zeros(1, np.int64)
            self.h = lib().oracle_client_new_keygen_parts(
                C.byref(p), seed, ptr(bv_a), ptr(bv_e, C.c_int64), ptr(k["gsw_a"]),
                ptr(k["gsw_e"], C.c_int64))
            self.keygen = k
        else:
            self.h = lib().oracle_client_new(C.byref(p), seed)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_client_free(self.h)
            self.h = None

    def bv_keys(self) -> np.ndarray:
        p = self.p
        out = np.zeros((max(p.expansion_height, 0), p.l_ks, 2, p.N), dtype=np.uint64)
        if p.expansion_height:
            lib().oracle_client_bv_keys(self.h, ptr(out))
        return out

    def gsw_key(self) -> np.ndarray:
        p = self.p
        out = np.zeros((2 * p.l_key, 2, p.N), dtype=np.uint64)
        lib().oracle_client_gsw_key(self.h, ptr(out))
        return out

    def query(self, idx: int) -> np.ndarray:
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        if lib().oracle_client_query(self.h, idx, ptr(out)) != 0:
            raise IndexError("plaintext index outside the layout")
        return out

    def query_with_a(self, idx: int, a: np.ndarray) -> np.ndarray:
        """The query for idx with c1 = a (a seed-compressed query)."""
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        aa = np.ascontiguousarray(a, dtype=np.uint64)
        if lib().oracle_client_query_with_a(self.h, idx, ptr(aa), ptr(out)) != 0:
            raise IndexError("plaintext index outside the layout")
        return out

    def decrypt(self, resp: np.ndarray) -> np.ndarray:
        resp = np.ascontiguousarray(resp, dtype=np.uint64)
        out = np.zeros(self.p.N, dtype=np.uint64)
        lib().oracle_client_decrypt(self.h, ptr(resp), ptr(out))
        return out

    def decrypt_noise(self, resp: np.ndarray) -> tuple[np.ndarray, int]:
        """decrypt_mod_q (client.cpp:364-410) and the max noise it reports."""
        resp = np.ascontiguousarray(resp, dtype=np.uint64)
        out = np.zeros(self.p.N, dtype=np.uint64)
        noise = np.zeros(1, dtype=np.uint64)
        lib().oracle_client_decrypt_noise(self.h, ptr(resp), ptr(out), ptr(noise))
        return out, int(noise[0])

    def secret(self) -> np.ndarray:
        """The ternary secret in coefficient form (N int8 in {-1, 0, 1})."""
        out = np.zeros(self.p.N, dtype=np.int8)
        lib().oracle_client_secret(self.h, ptr(out, C.c_int8))
        return out

    def query_parts(self, idx: int, a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """The query for idx with c1 = a, and the error e (N int64) it drew."""
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        e = np.zeros(self.p.N, dtype=np.int64)
        aa = np.ascontiguousarray(a, dtype=np.uint64)
        if lib().oracle_client_query_parts(self.h, idx, ptr(aa), ptr(out), ptr(e, C.c_int64)) != 0:
            raise IndexError("plaintext index outside the layout")
        return out, e

    def tree_query(self, N0: int, h_q: int, alpha: int, beta_bits, gamma_bits) -> np.ndarray:
        """make_tree_query (tree_query.cpp:142-196) for client coordinates."""
        bits = np.ascontiguousarray(np.asarray(list(beta_bits) + list(gamma_bits) or [0],
                                               dtype=np.uint8))
        groups = len(beta_bits) + len(gamma_bits)
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        if lib().oracle_client_tree_query(self.h, N0, h_q, alpha, ptr(bits, C.c_uint8), groups,
                                          ptr(out)) != 0:
            raise ValueError("tree query shape does not fit")
        return out

    def tree_query_parts(self, N0: int, h_q: int, alpha: int, beta_bits, gamma_bits,
                         a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """tree_query with c1 = a, and the error it drew."""
        bits = np.ascontiguousarray(np.asarray(list(beta_bits) + list(gamma_bits) or [0],
                                               dtype=np.uint8))
        groups = len(beta_bits) + len(gamma_bits)
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        e = np.zeros(self.p.N, dtype=np.int64)
        aa = np.ascontiguousarray(a, dtype=np.uint64)
        if lib().oracle_client_tree_query_parts(self.h, N0, h_q, alpha, ptr(bits, C.c_uint8),
                                                groups, ptr(aa), ptr(out),
                                                ptr(e, C.c_int64)) != 0:
            raise ValueError("tree query shape does not fit")
        return out, e

    def decrypt_q(self, ct: np.ndarray) -> np.ndarray:
        """decrypt_rns (rlwe.cpp:310-348) of a coefficient-form ciphertext mod q."""
        c = np.ascontiguousarray(ct, dtype=np.uint64)
        out = np.zeros(self.p.N, dtype=np.uint64)
        lib().oracle_client_decrypt_q(self.h, ptr(c), ptr(out))
        return out


class Server:
    def __init__(self, p: Params):
        self.p = p
        self.h = lib().oracle_server_new(C.byref(p))
        if not self.h:
            raise MemoryError("oracle server allocation failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_server_free(self.h)
            self.h = None

    def load_seeded(self, logical: int, seed: int):
        assert lib().oracle_server_load_seeded(self.h, logical, seed) == 0

    def load(self, coeffs: np.ndarray, logical: int | None = None):
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint16)
        n = coeffs.shape[0] if logical is None else logical
        rc = lib().oracle_server_load(self.h, n, ptr(coeffs, C.c_uint16))
        if rc != 0:
            raise ValueError("plaintext source rejected")

    def set_keys(self, bv: np.ndarray, gsw: np.ndarray):
        bv = np.ascontiguousarray(bv, dtype=np.uint64)
        gsw = np.ascontiguousarray(gsw, dtype=np.uint64)
        lib().oracle_server_set_keys(self.h, ptr(bv), ptr(gsw))

    def expand(self, query: np.ndarray) -> np.ndarray:
        out = np.zeros((self.p.useful, 2, self.p.N), dtype=np.uint64)
        q = np.ascontiguousarray(query, dtype=np.uint64)
        assert lib().oracle_server_expand(self.h, ptr(q), ptr(out)) == 0
        return out

    def complete_selectors(self, expanded: np.ndarray) -> np.ndarray:
        p = self.p
        out = np.zeros((max(p.num_dims - 1, 1), 2 * p.l_ep, 2, p.N), dtype=np.uint64)
        e = np.ascontiguousarray(expanded, dtype=np.uint64)
        assert lib().oracle_server_complete_selectors(self.h, ptr(e), ptr(out)) == 0
        return out[: p.num_dims - 1]

    def first_dim(self, fst_query: np.ndarray) -> np.ndarray:
        p = self.p
        out = np.zeros((p.other_dim_sz, 2, p.N), dtype=np.uint64)
        f = np.ascontiguousarray(fst_query[: p.fst_dim_sz], dtype=np.uint64)
        assert lib().oracle_server_first_dim(self.h, ptr(f), ptr(out)) == 0
        return out

    def other_dim(self, mid: np.ndarray, selectors: np.ndarray) -> np.ndarray:
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        m = np.array(mid, dtype=np.uint64, copy=True, order="C")
        s = np.ascontiguousarray(selectors, dtype=np.uint64)
        if s.size == 0:
            s = np.zeros(1, dtype=np.uint64)
        assert lib().oracle_server_other_dim(self.h, ptr(m), ptr(s), ptr(out)) == 0
        return out

    def make_query(self, query: np.ndarray) -> np.ndarray:
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        q = np.ascontiguousarray(query, dtype=np.uint64)
        assert lib().oracle_server_make_query(self.h, ptr(q), ptr(out)) == 0
        return out


def serialize(p: Params, resp: np.ndarray) -> bytes:
    r = np.ascontiguousarray(resp, dtype=np.uint64)
    buf = np.zeros(2 * p.N * 8, dtype=np.uint8)
    n = lib().oracle_serialize(C.byref(p), ptr(r), ptr(buf, C.c_uint8))
    return buf[:n].tobytes()


# ---------------------------------------------------------------- CONFIG_N4096_K2_MP
def c4_params(target: int, height: int, pow2: bool = True) -> C4Params:
    p = C4Params()
    if lib().oracle_c4_params_init(target, height, 1 if pow2 else 0, C.byref(p)) != 0:
        raise ValueError(f"invalid layout target={target} height={height}")
    return p


def k2mp_params(target: int, height: int, pow2: bool = True) -> C4Params:
    """CONFIG_N2048_K2_MP: the two-limb routines at N = 2048 with 29-bit limbs
    (the C4* classes and functions take these parameters too)."""
    p = C4Params()
    if lib().oracle_k2mp_params_init(target, height, 1 if pow2 else 0, C.byref(p)) != 0:
        raise ValueError(f"invalid layout target={target} height={height}")
    return p


def c4_db_plaintext(seed: int, pt: int, p: C4Params) -> np.ndarray:
    out = np.empty(p.N, dtype=np.uint64)
    lib().oracle_c4_db_plaintext(seed, pt, C.byref(p), ptr(out))
    return out


class C4Client:
    """Seeded two-limb client: the reference client (K = 2) with seeded generators.
    Ciphertexts are (2, 2, N): poly x limb x coefficient."""

    def __init__(self, p: C4Params, seed: int, keygen_parts: bool = False):
        """keygen_parts keeps the key-generation randomness in self.keygen:
        bv_a (h, L_KS, 2, N), bv_e (h, L_KS, N), gsw_a (2 L_KEY, 2, N),
        gsw_e (2 L_KEY, N)."""
        self.p = p
        if keygen_parts:
            h = max(p.expansion_height, 0)
            k = {"bv_a": np.zeros((h, p.l_ks, 2, p.N), np.uint64),
                 "bv_e": np.zeros((h, p.l_ks, p.N), np.int64),
                 "gsw_a": np.zeros((2 * p.l_key, 2, p.N), np.uint64),
                 "gsw_e": np.zeros((2 * p.l_key, p.N), np.int64)}
            bv_a = k["bv_a"] if h else np.zeros(1, np.uint64)
            bv_e = k["bv_e"] if h else np.zeros(1, np.int64)
            self.h = lib().oracle_c4_client_new_keygen_parts(
                C.byref(p), seed, ptr(bv_a), ptr(bv_e, C.c_int64), ptr(k["gsw_a"]),
                ptr(k["gsw_e"], C.c_int64))
            self.keygen = k
        else:
            self.h = lib().oracle_c4_client_new(C.byref(p), seed)

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_c4_client_free(self.h)
            self.h = None

    def bv_keys(self) -> np.ndarray:
        p = self.p
        out = np.zeros((max(p.expansion_height, 0), p.l_ks, 2, 2, p.N), dtype=np.uint64)
        if p.expansion_height:
            lib().oracle_c4_client_bv_keys(self.h, ptr(out))
        return out

    def gsw_key(self) -> np.ndarray:
        p = self.p
        out = np.zeros((2 * p.l_key, 2, 2, p.N), dtype=np.uint64)
        lib().oracle_c4_client_gsw_key(self.h, ptr(out))
        return out

    def query(self, idx: int) -> np.ndarray:
        out = np.zeros((2, 2, self.p.N), dtype=np.uint64)
        if lib().oracle_c4_client_query(self.h, idx, ptr(out)) != 0:
            raise IndexError("plaintext index outside the layout")
        return out

    def decrypt(self, resp: np.ndarray) -> np.ndarray:
        resp = np.ascontiguousarray(resp, dtype=np.uint64)
        out = np.zeros(self.p.N, dtype=np.uint64)
        lib().oracle_c4_client_decrypt(self.h, ptr(resp), ptr(out))
        return out

    def decrypt_noise(self, resp: np.ndarray) -> tuple[np.ndarray, int]:
        resp = np.ascontiguousarray(resp, dtype=np.uint64)
        out = np.zeros(self.p.N, dtype=np.uint64)
        noise = np.zeros(1, dtype=np.uint64)
        lib().oracle_c4_client_decrypt_noise(self.h, ptr(resp), ptr(out), ptr(noise))
        return out, int(noise[0])

    def secret(self) -> np.ndarray:
        out = np.zeros(self.p.N, dtype=np.int8)
        lib().oracle_c4_client_secret(self.h, ptr(out, C.c_int8))
        return out

    def query_parts(self, idx: int, a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """The query for idx with c1 = a (2, N limb-major), and the shared error e."""
        out = np.zeros((2, 2, self.p.N), dtype=np.uint64)
        e = np.zeros(self.p.N, dtype=np.int64)
        aa = np.ascontiguousarray(a, dtype=np.uint64)
        if lib().oracle_c4_client_query_parts(self.h, idx, ptr(aa), ptr(out),
                                              ptr(e, C.c_int64)) != 0:
            raise IndexError("plaintext index outside the layout")
        return out, e

    def tree_query_parts(self, N0: int, h_q: int, alpha: int, beta_bits, gamma_bits,
                         a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        bits = np.ascontiguousarray(np.asarray(list(beta_bits) + list(gamma_bits) or [0],
                                               dtype=np.uint8))
        groups = len(beta_bits) + len(gamma_bits)
        out = np.zeros((2, 2, self.p.N), dtype=np.uint64)
        e = np.zeros(self.p.N, dtype=np.int64)
        aa = np.ascontiguousarray(a, dtype=np.uint64)
        if lib().oracle_c4_client_tree_query_parts(self.h, N0, h_q, alpha, ptr(bits, C.c_uint8),
                                                   groups, ptr(aa), ptr(out),
                                                   ptr(e, C.c_int64)) != 0:
            raise ValueError("tree query shape does not fit")
        return out, e

    def tree_query(self, N0: int, h_q: int, alpha: int, beta_bits, gamma_bits) -> np.ndarray:
        """make_tree_query (tree_query.cpp:142-196), K = 2."""
        bits = np.ascontiguousarray(np.asarray(list(beta_bits) + list(gamma_bits) or [0],
                                               dtype=np.uint8))
        groups = len(beta_bits) + len(gamma_bits)
        out = np.zeros((2, 2, self.p.N), dtype=np.uint64)
        if lib().oracle_c4_client_tree_query(self.h, N0, h_q, alpha, ptr(bits, C.c_uint8), groups,
                                             ptr(out)) != 0:
            raise ValueError("tree query shape does not fit")
        return out


class C4Server:
    def __init__(self, p: C4Params):
        self.p = p
        self.h = lib().oracle_c4_server_new(C.byref(p))
        if not self.h:
            raise MemoryError("oracle server allocation failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_c4_server_free(self.h)
            self.h = None

    def load_seeded(self, logical: int, seed: int):
        assert lib().oracle_c4_server_load_seeded(self.h, logical, seed) == 0

    def set_keys(self, bv: np.ndarray, gsw: np.ndarray):
        bv = np.ascontiguousarray(bv, dtype=np.uint64)
        gsw = np.ascontiguousarray(gsw, dtype=np.uint64)
        if bv.size == 0:
            bv = np.zeros(1, dtype=np.uint64)
        lib().oracle_c4_server_set_keys(self.h, ptr(bv), ptr(gsw))

    def expand(self, query: np.ndarray) -> np.ndarray:
        out = np.zeros((self.p.useful, 2, 2, self.p.N), dtype=np.uint64)
        q = np.ascontiguousarray(query, dtype=np.uint64)
        assert lib().oracle_c4_server_expand(self.h, ptr(q), ptr(out)) == 0
        return out

    def complete_selectors(self, expanded: np.ndarray) -> np.ndarray:
        p = self.p
        out = np.zeros((max(p.num_dims - 1, 1), 2 * p.l_ep, 2, 2, p.N), dtype=np.uint64)
        e = np.ascontiguousarray(expanded, dtype=np.uint64)
        assert lib().oracle_c4_server_complete_selectors(self.h, ptr(e), ptr(out)) == 0
        return out[: p.num_dims - 1]

    def first_dim(self, fst_query: np.ndarray) -> np.ndarray:
        p = self.p
        out = np.zeros((p.other_dim_sz, 2, 2, p.N), dtype=np.uint64)
        f = np.ascontiguousarray(fst_query[: p.fst_dim_sz], dtype=np.uint64)
        assert lib().oracle_c4_server_first_dim(self.h, ptr(f), ptr(out)) == 0
        return out

    def other_dim(self, mid: np.ndarray, selectors: np.ndarray) -> np.ndarray:
        out = np.zeros((2, 2, self.p.N), dtype=np.uint64)
        m = np.array(mid, dtype=np.uint64, copy=True, order="C")
        s = np.ascontiguousarray(selectors, dtype=np.uint64)
        if s.size == 0:
            s = np.zeros(1, dtype=np.uint64)
        assert lib().oracle_c4_server_other_dim(self.h, ptr(m), ptr(s), ptr(out)) == 0
        return out

    def make_query(self, query: np.ndarray) -> np.ndarray:
        out = np.zeros((2, self.p.N), dtype=np.uint64)
        q = np.ascontiguousarray(query, dtype=np.uint64)
        assert lib().oracle_c4_server_make_query(self.h, ptr(q), ptr(out)) == 0
        return out


def c4_mod_switch(p: C4Params, ct: np.ndarray) -> np.ndarray:
    out = np.zeros((2, p.N), dtype=np.uint64)
    c = np.ascontiguousarray(ct, dtype=np.uint64)
    lib().oracle_c4_mod_switch(C.byref(p), ptr(c), ptr(out))
    return out


def c4_serialize(p: C4Params, resp: np.ndarray) -> bytes:
    r = np.ascontiguousarray(resp, dtype=np.uint64)
    buf = np.zeros(2 * p.N * 8, dtype=np.uint8)
    n = lib().oracle_c4_serialize(C.byref(p), ptr(r), ptr(buf, C.c_uint8))
    return buf[:n].tobytes()


# ----------------------------------------------------------------------------
# Row shards: the reference's evaluate_other_dim (server.cpp:599-649) split by
# MUX level, and the candidate rows that feed each level-1 position.

def ext_prod_mux(p, x: np.ndarray, y: np.ndarray, sel: np.ndarray) -> np.ndarray:
    """PirServer::ext_prod_mux (server.cpp:652-722): x + INTT(ExtProd(sel, y - x))."""
    xx = np.ascontiguousarray(x, dtype=np.uint64)
    yy = np.array(y, dtype=np.uint64, copy=True, order="C")
    ss = np.ascontiguousarray(sel, dtype=np.uint64)
    out = np.zeros_like(xx)
    if isinstance(p, C4Params):
        lib().oracle_c4_ext_prod_mux(C.byref(p), ptr(xx), ptr(yy), ptr(ss), ptr(out))
    else:
        lib().oracle_ext_prod_mux(C.byref(p), ptr(xx), ptr(yy), ptr(ss), ptr(out))
    return out


def mux_levels(p, mid: np.ndarray, selectors: np.ndarray, tree_h: int, begin: int,
               end: int) -> np.ndarray:
    """Levels [begin, end) of evaluate_other_dim's MUX tree of height tree_h
    over the candidates `mid` (level 0: rows offset + 2i and offset + 2i + 1
    into offset + i, offset = 2^tree_h - len(mid); level a >= 1: i and
    i + 2^(tree_h-a-1) into i), selector slot a at level a. Returns the
    positions left after level end - 1."""
    cur = [np.array(c, dtype=np.uint64) for c in mid]
    for a in range(begin, end):
        if a == 0:
            other = len(cur)
            last = 2 * other - (1 << tree_h)
            offset = other - last
            nxt = cur[:offset]
            for i in range(0, last, 2):
                nxt.append(ext_prod_mux(p, cur[offset + i], cur[offset + i + 1], selectors[0]))
        else:
            half = (1 << (tree_h - a)) >> 1
            nxt = [ext_prod_mux(p, cur[i], cur[i + half], selectors[a]) for i in range(half)]
        cur = nxt
    return np.stack(cur)


def shard_rows(other: int, num_dims: int, shard: int, num_shards: int) -> list[int]:
    """Candidate rows feeding the level-1 positions s = shard (mod num_shards):
    row s when s < offset (carried over at level 0), else rows 2s - offset and
    2s - offset + 1 (server.cpp:626-635), in increasing s."""
    h = num_dims - 1
    offset = other - (2 * other - (1 << h))
    rows = []
    for s in range(shard, 1 << (h - 1), num_shards):
        rows += [s] if s < offset else [2 * s - offset, 2 * s - offset + 1]
    return rows


def sharded_other_dim(p, mid: np.ndarray, selectors: np.ndarray, num_shards: int):
    """evaluate_other_dim computed as num_shards row shards plus a combine:
    returns (partials, result) with partials[g] = shard g's ciphertext after
    its levels 0 .. h - log2 G - 1 and result = the full tree's output."""
    h = p.num_dims - 1
    k = num_shards.bit_length() - 1
    partials = []
    for g in range(num_shards):
        rows = shard_rows(p.other_dim_sz, p.num_dims, g, num_shards)
        left = mux_levels(p, mid[rows], selectors, h - k, 0, h - k)
        assert len(left) == 1
        partials.append(left[0])
    result = mux_levels(p, np.stack(partials), selectors, h, h - k, h)
    return np.stack(partials), result[0]
