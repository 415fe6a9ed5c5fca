"""ctypes binding of libonionpir_b200.so (include/onionpir_b200.h).

The library is built in-tree (onionpirv2_b200/libonionpir_b200.so). Loading
fails loudly if it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libonionpir_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "onionpir_b200.h")

u64p = C.POINTER(C.c_uint64)
u32p = C.POINTER(C.c_uint32)
u16p = C.POINTER(C.c_uint16)
u8p = C.POINTER(C.c_uint8)


class Layout(C.Structure):
    _fields_ = [("target_num_pt", C.c_uint64), ("expansion_height", C.c_uint32),
                ("fst_dim_pow2", C.c_uint32)]


class Params(C.Structure):
    _fields_ = [
        ("poly_degree", C.c_uint32), ("num_limbs", C.c_uint32),
        ("q", C.c_uint64), ("q1", C.c_uint64), ("q2", C.c_uint64),
        ("w1", C.c_uint64), ("w2", C.c_uint64), ("w_crt", C.c_uint64),
        ("q1_inv_mod_q2", C.c_uint64), ("plain_mod", C.c_uint64), ("small_q", C.c_uint64),
        ("small_q_width", C.c_uint32), ("ct_mod_width", C.c_uint32),
        ("l_ep", C.c_uint32), ("l_key", C.c_uint32), ("l_ks", C.c_uint32),
        ("base_log2", C.c_uint32), ("base_log2_key", C.c_uint32), ("base_log2_ks", C.c_uint32),
        ("target_num_pt", C.c_uint64), ("num_pt", C.c_uint64), ("fst_dim_sz", C.c_uint64),
        ("other_dim_sz", C.c_uint64), ("num_dims", C.c_uint32), ("expansion_height", C.c_uint32),
        ("fst_dim_pow2", C.c_uint32), ("view", C.c_uint32),
    ]


class QueryShape(C.Structure):
    _fields_ = [("fst_dim_sz", C.c_uint64), ("num_selector_bits", C.c_uint32),
                ("expansion_height", C.c_uint32)]


class TreeParams(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in
                ("N", "L", "n", "g", "rho", "r", "N0", "a", "P", "B", "b",
                 "ell_beta", "ell_gamma", "w", "h_q", "W", "t")]


class TreeLevelPlan(C.Structure):
    _fields_ = [("level", C.c_uint64), ("R", C.c_uint64), ("select_case", C.c_uint32),
                ("reserved", C.c_uint32), ("coarsen_count", C.c_uint64),
                ("beta_begin", C.c_uint64), ("beta_count", C.c_uint64),
                ("gamma_begin", C.c_uint64), ("gamma_count", C.c_uint64),
                ("projection_depth", C.c_uint64)]


class MemoryPlan(C.Structure):
    _fields_ = [("database_bytes", C.c_uint64), ("client_key_bytes", C.c_uint64),
                ("scratch_bytes_per_query", C.c_uint64), ("scratch_bytes_fixed", C.c_uint64)]


SOURCE_CB = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64, u64p)

_SIGS = {
    "opir_version": ([], C.c_char_p),
    "opir_params_query_shape": ([C.POINTER(Params), C.POINTER(QueryShape), C.POINTER(Params)],
                                C.c_int),
    "opir_tree_params_make": ([C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64,
                               C.c_uint64, u64p, C.c_uint32, C.POINTER(TreeParams)], C.c_int),
    "opir_tree_params_init": ([C.c_uint64, C.c_uint64, C.POINTER(Params), C.POINTER(TreeParams)],
                              C.c_int),
    "opir_tree_level_plans": ([C.POINTER(TreeParams), C.POINTER(TreeLevelPlan)], C.c_int),
    "opir_tree_query_params": ([C.POINTER(TreeParams), C.POINTER(Params), C.POINTER(Params)],
                               C.c_int),
    "opir_tree_level_create": ([C.POINTER(Params), C.POINTER(TreeParams), C.c_uint64, u64p,
                                C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "opir_tree_select_level": ([C.c_void_p, u64p, u64p, u64p], C.c_int),
    "opir_tree_create": ([C.POINTER(Params), C.POINTER(TreeParams), C.POINTER(u64p), C.c_int,
                          C.POINTER(C.c_void_p)], C.c_int),
    "opir_tree_destroy": ([C.c_void_p], None),
    "opir_tree_last_error": ([C.c_void_p], C.c_char_p),
    "opir_tree_set_client_keys": ([C.c_void_p, C.c_uint64, u64p, u32p, C.c_uint32, u64p], C.c_int),
    "opir_tree_query": ([C.c_void_p, C.c_uint64, u64p, u64p], C.c_int),
    "opir_params_init": ([C.POINTER(Layout), C.POINTER(Params)], C.c_int),
    "opir_params_init_config": ([C.c_int, C.POINTER(Layout), C.POINTER(Params)], C.c_int),
    "opir_response_bytes": ([C.POINTER(Params)], C.c_size_t),
    "opir_server_create": ([C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "opir_server_destroy": ([C.c_void_p], None),
    "opir_server_last_error": ([C.c_void_p], C.c_char_p),
    "opir_server_params": ([C.c_void_p, C.POINTER(Params)], C.c_int),
    "opir_server_load_db": ([C.c_void_p, C.c_uint64, u64p], C.c_int),
    "opir_server_load_db_u16": ([C.c_void_p, C.c_uint64, u16p], C.c_int),
    "opir_server_load_db_source": ([C.c_void_p, C.c_uint64, SOURCE_CB, C.c_void_p], C.c_int),
    "opir_server_load_db_seeded": ([C.c_void_p, C.c_uint64, C.c_uint64], C.c_int),
    "opir_server_set_client_keys": ([C.c_void_p, C.c_uint64, u64p, u32p, C.c_uint32, u64p], C.c_int),
    "opir_server_set_client_keys_ex": ([C.c_void_p, C.c_uint64, u64p, u32p, C.c_uint32, u64p,
                                        C.c_uint32], C.c_int),
    "opir_server_remove_client": ([C.c_void_p, C.c_uint64], C.c_int),
    "opir_server_make_query": ([C.c_void_p, C.c_uint64, u64p, u64p], C.c_int),
    "opir_server_make_query_batch": ([C.c_void_p, C.c_uint32, u64p, u64p, u64p], C.c_int),
    "opir_server_make_query_batch_device": ([C.c_void_p, C.c_uint32, u64p, C.c_void_p,
                                             C.c_void_p, C.c_void_p], C.c_int),
    "opir_row_shard_rows": ([C.POINTER(Params), C.c_uint32, C.c_uint32, u32p, u64p, u32p],
                            C.c_int),
    "opir_server_create_row_shard": ([C.POINTER(Params), C.c_uint32, C.c_uint32, C.c_int,
                                      C.POINTER(C.c_void_p)], C.c_int),
    "opir_server_make_query_shard_batch": ([C.c_void_p, C.c_uint32, u64p, u64p, u64p], C.c_int),
    "opir_server_make_query_shard_batch_device": ([C.c_void_p, C.c_uint32, u64p, C.c_void_p,
                                                   C.c_void_p, C.c_void_p], C.c_int),
    "opir_server_combine_shards": ([C.c_void_p, C.c_uint32, u64p, u64p, u64p], C.c_int),
    "opir_server_combine_shards_device": ([C.c_void_p, C.c_uint32, u64p, C.c_void_p,
                                           C.c_void_p, C.c_void_p], C.c_int),
    "opir_prf_expand": ([C.POINTER(Params), u8p, C.c_uint32, C.c_uint64, u64p], C.c_int),
    "opir_query_wire_bytes": ([C.POINTER(Params)], C.c_size_t),
    "opir_keys_wire_bytes": ([C.POINTER(Params)], C.c_size_t),
    "opir_query_encode": ([C.POINTER(Params), u8p, u64p, u8p, C.c_size_t], C.c_int),
    "opir_query_decode": ([C.POINTER(Params), u8p, C.c_size_t, u64p], C.c_int),
    "opir_keys_encode": ([C.POINTER(Params), u8p, u64p, u64p, u8p, C.c_size_t], C.c_int),
    "opir_keys_decode": ([C.POINTER(Params), u8p, C.c_size_t, u64p, u32p, u64p], C.c_int),
    "opir_plan_memory": ([C.POINTER(Params), C.POINTER(MemoryPlan)], C.c_int),
    "opir_server_reserve": ([C.c_void_p, C.c_uint32], C.c_int),
    "opir_server_set_priority": ([C.c_void_p, C.c_int], C.c_int),
    "opir_server_set_scan_wait_limit": ([C.c_void_p, C.c_uint64], C.c_int),
    "opir_server_level_splits": ([C.c_void_p, C.c_uint32, C.POINTER(C.c_uint8),
                                  C.POINTER(C.c_uint8)], C.c_int),
    "opir_server_autotune": ([C.c_void_p, C.c_uint32], C.c_int),
    "opir_server_scan_tile": ([C.c_void_p, C.c_uint32, u32p, u32p, u32p], C.c_int),
    "opir_server_set_stage_timing": ([C.c_void_p, C.c_int], C.c_int),
    "opir_server_stage_times": ([C.c_void_p, C.POINTER(C.c_float), u32p], C.c_int),
    "opir_launch_count": ([], C.c_uint64),
    "opir_measure_butterfly_rate": ([C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "opir_measure_recombine_rate": ([C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "opir_server_expand_query": ([C.c_void_p, C.c_uint64, u64p, u64p], C.c_int),
    "opir_server_complete_selectors": ([C.c_void_p, C.c_uint64, u64p, u64p], C.c_int),
    "opir_server_evaluate_first_dim": ([C.c_void_p, u64p, u64p], C.c_int),
    "opir_server_evaluate_other_dim": ([C.c_void_p, u64p, u64p, u64p], C.c_int),
    "opir_server_ext_prod_mux": ([C.c_void_p, u64p, u64p, u64p, u64p], C.c_int),
    "opir_save_response": ([C.POINTER(Params), u64p, u8p, C.c_size_t], C.c_size_t),
    "opir_client_create": ([C.POINTER(Params), C.POINTER(C.c_int8), C.c_int,
                            C.POINTER(C.c_void_p)], C.c_int),
    "opir_client_destroy": ([C.c_void_p], None),
    "opir_client_last_error": ([C.c_void_p], C.c_char_p),
    "opir_client_generate_queries_device": ([C.c_void_p, C.c_uint32, u64p, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "opir_client_decrypt_device": ([C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p], C.c_int),
    "opir_client_keygen_device": ([C.c_void_p] + [C.c_void_p] * 6 + [C.c_void_p], C.c_int),
    "opir_client_generate_queries": ([C.c_void_p, C.c_uint32, u64p, u64p,
                                      C.POINTER(C.c_int64), u64p], C.c_int),
    "opir_client_decrypt": ([C.c_void_p, C.c_uint32, u64p, u64p, u64p], C.c_int),
    "opir_client_generate_tree_queries": ([C.c_void_p, C.POINTER(TreeParams), C.c_uint32, u64p,
                                           u8p, C.c_uint32, u64p, C.POINTER(C.c_int64), u64p],
                                          C.c_int),
    "opir_client_keygen": ([C.c_void_p, u64p, C.POINTER(C.c_int64), u64p,
                            C.POINTER(C.c_int64), u64p, u64p], C.c_int),
    "opir_ext_prod_mux_noalloc": ([C.POINTER(Params), C.c_uint32, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
}

_lib = None


def load():
    """Load the in-tree library (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m onionpirv2_b200.build` "
                "(there is no non-CUDA implementation)")
        lib = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def header_symbols() -> list[str]:
    """Every function the public header declares."""
    with open(HEADER) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)   # drop comments
    return sorted(set(re.findall(r"\b(opir_[a-z0-9_]+)\s*\(", text)))
