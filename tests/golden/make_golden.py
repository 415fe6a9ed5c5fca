"""Regenerates the golden fixtures in this folder from the reference itself.

Runs oracle/_ref/opir_ref (the unmodified OnionPIRv2 reference sources, built
by `make -C oracle ref` against the HEXL stand-in) on seeded inputs and stores,
per case: the layout, seeds and index, the serialized 22-bit response stream
(<name>.resp.bin, as written by PirServer::save_resp_to_stream), and SHA-256
digests of the response u64 array and of the client material (query, BV keys,
RGSW key) so a seeded client can be checked against the reference client
without committing megabytes of keys.

A second set (golden_c4.json, c4_*.resp.bin) comes from oracle/_ref/opir_ref_c4,
the same reference built with CONFIG_N4096_K2_MP (N = 4096, two 60-bit RNS
limbs); those cases also store SHA-256 digests of the outputs of the
reference's public stage methods (expand_query, complete_selectors,
evaluate_first_dim, evaluate_other_dim) in the reference's own flat layouts.

Two more sets come from the reference built with the other two parameter
sets it ships: golden_k2mp.json / k2mp_*.resp.bin from oracle/_ref/opir_ref_k2mp
(CONFIG_N2048_K2_MP: N = 2048, two 29-bit RNS limbs, the MP gadget) and
golden_k1p.json / k1p_*.resp.bin from oracle/_ref/opir_ref_k1
(CONFIG_N2048_K1, the reference's default: N = 2048, one 60-bit prime), with
the same stage digests as the CONFIG_N4096_K2_MP set.

A third set (golden_tree.json) runs the reference's tree PIR layer
(src/tree_*.cpp) through the driver's "tree" mode: one packed tree query per
case on the default scheme, unpacked by unpack_tree_query, and the digests of
the query, the alpha one-hot, the beta selectors and select_level's output at
every level (the reference's own Milestone-2 gate, every level decrypting to
its packed plaintext, must hold).

Only needed when the fixtures must change; tests never run it.
    python tests/golden/make_golden.py            # CONFIG_N2048_K1_COMP set
    python tests/golden/make_golden.py --c4       # CONFIG_N4096_K2_MP set
    python tests/golden/make_golden.py --k2mp     # CONFIG_N2048_K2_MP set
    python tests/golden/make_golden.py --k1p      # CONFIG_N2048_K1 set
    python tests/golden/make_golden.py --tree     # tree PIR select_level set
    python tests/golden/make_golden.py --tree --c4  # the same under CONFIG_N4096_K2_MP
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref", "opir_ref")
REF_BIN_C4 = os.path.join(REPO, "oracle", "_ref", "opir_ref_c4")
REF_BIN_K2 = os.path.join(REPO, "oracle", "_ref", "opir_ref_k2mp")
REF_BIN_K1 = os.path.join(REPO, "oracle", "_ref", "opir_ref_k1")

# name, target_num_pt, expansion_height, fst_dim_pow2, db_seed, client_seed, index
CASES = [
    ("c1_16384_h9", 16384, 9, 1, 11, 22, 12345),
    ("c1_16384_h9_first", 16384, 9, 1, 12, 23, 0),
    ("c1_16384_h9_last", 16384, 9, 1, 13, 24, 16383),
    ("c2_262144_h10", 262144, 10, 1, 101, 202, 200003),
    ("ragged_43_h5", 43, 5, 1, 5, 6, 42),
    ("ragged_43_h5_pad", 43, 5, 1, 7, 8, 47),
    ("tight_43_h5", 43, 5, 0, 5, 6, 42),
    ("singleton_1_h0", 1, 0, 1, 5, 6, 0),
    ("small_1000_h7", 1000, 7, 1, 5, 6, 999),
    ("flat_349526_h10", 349526, 10, 1, 31, 32, 349525),
]


# CONFIG_N4096_K2_MP: same columns
CASES_C4 = [
    ("c4_2048_h7", 2048, 7, 1, 3, 4, 777),
    ("c4_2048_h7_last", 2048, 7, 1, 5, 6, 2047),
    ("c4_ragged_43_h5", 43, 5, 1, 7, 8, 42),
    ("c4_tight_100_h6", 100, 6, 0, 9, 10, 57),
    ("c4_singleton_1_h0", 1, 0, 1, 11, 12, 0),
    ("c4_16384_h9", 16384, 9, 1, 13, 14, 9999),
]


# CONFIG_N2048_K2_MP and CONFIG_N2048_K1: same columns
CASES_K2 = [
    ("k2mp_1000_h7", 1000, 7, 1, 3, 4, 777),
    ("k2mp_1000_h7_last", 1000, 7, 1, 5, 6, 999),
    ("k2mp_ragged_43_h5", 43, 5, 1, 7, 8, 42),
    ("k2mp_tight_100_h6", 100, 6, 0, 9, 10, 57),
    ("k2mp_singleton_1_h0", 1, 0, 1, 11, 12, 0),
    ("k2mp_16384_h9", 16384, 9, 1, 13, 14, 9999),
]
CASES_K1 = [(n.replace("k2mp_", "k1p_"), t, h, pw, d + 100, c + 100, i)
            for n, t, h, pw, d, c, i in CASES_K2]

# per set: reference binary, cases, manifest, whether stage digests are kept
SETS = {
    "k1": (REF_BIN, CASES, "golden.json", False,
           "oracle/_ref/opir_ref (reference sources + HEXL stand-in)"),
    "c4": (REF_BIN_C4, CASES_C4, "golden_c4.json", True,
           "oracle/_ref/opir_ref_c4 (reference sources, CONFIG_N4096_K2_MP, + HEXL stand-in)"),
    "k2mp": (REF_BIN_K2, CASES_K2, "golden_k2mp.json", True,
             "oracle/_ref/opir_ref_k2mp (reference sources, CONFIG_N2048_K2_MP, + HEXL stand-in)"),
    "k1p": (REF_BIN_K1, CASES_K1, "golden_k1p.json", True,
            "oracle/_ref/opir_ref_k1 (reference sources, CONFIG_N2048_K1, + HEXL stand-in)"),
}


# (name, L, a, client seed, leaf): the shapes and the boundary, mixed-bit and
# beta-asymmetric leaves of src/tests/test_tree_select.cpp:103-123
def tree_cases():
    out = []
    for L, a, seed in ((16, 3, 31), (13, 2, 32)):
        N, r = 1 << L, 11
        b = L - r - a
        P, B = N >> r, 1 << b
        leaves = [0, N - 1, 0x2BADBEEF % N, P + B + (1 if b >= 2 else 0)]
        for k, leaf in enumerate(leaves):
            out.append((f"tree_L{L}_a{a}_leaf{leaf}", L, a, seed + 10 * k, leaf))
    return out


# the same shapes under CONFIG_N4096_K2_MP (r = log2 4096 = 12): (17, 3) and
# (16, 2), b = 2 for both
def tree_cases_c4():
    out = []
    for L, a, seed in ((17, 3, 41), (16, 2, 42)):
        N, r = 1 << L, 12
        b = L - r - a
        P, B = N >> r, 1 << b
        leaves = [0, N - 1, 0x2BADBEEF % N, P + B + (1 if b >= 2 else 0)]
        for k, leaf in enumerate(leaves):
            out.append((f"tree_c4_L{L}_a{a}_leaf{leaf}", L, a, seed + 10 * k, leaf))
    return out


def sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main_tree(c4: bool = False) -> int:
    ref_bin = REF_BIN_C4 if c4 else REF_BIN
    if not os.path.exists(ref_bin):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref"], check=True)
    manifest = []
    for name, L, a, seed, leaf in (tree_cases_c4() if c4 else tree_cases()):
        with tempfile.TemporaryDirectory() as tmp:
            out = subprocess.run(
                [ref_bin, "--mode", "tree", "--tree-L", str(L), "--tree-a", str(a),
                 "--client-seed", str(seed), "--leaf", str(leaf), "--out", tmp],
                check=True, capture_output=True, text=True)
            info = json.loads(out.stdout.strip().splitlines()[-1])
            if not info["ok"]:
                raise RuntimeError(f"{name}: reference select_level does not decrypt")
            import numpy as np
            levels = np.fromfile(os.path.join(tmp, "levels.u64"), dtype=np.uint64)
            per = levels.reshape(L + 1, -1)
            manifest.append({
                "name": name, "L": L, "a": a, "client_seed": seed, "leaf": leaf,
                "N0": info["N0"], "b": info["b"], "r": info["r"], "h_q": info["h_q"],
                "w": info["w"], "alpha": info["alpha"],
                "sha256_query_u64": sha(os.path.join(tmp, "query.u64")),
                "sha256_alpha_u64": sha(os.path.join(tmp, "alpha.u64")),
                "sha256_beta_selectors_u64": sha(os.path.join(tmp, "beta.u64")),
                "sha256_levels_u64": [hashlib.sha256(per[i].tobytes()).hexdigest()
                                      for i in range(L + 1)],
            })
            print(f"{name}: ok", flush=True)
    with open(os.path.join(HERE, "golden_tree_c4.json" if c4 else "golden_tree.json"), "w") as f:
        json.dump({"generator": f"oracle/_ref/{os.path.basename(ref_bin)} --mode tree (reference "
                                "sources incl. src/tree_*.cpp + HEXL stand-in), default PirParams "
                                f"scheme{' under CONFIG_N4096_K2_MP' if c4 else ''}",
                   "node_source": "synthetic_tree_node_value (src/tree_select.cpp:44-53)",
                   "cases": manifest}, f, indent=1)
    return 0


def main() -> int:
    if "--tree" in sys.argv[1:]:
        return main_tree(c4="--c4" in sys.argv[1:])
    which = next((k for k in ("c4", "k2mp", "k1p") if "--" + k in sys.argv[1:]), "k1")
    ref_bin, cases_, manifest_name, c4, generator = SETS[which]
    if not os.path.exists(ref_bin):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref"], check=True)
    manifest = []
    for name, target, h, pow2, dbs, cs, idx in cases_:
        with tempfile.TemporaryDirectory() as tmp:
            out = subprocess.run(
                [ref_bin, "--mode", "golden", "--target", str(target), "--height", str(h),
                 "--pow2", str(pow2), "--db-seed", str(dbs), "--client-seed", str(cs),
                 "--index", str(idx), "--out", tmp, "--dump-inputs"]
                + (["--stages", tmp] if c4 else []),
                check=True, capture_output=True, text=True)
            info = json.loads(out.stdout.strip().splitlines()[-1])
            if not info["ok"]:
                raise RuntimeError(f"{name}: reference decryption failed")
            with open(os.path.join(tmp, "response.bin"), "rb") as f:
                stream = f.read()
            with open(os.path.join(HERE, f"{name}.resp.bin"), "wb") as f:
                f.write(stream)
            manifest.append({
                "name": name, "target_num_pt": target, "expansion_height": h,
                "fst_dim_pow2": bool(pow2), "db_seed": dbs, "client_seed": cs,
                "index": idx,
                "num_pt": info["num_pt"], "fst_dim_sz": info["fst_dim_sz"],
                "num_dims": info["num_dims"], "other_dim_sz": info["other_dim_sz"],
                "q": info["q"], "q1": info["q1"], "q2": info["q2"],
                "w1": info["w1"], "w2": info["w2"], "t": info["t"],
                "small_q": info["small_q"], "resp_bytes": info["resp_bytes"],
                "sha256_response_u64": sha(os.path.join(tmp, "response.u64")),
                "sha256_response_stream": hashlib.sha256(stream).hexdigest(),
                "sha256_query_u64": sha(os.path.join(tmp, "query.u64")),
                "sha256_bv_keys_u64": sha(os.path.join(tmp, "bv_keys.u64")),
                "sha256_gsw_key_u64": sha(os.path.join(tmp, "gsw_key.u64")),
            })
            if c4:
                manifest[-1].update({
                    "K": info["K"], "q_limbs": [info["q"], info["q_limb1"]],
                    "base_log2": info["base_log2"], "base_log2_key": info["base_log2_key"],
                    "sha256_stage_expand": sha(os.path.join(tmp, "expand.u64")),
                    "sha256_stage_selectors": sha(os.path.join(tmp, "selectors.u64")),
                    "sha256_stage_first_dim": sha(os.path.join(tmp, "first_dim.u64")),
                    "sha256_stage_other_dim": sha(os.path.join(tmp, "other_dim.u64")),
                })
            print(f"{name}: ok ({info['num_pt']} pts, load {info['load_s']}s)", flush=True)
    with open(os.path.join(HERE, manifest_name), "w") as f:
        json.dump({"generator": generator,
                   "db_coeff": "mix64(db_seed + (pt*N + c + 1) * 0x9E3779B97F4A7C15) % t",
                   "cases": manifest}, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
