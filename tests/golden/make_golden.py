"""Regenerates the golden fixtures in this folder from the reference itself.

Runs oracle/_ref/opir_ref (the unmodified OnionPIRv2 reference sources, built
by `make -C oracle ref` against the HEXL stand-in) on seeded inputs and stores,
per case: the layout, seeds and index, the serialized 22-bit response stream
(<name>.resp.bin, as written by PirServer::save_resp_to_stream), and SHA-256
digests of the response u64 array and of the client material (query, BV keys,
RGSW key) so a seeded client can be checked against the reference client
without committing megabytes of keys.

Only needed when the fixtures must change; tests never run it.
    python tests/golden/make_golden.py
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


def sha(path: str) -> str:
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def main() -> int:
    if not os.path.exists(REF_BIN):
        subprocess.run(["make", "-C", os.path.join(REPO, "oracle"), "ref"], check=True)
    manifest = []
    for name, target, h, pow2, dbs, cs, idx in CASES:
        with tempfile.TemporaryDirectory() as tmp:
            out = subprocess.run(
                [REF_BIN, "--mode", "golden", "--target", str(target), "--height", str(h),
                 "--pow2", str(pow2), "--db-seed", str(dbs), "--client-seed", str(cs),
                 "--index", str(idx), "--out", tmp, "--dump-inputs"],
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
            print(f"{name}: ok ({info['num_pt']} pts, load {info['load_s']}s)", flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/opir_ref (reference sources + HEXL stand-in)",
                   "db_coeff": "mix64(db_seed + (pt*N + c + 1) * 0x9E3779B97F4A7C15) % t",
                   "cases": manifest}, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
