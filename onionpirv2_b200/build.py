"""Builds libonionpir_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m onionpirv2_b200.build          # incremental
    python -m onionpirv2_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libonionpir_b200.so")
SOURCES = ["opir_kernels.cu", "opir_server.cu", "opir_params.cpp", "opir_noalloc.cu",
           "opir_scan_tc.cu", "opir_c4_kernels.cu", "opir_c4_server.cu", "opir_c4_scan_tc.cu", "opir_k1p_kernels.cu", "opir_tree.cpp",
           "opir_shard.cpp", "opir_codec.cpp", "opir_codec_abi.cpp", "opir_client.cu"]
HEADERS = ["opir_device.cuh", "opir_kernels.h", "opir_params.h", "opir_scan_tc.h", "opir_ntt.cuh",
           "opir_host.h", "opir_c4_device.cuh", "opir_c4_kernels.h", "opir_c4_server.h", "opir_k1p_kernels.h", "opir_tc.cuh", "opir_tree.h",
           "opir_shard.h", "opir_codec.h", "opir_client.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3",
                     "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [
        os.path.join(os.path.dirname(PKG), "include", "onionpir_b200.h")]
    newest_dep = max(_mtime(d) for d in deps)
    objs, cmds = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _mtime(o) < max(_mtime(s), newest_dep):
            cmds.append([nvcc()] + NVCC_FLAGS + ["-c", s, "-o", o])

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(compile_one, c) for c in cmds]:
            f.result()
    if force or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
