"""Loader for the reference-generated golden fixtures in tests/golden/."""
import hashlib
import json
import os

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)["cases"]


def case(name):
    for c in cases():
        if c["name"] == name:
            return c
    raise KeyError(name)


def cases_c4():
    """CONFIG_N4096_K2_MP cases (reference built with that configuration)."""
    with open(os.path.join(GOLDEN_DIR, "golden_c4.json")) as f:
        return json.load(f)["cases"]


def case_c4(name):
    for c in cases_c4():
        if c["name"] == name:
            return c
    raise KeyError(name)


def cases_set(which):
    """The cases of another parameter set: "k2mp" (CONFIG_N2048_K2_MP) or
    "k1p" (CONFIG_N2048_K1), each made by the reference built with it."""
    with open(os.path.join(GOLDEN_DIR, f"golden_{which}.json")) as f:
        return json.load(f)["cases"]


def case_set(which, name):
    for c in cases_set(which):
        if c["name"] == name:
            return c
    raise KeyError(name)


def cases_tree():
    """Tree PIR select_level cases (reference tree layer, default scheme)."""
    with open(os.path.join(GOLDEN_DIR, "golden_tree.json")) as f:
        return json.load(f)["cases"]


def cases_tree_c4():
    """Tree PIR select_level cases under CONFIG_N4096_K2_MP (reference tree
    layer built with that configuration, default scheme)."""
    with open(os.path.join(GOLDEN_DIR, "golden_tree_c4.json")) as f:
        return json.load(f)["cases"]


def stream(c):
    with open(os.path.join(GOLDEN_DIR, c["name"] + ".resp.bin"), "rb") as f:
        return f.read()


def sha256(arr) -> str:
    if getattr(arr, "size", 1) == 0:   # memoryview cannot cast empty shapes
        return hashlib.sha256(b"").hexdigest()
    return hashlib.sha256(memoryview(arr).cast("B")).hexdigest()
