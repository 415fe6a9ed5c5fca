"""The C++ facade (include/onionpir_b200.hpp): it compiles self-contained
with warnings as errors, and its parity programs (tests/cpp/
test_server_facade.cpp and test_client_facade.cpp, written like the
reference's test_pir.cpp) build against the library and the oracle on CPU and
pass on a GPU."""
import os
import shutil
import subprocess

import pytest

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "onionpirv2_b200")
ORACLE = os.path.join(ROOT, "oracle")
CXX = shutil.which("g++")

pytestmark = pytest.mark.skipif(CXX is None, reason="no C++ compiler")


def build(tmp_path, name: str = "test_server_facade") -> str:
    O.build()
    exe = str(tmp_path / name)
    subprocess.run([CXX, "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-I", ORACLE,
                    os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                    "-L", PKG, "-lonionpir_b200", "-L", ORACLE, "-lopir_oracle",
                    f"-Wl,-rpath,{PKG}:{ORACLE}", "-o", exe], check=True)
    return exe


def test_header_is_self_contained(tmp_path):
    src = tmp_path / "only_header.cpp"
    src.write_text('#include "onionpir_b200.hpp"\n'
                   'int main() { onionpir_b200::RlweCt ct; ct.resize(4); return ct.poly_size() == 4 ? 0 : 1; }\n')
    subprocess.run([CXX, "-std=c++17", "-Wall", "-Wextra", "-Wpedantic", "-Werror",
                    "-I", os.path.join(ROOT, "include"), "-c", str(src),
                    "-o", str(tmp_path / "only_header.o")], check=True)


def test_parity_program_builds(tmp_path):
    assert os.path.exists(build(tmp_path))


@pytest.mark.gpu
def test_parity_program_passes(tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    assert r.stdout.strip().endswith("ok")


def test_client_parity_program_builds(tmp_path):
    assert os.path.exists(build(tmp_path, "test_client_facade"))


@pytest.mark.gpu
def test_client_parity_program_passes(tmp_path):
    exe = build(tmp_path, "test_client_facade")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-4000:]
    assert r.stdout.strip().endswith("ok")
