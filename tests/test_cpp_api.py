"""The C++ host API (include/vsdmo/DMO.hpp) compiles against the C ABI (CPU) and runs the
reference-style build -> optimize -> query sequence on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cpp_api.cpp")


def _compile(vsdmo, tmp_path):
    from volumesurfacediscretemeshoptimization_b200 import build
    exe = str(tmp_path / "test_cpp_api")
    libdir = os.path.dirname(build.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", libdir, "-lvsdmo", "-Wl,-rpath," + libdir], check=True)
    return exe


def test_cpp_api_compiles(vsdmo, tmp_path):
    assert os.path.exists(_compile(vsdmo, tmp_path))


@pytest.mark.gpu
def test_cpp_api_runs(vsdmo, tmp_path):
    exe = _compile(vsdmo, tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "cpp api ok" in out.stdout
