"""The C++ mirror of FIDESlib's api/fideslib.hpp surface (header-only over the
C ABI): it compiles on CPU, and its example runs end to end on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
API = os.path.join(ROOT, "pyfideslib_b200", "csrc", "api")


def _compile(out):
    cmd = ["g++", "-O2", "-std=c++17", "-I", "/usr/local/cuda/include", os.path.join(API, "example_ckks.cpp"),
           "-o", out, "-L", os.path.join(ROOT, "pyfideslib_b200"), "-lfidesb200",
           "-Wl,-rpath," + os.path.join(ROOT, "pyfideslib_b200")]
    subprocess.run(cmd, check=True)


def test_cpp_api_compiles(tmp_path):
    _compile(str(tmp_path / "ex"))


@pytest.mark.gpu
def test_cpp_api_example_runs(tmp_path):
    exe = str(tmp_path / "ex")
    _compile(exe)
    r = subprocess.run([exe, "13"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "OK" in r.stdout, r.stdout + r.stderr
