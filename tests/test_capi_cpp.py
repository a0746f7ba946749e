"""The C ABI from a compiled C++ client (tests/cpp/capi_client.cpp): it builds
against include/tn_cuda.h and links libtn_cuda.so on the CPU; on a GPU it
reproduces the reference's golden energy (test_Unittest1.py:22)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "tensornetworks_b200", "lib")
EXE = os.path.join(ROOT, "_build", "capi_client")


def _build():
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    os.makedirs(os.path.dirname(EXE), exist_ok=True)
    cmd = [cxx, "-O2", "-std=c++17", os.path.join(ROOT, "tests", "cpp", "capi_client.cpp"),
           "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + LIB, "-ltn_cuda",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIB, "-Wl,-rpath,/usr/local/cuda/lib64", "-o", EXE]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_client_builds():
    _build()
    assert os.path.exists(EXE)


@pytest.mark.gpu
def test_cpp_client_runs():
    _build()
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "golden" in r.stdout
