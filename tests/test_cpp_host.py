"""The C++ host API (include/geofem.hpp) over the C ABI: built and linked on the
CPU, run on the GPU (tests/cpp/host_api_test.cpp mirrors the reference's own
thermal-profile, 2x2 CG, patch-test and error-behaviour tests)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CPP = os.path.join(ROOT, "tests", "cpp")
BIN = os.path.join(CPP, "host_api_test")


def test_host_api_builds_and_links():
    subprocess.run(["make", "-s", "-C", CPP], check=True)
    out = subprocess.run(["ldd", BIN], capture_output=True, text=True, check=True).stdout
    assert "libgeofem.so" in out and "not found" not in out.split("libgeofem.so")[1].splitlines()[0]


@pytest.mark.gpu
def test_host_api_on_gpu(tmp_path):
    subprocess.run(["make", "-s", "-C", CPP], check=True)
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600, cwd=str(tmp_path))
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "PASSED: 0 failure(s)" in r.stdout
