"""Builds tests/cpp/test_dropin.cpp against the drop-in headers
(include/axhel/*.hpp) and libaxhel.so with g++, the way a C++ caller such as
SEAL links it, and runs it on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu


def cuda_include():
    for c in ("/usr/local/cuda/include", os.path.join(os.environ.get("CUDA_HOME", ""), "include")):
        if os.path.exists(os.path.join(c, "cuda_runtime.h")):
            return c
    pytest.skip("CUDA headers not found")


@pytest.mark.parametrize("pinned_max", [None, "0"], ids=["pinned-staging", "pageable-staging"])
def test_cpp_dropin(tmp_path, cuda, pinned_max):
    exe = tmp_path / "test_dropin"
    lib_dir = os.path.join(ROOT, "axhel_b200")
    orc = tmp_path / "axhel_oracle.o"
    subprocess.run(["gcc", "-O2", "-c", os.path.join(ROOT, "oracle", "axhel_oracle.c"), "-o", str(orc)], check=True)
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I" + cuda_include(),
           os.path.join(ROOT, "tests", "cpp", "test_dropin.cpp"), str(orc), "-L" + lib_dir, "-laxhel",
           "-Wl,-rpath," + lib_dir, "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath,/usr/local/cuda/lib64",
           "-lpthread", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    env = dict(os.environ)
    if pinned_max is not None:  # host operands handed to cudaMemcpyAsync as they are
        env["AXHEL_PINNED_STAGING_MAX"] = pinned_max
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "all checks passed" in r.stdout
