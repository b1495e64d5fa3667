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


# Host operands take three routes: small ones are read and written by the
# kernels in the mapped pinned buffers (by default up to 512 KiB for
# element-wise calls, 256 / 128 KiB for the inverse / forward transform), larger
# ones go by DMA through the pinned buffers, or, with pinned staging off,
# straight from the pageable memory.
STAGING = {
    "default": {},
    "pinned-dma": {"AXHEL_ZERO_COPY_MAX": "0"},
    "all-zero-copy": {"AXHEL_ZERO_COPY_MAX": str(1 << 30)},
    "pageable-staging": {"AXHEL_PINNED_STAGING_MAX": "0"},
}


@pytest.mark.parametrize("staging", list(STAGING))
def test_cpp_dropin(tmp_path, cuda, staging):
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
    env.update(STAGING[staging])
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-4000:]
    assert "all checks passed" in r.stdout
