"""Build recipe for the in-tree CUDA library ``axhel_b200/libaxhel.so``.

Compiles every source under ``axhel_b200/csrc`` for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``), in parallel, and links one
shared library exporting the C-ABI (``include/axhel_cuda.h``) and the C++
drop-in (``include/axhel/*.hpp``).  nvcc cross-compiles without a GPU.

    python -m axhel_b200.build           # build if sources changed
    python -m axhel_b200.build --force   # rebuild everything
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libaxhel.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                     "-I" + os.path.join(ROOT, "include")]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home():
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc())))


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(ROOT, "include")
    for dp, _, fs in os.walk(inc):
        hs += [os.path.join(dp, f) for f in fs]
    return hs


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _compile(src, verbose_ptxas=False):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if src.endswith(".cu"):
        cmd = [nvcc(), *NVCC_FLAGS, "-c", src, "-o", obj]
        if verbose_ptxas:
            cmd.insert(1, "-Xptxas=-v")
    else:
        cmd = ["g++", *CXX_FLAGS, "-I" + os.path.join(cuda_home(), "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


TOOLS = os.path.join(PKG, "tools")


def build_tools(force=False):
    """The measuring programs of ``axhel_b200/tools`` (C++ callers of the
    public API), linked against libaxhel.so next to them."""
    for f in sorted(os.listdir(TOOLS)):
        if not f.endswith(".cpp"):
            continue
        src = os.path.join(TOOLS, f)
        exe = os.path.join(PKG, f[:-4])
        if not force and os.path.exists(exe) and os.path.getmtime(exe) >= _newest([src, LIB] + headers()):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-DAXHEL_RNS", "-I" + os.path.join(ROOT, "include"), src, "-L" + PKG,
               "-laxhel", "-Wl,-rpath,$ORIGIN", "-lpthread", "-o", exe]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"tool build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force=False, verbose_ptxas=False, quiet=False):
    """Compile and link libaxhel.so (and the tools); returns its path."""
    lib = _build_lib(force, verbose_ptxas, quiet)
    build_tools(force)
    return lib


def _build_lib(force=False, verbose_ptxas=False, quiet=False):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _newest(srcs + headers() + [__file__]):
        return LIB
    jobs = min(len(srcs), os.cpu_count() or 4)
    logs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        futs = [ex.submit(_compile, s, verbose_ptxas) for s in srcs]
        objs = []
        for f in futs:
            o, log = f.result()
            objs.append(o)
            if log:
                logs.append(log)
    cmd = [nvcc(), *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(LIB + ".tmp", LIB)
    if verbose_ptxas and not quiet:
        sys.stderr.write("".join(logs))
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print registers / spills per kernel")
    ap.add_argument("--debug-log", action="store_true",
                    help="define AXHEL_DEBUG: every drop-in call logs its dispatch to stderr (AXHEL_LOG)")
    a = ap.parse_args()
    if a.debug_log:
        NVCC_FLAGS.append("-DAXHEL_DEBUG")
        CXX_FLAGS.append("-DAXHEL_DEBUG")
    print(build(force=a.force or a.ptxas_v or a.debug_log, verbose_ptxas=a.ptxas_v))


if __name__ == "__main__":
    main()
