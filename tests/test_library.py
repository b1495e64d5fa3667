"""CPU: the C-ABI library loads and exports every symbol the public headers
declare (C-ABI and the unipi::axhel C++ drop-in); host-side planner logic and
the workload parameter helpers.  No GPU calls."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "axhel_b200", "libaxhel.so")


def declared_c_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"^\s*[A-Za-z_][\w \*]*?\b(axhel_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_built():
    assert os.path.exists(LIB), "run python -m axhel_b200.build"


def test_every_declared_c_symbol_is_exported():
    names = declared_c_functions()
    assert len(names) >= 30
    missing = [n for n in names if n not in exported()]
    assert not missing, missing


def test_cpp_dropin_symbols_exported():
    out = subprocess.run(["nm", "-DC", "--defined-only", LIB], capture_output=True, text=True, check=True).stdout
    for sig in ("unipi::axhel::EltwiseAddMod(unsigned long*, unsigned long const*, unsigned long const*",
                "unipi::axhel::EltwiseAddMod(unsigned long*, unsigned long const*, unsigned long,",
                "unipi::axhel::EltwiseSubMod(unsigned long*, unsigned long const*, unsigned long const*",
                "unipi::axhel::EltwiseSubMod(unsigned long*, unsigned long const*, unsigned long,",
                "unipi::axhel::EltwiseMulMod(", "unipi::axhel::EltwiseFMAMod(", "unipi::axhel::EltwiseReduceMod(",
                "unipi::axhel::NTT::NTT(unsigned long, unsigned long, unsigned long)",
                "unipi::axhel::NTT::NTT(unsigned long, unsigned long, unipi::axhel::NTTMultiplyOperand const*",
                "unipi::axhel::NTT::ComputeForward(", "unipi::axhel::NTT::ComputeInverse(",
                "unipi::axhel::NTT::Degree() const", "unipi::axhel::NTT::Modulus() const",
                "unipi::axhel::ComputeForwardRNS(unipi::axhel::NTT const*",
                "unipi::axhel::ComputeInverseRNS(unipi::axhel::NTT const*"):
        assert sig in out, sig


def test_ctypes_load_and_cpu_side_calls():
    from axhel_b200 import capi

    L = capi.lib()
    assert L.axhel_version() >= 100
    assert L.axhel_status_string(4) == b"unsupported configuration"
    # argument checks fail before touching a device
    with pytest.raises(capi.AxhelError) as e:
        capi.NTT(12, 97, 3)
    assert e.value.status == 4
    # n == 0 is a no-op with null pointers (reference loops run zero times)
    capi.add(0, 0, 0, 0, 97)
    capi.mul(0, 0, 0, 0, 97, 1)


def test_default_plans_are_valid():
    from axhel_b200 import capi

    for logn in range(1, 18):
        for inverse in (False, True):
            for count in (1, 24, 768):
                plan = capi.plan_get(inverse, logn, count)
                assert sum(p[0] for p in plan) == logn
                for lg, lr, tg in plan:
                    assert 1 <= lr <= lg and tg >= 1 and (tg & (tg - 1)) == 0
                    assert (tg << (lg - lr)) <= (256 if lr >= 5 else 512)
                if inverse:
                    # a fused chain runs the inverse plan, then the same passes
                    # reversed as its forward: that must be a valid forward plan
                    capi.plan_set(False, logn, list(reversed(plan)))
                    capi.plan_set(False, logn, [])


def test_plan_override_and_table(tmp_path):
    from axhel_b200 import capi

    capi.plan_set(False, 16, [(8, 4, 16), (8, 4, 4)])
    assert capi.plan_get(False, 16, 768) == [(8, 4, 16), (8, 4, 4)]
    with pytest.raises(capi.AxhelError):
        capi.plan_set(False, 16, [(8, 4, 16), (7, 4, 4)])  # stages do not sum to 16
    with pytest.raises(capi.AxhelError):
        capi.plan_set(False, 16, [(8, 3, 64), (8, 4, 4)])  # 64 x 32 threads > 512
    capi.plan_set(False, 16, [])
    t = tmp_path / "plans.txt"
    t.write_text("# inverse logn bucket npass lg lr tg ...\n0 15 3 2 8 4 8 7 4 16\n0 15 3 2 8 4 8 9 4 1\n")
    assert capi.plan_load(str(t)) == 1  # the second line does not sum to 15
    assert capi.plan_get(False, 15, 8) == [(8, 4, 8), (7, 4, 16)]


def test_cluster_plan_override():
    """The single-launch cluster form's configuration: built-in choices are
    valid, invalid ones are refused, and an override can be cleared."""
    from axhel_b200 import capi

    for kind in (capi.CLUSTER_FORWARD, capi.CLUSTER_INVERSE, capi.CLUSTER_CHAIN, capi.CLUSTER_PRODUCT):
        for logn in range(10, 18):
            lga, lr, cs, m = capi.cluster_plan_get(kind, logn)
            if kind >= capi.CLUSTER_CHAIN and logn > 15:
                assert (lga, m) == (0, 0)  # no fused cluster kernel compiled for 2^16, 2^17
                continue
            assert lga >= 5 and cs in (2, 4, 8, 16)
            capi.cluster_plan_set(kind, logn, lga, lr, cs, max(m, 1))  # valid as it stands
            capi.cluster_plan_set(kind, logn)
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(4, 12, 6, 2, 8, 1)  # no such kind
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(capi.CLUSTER_CHAIN, 12, 6, 3, 8, 1)  # fused kernels are radix-4 only
    default = capi.cluster_plan_get(False, 12)
    capi.cluster_plan_set(False, 12, 6, 2, 16, 5)
    assert capi.cluster_plan_get(False, 12) == (6, 2, 16, 5)
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(False, 12, 6, 4, 8, 1)  # not compiled
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(False, 12, 6, 3, 32, 1)  # more than 16 CTAs
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(False, 16, 8, 4, 4, 1)  # 1024 threads per CTA
    with pytest.raises(capi.AxhelError):
        capi.cluster_plan_set(False, 9, 5, 2, 4, 1)  # degree out of range
    capi.cluster_plan_set(False, 12, 6, 3, 8, 0)  # off
    assert capi.cluster_plan_get(False, 12)[3] == 0
    capi.cluster_plan_set(False, 12)
    assert capi.cluster_plan_get(False, 12) == default


def test_params_primes_match_reference_generator(oracle):
    from axhel_b200 import params

    for n in (1024, 1 << 16):
        for bits in (30, 50, 59, 62):
            for num, den in ((1, 4), (1, 2), (3, 4)):
                assert params.ntt_prime_near(n, bits, num, den) == oracle.find_ntt_prime_near(n, bits, num, den)
            q = params.ntt_prime_near(n, bits, 1, 2)
            assert params.primitive_root(n, q) == oracle.find_primitive_root(n, q)
    import random

    r = random.Random(5)
    for _ in range(2000):
        x = r.getrandbits(62) | 1
        assert params.is_prime(x) == bool(oracle.is_prime(x))
    mods = params.rns_moduli(1 << 16, 24, 50, 59)
    assert len({q for q, _ in mods}) == 24
    assert all((q - 1) % (1 << 17) == 0 and 50 <= q.bit_length() <= 59 for q, _ in mods)


def test_batch_split_table_and_override(tmp_path):
    from axhel_b200 import capi

    t = tmp_path / "plans.txt"
    t.write_text("B 15 7\nB 16 4\nB 12 9\n")  # the last two are outside the valid ranges
    assert capi.plan_load(str(t)) == 1
    assert capi.batch_split_get(15) == 7
    capi.batch_split_set(15, 6)
    assert capi.batch_split_get(15) == 6
    capi.batch_split_set(15, 0)  # back to the table
    assert capi.batch_split_get(15) == 7
    for logn, row in ((16, 4), (16, 12), (12, 8), (9, 5), (18, 9)):
        with pytest.raises(capi.AxhelError):
            capi.batch_split_set(logn, row)


def test_debug_log_build_compiles(tmp_path):
    """The AXHEL_DEBUG build of the drop-in (AXHEL_LOG lines on every call,
    axhel/util/debug.hpp) compiles; the default build compiles them out."""
    cuda_inc = "/usr/local/cuda/include"
    if not os.path.exists(os.path.join(cuda_inc, "cuda_runtime.h")):
        pytest.skip("CUDA headers not found")
    src = os.path.join(ROOT, "axhel_b200", "csrc", "dropin.cpp")
    for defs in (["-DAXHEL_DEBUG"], []):
        subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", *defs,
                        "-I" + os.path.join(ROOT, "include"), "-I" + cuda_inc, src], check=True)
    probe = tmp_path / "log.cpp"
    probe.write_text('#include <axhel/util/debug.hpp>\n#include <sstream>\n'
                     'int main() { AXHEL_LOG("x=" << 1); return 0; }\n')
    exe = tmp_path / "log"
    subprocess.run(["g++", "-std=c++17", "-DAXHEL_DEBUG", "-I" + os.path.join(ROOT, "include"), str(probe), "-o",
                    str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, check=True)
    assert r.stderr == "[AXHEL] x=1\n"


def test_cluster_table_lines(tmp_path):
    """`K` lines of a plan table set the cluster form per kind and degree
    (between an override and the built-in choice); invalid ones are skipped.
    Run in a fresh process: a loaded table stays for the process."""
    import sys

    t = tmp_path / "plans.txt"
    t.write_text("K 0 12 6 3 8 5\nK 2 13 7 2 16 3\nK 1 12 6 4 8 1\nK 3 16 8 2 16 2\nK 1 14 7 2 16 0\n")
    code = f"""
from axhel_b200 import capi
assert capi.plan_load({str(t)!r}) == 3, "two lines are invalid"
assert capi.cluster_plan_get(0, 12) == (6, 3, 8, 5)
assert capi.cluster_plan_get(2, 13) == (7, 2, 16, 3)
assert capi.cluster_plan_get(1, 14)[3] == 0          # turned off by the table
assert capi.cluster_plan_get(1, 12) != (6, 4, 8, 1)  # not compiled: built-in kept
capi.cluster_plan_set(0, 12, 6, 2, 8, 9)             # an override wins over the table
assert capi.cluster_plan_get(0, 12) == (6, 2, 8, 9)
capi.cluster_plan_set(0, 12)                         # cleared: back to the table
assert capi.cluster_plan_get(0, 12) == (6, 3, 8, 5)
print("ok")
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=120)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]
