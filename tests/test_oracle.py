"""CPU: pins the oracle restatement to the reference — its known-answer
vectors, the example's explicit tables, the committed golden fixtures (made by
running the reference), and, when built, the reference native backend itself
on fresh seeded inputs."""
import hashlib
import json
import os

import numpy as np
import pytest

from helpers import MODULUS_BITS, SEED, barrett_cases

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_known_vector_n8_q17(oracle):
    """tests/public/test_ntt.cpp:32-46"""
    fwd, inv, ninv = oracle.tables(8, 17, 3)
    x = np.arange(1, 9, dtype=np.uint64)
    y = oracle.forward(x, 17, fwd, 1, 1)
    assert y.tolist() == [5, 0, 13, 8, 9, 11, 5, 8]
    assert oracle.inverse(y, 17, inv, ninv, 1, 1).tolist() == list(range(1, 9))


def test_tables_match_example_n8(oracle):
    """example/example.cpp:314-345"""
    fwd, inv, ninv = oracle.tables(8, 17, 3)
    assert fwd.tolist() == [[1, 1085102592571150095], [13, 14106333703424951235], [9, 9765923333140350855],
                            [15, 16276538888567251425], [3, 3255307777713450285], [5, 5425512962855750475],
                            [10, 10851025925711500950], [11, 11936128518282651045]]
    assert inv.tolist() == [[0, 0], [6, 6510615555426900570], [7, 7595718147998050665], [12, 13021231110853801140],
                            [14, 15191436295996101330], [2, 2170205185142300190], [8, 8680820740569200760],
                            [4, 4340410370284600380]]
    assert ninv.tolist() == [15, 16276538888567251425]


def test_root_sanity(oracle):
    """test_ntt.cpp:48-57"""
    for n in (8, 1024, 32768, 131072):
        for bits in MODULUS_BITS:
            q = oracle.find_ntt_prime(n, bits)
            if q == 0:
                continue
            psi = oracle.find_primitive_root(n, q)
            assert oracle.pow_mod(psi, n, q) == q - 1 and oracle.pow_mod(psi, 2 * n, q) == 1


def test_mt19937_64_known_answer(oracle):
    """The 10000th output of mt19937_64 default-seeded (5489) is
    9981545732273789042 (C++ standard, [rand.predef])."""
    st = oracle.rng(5489)
    for _ in range(9999):
        oracle.next_u64(st)
    assert oracle.next_u64(st) == 9981545732273789042


def test_golden_ntt_small(oracle):
    g = np.load(os.path.join(GOLD, "ntt_small.npz"))
    keys = sorted({k.rsplit("_", 1)[0] for k in g.files})
    assert len(keys) == 30
    for key in keys:
        n = int(key.split("_")[0][1:])
        q, psi = (int(v) for v in g[key + "_q"])
        fwd, inv, ninv = oracle.tables(n, q, psi)
        x, y = g[key + "_x"], g[key + "_y"]
        np.testing.assert_array_equal(oracle.forward(x, q, fwd, 4, 4), g[key + "_fwd4"], err_msg=key)
        np.testing.assert_array_equal(oracle.forward(x, q, fwd, 4, 1), g[key + "_fwd1"], err_msg=key)
        np.testing.assert_array_equal(oracle.inverse(y, q, inv, ninv, 2, 2), g[key + "_inv2"], err_msg=key)
        np.testing.assert_array_equal(oracle.inverse(y, q, inv, ninv, 2, 1), g[key + "_inv1"], err_msg=key)


def test_golden_eltwise(oracle):
    g = np.load(os.path.join(GOLD, "eltwise.npz"))
    for bits in (20, 31, 45, 50, 55, 60, 62):
        k = f"b{bits}"
        q = int(g[k + "_q"][0])
        a1, b1, s1 = g[k + "_a1"], g[k + "_b1"], int(g[k + "_s1"][0])
        np.testing.assert_array_equal(oracle.add(a1, b1, q), g[k + "_add"])
        np.testing.assert_array_equal(oracle.sub(a1, b1, q), g[k + "_sub"])
        np.testing.assert_array_equal(oracle.add(a1, s1, q), g[k + "_adds"])
        np.testing.assert_array_equal(oracle.sub(a1, s1, q), g[k + "_subs"])
        for f in (1, 2, 4, 8):
            a, b, s = g[f"{k}_f{f}_a"], g[f"{k}_f{f}_b"], int(g[f"{k}_f{f}_s"][0])
            if f != 8:
                np.testing.assert_array_equal(oracle.mul(a, b, q, f), g[f"{k}_f{f}_mul"])
            np.testing.assert_array_equal(oracle.fma(a, s, b, q, f), g[f"{k}_f{f}_fma"])
            np.testing.assert_array_equal(oracle.fma(a, s, None, q, f), g[f"{k}_f{f}_fma0"])
        for i, j in ((2, 1), (4, 1), (4, 2)):
            np.testing.assert_array_equal(oracle.reduce(g[f"{k}_r{i}{j}_a"], q, i, j), g[f"{k}_r{i}{j}"])
        np.testing.assert_array_equal(oracle.reduce(g[f"{k}_rq_a"], q, q, 1), g[f"{k}_rq"])


def test_golden_hashes_large(oracle):
    """Full-size (2^12..2^17) lazy outputs of the reference, by SHA-256."""
    with open(os.path.join(GOLD, "ntt_hashes.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        n, q, psi = c["n"], c["q"], c["psi"]
        fwd, inv, ninv = oracle.tables(n, q, psi)
        st = oracle.rng(c["seed"])
        x = oracle.random_vector(st, n, 4 * q)
        y = oracle.random_vector(st, n, 2 * q)
        assert hashlib.sha256(oracle.forward(x, q, fwd, 4, 4).tobytes()).hexdigest() == c["fwd4_sha256"]
        assert hashlib.sha256(oracle.inverse(y, q, inv, ninv, 2, 2).tobytes()).hexdigest() == c["inv2_sha256"]


def test_oracle_matches_reference_live(oracle, reference):
    """Fresh seeded inputs through both the restatement and the reference."""
    st = oracle.rng(SEED ^ 0x11)
    for n in (2, 4, 32, 2048, 8192):
        for bits in (21, 37, 50, 61, 62):
            q = oracle.find_ntt_prime(n, bits)
            if q == 0:
                continue
            psi = oracle.find_primitive_root(n, q)
            for a, b in zip(oracle.tables(n, q, psi), reference.tables(n, q, psi)):
                np.testing.assert_array_equal(a, b)
            h = reference.ntt(n, q, psi)
            fwd, inv, ninv = oracle.tables(n, q, psi)
            x = oracle.random_vector(st, n, 4 * q)
            for of in (1, 2, 4):
                np.testing.assert_array_equal(oracle.forward(x, q, fwd, 4, of), h.forward(x, 4, of))
            y = oracle.random_vector(st, n, 2 * q)
            for of in (1, 2):
                np.testing.assert_array_equal(oracle.inverse(y, q, inv, ninv, 2, of), h.inverse(y, 2, of))
    for bits, q, _ in barrett_cases(oracle):
        n = 300
        for f in (1, 2, 4, 8):
            bound = min(f * q, 2 ** 64 - 1)
            a, b = oracle.random_vector(st, n, bound), oracle.random_vector(st, n, bound)
            s = oracle.bounded(st, bound)
            if f != 8:
                np.testing.assert_array_equal(oracle.mul(a, b, q, f), reference.mul(a, b, q, f))
            np.testing.assert_array_equal(oracle.fma(a, s, b, q, f), reference.fma(a, s, b, q, f))
        a = oracle.random_vector(st, n, 2 ** 64 - 1)
        np.testing.assert_array_equal(oracle.reduce(a, q, q, 1), reference.reduce(a, q, q, 1))
        for i, j in ((1, 1), (1, 2), (2, 2), (2, 1), (4, 1), (4, 2), (4, 4), (8, 1), (0, 2)):
            a = oracle.random_vector(st, n, q * max(i, 1))
            e1 = oracle.reduce(a, q, i, j, out=np.full(n, 3, np.uint64))
            e2 = reference.reduce(a, q, i, j, out=np.full(n, 3, np.uint64))
            np.testing.assert_array_equal(e1, e2)


def test_polymul_against_quadratic_oracle(oracle):
    """test_polymul.cpp:236-292 on the oracle: NTT, MulMod, INTT = negacyclic product."""
    st = oracle.rng(SEED ^ 0x504F4C594D554C)
    for n in (8, 16, 32, 64):
        for bits in (30, 40, 50, 60, 62):
            q = oracle.find_ntt_prime(n, bits)
            psi = oracle.find_primitive_root(n, q)
            fwd, inv, ninv = oracle.tables(n, q, psi)
            a = oracle.random_vector(st, n, q)
            b = oracle.random_vector(st, n, q)
            A, B = oracle.forward(a, q, fwd), oracle.forward(b, q, fwd)
            got = oracle.inverse(oracle.mul(A, B, q, 1), q, inv, ninv)
            exp = [0] * n
            for i in range(n):
                for j in range(n):
                    p = int(a[i]) * int(b[j]) % q
                    k = i + j
                    if k < n:
                        exp[k] = (exp[k] + p) % q
                    else:
                        exp[k - n] = (exp[k - n] - p) % q
            assert got.tolist() == exp
