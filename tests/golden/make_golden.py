"""Generates the golden fixtures in this directory by running the REFERENCE
native backend (oracle/_ref/libaxhel_ref.so, compiled from the reference
sources by oracle/Makefile) on seeded inputs.

    make -C oracle && python tests/golden/make_golden.py

Inputs come from the reference test suite's generator (mt19937_64 seeded with
test_seed() ^ case, rejection-sampled bounded draws; restated in
oracle/axhel_oracle.c), so they can be regenerated on a machine without the
reference.  Outputs:
  ntt_small.npz    forward (in 4q, out 4 and 1) and inverse (in 2q, out 2 and 1)
                   vectors for N <= 1024 over several modulus widths
  eltwise.npz      Mul/FMA/Reduce/Add/Sub vectors for several widths and factors
  ntt_hashes.json  SHA-256 of forward-lazy / inverse-lazy outputs at N = 2^12..2^17
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from pyoracle import Oracle, Reference  # noqa: E402

SEED = 0x415848454C


def case_seed(*parts):
    s = SEED
    for p in parts:
        s = (s * 1000003 ^ int(p)) & 0xFFFFFFFFFFFFFFFF
    return s


def main():
    o, r = Oracle(), Reference()
    small = {}
    for n in (8, 16, 64, 256, 1024):
        for bits in (20, 30, 40, 50, 59, 62):
            q = o.find_ntt_prime(n, bits)
            psi = o.find_primitive_root(n, q)
            h = r.ntt(n, q, psi)
            st = o.rng(case_seed(n, bits))
            x = o.random_vector(st, n, 4 * q)
            y = o.random_vector(st, n, 2 * q)
            key = f"n{n}_b{bits}"
            small[key + "_q"] = np.array([q, psi], np.uint64)
            small[key + "_x"] = x
            small[key + "_y"] = y
            small[key + "_fwd4"] = h.forward(x, 4, 4)
            small[key + "_fwd1"] = h.forward(x, 4, 1)
            small[key + "_inv2"] = h.inverse(y, 2, 2)
            small[key + "_inv1"] = h.inverse(y, 2, 1)
    np.savez_compressed(os.path.join(HERE, "ntt_small.npz"), **small)

    elt = {}
    n = 129
    for bits in (20, 31, 45, 50, 55, 60, 62):
        q = o.find_ntt_prime(1024, bits)
        st = o.rng(case_seed(7, bits))
        key = f"b{bits}"
        elt[key + "_q"] = np.array([q], np.uint64)
        a1 = o.random_vector(st, n, q)
        b1 = o.random_vector(st, n, q)
        elt[key + "_a1"], elt[key + "_b1"] = a1, b1
        elt[key + "_add"] = r.add(a1, b1, q)
        elt[key + "_sub"] = r.sub(a1, b1, q)
        s1 = o.bounded(st, q)
        elt[key + "_s1"] = np.array([s1], np.uint64)
        elt[key + "_adds"] = r.add(a1, s1, q)
        elt[key + "_subs"] = r.sub(a1, s1, q)
        for f in (1, 2, 4, 8):
            bound = min(f * q, 2 ** 64 - 1)
            a = o.random_vector(st, n, bound)
            b = o.random_vector(st, n, bound)
            s = o.bounded(st, bound)
            elt[f"{key}_f{f}_a"], elt[f"{key}_f{f}_b"] = a, b
            elt[f"{key}_f{f}_s"] = np.array([s], np.uint64)
            if f != 8:
                elt[f"{key}_f{f}_mul"] = r.mul(a, b, q, f)
            elt[f"{key}_f{f}_fma"] = r.fma(a, s, b, q, f)
            elt[f"{key}_f{f}_fma0"] = r.fma(a, s, None, q, f)
        for (i, j) in ((2, 1), (4, 1), (4, 2)):
            a = o.random_vector(st, n, i * q)
            elt[f"{key}_r{i}{j}_a"] = a
            elt[f"{key}_r{i}{j}"] = r.reduce(a, q, i, j)
        a = o.random_vector(st, n, 2 ** 64 - 1)
        elt[f"{key}_rq_a"] = a
        elt[f"{key}_rq"] = r.reduce(a, q, q, 1)
    np.savez_compressed(os.path.join(HERE, "eltwise.npz"), **elt)

    hashes = []
    for logn in range(12, 18):
        n = 1 << logn
        for bits in (50, 59, 62):
            q = o.find_ntt_prime(n, bits)
            psi = o.find_primitive_root(n, q)
            h = r.ntt(n, q, psi)
            st = o.rng(case_seed(n, bits, 99))
            x = o.random_vector(st, n, 4 * q)
            y = o.random_vector(st, n, 2 * q)
            hashes.append({
                "n": n, "bits": bits, "q": q, "psi": psi, "seed": case_seed(n, bits, 99),
                "fwd4_sha256": hashlib.sha256(h.forward(x, 4, 4).tobytes()).hexdigest(),
                "inv2_sha256": hashlib.sha256(h.inverse(y, 2, 2).tobytes()).hexdigest(),
            })
    with open(os.path.join(HERE, "ntt_hashes.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py (reference native backend, oracle/_ref)",
                   "inputs": "x = random_vector(mt19937_64(seed), n, 4q); y = random_vector(same stream, n, 2q)",
                   "cases": hashes}, f, indent=1)
    print("golden fixtures written")


if __name__ == "__main__":
    main()
