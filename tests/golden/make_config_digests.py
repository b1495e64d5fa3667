"""Writes config_digests.json: SHA-256 of every output of the benchmark
configurations at their full sizes, computed on the CPU.

    make -C oracle && python tests/golden/make_config_digests.py

* headline batch: 768 limbs of N = 2^16 (24 primes of 50-59 bits):
  ComputeForward(1,4) on every limb, then ReduceMod(4,2) -> ComputeInverse(2,1);
* tensor product: 64 pairs x 16 limbs of N = 2^15, the five-call sequence
  then ReduceMod(4,1) per result;
* uneven batch: each of the 512 jobs (N 2^12..2^17, 1..48 limbs, forward,
  inverse and INTT -> MulMod -> NTT).

Outputs come from the oracle's multi-threaded per-limb call sequences
(tests/configs_oracle.py) and are checked here, call by call, against the
reference native backend compiled from its sources (oracle/_ref) before they
are written; the script refuses to write if the two differ anywhere.  Inputs
are regenerated from their seeds by bench.py / axhel_b200/workloads.py, and
their own SHA-256 is stored too, so that a mismatch on another machine can be
told apart from a changed input generator.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    sys.path.insert(0, p)

from pyoracle import Oracle, Reference  # noqa: E402

import configs_oracle as co  # noqa: E402


def check(ok, what):
    if not ok:
        raise SystemExit(f"oracle and reference differ: {what}")


def headline(o, r):
    import bench

    mods, data = co.headline_case()
    fwd, back = co.headline_oracle(o, mods, data)
    refs = [r.ntt(bench.N, q, psi) for q, psi in mods]
    F = fwd.reshape(bench.COUNT, bench.N)
    B = back.reshape(bench.COUNT, bench.N)
    for i in range(bench.COUNT):
        h, q = refs[i % len(mods)], mods[i % len(mods)][0]
        f = h.forward(data[i], 1, 4)
        check(np.array_equal(f, F[i]), f"headline forward limb {i}")
        b = h.inverse(r.reduce(f, q, 4, 2), 2, 1)
        check(np.array_equal(b, B[i]), f"headline inverse limb {i}")
    check(np.array_equal(back, data.reshape(-1)), "headline round trip")
    return {"limbs": bench.COUNT, "degree": bench.N, "seed": bench.SEED,
            "input_sha256": co.digest(data), "forward_lazy_sha256": co.digest(fwd),
            "round_trip_sha256": co.digest(back)}


def tensor(o, r):
    from axhel_b200 import workloads

    n, qs, count, ins, outs = co.tensor_oracle(o)
    c0, c1, d0, d1 = ins
    R = [x.reshape(count, n) for x in outs]
    for i in range(count):
        q = qs[i % len(qs)]
        t0 = r.mul(c0[i], d0[i], q, 1)
        t1 = r.mul(c0[i], d1[i], q, 1)
        t1 = r.add(t1, r.mul(c1[i], d0[i], q, 1), q)
        t2 = r.mul(c1[i], d1[i], q, 1)
        for k, t in enumerate((t0, t1, t2)):
            check(np.array_equal(r.reduce(t, q, 4, 1), R[k][i]), f"tensor r{k} limb {i}")
    return {"shape": workloads.TENSOR_SHAPE, "moduli": [int(q) for q in qs],
            "input_sha256": [co.digest(a) for a in ins], "r_sha256": [co.digest(x) for x in outs]}


def uneven(o, r):
    from axhel_b200 import workloads

    jobs = co.uneven_case()
    tabs = co.Tables(o)
    refs = {}
    out = []
    for j, job in enumerate(jobs):
        x, v = workloads.uneven_arrays(job)
        got = co.uneven_oracle_job(o, tabs, job, x, v).reshape(job["L"], job["n"])
        n = job["n"]
        for i, key in enumerate(job["keys"]):
            q, psi = workloads.modulus(*key)
            if (n, q, psi) not in refs:
                refs[(n, q, psi)] = r.ntt(n, q, psi)
            h = refs[(n, q, psi)]
            if job["kind"] == 1:
                want = h.forward(x[i], job["in_f"], job["out_f"])
            else:
                y = r.reduce(x[i], q, 4, 2) if job["in_f"] == 4 else x[i]
                if job["kind"] == 2:
                    want = h.inverse(y, 2, job["out_f"])
                else:
                    y = r.mul(h.inverse(y, 2, 2), v[i], q, 2)
                    want = h.forward(y, 1, job["out_f"])
            check(np.array_equal(want, got[i]), f"uneven job {j} limb {i}")
        out.append({"kind": job["kind"], "n": n, "L": job["L"], "in_f": job["in_f"], "out_f": job["out_f"],
                    "input_sha256": co.digest(x), "sha256": co.digest(got)})
    return {"jobs": out, "limbs": sum(j["L"] for j in jobs),
            "limb_transforms": sum(j["L"] * (2 if j["kind"] == 3 else 1) for j in jobs)}


def main():
    o, r = Oracle(), Reference()
    t = time.time()
    doc = {"generator": "tests/golden/make_config_digests.py: oracle (oracle/axhel_oracle.c) per-limb call "
                        "sequences, each output checked against the reference native backend (oracle/_ref)",
           "hash": "SHA-256 of the uint64 little-endian output words, limbs in order"}
    doc["headline"] = headline(o, r)
    print(f"headline done {time.time() - t:.1f} s", flush=True)
    doc["tensor"] = tensor(o, r)
    print(f"tensor done {time.time() - t:.1f} s", flush=True)
    doc["uneven"] = uneven(o, r)
    print(f"uneven done {time.time() - t:.1f} s", flush=True)
    with open(os.path.join(HERE, "config_digests.json"), "w") as f:
        json.dump(doc, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
