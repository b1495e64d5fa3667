"""The benchmark configurations at their full sizes, on the CPU checkers.

TEST INFRASTRUCTURE: rebuilds the exact seeded inputs of the configurations
the bench runs (the headline batched round trip, the tensor-product chain
and the 512-polynomial uneven batch; generators in bench.py and
axhel_b200/workloads.py) and computes every output with the oracle's
multi-threaded per-limb call sequences (oracle/axhel_oracle.c
orc_job_batch / orc_tensor_batch, restating axhel/ntt/ntt.cpp:173-204 and
axhel/eltwise/eltwise-*-mod.cpp).  Used by the full-size GPU parity test and
by tests/golden/make_config_digests.py, which commits the SHA-256 of each
output so that a run without the oracle can still check its bits.
"""
from __future__ import annotations

import hashlib

import numpy as np


def digest(arr) -> str:
    """SHA-256 of a uint64 array's little-endian bytes (C order)."""
    a = np.ascontiguousarray(arr, dtype=np.uint64)
    return hashlib.sha256(a.astype("<u8", copy=False).tobytes()).hexdigest()


class Tables:
    """Oracle twiddle tables per (N, q, psi), built once."""

    def __init__(self, oracle):
        self.o, self.cache = oracle, {}

    def get(self, n, q, psi):
        k = (n, q, psi)
        if k not in self.cache:
            self.cache[k] = self.o.tables(n, q, psi)
        return self.cache[k]


# ------------------------------------------------------------ headline batch

def headline_case():
    """(mods, data): the bench step's 24 moduli and its 768 x 2^16 input."""
    import bench

    mods = bench.workload_moduli()
    return mods, bench.make_inputs(mods, bench.COUNT, bench.SEED)


def headline_oracle(oracle, mods, data, threads=0):
    """ComputeForward(1,4) on every limb, then ReduceMod(4,2) ->
    ComputeInverse(2,1) on those results: (forward_lazy, round_trip)."""
    import bench

    tabs = Tables(oracle)
    qs = [q for q, _ in mods]
    tl = [tabs.get(bench.N, q, psi) for q, psi in mods]
    flat = np.ascontiguousarray(data.reshape(-1))
    fwd = oracle.job_batch(1, flat, bench.N, bench.COUNT, qs, tl, 1, 4, threads=threads)
    back = oracle.job_batch(2, fwd, bench.N, bench.COUNT, qs, tl, 4, 1, threads=threads)
    return fwd, back


# ------------------------------------------------------------ tensor product

def tensor_oracle(oracle, inputs=None, threads=0):
    """(n, qs, count, inputs, (r0, r1, r2)) for the C3 chain at its full size."""
    from axhel_b200 import workloads

    n, qs, count, ins = inputs if inputs is not None else workloads.tensor_inputs(**workloads.TENSOR_SHAPE)
    flat = [np.ascontiguousarray(a.reshape(-1)) for a in ins]
    outs = oracle.tensor_batch(*flat, n, count, qs, 1, threads=threads)
    return n, qs, count, ins, outs


# ------------------------------------------------------------ uneven batch

def uneven_case():
    """The C4 job list (host specs: kind, n, L, per-limb (q, psi), factors, seed)."""
    from axhel_b200 import workloads

    return workloads.uneven_specs()


def uneven_oracle_job(oracle, tables, job, x=None, v=None, threads=0):
    """One C4 job's full output on the oracle: the per-limb call sequence of
    its kind on each of its L limbs (limb i with its own modulus)."""
    from axhel_b200 import workloads

    if x is None:
        x, v = workloads.uneven_arrays(job)
    n, L = job["n"], job["L"]
    mods = [workloads.modulus(*k) for k in job["keys"]]
    qs = [q for q, _ in mods]
    tl = [tables.get(n, q, psi) for q, psi in mods]
    vec = None if v is None else np.ascontiguousarray(v.reshape(-1))
    return oracle.job_batch(job["kind"], np.ascontiguousarray(x.reshape(-1)), n, L, qs, tl, job["in_f"],
                            job["out_f"], vec=vec, threads=threads)
