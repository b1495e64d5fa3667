"""Workload generators and timers for the batched, fused and serving forms.

    python -m axhel_b200.workloads tensor   # fused tensor-product chain vs per-limb calls
    python -m axhel_b200.workloads uneven   # 512 uneven polynomials in one launch vs per-limb calls
    python -m axhel_b200.workloads product  # fused NTT -> MulMod -> INTT vs three batched calls
    python -m axhel_b200.workloads serve    # Poisson arrivals at 50/70/90 % of capacity
    python -m axhel_b200.workloads eltwise  # streaming eltwise kernels, GB/s at 2^24 elements
    python -m axhel_b200.workloads case F   # a small case of kernel family F, for a profiler

Each prints one JSON line.  Inputs are seeded synthetic residues (uniform in
[0, f*q)), primes from the deterministic search of `params`.  GPU times are
CUDA-event device times; serving latencies are host wall times from submit to
the result being available (copies included).
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys
import threading
import time

import numpy as np

from . import capi, params

UNIT = "limb-transforms/s"


def _events():
    import torch

    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _dev(arr):
    import torch

    return torch.from_numpy(np.ascontiguousarray(arr).view(np.int64)).cuda()


class ModulusPool:
    """NTT handles per (N, bits, position), shared by all jobs (tables stay
    resident); `moduli` alone needs no GPU."""

    def __init__(self):
        self.cache = {}

    def get(self, n, bits, pos):
        key = (n, bits, pos)
        if key not in self.cache:
            q, psi = modulus(n, bits, pos)
            self.cache[key] = (q, capi.NTT(n, q, psi))
        return self.cache[key]


_MODULI = {}


def modulus(n, bits, pos):
    """(q, psi): the NTT-friendly prime of width `bits` nearest position
    pos/4 of its range, q = 1 mod 2n, and its primitive 2n-th root."""
    key = (n, bits, pos)
    if key not in _MODULI:
        q = params.ntt_prime_near(n, bits, pos, 4)
        _MODULI[key] = (q, params.primitive_root(n, q))
    return _MODULI[key]


def uniform_rows(rng, bounds, n):
    """One row of n residues per bound, uniform integers in [0, bound)."""
    b = np.asarray(bounds, dtype=np.uint64).reshape(-1, 1)
    return rng.integers(0, b, size=(b.shape[0], n), dtype=np.uint64)


# ------------------------------------------------------------------ tensor

TENSOR_SHAPE = dict(pairs=64, L=16, logn=15, seed=3)


def tensor_inputs(pairs=64, L=16, logn=15, seed=3):
    """C3 operands on the host: `pairs` ciphertext pairs x L limbs of
    N = 2^logn residues, 16 primes of 40-55 bits; c0, c1, d0, d1 as
    (pairs*L, N) arrays uniform in [0, q_i).  Returns (n, qs, count, arrays)."""
    n = 1 << logn
    qs = [params.ntt_prime_near(n, 40 + (i % 16), 1 + i // 16, 4) for i in range(L)]
    count = pairs * L
    rng = np.random.default_rng(seed)
    bounds = [qs[i % L] for i in range(count)]
    return n, qs, count, tuple(uniform_rows(rng, bounds, n) for _ in range(4))


def tensor_chain(pairs=64, L=16, logn=15, reps=5, seed=3, keep=False):
    """C3: (c0*d0, c0*d1 + c1*d0, c1*d1) then ReduceMod(4,1): one fused launch
    over all limbs vs the reference's per-limb call sequence.  keep=True
    also returns the fused results (device tensors) under "results"."""
    import torch

    n, qs, count, host_in = tensor_inputs(pairs, L, logn, seed)
    c0, c1, d0, d1 = (_dev(a) for a in host_in)
    del host_in
    r0, r1, r2 = (torch.empty_like(c0) for _ in range(3))
    t1 = torch.empty_like(c0)
    P = lambda t, i=0: t.data_ptr() + 8 * n * i

    def fused():
        capi.tensor_product(P(r0), P(r1), P(r2), P(c0), P(c1), P(d0), P(d1), n, count, qs, 1)

    def per_limb():
        for i in range(count):
            q = qs[i % L]
            capi.mul(P(r0, i), P(c0, i), P(d0, i), n, q, 1)
            capi.mul(P(r1, i), P(c0, i), P(d1, i), n, q, 1)
            capi.mul(P(t1, i), P(c1, i), P(d0, i), n, q, 1)
            capi.add(P(r1, i), P(r1, i), P(t1, i), n, q)
            capi.mul(P(r2, i), P(c1, i), P(d1, i), n, q, 1)
            for r in (r0, r1, r2):
                capi.reduce(P(r, i), P(r, i), n, q, 4, 1)

    def timed(fn, k):
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    per_limb()
    ref = [t.clone() for t in (r0, r1, r2)]
    ms_sep = timed(per_limb, 1)
    ms_fused = timed(fused, reps)
    same = all(torch.equal(a, b) for a, b in zip(ref, (r0, r1, r2)))
    elems = count * n
    alg = 56 * elems  # 4 reads + 3 writes of 8 bytes per coefficient-limb
    out = {"workload": f"tensor product chain, N=2^{logn}, L={L}, {pairs} ciphertext pairs",
           "elements": elems, "fused_ms": ms_fused, "per_limb_calls_ms": ms_sep,
           "speedup": ms_sep / ms_fused, "fused_GBps": alg / (ms_fused / 1e3) / 1e9, "same_bits": same}
    if keep:
        out["results"] = (r0, r1, r2)
    return out


# ------------------------------------------------------------------ product

def product_chain(logn=16, limbs=24, polys=32, reps=10, seed=5):
    """The polynomial product in evaluation form over the headline's shape
    (24 primes of 50-59 bits, 32 polynomials): per limb ComputeForward(x, 4, 4)
    -> EltwiseMulMod(., m, 4) -> ComputeInverse(2, 1), as the fused product
    (one pass fused at the transforms' common contiguous pass) and as three
    batched calls (forward batch, one element-wise MulMod job, inverse batch)."""
    import torch

    n = 1 << logn
    mods = params.rns_moduli(n, limbs, 50, 59)
    ntts = capi.NTT.create_many([(n, q, psi) for q, psi in mods])
    count = limbs * polys
    rng = np.random.default_rng(seed)
    bounds = [4 * mods[i % limbs][0] for i in range(count)]
    x = _dev(uniform_rows(rng, bounds, n))
    m = _dev(uniform_rows(rng, bounds, n))
    y, z = torch.empty_like(x), torch.empty_like(x)
    mul = capi.Batch([dict(kind=capi.JOB_MUL, ntts=ntts, count=count, result=z.data_ptr(), operand=z.data_ptr(),
                           vector=m.data_ptr(), in_f=4, out_f=1)])

    def fused():
        capi.product_batch(ntts, y.data_ptr(), x.data_ptr(), m.data_ptr(), count, 4, 1)

    def separate():
        capi.forward_batch(ntts, z.data_ptr(), x.data_ptr(), count, 4, 4)
        mul.launch(phased=True)
        capi.inverse_batch(ntts, z.data_ptr(), z.data_ptr(), count, 2, 1)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_f, ms_s = timed(fused), timed(separate)
    same = torch.equal(y, z)
    mul.close()
    # the two halves: forward then MulMod, MulMod then inverse
    w = torch.empty_like(x)
    mul_x = capi.Batch([dict(kind=capi.JOB_MUL, ntts=ntts, count=count, result=w.data_ptr(), operand=x.data_ptr(),
                             vector=m.data_ptr(), in_f=4, out_f=1)])
    halves = {}
    for name, fused_fn, sep_fn in (
            ("forward_mul", lambda: capi.forward_mul_batch(ntts, y.data_ptr(), x.data_ptr(), m.data_ptr(), count),
             lambda: (capi.forward_batch(ntts, z.data_ptr(), x.data_ptr(), count, 4, 4), mul.launch(phased=True))),
            ("mul_inverse", lambda: capi.mul_inverse_batch(ntts, y.data_ptr(), x.data_ptr(), m.data_ptr(), count, 1),
             lambda: (mul_x.launch(phased=True), capi.inverse_batch(ntts, z.data_ptr(), w.data_ptr(), count, 2, 1)))):
        if name == "forward_mul":
            mul = capi.Batch([dict(kind=capi.JOB_MUL, ntts=ntts, count=count, result=z.data_ptr(),
                                   operand=z.data_ptr(), vector=m.data_ptr(), in_f=4, out_f=1)])
        a, b = timed(fused_fn), timed(sep_fn)
        halves[name] = {"fused_ms": a, "separate_calls_ms": b, "speedup": b / a, "same_bits": torch.equal(y, z)}
        if name == "forward_mul":
            mul.close()
    mul_x.close()
    return {"workload": f"NTT -> MulMod -> INTT, N=2^{logn}, {count} limbs ({limbs} primes of 50-59 bits)",
            "fused_ms": ms_f, "separate_calls_ms": ms_s, "speedup": ms_s / ms_f,
            "fused_rate": 2 * count / (ms_f / 1e3), "unit": UNIT, "same_bits": same, **halves}


# ------------------------------------------------------------------ uneven

def uneven_specs(n_polys=512, seed=11, logn_lo=12, logn_hi=17, max_L=48):
    """C4 job list (host only): polynomials with N ~ U{2^12..2^17}, L ~
    U{1..48} limbs (primes of 30-60 bits), input factor ~ U{1,2,4}; a third
    forward, a third inverse, a third INTT -> MulMod -> NTT with a plaintext
    vector.  Each job: kind, n, L, mods [(q, psi)] per limb, in_f, out_f and
    the seed of its operands (`uneven_arrays`)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_polys):
        logn = int(rng.integers(logn_lo, logn_hi + 1))
        n = 1 << logn
        L = int(rng.integers(1, max_L + 1))
        kind = (1, 2, 3)[j % 3]
        keys = [(n, int(rng.integers(30, 61)), int(rng.integers(1, 4))) for _ in range(L)]
        in_f = int(rng.choice([1, 2, 4]))
        out_f = int(rng.choice([1, 2])) if kind == 2 else int(rng.choice([1, 4]))
        jobs.append(dict(kind=kind, n=n, L=L, keys=keys, mods=[modulus(*k) for k in keys], in_f=in_f, out_f=out_f,
                         seed=int(rng.integers(1 << 30))))
    return jobs


def uneven_arrays(job):
    """A C4 job's operands on the host: x (L, N) uniform in [0, in_f*q_i),
    and for chains the vector (L, N) uniform in [0, 2 q_i)."""
    rng = np.random.default_rng(job["seed"])
    qs = [q for q, _ in job["mods"]]
    x = uniform_rows(rng, [job["in_f"] * q for q in qs], job["n"])
    v = uniform_rows(rng, [2 * q for q in qs], job["n"]) if job["kind"] == 3 else None
    return x, v


def uneven_jobs(pool, n_polys=512, seed=11, logn_lo=12, logn_hi=17, max_L=48):
    """C4 jobs with device handles (`ModulusPool`) for their moduli."""
    jobs = uneven_specs(n_polys, seed, logn_lo, logn_hi, max_L)
    for job in jobs:
        job["mods"] = [pool.get(*k) for k in job["keys"]]
    return jobs


def _job_arrays(job):
    import torch

    x, v = uneven_arrays(job)
    job["x"] = _dev(x)
    job["y"] = torch.empty_like(job["x"])
    if v is not None:
        job["v"] = _dev(v)


def uneven_batch(n_polys=512, seed=11, reps=3, keep=False):
    """C4 timed three ways (per-limb calls, one persistent launch, per-phase
    launches), each checked against the per-limb results; keep=True also
    returns the jobs with their device results ("y", from the per-phase
    launches) under "jobs"."""
    import torch

    pool = ModulusPool()
    jobs = uneven_jobs(pool, n_polys, seed)
    for job in jobs:
        _job_arrays(job)
    specs = [dict(kind=j["kind"], ntts=[t for _, t in j["mods"]], count=j["L"], result=j["y"].data_ptr(),
                  operand=j["x"].data_ptr(), vector=j["v"].data_ptr() if j["kind"] == 3 else 0,
                  in_f=j["in_f"], out_f=j["out_f"]) for j in jobs]
    transforms = sum(j["L"] * (2 if j["kind"] == 3 else 1) for j in jobs)
    b = capi.Batch(specs)

    def one_launch():
        b.launch()

    def phased():
        b.launch(phased=True)

    def per_limb():
        for j in jobs:
            n = j["n"]
            for i, (q, t) in enumerate(j["mods"]):
                xo, yo = j["x"].data_ptr() + 8 * n * i, j["y"].data_ptr() + 8 * n * i
                if j["kind"] == 1:
                    t.forward(yo, xo, j["in_f"], j["out_f"])
                    continue
                src = xo
                if j["in_f"] == 4:
                    capi.reduce(yo, xo, n, q, 4, 2)
                    src = yo
                if j["kind"] == 2:
                    t.inverse(yo, src, 2, j["out_f"])
                else:
                    t.inverse(yo, src, 2, 2)
                    capi.mul(yo, yo, j["v"].data_ptr() + 8 * n * i, n, q, 2)
                    t.forward(yo, yo, 1, j["out_f"])

    def timed(fn, k):
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(k):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    per_limb()
    ref = [j["y"].clone() for j in jobs]
    ms_plain = timed(per_limb, 1)
    for j in jobs:
        j["y"].zero_()
    ms_batch = timed(one_launch, reps)
    st = b.status()
    same = st == 0 and all(torch.equal(r, j["y"]) for r, j in zip(ref, jobs))
    for j in jobs:
        j["y"].zero_()
    ms_phased = timed(phased, reps)
    same = same and b.status() == 0 and all(torch.equal(r, j["y"]) for r, j in zip(ref, jobs))
    b.close()
    del ref
    limbs = sum(j["L"] for j in jobs)
    out = {"workload": f"{n_polys} uneven polynomials, N in 2^12..2^17, L in 1..48, fwd/inv/chain mix",
           "limbs": limbs, "limb_transforms": transforms, "one_launch_ms": ms_batch,
           "one_launch_rate": transforms / (ms_batch / 1e3), "phased_ms": ms_phased,
           "phased_rate": transforms / (ms_phased / 1e3), "per_limb_calls_ms": ms_plain,
           "per_limb_rate": transforms / (ms_plain / 1e3), "speedup": ms_plain / ms_batch, "same_bits": same,
           "unit": UNIT}
    if keep:
        out["jobs"] = jobs
    return out


# ------------------------------------------------------------------ serving

class RequestPool:
    """C5 request templates: INTT -> MulMod/FMAMod -> NTT, N ~ U{2^13..2^17},
    L ~ U{2..40}, primes of 40-59 bits.  Inputs and vectors live in pinned
    host memory (host-staged requests) or in HBM (device-resident requests);
    `copies` output buffers per template."""

    def __init__(self, n_templates=32, seed=21, copies=4, device=False, logn_lo=13, logn_hi=17, L_lo=2, L_hi=40):
        import torch

        rng = np.random.default_rng(seed)
        self.pool = ModulusPool()
        self.t = []
        self.device = device
        for k in range(n_templates):
            logn = int(rng.integers(logn_lo, logn_hi + 1))
            n = 1 << logn
            L = int(rng.integers(L_lo, L_hi + 1))
            mods = [self.pool.get(n, 40 + (i % 20), 1 + (i // 20) % 3) for i in range(L)]
            qs = [2 * q for q, _ in mods]
            kind = 3 if k % 2 == 0 else 4

            def place(a):
                t = torch.from_numpy(a.reshape(-1).view(np.int64))
                return t.cuda() if device else t.pin_memory()

            x = place(uniform_rows(rng, qs, n))
            v = place(uniform_rows(rng, qs, n))
            outs = [torch.empty(L * n, dtype=torch.int64, device="cuda" if device else "cpu") for _ in range(copies)]
            if not device:
                outs = [o.pin_memory() for o in outs]
            sc = [int(rng.integers(0, 2 * int(q))) for q, _ in mods]
            self.t.append(dict(n=n, L=L, kind=kind, ntts=[t for _, t in mods], x=x, v=v, outs=outs,
                               free=list(range(copies)), sc=sc))
        self.lock = threading.Lock()

    def take(self, rng):
        with self.lock:
            for _ in range(4 * len(self.t)):
                k = int(rng.integers(len(self.t)))
                if self.t[k]["free"]:
                    return k, self.t[k]["free"].pop()
        return None

    def give(self, k, slot):
        with self.lock:
            self.t[k]["free"].append(slot)

    def submit(self, srv, k, slot):
        t = self.t[k]
        return srv.submit(t["kind"], t["ntts"], t["L"], t["x"].data_ptr(), t["outs"][slot].data_ptr(),
                          vector=t["v"].data_ptr(), scalars=t["sc"] if t["kind"] == 4 else None, in_f=2, out_f=4)


def _pct(v, p):
    v = sorted(v)
    return v[min(len(v) - 1, int(p * (len(v) - 1) + 0.5))] if v else None


def serving(loads=(0.5, 0.7, 0.9), seconds=4.0, budget=60 << 30, inflight=4, seed=5, n_templates=32,
            device=False, max_batch_words=0, persistent=False, plain=True, small_words=0, reserve=8 << 30,
            max_batch_requests=256, flags=0, aging_us=0, batch_size_ratio=0, small_pct=None):
    """Isolated latency of every template (alone on an idle server), capacity
    (a burst), then Poisson arrivals at each load fraction of capacity
    (host-staged requests: `reserve` bytes of the staging pool mapped up
    front): p50/p99 latency, p99 of each request's slowdown against its own isolated
    latency, and jobs/s; then the plain sequential GPU path."""
    rp = RequestPool(n_templates=n_templates, seed=seed, device=device)
    if small_pct is not None:  # two lanes split at this percentile of the templates' sizes
        sizes = sorted(t["n"] * t["L"] for t in rp.t)
        small_words = sizes[min(len(sizes) - 1, int(small_pct / 100 * (len(sizes) - 1)))]
    srv = capi.Server(budget_bytes=budget, max_inflight=inflight, max_batch_requests=max_batch_requests,
                      max_batch_words=max_batch_words, persistent=persistent, small_request_words=small_words,
                      reserve_bytes=0 if device else reserve, flags=flags, aging_us=aging_us,
                      batch_size_ratio=batch_size_ratio)
    rng = np.random.default_rng(seed)

    iso = []
    for k in range(len(rp.t)):
        runs = []
        for _ in range(3):
            rid = rp.submit(srv, k, 0)
            st, info = srv.wait(rid)
            assert st == 0
            runs.append(info.latency_ms)
        iso.append(statistics.median(runs))

    # capacity: a burst queued while admission is held, timed from its release
    caps = []
    for _ in range(3):
        burst = []
        srv.pause(True)
        for i in range(8 * len(rp.t)):
            got = rp.take(rng)
            if got is None:
                break
            burst.append((rp.submit(srv, *got), got))
        t0 = time.perf_counter()
        srv.pause(False)
        for rid, got in burst:
            st, _ = srv.wait(rid)
            assert st == 0
            rp.give(*got)
        caps.append(len(burst) / (time.perf_counter() - t0))
    cap = statistics.median(caps)
    srv.stats(reset=True)

    results = []
    templates = [dict(kind=t["kind"], ntts=t["ntts"], count=t["L"], input=t["x"].data_ptr(),
                      vector=t["v"].data_ptr(), scalars=t["sc"] if t["kind"] == 4 else None, in_f=2, out_f=4)
                 for t in rp.t]
    outputs = [[o.data_ptr() for o in t["outs"]] for t in rp.t]
    for frac in loads:
        d = srv.drive(templates, outputs, iso, frac * cap, seconds, seed=int(frac * 1000) + seed)
        results.append({"load": frac, "offered_per_s": frac * cap, "jobs_per_s": d["jobs_per_s"],
                        "p50_ms": d["p50_ms"], "p99_ms": d["p99_ms"], "isolated_p99_ms": d["isolated_p99_ms"],
                        "p99_over_isolated_p99": d["p99_ms"] / d["isolated_p99_ms"] if d["isolated_p99_ms"] else None,
                        "p50_slowdown": d["p50_slowdown"], "p99_slowdown": d["p99_slowdown"],
                        "p50_queue_ms": d["p50_queue_ms"], "p99_queue_ms": d["p99_queue_ms"],
                        "p99_large_ms": d["p99_large_ms"], "p99_rest_ms": d["p99_rest_ms"],
                        "requests": d["completed"], "skipped_no_buffer": d["skipped"], "failed": d["failed"]})
    st = srv.stats()
    srv.close()

    out = {"workload": "INTT->MulMod/FMAMod->NTT requests, N in 2^13..2^17, L in 2..40, Poisson arrivals",
           "operands": "device-resident" if device else "host pinned, staged per request",
           "launch": "persistent" if persistent else "per-phase class launches", "max_batch_words": max_batch_words,
           "small_request_words": small_words,
           "policy": policy_name(flags, aging_us) + (
               f"; two lanes split at {small_words} residues, the {'large' if flags & capi.SERVER_LARGE_FIRST else 'small'}"
               " one at high stream priority" if small_words else "") + (
               f"; {max_batch_requests} request(s) per batch" if max_batch_requests < 8 else ""),
           "batch_size_ratio": batch_size_ratio, "max_batch_requests_cfg": max_batch_requests,
           "capacity_jobs_per_s": cap, "isolated_median_ms": statistics.median(iso), "loads": results,
           "batches": st["batches"], "max_batch_requests": st["max_batch_requests"],
           "host_us_per_batch": st["host_us_per_batch"],
           "peak_in_use_bytes": st["peak_in_use_bytes"], "budget_bytes": budget, "max_inflight": inflight}
    if plain:
        out["plain_sequential_jobs_per_s"] = plain_sequential(rp)
    return out


def policy_name(flags, aging_us=0):
    """Readable name of the server's scheduling flags."""
    parts = []
    if flags & capi.SERVER_ARRIVAL_PRIORITY:
        parts.append("arrival-priority streams")
    if flags & capi.SERVER_SMALLEST_FIRST:
        parts.append(f"smallest-first admission (aging {aging_us} us)")
    if flags & capi.SERVER_LARGE_FIRST:
        parts.append("large-request lane at high priority")
    return ", ".join(parts) or "arrival-order admission"


def plain_sequential(rp, limit=16):
    """Each request as the reference call pattern: per limb ComputeInverse,
    MulMod / FMAMod, ComputeForward through the C-ABI, one request after the
    other, operands copied in and out as in the served form."""
    import torch

    n_req = min(len(rp.t), limit)
    t0 = time.perf_counter()
    for k in range(n_req):
        t = rp.t[k]
        n = t["n"]
        x = t["x"] if rp.device else t["x"].cuda(non_blocking=True)
        v = t["v"] if rp.device else t["v"].cuda(non_blocking=True)
        y = torch.empty_like(x)
        for i, h in enumerate(t["ntts"]):
            o = 8 * n * i
            h.inverse(y.data_ptr() + o, x.data_ptr() + o, 2, 2)
            if t["kind"] == 3:
                capi.mul(y.data_ptr() + o, y.data_ptr() + o, v.data_ptr() + o, n, h.modulus, 2)
            else:
                capi.fma(y.data_ptr() + o, y.data_ptr() + o, t["sc"][i], v.data_ptr() + o, n, h.modulus, 2)
            h.forward(y.data_ptr() + o, y.data_ptr() + o, 1, 4)
        t["outs"][0].copy_(y)
        torch.cuda.synchronize()
    return n_req / (time.perf_counter() - t0)


# ------------------------------------------------------------------ kernels

def eltwise_rates(n=1 << 24, reps=30):
    """Algorithmic GB/s of the streaming eltwise kernels on 2^24-element
    device vectors (128 MiB each, above the L2)."""
    import torch

    q = params.ntt_prime_near(1 << 16, 50, 1, 1)
    rng = np.random.default_rng(1)
    a, b, c = (_dev(rng.integers(0, q, n, dtype=np.uint64)) for _ in range(3))
    big = _dev(rng.integers(0, 2**63, n, dtype=np.uint64))
    r = torch.empty_like(a)
    P = lambda t: t.data_ptr()
    cases = [("add_vv", 24, lambda: capi.add(P(r), P(a), P(b), n, q)),
             ("add_vs", 16, lambda: capi.add(P(r), P(a), 5, n, q, scalar=True)),
             ("mul_f1", 24, lambda: capi.mul(P(r), P(a), P(b), n, q, 1)),
             ("fma_f1", 24, lambda: capi.fma(P(r), P(a), 12345, P(c), n, q, 1)),
             ("reduce_4to1", 16, lambda: capi.reduce(P(r), P(a), n, q, 4, 1)),
             ("reduce_barrett", 16, lambda: capi.reduce(P(r), P(big), n, q, q, 1))]
    out = {"elements": n, "unit": "GB/s (algorithmic bytes / CUDA-event time)"}
    for name, bpe, fn in cases:
        fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = bpe * n / (e0.elapsed_time(e1) / reps / 1e3) / 1e9
    return out


def kernel_case(family):
    """A small case of one kernel family, launched two or three times: the
    command a profiler runs (inputs above the L2, a few hundred MB)."""
    import torch

    rng = np.random.default_rng(1)
    if family in ("eltwise", "eltwise_unaligned"):  # add, mul, fma, Barrett reduce on 2^24 elements, twice
        n = 1 << 24
        q = params.ntt_prime_near(1 << 16, 50, 1, 1)
        a, b, c = (_dev(rng.integers(0, q, n, dtype=np.uint64)) for _ in range(3))
        r = torch.empty_like(a)
        off = 8 if family == "eltwise_unaligned" else 0  # 8-byte aligned operands: the scalar kernel
        m = n - 1 if off else n
        pa, pb, pc, pr = (t.data_ptr() + off for t in (a, b, c, r))
        for _ in range(2):
            capi.add(pr, pa, pb, m, q)
            capi.mul(pr, pa, pb, m, q, 1)
            capi.fma(pr, pa, 12345, pc, m, q, 1)
            capi.reduce(pr, pa, m, q, q, 1)
    elif family == "tensor":  # 16 pairs x 16 limbs of N = 2^15
        L, n, pairs = 16, 1 << 15, 16
        qs = [q for q, _ in params.rns_moduli(n, L, 40, 55)]
        cnt = pairs * L
        ins = [_dev(np.concatenate([rng.integers(0, qs[i % L], n, dtype=np.uint64) for i in range(cnt)]))
               for _ in range(4)]
        outs = [torch.empty_like(ins[0]) for _ in range(3)]
        for _ in range(2):
            capi.tensor_product(*[o.data_ptr() for o in outs], *[x.data_ptr() for x in ins], n, cnt, qs, 1)
    elif family == "peak":  # the register-only butterfly probe, forward then inverse (two launches each)
        n = 1 << 16
        q, psi = params.rns_moduli(n, 1, 50, 50)[0]
        t = capi.NTT(n, q, psi)
        for inv in (False, True):
            capi.butterfly_peak(t, inv)
    elif family == "cluster":  # one limb of N = 2^12, forward and inverse: the one-launch cluster form
        n = 1 << 12
        q, psi = params.rns_moduli(n, 1, 50, 59)[0]
        t = capi.NTT(n, q, psi)
        x = _dev(rng.integers(0, q, n, dtype=np.uint64))
        for _ in range(3):
            capi.forward_batch([t], x.data_ptr(), x.data_ptr(), 1, 4, 4)
            capi.inverse_batch([t], x.data_ptr(), x.data_ptr(), 1, 4, 1)
    elif family == "cluster_chain":  # one limb of N = 2^12: INTT -> MulMod -> NTT and NTT -> MulMod -> INTT
        n = 1 << 12
        q, psi = params.rns_moduli(n, 1, 50, 59)[0]
        t = capi.NTT(n, q, psi)
        x = _dev(rng.integers(0, q, n, dtype=np.uint64))
        m = _dev(rng.integers(0, q, n, dtype=np.uint64))
        for _ in range(3):
            capi.chain_mul_batch([t], x.data_ptr(), x.data_ptr(), m.data_ptr(), 1, 2, 1)
            capi.product_batch([t], x.data_ptr(), x.data_ptr(), m.data_ptr(), 1, 4, 1)
    elif family == "tables":  # 3 x 24 fresh contexts of N = 2^16
        for lo, hi in ((30, 40), (41, 51), (52, 62)):
            capi.NTT.create_many([(1 << 16, q, psi) for q, psi in params.rns_moduli(1 << 16, 24, lo, hi)])
    elif family in ("chain", "batch", "batch_phased", "batch_eltwise"):  # 384 limbs of N = 2^16 (192 MiB), 24 moduli
        n = 1 << 16
        mods = params.rns_moduli(n, 24, 50, 59)
        ntts = [capi.NTT(n, q, psi) for q, psi in mods]
        x = _dev(np.concatenate([rng.integers(0, mods[i % 24][0], n, dtype=np.uint64) for i in range(384)]))
        v = x.clone()
        if family == "chain":  # INTT -> MulMod -> NTT, fused
            for _ in range(2):
                capi.chain_mul_batch(ntts, x.data_ptr(), x.data_ptr(), v.data_ptr(), 384, 2, 4)
        elif family in ("batch", "batch_phased"):  # one forward job: one persistent launch, or one per phase
            b = capi.Batch([dict(kind=capi.JOB_FORWARD, ntts=ntts, count=384, result=x.data_ptr(),
                                 operand=x.data_ptr(), in_f=4, out_f=4)])
            for _ in range(3):
                b.launch(phased=family == "batch_phased")
        else:  # one MulMod job, one launch per phase
            b = capi.Batch([dict(kind=capi.JOB_MUL, ntts=ntts, count=384, result=x.data_ptr(), operand=x.data_ptr(),
                                 vector=v.data_ptr(), in_f=1, out_f=1)])
            for _ in range(2):
                b.launch(phased=True)
    else:
        raise SystemExit(f"unknown kernel family {family}")
    torch.cuda.synchronize()
    return {"case": family, "ok": True}


def small_transform_latency(counts=(1, 4, 16, 64), reps=40):
    """Device time per batched call on a few limbs, N = 2^10..2^17, in the
    one-launch cluster form (built-in choice) and in the pass form (two
    launches for a transform, three for a fused chain or product): forward,
    inverse, INTT -> MulMod -> NTT chain and NTT -> MulMod -> INTT product;
    `reps` calls captured in a CUDA graph and replayed (no host launch cost),
    best of 5 replays, microseconds per call."""
    import torch

    names = {capi.CLUSTER_FORWARD: "forward", capi.CLUSTER_INVERSE: "inverse", capi.CLUSTER_CHAIN: "chain_mul",
             capi.CLUSTER_PRODUCT: "product"}
    rows = []
    for logn in range(10, 18):
        n = 1 << logn
        mods = params.rns_moduli(n, 4, 50, 59)
        ntts = [capi.NTT(n, q, p) for q, p in mods]
        for count in counts:
            x = torch.randint(0, 1 << 40, (count * n,), dtype=torch.int64, device="cuda")
            y = torch.empty_like(x)
            m = torch.randint(0, 1 << 40, (count * n,), dtype=torch.int64, device="cuda")
            calls = {
                capi.CLUSTER_FORWARD: lambda st: capi.forward_batch(ntts, y.data_ptr(), x.data_ptr(), count, 4, 4,
                                                                    st),
                capi.CLUSTER_INVERSE: lambda st: capi.inverse_batch(ntts, y.data_ptr(), x.data_ptr(), count, 2, 2,
                                                                    st),
                capi.CLUSTER_CHAIN: lambda st: capi.chain_mul_batch(ntts, y.data_ptr(), x.data_ptr(), m.data_ptr(),
                                                                    count, 2, 4, st),
                capi.CLUSTER_PRODUCT: lambda st: capi.product_batch(ntts, y.data_ptr(), x.data_ptr(), m.data_ptr(),
                                                                    count, 4, 1, st),
            }
            for kind, call in calls.items():
                row = {"logn": logn, "count": count, "direction": names[kind]}
                cfg = capi.cluster_plan_get(kind, logn)
                for form in ("cluster", "passes"):
                    if form == "cluster" and cfg[3] < count:
                        continue
                    if cfg[0]:
                        capi.cluster_plan_set(kind, logn, *cfg[:3], 0 if form == "passes" else max(cfg[3], 1))
                    s = torch.cuda.Stream()
                    s.wait_stream(torch.cuda.current_stream())
                    with torch.cuda.stream(s):
                        for _ in range(3):
                            call(s.cuda_stream)
                    torch.cuda.synchronize()
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=s):
                        for _ in range(reps):
                            call(s.cuda_stream)
                    best = float("inf")
                    for _ in range(5):
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record()
                        g.replay()
                        e1.record()
                        torch.cuda.synchronize()
                        best = min(best, e0.elapsed_time(e1) * 1e3 / reps)
                    del g
                    row[f"{form}_us"] = round(best, 2)
                capi.cluster_plan_set(kind, logn)
                rows.append(row)
    return {"workload": "device time per call, a few limbs of N = 2^10..2^17 (CUDA-graph replay)",
            "cluster_form": {names[k]: {str(l): capi.cluster_plan_get(k, l) for l in range(10, 18)} for k in names},
            "rows": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["tensor", "uneven", "serve", "eltwise", "case", "product", "latency"])
    ap.add_argument("family", nargs="?", default="eltwise",
                    help="case: eltwise | eltwise_unaligned | tensor | tables | chain | batch | batch_phased | "
                         "batch_eltwise | peak | cluster | cluster_chain")
    ap.add_argument("--seconds", type=float, default=4.0)
    ap.add_argument("--device", action="store_true", help="device-resident request operands")
    ap.add_argument("--persistent", action="store_true", help="one persistent launch per batch")
    ap.add_argument("--max-batch-words", type=int, default=0)
    ap.add_argument("--inflight", type=int, default=4)
    ap.add_argument("--small-words", type=int, default=0, help="high-priority lane for requests up to this size")
    ap.add_argument("--max-batch-requests", type=int, default=256)
    ap.add_argument("--arrival-priority", action="store_true", help="batches in flight prioritised by launch order")
    ap.add_argument("--smallest-first", action="store_true", help="admit the smallest pending requests first")
    ap.add_argument("--aging-us", type=int, default=0, help="smallest-first: pending time after which arrival wins")
    ap.add_argument("--large-first", action="store_true", help="two lanes, the large-request lane at high priority")
    ap.add_argument("--small-pct", type=float, default=None,
                    help="two lanes split at this percentile of the templates' sizes")
    ap.add_argument("--size-ratio", type=int, default=0, help="batches only of requests within this size factor")
    ap.add_argument("--loads", default="0.5,0.7,0.9")
    ap.add_argument("--templates", type=int, default=24, help="request templates (the bench uses 24)")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain sequential comparison")
    a = ap.parse_args()
    if a.what == "tensor":
        out = tensor_chain()
    elif a.what == "eltwise":
        out = eltwise_rates()
    elif a.what == "case":
        out = kernel_case(a.family)
    elif a.what == "uneven":
        out = uneven_batch()
    elif a.what == "product":
        out = product_chain()
    elif a.what == "latency":
        out = small_transform_latency()
    else:
        flags = (capi.SERVER_ARRIVAL_PRIORITY if a.arrival_priority else 0) | \
            (capi.SERVER_SMALLEST_FIRST if a.smallest_first else 0) | (capi.SERVER_LARGE_FIRST if a.large_first else 0)
        out = serving(loads=tuple(float(x) for x in a.loads.split(",")), seconds=a.seconds, device=a.device,
                      persistent=a.persistent, max_batch_words=a.max_batch_words, inflight=a.inflight,
                      small_words=a.small_words, max_batch_requests=a.max_batch_requests, flags=flags,
                      aging_us=a.aging_us, n_templates=a.templates, plain=not a.no_plain,
                      batch_size_ratio=a.size_ratio, small_pct=a.small_pct)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
