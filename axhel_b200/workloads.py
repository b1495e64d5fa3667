"""Workload generators and timers for the batched, fused and serving forms.

    python -m axhel_b200.workloads tensor   # fused tensor-product chain vs per-limb calls
    python -m axhel_b200.workloads uneven   # 512 uneven polynomials in one launch vs per-limb calls
    python -m axhel_b200.workloads serve    # Poisson arrivals at 50/70/90 % of capacity

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
    """NTT handles per (N, bits), shared by all jobs (tables stay resident)."""

    def __init__(self):
        self.cache = {}

    def get(self, n, bits, pos):
        key = (n, bits, pos)
        if key not in self.cache:
            q = params.ntt_prime_near(n, bits, pos, 4)
            self.cache[key] = (q, capi.NTT(n, q, params.primitive_root(n, q)))
        return self.cache[key]


# ------------------------------------------------------------------ tensor

def tensor_chain(pairs=64, L=16, logn=15, reps=5, seed=3):
    """C3: (c0*d0, c0*d1 + c1*d0, c1*d1) then ReduceMod(4,1): one fused launch
    over all limbs vs the reference's per-limb call sequence."""
    import torch

    n = 1 << logn
    qs = [params.ntt_prime_near(n, 40 + (i % 16), 1 + i // 16, 4) for i in range(L)]
    count = pairs * L
    rng = np.random.default_rng(seed)
    bounds = np.array([qs[i % L] for i in range(count)], dtype=np.uint64)[:, None]
    c0, c1, d0, d1 = (_dev((rng.random((count, n)) * bounds).astype(np.uint64)) for _ in range(4))
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
    return {"workload": f"tensor product chain, N=2^{logn}, L={L}, {pairs} ciphertext pairs",
            "elements": elems, "fused_ms": ms_fused, "per_limb_calls_ms": ms_sep,
            "speedup": ms_sep / ms_fused, "fused_GBps": alg / (ms_fused / 1e3) / 1e9, "same_bits": same}


# ------------------------------------------------------------------ uneven

def uneven_jobs(pool, n_polys=512, seed=11, logn_lo=12, logn_hi=17, max_L=48):
    """C4: polynomials with N ~ U{2^12..2^17}, L ~ U{1..48} limbs (primes of
    30-60 bits), input factor ~ U{1,2,4}; a third forward, a third inverse,
    a third INTT -> MulMod -> NTT with a plaintext vector."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(n_polys):
        logn = int(rng.integers(logn_lo, logn_hi + 1))
        n = 1 << logn
        L = int(rng.integers(1, max_L + 1))
        kind = (1, 2, 3)[j % 3]
        mods = [pool.get(n, int(rng.integers(30, 61)), int(rng.integers(1, 4))) for _ in range(L)]
        in_f = int(rng.choice([1, 2, 4]))
        out_f = int(rng.choice([1, 2])) if kind == 2 else int(rng.choice([1, 4]))
        jobs.append(dict(kind=kind, n=n, L=L, mods=mods, in_f=in_f, out_f=out_f, seed=int(rng.integers(1 << 30))))
    return jobs


def _job_arrays(job):
    import torch

    n, L = job["n"], job["L"]
    rng = np.random.default_rng(job["seed"])
    qs = np.array([q for q, _ in job["mods"]], dtype=np.uint64)[:, None]
    x = (rng.random((L, n)) * (qs * np.uint64(job["in_f"]))).astype(np.uint64)
    job["x"] = _dev(x)
    job["y"] = torch.empty_like(job["x"])
    if job["kind"] == 3:
        job["v"] = _dev((rng.random((L, n)) * (2 * qs)).astype(np.uint64))


def uneven_batch(n_polys=512, seed=11, reps=3):
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
    b.close()
    limbs = sum(j["L"] for j in jobs)
    return {"workload": f"{n_polys} uneven polynomials, N in 2^12..2^17, L in 1..48, fwd/inv/chain mix",
            "limbs": limbs, "limb_transforms": transforms, "one_launch_ms": ms_batch,
            "one_launch_rate": transforms / (ms_batch / 1e3), "per_limb_calls_ms": ms_plain,
            "per_limb_rate": transforms / (ms_plain / 1e3), "speedup": ms_plain / ms_batch, "same_bits": same,
            "unit": UNIT}


# ------------------------------------------------------------------ serving

class RequestPool:
    """C5 request templates: INTT -> MulMod/FMAMod -> NTT, N ~ U{2^13..2^17},
    L ~ U{2..40}, primes of 40-59 bits; inputs and vectors in pinned host
    memory, `copies` pinned output buffers per template."""

    def __init__(self, n_templates=32, seed=21, copies=4, logn_lo=13, logn_hi=17, L_lo=2, L_hi=40):
        import torch

        rng = np.random.default_rng(seed)
        self.pool = ModulusPool()
        self.t = []
        for k in range(n_templates):
            logn = int(rng.integers(logn_lo, logn_hi + 1))
            n = 1 << logn
            L = int(rng.integers(L_lo, L_hi + 1))
            mods = [self.pool.get(n, 40 + (i % 20), 1 + (i // 20) % 3) for i in range(L)]
            qs = np.array([q for q, _ in mods], dtype=np.uint64)[:, None]
            kind = 3 if k % 2 == 0 else 4

            def pin(a):
                t = torch.from_numpy(a.reshape(-1).view(np.int64)).pin_memory()
                return t

            x = pin((rng.random((L, n)) * (2 * qs)).astype(np.uint64))
            v = pin((rng.random((L, n)) * (2 * qs)).astype(np.uint64))
            outs = [torch.empty(L * n, dtype=torch.int64).pin_memory() for _ in range(copies)]
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


def serving(loads=(0.5, 0.7, 0.9), seconds=4.0, budget=60 << 30, inflight=3, seed=5, n_templates=32):
    """Capacity (a burst), isolated latency (one at a time), then Poisson
    arrivals at each load fraction of capacity: p50/p99 and jobs/s."""
    rp = RequestPool(n_templates=n_templates, seed=seed)
    srv = capi.Server(budget_bytes=budget, max_inflight=inflight, max_batch_requests=256)
    rng = np.random.default_rng(seed)

    # isolated: each template alone on an idle server
    iso = []
    for k in range(len(rp.t)):
        for _ in range(2):
            rid = rp.submit(srv, k, 0)
            st, info = srv.wait(rid)
            assert st == 0
        iso.append(info.latency_ms)
    iso_med = statistics.median(iso)

    # capacity: a burst of requests submitted at once
    burst = []
    t0 = time.perf_counter()
    for i in range(8 * len(rp.t)):
        got = rp.take(rng)
        if got is None:
            break
        burst.append((rp.submit(srv, *got), got))
    for rid, got in burst:
        st, _ = srv.wait(rid)
        assert st == 0
        rp.give(*got)
    cap = len(burst) / (time.perf_counter() - t0)
    srv.stats(reset=True)

    results = []
    for frac in loads:
        rate = frac * cap
        stop = threading.Event()
        inflight_q = []
        qlock = threading.Lock()
        lat = []
        dropped = [0]

        def producer():
            t = time.perf_counter()
            end = t + seconds
            while t < end:
                t += rng.exponential(1.0 / rate)
                while True:
                    now = time.perf_counter()
                    if now >= t:
                        break
                    time.sleep(min(t - now, 0.001))
                got = rp.take(rng)
                if got is None:
                    dropped[0] += 1
                    continue
                rid = rp.submit(srv, *got)
                with qlock:
                    inflight_q.append((rid, got))
            stop.set()

        def consumer():
            while True:
                with qlock:
                    item = inflight_q.pop(0) if inflight_q else None
                if item is None:
                    if stop.is_set():
                        with qlock:
                            if not inflight_q:
                                return
                    time.sleep(0.0002)
                    continue
                rid, got = item
                st, info = srv.wait(rid)
                assert st == 0
                lat.append(info.latency_ms)
                rp.give(*got)

        t0 = time.perf_counter()
        th = [threading.Thread(target=producer), threading.Thread(target=consumer)]
        for x in th:
            x.start()
        for x in th:
            x.join()
        wall = time.perf_counter() - t0
        lat.sort()
        pct = lambda p: lat[min(len(lat) - 1, int(p * (len(lat) - 1) + 0.5))]
        results.append({"load": frac, "offered_per_s": rate, "jobs_per_s": len(lat) / wall, "p50_ms": pct(0.5),
                        "p99_ms": pct(0.99), "p99_over_isolated": pct(0.99) / iso_med, "requests": len(lat),
                        "skipped_no_buffer": dropped[0]})
    st = srv.stats()
    srv.close()

    # plain sequential GPU path: each request as per-limb C-ABI calls, one after another
    import torch

    seq_n = min(len(rp.t), 16)
    dbuf = {}
    t0 = time.perf_counter()
    for k in range(seq_n):
        t = rp.t[k]
        n, L = t["n"], t["L"]
        x = t["x"].cuda(non_blocking=True)
        v = t["v"].cuda(non_blocking=True)
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
        dbuf[k] = y
    torch.cuda.synchronize()
    seq_rate = seq_n / (time.perf_counter() - t0)
    return {"workload": "INTT->MulMod/FMAMod->NTT requests, N in 2^13..2^17, L in 2..40, Poisson arrivals",
            "capacity_jobs_per_s": cap, "isolated_median_ms": iso_med, "loads": results,
            "plain_sequential_jobs_per_s": seq_rate, "batches": st["batches"],
            "max_batch_requests": st["max_batch_requests"], "peak_in_use_bytes": st["peak_in_use_bytes"],
            "budget_bytes": budget, "max_inflight": inflight}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["tensor", "uneven", "serve"])
    ap.add_argument("--seconds", type=float, default=4.0)
    a = ap.parse_args()
    if a.what == "tensor":
        out = tensor_chain()
    elif a.what == "uneven":
        out = uneven_batch()
    else:
        out = serving(seconds=a.seconds)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
