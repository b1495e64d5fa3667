#!/usr/bin/env python
"""Benchmark: batched NTT+INTT limb-transforms/s at N = 2^16.

Workload (one step, per GPU): 16 ciphertexts x 2 polynomials x 24 RNS limbs =
768 limbs of N = 65536 residues (50..59-bit primes q = 1 mod 2N from a
deterministic search; residues uniform in [0, q), seeded).  A step is the
reference's lazy round trip on every limb,
    ComputeForward(1, 4) -> EltwiseReduceMod(4, 2) -> ComputeInverse(2, 1),
run as two batched C-ABI calls (forward_batch, inverse_batch with the 4->2
reduce fused on load): 1536 limb-transforms.  Inputs (384 MiB) exceed the
126 MB L2, so no flush is needed between steps.

Prints one JSON line (rank 0).  `--impl reference` times the reference's own
CPU implementation (oracle/_ref, compiled from the reference sources) on the
same workload and metric.  Multi-GPU (torchrun): every rank runs its own 768
limbs (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 1 << 16
LIMBS = 24
CIPHERTEXTS = 16
POLYS = 2
COUNT = CIPHERTEXTS * POLYS * LIMBS  # 768 limbs per GPU
SEED = 0x415848454C
METRIC = "batched NTT+INTT limb-transforms/s at N=2^16"
UNIT = "limb-transforms/s"
HBM_FALLBACK = 6650.0
# Serving-loop configuration of the bench line per operand placement.  Host-
# staged requests: batches of whatever is queued, 4 in flight (their copies
# share the PCIe link).  Device-resident requests: one request per batch, 8 in
# flight, so a small request never waits inside a large one's batch.
SERVE_CONFIG = {
    "host_staged": dict(inflight=4, max_batch_requests=256),
    "device_resident": dict(inflight=8, max_batch_requests=1),
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK, "fallback"


def workload_moduli():
    from axhel_b200 import params

    return params.rns_moduli(N, LIMBS, 50, 59)


def workload_config(world):
    """The `config` object of both arms' JSON lines (the same workload)."""
    return {"workload": "batched RNS NTT+INTT round trip, N=2^16, 24 limbs x 16 ciphertexts x 2 polys "
                        "(768 limbs per GPU, 1536 limb-transforms per step)",
            "limbs_per_gpu": COUNT, "degree": N, "moduli": "24 primes of 50-59 bits",
            "l2": "inputs 384 MiB > 126 MB L2, no flush",
            "parallelism": f"{world} independent GPU(s), no data-path collective"}


def make_inputs(mods, count=COUNT, seed=SEED):
    rng = np.random.default_rng(seed)
    qs = np.array([q for q, _ in mods], dtype=np.uint64)
    out = np.empty((count, N), np.uint64)
    for i in range(count):
        out[i] = rng.integers(0, qs[i % len(qs)], N, dtype=np.uint64)
    return out


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """Samples SM clock and throttle reasons on one GPU (NVML) while running."""

    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
               0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}

    def __init__(self, index, period=0.01):
        self.index, self.period = index, period
        self.samples, self.reasons = [], set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def start(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)

            def run():
                while not self._stop.is_set():
                    try:
                        self.samples.append(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for bit, name in self.REASONS.items():
                            if r & bit and bit != 0x1:
                                self.reasons.add(name)
                    except Exception:
                        pass
                    time.sleep(self.period)

            self._t = threading.Thread(target=run, daemon=True)
            self._t.start()
        except Exception:
            self._t = None
        return self

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join()
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ distributed

def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ------------------------------------------------------------------ CPU reference

def reference_roundtrip_rate(mods, data, threads, target_s):
    """Times the reference native backend (oracle/_ref) on a bounded sample of
    the workload: the lazy round trip on S limbs over `threads` host threads,
    repeated to about `target_s` seconds.  Returns (limb-transforms/s, S,
    repeats, seconds, table-generation seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Reference

    ref = Reference()
    t = time.perf_counter()
    ntts = [ref.ntt(N, q, psi) for q, psi in mods]  # GenerateNTTTables, one host thread
    tables_s = time.perf_counter() - t
    S = min(len(data), max(threads, 4 * threads))
    buf = np.ascontiguousarray(data[:S])
    t = time.perf_counter()
    ref.roundtrip_batch(ntts, buf, N, S, threads)
    once = max(time.perf_counter() - t, 1e-4)
    reps = max(1, int(round(target_s / once)))
    t = time.perf_counter()
    for _ in range(reps):
        ref.roundtrip_batch(ntts, buf, N, S, threads)
    dt = time.perf_counter() - t
    if not np.array_equal(buf, data[:S]):
        raise RuntimeError("reference round trip did not reproduce its input")
    return 2 * S * reps / dt, S, reps, dt, tables_s


def run_reference(args):
    world, rank, local = dist_init()
    if rank != 0:
        return 0
    mods = workload_moduli()
    threads = len(os.sched_getaffinity(0))
    data = make_inputs(mods, COUNT)
    # size each step so the whole run stays within ~2 minutes
    budget = min(10.0, 120.0 / max(1, args.steps + args.warmup))
    rate = reference_roundtrip_rate(mods, data, threads, 1.0)[0]
    S = int(min(COUNT, max(threads, round(budget * rate / 2 / threads) * threads)))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from pyoracle import Reference

    ref = Reference()
    ntts = [ref.ntt(N, q, psi) for q, psi in mods]
    buf = np.ascontiguousarray(data[:S])
    for _ in range(args.warmup):
        ref.roundtrip_batch(ntts, buf, N, S, threads)
    t = time.perf_counter()
    for _ in range(args.steps):
        ref.roundtrip_batch(ntts, buf, N, S, threads)
    dt = time.perf_counter() - t
    value = 2 * S * args.steps / dt
    sample = (f"{S} of the {COUNT} limbs per step (N=2^16, 24 primes), lazy round trip per limb, "
              f"{threads} host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": workload_config(world),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm

def run_ours(args):
    import torch

    from axhel_b200 import capi

    world, rank, local = dist_init()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    mods = workload_moduli()
    torch.cuda.synchronize()
    # cold start: the 24 contexts' tables generated on the device in one launch
    t_tab = time.perf_counter()
    ntts = capi.NTT.create_many([(N, q, psi) for q, psi in mods])
    tables_ms = 1e3 * (time.perf_counter() - t_tab)
    data = make_inputs(mods, COUNT, SEED + rank)
    x = torch.from_numpy(data.reshape(-1).view(np.int64)).to(dev)
    y = torch.empty_like(x)
    xp, yp = x.data_ptr(), y.data_ptr()

    def step():
        capi.forward_batch(ntts, yp, xp, COUNT, 1, 4, sh)
        capi.inverse_batch(ntts, yp, yp, COUNT, 4, 1, sh)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if not torch.equal(x, y):
        raise RuntimeError("round trip mismatch before timing")
    if args.profile_step:
        # one more step and exit: the command line the ncu summaries are taken on
        step()
        torch.cuda.synchronize()
        print(json.dumps({"profile_step": "ok", "launches_per_step": 4}), flush=True)
        return 0

    # ---- timed region (device time, CUDA events on the launching stream)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local).start()
    l0 = capi.launch_count()
    capi.profile_enable(True)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    capi.profile_enable(False)
    launches = capi.launch_count() - l0
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    prof = capi.profile_report()
    if pg:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
        pg.barrier()
    if not torch.equal(x, y):
        raise RuntimeError("round trip mismatch after timing")
    value = world * 2 * COUNT * args.steps / (ms / 1e3)

    # ---- dominant kernel roofline (algorithmic bytes: each pass reads and
    # writes every limb once -> 16 * N * COUNT bytes per launch)
    peak, peak_kind = peaks()
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roofline = None
    if dom:
        name, (cnt, tot) = dom
        alg = 16 * N * COUNT
        avg_s = tot / cnt / 1e3
        achieved = alg / avg_s / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        if os.path.exists(tpath):
            with open(tpath) as f:
                traffic = json.load(f).get(name)
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                    "traffic": traffic, "kernel": name, "launches": cnt, "avg_launch_ms": tot / cnt,
                    "alg_bytes_per_launch": alg, "peak_source": f"{peak_kind} hbm_gbs",
                    "share": tot / sum(v[1] for v in prof.values())}
        # The binding roofline is the integer pipe: butterflies of the
        # reference algebra per second against the register-only probe.
        lg = int(name.split("lg=")[1].split()[0])
        bfly_launch = COUNT * (N // 2) * lg
        bpeak = max(capi.butterfly_peak(ntts[0], False, sh) for _ in range(3))
        step_bfly = 2 * COUNT * (N // 2) * 16
        int_roof = {"bound": "int_pipe", "achieved": bfly_launch / avg_s, "peak": bpeak, "unit": "butterflies/s",
                    "frac": bfly_launch / avg_s / bpeak, "kernel": name,
                    "step_frac": step_bfly / (ms / 1e3 / args.steps) / bpeak,
                    "peak_source": "measured: reference butterflies on registers over the full device "
                                   "(axhel_cuda_butterfly_peak)"}

    # ---- plain per-limb drop-in on the same device data (one call per limb
    # per operation, as the reference API is used), for the batching speed-up
    plain = plain_per_limb(capi, ntts, x, y, sh, limbs=min(COUNT, 768))

    # ---- e2e through the C-ABI with pinned host buffers, copies inside the timed region
    e2e = end_to_end(capi, ntts, data, dev, steps=max(1, min(args.steps, 10)))
    if pg:  # whole-job rate: every rank moves its own batch over its own link; slowest rank's time
        t = torch.tensor([e2e["ms_per_step"]], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e["ms_per_step"] = float(t.item())
        e2e["value"] = world * 2 * COUNT / (e2e["ms_per_step"] / 1e3)
        e2e["h2d_bytes_per_step"] *= world
        e2e["d2h_bytes_per_step"] *= world

    # ---- the other configurations' workloads, once each, outside the timed
    # region: the fused tensor product (C3) and the 512-polynomial uneven
    # batch (C4).  `same_bits` compares every output word with the oracle's
    # results, through the SHA-256 digests committed beside the test
    # fixtures (tests/golden/config_digests.json, made by the oracle and
    # checked there against the reference); `same_as_per_limb_calls` with the
    # GPU's own per-limb call sequence.
    others = None
    if rank == 0 and not args.no_others:
        from axhel_b200 import workloads

        want = oracle_digests()
        t = workloads.tensor_chain(keep=True)
        t_ok = None
        if want:
            t_ok = [digest_of(r) for r in t.pop("results")] == want["tensor"]["r_sha256"]
        t.pop("results", None)
        u = workloads.uneven_batch(keep=True)
        u_ok = None
        if want:
            u_ok = all(digest_of(j["y"]) == w["sha256"] for j, w in zip(u["jobs"], want["uneven"]["jobs"]))
        u.pop("jobs", None)
        torch.cuda.empty_cache()
        pr = workloads.product_chain()
        others = {
            "tensor_product": {"workload": t["workload"], "ms": t["fused_ms"], "GBps": t["fused_GBps"],
                               "per_limb_calls_ms": t["per_limb_calls_ms"], "speedup": t["speedup"],
                               "same_bits": t_ok, "same_as_per_limb_calls": t["same_bits"]},
            "uneven_batch": {"workload": u["workload"], "limb_transforms": u["limb_transforms"],
                             "persistent_rate": u["one_launch_rate"], "phased_rate": u["phased_rate"],
                             "per_limb_rate": u["per_limb_rate"], "unit": u["unit"], "same_bits": u_ok,
                             "same_as_per_limb_calls": u["same_bits"]},
            "ntt_mulmod_intt": {"workload": pr["workload"], "fused_ms": pr["fused_ms"],
                                "separate_calls_ms": pr["separate_calls_ms"], "speedup": pr["speedup"],
                                "fused_rate": pr["fused_rate"], "unit": pr["unit"],
                                "same_as_separate_calls": pr["same_bits"]},
            "headline": headline_digest_check(capi, ntts, xp, y, sh, want),
            "same_bits_means": "every output word equal to the oracle's (SHA-256 against "
                               "tests/golden/config_digests.json)",
        }

    # ---- serving loop (continuous batching): Poisson arrivals at 50, 70 and
    # 90 % of its measured capacity, host-staged requests (copies in the
    # loop) and device-resident ones; latency against each request's
    # isolated latency two ways: p99 over the isolated p99, and the p99 of
    # per-request slowdowns
    serve = None
    if rank == 0 and not args.no_serve:
        from axhel_b200 import workloads

        serve = {}
        for mode, device in (("host_staged", False), ("device_resident", True)):
            r = workloads.serving(loads=(0.5, 0.7, 0.9), seconds=3.0, n_templates=24, device=device, plain=True,
                                  **SERVE_CONFIG[mode])
            m = {"capacity_jobs_per_s": r["capacity_jobs_per_s"], "isolated_median_ms": r["isolated_median_ms"],
                 "plain_sequential_jobs_per_s": r["plain_sequential_jobs_per_s"], "policy": r["policy"],
                 "config": {k: r[k] for k in ("max_inflight", "max_batch_requests_cfg", "small_request_words")}}
            for l in r["loads"]:
                m[f"load_{int(round(100 * l['load']))}"] = {
                    k: l[k] for k in ("jobs_per_s", "p50_ms", "p99_ms", "isolated_p99_ms", "p99_over_isolated_p99",
                                      "p50_slowdown", "p99_slowdown", "p99_queue_ms", "p99_large_ms", "p99_rest_ms",
                                      "requests")}
            l70 = m["load_70"]
            m.update({"jobs_per_s_at_70pct": l70["jobs_per_s"], "p50_ms": l70["p50_ms"], "p99_ms": l70["p99_ms"],
                      "isolated_p99_ms": l70["isolated_p99_ms"], "p99_over_isolated_p99": l70["p99_over_isolated_p99"],
                      "p99_slowdown": l70["p99_slowdown"]})
            serve[mode] = m
        serve["workload"] = ("INTT->MulMod/FMAMod->NTT requests, N in 2^13..2^17, L in 2..40, 24 templates, "
                             "Poisson arrivals at 50/70/90 % of capacity, HBM budget 60 GB; headline figures at 70 %")

    dropin = None
    if rank == 0 and not args.no_dropin:
        try:
            dropin = dropin_host(with_reference=world == 1 and not args.no_cpu)
        except Exception as e:  # the timer is a separate program; report why it did not run
            dropin = {"unavailable": str(e)[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            threads = len(os.sched_getaffinity(0))
            rate, S, reps, secs, tables_s = reference_roundtrip_rate(mods, data, threads, args.cpu_seconds)
            cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"{S} limbs of the N=2^16 workload x {reps} repeats, lazy round trip "
                             f"(forward, ReduceMod 4->2, inverse), {secs:.1f} s",
                   "tables_ms": 1e3 * tables_s}
            # the same on one host thread (the library itself is single-threaded)
            r1, S1, reps1, secs1, _ = reference_roundtrip_rate(mods, data, 1, min(args.cpu_seconds, 3.0))
            cpu["single_thread"] = {"value": r1, "unit": UNIT, "cores": 1,
                                    "sample": f"{S1} limbs x {reps1} repeats, {secs1:.1f} s"}
        except Exception as e:  # the reference build is test infrastructure; report its absence
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": workload_config(world),
            "gpu_launches": launches,
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "roofline": roofline,
            "int_roofline": int_roof if dom else None,
            "plain_per_limb": plain,
            "e2e": e2e,
            "serve": serve,
            "configs": others,
            "dropin_host": dropin,
            "tables": {"contexts": len(mods), "degree": N, "device_ms": tables_ms,
                       "reference_cpu_ms": cpu["tables_ms"] if cpu and "tables_ms" in cpu else None,
                       "note": "cold start: twiddle tables of the 24 moduli, device generation (one launch, "
                               "wall clock incl. allocation) vs the reference's GenerateNTTTables on one host "
                               "thread"},
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()
    return 0


def oracle_digests():
    """The committed SHA-256 digests of the configurations' oracle outputs
    (None when the fixture file is absent)."""
    path = os.path.join(ROOT, "tests", "golden", "config_digests.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


def digest_of(t):
    """SHA-256 of a device tensor's words (uint64 little-endian)."""
    import hashlib

    a = t.detach().cpu().numpy().view(np.uint64)
    return hashlib.sha256(np.ascontiguousarray(a).astype("<u8", copy=False).tobytes()).hexdigest()


def headline_digest_check(capi, ntts, xp, y, sh, want):
    """One more step outside the timed region: the forward outputs (lazy,
    [0, 4q)) and the round trip against the oracle's digests."""
    import torch

    capi.forward_batch(ntts, y.data_ptr(), xp, COUNT, 1, 4, sh)
    torch.cuda.synchronize()
    f = digest_of(y)
    capi.inverse_batch(ntts, y.data_ptr(), y.data_ptr(), COUNT, 4, 1, sh)
    torch.cuda.synchronize()
    b = digest_of(y)
    if not want:
        return {"same_bits": None}
    return {"same_bits": f == want["headline"]["forward_lazy_sha256"] and b == want["headline"]["round_trip_sha256"],
            "checked": "forward lazy outputs and round-trip outputs of all 768 limbs"}


def dropin_cases():
    """(logn, q, psi) per degree 2^12..2^17: a 50-bit NTT prime of each."""
    from axhel_b200 import params

    out = []
    for logn in range(12, 18):
        n = 1 << logn
        q = params.ntt_prime_near(n, 50, 1, 4)
        out.append((logn, q, params.primitive_root(n, q)))
    return out


def dropin_timer(exe, threads, seconds, cases):
    """Runs a build of axhel_b200/tools/dropin_bench.cpp: {(op, logn): us per call}."""
    args = [exe, str(threads), str(seconds)] + [f"{l}:{q}:{p}" for l, q, p in cases]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} failed: {r.stderr[-400:]}")
    out = {}
    for line in r.stdout.splitlines():
        d = json.loads(line)
        out[(d["op"], d["logn"])] = d
    return out


def dropin_host(with_reference, threads_list=(1, 8), seconds=0.2):
    """SEAL's call pattern through the C++ drop-in: host (pageable) pointers,
    one limb per call, in place, threads sharing one cached NTT object --
    ComputeForward(p,p,4,4), ComputeInverse(p,p,2,1), EltwiseMulMod(p,p,b,N,q,4)
    and the N-point plain round trip (two forwards, MulMod, AddMod with a
    scalar, inverse) -- against the same program linked to the reference
    native backend (oracle/_ref/dropin_bench_ref).  Mean microseconds per call
    seen by a thread; the crossover is the smallest degree from which the GPU
    call is faster than the reference's."""
    cases = dropin_cases()
    ours_exe = os.path.join(ROOT, "axhel_b200", "dropin_bench")
    ref_exe = os.path.join(ROOT, "oracle", "_ref", "dropin_bench_ref")
    out = {"unit": "us per call (mean per thread)", "pattern": "host pageable buffers, one limb per call, in place, "
           "threads share one const NTT per degree; 50-bit primes", "rows": []}
    crossover = {}
    for threads in threads_list:
        ours = dropin_timer(ours_exe, threads, seconds, cases)
        ref = dropin_timer(ref_exe, threads, seconds, cases) if with_reference and os.path.exists(ref_exe) else {}
        for (op, logn), d in sorted(ours.items(), key=lambda kv: (kv[0][0], kv[0][1])):
            row = {"op": op, "logn": logn, "threads": threads, "us": d["us_per_call"],
                   "calls_per_s": d["calls_per_s"]}
            if op.startswith("rns24") and ("forward_4_4", logn) in ref:
                # the reference's cost of the same polynomial: 24 per-limb calls
                r = ref[("forward_4_4", logn)]
                row.update({"reference_us": 24 * r["us_per_call"],
                            "speedup": 24 * r["us_per_call"] / d["us_per_call"]})
            elif (op, logn) in ref:
                r = ref[(op, logn)]
                row.update({"reference_us": r["us_per_call"], "reference_calls_per_s": r["calls_per_s"],
                            "speedup": r["us_per_call"] / d["us_per_call"]})
            if "speedup" in row:
                key = f"{op}@{threads}t"
                if row["speedup"] > 1 and key not in crossover:
                    crossover[key] = 1 << logn
            out["rows"].append(row)
    out["crossover_degree"] = crossover
    return out


def plain_per_limb(capi, ntts, x, y, sh, limbs):
    """The reference's call pattern on the GPU drop-in: for each limb,
    ComputeForward(1,4), EltwiseReduceMod(4,2), ComputeInverse(2,1) as three
    separate C-ABI calls on device-resident data -- issued eagerly, and
    replayed from a CUDA graph (no host launch cost)."""
    import torch

    L = len(ntts)

    def run(stream_handle):
        for i in range(limbs):
            off = 8 * N * i
            t = ntts[i % L]
            t.forward(y.data_ptr() + off, x.data_ptr() + off, 1, 4, stream_handle)
            capi.reduce(y.data_ptr() + off, y.data_ptr() + off, N, t.modulus, 4, 2, stream_handle)
            t.inverse(y.data_ptr() + off, y.data_ptr() + off, 2, 1, stream_handle)

    s = torch.cuda.current_stream()
    run(s.cuda_stream)
    torch.cuda.synchronize()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    ms = timed(lambda: run(s.cuda_stream))
    y.zero_()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        run(torch.cuda.current_stream().cuda_stream)
    g.replay()
    torch.cuda.synchronize()
    ms_graph = timed(g.replay)
    ok = torch.equal(x[: limbs * N], y[: limbs * N])
    del g
    return {"value": 2 * limbs / (ms / 1e3), "unit": UNIT, "limbs": limbs, "ms": ms, "calls_per_limb": 3,
            "graph_value": 2 * limbs / (ms_graph / 1e3), "graph_ms": ms_graph, "bitexact_roundtrip": ok}


def end_to_end(capi, ntts, data, dev, steps, chunks=8):
    """Same metric through the C-ABI from pinned HOST memory: per step, every
    chunk of limbs is copied host->device, transformed (forward, inverse) and
    copied back, pipelined over 3 streams; steps follow each other without a
    barrier, as a stream of batches would.  Timed with CUDA events.  The bound
    is PCIe: a step moves 384 MiB each way."""
    import torch

    flat = data.reshape(-1)
    hin = torch.from_numpy(flat.view(np.int64)).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    dbuf = torch.empty(hin.numel(), dtype=torch.int64, device=dev)
    per = COUNT // chunks
    assert per % LIMBS == 0
    streams = [torch.cuda.Stream(dev) for _ in range(3)]
    main = torch.cuda.current_stream(dev)

    def one_step():
        for c in range(chunks):
            s = streams[c % len(streams)]
            lo, hi = c * per * N, (c + 1) * per * N
            with torch.cuda.stream(s):
                dbuf[lo:hi].copy_(hin[lo:hi], non_blocking=True)
                p = dbuf.data_ptr() + 8 * lo
                capi.forward_batch(ntts, p, p, per, 1, 4, s.cuda_stream)
                capi.inverse_batch(ntts, p, p, per, 4, 1, s.cuda_stream)
                hout[lo:hi].copy_(dbuf[lo:hi], non_blocking=True)

    for s in streams:
        s.wait_stream(main)
    one_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(main)
    for s in streams:
        s.wait_stream(main)
    for _ in range(steps):
        one_step()
    for s in streams:
        main.wait_stream(s)
    e1.record(main)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ok = torch.equal(hin, hout)
    nbytes = flat.nbytes
    return {"value": 2 * COUNT * steps / (ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "ms_per_step": ms / steps, "bitexact_roundtrip": ok,
            "pipeline": f"{chunks} chunks over 3 streams, steps back to back"}


def run_kernel_table(args):
    """The per-kernel comparison table: every public kernel over the reference
    benchmark's scenario matrix (degrees 2048..32768 x widths 20..62), timed
    on the GPU by axhel_b200.harness (device time per call) and, as the CPU
    baseline, the reference native backend (oracle/_ref/kernel_timer_ref,
    wall time per call on one host thread); both summaries in the reference's
    summary.csv columns, joined into speedup.csv, plus a markdown digest."""
    from pathlib import Path

    import torch

    from axhel_b200 import harness, params

    out = Path(args.kernel_table)
    out.mkdir(parents=True, exist_ok=True)
    reps, warm = 30, 5
    torch.cuda.set_device(0)
    harness.main(["run", "--output", str(out / "b200"), "--repetitions", str(reps), "--warmup", str(warm),
                  "--no-raw"])
    exe = os.path.join(ROOT, "oracle", "_ref", "kernel_timer_ref")
    cases = []
    for d in harness.DEGREES:
        for b in harness.BITS:
            q = harness.largest_ntt_prime(d, b)
            cases.append(f"{d}:{b}:{q}:{params.primitive_root(d, q)}")
    r = subprocess.run([exe, str(reps), str(warm), "1"] + cases, capture_output=True, text=True, timeout=1800)
    if r.returncode != 0:
        raise RuntimeError(f"kernel_timer_ref failed: {r.stderr[-400:]}")
    (out / "reference").mkdir(exist_ok=True)
    recs = [json.loads(l) for l in r.stdout.splitlines() if l.strip()]
    harness.write_summary(out / "reference" / "summary.csv", recs, "reference-native-1thread")
    harness.main(["compare", str(out / "reference" / "summary.csv"), str(out / "b200" / "summary.csv"),
                  str(out / "speedup.csv"), "--cpu-unit", "ns"])
    table = harness.speedup_table(out / "speedup.csv")
    (out / "speedup.md").write_text(table + "\n")
    print(table, flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample length")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-others", action="store_true", help="skip the tensor-product and uneven-batch workloads")
    ap.add_argument("--no-dropin", action="store_true", help="skip the C++ drop-in per-call timings")
    ap.add_argument("--profile-step", action="store_true",
                    help="warm up, run one step and exit (the command profiled by ncu)")
    ap.add_argument("--kernel-table", metavar="DIR", default=None,
                    help="write the per-kernel GPU vs reference table (summary.csv both sides, speedup.csv) to DIR "
                         "and exit")
    args = ap.parse_args()
    if args.kernel_table:
        return run_kernel_table(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
