"""Autotuner for the NTT pass plans and the uneven-batch engine's split.

For each direction, degree N = 2^logn and limb-count bucket, times every
candidate split of the log2 N stages into passes (1 or 2 passes), register
depth LR in {3, 4, 5} and tile width TG on the GPU (CUDA events, median of
several launches of the batched C-ABI call) and writes the fastest to
``axhel_b200/ntt_plans.txt``, which the library loads at first use:

    <inverse> <logn> <limb-bucket> <npass> (<lg> <lr> <tg>)...

limb-bucket = floor(log2(limbs)).  For the uneven-batch engine (fixed
1024-residue tiles) it times, per degree, every split of a job's stages into
its strided and contiguous passes on a batch of forward, inverse and chained
jobs, and writes

    B <logn> <contiguous-pass stages>

For the one-launch cluster form of small calls (transforms, fused chains and
products of a few limbs) it times every compiled (lga, lr, csize) on one
limb and the limb counts up to which the fastest beats the pass form:

    K <kind> <logn> <lga> <lr> <csize> <max-limbs>

Every candidate computes the same bits (tests/test_ntt_gpu.py::
test_every_plan_bitexact, tests/test_batch_gpu.py), so the choice only
affects speed.

    python -m axhel_b200.autotune [--what all|passes|batch|cluster] [--logn 12-17] [--buckets 0,3,6,9]
"""
from __future__ import annotations

import argparse
import os
import statistics
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "ntt_plans.txt")


def candidates(logn, inverse):
    out = []
    if logn <= 13:
        for lr in (3, 4, 5):
            if lr <= logn and (1 << (logn - lr)) <= (256 if lr >= 5 else 512):
                out.append([(logn, lr, 1)])
    if logn >= 6:
        for a in range(3, min(13, logn - 3) + 1):  # a = strided column pass
            b = logn - a
            if b > 13 or b < 3:
                continue
            for lra in (3, 4, 5):
                for lrb in (3, 4, 5):
                    if lra > a or lrb > b:
                        continue
                    for tga in (4, 8, 16, 32):
                        for tgb in (1, 2, 4, 8, 16, 32):
                            col = (a, lra, tga)
                            row = (b, lrb, tgb)
                            if tga > (1 << b) or tgb > (1 << a):
                                continue
                            if (tga << (a - lra)) > (256 if lra >= 5 else 512):
                                continue
                            if (tgb << (b - lrb)) > (256 if lrb >= 5 else 512):
                                continue
                            if (tga << (a - lra)) < 64 or (tgb << (b - lrb)) < 64:
                                continue
                            out.append([row, col] if inverse else [col, row])
    return out


def time_plan(capi, torch, ntts, x, y, count, inverse, reps=5):
    if inverse:
        fn = lambda: capi.inverse_batch(ntts, y.data_ptr(), x.data_ptr(), count, 2, 2)
    else:
        fn = lambda: capi.forward_batch(ntts, y.data_ptr(), x.data_ptr(), count, 4, 4)
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def tune(lognums, buckets, limbs_cap_bytes=1 << 30, verbose=True):
    import torch

    from axhel_b200 import capi, params

    lines = []
    for logn in lognums:
        n = 1 << logn
        mods = params.rns_moduli(n, 8, 50, 59)
        ntts = [capi.NTT(n, q, psi) for q, psi in mods]
        for bucket in buckets:
            count = 1 << bucket
            if count * n * 8 > limbs_cap_bytes:
                count = max(1, limbs_cap_bytes // (n * 8))
            rng = np.random.default_rng(logn * 100 + bucket)
            data = np.concatenate([rng.integers(0, mods[i % 8][0], n, dtype=np.uint64) for i in range(count)])
            x = torch.from_numpy(data.view(np.int64)).cuda()
            y = torch.empty_like(x)
            for inverse in (False, True):
                best = None
                for plan in candidates(logn, inverse):
                    try:
                        capi.plan_set(inverse, logn, plan)
                    except capi.AxhelError:
                        continue
                    ms = time_plan(capi, torch, ntts, x, y, count, inverse)
                    if best is None or ms < best[0]:
                        best = (ms, plan)
                capi.plan_set(inverse, logn, [])
                if best is None:
                    continue
                ms, plan = best
                flat = " ".join(f"{lg} {lr} {tg}" for lg, lr, tg in plan)
                lines.append(f"{int(inverse)} {logn} {bucket} {len(plan)} {flat}")
                if verbose:
                    rate = count / (ms / 1e3)
                    print(f"inv={int(inverse)} logn={logn} limbs={count}: {plan} {ms:.4f} ms "
                          f"({rate:,.0f} limb-transforms/s)", flush=True)
    return lines


def tune_batch(lognums, bytes_per_job=128 << 20, reps=5, verbose=True):
    """Per degree, the batch engine's contiguous-pass width that runs a
    forward, an inverse and a chained job of ~128 MiB each fastest: the sum
    of the persistent launch's and the per-phase launches' times (one split
    serves both forms)."""
    import torch

    from axhel_b200 import capi, params

    lines = []
    for logn in lognums:
        if not 10 <= logn <= 17:
            continue
        n = 1 << logn
        mods = params.rns_moduli(n, 8, 50, 59)
        ntts = [capi.NTT(n, q, psi) for q, psi in mods]
        count = max(8, bytes_per_job // (n * 8)) // 8 * 8
        rng = np.random.default_rng(logn)
        data = np.concatenate([rng.integers(0, mods[i % 8][0], n, dtype=np.uint64) for i in range(count)])
        bufs = [torch.from_numpy(data.view(np.int64)).cuda() for _ in range(4)]
        outs = [torch.empty_like(bufs[0]) for _ in range(3)]
        specs = [dict(kind=capi.JOB_FORWARD, ntts=ntts, count=count, result=outs[0].data_ptr(),
                      operand=bufs[0].data_ptr(), in_f=1, out_f=4),
                 dict(kind=capi.JOB_INVERSE, ntts=ntts, count=count, result=outs[1].data_ptr(),
                      operand=bufs[1].data_ptr(), in_f=2, out_f=1),
                 dict(kind=capi.JOB_CHAIN_MUL, ntts=ntts, count=count, result=outs[2].data_ptr(),
                      operand=bufs[2].data_ptr(), vector=bufs[3].data_ptr(), in_f=2, out_f=4)]
        best = None
        for row in range(max(5, logn - 9), min(9, logn - 5) + 1):
            capi.batch_split_set(logn, row)
            b = capi.Batch(specs)
            form_ms = []
            for phased in (False, True):
                b.launch(phased=phased)
                torch.cuda.synchronize()
                ts = []
                for _ in range(reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    b.launch(phased=phased)
                    e1.record()
                    torch.cuda.synchronize()
                    ts.append(e0.elapsed_time(e1))
                form_ms.append(statistics.median(ts))
            b.close()
            ms = sum(form_ms)
            if verbose:
                print(f"batch logn={logn} row={row}: persistent {form_ms[0]:.3f} ms, per phase {form_ms[1]:.3f} ms",
                      flush=True)
            if best is None or ms < best[0]:
                best = (ms, row)
        capi.batch_split_set(logn, 0)
        lines.append(f"B {logn} {best[1]}")
    return lines


def graph_time_us(torch, call, reps=30):
    """Device time per call: `reps` calls captured in a CUDA graph, best of 5
    replays (no host launch cost: what a small latency-bound call costs)."""
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
    return best


def tune_cluster(lognums, counts=(1, 2, 4, 8, 16, 32, 64), verbose=True):
    """The one-launch cluster form of small calls (forward, inverse, the
    INTT -> MulMod -> NTT chain, the NTT -> MulMod -> INTT product): per kind
    and degree the fastest compiled (lga, lr, csize) on one limb, and the
    largest limb count up to which it beats the pass form (0: never)."""
    import torch

    from axhel_b200 import capi, params

    names = {capi.CLUSTER_FORWARD: "forward", capi.CLUSTER_INVERSE: "inverse", capi.CLUSTER_CHAIN: "chain",
             capi.CLUSTER_PRODUCT: "product"}
    lines = []
    for logn in lognums:
        n = 1 << logn
        mods = params.rns_moduli(n, 4, 50, 59)
        ntts = [capi.NTT(n, q, psi) for q, psi in mods]
        cmax = max(counts)
        x = torch.randint(0, 1 << 40, (cmax * n,), dtype=torch.int64, device="cuda")
        y = torch.empty_like(x)
        m = torch.randint(0, 1 << 40, (cmax * n,), dtype=torch.int64, device="cuda")

        def caller(kind, count):
            xp, yp, mp = x.data_ptr(), y.data_ptr(), m.data_ptr()
            if kind == capi.CLUSTER_FORWARD:
                return lambda st: capi.forward_batch(ntts, yp, xp, count, 4, 4, st)
            if kind == capi.CLUSTER_INVERSE:
                return lambda st: capi.inverse_batch(ntts, yp, xp, count, 2, 2, st)
            if kind == capi.CLUSTER_CHAIN:
                return lambda st: capi.chain_mul_batch(ntts, yp, xp, mp, count, 2, 4, st)
            return lambda st: capi.product_batch(ntts, yp, xp, mp, count, 4, 1, st)

        for kind in names:
            # every compiled shape, timed on 1, 4, 16 and 64 limbs; the one with
            # the smallest summed time relative to the fastest shape at each
            # count (the best on one limb alone can be 20-35 % slower on 16)
            obj = (1, 4, 16, 64)
            timed = {}
            for lga in range(5, 10):
                for lr in (2, 3, 4):
                    for cs in (2, 4, 8, 16):
                        try:
                            capi.cluster_plan_set(kind, logn, lga, lr, cs, cmax)
                            timed[(lga, lr, cs)] = [graph_time_us(torch, caller(kind, c)) for c in obj]
                        except (capi.AxhelError, RuntimeError):
                            continue  # not compiled, or not schedulable on this GPU
            if not timed:
                capi.cluster_plan_set(kind, logn)
                continue
            fastest = [min(t[i] for t in timed.values()) for i in range(len(obj))]
            lga, lr, cs = min(timed, key=lambda c: sum(timed[c][i] / fastest[i] for i in range(len(obj))))
            best = (timed[(lga, lr, cs)][0],)
            max_limbs = 0
            for count in counts:
                capi.cluster_plan_set(kind, logn, lga, lr, cs, cmax)
                t_cluster = graph_time_us(torch, caller(kind, count))
                capi.cluster_plan_set(kind, logn, lga, lr, cs, 0)
                t_passes = graph_time_us(torch, caller(kind, count))
                if t_cluster >= t_passes:
                    break
                max_limbs = count
            capi.cluster_plan_set(kind, logn)
            lines.append(f"K {kind} {logn} {lga} {lr} {cs} {max_limbs}")
            if verbose:
                print(f"{names[kind]} logn={logn}: lga={lga} lr={lr} csize={cs}, one limb {best[0]:.2f} us, "
                      f"cluster form up to {max_limbs} limbs", flush=True)
    return lines


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--what", choices=["all", "passes", "batch", "cluster"], default="all")
    ap.add_argument("--logn", default="12-17")
    ap.add_argument("--buckets", default="0,3,5,7,9")
    ap.add_argument("--out", default=TABLE)
    a = ap.parse_args()
    lo, _, hi = a.logn.partition("-")
    lognums = list(range(int(lo), int(hi or lo) + 1))
    buckets = [int(b) for b in a.buckets.split(",")]
    t = time.time()
    old = []
    if os.path.exists(a.out):
        with open(a.out) as f:
            old = [l.rstrip("\n") for l in f if l.strip() and not l.startswith("#")]
    # lines of the parts not re-tuned are kept
    def part(line):
        return "batch" if line.startswith("B") else "cluster" if line.startswith("K") else "passes"

    keep = [l for l in old if a.what != "all" and part(l) != a.what]
    lines = []
    if a.what in ("all", "passes"):
        lines += tune(lognums, buckets)
    if a.what in ("all", "batch"):
        lines += tune_batch(list(range(10, 18)) if a.what == "all" else lognums)
    if a.what in ("all", "cluster"):
        lines += tune_cluster(list(range(10, 18)) if a.what == "all" else lognums)
    merged = sorted(keep + lines, key=lambda l: ({"passes": 0, "batch": 1, "cluster": 2}[part(l)], l))
    with open(a.out, "w") as f:
        f.write("# NTT pass plans chosen by axhel_b200/autotune.py on one B200\n")
        f.write("# inverse logn limb-bucket npass (lg lr tg)...  |  B logn contiguous-pass-stages (batch engine)\n")
        f.write("# K kind logn lga lr csize max-limbs (cluster form: 0 forward, 1 inverse, 2 chain, 3 product)\n")
        f.write("\n".join(merged) + "\n")
    print(f"wrote {a.out} ({len(lines)} lines tuned, {len(keep)} kept, {time.time() - t:.0f} s)")


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(HERE))
    main()
