"""Per-kernel benchmark of the GPU library in the reference harness's format.

The reference's benchmark (benchmark/src/axhel_benchmark.cpp) times every
public kernel over a matrix of degrees x modulus widths, filters each
scenario's samples with Tukey's IQR fences and writes ``summary.csv``
(axhel_benchmark.cpp:976-1024); ``compare_results.py`` joins the summaries
of several backends into a speed-up table.  This module does the same for
this library on one GPU, with the same scenario matrix (degrees
2048..32768, widths 20..62; axhel_benchmark.cpp:48-50), kernel names
(add_vv ... ntt_inverse_lazy; :1047-1166), moduli (the largest prime
q = 1 mod 2N below 2^bits and its smallest-generator root; :683-722),
statistics (linear quantiles, fences Q1 - 1.5 IQR / Q3 + 1.5 IQR; :741-794)
and columns, so that its summary sits beside a CPU summary row for row:

    python -m axhel_b200.harness run --output results/b200
    python -m axhel_b200.harness compare cpu/summary.csv results/b200/summary.csv \\
        speedup.csv --cpu-ghz 2.7

Each sample is ``--batch`` consecutive calls on device-resident operands
through the C-ABI, bracketed by CUDA events on the launching stream, queued
while a short device-side sleep holds the GPU (so the events measure device
time, not the host's call latency); the "cycles" columns hold NANOSECONDS
per call (metadata.txt says so).  The
compare step converts the CPU summary's cycles with ``--cpu-ghz``.  NTT
samples transform in place (table generation outside the timed region, as
in the reference); element-wise samples write a separate result.
"""
from __future__ import annotations

import argparse
import csv
import math
import os
import platform
import time
from pathlib import Path

import numpy as np

from . import capi, params

DEGREES = [2048, 4096, 8192, 16384, 32768]
BITS = [20, 25, 30, 40, 50, 52, 54, 56, 58, 60, 61, 62]
KERNELS = ["add_vv", "sub_vv", "add_vs", "sub_vs", "mul_f1", "mul_f2", "mul_f4", "fma_f1", "fma_f2", "fma_f4",
           "fma_f8", "reduce_2to1", "reduce_4to1", "reduce_4to2", "reduce_barrett", "ntt_forward",
           "ntt_forward_lazy", "ntt_inverse", "ntt_inverse_lazy"]
KEYS = ["kernel", "poly_degree", "qi_bits", "modulus", "mod_factor", "input_mod_factor", "output_mod_factor"]
METRICS = ["samples_total", "samples_kept", "outliers_removed", "raw_min_cycles", "raw_max_cycles", "q1_cycles",
           "q3_cycles", "iqr_cycles", "lower_fence_cycles", "upper_fence_cycles", "min_cycles", "max_cycles",
           "mean_cycles", "median_cycles", "stddev_cycles", "cv_percent", "mean_cycles_per_coeff",
           "median_cycles_per_coeff", "perf_scaled"]
BACKEND = "B200"


def largest_ntt_prime(degree, bits):
    """The largest prime q = 1 mod 2*degree below 2^bits."""
    return params.ntt_prime_near(degree, bits, 1, 1)


def quantile_sorted(v, p):
    if len(v) == 1:
        return v[0]
    pos = p * (len(v) - 1)
    lo, hi = math.floor(pos), math.ceil(pos)
    return v[lo] + (pos - lo) * (v[hi] - v[lo])


def statistics(samples):
    """Tukey-filtered statistics of one scenario's per-call times."""
    v = sorted(samples)
    q1, q3 = quantile_sorted(v, 0.25), quantile_sorted(v, 0.75)
    iqr = q3 - q1
    lo, hi = q1 - 1.5 * iqr, q3 + 1.5 * iqr
    kept = [x for x in v if lo <= x <= hi]
    mean = sum(kept) / len(kept)
    sd = math.sqrt(sum((x - mean) ** 2 for x in kept) / (len(kept) - 1)) if len(kept) > 1 else 0.0
    return dict(samples_total=len(v), samples_kept=len(kept), outliers_removed=len(v) - len(kept),
                raw_min=v[0], raw_max=v[-1], q1=q1, q3=q3, iqr=iqr, lower_fence=lo, upper_fence=hi, min=kept[0],
                max=kept[-1], mean=mean, median=quantile_sorted(kept, 0.5), stddev=sd,
                cv_percent=100.0 * sd / mean if mean else 0.0)


def _uniform(rng, n, bound):
    """n residues uniform in [0, bound) (bound <= 2^64)."""
    if bound >= 1 << 64:
        return rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    return rng.integers(0, bound, n, dtype=np.uint64)


class Runner:
    def __init__(self, repetitions, warmup, batch, write_raw, out_dir, seed):
        import torch

        self.torch = torch
        self.rep, self.warm, self.batch = repetitions, warmup, batch
        self.sleep_cycles = int(2000 * (50 + 20 * batch))  # 2000 cycles/us: ~50 us + 20 us per queued call
        self.seed = seed
        self.stream = torch.cuda.current_stream().cuda_stream
        self.summary = open(out_dir / "summary.csv", "w", newline="")
        self.sw = csv.writer(self.summary)
        self.sw.writerow(["backend"] + KEYS + METRICS)
        self.raw = None
        if write_raw:
            self.raw = open(out_dir / "raw_samples.csv", "w", newline="")
            self.rw = csv.writer(self.raw)
            self.rw.writerow(["backend"] + KEYS + ["repetition", "batch", "raw_ns", "ns"])

    def dev(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()

    def measure(self, call):
        torch = self.torch
        for _ in range(self.warm):
            call()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(self.rep)]
        for a, b in ev:
            # keep the GPU busy while the host queues the sample, so the
            # events bracket device time only, not the host's call latency
            torch.cuda._sleep(self.sleep_cycles)
            a.record()
            for _ in range(self.batch):
                call()
            b.record()
            torch.cuda.synchronize()
        return [1e6 * a.elapsed_time(b) for a, b in ev]  # ns per sample (batch calls)

    def report(self, name, degree, bits, q, mod_f, in_f, out_f, raw_ns):
        per_call = [x / self.batch for x in raw_ns]
        st = statistics(per_call)
        key = [name, degree, bits, q, mod_f, in_f, out_f]
        if self.raw:
            for i, (r, c) in enumerate(zip(raw_ns, per_call)):
                self.rw.writerow([BACKEND] + key + [i, self.batch, f"{r:.3f}", f"{c:.3f}"])
        f3 = lambda x: f"{x:.3f}"
        self.sw.writerow([BACKEND] + key + [
            st["samples_total"], st["samples_kept"], st["outliers_removed"], f3(st["raw_min"]), f3(st["raw_max"]),
            f3(st["q1"]), f3(st["q3"]), f3(st["iqr"]), f3(st["lower_fence"]), f3(st["upper_fence"]), f3(st["min"]),
            f3(st["max"]), f3(st["mean"]), f3(st["median"]), f3(st["stddev"]), f3(st["cv_percent"]),
            f3(st["mean"] / degree), f3(st["median"] / degree), 0])
        self.summary.flush()
        return st

    def scenario(self, degree, bits, kernels):
        q = largest_ntt_prime(degree, bits)
        root = params.primitive_root(degree, q)
        n, s = degree, self.stream
        rng = np.random.default_rng([self.seed, degree, bits])
        res = self.dev(np.zeros(n, np.uint64))
        r = res.data_ptr()
        out = []

        def run(name, call, mod_f=0, in_f=0, out_f=0):
            if name in kernels:
                st = self.report(name, degree, bits, q, mod_f, in_f, out_f, self.measure(call))
                out.append((name, st["median"]))

        a1, b1 = self.dev(_uniform(rng, n, q)), self.dev(_uniform(rng, n, q))
        pa, pb = a1.data_ptr(), b1.data_ptr()
        sc = int(_uniform(rng, 1, q)[0])
        run("add_vv", lambda: capi.add(r, pa, pb, n, q, s))
        run("sub_vv", lambda: capi.sub(r, pa, pb, n, q, s))
        run("add_vs", lambda: capi.add(r, pa, sc, n, q, s, scalar=True))
        run("sub_vs", lambda: capi.sub(r, pa, sc, n, q, s, scalar=True))
        for f in (1, 2, 4):
            x, y = self.dev(_uniform(rng, n, f * q)), self.dev(_uniform(rng, n, f * q))
            run(f"mul_f{f}", lambda x=x, y=y, f=f: capi.mul(r, x.data_ptr(), y.data_ptr(), n, q, f, s), mod_f=f)
        for f in (1, 2, 4, 8):
            x, c = self.dev(_uniform(rng, n, f * q)), self.dev(_uniform(rng, n, f * q))
            sf = int(_uniform(rng, 1, f * q)[0])
            run(f"fma_f{f}", lambda x=x, c=c, f=f, sf=sf: capi.fma(r, x.data_ptr(), sf, c.data_ptr(), n, q, f, s),
                mod_f=f)
        for name, fi, fo, arbitrary in (("reduce_2to1", 2, 1, False), ("reduce_4to1", 4, 1, False),
                                        ("reduce_4to2", 4, 2, False), ("reduce_barrett", 0, 1, True)):
            x = self.dev(_uniform(rng, n, 1 << 64) if arbitrary else _uniform(rng, n, fi * q))
            pin = q if arbitrary else fi
            run(name, lambda x=x, pin=pin, fo=fo: capi.reduce(r, x.data_ptr(), n, q, pin, fo, s), in_f=pin, out_f=fo)
        if any(k.startswith("ntt_") for k in kernels):
            t = capi.NTT(n, q, root)  # tables outside the timed region
            w = self.dev(_uniform(rng, n, q))
            pw = w.data_ptr()
            run("ntt_forward", lambda: t.forward(pw, pw, 1, 1, s), in_f=1, out_f=1)
            run("ntt_forward_lazy", lambda: t.forward(pw, pw, 1, 4, s), in_f=1, out_f=4)
            t.forward(pw, pw, 1, 1, s)  # inverse inputs in [0, q)
            run("ntt_inverse", lambda: t.inverse(pw, pw, 1, 1, s), in_f=1, out_f=1)
            run("ntt_inverse_lazy", lambda: t.inverse(pw, pw, 1, 2, s), in_f=1, out_f=2)
        return q, out

    def close(self):
        self.summary.close()
        if self.raw:
            self.raw.close()


def write_metadata(out_dir, args):
    import torch

    p = torch.cuda.get_device_properties(0)
    lines = [f"backend={BACKEND}", f"device={p.name}", f"sm_count={p.multi_processor_count}",
             f"host={platform.node()}", f"python={platform.python_version()}", f"torch={torch.__version__}",
             f"library={capi.LIB_PATH}", f"repetitions={args.repetitions}", f"warmup={args.warmup}",
             f"batch={args.batch}", f"degrees={','.join(map(str, args.degrees))}",
             f"bits={','.join(map(str, args.bits))}", f"kernels={','.join(args.kernels)}",
             "unit=nanoseconds per call in every *_cycles column (CUDA events on the launching stream)",
             "timing=device time: each sample queued behind a device-side sleep, host call latency excluded",
             "outlier_filter=Tukey IQR, fences Q1-1.5*IQR and Q3+1.5*IQR",
             "quantiles=linear interpolation over sorted samples",
             "ntt_mode=in-place on device-resident data; NTT table construction excluded from measurement",
             "input_mode=seeded uniform residues in the kernel's input range, device-resident",
             "batch_semantics=raw_ns is the time of `batch` consecutive calls; statistics are per call",
             f"date={time.strftime('%Y-%m-%dT%H:%M:%S')}"]
    (out_dir / "metadata.txt").write_text("\n".join(lines) + "\n")


def cmd_run(args):
    out_dir = Path(args.output)
    out_dir.mkdir(parents=True, exist_ok=True)
    unknown = set(args.kernels) - set(KERNELS)
    if unknown:
        raise SystemExit(f"unknown kernels: {sorted(unknown)}")
    write_metadata(out_dir, args)
    run = Runner(args.repetitions, args.warmup, args.batch, not args.no_raw, out_dir, args.seed)
    try:
        total = len(args.degrees) * len(args.bits)
        for i, degree in enumerate(args.degrees):
            for j, bits in enumerate(args.bits):
                q, res = run.scenario(degree, bits, set(args.kernels))
                k = i * len(args.bits) + j + 1
                print(f"scenario {k}/{total} N={degree} qi_bits={bits} q={q}: " +
                      " ".join(f"{name}={med:.0f}ns" for name, med in res), flush=True)
    finally:
        run.close()
    return 0


def write_summary(path, records, backend):
    """Writes summary.csv rows for timed scenarios given as records with the
    scenario keys and `raw_ns` (per sample, `batch` calls each) -- e.g. a CPU
    backend timed by wall clock -- with the same statistics and columns as
    `run` (times in nanoseconds per call)."""
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["backend"] + KEYS + METRICS)
        f3 = lambda x: f"{x:.3f}"
        for rec in records:
            per_call = [x / rec["batch"] for x in rec["raw_ns"]]
            st = statistics(per_call)
            degree = int(rec["poly_degree"])
            w.writerow([backend] + [rec[k] for k in KEYS] + [
                st["samples_total"], st["samples_kept"], st["outliers_removed"], f3(st["raw_min"]),
                f3(st["raw_max"]), f3(st["q1"]), f3(st["q3"]), f3(st["iqr"]), f3(st["lower_fence"]),
                f3(st["upper_fence"]), f3(st["min"]), f3(st["max"]), f3(st["mean"]), f3(st["median"]),
                f3(st["stddev"]), f3(st["cv_percent"]), f3(st["mean"] / degree), f3(st["median"] / degree), 0])


def speedup_table(path):
    """Markdown table of a compare output: per kernel and degree, the median
    over modulus widths of the CPU / GPU median-time ratio."""
    with open(path, newline="") as f:
        rows = list(csv.DictReader(f))
    by = {}
    for r in rows:
        by.setdefault((r["kernel"], int(r["poly_degree"])), []).append(
            (float(r["speedup_median_cpu_over_gpu"]), float(r["cpu_median_ns"]), float(r["gpu_median_ns"])))
    degrees = sorted({d for _, d in by})
    kernels = [k for k in KERNELS if any((k, d) in by for d in degrees)]
    med = lambda v: sorted(v)[len(v) // 2]
    lines = ["| kernel | " + " | ".join(f"N={d}" for d in degrees) + " |",
             "|---|" + "---|" * len(degrees)]
    for k in kernels:
        cells = []
        for d in degrees:
            v = by.get((k, d))
            if not v:
                cells.append("")
                continue
            cells.append(f"{med([x[0] for x in v]):.2f}x ({med([x[1] for x in v]) / 1e3:.1f} / "
                         f"{med([x[2] for x in v]) / 1e3:.1f} us)")
        lines.append(f"| {k} | " + " | ".join(cells) + " |")
    return "\n".join(lines)


def load_summary(path):
    with open(path, newline="") as f:
        rows = list(csv.DictReader(f))
    return {tuple(row[k] for k in KEYS): row for row in rows}


def cmd_compare(args):
    """Joins a CPU summary (cycles) and this library's (ns) on the scenario
    keys: per scenario both medians and means in ns and the CPU / GPU ratios."""
    cpu, gpu = load_summary(args.cpu_summary), load_summary(args.gpu_summary)
    common = sorted(set(cpu) & set(gpu), key=lambda k: (k[0], int(k[1]), int(k[2])))
    if not common:
        raise SystemExit("no scenario appears in both summaries")
    ghz = 1.0 if args.cpu_unit == "ns" else args.cpu_ghz
    if ghz is None:
        raise SystemExit("--cpu-ghz is required for a CPU summary in cycles")
    Path(args.output).parent.mkdir(parents=True, exist_ok=True)
    with open(args.output, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(KEYS + ["cpu_backend", "cpu_median_ns", "cpu_mean_ns", "gpu_median_ns", "gpu_mean_ns",
                           "speedup_median_cpu_over_gpu", "speedup_mean_cpu_over_gpu"])
        for k in common:
            c, g = cpu[k], gpu[k]
            cm, ca = float(c["median_cycles"]) / ghz, float(c["mean_cycles"]) / ghz
            gm, ga = float(g["median_cycles"]), float(g["mean_cycles"])
            w.writerow(list(k) + [c.get("backend", ""), f"{cm:.3f}", f"{ca:.3f}", f"{gm:.3f}", f"{ga:.3f}",
                                  f"{cm / gm:.6f}" if gm else "", f"{ca / ga:.6f}" if ga else ""])
    print(f"{len(common)} scenarios -> {args.output} "
          f"({len(set(cpu) - set(gpu))} CPU-only, {len(set(gpu) - set(cpu))} GPU-only skipped)")
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run", help="time every kernel over the scenario matrix on the GPU")
    r.add_argument("--output", default="results/" + BACKEND.lower())
    r.add_argument("--degrees", type=lambda s: [int(x) for x in s.split(",")], default=DEGREES)
    r.add_argument("--bits", type=lambda s: [int(x) for x in s.split(",")], default=BITS)
    r.add_argument("--kernels", type=lambda s: s.split(","), default=KERNELS)
    r.add_argument("--repetitions", type=int, default=100)
    r.add_argument("--warmup", type=int, default=10)
    r.add_argument("--batch", type=int, default=1)
    r.add_argument("--seed", type=int, default=0x415848454C42454E)
    r.add_argument("--no-raw", action="store_true")
    c = sub.add_parser("compare", help="join a CPU summary.csv and this library's into a speed-up table")
    c.add_argument("cpu_summary")
    c.add_argument("gpu_summary")
    c.add_argument("output")
    c.add_argument("--cpu-ghz", type=float, default=None, help="clock converting the CPU summary's cycles to ns")
    c.add_argument("--cpu-unit", choices=["cycles", "ns"], default="cycles",
                   help="unit of the CPU summary's *_cycles columns (ns: a wall-clock summary)")
    a = ap.parse_args(argv)
    return cmd_run(a) if a.cmd == "run" else cmd_compare(a)


if __name__ == "__main__":
    raise SystemExit(main())
