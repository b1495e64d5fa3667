"""The per-kernel harness (axhel_b200/harness.py): its statistics follow the
reference benchmark's (linear quantiles, Tukey fences), its scenario moduli
are the reference benchmark's (the largest prime q = 1 mod 2N below 2^bits),
the compare step joins summaries on the scenario keys; on a GPU, one small
run writes a summary.csv with the reference's columns and every kernel."""
import csv

import pytest

from axhel_b200 import harness


def test_statistics_follow_the_reference_definitions():
    st = harness.statistics([4.0, 1.0, 3.0, 100.0, 2.0])
    assert (st["q1"], st["q3"], st["iqr"]) == (2.0, 4.0, 2.0)
    assert (st["lower_fence"], st["upper_fence"]) == (-1.0, 7.0)
    assert (st["samples_total"], st["samples_kept"], st["outliers_removed"]) == (5, 4, 1)
    assert st["median"] == 2.5 and st["mean"] == 2.5 and st["raw_max"] == 100.0
    assert abs(st["stddev"] - (5.0 / 3.0) ** 0.5) < 1e-12
    one = harness.statistics([7.0])
    assert one["median"] == 7.0 and one["stddev"] == 0.0


def test_scenario_moduli_are_the_reference_benchmarks(oracle):
    for degree in harness.DEGREES:
        for bits in harness.BITS:
            assert harness.largest_ntt_prime(degree, bits) == oracle.find_ntt_prime(degree, bits), (degree, bits)


def test_compare_joins_cpu_and_gpu_summaries(tmp_path):
    cols = ["backend"] + harness.KEYS + harness.METRICS
    def write(path, backend, rows):
        with open(path, "w", newline="") as f:
            w = csv.writer(f)
            w.writerow(cols)
            for kernel, med, mean in rows:
                vals = {m: "0" for m in harness.METRICS}
                vals.update(median_cycles=str(med), mean_cycles=str(mean))
                w.writerow([backend, kernel, 4096, 50, 1125899906826241, 0, 1, 1] + [vals[m] for m in harness.METRICS])
    write(tmp_path / "cpu.csv", "Native", [("ntt_forward", 27000.0, 27500.0), ("add_vv", 2700.0, 2700.0)])
    write(tmp_path / "gpu.csv", "B200", [("ntt_forward", 5000.0, 5000.0), ("mul_f1", 3000.0, 3000.0)])
    assert harness.main(["compare", str(tmp_path / "cpu.csv"), str(tmp_path / "gpu.csv"), str(tmp_path / "s.csv"),
                         "--cpu-ghz", "2.7"]) == 0
    rows = list(csv.DictReader(open(tmp_path / "s.csv")))
    assert len(rows) == 1 and rows[0]["kernel"] == "ntt_forward"
    assert float(rows[0]["cpu_median_ns"]) == pytest.approx(10000.0)
    assert float(rows[0]["speedup_median_cpu_over_gpu"]) == pytest.approx(2.0)


@pytest.mark.gpu
def test_small_run_writes_every_kernel(tmp_path, cuda):
    assert harness.main(["run", "--output", str(tmp_path), "--degrees", "2048,4096", "--bits", "50,62",
                         "--repetitions", "7", "--warmup", "2"]) == 0
    rows = list(csv.DictReader(open(tmp_path / "summary.csv")))
    assert list(rows[0].keys()) == ["backend"] + harness.KEYS + harness.METRICS
    assert len(rows) == 4 * len(harness.KERNELS)
    assert {r["kernel"] for r in rows} == set(harness.KERNELS)
    for r in rows:
        assert r["backend"] == "B200" and int(r["samples_total"]) == 7
        assert 0 < float(r["median_cycles"]) < 1e7  # ns per call
    assert (tmp_path / "metadata.txt").read_text().count("unit=nanoseconds") == 1
