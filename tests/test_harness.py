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


def test_wall_clock_summary_joins_in_nanoseconds(tmp_path):
    """A CPU backend timed by wall clock (records of raw ns samples) gets the
    same summary columns and statistics, and joins without a clock rate."""
    recs = [dict(kernel="ntt_forward", poly_degree=4096, qi_bits=50, modulus=1125899906826241, mod_factor=0,
                 input_mod_factor=1, output_mod_factor=1, batch=2, raw_ns=[20000.0, 21000.0, 20500.0, 90000.0]),
            dict(kernel="add_vv", poly_degree=4096, qi_bits=50, modulus=1125899906826241, mod_factor=0,
                 input_mod_factor=0, output_mod_factor=0, batch=1, raw_ns=[3000.0, 3100.0, 2900.0])]
    harness.write_summary(tmp_path / "cpu.csv", recs, "reference-native-1thread")
    rows = {r["kernel"]: r for r in csv.DictReader(open(tmp_path / "cpu.csv"))}
    assert list(next(iter(rows.values())).keys()) == ["backend"] + harness.KEYS + harness.METRICS
    assert int(rows["ntt_forward"]["outliers_removed"]) == 1
    assert float(rows["ntt_forward"]["median_cycles"]) == pytest.approx(10250.0)
    gpu = {**recs[0], "raw_ns": [2050.0] * 4, "batch": 1}
    harness.write_summary(tmp_path / "gpu.csv", [gpu], "B200")
    assert harness.main(["compare", str(tmp_path / "cpu.csv"), str(tmp_path / "gpu.csv"), str(tmp_path / "s.csv"),
                         "--cpu-unit", "ns"]) == 0
    out = list(csv.DictReader(open(tmp_path / "s.csv")))
    assert len(out) == 1 and float(out[0]["speedup_median_cpu_over_gpu"]) == pytest.approx(5.0)
    md = harness.speedup_table(tmp_path / "s.csv")
    assert "| ntt_forward | 5.00x" in md
