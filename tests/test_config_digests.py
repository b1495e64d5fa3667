"""CPU: the committed full-size digests (tests/golden/config_digests.json) are
reproduced by the oracle on the regenerated seeded inputs -- the headline
batch, the tensor product, and a sample of the uneven batch's jobs (the
generator script checks all of them against the reference itself)."""
import json
import os

import pytest

import configs_oracle as co

DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_digests.json")


@pytest.fixture(scope="module")
def digests():
    with open(DIGESTS) as f:
        return json.load(f)


def test_headline_digests(oracle, digests):
    mods, data = co.headline_case()
    want = digests["headline"]
    assert co.digest(data) == want["input_sha256"]
    fwd, back = co.headline_oracle(oracle, mods, data)
    assert co.digest(fwd) == want["forward_lazy_sha256"]
    assert co.digest(back) == want["round_trip_sha256"] == co.digest(data)


def test_tensor_digests(oracle, digests):
    want = digests["tensor"]
    n, qs, count, ins, outs = co.tensor_oracle(oracle)
    assert qs == want["moduli"]
    assert [co.digest(a) for a in ins] == want["input_sha256"]
    assert [co.digest(o) for o in outs] == want["r_sha256"]


def test_uneven_digests_sample(oracle, digests):
    from axhel_b200 import workloads

    want = digests["uneven"]["jobs"]
    jobs = co.uneven_case()
    assert len(jobs) == len(want)
    assert sum(j["L"] for j in jobs) == digests["uneven"]["limbs"]
    tabs = co.Tables(oracle)
    sample = [j for j in range(len(jobs)) if jobs[j]["n"] <= 1 << 14][:24]
    sample += [j for j in range(len(jobs)) if jobs[j]["n"] == 1 << 17][:2]
    kinds = {jobs[j]["kind"] for j in sample}
    assert kinds == {1, 2, 3}
    for j in sample:
        job = jobs[j]
        x, v = workloads.uneven_arrays(job)
        assert co.digest(x) == want[j]["input_sha256"]
        assert co.digest(co.uneven_oracle_job(oracle, tabs, job, x, v)) == want[j]["sha256"], f"job {j}"
