"""GPU: the benchmark configurations at their FULL sizes, every output word
checked against the oracle's per-limb call sequences on the same seeded
inputs, and against the committed SHA-256 digests of those outputs
(tests/golden/config_digests.json, made by running the oracle and checked
there against the reference native backend compiled from its sources):

* headline batch: 768 limbs of N = 2^16 (24 primes of 50-59 bits),
  forward(1,4) then inverse with ReduceMod(4,2) fused, out factor 1;
* tensor product: 64 ciphertext pairs x 16 limbs of N = 2^15 in one launch;
* uneven batch: 512 polynomials (N 2^12..2^17, 1..48 limbs, primes of
  30-60 bits, input factors 1/2/4; forward, inverse and INTT -> MulMod -> NTT
  jobs), as one persistent launch and as per-phase launches.
"""
import json
import os

import numpy as np
import pytest

import configs_oracle as co
from helpers import dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu

DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_digests.json")


@pytest.fixture(scope="module")
def digests():
    with open(DIGESTS) as f:
        return json.load(f)


def test_headline_batch_full_size(cuda, oracle, digests):
    import bench

    mods, data = co.headline_case()
    want = digests["headline"]
    assert co.digest(data) == want["input_sha256"], "input generator changed"
    ntts = [cuda.NTT(bench.N, q, psi) for q, psi in mods]
    x = dev(data.reshape(-1))
    y = dev_empty(data.size)
    cuda.forward_batch(ntts, ptr(y), ptr(x), bench.COUNT, 1, 4)
    fwd = host(y, data.size)
    cuda.inverse_batch(ntts, ptr(y), ptr(y), bench.COUNT, 4, 1)
    back = host(y, data.size)
    o_fwd, o_back = co.headline_oracle(oracle, mods, data)
    for name, got, exp in (("forward", fwd, o_fwd), ("round trip", back, o_back)):
        g, e = got.reshape(bench.COUNT, -1), exp.reshape(bench.COUNT, -1)
        bad = np.nonzero((g != e).any(axis=1))[0]
        assert bad.size == 0, f"{name}: limbs {bad[:8].tolist()} differ from the oracle"
    assert co.digest(fwd) == want["forward_lazy_sha256"]
    assert co.digest(back) == want["round_trip_sha256"]


def test_tensor_product_full_size(cuda, oracle, digests):
    from axhel_b200 import workloads

    want = digests["tensor"]
    n, qs, count, ins = workloads.tensor_inputs(**workloads.TENSOR_SHAPE)
    assert [co.digest(a) for a in ins] == want["input_sha256"], "input generator changed"
    bufs = [dev(a.reshape(-1)) for a in ins]
    outs = [dev_empty(n * count) for _ in range(3)]
    cuda.tensor_product(*[ptr(t) for t in outs], *[ptr(t) for t in bufs], n, count, qs, 1)
    got = [host(t, n * count) for t in outs]
    del bufs, outs
    *_, exp = co.tensor_oracle(oracle, (n, qs, count, ins))
    for k in range(3):
        g, e = got[k].reshape(count, n), exp[k].reshape(count, n)
        bad = np.nonzero((g != e).any(axis=1))[0]
        assert bad.size == 0, f"r{k}: limbs {bad[:8].tolist()} differ from the oracle"
        assert co.digest(got[k]) == want["r_sha256"][k]


def test_uneven_batch_full_size_both_launch_forms(cuda, oracle, digests):
    import torch

    from axhel_b200 import workloads

    want = digests["uneven"]["jobs"]
    pool = workloads.ModulusPool()
    jobs = workloads.uneven_jobs(pool)
    assert len(jobs) == len(want) == 512
    host_in, dev_in, results = [], [], []
    for j, job in enumerate(jobs):
        x, v = workloads.uneven_arrays(job)
        assert co.digest(x) == want[j]["input_sha256"], f"job {j}: input generator changed"
        host_in.append((x, v))
        dx = dev(x.reshape(-1))
        dv = dev(v.reshape(-1)) if v is not None else None
        dev_in.append((dx, dv))
        results.append(dev_empty(x.size))
    specs = [dict(kind=job["kind"], ntts=[t for _, t in job["mods"]], count=job["L"], result=ptr(results[j]),
                  operand=ptr(dev_in[j][0]), vector=ptr(dev_in[j][1]) if dev_in[j][1] is not None else 0,
                  in_f=job["in_f"], out_f=job["out_f"]) for j, job in enumerate(jobs)]
    b = cuda.Batch(specs)
    tabs = co.Tables(oracle)
    try:
        for phased in (False, True):
            for r in results:
                r.fill_(-1)
            b.launch(phased=phased)
            assert b.status() == 0
            torch.cuda.synchronize()
            for j, job in enumerate(jobs):
                got = host(results[j], job["L"] * job["n"])
                if not phased:  # the oracle once per job; the second form is held to the same words
                    x, v = host_in[j]
                    exp = co.uneven_oracle_job(oracle, tabs, job, x, v)
                    bad = np.nonzero((got.reshape(job["L"], -1) != exp.reshape(job["L"], -1)).any(axis=1))[0]
                    assert bad.size == 0, f"job {j} (kind {job['kind']}, N={job['n']}): limbs {bad[:8].tolist()}"
                assert co.digest(got) == want[j]["sha256"], f"job {j}, {'phased' if phased else 'persistent'}"
    finally:
        b.close()
