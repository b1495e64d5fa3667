"""GPU: edge cases of the batched forms -- jobs with no limbs beside real
ones, batches with nothing to do, 8-byte (not 16-byte) aligned operands and
results, and the largest degree -- each against the oracle or untouched."""
import numpy as np
import pytest

import test_batch_gpu as tb
from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


def test_jobs_without_limbs_are_skipped(cuda, oracle):
    rng = np.random.default_rng(5)
    jobs = tb.make_jobs(cuda, oracle, rng, 4, [11, 14], 2, 2)
    specs, bufs = tb.specs_for(cuda, jobs)
    canary = dev_empty(64, fill=0x5A5A5A5A)
    q = jobs[0]["mods"][0][0]
    empty = [dict(kind=k, ntts=jobs[0]["ntts"], count=0, result=ptr(canary), operand=ptr(canary),
                  vector=ptr(canary), scalars=[1] * len(jobs[0]["ntts"]), in_f=1, out_f=1)
             for k in (1, 2, 3, 4, 5, 7, 9)]
    cuda.batch_run(empty[:3] + specs + empty[3:])
    tb.check(oracle, jobs, bufs)
    assert np.all(host(canary, 64) == np.uint64(0x5A5A5A5A)), "a job without limbs wrote"
    l0 = cuda.launch_count()
    cuda.batch_run(empty)  # nothing to do: no launch, no error
    b = cuda.Batch(empty)
    b.launch()
    assert b.status() == 0
    b.close()
    assert cuda.launch_count() == l0
    assert np.all(host(canary, 64) == np.uint64(0x5A5A5A5A))
    t = jobs[0]["ntts"][0]
    cuda.forward_batch([t], ptr(canary), ptr(canary), 0, 1, 4)  # count 0: a no-op
    cuda.inverse_batch([t], ptr(canary), ptr(canary), 0, 2, 1)
    assert np.all(host(canary, 64) == np.uint64(0x5A5A5A5A))


@pytest.mark.parametrize("off", [1, 3])
def test_eight_byte_aligned_operands(cuda, oracle, off):
    """Operands and results 8 bytes off a 16-byte boundary (the reference
    accepts any uint64_t*): every job kind, element-wise jobs included."""
    from helpers import eltwise_expected, eltwise_job_data

    rng = np.random.default_rng(40 + off)
    jobs = tb.make_jobs(cuda, oracle, rng, 6, [10, 13, 16], 2, 3)
    specs, keep = [], []
    for jb in jobs:
        d = dev_empty(jb["x"].size + off)
        d[off:] = dev(jb["x"])[: jb["x"].size]
        o = dev_empty(jb["x"].size + off, fill=0)
        dv = None
        if jb["vec"] is not None:
            dv = dev_empty(jb["vec"].size + off)
            dv[off:] = dev(jb["vec"])[: jb["vec"].size]
        keep.append((d, o, dv))
        specs.append(dict(kind=jb["kind"], ntts=jb["ntts"], count=jb["count"], result=ptr(o, off),
                          operand=ptr(d, off), vector=ptr(dv, off) if dv is not None else 0,
                          scalars=jb["scalars"], in_f=jb["in_f"], out_f=jb["out_f"]))
    n = 1 << 12
    q = oracle.find_ntt_prime(n, 50)
    mods = [(q, oracle.find_primitive_root(n, q))]
    ex, ev, es = eltwise_job_data(oracle, oracle.rng(SEED ^ off), 7, True, 2, mods, n, 2)
    de, dve, deo = dev_empty(ex.size + off), dev_empty(ex.size + off), dev_empty(ex.size + off, fill=0)
    de[off:] = dev(ex)[: ex.size]
    dve[off:] = dev(ev)[: ev.size]
    specs.append(dict(kind=7, ntts=[cuda.NTT(n, q, mods[0][1])], count=2, result=ptr(deo, off),
                      operand=ptr(de, off), vector=ptr(dve, off), in_f=2, out_f=1))
    cuda.batch_run(specs)
    for idx, (jb, (d, o, dv)) in enumerate(zip(jobs, keep)):
        got = host(o, jb["x"].size + off)[off:]
        np.testing.assert_array_equal(got, tb.expected(oracle, jb), err_msg=f"job {idx} kind {jb['kind']}")
    np.testing.assert_array_equal(host(deo, ex.size + off)[off:],
                                  eltwise_expected(oracle, 7, True, 2, 1, mods, n, 2, ex, ev, es))


def test_largest_degree_all_kinds(cuda, oracle):
    rng = np.random.default_rng(17)
    for kind in (1, 2, 3, 4):
        jobs = tb.make_jobs(cuda, oracle, rng, 1, [17], 1, 1, kinds=(kind,))
        specs, bufs = tb.specs_for(cuda, jobs)
        cuda.batch_run(specs)
        tb.check(oracle, jobs, bufs)
        specs, bufs = tb.specs_for(cuda, jobs)
        b = cuda.Batch(specs)
        b.launch(phased=True)
        assert b.status() == 0
        tb.check(oracle, jobs, bufs)
        b.close()
