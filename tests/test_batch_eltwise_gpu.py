"""GPU: element-wise jobs of the batch engine -- EltwiseAdd/Sub/Mul/FMA/
ReduceMod over every limb of a job, limb i with the modulus of ntts[i % L] --
bit-exact against the reference's per-limb calls on the oracle, for every
mod-factor and form the reference has; alone, in place, and mixed with
transform jobs in one launch; factor pairs the reference ignores are refused."""
import numpy as np
import pytest

import test_batch_gpu as tb
from helpers import ELT_CASES, SEED, dev, dev_empty, eltwise_expected, eltwise_job_data, host, ptr

pytestmark = pytest.mark.gpu


def elt_jobs(cuda, oracle, seed, logns=(10, 13), L=3, count=5):
    rng = np.random.default_rng(seed)
    jobs = []
    for c, (kind, has_vec, in_f, out_f) in enumerate(ELT_CASES):
        n = 1 << int(rng.choice(logns))
        mods = []
        for i in range(L):
            q = oracle.find_ntt_prime_near(n, int(rng.integers(30, 61)), int(rng.integers(1, 4)), 4)
            mods.append((q, oracle.find_primitive_root(n, q)))
        st = oracle.rng(SEED ^ (seed * 977 + c))
        x, vec, sc = eltwise_job_data(oracle, st, kind, has_vec, in_f, mods, n, count)
        jobs.append(dict(kind=kind, has_vec=has_vec, in_f=in_f, out_f=out_f, mods=mods, n=n, count=count, x=x,
                         vec=vec, sc=sc, ntts=[cuda.NTT(n, q, psi) for q, psi in mods]))
    return jobs


def elt_specs(cuda, jobs, in_place=False):
    specs, bufs = [], []
    for jb in jobs:
        d = dev(jb["x"])
        o = d if in_place else dev_empty(jb["x"].size, fill=0xA5A5A5A5)
        dv = dev(jb["vec"]) if jb["has_vec"] else None
        bufs.append((d, o, dv))
        in_f = cuda.FACTOR_MODULUS if jb["in_f"] == "q" else jb["in_f"]
        specs.append(dict(kind=jb["kind"], ntts=jb["ntts"], count=jb["count"], result=ptr(o), operand=ptr(d),
                          vector=ptr(dv) if dv is not None else 0, scalars=jb["sc"], in_f=in_f, out_f=jb["out_f"]))
    return specs, bufs


def want(oracle, jb):
    return eltwise_expected(oracle, jb["kind"], jb["has_vec"], jb["in_f"], jb["out_f"], jb["mods"], jb["n"],
                            jb["count"], jb["x"], jb["vec"], jb["sc"])


@pytest.mark.parametrize("in_place", [False, True])
def test_eltwise_jobs_match_per_limb_calls(cuda, oracle, in_place):
    jobs = elt_jobs(cuda, oracle, 31 + in_place)
    specs, bufs = elt_specs(cuda, jobs, in_place)
    l0 = cuda.launch_count()
    cuda.batch_run(specs)
    assert cuda.launch_count() - l0 == 1
    for k, (jb, (d, o, dv)) in enumerate(zip(jobs, bufs)):
        np.testing.assert_array_equal(host(o, jb["x"].size), want(oracle, jb),
                                      err_msg=f"case {ELT_CASES[k]} n={jb['n']}")


def test_eltwise_and_transform_jobs_in_one_launch(cuda, oracle):
    rng = np.random.default_rng(77)
    tjobs = tb.make_jobs(cuda, oracle, rng, 8, [10, 12, 14, 16], 3, 3)
    tspecs, tbufs = tb.specs_for(cuda, tjobs)
    ejobs = elt_jobs(cuda, oracle, 78, logns=(11, 15), L=2, count=4)
    especs, ebufs = elt_specs(cuda, ejobs)
    b = cuda.Batch(tspecs + especs)
    for graph, phased in ((False, False), (True, False), (False, True)):
        for _, o, _ in tbufs + ebufs:
            o.zero_()
        b.launch(graph=graph, phased=phased)
        assert b.status() == 0
        tb.check(oracle, tjobs, tbufs)
        for jb, (d, o, dv) in zip(ejobs, ebufs):
            np.testing.assert_array_equal(host(o, jb["x"].size), want(oracle, jb))
    b.close()


def test_eltwise_static_scratch_matches(cuda, oracle):
    jobs = elt_jobs(cuda, oracle, 90, logns=(12,), L=2, count=3)
    specs, bufs = elt_specs(cuda, jobs)
    cuda.batch_run_static(specs)
    for jb, (d, o, dv) in zip(jobs, bufs):
        np.testing.assert_array_equal(host(o, jb["x"].size), want(oracle, jb))


def test_eltwise_jobs_refuse_what_the_reference_ignores(cuda, oracle):
    n = 1024
    q = oracle.find_ntt_prime(n, 45)
    t = cuda.NTT(n, q, oracle.find_primitive_root(n, q))
    d = dev_empty(n)
    base = dict(ntts=[t], count=1, result=ptr(d), operand=ptr(d))
    bad = [dict(kind=7, vector=ptr(d), in_f=3),            # MulMod factor 3 (a no-op in the reference)
           dict(kind=8, scalars=[1], in_f=16),             # FMAMod factor 16
           dict(kind=9, in_f=2, out_f=4),                  # unmatched ReduceMod pair
           dict(kind=9, in_f=8, out_f=1),
           dict(kind=5),                                   # neither vector nor scalars
           dict(kind=7, in_f=1),                           # multiplicand missing
           dict(kind=8, in_f=1),                           # scalars missing
           dict(kind=10)]                                  # unknown kind
    for b in bad:
        with pytest.raises(cuda.AxhelError) as e:
            cuda.batch_run([dict(base, **b)])
        assert e.value.status == 1, b  # AXHEL_ERR_INVALID


def test_single_job_batches_per_phase_every_kind(cuda, oracle):
    """A batch of one job runs its per-phase launches with the job's entry as
    a kernel parameter: every transform kind (at a split of each width) and
    every element-wise form, alone, against the reference's per-limb calls."""
    rng = np.random.default_rng(123)
    for kind in (1, 2, 3, 4):
        for logn in (11, 14, 16, 17):
            jobs = tb.make_jobs(cuda, oracle, rng, 1, [logn], 3, 3, kinds=(kind,))
            specs, bufs = tb.specs_for(cuda, jobs)
            b = cuda.Batch(specs)
            b.launch(phased=True)
            assert b.status() == 0
            tb.check(oracle, jobs, bufs)
            b.close()
    for jb in elt_jobs(cuda, oracle, 124, logns=(10, 14), L=2, count=3):
        specs, bufs = elt_specs(cuda, [jb])
        b = cuda.Batch(specs)
        b.launch(phased=True)
        assert b.status() == 0
        np.testing.assert_array_equal(host(bufs[0][1], jb["x"].size), want(oracle, jb))
        b.close()


def test_random_mixed_batches_both_forms(cuda, oracle):
    """Seeded random batches: 1-11 transform and chain jobs over up to three
    degrees, 0-3 element-wise jobs, in shuffled order; the persistent launch
    and the per-phase launches each match the reference's per-limb calls."""
    for seed in range(24):
        rng = np.random.default_rng(50000 + seed)
        logns = sorted(set(int(x) for x in rng.integers(10, 18, 3)))
        jobs = tb.make_jobs(cuda, oracle, rng, int(rng.integers(1, 12)), logns, int(rng.integers(1, 10)),
                            int(rng.integers(1, 5)))
        ejobs = elt_jobs(cuda, oracle, 7000 + seed, logns=(10, 12), L=2,
                         count=int(rng.integers(1, 4)))[: int(rng.integers(0, 4))]
        for phased in (False, True):
            specs, bufs = tb.specs_for(cuda, jobs)
            especs, ebufs = elt_specs(cuda, ejobs)
            every = specs + especs
            order = rng.permutation(len(every))
            b = cuda.Batch([every[i] for i in order])
            b.launch(phased=phased)
            assert b.status() == 0
            b.close()
            tb.check(oracle, jobs, bufs)
            for jb, (d, o, dv) in zip(ejobs, ebufs):
                np.testing.assert_array_equal(host(o, jb["x"].size), want(oracle, jb),
                                              err_msg=f"seed {seed} phased={phased}")
