"""GPU: uneven batches (mixed degree, limb count, kind and input factor) in one
persistent launch, each job bit-exact against the reference call sequence on
the oracle; relaunch and CUDA-graph replay; the bounded dependency wait."""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


def make_jobs(cuda, oracle, rng, n_jobs, logns, max_count, max_L, kinds=(1, 2, 3, 4)):
    jobs = []
    for j in range(n_jobs):
        logn = int(rng.choice(logns))
        n = 1 << logn
        L = int(rng.integers(1, max_L + 1))
        count = int(rng.integers(1, max_count + 1))
        kind = int(rng.choice(kinds))
        mods = []
        for i in range(L):
            bits = int(rng.integers(30, 61))
            q = oracle.find_ntt_prime_near(n, bits, int(rng.integers(1, 4)), 4)
            mods.append((q, oracle.find_primitive_root(n, q)))
        in_f = int(rng.choice([1, 2, 4]))
        if kind == 1:
            out_f = int(rng.choice([1, 4]))
        elif kind == 2:
            out_f = int(rng.choice([1, 2]))
        else:
            out_f = int(rng.choice([1, 4]))
        st = oracle.rng(SEED ^ (j * 7919 + logn))
        bound_in = lambda q: in_f * q  # lazy input factor: residues in [0, in_f * q)
        x = np.concatenate([oracle.random_vector(st, n, bound_in(mods[i % L][0])) for i in range(count)])
        vec = None
        if kind in (3, 4):
            vec = np.concatenate([oracle.random_vector(st, n, 2 * mods[i % L][0]) for i in range(count)])
        scal = [oracle.bounded(st, 2 * q) for q, _ in mods] if kind == 4 else None
        jobs.append(dict(kind=kind, n=n, L=L, count=count, mods=mods, x=x, vec=vec, scalars=scal, in_f=in_f,
                         out_f=out_f, ntts=[cuda.NTT(n, q, psi) for q, psi in mods]))
    return jobs


def expected(oracle, jb):
    n, L, out = jb["n"], jb["L"], []
    for i in range(jb["count"]):
        q, psi = jb["mods"][i % L]
        fwd, inv, ninv = oracle.tables(n, q, psi)
        x = jb["x"][i * n:(i + 1) * n]
        k = jb["kind"]
        if k == 1:
            out.append(oracle.forward(x, q, fwd, jb["in_f"], jb["out_f"]))
            continue
        if jb["in_f"] == 4:
            x = oracle.reduce(x, q, 4, 2)
        if k == 2:
            out.append(oracle.inverse(x, q, inv, ninv, 2, jb["out_f"]))
            continue
        y = oracle.inverse(x, q, inv, ninv, 2, 2)
        v = jb["vec"][i * n:(i + 1) * n]
        y = oracle.mul(y, v, q, 2) if k == 3 else oracle.fma(y, jb["scalars"][i % L], v, q, 2)
        out.append(oracle.forward(y, q, fwd, 1, jb["out_f"]))
    return np.concatenate(out)


def specs_for(cuda, jobs):
    specs, bufs = [], []
    for jb in jobs:
        d = dev(jb["x"])
        o = dev_empty(jb["x"].size)
        dv = dev(jb["vec"]) if jb["vec"] is not None else None
        bufs.append((d, o, dv))
        specs.append(dict(kind=jb["kind"], ntts=jb["ntts"], count=jb["count"], result=ptr(o), operand=ptr(d),
                          vector=ptr(dv) if dv is not None else 0, scalars=jb["scalars"], in_f=jb["in_f"],
                          out_f=jb["out_f"]))
    return specs, bufs


def check(oracle, jobs, bufs):
    for idx, (jb, (d, o, dv)) in enumerate(zip(jobs, bufs)):
        np.testing.assert_array_equal(host(o, jb["x"].size), expected(oracle, jb),
                                      err_msg=f"job {idx} kind={jb['kind']} n={jb['n']} count={jb['count']}")


def test_uneven_batch_one_launch_bitexact(cuda, oracle):
    rng = np.random.default_rng(4)
    jobs = make_jobs(cuda, oracle, rng, 24, [10, 11, 12, 13, 14, 15, 16, 17], 4, 5)
    specs, bufs = specs_for(cuda, jobs)
    l0 = cuda.launch_count()
    cuda.batch_run(specs)
    assert cuda.launch_count() - l0 == 1, "the whole batch is one kernel launch"
    check(oracle, jobs, bufs)


def test_batch_relaunch_and_graph_replay(cuda, oracle):
    rng = np.random.default_rng(9)
    jobs = make_jobs(cuda, oracle, rng, 10, [12, 16, 17], 3, 4)
    specs, bufs = specs_for(cuda, jobs)
    b = cuda.Batch(specs)
    for graph, phased in ((False, False), (False, False), (True, False), (True, False), (False, True)):
        for _, o, _ in bufs:
            o.zero_()
        b.launch(graph=graph, phased=phased)
        assert b.status() == 0
        check(oracle, jobs, bufs)
    b.close()


def test_batch_in_place_and_kinds(cuda, oracle):
    """result == operand, every kind, and the 1 / 2 / 4 input factors."""
    rng = np.random.default_rng(21)
    for kind in (1, 2, 3, 4):
        jobs = make_jobs(cuda, oracle, rng, 4, [10, 15], 2, 3, kinds=(kind,))
        specs, bufs = specs_for(cuda, jobs)
        for sp, (d, o, dv) in zip(specs, bufs):
            sp["result"] = sp["operand"]
        cuda.batch_run(specs)
        for jb, (d, o, dv) in zip(jobs, bufs):
            np.testing.assert_array_equal(host(d, jb["x"].size), expected(oracle, jb))


def test_batch_rejects_bad_jobs(cuda, oracle):
    q = oracle.find_ntt_prime(256, 40)
    t = cuda.NTT(256, q, oracle.find_primitive_root(256, q))
    d = dev_empty(256)
    with pytest.raises(cuda.AxhelError):  # degree below the batched range
        cuda.batch_run([dict(kind=1, ntts=[t], count=1, result=ptr(d), operand=ptr(d))])
    q2 = oracle.find_ntt_prime(1024, 40)
    t2 = cuda.NTT(1024, q2, oracle.find_primitive_root(1024, q2))
    with pytest.raises(cuda.AxhelError):  # handles of two degrees in one job
        cuda.batch_run([dict(kind=1, ntts=[t2, t], count=1, result=ptr(d), operand=ptr(d))])
    with pytest.raises(cuda.AxhelError):  # chain without its multiplicand
        cuda.batch_run([dict(kind=3, ntts=[t2], count=1, result=ptr(d), operand=ptr(d))])


def test_dependency_wait_times_out_and_device_recovers(cuda, oracle):
    """Failure detection without a GPU fault: a dependency that can never be
    met ends the launch with AXHEL_ERR_TIMEOUT after the bounded wait, and
    the same context then runs a batch correctly."""
    rng = np.random.default_rng(33)
    jobs = make_jobs(cuda, oracle, rng, 3, [12], 2, 2, kinds=(1,))
    specs, bufs = specs_for(cuda, jobs)
    b = cuda.Batch(specs)
    b.set_wait_ns(50_000_000)  # 50 ms
    b.debug_unreachable(1)
    b.launch()
    assert b.status() == 6  # AXHEL_ERR_TIMEOUT
    b.close()
    b = cuda.Batch(specs)
    b.launch()
    assert b.status() == 0
    check(oracle, jobs, bufs)
    b.close()


def test_every_batch_split_bitexact(cuda, oracle):
    """Every strided/contiguous split the autotuner may pick gives the same bits."""
    rng = np.random.default_rng(61)
    for logn in (10, 13, 15, 17):
        jobs = make_jobs(cuda, oracle, rng, 3, [logn], 2, 2)
        for row in range(max(5, logn - 9), min(9, logn - 5) + 1):
            cuda.batch_split_set(logn, row)
            try:
                specs, bufs = specs_for(cuda, jobs)
                cuda.batch_run(specs)
                check(oracle, jobs, bufs)
                specs, bufs = specs_for(cuda, jobs)  # the per-phase launches of every width
                b = cuda.Batch(specs)
                b.launch(phased=True)
                assert b.status() == 0
                check(oracle, jobs, bufs)
                b.close()
            finally:
                cuda.batch_split_set(logn, 0)


def test_relaunches_stay_bit_identical(cuda, oracle):
    """Cross-CTA dependencies under repetition: a mixed batch (chains across
    three phases included) relaunched 40 times, eagerly and from its graph,
    reproduces its oracle-checked first result every time."""
    import torch

    rng = np.random.default_rng(1001)
    jobs = make_jobs(cuda, oracle, rng, 16, [10, 12, 14, 16, 17], 5, 5)
    specs, bufs = specs_for(cuda, jobs)
    b = cuda.Batch(specs)
    b.launch()
    assert b.status() == 0
    check(oracle, jobs, bufs)
    ref = [o.clone() for _, o, _ in bufs]
    for rep in range(40):
        for _, o, _ in bufs:
            o.fill_(-1)
        b.launch(graph=rep % 2 == 1)
        assert b.status() == 0
        assert all(torch.equal(r, o) for r, (_, o, _) in zip(ref, bufs)), f"relaunch {rep}"
    b.close()


def test_phased_launch_replays_from_a_captured_graph(cuda, oracle):
    """The per-phase launches fork each phase over extra streams and join
    them back into the caller's stream: captured into a CUDA graph on that
    stream, the batch replays to its oracle-checked result."""
    import torch

    rng = np.random.default_rng(2024)
    jobs = make_jobs(cuda, oracle, rng, 12, [12, 14, 16, 17], 4, 4)
    specs, bufs = specs_for(cuda, jobs)
    b = cuda.Batch(specs)
    b.launch(phased=True)
    assert b.status() == 0
    check(oracle, jobs, bufs)
    ref = [o.clone() for _, o, _ in bufs]
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        b.launch(stream=s.cuda_stream, phased=True)
    for rep in range(4):
        for _, o, _ in bufs:
            o.fill_(-1)
        g.replay()
        torch.cuda.synchronize()
        assert all(torch.equal(r, o) for r, (_, o, _) in zip(ref, bufs)), f"replay {rep}"
    del g
    b.close()


def test_phased_large_entries_alone_and_grouped(cuda, oracle):
    """Entries of 512 tiles or more (here 4-8 limbs at N = 2^16, 2^17) get
    per-phase launches of their own beside the grouped small entries, spread
    over the extra streams; every kind matches its per-limb calls, and the
    persistent launch of the same batch gives the same bits."""
    import torch

    rng = np.random.default_rng(4242)
    jobs = make_jobs(cuda, oracle, rng, 6, [16, 17], 8, 3) + make_jobs(cuda, oracle, rng, 10, [10, 11, 12, 13], 3, 3)
    specs, bufs = specs_for(cuda, jobs)
    b = cuda.Batch(specs)
    b.launch(phased=True)
    assert b.status() == 0
    check(oracle, jobs, bufs)
    ref = [o.clone() for _, o, _ in bufs]
    for _, o, _ in bufs:
        o.fill_(-1)
    b.launch()
    assert b.status() == 0
    assert all(torch.equal(r, o) for r, (_, o, _) in zip(ref, bufs))
    b.close()
