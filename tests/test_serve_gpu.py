"""GPU: the serving loop.  Requests of mixed degree and limb count, from host
(pinned) and device memory, give the same bits alone and in a concurrent mix
(and match the reference call sequence on the oracle); admission respects the
HBM budget; host-side failure cases (rejection, cancellation, a held queue
and a bounded wait) leave the server healthy."""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


def pinned(arr):
    import torch

    t = torch.empty(max(arr.size, 1), dtype=torch.int64).pin_memory()
    t.numpy().view(np.uint64)[: arr.size] = arr
    return t


def make_requests(cuda, oracle, seed, specs):
    rng = np.random.default_rng(seed)
    reqs = []
    for j, (logn, L, count, kind) in enumerate(specs):
        n = 1 << logn
        mods = []
        for i in range(L):
            q = oracle.find_ntt_prime_near(n, int(rng.integers(40, 60)), int(rng.integers(1, 4)), 4)
            mods.append((q, oracle.find_primitive_root(n, q)))
        st = oracle.rng(SEED ^ (seed * 1000 + j))
        x = np.concatenate([oracle.random_vector(st, n, 2 * mods[i % L][0]) for i in range(count)])
        v = np.concatenate([oracle.random_vector(st, n, 2 * mods[i % L][0]) for i in range(count)])
        sc = [oracle.bounded(st, 2 * q) for q, _ in mods]
        reqs.append(dict(n=n, L=L, count=count, kind=kind, mods=mods, x=x, v=v, sc=sc,
                         ntts=[cuda.NTT(n, q, psi) for q, psi in mods]))
    return reqs


def expected(oracle, r):
    n, out = r["n"], []
    for i in range(r["count"]):
        q, psi = r["mods"][i % r["L"]]
        fwd, inv, ninv = oracle.tables(n, q, psi)
        s = slice(i * n, (i + 1) * n)
        y = oracle.inverse(r["x"][s], q, inv, ninv, 2, 2)
        y = oracle.mul(y, r["v"][s], q, 2) if r["kind"] == 3 else oracle.fma(y, r["sc"][i % r["L"]], r["v"][s], q, 2)
        out.append(oracle.forward(y, q, fwd, 1, 4))
    return np.concatenate(out)


def submit(srv, r, on_device):
    if on_device:
        bi, bo, bv = dev(r["x"]), dev_empty(r["x"].size), dev(r["v"])
        pi, po, pv = ptr(bi), ptr(bo), ptr(bv)
    else:
        bi, bo, bv = pinned(r["x"]), pinned(np.zeros(r["x"].size, np.uint64)), pinned(r["v"])
        pi, po, pv = bi.data_ptr(), bo.data_ptr(), bv.data_ptr()
    rid = srv.submit(r["kind"], r["ntts"], r["count"], pi, po, vector=pv,
                     scalars=r["sc"] if r["kind"] == 4 else None, in_f=2, out_f=4)
    return rid, (bi, bo, bv)


def result(bufs, size, on_device):
    if on_device:
        return host(bufs[1], size)
    return bufs[1].numpy().view(np.uint64)[:size].copy()


SPECS = [(13, 4, 4, 3), (14, 2, 2, 4), (15, 6, 6, 3), (16, 3, 3, 4), (17, 2, 2, 3), (13, 8, 8, 4), (16, 5, 5, 3),
         (12, 3, 3, 4)]


@pytest.mark.parametrize("cfg", [{}, {"persistent": True}, {"small_request_words": 1 << 16}, {"flags": 2},
                                 {"flags": 4, "aging_us": 500}, {"max_batch_requests": 1, "max_inflight": 8},
                                 {"small_request_words": 1 << 16, "flags": 8}, {"batch_size_ratio": 2}],
                         ids=["per-phase", "persistent", "two-lanes", "arrival-priority", "smallest-first",
                              "one-per-batch", "large-first", "size-ratio"])
def test_same_bits_alone_and_in_a_mix(cuda, oracle, cfg):
    reqs = make_requests(cuda, oracle, 5, SPECS)
    srv = cuda.Server(**{"budget_bytes": 8 << 30, "max_inflight": 2, "max_batch_requests": 64, **cfg})
    alone = []
    for k, r in enumerate(reqs):  # one at a time on an idle server
        rid, bufs = submit(srv, r, on_device=k % 2 == 0)
        st, info = srv.wait(rid)
        assert st == 0 and info.batch_size == 1
        alone.append(result(bufs, r["x"].size, k % 2 == 0))
        np.testing.assert_array_equal(alone[-1], expected(oracle, r), err_msg=f"request {k}")
    # everything at once, twice over: admission held while the requests
    # arrive, then released, so batches mix requests (and two run at a time)
    handles = []
    srv.pause(True)
    for rep in range(2):
        for k, r in enumerate(reqs):
            rid, bufs = submit(srv, r, on_device=(k + rep) % 2 == 0)
            handles.append((k, rid, bufs, (k + rep) % 2 == 0))
    srv.pause(False)
    sizes = []
    for k, rid, bufs, on_dev in handles:
        st, info = srv.wait(rid)
        assert st == 0
        sizes.append(info.batch_size)
        np.testing.assert_array_equal(result(bufs, reqs[k]["x"].size, on_dev), alone[k], err_msg=f"mix {k}")
    if cfg.get("max_batch_requests", 64) > 1:
        assert max(sizes) > 1, "concurrent requests were batched together"
    else:
        assert max(sizes) == 1
    stats = srv.stats()
    assert stats["completed"] == 3 * len(reqs) and stats["p99_ms"] >= stats["p50_ms"] > 0
    srv.close()


def test_admission_respects_the_budget(cuda, oracle):
    reqs = make_requests(cuda, oracle, 6, [(16, 4, 4, 3)] * 6)
    one = 3 * reqs[0]["x"].nbytes  # input, output and vector staged per request
    srv = cuda.Server(budget_bytes=2 * one, max_inflight=4, max_batch_requests=16)
    hs = [submit(srv, r, on_device=False) for r in reqs]
    for (rid, bufs), r in zip(hs, reqs):
        st, _ = srv.wait(rid)
        assert st == 0
        np.testing.assert_array_equal(result(bufs, r["x"].size, False), expected(oracle, r))
    assert srv.stats()["peak_in_use_bytes"] <= 2 * one
    srv.close()


def test_rejection_cancel_and_bounded_wait(cuda, oracle):
    reqs = make_requests(cuda, oracle, 7, [(13, 2, 2, 3), (13, 2, 2, 4), (13, 2, 2, 3)])
    one = 3 * reqs[0]["x"].nbytes
    srv = cuda.Server(budget_bytes=one, max_inflight=1, max_batch_requests=4)
    big = make_requests(cuda, oracle, 8, [(14, 2, 4, 3)])[0]
    with pytest.raises(cuda.AxhelError) as e:  # alone over the budget
        submit(srv, big, on_device=False)
    assert e.value.status == 7
    srv.pause(True)  # a held queue: nothing is admitted
    a, abufs = submit(srv, reqs[0], on_device=False)
    b, bbufs = submit(srv, reqs[1], on_device=False)
    c, cbufs = submit(srv, reqs[2], on_device=False)
    st, _ = srv.wait(a, timeout_s=0.02)
    assert st == 6  # bounded wait: still queued
    assert srv.cancel(b) == 0
    srv.pause(False)
    st, info = srv.wait(b)
    assert st == 8  # cancelled, never ran
    for rid, bufs, r in ((a, abufs, reqs[0]), (c, cbufs, reqs[2])):
        st, _ = srv.wait(rid)
        assert st == 0
        np.testing.assert_array_equal(result(bufs, r["x"].size, False), expected(oracle, r))
    srv.close()


def test_eltwise_requests_alone_and_in_a_mix(cuda, oracle):
    """Element-wise requests (Add/Sub/Mul/FMA/ReduceMod over all limbs) are
    admitted beside transform chains: each result equals the reference's
    per-limb calls alone, and is the same in a concurrent mix."""
    from helpers import eltwise_expected, eltwise_job_data

    rng = np.random.default_rng(12)
    cases = [(5, True, 1, 1), (6, False, 1, 1), (7, True, 2, 1), (8, True, 4, 1), (8, False, 8, 1),
             (9, False, 4, 1), (9, False, "q", 1)]
    ereqs = []
    for c, (kind, has_vec, in_f, out_f) in enumerate(cases):
        n, L, count = 1 << (13 + c % 3), 3, 4
        mods = []
        for i in range(L):
            q = oracle.find_ntt_prime_near(n, int(rng.integers(40, 60)), int(rng.integers(1, 4)), 4)
            mods.append((q, oracle.find_primitive_root(n, q)))
        x, vec, sc = eltwise_job_data(oracle, oracle.rng(SEED ^ (4242 + c)), kind, has_vec, in_f, mods, n, count)
        ereqs.append(dict(kind=kind, has_vec=has_vec, in_f=in_f, out_f=out_f, mods=mods, n=n, count=count, x=x,
                          vec=vec, sc=sc, ntts=[cuda.NTT(n, q, psi) for q, psi in mods]))
    chains = make_requests(cuda, oracle, 9, SPECS[:4])

    def esubmit(srv, r, on_device):
        if on_device:
            bi, bo = dev(r["x"]), dev_empty(r["x"].size)
            bv = dev(r["vec"]) if r["has_vec"] else None
            pi, po, pv = ptr(bi), ptr(bo), ptr(bv) if bv is not None else 0
        else:
            bi, bo = pinned(r["x"]), pinned(np.zeros(r["x"].size, np.uint64))
            bv = pinned(r["vec"]) if r["has_vec"] else None
            pi, po, pv = bi.data_ptr(), bo.data_ptr(), bv.data_ptr() if bv is not None else 0
        in_f = cuda.FACTOR_MODULUS if r["in_f"] == "q" else r["in_f"]
        rid = srv.submit(r["kind"], r["ntts"], r["count"], pi, po, vector=pv, scalars=r["sc"], in_f=in_f,
                         out_f=r["out_f"])
        return rid, (bi, bo, bv)

    srv = cuda.Server(budget_bytes=8 << 30, max_inflight=2, max_batch_requests=64)
    alone = []
    for k, r in enumerate(ereqs):
        rid, bufs = esubmit(srv, r, on_device=k % 2 == 1)
        st, info = srv.wait(rid)
        assert st == 0 and info.batch_size == 1
        alone.append(result(bufs, r["x"].size, k % 2 == 1))
        np.testing.assert_array_equal(
            alone[-1], eltwise_expected(oracle, r["kind"], r["has_vec"], r["in_f"], r["out_f"], r["mods"], r["n"],
                                        r["count"], r["x"], r["vec"], r["sc"]), err_msg=f"request {cases[k]}")
    chain_alone = [expected(oracle, r) for r in chains]
    handles = []
    srv.pause(True)
    for k, r in enumerate(ereqs):
        rid, bufs = esubmit(srv, r, on_device=k % 2 == 0)
        handles.append(("e", k, rid, bufs, k % 2 == 0))
    for k, r in enumerate(chains):
        rid, bufs = submit(srv, r, on_device=k % 2 == 1)
        handles.append(("c", k, rid, bufs, k % 2 == 1))
    srv.pause(False)
    sizes = []
    for what, k, rid, bufs, on_dev in handles:
        st, info = srv.wait(rid)
        assert st == 0
        sizes.append(info.batch_size)
        if what == "e":
            np.testing.assert_array_equal(result(bufs, ereqs[k]["x"].size, on_dev), alone[k], err_msg=f"mix {k}")
        else:
            np.testing.assert_array_equal(result(bufs, chains[k]["x"].size, on_dev), chain_alone[k])
    assert max(sizes) > 1
    with pytest.raises(cuda.AxhelError):  # refused at submit, alone: MulMod factor 3
        r = ereqs[2]
        d = dev(r["x"])
        srv.submit(7, r["ntts"], r["count"], ptr(d), ptr(d), vector=ptr(d), in_f=3, out_f=1)
    srv.close()


def test_pageable_host_buffers(cuda, oracle):
    """Requests on ordinary (pageable, unpinned) host memory: same results;
    the copies are simply not asynchronous."""
    reqs = make_requests(cuda, oracle, 23, SPECS[:4])
    srv = cuda.Server(budget_bytes=4 << 30, max_inflight=2, max_batch_requests=8)
    outs, ids = [], []
    for r in reqs:
        x = np.ascontiguousarray(r["x"])
        v = np.ascontiguousarray(r["v"])
        o = np.zeros_like(x)
        outs.append((x, v, o))
        ids.append(srv.submit(r["kind"], r["ntts"], r["count"], x.ctypes.data, o.ctypes.data, vector=v.ctypes.data,
                              scalars=r["sc"] if r["kind"] == 4 else None, in_f=2, out_f=4))
    for rid, r, (x, v, o) in zip(ids, reqs, outs):
        st, _ = srv.wait(rid)
        assert st == 0
        np.testing.assert_array_equal(o, expected(oracle, r))
    srv.close()


def test_staging_failure_frees_what_it_staged(cuda, oracle):
    """A device allocation failure part-way through staging a batch (injected
    on the host at its third request): every request of that batch ends with
    AXHEL_ERR_NOMEM, the buffers staged for the first ones go back to the
    pool, the budget returns to zero, and the server keeps serving."""
    reqs = make_requests(cuda, oracle, 31, [(13, 2, 2, 3), (14, 2, 2, 4), (13, 3, 3, 3), (14, 2, 2, 3)])
    srv = cuda.Server(budget_bytes=1 << 30, max_inflight=1, max_batch_requests=16)
    srv.pause(True)
    hs = [submit(srv, r, on_device=False) for r in reqs]
    srv.debug_fail_staging(2)
    srv.pause(False)
    for rid, _ in hs:
        st, _ = srv.wait(rid)
        assert st == 3  # AXHEL_ERR_NOMEM
    s = srv.stats()
    assert s["in_use_bytes"] == 0
    assert s["pool_used_bytes"] == 0
    hs = [submit(srv, r, on_device=False) for r in reqs]
    for (rid, bufs), r in zip(hs, reqs):
        st, _ = srv.wait(rid)
        assert st == 0
        np.testing.assert_array_equal(result(bufs, r["x"].size, False), expected(oracle, r))
    assert srv.stats()["pool_used_bytes"] == 0
    srv.close()


@pytest.mark.parametrize("aging_us", [0, 10_000_000])
def test_smallest_first_admission_and_aging(cuda, oracle, aging_us):
    """Smallest-first admission, one request per batch on one stream: held
    requests run smallest first; with an aging bound of 0 every request has
    aged, so they run in arrival order.  Results are the same either way."""
    specs = [(15, 4, 4, 3), (13, 2, 2, 4), (16, 3, 3, 3), (13, 1, 1, 3), (14, 2, 2, 4)]
    reqs = make_requests(cuda, oracle, 41, specs)
    srv = cuda.Server(budget_bytes=4 << 30, max_inflight=1, max_batch_requests=1, flags=cuda.SERVER_SMALLEST_FIRST,
                      aging_us=aging_us)
    srv.pause(True)
    hs = [submit(srv, r, on_device=True) for r in reqs]
    srv.pause(False)
    batch = []
    for (rid, bufs), r in zip(hs, reqs):
        st, info = srv.wait(rid)
        assert st == 0 and info.batch_size == 1
        batch.append(info.batch_id)
        np.testing.assert_array_equal(result(bufs, r["x"].size, True), expected(oracle, r))
    words = [r["n"] * r["count"] for r in reqs]
    order = sorted(range(len(reqs)), key=lambda k: batch[k])
    if aging_us:
        assert [words[k] for k in order] == sorted(words)
    else:
        assert order == list(range(len(reqs)))
    srv.close()
