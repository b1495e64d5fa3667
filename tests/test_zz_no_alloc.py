"""GPU: the batch entry point that allocates nothing, axhel_cuda_batch_run_static.

It serves callers that cannot call cudaMalloc while they run -- a process
whose device memory is reserved up front by its own allocator or a fixed
budget, or a latency-critical loop where cudaMalloc / cudaFree would
synchronize the device.  Its scratch lives in the library's static device
array, so these tests check, through the C-ABI, that two calls in a row give
exactly the results of the allocating entry point, axhel_cuda_batch_run, and
that a batch larger than the array is refused with a clear error.

This file is named to be collected last; it also passes run alone.
"""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


def _jobs(cuda, oracle):
    rng = np.random.default_rng(2024)
    specs, outs, inputs = [], [], []
    for j, (logn, kind, count, L) in enumerate([(10, 1, 3, 2), (12, 2, 2, 3), (13, 3, 2, 2), (14, 4, 1, 2),
                                                 (16, 1, 2, 3), (17, 3, 1, 1)]):
        n = 1 << logn
        mods = []
        for i in range(L):
            q = oracle.find_ntt_prime_near(n, 40 + 5 * i, 1, 2)
            mods.append((q, oracle.find_primitive_root(n, q)))
        st = oracle.rng(SEED ^ (j + 101))
        in_f = 4 if kind != 1 else 1
        x = np.concatenate([oracle.random_vector(st, n, in_f * mods[i % L][0]) for i in range(count)])
        vec = np.concatenate([oracle.random_vector(st, n, 2 * mods[i % L][0]) for i in range(count)])
        scal = [oracle.bounded(st, 2 * q) for q, _ in mods]
        d, dv = dev(x), dev(vec)
        inputs.append((d, dv))
        outs.append(x.size)
        specs.append(dict(kind=kind, ntts=[cuda.NTT(n, q, psi) for q, psi in mods], count=count, result=0,
                          operand=ptr(d), vector=ptr(dv) if kind in (3, 4) else 0,
                          scalars=scal if kind == 4 else None, in_f=in_f, out_f=4 if kind != 2 else 1))
    return specs, outs, inputs


def _run(cuda, specs, outs, fn):
    bufs = [dev_empty(size, fill=0xA5A5A5A5) for size in outs]
    for sp, b in zip(specs, bufs):
        sp["result"] = ptr(b)
    fn(specs)
    return [host(b, size) for b, size in zip(bufs, outs)]


def test_static_scratch_batch_matches_allocating_batch_twice(cuda, oracle):
    specs, outs, inputs = _jobs(cuda, oracle)
    want = _run(cuda, specs, outs, cuda.batch_run)
    for call in range(2):  # the shared scratch keeps the previous call's contents
        got = _run(cuda, specs, outs, cuda.batch_run_static)
        for j, (g, w) in enumerate(zip(got, want)):
            np.testing.assert_array_equal(g, w, err_msg=f"call {call} job {j}")


def test_static_scratch_refuses_batches_beyond_its_size(cuda, oracle):
    n, jobs = 1024, 4096
    q = oracle.find_ntt_prime(n, 40)
    t = cuda.NTT(n, q, oracle.find_primitive_root(n, q))
    # 4096 one-limb jobs need about 1.3 MB of descriptors: more than the
    # 1 MiB array.  Every job has its own limb of a real buffer (32 MiB), so
    # nothing could run past an allocation even if the batch got through;
    # it is refused on the host, before any copy or launch.
    d = dev_empty(jobs * n)
    spec = [dict(kind=1, ntts=[t], count=1, result=ptr(d, j * n), operand=ptr(d, j * n), in_f=1, out_f=4)
            for j in range(jobs)]
    with pytest.raises(cuda.AxhelError) as e:
        cuda.batch_run_static(spec)
    assert e.value.status == 4  # AXHEL_ERR_UNSUPPORTED
    assert "static scratch holds 1048576 bytes" in str(e.value)
    # the same batch through the allocating entry point runs
    cuda.batch_run(spec)
