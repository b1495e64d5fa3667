"""GPU: the benchmark configurations' own call sequences against the
reference native backend compiled from its sources (oracle/_ref), bit for
bit -- the plain single-limb round trip (N = 4096, a 50-bit prime
q = 1 mod 8192: ComputeForward(1,1), EltwiseMulMod of two such vectors,
EltwiseAddMod with a scalar, ComputeInverse normalized), and the batched
RNS round trip of the headline workload on a slice of its limbs (24 primes
of 50-59 bits, q = 1 mod 2^17, forward(1,4), inverse(4,1))."""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pos", [1, 2, 3])
def test_plain_single_limb_round_trip(cuda, oracle, reference, pos):
    n = 4096
    q = oracle.find_ntt_prime_near(n, 50, pos, 4)
    assert q % (2 * n) == 1 and q.bit_length() == 50
    psi = oracle.find_primitive_root(n, q)
    st = oracle.rng(SEED ^ (0xC1 + pos))
    a, b = oracle.random_vector(st, n, q), oracle.random_vector(st, n, q)
    s = oracle.bounded(st, q)
    # the reference, on the host
    r = reference.ntt(n, q, psi)
    A, B = r.forward(a, 1, 1), r.forward(b, 1, 1)
    want = r.inverse(reference.add(reference.mul(A, B, q, 1), s, q), 1, 1)
    # the same calls on the GPU, through the C-ABI
    t = cuda.NTT(n, q, psi)
    da, db, dc = dev(a), dev(b), dev_empty(n)
    t.forward(ptr(da), ptr(da), 1, 1)
    t.forward(ptr(db), ptr(db), 1, 1)
    np.testing.assert_array_equal(host(da, n), A)
    cuda.mul(ptr(dc), ptr(da), ptr(db), n, q, 1)
    cuda.add(ptr(dc), ptr(dc), s, n, q, scalar=True)
    t.inverse(ptr(dc), ptr(dc), 1, 1)
    np.testing.assert_array_equal(host(dc, n), want)


def test_headline_round_trip_slice_against_reference(cuda, reference):
    """The bench step (forward lazy, fused ReduceMod 4->2, inverse normalized)
    on 48 of its 768 limbs, each limb checked against the reference's
    ComputeForward(1,4) / EltwiseReduceMod(4,2) / ComputeInverse(2,1)."""
    import bench

    mods = bench.workload_moduli()
    count = 48
    data = bench.make_inputs(mods, count)
    ntts = [cuda.NTT(bench.N, q, psi) for q, psi in mods]
    x = dev(data.reshape(-1))
    y = dev_empty(data.size)
    cuda.forward_batch(ntts, ptr(y), ptr(x), count, 1, 4)
    fwd = host(y, data.size).reshape(count, bench.N)
    cuda.inverse_batch(ntts, ptr(y), ptr(y), count, 4, 1)
    back = host(y, data.size).reshape(count, bench.N)
    refs = [reference.ntt(bench.N, q, psi) for q, psi in mods]
    for i in range(count):
        q = mods[i % 24][0]
        r = refs[i % 24]
        f = r.forward(data[i], 1, 4)
        np.testing.assert_array_equal(fwd[i], f, err_msg=f"forward limb {i}")
        inv = r.inverse(reference.reduce(f, q, 4, 2), 2, 1)
        np.testing.assert_array_equal(back[i], inv, err_msg=f"inverse limb {i}")
        np.testing.assert_array_equal(back[i], data[i])
