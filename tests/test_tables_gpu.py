"""GPU: twiddle tables generated on the device (axhel_cuda_ntt_create /
axhel_cuda_ntt_create_many) equal GenerateNTTTables' tables entry for entry
-- roots, Shoup quotients, N^-1 -- for every degree 2..2^17 and modulus
widths 20..62, including batches of more than one launch, duplicate and
cached parameters; invalid parameters are refused without handles."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def params(oracle, degrees, widths, k=1):
    out = []
    for n in degrees:
        for bits in widths:
            q = oracle.find_ntt_prime_near(n, bits, k, 4)
            out.append((n, q, oracle.find_primitive_root(n, q)))
    return out


def check_tables(oracle, t, n, q, psi):
    fwd, inv, ninv = t.read_tables()
    F, I, N = oracle.tables(n, q, psi)
    np.testing.assert_array_equal(fwd, F, err_msg=f"fwd n={n} q={q}")
    np.testing.assert_array_equal(inv, I, err_msg=f"inv n={n} q={q}")
    np.testing.assert_array_equal(ninv, N, err_msg=f"ninv n={n} q={q}")


def test_device_tables_equal_reference_tables(cuda, oracle):
    ps = params(oracle, [2, 4, 8, 16, 1024, 4096], [20, 31, 45, 53, 60, 61, 62], k=2)
    ps += params(oracle, [1 << 15, 1 << 16, 1 << 17], [30, 50, 59, 62], k=3)
    ts = cuda.NTT.create_many(ps)
    for t, (n, q, psi) in zip(ts, ps):
        check_tables(oracle, t, n, q, psi)


# The explicit N = 8, q = 17, psi = 3 tables of the reference's example
# (example/example.cpp:314-345): {w, floor(w 2^64 / q)} pairs.
KAT_FWD = [(1, 1085102592571150095), (13, 14106333703424951235), (9, 9765923333140350855),
           (15, 16276538888567251425), (3, 3255307777713450285), (5, 5425512962855750475),
           (10, 10851025925711500950), (11, 11936128518282651045)]
KAT_INV = [(0, 0), (6, 6510615555426900570), (7, 7595718147998050665), (12, 13021231110853801140),
           (14, 15191436295996101330), (2, 2170205185142300190), (8, 8680820740569200760),
           (4, 4340410370284600380)]
KAT_NINV = (15, 16276538888567251425)


def test_known_answer_tables_n8(cuda, oracle):
    t = cuda.NTT(8, 17, 3)
    fwd, inv, ninv = t.read_tables()
    assert [tuple(int(v) for v in r) for r in fwd] == KAT_FWD
    assert [tuple(int(v) for v in r) for r in inv] == KAT_INV
    assert tuple(int(v) for v in ninv) == KAT_NINV


def test_many_contexts_over_several_launches_and_the_cache(cuda, oracle):
    ps = []
    for i in range(130):  # two launches of at most 96 contexts
        n = 1 << (10 + i % 4)
        q = oracle.find_ntt_prime_near(n, 30 + i % 31, 1 + (i // 31) % 3, 4)  # distinct (n, q) per i
        ps.append((n, q, oracle.find_primitive_root(n, q)))
    ps.append(ps[3])  # a duplicate inside the call shares one context
    l0 = cuda.launch_count()
    ts = cuda.NTT.create_many(ps)
    launches = cuda.launch_count() - l0
    assert ts[3].h.value == ts[-1].h.value
    for t, (n, q, psi) in zip(ts[::7], ps[::7]):
        check_tables(oracle, t, n, q, psi)
    # cached now: the same parameters again launch nothing and share handles
    l1 = cuda.launch_count()
    again = cuda.NTT.create_many(ps[:5])
    assert cuda.launch_count() == l1
    assert [a.h.value for a in again] == [t.h.value for t in ts[:5]]
    assert launches <= 2 or launches == 0  # zero if an earlier test created these already


def test_invalid_parameters_are_refused(cuda, oracle):
    q = oracle.find_ntt_prime(1024, 40)
    psi = oracle.find_primitive_root(1024, q)
    for bad in ([(1024, q + 1, psi)],           # even modulus
                [(1024, q, 0)], [(1024, q, q)],  # root outside [1, q)
                [(1000, q, psi)],                # not a power of two
                [(1024, q, psi), (1 << 18, q, psi)]):  # one bad entry fails the whole call
        with pytest.raises(cuda.AxhelError):
            cuda.NTT.create_many(bad)
