"""GPU parity of the element-wise kernels (C-ABI) against the oracle and the
u128 reference formulas, restating tests/public/test_eltwise.cpp and
tests/public/test_reduce.cpp: boundary values for every mod-factor and every
Barrett width 20..62, seeded random inputs, aliasing, unaligned offsets and
guard canaries around the output."""
import numpy as np
import pytest

from helpers import (MODULUS_BITS, SEED, barrett_cases, boundary_values, boundary_values_u64, dev, dev_empty,
                     element_sizes, host, pattern, ptr)

pytestmark = pytest.mark.gpu

LEFT, RIGHT = 0x13579BDF2468ACE0, 0xFDB97531ECA86420  # canaries, test_eltwise.cpp:29-30
GUARD = 8


def guarded(cuda_vals, n, fill=0):
    """A device buffer with GUARD canary words on each side; returns (buf, base offset)."""
    a = np.full(n + 2 * GUARD, fill, np.uint64)
    a[:GUARD] = LEFT
    a[GUARD + n:] = RIGHT
    if cuda_vals is not None:
        a[GUARD:GUARD + n] = cuda_vals
    return dev(a)


def check_guards(buf, n):
    h = host(buf, n + 2 * GUARD)
    assert (h[:GUARD] == LEFT).all() and (h[GUARD + n:] == RIGHT).all(), "canary overwritten"
    return h[GUARD:GUARD + n]


def run_vv(cuda, fn, a, b, q, *extra):
    n = a.size
    da, db, do = guarded(a, n), guarded(b, n), guarded(None, n)
    fn(ptr(do, GUARD), ptr(da, GUARD), ptr(db, GUARD), n, q, *extra)
    out = check_guards(do, n)
    np.testing.assert_array_equal(check_guards(da, n), a)
    np.testing.assert_array_equal(check_guards(db, n), b)
    return out


def py_add(a, b, q):
    return ((a.astype(object) + b.astype(object)) % q).astype(np.uint64)


def py_sub(a, b, q):
    return ((a.astype(object) - b.astype(object)) % q).astype(np.uint64)


def py_mul(a, b, q):
    return ((a.astype(object) % q) * (b.astype(object) % q) % q).astype(np.uint64)


SIZES = [n for n in element_sizes() if n <= 8193]


def test_add_sub_boundary_vector_vector(cuda, oracle):
    for bits in MODULUS_BITS:
        q = oracle.find_ntt_prime(1024, bits)
        vals = boundary_values(q, 1)
        for n in SIZES:
            a, b = pattern(n, vals), pattern(n, vals[::-1])
            if n == 0:
                cuda.add(0, 0, 0, 0, q)  # n == 0 is a no-op, null pointers allowed
                continue
            np.testing.assert_array_equal(run_vv(cuda, cuda.add, a, b, q), py_add(a, b, q))
            np.testing.assert_array_equal(run_vv(cuda, cuda.sub, a, b, q), py_sub(a, b, q))


def test_add_sub_vector_scalar_corners(cuda, oracle):
    for bits in MODULUS_BITS:
        q = oracle.find_ntt_prime(1024, bits)
        vals = boundary_values(q, 1)
        a = pattern(5, vals)
        for s in vals:
            da, do = dev(a), dev_empty(5)
            cuda.add(ptr(do), ptr(da), s, 5, q, scalar=True)
            np.testing.assert_array_equal(host(do, 5), py_add(a, np.full(5, s, np.uint64), q))
            cuda.sub(ptr(do), ptr(da), s, 5, q, scalar=True)
            np.testing.assert_array_equal(host(do, 5), py_sub(a, np.full(5, s, np.uint64), q))


def test_mul_boundary_all_factors_all_barrett_widths(cuda, oracle):
    for bits, q, _ in barrett_cases(oracle):
        for f in (1, 2, 4):
            vals = boundary_values(q, f)
            for n in (1, 3, 33, 257, 1025):
                a, b = pattern(n, vals), pattern(n, vals[::-1])
                got = run_vv(cuda, cuda.mul, a, b, q, f)
                np.testing.assert_array_equal(got, py_mul(a, b, q), err_msg=f"bits={bits} f={f} n={n}")


def test_mul_random_all_barrett_widths(cuda, oracle):
    st = oracle.rng(SEED)
    for bits, q, var in barrett_cases(oracle):
        for f in (1, 2, 4):
            n = 4099
            a = oracle.random_vector(st, n, q * f)
            b = oracle.random_vector(st, n, q * f)
            da, db, do = dev(a), dev(b), dev_empty(n)
            cuda.mul(ptr(do), ptr(da), ptr(db), n, q, f)
            np.testing.assert_array_equal(host(do, n), oracle.mul(a, b, q, f), err_msg=f"bits={bits} q={q} f={f}")


def test_fma_boundary_and_random(cuda, oracle):
    st = oracle.rng(SEED ^ 0x464D4152414E44)
    for bits, q, _ in barrett_cases(oracle):
        for f in (1, 2, 4, 8):
            vals = boundary_values_u64(q, f)
            n = 257
            a, c = pattern(n, vals), pattern(n, vals[::-1])
            s = vals[len(vals) // 2]
            exp = ((a.astype(object) % q) * (s % q) + (c.astype(object) % q)) % q
            got = run_vv(cuda, lambda o, x, y, n_, q_: cuda.fma(o, x, s, y, n_, q_, f), a, c, q)
            np.testing.assert_array_equal(got, exp.astype(np.uint64), err_msg=f"bits={bits} f={f}")
            bound = min(q * f, 2 ** 64 - 1)
            a = oracle.random_vector(st, 1031, bound)
            c = oracle.random_vector(st, 1031, bound)
            s = oracle.bounded(st, bound)
            da, dc, do = dev(a), dev(c), dev_empty(1031)
            cuda.fma(ptr(do), ptr(da), s, ptr(dc), 1031, q, f)
            np.testing.assert_array_equal(host(do, 1031), oracle.fma(a, s, c, q, f))
            cuda.fma(ptr(do), ptr(da), s, 0, 1031, q, f)  # null addend == plain multiply
            np.testing.assert_array_equal(host(do, 1031), oracle.fma(a, s, None, q, f))


def test_unsupported_factor_leaves_result_untouched(cuda, oracle):
    q = oracle.find_ntt_prime(1024, 50)
    a = np.arange(100, dtype=np.uint64)
    da, do = dev(a), dev_empty(100, fill=0xDEADBEEF)
    cuda.mul(ptr(do), ptr(da), ptr(da), 100, q, 3)
    cuda.fma(ptr(do), ptr(da), 5, 0, 100, q, 16)
    cuda.reduce(ptr(do), ptr(da), 100, q, 4, 4)
    cuda.reduce(ptr(do), ptr(da), 100, q, 8, 1)
    assert (host(do, 100) == 0xDEADBEEF).all()


@pytest.mark.parametrize("pair", [(1, 1), (1, 2), (2, 2), (2, 1), (4, 1), (4, 2), (0, 2)])
def test_reduce_pairs_match_oracle(cuda, oracle, pair):
    """test_reduce.cpp:117-268: identity, thresholds, random; in and out of place."""
    in_f, out_f = pair
    st = oracle.rng(SEED ^ 0x524544554345)
    for bits in MODULUS_BITS:
        q = oracle.find_ntt_prime(1024, bits)
        bound = q * max(in_f, 1)
        for n in (0, 1, 7, 9, 8193):
            x = np.concatenate([pattern(min(n, 20), boundary_values(q, max(in_f, 1))),
                                oracle.random_vector(st, max(n - 20, 0), bound)])[:n]
            exp = oracle.reduce(x, q, in_f, out_f, out=np.full(n, 7, np.uint64))
            if n == 0:
                cuda.reduce(0, 0, 0, q, in_f, out_f)
                continue
            d, o = dev(x), dev_empty(n, fill=7)
            cuda.reduce(ptr(o), ptr(d), n, q, in_f, out_f)
            np.testing.assert_array_equal(host(o, n), exp)
            cuda.reduce(ptr(d), ptr(d), n, q, in_f, out_f)
            np.testing.assert_array_equal(host(d, n), exp)


def test_reduce_barrett_arbitrary_u64(cuda, oracle):
    """The in_factor == modulus branch (eltwise-reduce-mod.cpp:109-127), any uint64 input."""
    st = oracle.rng(SEED ^ 0xBA77E77)
    for bits, q, _ in barrett_cases(oracle):
        x = np.concatenate([oracle.random_vector(st, 3000, 2 ** 64 - 1),
                            np.array([0, 1, q - 1, q, q + 1, 2 ** 64 - 1, 2 ** 63, q * q % 2 ** 64], np.uint64)])
        d, o = dev(x), dev_empty(x.size)
        cuda.reduce(ptr(o), ptr(d), x.size, q, q, 1)
        got = host(o, x.size)
        np.testing.assert_array_equal(got, oracle.reduce(x, q, q, 1))
        np.testing.assert_array_equal(got, (x.astype(object) % q).astype(np.uint64))


def test_in_place_aliasing(cuda, oracle):
    """test_eltwise.cpp:439-516"""
    q = oracle.find_ntt_prime(1024, 50)
    vals = boundary_values(q, 1)
    n = 7
    a, b = pattern(n, vals), pattern(n, vals[::-1])
    for fn, ref in ((cuda.add, py_add), (cuda.sub, py_sub)):
        d1, d2 = dev(a), dev(b)
        fn(ptr(d1), ptr(d1), ptr(d2), n, q)
        np.testing.assert_array_equal(host(d1, n), ref(a, b, q))
        d1, d2 = dev(a), dev(b)
        fn(ptr(d2), ptr(d1), ptr(d2), n, q)
        np.testing.assert_array_equal(host(d2, n), ref(a, b, q))
    d = dev(a)
    cuda.sub(ptr(d), ptr(d), ptr(d), n, q)
    assert (host(d, n) == 0).all()
    d1, d2 = dev(a), dev(b)
    cuda.mul(ptr(d1), ptr(d1), ptr(d2), n, q, 1)
    np.testing.assert_array_equal(host(d1, n), py_mul(a, b, q))


def test_unaligned_offsets(cuda, oracle):
    """test_eltwise.cpp:518-561: 8-byte aligned but not 16-byte aligned pointers."""
    q = oracle.find_ntt_prime(1024, 50)
    n = 4103
    i = np.arange(n, dtype=np.uint64)
    for off in range(4):
        sa = np.zeros(n + 8, np.uint64)
        sb = np.zeros(n + 8, np.uint64)
        sa[off:off + n] = (i * 17 + 3) % q
        sb[off:off + n] = (i * 29 + 5) % q
        da, db, do = dev(sa), dev(sb), dev_empty(n + 8)
        a, b = sa[off:off + n], sb[off:off + n]
        cuda.add(ptr(do, off), ptr(da, off), ptr(db, off), n, q)
        np.testing.assert_array_equal(host(do)[off:off + n], py_add(a, b, q))
        cuda.sub(ptr(do, off), ptr(da, off), ptr(db, off), n, q)
        np.testing.assert_array_equal(host(do)[off:off + n], py_sub(a, b, q))
        cuda.mul(ptr(do, off), ptr(da, off), ptr(db, off), n, q, 1)
        np.testing.assert_array_equal(host(do)[off:off + n], py_mul(a, b, q))


def test_guard_canaries_mul4_fma8_62bit(cuda, oracle):
    """test_eltwise.cpp:563-636 on the widest lazy domains with a 62-bit q."""
    q = oracle.find_ntt_prime(1024, 62)
    for n in (1, 2, 3, 31, 32, 33, 127, 129, 1023, 1025, 8191, 8193):
        v4 = boundary_values(q, 4)
        m1, m2 = pattern(n, v4), pattern(n, v4[::-1])
        np.testing.assert_array_equal(run_vv(cuda, cuda.mul, m1, m2, q, 4), py_mul(m1, m2, q))
        v8 = boundary_values_u64(q, 8)
        f1, f3 = pattern(n, v8), pattern(n, v8[::-1])
        s = v8[len(v8) // 2]
        got = run_vv(cuda, lambda o, x, y, n_, q_: cuda.fma(o, x, s, y, n_, q_, 8), f1, f3, q)
        exp = ((f1.astype(object) % q) * (s % q) + f3.astype(object) % q) % q
        np.testing.assert_array_equal(got, exp.astype(np.uint64))


def test_large_vectors_all_ops_match_oracle(cuda, oracle):
    """Full-size streaming (2^24 elements) for every op against the oracle."""
    n = 1 << 24
    q = oracle.find_ntt_prime(1 << 16, 59)
    rng = np.random.default_rng(7)
    a = rng.integers(0, 4 * q, n, dtype=np.uint64)
    b = rng.integers(0, 4 * q, n, dtype=np.uint64)
    da, db, do = dev(a), dev(b), dev_empty(n)
    cuda.mul(ptr(do), ptr(da), ptr(db), n, q, 4)
    np.testing.assert_array_equal(host(do, n), oracle.mul(a, b, q, 4))
    cuda.fma(ptr(do), ptr(da), 12345, ptr(db), n, q, 4)
    np.testing.assert_array_equal(host(do, n), oracle.fma(a, 12345, b, q, 4))
    cuda.reduce(ptr(do), ptr(da), n, q, 4, 1)
    np.testing.assert_array_equal(host(do, n), oracle.reduce(a, q, 4, 1))


@pytest.mark.parametrize("in_place", [False, True])
def test_unaligned_large_all_ops(cuda, oracle, in_place):
    """8-byte aligned (not 16-byte) operands long enough for the unaligned
    kernel's four-elements-per-thread steps and its tail: every op against
    the oracle, out of place and in place (result aliasing the first operand)."""
    q = oracle.find_ntt_prime(1 << 16, 59)
    n = (1 << 21) + 5
    st = oracle.rng(SEED ^ 0x51)
    a = oracle.random_vector(st, n, 2 * q)
    b = oracle.random_vector(st, n, 2 * q)
    c = oracle.random_vector(st, n, q)
    cases = [
        (lambda o, x, y, z: cuda.add(o, x, z, n, q), lambda: oracle.add(a % q, c, q), True),
        (lambda o, x, y, z: cuda.sub(o, x, z, n, q), lambda: oracle.sub(a % q, c, q), True),
        (lambda o, x, y, z: cuda.mul(o, x, y, n, q, 2), lambda: oracle.mul(a, b, q, 2), False),
        (lambda o, x, y, z: cuda.fma(o, x, 12345, z, n, q, 2), lambda: oracle.fma(a, 12345, c, q, 2), False),
        (lambda o, x, y, z: cuda.reduce(o, x, n, q, q, 1), lambda: oracle.reduce(a, q, q, 1), False),
    ]
    for k, (run, want, canonical_a) in enumerate(cases):
        x = a % q if canonical_a else a
        da, db, dc = dev_empty(n + 1), dev_empty(n + 1), dev_empty(n + 1)
        da[1:] = dev(x)[:n]
        db[1:] = dev(b)[:n]
        dc[1:] = dev(c)[:n]
        do = da if in_place else dev_empty(n + 1, fill=0)
        run(ptr(do, 1), ptr(da, 1), ptr(db, 1), ptr(dc, 1))
        np.testing.assert_array_equal(host(do, n + 1)[1:], want(), err_msg=f"op {k} in_place={in_place}")
