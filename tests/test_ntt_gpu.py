"""GPU parity of the NTT/INTT (C-ABI) against the oracle, bit for bit,
including the lazy [0,4q) / [0,2q) representatives.  Restates the reference's
tests/public/test_ntt.cpp cases, plus batched and per-plan coverage."""
import numpy as np
import pytest

from helpers import (MODULUS_BITS, NTT_DEGREES, SEED, barrett_cases, dev, dev_empty, host, ntt_params, ptr)

pytestmark = pytest.mark.gpu


def special_input(n, q, pattern):
    """test_ntt.cpp:15-30"""
    v = np.zeros(n, np.uint64)
    if pattern == 1:
        v[0] = 1
    elif pattern == 2:
        v[:] = 1
    elif pattern == 3:
        v[:] = q - 1
    elif pattern == 4:
        v[1::2] = q - 1
    elif pattern == 5:
        v[-1] = q - 1
    return v


def gpu_fwd(cuda, ntt, x, in_f=1, out_f=1, inplace=True):
    d = dev(x)
    if inplace:
        ntt.forward(ptr(d), ptr(d), in_f, out_f)
        return host(d)
    o = dev_empty(x.size)
    ntt.forward(ptr(o), ptr(d), in_f, out_f)
    return host(o)


def gpu_inv(cuda, ntt, x, in_f=1, out_f=1, inplace=True):
    d = dev(x)
    if inplace:
        ntt.inverse(ptr(d), ptr(d), in_f, out_f)
        return host(d)
    o = dev_empty(x.size)
    ntt.inverse(ptr(o), ptr(d), in_f, out_f)
    return host(o)


def test_known_vector_n8_q17(cuda):
    """test_ntt.cpp:32-46"""
    ntt = cuda.NTT(8, 17, 3)
    x = np.arange(1, 9, dtype=np.uint64)
    y = gpu_fwd(cuda, ntt, x, 1, 1)
    assert y.tolist() == [5, 0, 13, 8, 9, 11, 5, 8]
    assert gpu_inv(cuda, ntt, y, 1, 1).tolist() == list(range(1, 9))


def test_tables_match_oracle(cuda, oracle):
    for n in (8, 1024, 65536, 131072):
        for bits in (30, 50, 62):
            q, psi = ntt_params(oracle, n, bits)
            ntt = cuda.NTT(n, q, psi)
            got = ntt.read_tables()
            exp = oracle.tables(n, q, psi)
            for g, e in zip(got, exp):
                np.testing.assert_array_equal(g, e)


def test_external_tables_example_n8(cuda):
    """The explicit N=8, q=17 tables of example/example.cpp:314-345."""
    fwd = np.array([[1, 1085102592571150095], [13, 14106333703424951235], [9, 9765923333140350855],
                    [15, 16276538888567251425], [3, 3255307777713450285], [5, 5425512962855750475],
                    [10, 10851025925711500950], [11, 11936128518282651045]], np.uint64)
    inv = np.array([[0, 0], [6, 6510615555426900570], [7, 7595718147998050665], [12, 13021231110853801140],
                    [14, 15191436295996101330], [2, 2170205185142300190], [8, 8680820740569200760],
                    [4, 4340410370284600380]], np.uint64)
    ninv = np.array([15, 16276538888567251425], np.uint64)
    ntt = cuda.NTT(8, 17, tables=(fwd, inv, ninv))
    x = np.arange(1, 9, dtype=np.uint64)
    y = gpu_fwd(cuda, ntt, x)
    assert y.tolist() == [5, 0, 13, 8, 9, 11, 5, 8]
    assert gpu_inv(cuda, ntt, y).tolist() == list(range(1, 9))


@pytest.mark.parametrize("n", NTT_DEGREES + [65536, 131072])
def test_forward_inverse_bitexact_lazy_and_normalized(cuda, oracle, n):
    """Lazy outputs are algorithm-dependent: they must equal the reference's exactly."""
    st = oracle.rng(SEED ^ n)
    bits_list = MODULUS_BITS if n <= 16384 else [50, 59, 62]
    for bits in bits_list:
        q, psi = ntt_params(oracle, n, bits)
        ntt = cuda.NTT(n, q, psi)
        fwd, inv, ninv = oracle.tables(n, q, psi)
        x = oracle.random_vector(st, n, 4 * q)
        for out_f in (4, 1, 2):
            np.testing.assert_array_equal(gpu_fwd(cuda, ntt, x, 4, out_f), oracle.forward(x, q, fwd, 4, out_f),
                                          err_msg=f"fwd n={n} bits={bits} out_f={out_f}")
        y = oracle.random_vector(st, n, 2 * q)
        for out_f in (2, 1):
            np.testing.assert_array_equal(gpu_inv(cuda, ntt, y, 2, out_f),
                                          oracle.inverse(y, q, inv, ninv, 2, out_f),
                                          err_msg=f"inv n={n} bits={bits} out_f={out_f}")


@pytest.mark.parametrize("n", [8, 64, 1024, 32768])
def test_special_patterns_normalized_vs_lazy(cuda, oracle, n):
    """test_ntt.cpp:59-79"""
    for bits in MODULUS_BITS:
        q, psi = ntt_params(oracle, n, bits)
        ntt = cuda.NTT(n, q, psi)
        for pat in range(6):
            a = special_input(n, q, pat)
            norm = gpu_fwd(cuda, ntt, a, 1, 1)
            lazy = gpu_fwd(cuda, ntt, a, 1, 4)
            assert (norm < q).all() and (lazy < 4 * q).all()
            np.testing.assert_array_equal(norm, lazy % np.uint64(q))


@pytest.mark.parametrize("n", [8, 256, 4096, 16384, 65536])
def test_round_trips(cuda, oracle, n):
    """test_ntt.cpp:81-162: factor-4 forward input, factor-2 inverse input and
    the lazy composition forward(1,4) -> ReduceMod(4,2) -> inverse(2,1)."""
    st = oracle.rng(SEED ^ 0x4E5454 ^ n)
    for bits in (MODULUS_BITS if n <= 4096 else [40, 59, 62]):
        q, psi = ntt_params(oracle, n, bits)
        ntt = cuda.NTT(n, q, psi)
        orig = oracle.random_vector(st, n, q)
        lazy_in = orig + (np.arange(n, dtype=np.uint64) % 4) * np.uint64(q)
        spec = gpu_fwd(cuda, ntt, orig, 1, 1)
        np.testing.assert_array_equal(gpu_fwd(cuda, ntt, lazy_in, 4, 1), spec)
        spec2 = spec.copy()
        spec2[1::2] += np.uint64(q)
        np.testing.assert_array_equal(gpu_inv(cuda, ntt, spec2, 2, 1), orig)
        x = gpu_fwd(cuda, ntt, orig, 1, 4)
        assert (x < 4 * q).all()
        d = dev(x)
        cuda.reduce(ptr(d), ptr(d), n, q, 4, 2)
        x2 = host(d)
        assert (x2 < 2 * q).all()
        np.testing.assert_array_equal(gpu_inv(cuda, ntt, x2, 2, 1), orig)
        y = gpu_inv(cuda, ntt, spec, 1, 2)
        assert (y < 2 * q).all()
        np.testing.assert_array_equal(y % np.uint64(q), orig)


def test_critical_modulus_variants(cuda, oracle):
    """test_ntt.cpp:164-184"""
    n = 1024
    st = oracle.rng(SEED ^ 0x4E545451564152)
    for bits, q, _ in barrett_cases(oracle):
        if bits not in (50, 52, 59, 60, 61, 62):
            continue
        psi = oracle.find_primitive_root(n, q)
        ntt = cuda.NTT(n, q, psi)
        fwd, inv, ninv = oracle.tables(n, q, psi)
        for _ in range(2):
            orig = oracle.random_vector(st, n, q)
            x = gpu_fwd(cuda, ntt, orig, 1, 4)
            np.testing.assert_array_equal(x, oracle.forward(orig, q, fwd, 1, 4))
            x = oracle.reduce(x, q, 4, 2)
            np.testing.assert_array_equal(gpu_inv(cuda, ntt, x, 2, 1), orig)


@pytest.mark.parametrize("n", [8, 128, 1024, 8192, 32768, 131072])
def test_out_of_place_matches_in_place(cuda, oracle, n):
    """test_ntt.cpp:186-207"""
    q, psi = ntt_params(oracle, n, 62)
    ntt = cuda.NTT(n, q, psi)
    x = oracle.random_vector(oracle.rng(SEED ^ n), n, q)
    a = gpu_fwd(cuda, ntt, x, inplace=True)
    b = gpu_fwd(cuda, ntt, x, inplace=False)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(gpu_inv(cuda, ntt, a, inplace=False), x)


@pytest.mark.parametrize("n", [4096, 16384, 65536])
def test_batch_matches_per_limb(cuda, oracle, n):
    """Batched launches (limb i uses modulus i % L) equal per-limb results bit for bit."""
    L, count = 5, 13
    ntts, tabs, qs = [], [], []
    for i in range(L):
        q = oracle.find_ntt_prime_near(n, 50 + i, 1, 3)
        psi = oracle.find_primitive_root(n, q)
        ntts.append(cuda.NTT(n, q, psi))
        tabs.append(oracle.tables(n, q, psi))
        qs.append(q)
    st = oracle.rng(SEED ^ 0xBA7C4 ^ n)
    x = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % L]) for i in range(count)])
    d = dev(x)
    o = dev_empty(x.size)
    cuda.forward_batch(ntts, ptr(o), ptr(d), count, 1, 4)
    got = host(o)
    for i in range(count):
        k = i % L
        np.testing.assert_array_equal(got[i * n:(i + 1) * n],
                                      oracle.forward(x[i * n:(i + 1) * n], qs[k], tabs[k][0], 1, 4))
    # inverse with the fused ReduceMod(4 -> 2) on load, normalized output
    cuda.inverse_batch(ntts, ptr(o), ptr(o), count, 4, 1)
    back = host(o)
    for i in range(count):
        k = i % L
        lazy = got[i * n:(i + 1) * n]
        exp = oracle.inverse(oracle.reduce(lazy, qs[k], 4, 2), qs[k], tabs[k][1], tabs[k][2], 2, 1)
        np.testing.assert_array_equal(back[i * n:(i + 1) * n], exp)
        np.testing.assert_array_equal(back[i * n:(i + 1) * n], x[i * n:(i + 1) * n] % np.uint64(qs[k]))


def plan_candidates(logn, inverse):
    """A spread of valid pass splits for the autotuner's search space."""
    out = []
    if logn <= 13:
        for lr in (3, 4, 5):
            if lr <= logn:
                out.append([(logn, lr, 1)])
    for a in range(max(1, logn - 13), min(13, logn - 1) + 1):
        b = logn - a
        for lr in (3, 4, 5):
            if lr > a or lr > b:
                continue
            for tga in (4, 16):
                for tgb in (1, 8):
                    col = (a, lr, min(tga, 1 << b))
                    row = (b, lr, min(tgb, 1 << a))
                    out.append([row, col] if inverse else [col, row])
    return out


@pytest.mark.parametrize("logn", [6, 10, 12, 14, 16, 17])
def test_every_plan_bitexact(cuda, oracle, logn):
    """Each autotuner candidate split computes the same bits."""
    n = 1 << logn
    q, psi = ntt_params(oracle, n, 59)
    ntt = cuda.NTT(n, q, psi)
    fwd, inv, ninv = oracle.tables(n, q, psi)
    st = oracle.rng(SEED ^ 0x9 ^ logn)
    count = 3
    x = np.concatenate([oracle.random_vector(st, n, 4 * q) for _ in range(count)])
    y = np.concatenate([oracle.random_vector(st, n, 2 * q) for _ in range(count)])
    ef = np.concatenate([oracle.forward(x[i * n:(i + 1) * n], q, fwd, 4, 4) for i in range(count)])
    ei = np.concatenate([oracle.inverse(y[i * n:(i + 1) * n], q, inv, ninv, 2, 2) for i in range(count)])
    checked = 0
    try:
        for inverse in (False, True):
            for plan in plan_candidates(logn, inverse):
                # skip splits whose tile widths are invalid for this direction
                try:
                    cuda.plan_set(inverse, logn, plan)
                except cuda.AxhelError:
                    continue
                src = dev(y if inverse else x)
                o = dev_empty(src.numel())
                if inverse:
                    cuda.inverse_batch([ntt], ptr(o), ptr(src), count, 2, 2)
                else:
                    cuda.forward_batch([ntt], ptr(o), ptr(src), count, 4, 4)
                np.testing.assert_array_equal(host(o), ei if inverse else ef, err_msg=f"inverse={inverse} {plan}")
                checked += 1
    finally:
        cuda.plan_set(False, logn, [])
        cuda.plan_set(True, logn, [])
    assert checked >= 2


def test_rejects_bad_arguments(cuda, oracle):
    with pytest.raises(cuda.AxhelError):
        cuda.NTT(12, 97, 3)  # not a power of two
    with pytest.raises(cuda.AxhelError):
        cuda.NTT(1 << 18, 2 ** 61 - 1, 3)  # degree beyond the supported maximum
    with pytest.raises(cuda.AxhelError):
        cuda.NTT(8, 2 ** 62 + 1, 3)  # modulus too wide


def schoolbook_negacyclic(a, b, q):
    """Product in Z_q[x]/(x^n + 1) the quadratic way (test_polymul.cpp)."""
    n = len(a)
    A = [int(v) for v in a]
    B = np.array([int(v) for v in b], dtype=object)
    acc = np.zeros(2 * n, dtype=object)
    for i in range(n):
        acc[i:i + n] += A[i] * B
    return np.array([(acc[k] - acc[k + n]) % q for k in range(n)], dtype=np.uint64)


@pytest.mark.parametrize("n", [64, 256, 512])
def test_polymul_matches_schoolbook(cuda, oracle, n):
    """test_polymul.cpp:236-292 on the GPU path: ComputeForward on both
    factors, EltwiseMulMod, ComputeInverse is the negacyclic product -- an
    algorithm-independent check -- with lazy ([0,4q), MulMod factor 4) and
    normalized forward outputs, widths up to 62 bits."""
    st = oracle.rng(SEED ^ 0x504F4C59 ^ n)
    for bits in (30, 50, 61, 62):
        q, psi = ntt_params(oracle, n, bits)
        t = cuda.NTT(n, q, psi)
        a, b = oracle.random_vector(st, n, q), oracle.random_vector(st, n, q)
        want = schoolbook_negacyclic(a, b, q)
        da, db, dc = dev(a), dev(b), dev_empty(n)
        t.forward(ptr(da), ptr(da), 1, 4)   # lazy forward outputs feed MulMod with factor 4
        t.forward(ptr(db), ptr(db), 1, 4)
        cuda.mul(ptr(dc), ptr(da), ptr(db), n, q, 4)
        t.inverse(ptr(dc), ptr(dc), 1, 1)
        np.testing.assert_array_equal(host(dc, n), want, err_msg=f"per call, q bits {bits}")
        # normalized forward outputs, MulMod factor 1
        A, B = dev(a), dev(b)
        t.forward(ptr(A), ptr(A), 1, 1)
        t.forward(ptr(B), ptr(B), 1, 1)
        prod = dev_empty(n)
        cuda.mul(ptr(prod), ptr(A), ptr(B), n, q, 1)  # dyadic product in the NTT domain
        t.inverse(ptr(prod), ptr(prod), 1, 1)
        np.testing.assert_array_equal(host(prod, n), want, err_msg=f"normalized, q bits {bits}")
        # the fused NTT -> MulMod -> INTT product, with b's lazy forward as multiplicand
        db = dev(b)
        t.forward(ptr(db), ptr(db), 1, 4)
        da, out = dev(a), dev_empty(n)
        cuda.product_batch([t], ptr(out), ptr(da), ptr(db), 1, 1, 1)
        np.testing.assert_array_equal(host(out, n), want, err_msg=f"fused product, q bits {bits}")


def test_refresh_external_tables(cuda, oracle):
    """axhel_cuda_ntt_refresh_external: a handle made from external tables
    re-reads them (the reference borrows them); other handles refuse."""
    import ctypes as C

    n = 1024
    q, psi1 = ntt_params(oracle, n, 50)
    psi2 = oracle.pow_mod(psi1, 3, q)
    f1, i1, n1 = oracle.tables(n, q, psi1)
    f2, i2, n2 = oracle.tables(n, q, psi2)
    t = cuda.NTT(n, q, tables=(f1, i1, n1))
    x = oracle.random_vector(oracle.rng(SEED ^ 0xEF), n, q)
    d, o = dev(x), dev_empty(n)
    t.forward(ptr(o), ptr(d), 1, 4)
    np.testing.assert_array_equal(host(o, n), oracle.forward(x, q, f1, 1, 4))
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    L = cuda.lib()
    assert L.axhel_cuda_ntt_refresh_external(t.h, P(f2), P(i2), P(n2), None) == 0
    t.forward(ptr(o), ptr(d), 1, 4)
    np.testing.assert_array_equal(host(o, n), oracle.forward(x, q, f2, 1, 4))
    t.inverse(ptr(o), ptr(d), 1, 1)
    np.testing.assert_array_equal(host(o, n), oracle.inverse(x, q, i2, n2, 1, 1))
    auto = cuda.NTT(n, q, psi1)
    assert L.axhel_cuda_ntt_refresh_external(auto.h, P(f2), None, None, None) == 1  # not an external-table handle
    assert L.axhel_cuda_ntt_refresh_external(t.h, None, P(i2), None, None) == 1  # inverse table without N^-1
