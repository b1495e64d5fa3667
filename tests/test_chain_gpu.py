"""GPU parity of the fused forms against the reference's per-limb call
sequences, run on the oracle: INTT -> MulMod/FMAMod -> NTT chains and the
tensor-product eltwise chain."""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu


def moduli(oracle, n, L, bits0):
    out = []
    for i in range(L):
        q = oracle.find_ntt_prime_near(n, bits0 + (i % 10), i + 1, L + 2)
        psi = oracle.find_primitive_root(n, q)
        out.append((q, psi))
    return out


@pytest.mark.parametrize("n", [8, 1024, 4096, 16384, 65536, 131072])
@pytest.mark.parametrize("op", ["mul", "fma", "fma_noadd"])
def test_chain_matches_call_sequence(cuda, oracle, n, op):
    L, count = 3, 4
    ms = moduli(oracle, n, L, 45)
    ntts = [cuda.NTT(n, q, psi) for q, psi in ms]
    tabs = [oracle.tables(n, q, psi) for q, psi in ms]
    st = oracle.rng(SEED ^ 0xC4A1 ^ n)
    x = np.concatenate([oracle.random_vector(st, n, 4 * ms[i % L][0]) for i in range(count)])
    m = np.concatenate([oracle.random_vector(st, n, 2 * ms[i % L][0]) for i in range(count)])
    scalars = [oracle.bounded(st, 2 * q) for q, _ in ms]
    for in_f, out_f in ((4, 4), (2, 1)):
        xin = x if in_f == 4 else np.concatenate(
            [oracle.reduce(x[i * n:(i + 1) * n], ms[i % L][0], 4, 2) for i in range(count)])
        d, o, dm = dev(xin), dev_empty(xin.size), dev(m)
        if op == "mul":
            cuda.chain_mul_batch(ntts, ptr(o), ptr(d), ptr(dm), count, in_f, out_f)
        else:
            cuda.chain_fma_batch(ntts, ptr(o), ptr(d), scalars, ptr(dm) if op == "fma" else 0, count, in_f, out_f)
        got = host(o)
        for i in range(count):
            q = ms[i % L][0]
            fwd, inv, ninv = tabs[i % L]
            seg = xin[i * n:(i + 1) * n]
            if in_f == 4:
                seg = oracle.reduce(seg, q, 4, 2)
            y = oracle.inverse(seg, q, inv, ninv, 2, 2)
            mi = m[i * n:(i + 1) * n]
            if op == "mul":
                y = oracle.mul(y, mi, q, 2)
            else:
                y = oracle.fma(y, scalars[i % L], mi if op == "fma" else None, q, 2)
            exp = oracle.forward(y, q, fwd, 1, out_f)
            np.testing.assert_array_equal(got[i * n:(i + 1) * n], exp, err_msg=f"limb {i} in_f={in_f}")


@pytest.mark.parametrize("factor", [1, 2, 4])
def test_tensor_product_matches_call_sequence(cuda, oracle, factor):
    n, L, pairs = 4096, 4, 3
    qs = [q for q, _ in moduli(oracle, n, L, 40)]
    count = pairs * L
    st = oracle.rng(SEED ^ 0x7E45 ^ factor)
    bound = lambda i: factor * qs[i % L]
    c0, c1, d0, d1 = (np.concatenate([oracle.random_vector(st, n, bound(i)) for i in range(count)]) for _ in range(4))
    bufs = [dev(v) for v in (c0, c1, d0, d1)]
    outs = [dev_empty(n * count) for _ in range(3)]
    cuda.tensor_product(*[ptr(t) for t in outs], *[ptr(t) for t in bufs], n, count, qs, factor)
    r0, r1, r2 = (host(t) for t in outs)
    for i in range(count):
        q = qs[i % L]
        s = slice(i * n, (i + 1) * n)
        t0 = oracle.mul(c0[s], d0[s], q, factor)
        t1 = oracle.mul(c0[s], d1[s], q, factor)
        u = oracle.mul(c1[s], d0[s], q, factor)
        t1 = oracle.add(t1, u, q)
        t2 = oracle.mul(c1[s], d1[s], q, factor)
        np.testing.assert_array_equal(r0[s], oracle.reduce(t0, q, 4, 1))
        np.testing.assert_array_equal(r1[s], oracle.reduce(t1, q, 4, 1))
        np.testing.assert_array_equal(r2[s], oracle.reduce(t2, q, 4, 1))


@pytest.mark.parametrize("n", [8, 64, 1024, 4096, 16384, 65536, 131072])
def test_product_matches_call_sequence(cuda, oracle, n):
    """The fused NTT -> MulMod -> INTT product equals, limb by limb, the
    reference call sequence ComputeForward(x, 4, 4) -> EltwiseMulMod(., m, 4)
    -> ComputeInverse(2, out_f): lazy and normalized outputs, in place and out
    of place."""
    L, count = 3, 5
    ms = moduli(oracle, n, L, 45)
    ntts = [cuda.NTT(n, q, psi) for q, psi in ms]
    tabs = [oracle.tables(n, q, psi) for q, psi in ms]
    st = oracle.rng(SEED ^ 0x9D0C ^ n)
    x = np.concatenate([oracle.random_vector(st, n, 4 * ms[i % L][0]) for i in range(count)])
    m = np.concatenate([oracle.random_vector(st, n, 4 * ms[i % L][0]) for i in range(count)])
    for out_f in (2, 1):
        exp = []
        for i in range(count):
            q = ms[i % L][0]
            fwd, inv, ninv = tabs[i % L]
            seg = slice(i * n, (i + 1) * n)
            y = oracle.forward(x[seg], q, fwd, 4, 4)
            y = oracle.mul(y, m[seg], q, 4)
            exp.append(oracle.inverse(y, q, inv, ninv, 2, out_f))
        exp = np.concatenate(exp)
        d, o, dm = dev(x), dev_empty(x.size), dev(m)
        cuda.product_batch(ntts, ptr(o), ptr(d), ptr(dm), count, 4, out_f)
        np.testing.assert_array_equal(host(o), exp, err_msg=f"out of place, out_f={out_f}")
        cuda.product_batch(ntts, ptr(d), ptr(d), ptr(dm), count, 4, out_f)
        np.testing.assert_array_equal(host(d), exp, err_msg=f"in place, out_f={out_f}")
    with pytest.raises(cuda.AxhelError):  # the multiplicand may not be the result
        cuda.product_batch(ntts, ptr(dm), ptr(d), ptr(dm), count, 4, 1)


@pytest.mark.parametrize("n", [8, 1024, 4096, 16384, 65536, 131072])
@pytest.mark.parametrize("count", [1, 5, 80])
def test_forward_mul_and_mul_inverse_match_call_sequences(cuda, oracle, n, count):
    """The dyadic product fused after a forward transform equals
    ComputeForward(x, 4, 4) -> EltwiseMulMod(., m, 4), and fused ahead of an
    inverse equals EltwiseMulMod(x, m, 4) -> ComputeInverse(2, out_f), limb by
    limb; one limb and a few take the one-launch cluster form at 2^10..2^15,
    80 limbs the pass form."""
    if n * count > (1 << 21):
        count = max(1, (1 << 21) // n)
    L = 3
    ms = moduli(oracle, n, L, 47)
    ntts = [cuda.NTT(n, q, psi) for q, psi in ms]
    tabs = [oracle.tables(n, q, psi) for q, psi in ms]
    st = oracle.rng(SEED ^ 0xF3A1 ^ n ^ count)
    x = np.concatenate([oracle.random_vector(st, n, 4 * ms[i % L][0]) for i in range(count)])
    m = np.concatenate([oracle.random_vector(st, n, 4 * ms[i % L][0]) for i in range(count)])
    segs = [slice(i * n, (i + 1) * n) for i in range(count)]
    exp_f = np.concatenate([oracle.mul(oracle.forward(x[s], ms[i % L][0], tabs[i % L][0], 4, 4), m[s],
                                       ms[i % L][0], 4) for i, s in enumerate(segs)])
    d, o, dm = dev(x), dev_empty(x.size), dev(m)
    cuda.forward_mul_batch(ntts, ptr(o), ptr(d), ptr(dm), count)
    np.testing.assert_array_equal(host(o), exp_f, err_msg="forward then MulMod, out of place")
    cuda.forward_mul_batch(ntts, ptr(d), ptr(d), ptr(dm), count)
    np.testing.assert_array_equal(host(d), exp_f, err_msg="forward then MulMod, in place")
    for out_f in (2, 1):
        exp_i = np.concatenate([oracle.inverse(oracle.mul(x[s], m[s], ms[i % L][0], 4), ms[i % L][0],
                                               tabs[i % L][1], tabs[i % L][2], 2, out_f) for i, s in enumerate(segs)])
        d = dev(x)
        cuda.mul_inverse_batch(ntts, ptr(o), ptr(d), ptr(dm), count, out_f)
        np.testing.assert_array_equal(host(o), exp_i, err_msg=f"MulMod then inverse, out_f={out_f}")
        cuda.mul_inverse_batch(ntts, ptr(d), ptr(d), ptr(dm), count, out_f)
        np.testing.assert_array_equal(host(d), exp_i, err_msg=f"MulMod then inverse in place, out_f={out_f}")
    with pytest.raises(cuda.AxhelError):  # the multiplicand may not be the result
        cuda.forward_mul_batch(ntts, ptr(dm), ptr(d), ptr(dm), count)
    with pytest.raises(cuda.AxhelError):
        cuda.mul_inverse_batch(ntts, ptr(dm), ptr(d), ptr(dm), count, 1)
