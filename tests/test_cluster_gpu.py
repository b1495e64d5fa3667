"""The single-launch cluster form of small transforms (one thread-block
cluster per limb, the two passes exchanging the limb through distributed
shared memory) against the oracle, for every compiled configuration."""
import numpy as np
import pytest

from helpers import SEED, dev, dev_empty, host, ptr

pytestmark = pytest.mark.gpu

# (first-pass stages, second-pass stages, register stages) compiled in ntt_cluster.cu
COMPILED = [(6, 6, 2), (6, 6, 3), (5, 7, 3), (7, 5, 3), (6, 7, 3), (7, 6, 3), (7, 7, 3), (7, 8, 3), (8, 7, 3),
            (8, 8, 3), (8, 8, 4), (8, 9, 4), (9, 8, 4), (6, 7, 2), (7, 6, 2), (7, 7, 2), (7, 8, 2), (8, 7, 2),
            (5, 5, 2), (5, 6, 2), (6, 5, 2)]


def configs(logn):
    """Valid (lga, lr, csize) for N = 2^logn: threads per CTA in [32, 512]
    (256 at 32 registers per element), at most 16 CTAs, shared memory within
    227 KiB."""
    out = []
    for a, b, lr in COMPILED:
        if a + b != logn:
            continue
        for c in (1, 2, 3, 4):
            lgt = logn - c - lr
            if c > min(a, b) or lgt < 5 or (1 << lgt) > (256 if lr >= 5 else 512):
                continue
            if 2 * 8 * (1 << (logn - c)) > 227 * 1024:
                continue
            out.append((a, lr, 1 << c))
    return out


def moduli(oracle, n, L):
    ntts, tabs, qs = [], [], []
    for i in range(L):
        q = oracle.find_ntt_prime_near(n, 52 + 3 * i, 1, 3)
        psi = oracle.find_primitive_root(n, q)
        ntts.append((q, psi))
        tabs.append(oracle.tables(n, q, psi))
        qs.append(q)
    return ntts, tabs, qs


@pytest.mark.parametrize("logn", [10, 11, 12, 13, 14, 15, 16, 17])
def test_cluster_configs_bitexact(cuda, oracle, logn):
    n = 1 << logn
    # one limb and a few run one wave of clusters (twiddles prefetched into
    # registers up to 2^14); 160 limbs take more than one CTA per SM (the
    # variant without prefetching)
    L, count = 2, (160 if logn <= 14 else 3)
    params, tabs, qs = moduli(oracle, n, L)
    ntts = [cuda.NTT(n, q, psi) for q, psi in params]
    st = oracle.rng(SEED ^ 0xC1A5 ^ logn)
    x = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % L]) for i in range(count)])
    ef4 = [oracle.forward(x[i * n:(i + 1) * n], qs[i % L], tabs[i % L][0], 4, 4) for i in range(count)]
    ef1 = [oracle.forward(x[i * n:(i + 1) * n], qs[i % L], tabs[i % L][0], 4, 1) for i in range(count)]
    # inverse inputs in [0, 4q): the batch form reduces 4 -> 2 on load
    ei2 = [oracle.inverse(oracle.reduce(ef4[i], qs[i % L], 4, 2), qs[i % L], tabs[i % L][1], tabs[i % L][2], 2, 2)
           for i in range(count)]
    ei1 = [oracle.inverse(oracle.reduce(ef4[i], qs[i % L], 4, 2), qs[i % L], tabs[i % L][1], tabs[i % L][2], 2, 1)
           for i in range(count)]
    cfgs = configs(logn)
    assert cfgs
    try:
        for lga, lr, cs in cfgs:
            for inverse in (False, True):
                cuda.cluster_plan_set(inverse, logn, lga, lr, cs, count)
            tag = f"lga={lga} lr={lr} csize={cs}"
            for k in (1, count):
                src = dev(x[:k * n])
                out = dev_empty(k * n)
                cuda.forward_batch(ntts, ptr(out), ptr(src), k, 4, 4)
                got4 = host(out)
                np.testing.assert_array_equal(got4, np.concatenate(ef4[:k]), err_msg=f"forward 4->4 {tag} k={k}")
                cuda.forward_batch(ntts, ptr(src), ptr(src), k, 4, 1)  # in place
                np.testing.assert_array_equal(host(src), np.concatenate(ef1[:k]), err_msg=f"forward ->1 {tag}")
                cuda.inverse_batch(ntts, ptr(src), ptr(out), k, 4, 2)
                np.testing.assert_array_equal(host(src), np.concatenate(ei2[:k]), err_msg=f"inverse ->2 {tag}")
                cuda.inverse_batch(ntts, ptr(out), ptr(out), k, 4, 1)  # in place
                np.testing.assert_array_equal(host(out), np.concatenate(ei1[:k]), err_msg=f"inverse ->1 {tag}")
                np.testing.assert_array_equal(
                    host(out), np.concatenate([x[i * n:(i + 1) * n] % np.uint64(qs[i % L]) for i in range(k)]))
    finally:
        for inverse in (False, True):
            cuda.cluster_plan_set(inverse, logn)


@pytest.mark.parametrize("logn", [12, 13, 14, 15])
def test_cluster_form_matches_pass_form(cuda, oracle, logn):
    """The built-in choice for one limb against the two-launch pass form."""
    n = 1 << logn
    params, tabs, qs = moduli(oracle, n, 1)
    ntt = cuda.NTT(n, *params[0])
    st = oracle.rng(SEED ^ 0xC1A6 ^ logn)
    x = oracle.random_vector(st, n, 4 * qs[0])
    outs = []
    try:
        for enabled in (True, False):
            for inverse in (False, True):
                if enabled:
                    cuda.cluster_plan_set(inverse, logn)
                else:
                    lga, lr, cs, _ = cuda.cluster_plan_get(inverse, logn)
                    cuda.cluster_plan_set(inverse, logn, lga, lr, cs, 0)
            a = dev(x)
            ntt.forward(ptr(a), ptr(a), 4, 4)
            f = host(a)
            b = dev(oracle.reduce(f, qs[0], 4, 2))
            ntt.inverse(ptr(b), ptr(b), 2, 1)
            outs.append((f, host(b)))
    finally:
        for inverse in (False, True):
            cuda.cluster_plan_set(inverse, logn)
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][0], oracle.forward(x, qs[0], tabs[0][0], 4, 4))


@pytest.mark.parametrize("logn", [10, 12, 14, 16])
@pytest.mark.parametrize("count", [1, 40])
def test_transforms_on_8_byte_aligned_pointers(cuda, oracle, logn, count):
    """Operands that are 8- but not 16-byte aligned (the reference accepts any
    uint64_t pointer) take the scalar-access path of the pass and cluster
    kernels and of the fused product: same bits as the oracle."""
    import torch

    n = 1 << logn
    params, tabs, qs = moduli(oracle, n, 2)
    ntts = [cuda.NTT(n, q, psi) for q, psi in params]
    st = oracle.rng(SEED ^ 0xA11 ^ logn ^ count)
    x = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % 2]) for i in range(count)])
    m = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % 2]) for i in range(count)])
    segs = [slice(i * n, (i + 1) * n) for i in range(count)]

    def odd(a):  # a device copy starting 8 bytes into its allocation
        t = torch.empty(a.size + 1, dtype=torch.int64, device="cuda")
        t[1:].copy_(torch.from_numpy(a.view(np.int64)))
        return t

    def back(t):
        return t[1:].cpu().numpy().view(np.uint64)

    def p(t):
        return t.data_ptr() + 8

    d, o, dm = odd(x), odd(np.zeros_like(x)), odd(m)
    assert p(d) % 16 == 8
    ef = np.concatenate([oracle.forward(x[s], qs[i % 2], tabs[i % 2][0], 4, 4) for i, s in enumerate(segs)])
    cuda.forward_batch(ntts, p(o), p(d), count, 4, 4)
    np.testing.assert_array_equal(back(o), ef)
    ei = np.concatenate([oracle.inverse(oracle.reduce(ef[s], qs[i % 2], 4, 2), qs[i % 2], tabs[i % 2][1],
                                        tabs[i % 2][2], 2, 1) for i, s in enumerate(segs)])
    cuda.inverse_batch(ntts, p(o), p(o), count, 4, 1)
    np.testing.assert_array_equal(back(o), ei)
    efm = np.concatenate([oracle.mul(ef[s], m[s], qs[i % 2], 4) for i, s in enumerate(segs)])
    cuda.forward_mul_batch(ntts, p(o), p(d), p(dm), count)
    np.testing.assert_array_equal(back(o), efm)


FUSED = [(5, 5, 2), (6, 5, 2), (5, 6, 2), (6, 6, 2), (7, 6, 2), (6, 7, 2), (7, 7, 2), (8, 7, 2), (7, 8, 2)]


def fused_configs(logn):
    """Valid (row stages, lr, csize) of the fused chain / product kernels."""
    out = []
    for a, b, lr in FUSED:
        if a + b != logn:
            continue
        for c in (1, 2, 3, 4):
            lgt = logn - c - lr
            if c > min(a, b) or lgt < 5 or (1 << lgt) > 512 or 3 * 8 * (1 << (logn - c)) > 227 * 1024:
                continue
            out.append((a, lr, 1 << c))
    return out


@pytest.mark.parametrize("logn", [10, 11, 12, 13, 14, 15])
def test_fused_cluster_chains_bitexact(cuda, oracle, logn):
    """INTT -> MulMod/FMAMod -> NTT and NTT -> MulMod -> INTT in one cluster
    launch per limb, every compiled configuration, against the reference call
    sequences computed by the oracle (lazy and normalized, in place)."""
    n = 1 << logn
    L, count = 2, 3
    params, tabs, qs = moduli(oracle, n, L)
    ntts = [cuda.NTT(n, q, psi) for q, psi in params]
    st = oracle.rng(SEED ^ 0xF05E ^ logn)
    x = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % L]) for i in range(count)])
    m2 = np.concatenate([oracle.random_vector(st, n, 2 * qs[i % L]) for i in range(count)])
    m4 = np.concatenate([oracle.random_vector(st, n, 4 * qs[i % L]) for i in range(count)])
    scalars = [oracle.bounded(st, 2 * q) for q in qs]
    segs = [slice(i * n, (i + 1) * n) for i in range(count)]

    def chain_exp(op, out_f, k):
        out = []
        for i, s in enumerate(segs[:k]):
            q, (fwd, inv, ninv) = qs[i % L], tabs[i % L]
            y = oracle.inverse(oracle.reduce(x[s], q, 4, 2), q, inv, ninv, 2, 2)
            if op == "mul":
                y = oracle.mul(y, m2[s], q, 2)
            else:
                y = oracle.fma(y, scalars[i % L], m2[s] if op == "fma" else None, q, 2)
            out.append(oracle.forward(y, q, fwd, 1, out_f))
        return np.concatenate(out)

    def product_exp(out_f, k):
        out = []
        for i, s in enumerate(segs[:k]):
            q, (fwd, inv, ninv) = qs[i % L], tabs[i % L]
            y = oracle.mul(oracle.forward(x[s], q, fwd, 4, 4), m4[s], q, 4)
            out.append(oracle.inverse(y, q, inv, ninv, 2, out_f))
        return np.concatenate(out)

    cfgs = fused_configs(logn)
    assert cfgs
    try:
        for lgr, lr, cs in cfgs:
            for kind in (cuda.CLUSTER_CHAIN, cuda.CLUSTER_PRODUCT):
                cuda.cluster_plan_set(kind, logn, lgr, lr, cs, count)
            tag = f"lgr={lgr} lr={lr} csize={cs}"
            for k in (1, count):
                dm2, dm4, o = dev(m2[:k * n]), dev(m4[:k * n]), dev_empty(k * n)
                for op in ("mul", "fma", "fma_noadd"):
                    for out_f in (4, 1):
                        d = dev(x[:k * n])
                        if op == "mul":
                            cuda.chain_mul_batch(ntts, ptr(o), ptr(d), ptr(dm2), k, 4, out_f)
                        else:
                            cuda.chain_fma_batch(ntts, ptr(d), ptr(d), scalars, ptr(dm2) if op == "fma" else 0, k,
                                                 4, out_f)
                            o, d = d, o
                        np.testing.assert_array_equal(host(o), chain_exp(op, out_f, k),
                                                      err_msg=f"chain {op} out_f={out_f} k={k} {tag}")
                for out_f in (2, 1):
                    d = dev(x[:k * n])
                    cuda.product_batch(ntts, ptr(d), ptr(d), ptr(dm4), k, 4, out_f)
                    np.testing.assert_array_equal(host(d), product_exp(out_f, k),
                                                  err_msg=f"product out_f={out_f} k={k} {tag}")
    finally:
        for kind in (cuda.CLUSTER_CHAIN, cuda.CLUSTER_PRODUCT):
            cuda.cluster_plan_set(kind, logn)
