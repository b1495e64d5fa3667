"""Test helpers: device buffers (torch as plumbing), the reference test suite's
parameter matrix (tests/common/parameters.hpp) restated, and special inputs."""
import numpy as np

SEED = 0x415848454C  # test_seed(), tests/common/parameters.hpp:142-146

# parameters.hpp:200-203, :246-251
MODULUS_BITS = [20, 30, 40, 50, 52, 55, 59, 60, 61, 62]
NTT_DEGREES = [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384, 32768]
CRITICAL_BITS = {50, 52, 59, 60, 61, 62}  # parameters.hpp:216-218


def element_sizes():
    """parameters.hpp:158-183 with the native surrogate of 2 lanes."""
    v = {0, 1, 2, 3, 4, 5, 6, 7, 31, 32, 33, 127, 128, 129, 255, 256, 257, 1023, 1024, 1025, 8191, 8192, 8193,
         16383, 16384, 16385, 32767, 32768, 32769}
    for k in (1, 2, 3, 4, 7, 8, 16):
        x = 2 * k
        v |= {x - 1, x, x + 1}
    return sorted(v)


def barrett_cases(oracle):
    """parameters.hpp:222-239: one high q per width 20..62, plus low / mid for critical widths."""
    out = []
    for bits in range(20, 63):
        hi = oracle.find_ntt_prime(1024, bits)
        out.append((bits, hi, 0))
        if bits in CRITICAL_BITS:
            lo = oracle.find_ntt_prime_near(1024, bits, 1, 4)
            mid = oracle.find_ntt_prime_near(1024, bits, 1, 2)
            if lo != hi:
                out.append((bits, lo, 1))
            if mid not in (hi, lo):
                out.append((bits, mid, 2))
    return out


def boundary_values(q, factor):
    """parameters.hpp:272-293"""
    B = q * factor
    v = {0, 1}

    def add(x):
        if 0 <= x < B and x < 2 ** 64:
            v.add(x)

    for k in range(1, factor):
        t = k * q
        for d in (-2, -1, 0, 1):
            add(t + d)
    add(B - 2)
    add(B - 1)
    return sorted(v)


def boundary_values_u64(q, factor):
    """parameters.hpp:295-325"""
    bound = min(q * factor, 2 ** 64)
    v = {0, 1}

    def add(x):
        if 0 <= x < bound:
            v.add(x)

    add(q - 2)
    for m in (1, 2, 3, 4, 7):
        for d in (-1, 0, 1):
            add(m * q + d)
    add(bound - 2)
    add(bound - 1)
    return sorted(v)


def pattern(n, vals):
    vals = np.array(vals, dtype=np.uint64)
    if n == 0:
        return np.zeros(0, np.uint64)
    return vals[np.arange(n) % len(vals)].copy()


# ------------------------------------------------------------ device I/O

def dev(arr):
    """Copy a numpy uint64 array to a new device buffer (torch int64 storage)."""
    import torch

    a = np.ascontiguousarray(arr, dtype=np.uint64)
    if a.size == 0:
        return torch.zeros(1, dtype=torch.int64, device="cuda")
    return torch.from_numpy(a.view(np.int64)).to("cuda")


def dev_empty(n, fill=None):
    import torch

    t = torch.empty(max(n, 1), dtype=torch.int64, device="cuda")
    if fill is not None:
        t.fill_(np.int64(np.uint64(fill).view(np.int64)))
    return t


def host(t, n=None):
    import torch

    torch.cuda.synchronize()
    a = t.cpu().numpy().view(np.uint64)
    return a[:n].copy() if n is not None else a.copy()


def ptr(t, offset_words=0):
    return t.data_ptr() + 8 * offset_words


def ntt_params(oracle, n, bits):
    q = oracle.find_ntt_prime(n, bits)
    return q, oracle.find_primitive_root(n, q)


# Element-wise batch jobs: (kind, has_vector, in_f, out_f); in_f "q" is the
# ReduceMod Barrett branch (input factor equal to the modulus).
ELT_CASES = [
    (5, True, 1, 1), (5, False, 1, 1), (6, True, 1, 1), (6, False, 1, 1),
    (7, True, 1, 1), (7, True, 2, 1), (7, True, 4, 1),
    (8, False, 1, 1), (8, True, 2, 1), (8, True, 4, 1), (8, False, 8, 1), (8, True, 8, 1),
    (9, False, 1, 1), (9, False, 2, 2), (9, False, 2, 1), (9, False, 4, 1), (9, False, 4, 2), (9, False, "q", 1),
]


def eltwise_job_data(oracle, st, kind, has_vec, in_f, mods, n, count):
    """Operands of an element-wise job, drawn in the reference's input ranges:
    [0, q) for Add/Sub, [0, F*q) for Mul/FMA, [0, in_f*q) or any 64-bit value
    (Barrett branch) for ReduceMod."""
    L = len(mods)
    qs = [mods[i % L][0] for i in range(count)]
    if kind in (5, 6):
        bound = lambda q: q
    elif kind == 9 and in_f == "q":
        bound = lambda q: 2**64 - 1
    else:
        bound = lambda q: in_f * q
    x = np.concatenate([oracle.random_vector(st, n, bound(q)) for q in qs])
    vec = np.concatenate([oracle.random_vector(st, n, bound(q)) for q in qs]) if has_vec else None
    sc = None
    if kind in (5, 6) and not has_vec:
        sc = [oracle.bounded(st, q) for q, _ in mods]
    elif kind == 8:
        sc = [oracle.bounded(st, in_f * q) for q, _ in mods]
    return x, vec, sc


def eltwise_expected(oracle, kind, has_vec, in_f, out_f, mods, n, count, x, vec, sc):
    """The reference's per-limb eltwise call on every limb (oracle)."""
    L, out = len(mods), []
    for i in range(count):
        q = mods[i % L][0]
        s = slice(i * n, (i + 1) * n)
        a, b = x[s], (vec[s] if has_vec else None)
        if kind == 5:
            out.append(oracle.add(a, b if has_vec else sc[i % L], q))
        elif kind == 6:
            out.append(oracle.sub(a, b if has_vec else sc[i % L], q))
        elif kind == 7:
            out.append(oracle.mul(a, b, q, in_f))
        elif kind == 8:
            out.append(oracle.fma(a, sc[i % L], b, q, in_f))
        else:
            out.append(oracle.reduce(a, q, q if in_f == "q" else in_f, out_f))
    return np.concatenate(out)
