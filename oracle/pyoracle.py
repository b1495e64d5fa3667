"""ctypes bindings for the two CPU checkers built by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY.  ``Oracle`` wraps the plain-C restatement
(``liboracle.so``); ``Reference`` wraps the reference AXHEL native backend
compiled from its own sources (``_ref/libaxhel_ref.so``).  Only the test
suite, the smoke check and the bench's CPU-baseline leg import this module;
the shipped library never does.

All arrays are numpy ``uint64``.  Twiddle tables are ``(N, 2)`` arrays of
``{operand, Shoup quotient}`` rows, the layout of ``NTTMultiplyOperand``
(axhel/include/axhel/ntt/ntt.hpp:14-18).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libaxhel_ref.so")

u64 = C.c_uint64
p64 = C.POINTER(C.c_uint64)


def _ptr(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(p64)


def build_port():
    """Compile the restatement with gcc when the prebuilt library is absent."""
    if not os.path.exists(PORT_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "port"])


class _Common:
    lib: C.CDLL
    prefix: str

    def _fn(self, name, restype, *argtypes):
        f = getattr(self.lib, self.prefix + name)
        f.restype = restype
        f.argtypes = list(argtypes)
        return f

    def _bind_eltwise(self):
        self._add_vv = self._fn("add_vv", None, p64, p64, p64, u64, u64)
        self._add_vs = self._fn("add_vs", None, p64, p64, u64, u64, u64)
        self._sub_vv = self._fn("sub_vv", None, p64, p64, p64, u64, u64)
        self._sub_vs = self._fn("sub_vs", None, p64, p64, u64, u64, u64)
        self._mul = self._fn("mul", None, p64, p64, p64, u64, u64, u64)
        self._fma = self._fn("fma", None, p64, p64, u64, p64, u64, u64, u64)
        self._reduce = self._fn("reduce", None, p64, p64, u64, u64, u64, u64)

    # --- element-wise, numpy in / numpy out (out may be passed to test aliasing)
    def add(self, a, b, q, out=None):
        out = np.zeros_like(a) if out is None else out
        if np.isscalar(b) or isinstance(b, (int, np.integer)):
            self._add_vs(_ptr(out), _ptr(a), int(b), a.size, q)
        else:
            self._add_vv(_ptr(out), _ptr(a), _ptr(b), a.size, q)
        return out

    def sub(self, a, b, q, out=None):
        out = np.zeros_like(a) if out is None else out
        if np.isscalar(b) or isinstance(b, (int, np.integer)):
            self._sub_vs(_ptr(out), _ptr(a), int(b), a.size, q)
        else:
            self._sub_vv(_ptr(out), _ptr(a), _ptr(b), a.size, q)
        return out

    def mul(self, a, b, q, factor, out=None):
        out = np.zeros_like(a) if out is None else out
        self._mul(_ptr(out), _ptr(a), _ptr(b), a.size, q, factor)
        return out

    def fma(self, a, s, c, q, factor, out=None):
        out = np.zeros_like(a) if out is None else out
        self._fma(_ptr(out), _ptr(a), int(s), _ptr(c), a.size, q, factor)
        return out

    def reduce(self, a, q, in_f, out_f, out=None):
        out = np.zeros_like(a) if out is None else out
        self._reduce(_ptr(out), _ptr(a), a.size, q, in_f, out_f)
        return out

    def tables(self, n, q, psi):
        fwd = np.zeros((n, 2), np.uint64)
        inv = np.zeros((n, 2), np.uint64)
        ninv = np.zeros(2, np.uint64)
        rc = self._tables(n, q, psi, _ptr(fwd), _ptr(inv), _ptr(ninv))
        assert rc == 0
        return fwd, inv, ninv


class Oracle(_Common):
    """The plain-C restatement (oracle/axhel_oracle.c)."""

    prefix = "orc_"

    def __init__(self):
        build_port()
        self.lib = C.CDLL(PORT_SO)
        self._bind_eltwise()
        self._tables = self._fn("ntt_tables", C.c_int, u64, u64, u64, p64, p64, p64)
        self._fwd = self._fn("ntt_compute_forward", None, p64, p64, u64, u64, p64, u64, u64)
        self._inv = self._fn("ntt_compute_inverse", None, p64, p64, u64, u64, p64, p64, u64, u64)
        PP = C.POINTER(p64)
        self._job = self._fn("job_batch", None, C.c_uint32, p64, p64, p64, p64, u64, u64, p64, PP, PP, PP, u64,
                             u64, u64, C.c_int)
        self._tensor = self._fn("tensor_batch", None, p64, p64, p64, p64, p64, p64, p64, u64, u64, p64, u64, u64,
                                C.c_int)
        self.is_prime = self._fn("is_prime", C.c_int, u64)
        self.find_ntt_prime = self._fn("find_ntt_prime", u64, u64, C.c_uint)
        self.find_ntt_prime_near = self._fn("find_ntt_prime_near", u64, u64, C.c_uint, u64, u64)
        root = self._fn("find_primitive_root", u64, u64, u64)

        def find_primitive_root(n, q):
            if q < 3 or q % (2 * n) != 1:  # also guards the C search against q = 0 (a failed prime search)
                raise ValueError(f"no primitive 2N-th root: q={q} is not 1 mod 2N={2 * n}")
            return root(n, q)

        self.find_primitive_root = find_primitive_root
        self.pow_mod = self._fn("pow_mod", u64, u64, u64, u64)
        self.barrett_factor = self._fn("barrett_factor", u64, u64)
        self.shoup_quotient = self._fn("shoup_quotient", u64, u64, u64)
        self._seed = self._fn("mt64_seed", None, p64, u64)
        self._next = self._fn("mt64_next", u64, p64)
        self._bounded = self._fn("bounded_random", u64, p64, u64)
        self._randvec = self._fn("random_vector", None, p64, u64, u64, p64)

    def forward(self, x, q, fwd, in_f=1, out_f=1, out=None):
        out = np.zeros_like(x) if out is None else out
        self._fwd(_ptr(out), _ptr(x), x.size, q, _ptr(fwd), in_f, out_f)
        return out

    def job_batch(self, kind, x, n, count, qs, tables, in_f, out_f, vec=None, scalars=None, threads=0, out=None):
        """The reference's per-limb call sequence of a batch job (kind 1..4 as
        the C-ABI's AXHEL_JOB_*) over `count` limbs of degree n stored back to
        back; limb i uses qs[i % len(qs)] and tables[i % len(qs)] = (fwd, inv,
        ninv).  Multi-threaded over limbs (threads 0 = every core)."""
        nq = len(qs)
        assert len(tables) == nq and x.size == n * count
        out = np.zeros_like(x) if out is None else out
        PP = p64 * nq
        fw = PP(*[_ptr(t[0]) for t in tables])
        iv = PP(*[_ptr(t[1]) for t in tables])
        ni = PP(*[_ptr(t[2]) for t in tables])
        qa = np.ascontiguousarray(qs, dtype=np.uint64)
        sc = None if scalars is None else np.ascontiguousarray(scalars, dtype=np.uint64)
        self._job(kind, _ptr(out), _ptr(x), _ptr(vec), _ptr(sc), n, count, _ptr(qa), fw, iv, ni, nq, in_f, out_f,
                  threads)
        return out

    def tensor_batch(self, c0, c1, d0, d1, n, count, qs, factor, threads=0):
        """The tensor-product per-limb call sequence (three results)."""
        outs = [np.zeros_like(c0) for _ in range(3)]
        qa = np.ascontiguousarray(qs, dtype=np.uint64)
        self._tensor(*[_ptr(o) for o in outs], _ptr(c0), _ptr(c1), _ptr(d0), _ptr(d1), n, count, _ptr(qa), len(qs),
                     factor, threads)
        return outs

    def inverse(self, x, q, inv, ninv, in_f=1, out_f=1, out=None):
        out = np.zeros_like(x) if out is None else out
        self._inv(_ptr(out), _ptr(x), x.size, q, _ptr(inv), _ptr(ninv), in_f, out_f)
        return out

    # --- the reference tests' deterministic generator (mt19937_64 + rejection)
    def rng(self, seed):
        st = np.zeros(313, np.uint64)
        self._seed(_ptr(st), seed & 0xFFFFFFFFFFFFFFFF)
        return st

    def next_u64(self, st):
        return int(self._next(_ptr(st)))

    def bounded(self, st, bound):
        return int(self._bounded(_ptr(st), bound))

    def random_vector(self, st, n, bound):
        out = np.zeros(n, np.uint64)
        self._randvec(_ptr(out), n, bound, _ptr(st))
        return out


class Reference(_Common):
    """The reference AXHEL native backend compiled from source (oracle/_ref)."""

    prefix = "ref_"

    @staticmethod
    def available():
        return os.path.exists(REF_SO)

    def __init__(self):
        self.lib = C.CDLL(REF_SO)
        self._bind_eltwise()
        self._tables = self._fn("ntt_tables", C.c_int, u64, u64, u64, p64, p64, p64)
        self._create = self._fn("ntt_create", C.c_void_p, u64, u64, u64)
        self._create_ext = self._fn("ntt_create_external", C.c_void_p, u64, u64, p64, p64, p64)
        self._destroy = self._fn("ntt_destroy", None, C.c_void_p)
        self._fwd = self._fn("ntt_forward", None, C.c_void_p, p64, p64, u64, u64)
        self._inv = self._fn("ntt_inverse", None, C.c_void_p, p64, p64, u64, u64)
        self._roundtrip = self._fn("roundtrip_batch", None, C.POINTER(C.c_void_p), u64, p64, u64, u64, C.c_int)

    def ntt(self, n, q, psi):
        return _RefNTT(self, self._create(n, q, psi), n, q)

    def ntt_external(self, n, q, fwd, inv, ninv):
        h = _RefNTT(self, self._create_ext(n, q, _ptr(fwd), _ptr(inv), _ptr(ninv)), n, q)
        h._keep = (fwd, inv, ninv)
        return h

    def roundtrip_batch(self, ntts, data, n, count, threads):
        hs = (C.c_void_p * len(ntts))(*[t.h for t in ntts])
        self._roundtrip(hs, len(ntts), _ptr(data), n, count, threads)


class _RefNTT:
    def __init__(self, ref, h, n, q):
        self.ref, self.h, self.n, self.q = ref, h, n, q

    def forward(self, x, in_f=1, out_f=1, out=None):
        out = np.zeros_like(x) if out is None else out
        self.ref._fwd(self.h, _ptr(out), _ptr(x), in_f, out_f)
        return out

    def inverse(self, x, in_f=1, out_f=1, out=None):
        out = np.zeros_like(x) if out is None else out
        self.ref._inv(self.h, _ptr(out), _ptr(x), in_f, out_f)
        return out

    def __del__(self):
        try:
            self.ref._destroy(self.h)
        except Exception:
            pass
