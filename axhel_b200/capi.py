"""ctypes binding of the C-ABI in ``include/axhel_cuda.h``.

Loads the in-tree ``axhel_b200/libaxhel.so`` (built by ``axhel_b200.build``)
and raises if it is missing: there is no CPU fallback.  Data arguments are
raw device addresses (``int``), e.g. ``torch.Tensor.data_ptr()``; streams are
``cudaStream_t`` values as ``int`` (``torch.cuda.Stream.cuda_stream``) or 0.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaxhel.so")

u64 = C.c_uint64
u32 = C.c_uint32
vp = C.c_void_p
st_t = C.c_int32

OK = 0
STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported", 5: "busy",
          6: "timeout", 7: "rejected", 8: "cancelled"}


JOB_FORWARD, JOB_INVERSE, JOB_CHAIN_MUL, JOB_CHAIN_FMA = 1, 2, 3, 4
JOB_ADD, JOB_SUB, JOB_MUL, JOB_FMA, JOB_REDUCE = 5, 6, 7, 8, 9  # element-wise jobs
FACTOR_MODULUS = 2**64 - 1  # ReduceMod input factor equal to each limb's modulus (Barrett branch)


class Job(C.Structure):
    """axhel_job_t"""

    _fields_ = [("kind", C.c_uint32), ("n_ntts", C.c_uint32), ("ntts", C.POINTER(C.c_void_p)),
                ("count", C.c_uint64), ("result", C.c_void_p), ("operand", C.c_void_p), ("vector", C.c_void_p),
                ("scalars", C.POINTER(C.c_uint64)), ("input_mod_factor", C.c_uint64),
                ("output_mod_factor", C.c_uint64)]


SERVER_PERSISTENT = 1
SERVER_ARRIVAL_PRIORITY = 2
SERVER_SMALLEST_FIRST = 4
SERVER_LARGE_FIRST = 8


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_batch_words", C.c_uint64),
                ("small_request_words", C.c_uint64), ("max_inflight", C.c_uint32),
                ("max_batch_requests", C.c_uint32), ("flags", C.c_uint32), ("aging_us", C.c_uint32),
                ("reserve_bytes", C.c_uint64), ("batch_size_ratio", C.c_uint32), ("reserved", C.c_uint32)]


class Request(C.Structure):
    """axhel_request_t"""

    _fields_ = [("kind", C.c_uint32), ("n_ntts", C.c_uint32), ("ntts", C.POINTER(C.c_void_p)),
                ("count", C.c_uint64), ("input", C.c_void_p), ("output", C.c_void_p), ("vector", C.c_void_p),
                ("scalars", C.POINTER(C.c_uint64)), ("input_mod_factor", C.c_uint64),
                ("output_mod_factor", C.c_uint64)]


class RequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("batch_size", C.c_uint32), ("batch_id", C.c_uint64),
                ("queue_ms", C.c_double), ("latency_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("batches", C.c_uint64), ("max_batch_requests", C.c_uint64),
                ("pending", C.c_uint64), ("in_use_bytes", C.c_uint64), ("peak_in_use_bytes", C.c_uint64),
                ("samples", C.c_uint64), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("pool_used_bytes", C.c_uint64), ("host_us_per_batch", C.c_double)]


class DriveResult(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("skipped", C.c_uint64),
                ("failed", C.c_uint64), ("wall_s", C.c_double), ("jobs_per_s", C.c_double),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p50_slowdown", C.c_double),
                ("p99_slowdown", C.c_double), ("isolated_p99_ms", C.c_double), ("p50_queue_ms", C.c_double),
                ("p99_queue_ms", C.c_double), ("p99_large_ms", C.c_double), ("p99_rest_ms", C.c_double)]


class AxhelError(RuntimeError):
    def __init__(self, status, where, msg):
        super().__init__(f"{where}: {STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib():
    """The loaded shared library (loaded once)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"AXHEL CUDA library not built: {LIB_PATH} (run python -m axhel_b200.build)")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    def d(name, res, *args):
        f = getattr(L, name)
        f.restype = res
        f.argtypes = list(args)

    d("axhel_status_string", C.c_char_p, st_t)
    d("axhel_last_error", C.c_char_p)
    d("axhel_version", C.c_int)
    d("axhel_cuda_ntt_create", st_t, u64, u64, u64, C.POINTER(vp))
    d("axhel_cuda_ntt_create_many", st_t, u64, C.POINTER(u64), C.POINTER(u64), C.POINTER(u64), C.POINTER(vp))
    d("axhel_cuda_ntt_create_external", st_t, u64, u64, vp, vp, vp, C.POINTER(vp))
    d("axhel_cuda_ntt_refresh_external", st_t, vp, vp, vp, vp, vp)
    d("axhel_cuda_ntt_retain", st_t, vp)
    d("axhel_cuda_ntt_release", st_t, vp)
    d("axhel_cuda_ntt_degree", u64, vp)
    d("axhel_cuda_ntt_modulus", u64, vp)
    d("axhel_cuda_ntt_read_tables", st_t, vp, vp, vp, vp)
    d("axhel_cuda_ntt_forward", st_t, vp, vp, vp, u64, u64, vp)
    d("axhel_cuda_ntt_inverse", st_t, vp, vp, vp, u64, u64, vp)
    d("axhel_cuda_ntt_forward_batch", st_t, C.POINTER(vp), u64, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_ntt_inverse_batch", st_t, C.POINTER(vp), u64, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_ntt_chain_mul_batch", st_t, C.POINTER(vp), u64, vp, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_ntt_chain_fma_batch", st_t, C.POINTER(vp), u64, vp, vp, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_ntt_product_batch", st_t, C.POINTER(vp), u64, vp, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_ntt_forward_mul_batch", st_t, C.POINTER(vp), u64, vp, vp, vp, u64, vp)
    d("axhel_cuda_ntt_mul_inverse_batch", st_t, C.POINTER(vp), u64, vp, vp, vp, u64, u64, vp)
    d("axhel_cuda_eltwise_add_vv", st_t, vp, vp, vp, u64, u64, vp)
    d("axhel_cuda_eltwise_add_vs", st_t, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_eltwise_sub_vv", st_t, vp, vp, vp, u64, u64, vp)
    d("axhel_cuda_eltwise_sub_vs", st_t, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_eltwise_mul", st_t, vp, vp, vp, u64, u64, u64, vp)
    d("axhel_cuda_eltwise_fma", st_t, vp, vp, u64, vp, u64, u64, u64, vp)
    d("axhel_cuda_eltwise_reduce", st_t, vp, vp, u64, u64, u64, u64, vp)
    d("axhel_cuda_tensor_product", st_t, vp, vp, vp, vp, vp, vp, vp, u64, u64, vp, u64, u64, vp)
    d("axhel_cuda_plan_set", st_t, C.c_int, u32, u32, vp, vp, vp)
    d("axhel_cuda_plan_get", st_t, C.c_int, u32, u64, vp, vp, vp, vp)
    d("axhel_cuda_cluster_plan_set", st_t, C.c_int, u32, u32, u32, u32, u64)
    d("axhel_cuda_cluster_plan_get", st_t, C.c_int, u32, vp, vp, vp, vp)
    d("axhel_cuda_plan_load", st_t, C.c_char_p, C.POINTER(u32))
    d("axhel_cuda_batch_split_set", st_t, u32, u32)
    d("axhel_cuda_batch_split_get", st_t, u32, C.POINTER(u32))
    d("axhel_cuda_is_device_pointer", C.c_int, vp)
    d("axhel_cuda_launch_count", u64)
    d("axhel_cuda_profile_enable", st_t, C.c_int)
    d("axhel_cuda_profile_report", st_t, C.c_char_p, u64, C.POINTER(u64))
    d("axhel_cuda_butterfly_peak", st_t, vp, C.c_int, C.POINTER(C.c_double), vp)
    d("axhel_cuda_batch_create", st_t, C.POINTER(Job), u64, C.POINTER(vp))
    d("axhel_cuda_batch_launch", st_t, vp, vp)
    d("axhel_cuda_batch_graph_launch", st_t, vp, vp)
    d("axhel_cuda_batch_launch_phased", st_t, vp, vp)
    d("axhel_cuda_batch_status", st_t, vp, vp)
    d("axhel_cuda_batch_destroy", st_t, vp)
    d("axhel_cuda_batch_run", st_t, C.POINTER(Job), u64, vp)
    d("axhel_cuda_batch_last_error", C.c_char_p)
    d("axhel_cuda_batch_set_wait_ns", st_t, vp, u64)
    d("axhel_cuda_batch_run_static", st_t, C.POINTER(Job), u64, vp)
    d("axhel_server_create", st_t, C.POINTER(ServerConfig), C.POINTER(vp))
    d("axhel_server_submit", st_t, vp, C.POINTER(Request), C.POINTER(u64))
    d("axhel_server_wait", st_t, vp, u64, u64, C.POINTER(RequestInfo))
    d("axhel_server_cancel", st_t, vp, u64)
    d("axhel_server_pause", st_t, vp, C.c_int)
    d("axhel_server_stats", st_t, vp, C.POINTER(ServerStats), C.c_int)
    d("axhel_server_destroy", st_t, vp)
    d("axhel_server_last_error", C.c_char_p)
    d("axhel_server_drive", st_t, vp, C.POINTER(Request), C.c_uint32, C.POINTER(C.c_void_p), C.c_uint32,
      C.POINTER(C.c_double), C.c_double, C.c_double, u64, C.POINTER(DriveResult))
    d("axhel_cuda_batch_debug_unreachable", st_t, vp, u64)
    d("axhel_server_debug_fail_staging", st_t, vp, u32)


def check(status, where):
    if status != OK:
        raise AxhelError(status, where, lib().axhel_last_error().decode())


def launch_count():
    return int(lib().axhel_cuda_launch_count())


def profile_enable(on=True):
    check(lib().axhel_cuda_profile_enable(1 if on else 0), "profile_enable")


def profile_report():
    """Drains the event records: {kernel configuration: (launches, total_ms)}."""
    need = u64()
    buf = C.create_string_buffer(1 << 16)
    check(lib().axhel_cuda_profile_report(buf, len(buf), C.byref(need)), "profile_report")
    out = {}
    for line in buf.value.decode().splitlines():
        parts = line.rsplit(" ", 2)
        if len(parts) == 3:
            out[parts[0]] = (int(parts[1]), float(parts[2]))
    return out


def butterfly_peak(ntt, inverse=False, stream=0):
    """Measured butterflies/s of the reference butterfly on registers only."""
    r = C.c_double()
    check(lib().axhel_cuda_butterfly_peak(ntt.h, int(inverse), C.byref(r), stream), "butterfly_peak")
    return r.value


def make_jobs(specs):
    """specs: list of dicts {kind, ntts, count, result, operand, vector=0,
    scalars=None, in_f, out_f}; returns (ctypes array of Job, keep-alive list)."""
    arr = (Job * len(specs))()
    keep = []
    for i, sp in enumerate(specs):
        hs = (C.c_void_p * len(sp["ntts"]))(*[t.h.value for t in sp["ntts"]])
        keep.append(hs)
        j = arr[i]
        j.kind = sp["kind"]
        j.n_ntts = len(sp["ntts"])
        j.ntts = C.cast(hs, C.POINTER(C.c_void_p))
        j.count = sp["count"]
        j.result = sp["result"]
        j.operand = sp["operand"]
        j.vector = sp.get("vector") or None
        if sp.get("scalars") is not None:
            sc = (C.c_uint64 * len(sp["scalars"]))(*[int(v) for v in sp["scalars"]])
            keep.append(sc)
            j.scalars = C.cast(sc, C.POINTER(C.c_uint64))
        j.input_mod_factor = sp.get("in_f", 1)
        j.output_mod_factor = sp.get("out_f", 1)
    return arr, keep


def _bcheck(status, where):
    if status != OK:
        raise AxhelError(status, where, lib().axhel_cuda_batch_last_error().decode())


class Batch:
    """A batch of uneven jobs run by one persistent kernel launch."""

    def __init__(self, specs):
        self.jobs, self._keep = make_jobs(specs)
        self.h = vp()
        _bcheck(lib().axhel_cuda_batch_create(self.jobs, len(specs), C.byref(self.h)), "batch_create")

    def launch(self, stream=0, graph=False, phased=False):
        if phased:
            f = lib().axhel_cuda_batch_launch_phased
        else:
            f = lib().axhel_cuda_batch_graph_launch if graph else lib().axhel_cuda_batch_launch
        _bcheck(f(self.h, stream), "batch_launch")

    def status(self, stream=0):
        return int(lib().axhel_cuda_batch_status(self.h, stream))

    def set_wait_ns(self, ns):
        _bcheck(lib().axhel_cuda_batch_set_wait_ns(self.h, ns), "batch_set_wait_ns")

    def debug_unreachable(self, job):
        _bcheck(lib().axhel_cuda_batch_debug_unreachable(self.h, job), "batch_debug_unreachable")

    def close(self):
        if self.h:
            lib().axhel_cuda_batch_destroy(self.h)
            self.h = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_run(specs, stream=0):
    jobs, keep = make_jobs(specs)
    _bcheck(lib().axhel_cuda_batch_run(jobs, len(specs), stream), "batch_run")


def batch_run_static(specs, stream=0):
    """axhel_cuda_batch_run_static: the batch with its scratch in the library's
    static device array (no device allocation)."""
    jobs, keep = make_jobs(specs)
    _bcheck(lib().axhel_cuda_batch_run_static(jobs, len(specs), stream), "batch_run_static")


def _scheck(status, where):
    if status != OK:
        raise AxhelError(status, where, lib().axhel_server_last_error().decode())


class Server:
    """The continuous-batching serving loop (axhel_server_*)."""

    def __init__(self, budget_bytes, max_inflight=2, max_batch_requests=256, max_batch_words=0, persistent=False,
                 small_request_words=0, reserve_bytes=0, flags=0, aging_us=0, batch_size_ratio=0):
        flags |= SERVER_PERSISTENT if persistent else 0
        cfg = ServerConfig(budget_bytes, max_batch_words, small_request_words, max_inflight, max_batch_requests,
                           flags, aging_us, reserve_bytes, batch_size_ratio, 0)
        self.h = vp()
        _scheck(lib().axhel_server_create(C.byref(cfg), C.byref(self.h)), "server_create")
        self._keep = {}

    def submit(self, kind, ntts, count, input, output, vector=0, scalars=None, in_f=1, out_f=1):
        hs = (C.c_void_p * len(ntts))(*[t.h.value for t in ntts])
        r = Request(kind, len(ntts), C.cast(hs, C.POINTER(C.c_void_p)), count, input, output, vector or None,
                    None, in_f, out_f)
        keep = [hs]
        if scalars is not None:
            sc = (C.c_uint64 * len(scalars))(*[int(v) for v in scalars])
            r.scalars = C.cast(sc, C.POINTER(C.c_uint64))
            keep.append(sc)
        rid = u64()
        _scheck(lib().axhel_server_submit(self.h, C.byref(r), C.byref(rid)), "server_submit")
        self._keep[rid.value] = keep
        return rid.value

    def wait(self, rid, timeout_s=60.0):
        """Returns (status, RequestInfo); status AXHEL_ERR_TIMEOUT (6) leaves the request queued."""
        info = RequestInfo()
        st = int(lib().axhel_server_wait(self.h, rid, int(timeout_s * 1e6), C.byref(info)))
        if st != 6:
            self._keep.pop(rid, None)
        return st, info

    def cancel(self, rid):
        return int(lib().axhel_server_cancel(self.h, rid))

    def pause(self, paused=True):
        _scheck(lib().axhel_server_pause(self.h, 1 if paused else 0), "server_pause")

    def debug_fail_staging(self, request):
        """The next batch's staging fails at its request `request` (tests)."""
        _scheck(lib().axhel_server_debug_fail_staging(self.h, request), "server_debug_fail_staging")

    def stats(self, reset=False):
        s = ServerStats()
        _scheck(lib().axhel_server_stats(self.h, C.byref(s), 1 if reset else 0), "server_stats")
        return {k: getattr(s, k) for k, _ in ServerStats._fields_}

    def drive(self, templates, outputs, isolated_ms, rate, seconds, seed=1):
        """axhel_server_drive: Poisson load from a C++ thread.  templates: list
        of dicts as submit() takes (output ignored); outputs: per template a
        list of `copies` output addresses."""
        n = len(templates)
        copies = len(outputs[0])
        arr = (Request * n)()
        keep = []
        for i, t in enumerate(templates):
            hs = (C.c_void_p * len(t["ntts"]))(*[h.h.value for h in t["ntts"]])
            keep.append(hs)
            r = arr[i]
            r.kind, r.n_ntts, r.ntts, r.count = t["kind"], len(t["ntts"]), C.cast(hs, C.POINTER(C.c_void_p)), t["count"]
            r.input, r.output, r.vector = t["input"], outputs[i][0], t.get("vector") or None
            if t.get("scalars") is not None:
                sc = (C.c_uint64 * len(t["scalars"]))(*[int(v) for v in t["scalars"]])
                keep.append(sc)
                r.scalars = C.cast(sc, C.POINTER(C.c_uint64))
            r.input_mod_factor, r.output_mod_factor = t.get("in_f", 1), t.get("out_f", 1)
        outs = (C.c_void_p * (n * copies))(*[o for row in outputs for o in row])
        iso = (C.c_double * n)(*isolated_ms) if isolated_ms is not None else None
        res = DriveResult()
        _scheck(lib().axhel_server_drive(self.h, arr, n, outs, copies, iso, rate, seconds, seed, C.byref(res)),
                "server_drive")
        return {k: getattr(res, k) for k, _ in DriveResult._fields_}

    def close(self):
        if self.h:
            lib().axhel_server_destroy(self.h)
            self.h = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _arr64(values):
    a = (u64 * len(values))(*[int(v) for v in values])
    return a


class NTT:
    """A device-resident (N, q) table context (``axhel_ntt_t``)."""

    def __init__(self, degree, modulus, root=None, tables=None, handle=None):
        h = vp()
        if handle is not None:
            h = handle
        elif tables is None:
            check(lib().axhel_cuda_ntt_create(degree, modulus, root, C.byref(h)), "ntt_create")
        else:
            import numpy as np

            fwd, inv, ninv = (np.ascontiguousarray(t, dtype=np.uint64) for t in tables)
            check(lib().axhel_cuda_ntt_create_external(degree, modulus, fwd.ctypes.data, inv.ctypes.data,
                                                       ninv.ctypes.data, C.byref(h)), "ntt_create_external")
        self.h = h
        self.degree = degree
        self.modulus = modulus

    @staticmethod
    def create_many(params):
        """NTT objects for a list of (degree, modulus, root), the missing
        tables generated on the device in one launch
        (axhel_cuda_ntt_create_many)."""
        k = len(params)
        arr = lambda col: (u64 * max(k, 1))(*[int(p[col]) for p in params])
        hs = (vp * max(k, 1))()
        check(lib().axhel_cuda_ntt_create_many(k, arr(0), arr(1), arr(2), hs), "ntt_create_many")
        return [NTT(d, q, handle=vp(hs[i])) for i, (d, q, _) in enumerate(params)]

    def close(self):
        if self.h:
            lib().axhel_cuda_ntt_release(self.h)
            self.h = vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def read_tables(self):
        import numpy as np

        fwd = np.zeros((self.degree, 2), np.uint64)
        inv = np.zeros((self.degree, 2), np.uint64)
        ninv = np.zeros(2, np.uint64)
        check(lib().axhel_cuda_ntt_read_tables(self.h, fwd.ctypes.data, inv.ctypes.data, ninv.ctypes.data),
              "read_tables")
        return fwd, inv, ninv

    def forward(self, dst, src, in_f=1, out_f=1, stream=0):
        check(lib().axhel_cuda_ntt_forward(self.h, dst, src, in_f, out_f, stream), "ntt_forward")

    def inverse(self, dst, src, in_f=1, out_f=1, stream=0):
        check(lib().axhel_cuda_ntt_inverse(self.h, dst, src, in_f, out_f, stream), "ntt_inverse")


def _handles(ntts):
    return (vp * len(ntts))(*[t.h.value for t in ntts])


def forward_batch(ntts, dst, src, count, in_f=1, out_f=1, stream=0):
    check(lib().axhel_cuda_ntt_forward_batch(_handles(ntts), len(ntts), dst, src, count, in_f, out_f, stream),
          "ntt_forward_batch")


def inverse_batch(ntts, dst, src, count, in_f=1, out_f=1, stream=0):
    check(lib().axhel_cuda_ntt_inverse_batch(_handles(ntts), len(ntts), dst, src, count, in_f, out_f, stream),
          "ntt_inverse_batch")


def forward_mul_batch(ntts, dst, src, multiplicand, count, stream=0):
    """Forward transform of each limb, then the dyadic product with `multiplicand`."""
    check(lib().axhel_cuda_ntt_forward_mul_batch(_handles(ntts), len(ntts), dst, src, multiplicand, count, stream),
          "ntt_forward_mul_batch")


def mul_inverse_batch(ntts, dst, src, multiplicand, count, out_f=1, stream=0):
    """Dyadic product with `multiplicand`, then the inverse transform of each limb."""
    check(lib().axhel_cuda_ntt_mul_inverse_batch(_handles(ntts), len(ntts), dst, src, multiplicand, count, out_f,
                                                 stream), "ntt_mul_inverse_batch")


def chain_mul_batch(ntts, dst, src, multiplicand, count, in_f=2, out_f=1, stream=0):
    check(lib().axhel_cuda_ntt_chain_mul_batch(_handles(ntts), len(ntts), dst, src, multiplicand, count, in_f, out_f,
                                               stream), "ntt_chain_mul_batch")


def product_batch(ntts, dst, src, multiplicand, count, in_f=4, out_f=1, stream=0):
    """Fused NTT -> MulMod(., multiplicand, 4) -> INTT over a batch."""
    hs = _handles(ntts)
    check(lib().axhel_cuda_ntt_product_batch(hs, len(ntts), dst, src, multiplicand, count, in_f, out_f, stream),
          "ntt_product_batch")


def chain_fma_batch(ntts, dst, src, scalars, addend, count, in_f=2, out_f=1, stream=0):
    sc = _arr64(scalars)
    check(lib().axhel_cuda_ntt_chain_fma_batch(_handles(ntts), len(ntts), dst, src, C.cast(sc, vp), addend, count,
                                               in_f, out_f, stream), "ntt_chain_fma_batch")


def add(dst, a, b, n, q, stream=0, scalar=False):
    f = lib().axhel_cuda_eltwise_add_vs if scalar else lib().axhel_cuda_eltwise_add_vv
    check(f(dst, a, b, n, q, stream), "eltwise_add")


def sub(dst, a, b, n, q, stream=0, scalar=False):
    f = lib().axhel_cuda_eltwise_sub_vs if scalar else lib().axhel_cuda_eltwise_sub_vv
    check(f(dst, a, b, n, q, stream), "eltwise_sub")


def mul(dst, a, b, n, q, factor, stream=0):
    check(lib().axhel_cuda_eltwise_mul(dst, a, b, n, q, factor, stream), "eltwise_mul")


def fma(dst, a, s, c, n, q, factor, stream=0):
    check(lib().axhel_cuda_eltwise_fma(dst, a, s, c, n, q, factor, stream), "eltwise_fma")


def reduce(dst, a, n, q, in_f, out_f, stream=0):
    check(lib().axhel_cuda_eltwise_reduce(dst, a, n, q, in_f, out_f, stream), "eltwise_reduce")


def tensor_product(r0, r1, r2, c0, c1, d0, d1, n, count, moduli, factor=1, stream=0):
    m = _arr64(moduli)
    check(lib().axhel_cuda_tensor_product(r0, r1, r2, c0, c1, d0, d1, n, count, C.cast(m, vp), len(moduli), factor,
                                          stream), "tensor_product")


def plan_set(inverse, logn, passes):
    """passes: list of (lg, lr, tg); [] restores the default."""
    n = len(passes)
    lg = (u32 * 3)(*[p[0] for p in passes])
    lr = (u32 * 3)(*[p[1] for p in passes])
    tg = (u32 * 3)(*[p[2] for p in passes])
    check(lib().axhel_cuda_plan_set(int(inverse), logn, n, C.cast(lg, vp), C.cast(lr, vp), C.cast(tg, vp)),
          "plan_set")


def plan_get(inverse, logn, count):
    npass = u32()
    lg, lr, tg = (u32 * 3)(), (u32 * 3)(), (u32 * 3)()
    check(lib().axhel_cuda_plan_get(int(inverse), logn, count, C.byref(npass), C.cast(lg, vp), C.cast(lr, vp),
                                    C.cast(tg, vp)), "plan_get")
    return [(lg[i], lr[i], tg[i]) for i in range(npass.value)]


CLUSTER_FORWARD, CLUSTER_INVERSE, CLUSTER_CHAIN, CLUSTER_PRODUCT = 0, 1, 2, 3


def cluster_plan_set(kind, logn, lga=0, lr=0, csize=0, max_limbs=0):
    """Single-launch cluster form of up to `max_limbs` limbs for `kind`
    (CLUSTER_FORWARD / _INVERSE transforms, or a bool for those two;
    CLUSTER_CHAIN / _PRODUCT fused chains); lga = 0 restores the built-in
    choice, max_limbs = 0 turns it off."""
    check(lib().axhel_cuda_cluster_plan_set(int(kind), logn, lga, lr, csize, max_limbs), "cluster_plan_set")


def cluster_plan_get(kind, logn):
    """(lga, lr, csize, max_limbs) of the cluster form of `kind` for N = 2^logn."""
    a, b, c = u32(), u32(), u32()
    m = u64()
    check(lib().axhel_cuda_cluster_plan_get(int(kind), logn, C.byref(a), C.byref(b), C.byref(c), C.byref(m)),
          "cluster_plan_get")
    return a.value, b.value, c.value, m.value


def batch_split_set(logn, row_stages):
    """Contiguous-pass stages of the batch engine for N = 2^logn (0 restores)."""
    check(lib().axhel_cuda_batch_split_set(logn, row_stages), "batch_split_set")


def batch_split_get(logn):
    r = u32()
    check(lib().axhel_cuda_batch_split_get(logn, C.byref(r)), "batch_split_get")
    return r.value


def plan_load(path=None):
    n = u32()
    check(lib().axhel_cuda_plan_load(path.encode() if path else None, C.byref(n)), "plan_load")
    return n.value
