"""rssieve_b200 -- B200 (sm_100a) implementation of RSSieve's BSGS sieve path.

Python binding of the C ABI in include/rssieve_b200.h (librssieve_b200.so,
built in-tree by rssieve_b200.build).  The product is the shared library and
the `rssieve` command-line drop-in next to it; this module is the host-side
mirror used by tests and bench.py.  There is no CPU fallback: device entry
points raise RuntimeError when the library or a CUDA device is missing.
"""
import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "_lib", "librssieve_b200.so")
CLI_PATH = os.path.join(PKG, "_lib", "rssieve")
MAX_SEQ = 100

RS_OK, RS_EARG, RS_ECUDA, RS_ENOMEM, RS_EDEVICE, RS_EIO, RS_EPARSE, RS_ESTATE, RS_EVERIFY, RS_ENODEV, RS_EBUSY = (
    0, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10)

FACTOR_DT = np.dtype([("p", "<u8"), ("n", "<u4"), ("seq", "<u4")])
COUNTER_FIELDS = ("primes", "skipped", "full", "parity", "targets", "baby", "giant", "small_order",
                  "candidates", "hits", "factors", "dups", "sieve_cands")


class _Seqs(C.Structure):
    _fields_ = [("base", C.c_uint32), ("kcount", C.c_uint32), ("nmin", C.c_uint32), ("nmax", C.c_uint32),
                ("k", C.c_uint64 * MAX_SEQ), ("c", C.c_int32 * MAX_SEQ), ("words_per_seq", C.c_uint64),
                ("bitmap", C.POINTER(C.c_uint32))]


class _Counters(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in COUNTER_FIELDS]


class _State(C.Structure):
    _fields_ = [(f, C.c_uint64) for f in ("pmin", "pmax", "p", "checksum", "primecount", "factorcount",
                                          "last_trickle", "dupcount")]


class _Factor(C.Structure):
    _fields_ = [("p", C.c_uint64), ("n", C.c_uint32), ("seq", C.c_uint32)]


# every symbol include/rssieve_b200.h declares
EXPORTS = (
    "rs_version", "rs_strerror", "rs_last_error", "rs_abcd_parse", "rs_abcd_read", "rs_seqs_create",
    "rs_seqs_free", "rs_seqs_count", "rs_verify_factor", "rs_is_prime", "rs_format_factor",
    "rs_factors_file_apply", "rs_factors_commit", "rs_factors_finalize", "rs_state_write", "rs_state_read",
    "rs_state_resume", "rs_ctx_create", "rs_ctx_destroy", "rs_ctx_set_stream", "rs_device_count",
    "rs_job_load", "rs_run_range", "rs_factors_fetch", "rs_bitmap_download", "rs_counters_get",
    "rs_primes_generate", "rs_last_timing", "rs_mulmod_peak", "rs_widemul_peak", "rs_fpmul_peak", "rs_primes_generate_noalloc",
    "rs_set_baby_steps", "rs_get_baby_steps", "rs_set_wait_limit",
    "rs_batch_create", "rs_batch_destroy", "rs_batch_set_stream", "rs_batch_add", "rs_batch_add_clone",
    "rs_batch_free_slots", "rs_batch_job_bytes", "rs_batch_reserve", "rs_batch_release", "rs_batch_set_budget",
    "rs_batch_poll", "rs_batch_run",
    "rs_batch_factors_fetch", "rs_batch_bitmap_download", "rs_batch_job_info", "rs_batch_counters",
)
BABY_STEPS = (1024, 2048, 4096, 8192, 16384)   # accepted by rs_set_baby_steps (0: automatic)
NOALLOC_MAX_WIDTH = 1 << 22     # RS_NOALLOC_MAX_WIDTH

_lib = None


def lib():
    """Load librssieve_b200.so (building it first when absent and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build
        build.build()
    L = C.CDLL(LIB_PATH)
    u64, u32, i32, vp, sz = C.c_uint64, C.c_uint32, C.c_int32, C.c_void_p, C.c_size_t
    PS = C.POINTER(_Seqs)
    sig = {
        "rs_version": (C.c_char_p, []),
        "rs_strerror": (C.c_char_p, [C.c_int]),
        "rs_last_error": (C.c_char_p, []),
        "rs_abcd_parse": (C.c_int, [C.c_char_p, sz, C.POINTER(PS)]),
        "rs_abcd_read": (C.c_int, [C.c_char_p, C.POINTER(PS)]),
        "rs_seqs_create": (C.c_int, [u32, u32, vp, vp, u32, u32, vp, C.POINTER(PS)]),
        "rs_seqs_free": (None, [PS]),
        "rs_seqs_count": (u64, [PS]),
        "rs_verify_factor": (C.c_int, [u64, u64, u32, i32, u32]),
        "rs_is_prime": (C.c_int, [u64]),
        "rs_format_factor": (C.c_int, [PS, C.POINTER(_Factor), C.c_char_p, sz]),
        "rs_factors_file_apply": (C.c_int, [C.c_char_p, PS, C.POINTER(u64)]),
        "rs_factors_commit": (C.c_int, [C.c_char_p, PS, vp, sz, C.POINTER(_State)]),
        "rs_factors_finalize": (C.c_int, [C.c_char_p, C.POINTER(_State)]),
        "rs_state_write": (C.c_int, [C.c_char_p, C.POINTER(_State), PS]),
        "rs_state_read": (C.c_int, [C.c_char_p, C.POINTER(_State), PS]),
        "rs_state_resume": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_State), PS, C.POINTER(C.c_int)]),
        "rs_ctx_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
        "rs_ctx_destroy": (None, [vp]),
        "rs_ctx_set_stream": (C.c_int, [vp, vp]),
        "rs_device_count": (C.c_int, []),
        "rs_job_load": (C.c_int, [vp, PS]),
        "rs_run_range": (C.c_int, [vp, u64, u64, C.POINTER(_Counters)]),
        "rs_factors_fetch": (C.c_int, [vp, vp, sz, C.POINTER(sz)]),
        "rs_bitmap_download": (C.c_int, [vp, vp, sz]),
        "rs_counters_get": (C.c_int, [vp, C.POINTER(_Counters)]),
        "rs_primes_generate": (C.c_int, [vp, u64, u64, vp, sz, C.POINTER(sz)]),
        "rs_last_timing": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(u32),
                                     C.POINTER(u32)]),
        "rs_mulmod_peak": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "rs_widemul_peak": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "rs_fpmul_peak": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "rs_primes_generate_noalloc": (C.c_int, [u64, u64, vp, u32, vp, vp]),
        "rs_set_baby_steps": (C.c_int, [vp, u32]),
        "rs_batch_create": (C.c_int, [C.c_int, u32, u32, C.POINTER(vp)]),
        "rs_batch_release": (C.c_int, [vp, u32]),
        "rs_batch_add_clone": (C.c_int, [vp, u32, u64, u64, u32, C.POINTER(u32)]),
        "rs_batch_free_slots": (C.c_int, [vp, C.POINTER(u32), C.POINTER(u32)]),
        "rs_batch_job_bytes": (C.c_int, [vp, u32, C.POINTER(C.c_uint64)]),
        "rs_batch_reserve": (C.c_int, [vp, C.c_uint64]),
        "rs_batch_set_budget": (C.c_int, [vp, u32, u64]),
        "rs_batch_poll": (C.c_int, [vp, vp, vp, vp]),
        "rs_batch_destroy": (None, [vp]),
        "rs_batch_set_stream": (C.c_int, [vp, vp]),
        "rs_batch_add": (C.c_int, [vp, PS, u64, u64, u32, C.POINTER(u32)]),
        "rs_batch_run": (C.c_int, [vp, u32, C.POINTER(C.c_int)]),
        "rs_batch_factors_fetch": (C.c_int, [vp, u32, vp, sz, C.POINTER(sz)]),
        "rs_batch_bitmap_download": (C.c_int, [vp, u32, vp, sz]),
        "rs_batch_job_info": (C.c_int, [vp, u32, C.POINTER(u32), C.POINTER(u64), C.POINTER(C.c_int)]),
        "rs_batch_counters": (C.c_int, [vp, C.POINTER(_Counters)]),
        "rs_get_baby_steps": (C.c_int, [vp, C.POINTER(u32), C.POINTER(C.c_int)]),
        "rs_set_wait_limit": (C.c_int, [vp, u32, C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _lib = L
    return L


class RSError(RuntimeError):
    def __init__(self, code, what=""):
        L = lib()
        msg = "%s: %s (%s)" % (what, L.rs_strerror(code).decode(), L.rs_last_error().decode())
        super().__init__(msg)
        self.code = code


def _check(rc, what):
    if rc != RS_OK:
        raise RSError(rc, what)


class Seqs:
    """A job: up to 100 sequences k*b^n+c over [nmin,nmax] with a candidate bitmap (rs_seqs)."""

    def __init__(self, ptr):
        self._p = ptr

    @classmethod
    def from_abcd_text(cls, text):
        L = lib()
        p = C.POINTER(_Seqs)()
        data = text.encode() if isinstance(text, str) else text
        _check(L.rs_abcd_parse(data, len(data), C.byref(p)), "rs_abcd_parse")
        return cls(p)

    @classmethod
    def from_abcd_file(cls, path):
        L = lib()
        p = C.POINTER(_Seqs)()
        _check(L.rs_abcd_read(os.fsencode(path), C.byref(p)), "rs_abcd_read")
        return cls(p)

    @classmethod
    def create(cls, base, ks, cs, nmin, nmax, bitmap=None):
        L = lib()
        ks = np.ascontiguousarray(ks, dtype=np.uint64)
        cs = np.ascontiguousarray(cs, dtype=np.int32)
        bm = None if bitmap is None else np.ascontiguousarray(bitmap, dtype=np.uint32)
        p = C.POINTER(_Seqs)()
        _check(L.rs_seqs_create(base, len(ks), ks.ctypes.data, cs.ctypes.data, nmin, nmax,
                                None if bm is None else bm.ctypes.data, C.byref(p)), "rs_seqs_create")
        return cls(p)

    def __del__(self):
        if getattr(self, "_p", None) and _lib is not None:
            _lib.rs_seqs_free(self._p)
            self._p = None

    @property
    def s(self):
        return self._p.contents

    base = property(lambda self: self.s.base)
    kcount = property(lambda self: self.s.kcount)
    nmin = property(lambda self: self.s.nmin)
    nmax = property(lambda self: self.s.nmax)
    words_per_seq = property(lambda self: self.s.words_per_seq)

    @property
    def k(self):
        return [int(self.s.k[i]) for i in range(self.kcount)]

    @property
    def c(self):
        return [int(self.s.c[i]) for i in range(self.kcount)]

    @property
    def bitmap(self):
        """numpy view [kcount, words_per_seq] of the library-owned bitmap."""
        n = self.kcount * self.words_per_seq
        arr = np.ctypeslib.as_array(self.s.bitmap, shape=(n,))
        return arr.reshape(self.kcount, self.words_per_seq)

    def count(self):
        return int(lib().rs_seqs_count(self._p))

    def format_factor(self, p, n, seq):
        f = _Factor(p, n, seq)
        buf = C.create_string_buffer(160)
        _check(lib().rs_format_factor(self._p, C.byref(f), buf, 160), "rs_format_factor")
        return buf.value.decode()

    def apply_factor_file(self, path):
        lines = C.c_uint64(0)
        _check(lib().rs_factors_file_apply(os.fsencode(path), self._p, C.byref(lines)), "rs_factors_file_apply")
        return int(lines.value)


class State:
    """Checkpoint scalars (workStatus)."""

    def __init__(self, **kw):
        self.st = _State(**kw)

    def __getattr__(self, k):
        return getattr(self.__dict__["st"], k)

    def write(self, path, seqs):
        _check(lib().rs_state_write(os.fsencode(path), C.byref(self.st), seqs._p), "rs_state_write")

    @classmethod
    def read(cls, path, seqs, pmin, pmax):
        """The state in path, which must belong to seqs and to the p-range [pmin, pmax)."""
        s = cls(pmin=pmin, pmax=pmax)
        rc = lib().rs_state_read(os.fsencode(path), C.byref(s.st), seqs._p)
        if rc != RS_OK:
            raise RSError(rc, "rs_state_read")
        return s

    @classmethod
    def resume(cls, path_a, path_b, seqs, pmin, pmax):
        """The newer valid one of two A/B state files of seqs over [pmin, pmax)."""
        s = cls(pmin=pmin, pmax=pmax)
        which = C.c_int(-1)
        r = lib().rs_state_resume(os.fsencode(path_a), os.fsencode(path_b), C.byref(s.st), seqs._p, C.byref(which))
        return (s, which.value) if r == 1 else (None, -1)

    def commit(self, path, seqs, factors):
        f = np.ascontiguousarray(factors, dtype=FACTOR_DT).copy()
        _check(lib().rs_factors_commit(os.fsencode(path), seqs._p, f.ctypes.data, len(f), C.byref(self.st)),
               "rs_factors_commit")
        return f

    def finalize(self, path):
        _check(lib().rs_factors_finalize(os.fsencode(path), C.byref(self.st)), "rs_factors_finalize")


def verify_factor(p, k, n, c, base):
    return lib().rs_verify_factor(p, k, n, c, base)


def is_prime(n):
    return bool(lib().rs_is_prime(n))


def device_count():
    return lib().rs_device_count()


class Sieve:
    """A device context running jobs (rs_ctx).  Raises when no CUDA device is present."""

    def __init__(self, device=0):
        L = lib()
        self._c = C.c_void_p()
        _check(L.rs_ctx_create(device, C.byref(self._c)), "rs_ctx_create")
        self.seqs = None

    def close(self):
        if getattr(self, "_c", None) and self._c.value:
            lib().rs_ctx_destroy(self._c)
            self._c = C.c_void_p()

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle):
        _check(lib().rs_ctx_set_stream(self._c, C.c_void_p(stream_handle)), "rs_ctx_set_stream")

    def load(self, seqs):
        _check(lib().rs_job_load(self._c, seqs._p), "rs_job_load")
        self.seqs = seqs

    def run(self, p0, p1):
        d = _Counters()
        _check(lib().rs_run_range(self._c, p0, p1, C.byref(d)), "rs_run_range")
        return {f: int(getattr(d, f)) for f in COUNTER_FIELDS}

    def counters(self):
        d = _Counters()
        _check(lib().rs_counters_get(self._c, C.byref(d)), "rs_counters_get")
        return {f: int(getattr(d, f)) for f in COUNTER_FIELDS}

    def factors(self):
        L = lib()
        n = C.c_size_t(0)
        rc = L.rs_factors_fetch(self._c, None, 0, C.byref(n))
        if rc not in (RS_OK, RS_EARG):
            _check(rc, "rs_factors_fetch")
        out = np.zeros(max(n.value, 1), dtype=FACTOR_DT)
        _check(L.rs_factors_fetch(self._c, out.ctypes.data, len(out), C.byref(n)), "rs_factors_fetch")
        return out[: n.value].copy()

    def bitmap(self):
        s = self.seqs
        out = np.zeros(s.kcount * s.words_per_seq, dtype=np.uint32)
        _check(lib().rs_bitmap_download(self._c, out.ctypes.data, len(out)), "rs_bitmap_download")
        return out.reshape(s.kcount, s.words_per_seq)

    def primes(self, p0, p1, cap=None):
        L = lib()
        n = C.c_size_t(0)
        if cap is None:
            _check(L.rs_primes_generate(self._c, p0, p1, None, 0, C.byref(n)), "rs_primes_generate")
            cap = n.value
        out = np.zeros(max(cap, 1), dtype=np.uint64)
        _check(L.rs_primes_generate(self._c, p0, p1, out.ctypes.data, cap, C.byref(n)), "rs_primes_generate")
        return out[: n.value].copy()

    def set_baby_steps(self, q):
        """Force Q baby steps per prime (one of BABY_STEPS), or 0 to choose per job."""
        _check(lib().rs_set_baby_steps(self._c, q), "rs_set_baby_steps")

    def baby_steps(self):
        """(Q in use, whether the per-job tuner is still timing candidates)."""
        q, t = C.c_uint32(0), C.c_int(0)
        _check(lib().rs_get_baby_steps(self._c, C.byref(q), C.byref(t)), "rs_get_baby_steps")
        return q.value, bool(t.value)

    def set_wait_limit(self, tries=0, test_stall=False):
        """Bound on the BSGS kernel's record-copy waits (0: default); test_stall
        makes every CTA's first wait run out, to exercise the error path."""
        _check(lib().rs_set_wait_limit(self._c, tries, 1 if test_stall else 0), "rs_set_wait_limit")

    def widemul_peak(self):
        """10^9 32x32->64 multiplies/s of independent chains on this device."""
        g, ms = C.c_double(0), C.c_double(0)
        _check(lib().rs_widemul_peak(self._c, C.byref(g), C.byref(ms)), "rs_widemul_peak")
        return g.value

    def fpmul_peak(self):
        """10^9 FP64 modular products/s (the steps' product below 2^51) on this device."""
        g, ms = C.c_double(0), C.c_double(0)
        _check(lib().rs_fpmul_peak(self._c, C.byref(g), C.byref(ms)), "rs_fpmul_peak")
        return g.value

    def mulmod_peak(self):
        """10^9 Montgomery products/s of independent chains on this device."""
        g, ms = C.c_double(0), C.c_double(0)
        _check(lib().rs_mulmod_peak(self._c, C.byref(g), C.byref(ms)), "rs_mulmod_peak")
        return g.value

    def last_timing(self):
        b, t = C.c_double(0), C.c_double(0)
        bl, kl = C.c_uint32(0), C.c_uint32(0)
        _check(lib().rs_last_timing(self._c, C.byref(b), C.byref(t), C.byref(bl), C.byref(kl)), "rs_last_timing")
        return {"bsgs_ms_avg": b.value, "total_ms": t.value, "bsgs_launches": bl.value, "kernel_launches": kl.value}


class Batch:
    """Many independent jobs sieved together on one device (rs_batch_*)."""

    def __init__(self, device=0, max_jobs=0, range_slots=0):
        L = lib()
        self._b = C.c_void_p()
        _check(L.rs_batch_create(device, max_jobs, range_slots, C.byref(self._b)), "rs_batch_create")
        self._seqs = {}
        self.max_jobs = max_jobs or 64

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            lib().rs_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        """Run the batch's rounds on a caller stream (not the legacy default stream)."""
        _check(lib().rs_batch_set_stream(self._b, C.c_void_p(stream_handle)), "rs_batch_set_stream")

    def add(self, seqs, p0, p1, q=0):
        """Add a job over [p0, p1) (p0 == p1: a resident template); q fixes its baby steps,
        0 takes a measured or modelled choice.  Returns its slot, or None when no slot is free."""
        j = C.c_uint32(0)
        rc = lib().rs_batch_add(self._b, seqs._p, p0, p1, q, C.byref(j))
        if rc == RS_EBUSY:
            return None
        _check(rc, "rs_batch_add")
        self._seqs[j.value] = seqs
        return j.value

    def add_clone(self, src, p0, p1, nsplit=1):
        """A job copying slot src's sequences and bitmap on the device, its p-range cut into
        nsplit range slots; None when no slot is free."""
        j = C.c_uint32(0)
        rc = lib().rs_batch_add_clone(self._b, src, p0, p1, nsplit, C.byref(j))
        self.last_rc = rc
        if rc in (RS_EBUSY, RS_ENOMEM):
            self.last_error = lib().rs_last_error().decode()
            return None
        _check(rc, "rs_batch_add_clone")
        self._seqs[j.value] = self._seqs[src]
        return j.value

    def job_bytes(self, job):
        """Device memory a job (or a clone of it) holds while admitted."""
        n = C.c_uint64(0)
        _check(lib().rs_batch_job_bytes(self._b, job, C.byref(n)), "rs_batch_job_bytes")
        return n.value

    def reserve(self, nbytes):
        """Map nbytes into the batch's job pool ahead of admissions; False if the device lacks them."""
        rc = lib().rs_batch_reserve(self._b, C.c_uint64(int(nbytes)))
        if rc == RS_ENOMEM:
            return False
        _check(rc, "rs_batch_reserve")
        return True

    def free_slots(self):
        """(free job slots, free range slots)."""
        j, r = C.c_uint32(0), C.c_uint32(0)
        _check(lib().rs_batch_free_slots(self._b, C.byref(j), C.byref(r)), "rs_batch_free_slots")
        return j.value, r.value

    def set_budget(self, job, primes):
        """Primes the job should cover per round from now on (0 pauses it)."""
        _check(lib().rs_batch_set_budget(self._b, job, int(primes)), "rs_batch_set_budget")

    def poll(self):
        """(done, primes tested, p-range left) for every job slot, from one device read."""
        d = np.zeros(self.max_jobs, dtype=np.uint8)
        n = np.zeros(self.max_jobs, dtype=np.uint64)
        r = np.zeros(self.max_jobs, dtype=np.uint64)
        _check(lib().rs_batch_poll(self._b, d.ctypes.data, n.ctypes.data, r.ctypes.data), "rs_batch_poll")
        return d.astype(bool), n, r

    def release(self, job):
        _check(lib().rs_batch_release(self._b, job), "rs_batch_release")
        self._seqs.pop(job, None)

    def run(self, max_rounds=0):
        """Run up to max_rounds rounds (0: to completion); True once every job is done."""
        d = C.c_int(0)
        _check(lib().rs_batch_run(self._b, max_rounds, C.byref(d)), "rs_batch_run")
        return bool(d.value)

    def factors(self, job):
        L = lib()
        n = C.c_size_t(0)
        rc = L.rs_batch_factors_fetch(self._b, job, None, 0, C.byref(n))
        if rc not in (RS_OK, RS_EARG):
            _check(rc, "rs_batch_factors_fetch")
        out = np.zeros(max(n.value, 1), dtype=FACTOR_DT)
        _check(L.rs_batch_factors_fetch(self._b, job, out.ctypes.data, len(out), C.byref(n)), "rs_batch_factors_fetch")
        return out[: n.value].copy()

    def bitmap(self, job):
        s = self._seqs[job]
        out = np.zeros(s.kcount * s.words_per_seq, dtype=np.uint32)
        _check(lib().rs_batch_bitmap_download(self._b, job, out.ctypes.data, len(out)), "rs_batch_bitmap_download")
        return out.reshape(s.kcount, s.words_per_seq)

    def job_info(self, job):
        """(baby steps Q, primes tested, done)."""
        q, n, d = C.c_uint32(0), C.c_uint64(0), C.c_int(0)
        _check(lib().rs_batch_job_info(self._b, job, C.byref(q), C.byref(n), C.byref(d)), "rs_batch_job_info")
        return q.value, n.value, bool(d.value)

    def counters(self):
        d = _Counters()
        _check(lib().rs_batch_counters(self._b, C.byref(d)), "rs_batch_counters")
        return {f: int(getattr(d, f)) for f in COUNTER_FIELDS}


def term_set(factors):
    """Eliminated terms (seq, n): what the reference README says to compare across runs."""
    return set(zip(factors["seq"].tolist(), factors["n"].tolist()))
