"""ctypes wrapper for the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  It wraps oracle/_build/liboracle.so (the plain-C restatement of
the reference algorithm, see oracle/rsoracle.h) and, when present,
oracle/_ref/librsref.so (the reference's own kernels/setup.cl, sort.cl and
verify_factor.c compiled for the CPU, see oracle/ref_kernels.cpp).
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "librsref.so")
MAX_SEQ = 100

FACTOR_DT = np.dtype([("p", "<u8"), ("n", "<u4"), ("seq", "<u4")])
KDATA_DT = np.dtype([("hadj", "<u8"), ("parity", "<i4"), ("kidx", "<i4")])


class _Job(C.Structure):
    _fields_ = [
        ("base", C.c_uint32), ("kcount", C.c_uint32), ("nmin", C.c_uint32), ("nmax", C.c_uint32),
        ("words_per_seq", C.c_uint32), ("k", C.c_uint64 * MAX_SEQ), ("c", C.c_int32 * MAX_SEQ),
        ("bitmap", C.POINTER(C.c_uint32)),
    ]


class _Params(C.Structure):
    _fields_ = [("Q", C.c_uint32), ("hsize", C.c_uint32), ("m", C.c_uint32), ("QQ", C.c_uint32), ("mm", C.c_uint32)]


class _Stats(C.Structure):
    _fields_ = [("mulmods", C.c_uint64), ("lookups", C.c_uint64), ("dup_ref", C.c_uint64),
                ("dup_inrange", C.c_uint64), ("skipped", C.c_uint64)]


_lib = None
_ref = None


def build(refdir=None):
    """Compile the oracle, and the reference kernels when refdir (default: the
    RSSIEVE_REFERENCE_DIR environment variable) names the reference checkout."""
    refdir = refdir or os.environ.get("RSSIEVE_REFERENCE_DIR", "")
    cmd = ["make", "-s", "-C", HERE]
    if refdir:
        cmd.append("REFDIR=" + os.path.abspath(refdir))
    subprocess.run(cmd, check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u64, u32, i32, p64 = C.c_uint64, C.c_uint32, C.c_int32, C.POINTER(C.c_uint64)
        L.or_primes.restype = C.c_size_t
        L.or_primes.argtypes = [u64, u64, p64, C.c_size_t]
        L.or_prp2.restype = C.c_size_t
        L.or_prp2.argtypes = [u64, u64, p64, C.c_size_t]
        L.or_is_prime.restype = C.c_int
        L.or_is_prime.argtypes = [u64]
        L.or_sprp2.restype = C.c_int
        L.or_sprp2.argtypes = [u64]
        L.or_verify_factor.restype = C.c_int
        L.or_verify_factor.argtypes = [u64, u64, u32, i32, u32]
        L.or_brute.restype = C.c_size_t
        L.or_brute.argtypes = [C.POINTER(_Job), p64, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t, p64]
        L.or_bsgs.restype = C.c_size_t
        L.or_bsgs.argtypes = [C.POINTER(_Job), p64, C.c_size_t, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(_Stats)]
        L.or_ref_params.restype = _Params
        L.or_ref_params.argtypes = [u32, u32]
        L.or_setup.restype = None
        L.or_setup.argtypes = [C.POINTER(_Job), u32, p64, C.c_size_t, p64, C.c_void_p]
        L.or_verify_and_sort.restype = C.c_size_t
        L.or_verify_and_sort.argtypes = [C.POINTER(_Job), C.c_void_p, C.c_size_t, C.POINTER(C.c_int), p64]
        L.or_plant.restype = C.c_int
        L.or_plant.argtypes = [u64, u32, i32, u32, u32, u64, C.c_int, p64, C.POINTER(u32)]
        L.or_m_mul.restype = u64
        L.or_m_mul.argtypes = [u64, u64, u64, u64]
        L.or_invert.restype = u64
        L.or_invert.argtypes = [u64]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(REF_PATH)


def ref():
    global _ref
    if _ref is None:
        R = C.CDLL(REF_PATH)
        u64, u32, i32 = C.c_uint64, C.c_uint32, C.c_int32
        R.rsref_setup_sort.restype = C.c_int
        R.rsref_setup_sort.argtypes = [u32, u32, C.c_void_p, u32, u32, u32, C.c_void_p, u32] + [C.c_void_p] * 9
        R.rsref_verify_factor.restype = C.c_int
        R.rsref_verify_factor.argtypes = [u64, u64, u32, i32, u32]
        R.rsref_is_prime.restype = C.c_int
        R.rsref_is_prime.argtypes = [u64]
        R.rsref_sprp2.restype = C.c_int
        R.rsref_sprp2.argtypes = [u64]
        _ref = R
    return _ref


def _p64(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


class Job:
    """A sieve job: sequences k_i*b^n+c_i with candidate bitmap over [nmin,nmax]."""

    def __init__(self, base, ks, cs, nmin, nmax, bitmap):
        assert len(ks) == len(cs) and 0 < len(ks) <= MAX_SEQ
        self.base, self.ks, self.cs = int(base), [int(k) for k in ks], [int(c) for c in cs]
        self.nmin, self.nmax = int(nmin), int(nmax)
        self.words = (self.nmax - self.nmin + 1 + 31) // 32
        self.bitmap = np.ascontiguousarray(bitmap, dtype=np.uint32).reshape(len(ks), self.words).copy()

    def _c(self, bitmap):
        j = _Job()
        j.base, j.kcount, j.nmin, j.nmax, j.words_per_seq = self.base, len(self.ks), self.nmin, self.nmax, self.words
        for i, (k, c) in enumerate(zip(self.ks, self.cs)):
            j.k[i], j.c[i] = k, c
        j.bitmap = bitmap.ctypes.data_as(C.POINTER(C.c_uint32))
        return j


def primes(lo, hi):
    L = lib()
    n = L.or_primes(lo, hi, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    L.or_primes(lo, hi, _p64(out), n)
    return out[:n]


def prp2(lo, hi):
    L = lib()
    n = L.or_prp2(lo, hi, None, 0)
    out = np.zeros(max(n, 1), dtype=np.uint64)
    L.or_prp2(lo, hi, _p64(out), n)
    return out[:n]


def is_prime(n):
    return bool(lib().or_is_prime(n))


def verify_factor(p, k, n, c, base):
    return lib().or_verify_factor(p, k, n, c, base)


def brute(job, plist, ref_skip=True, cap=1 << 22):
    """Brute-force term oracle; returns (factors, dups, bitmap_after)."""
    L = lib()
    bm = job.bitmap.copy()
    j = job._c(bm)
    pl = np.ascontiguousarray(plist, dtype=np.uint64)
    out = np.zeros(cap, dtype=FACTOR_DT)
    d = C.c_uint64(0)
    n = L.or_brute(C.byref(j), _p64(pl), len(pl), 1 if ref_skip else 0, out.ctypes.data, cap, C.byref(d))
    assert n <= cap, "oracle factor buffer overflow"
    return out[:n].copy(), int(d.value), bm


def bsgs(job, plist, nthreads=1, cap=1 << 22):
    """CPU port of the reference BSGS pipeline; returns (factors, stats dict, bitmap_after)."""
    L = lib()
    bm = job.bitmap.copy()
    j = job._c(bm)
    pl = np.ascontiguousarray(plist, dtype=np.uint64)
    out = np.zeros(cap, dtype=FACTOR_DT)
    st = _Stats()
    n = L.or_bsgs(C.byref(j), _p64(pl), len(pl), nthreads, out.ctypes.data, cap, C.byref(st))
    assert n <= cap, "oracle factor buffer overflow"
    stats = {f: int(getattr(st, f)) for f, _ in _Stats._fields_}
    return out[:n].copy(), stats, bm


def plant(p, base, c, n_lo, n_hi, kmax, parity=-1):
    """(k, n) with p | k*base^n+c, n in [n_lo, n_hi), k < kmax of the given
    parity (0 even, 1 odd, -1 any), the first such n; None when none exists."""
    k, n = C.c_uint64(0), C.c_uint32(0)
    ok = lib().or_plant(p, base, c, n_lo, n_hi, kmax, parity, C.byref(k), C.byref(n))
    return (int(k.value), int(n.value)) if ok else None


def ref_params(nmin, nmax):
    r = lib().or_ref_params(nmin, nmax)
    return {f: int(getattr(r, f)) for f, _ in _Params._fields_}


def setup(job, Q, plist):
    """Restated setup.cl: returns (rows[np,8], kdata[np,kcount])."""
    L = lib()
    pl = np.ascontiguousarray(plist, dtype=np.uint64)
    rows = np.zeros((len(pl), 8), dtype=np.uint64)
    kd = np.zeros((len(pl), len(job.ks)), dtype=KDATA_DT)
    j = job._c(job.bitmap)
    L.or_setup(C.byref(j), Q, _p64(pl), len(pl), _p64(rows), kd.ctypes.data)
    return rows, kd


def ref_setup_sort(job, Q, LS, plist):
    """The reference's own setup.cl + sort.cl (compiled for the CPU); needs k < 2^31."""
    R = ref()
    K = len(job.ks)
    kl = np.array([k if c > 0 else -k for k, c in zip(job.ks, job.cs)], dtype=np.int32)
    assert all(k < 2 ** 31 for k in job.ks)
    pl = np.ascontiguousarray(plist, dtype=np.uint64)
    npr = len(pl)
    rows = np.zeros((npr, 8), dtype=np.uint64)
    hadj = np.zeros((npr, K), dtype=np.uint64)
    par = np.zeros((npr, K), dtype=np.int32)
    kidx = np.zeros((npr, K), dtype=np.int32)
    counts = np.zeros(3, dtype=np.uint32)
    rows_cls = np.zeros((3, npr, 8), dtype=np.uint64)
    kp_hadj = np.zeros((3, npr, K), dtype=np.uint64)
    kp_kidx = np.zeros((3, npr, K), dtype=np.int32)
    kcounts = np.zeros((3, npr), dtype=np.int32)
    rc = R.rsref_setup_sort(job.base, K, kl.ctypes.data, job.nmin, Q, LS, pl.ctypes.data, npr,
                            rows.ctypes.data, hadj.ctypes.data, par.ctypes.data, kidx.ctypes.data,
                            counts.ctypes.data, rows_cls.ctypes.data, kp_hadj.ctypes.data,
                            kp_kidx.ctypes.data, kcounts.ctypes.data)
    if rc != 0:
        raise ValueError("no compiled reference namespace for base %d" % job.base)
    kd = np.zeros((npr, K), dtype=KDATA_DT)
    kd["hadj"], kd["parity"], kd["kidx"] = hadj, par, kidx
    return dict(rows=rows, kd=kd, counts=counts, rows_cls=rows_cls, kp_hadj=kp_hadj, kp_kidx=kp_kidx,
                kcounts=kcounts)


def ref_verify_factor(p, k, n, c, base):
    return ref().rsref_verify_factor(p, k, n, c, base)


def ref_is_prime(p):
    return bool(ref().rsref_is_prime(p))


def ref_sprp2(n):
    return bool(ref().rsref_sprp2(n))


def sprp2(n):
    return bool(lib().or_sprp2(n))


def verify_and_sort(job, factors):
    L = lib()
    f = np.ascontiguousarray(factors.copy())
    bad = C.c_int(0)
    cs = C.c_uint64(0)
    j = job._c(job.bitmap)
    n = L.or_verify_and_sort(C.byref(j), f.ctypes.data, len(f), C.byref(bad), C.byref(cs))
    return f[:n].copy(), bool(bad.value), int(cs.value)


def term_set(factors):
    """Set of eliminated terms (seq, n) -- what the reference README says to compare."""
    return set(zip(factors["seq"].tolist(), factors["n"].tolist()))
