"""Seeded synthetic sieve jobs with the shapes of the benchmark configurations.

No public dataset is involved: jobs are drawn from a seeded splitmix64 stream
(k values, signs, bases, ranges) and numpy's PCG64 (candidate bitmaps), and
can be written as sr2sieve/sr5sieve ABCD text for the command line.

  config 1  8 seqs k*2^n-1, k odd in [3,2^20), n in [1e5,3e5) kept w.p. 0.06,
            p in [1e12, 1e12+1e8)
  config 2  100 seqs b=2 (50 with +1, 50 with -1), k odd in [3,2^32),
            n in [4e6,1e7) kept w.p. 0.03, p in [2^50, 2^50+2^38)
  config 3  48 jobs: 1..100 seqs, b in {2,3,5,6,10}, k in [2,2^31) with the
            parity that makes every term odd, n from 1e6 over a log-uniform
            width in [1e5,1e7], survival in [0.02,0.10], p-range of width 2^32
            starting log-uniformly in [2^44,2^60]
  config 4  20 seqs b=5, k even in [2,2^40), c alternating, n in [1e6,3e6)
            kept w.p. 0.05, p in [2^64-2^36, 2^64-1)
  config 5  work units: slices of width 2^U{30..36} starting log-uniformly
            in [2^44,2^62] over one of 16 config-2-style files of 1..100 seqs
"""
import math

import numpy as np

MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.x = seed & MASK64

    def next(self):
        self.x = (self.x + 0x9E3779B97F4A7C15) & MASK64
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self, lo, hi):
        """integer in [lo, hi)"""
        return lo + self.next() % (hi - lo)

    def real(self):
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def log_uniform(self, lo, hi):
        return int(math.exp(math.log(lo) + self.real() * (math.log(hi) - math.log(lo))))


def random_bitmap(kcount, nmin, nmax, keep, seed, n_lo=None, n_hi=None):
    """kcount x words bitmap; bit (n-nmin) set with probability keep for n in [n_lo, n_hi)."""
    L = nmax - nmin + 1
    words = (L + 31) // 32
    n_lo = nmin if n_lo is None else n_lo
    n_hi = nmax + 1 if n_hi is None else n_hi
    rng = np.random.Generator(np.random.PCG64(seed))
    out = np.zeros((kcount, words), dtype=np.uint32)
    for i in range(kcount):
        bits = np.zeros(words * 32, dtype=bool)
        a, b = n_lo - nmin, n_hi - nmin
        bits[a:b] = rng.random(b - a, dtype=np.float32) < keep
        out[i] = np.packbits(bits, bitorder="little").view(np.uint32)
    return out


def _distinct(gen, count, draw):
    seen, out = set(), []
    while len(out) < count:
        v = draw()
        if v not in seen:
            seen.add(v)
            out.append(v)
    return out


def job_dict(base, ks, cs, nmin, nmax, bitmap, prange=None, name=""):
    return {"name": name, "base": int(base), "k": [int(x) for x in ks], "c": [int(x) for x in cs],
            "nmin": int(nmin), "nmax": int(nmax), "bitmap": bitmap, "prange": prange}


def config1(seed=1):
    g = SplitMix64(seed)
    ks = _distinct(g, 8, lambda: g.uniform(3, 1 << 20) | 1)
    nmin, nmax = 100000, 299999
    bm = random_bitmap(8, nmin, nmax, 0.06, seed)
    return job_dict(2, ks, [-1] * 8, nmin, nmax, bm, (10 ** 12, 10 ** 12 + 10 ** 8), "config1")


def config2(seed=2, kcount=100):
    g = SplitMix64(seed)
    ks = _distinct(g, kcount, lambda: g.uniform(3, 1 << 32) | 1)
    cs = [1 if i < kcount // 2 else -1 for i in range(kcount)]
    nmin, nmax = 4000000, 9999999
    bm = random_bitmap(kcount, nmin, nmax, 0.03, seed)
    return job_dict(2, ks, cs, nmin, nmax, bm, (1 << 50, (1 << 50) + (1 << 38)), "config2")


def config3(seed=3, njobs=48):
    g = SplitMix64(seed)
    jobs = []
    for j in range(njobs):
        kc = g.uniform(1, 101)
        b = [2, 3, 5, 6, 10][g.uniform(0, 5)]

        def draw_k():
            k = g.uniform(2, 1 << 31)
            return (k & ~1) if (b & 1) else (k | 1)     # even k for odd b, odd k for even b: odd terms

        ks = _distinct(g, kc, draw_k)
        cs = [1 if g.next() & 1 else -1 for _ in range(kc)]
        nmin = 1000000
        width = g.log_uniform(10 ** 5, 10 ** 7)
        nmax = nmin + width - 1
        keep = 0.02 + 0.08 * g.real()
        p0 = g.log_uniform(1 << 44, 1 << 60)
        bm = random_bitmap(kc, nmin, nmax, keep, seed * 1000 + j)
        jobs.append(job_dict(b, ks, cs, nmin, nmax, bm, (p0, p0 + (1 << 32)), "config3.%d" % j))
    return jobs


def config4(seed=4):
    g = SplitMix64(seed)
    ks = _distinct(g, 20, lambda: g.uniform(2, 1 << 40) & ~1 or 2)
    cs = [1 if i % 2 == 0 else -1 for i in range(20)]
    nmin, nmax = 1000000, 2999999
    bm = random_bitmap(20, nmin, nmax, 0.05, seed)
    return job_dict(5, ks, cs, nmin, nmax, bm, ((1 << 64) - (1 << 36), (1 << 64) - 1), "config4")


def config5_files(seed=5, nfiles=16):
    g = SplitMix64(seed)
    files = []
    for f in range(nfiles):
        kc = g.uniform(1, 101)
        ks = _distinct(g, kc, lambda: g.uniform(3, 1 << 32) | 1)
        cs = [1 if g.next() & 1 else -1 for _ in range(kc)]
        nmin, nmax = 4000000, 9999999
        bm = random_bitmap(kc, nmin, nmax, 0.03, seed * 100 + f)
        files.append(job_dict(2, ks, cs, nmin, nmax, bm, None, "config5.file%d" % f))
    return files


def config5_units(seed=5, nunits=10000, rate=100.0, nfiles=16, width_log2=(30, 36)):
    """Poisson arrivals: list of (arrival_s, file_index, p0, p1); widths 2^U{width_log2}
    (30..36 for the full workload; a scaled-down run passes smaller exponents)."""
    g = SplitMix64(seed + 77)
    t, units = 0.0, []
    for _ in range(nunits):
        t += -math.log(1.0 - g.real()) / rate
        w = 1 << g.uniform(width_log2[0], width_log2[1] + 1)
        p0 = g.log_uniform(1 << 44, 1 << 62)
        units.append((t, g.uniform(0, nfiles), p0, p0 + w))
    return units


def small_job(seed, kcount=8, base=2, nmin=1000, nmax=5000, keep=0.3, kmax=1 << 20, parity_odd_terms=True,
              signs="mixed"):
    """Small random job for parity tests (many factors at small p)."""
    g = SplitMix64(seed)

    def draw_k():
        k = g.uniform(2, kmax)
        if parity_odd_terms:
            k = (k & ~1 or 2) if (base & 1) else (k | 1)
        return k

    ks = _distinct(g, kcount, draw_k)
    if signs == "mixed":
        cs = [1 if g.next() & 1 else -1 for _ in range(kcount)]
    else:
        cs = [int(signs)] * kcount
    bm = random_bitmap(kcount, nmin, nmax, keep, seed)
    return job_dict(base, ks, cs, nmin, nmax, bm, None, "small%d" % seed)


def to_abcd(job):
    """sr2sieve/sr5sieve ABCD text of a job (inputfile.cpp:1-22): header with n0, then deltas."""
    lines = []
    nmin = job["nmin"]
    for i, (k, c) in enumerate(zip(job["k"], job["c"])):
        row = np.unpackbits(job["bitmap"][i].view(np.uint8), bitorder="little")
        ns = (np.nonzero(row)[0] + nmin).tolist()
        ns = [n for n in ns if n <= job["nmax"] and n > 0]
        if not ns:
            continue
        lines.append("ABCD %d*%d^$a%+d [%d]" % (k, job["base"], c, ns[0]))
        prev = ns[0]
        for n in ns[1:]:
            lines.append("%d" % (n - prev))
            prev = n
    return "\n".join(lines) + "\n"


def seqs_of(job):
    """rssieve_b200.Seqs of a job dict."""
    from . import Seqs
    return Seqs.create(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])
