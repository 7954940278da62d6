"""The benchmark configurations' own jobs against the brute-force oracle.

The bench numbers are measured on the config-2 job (100 sequences k*2^n+-1,
k < 2^32, n in [4e6, 1e7)) at p from 2^50, the config-4 job (b = 5, k < 2^40)
just below 2^64, and batches of config-3 jobs.  At those p a random job has
almost no factors, so two kinds of windows are checked, each through the C ABI
against oracle.brute (which evaluates k*b^n mod p for every prime and n):

  - the unchanged jobs over low p-windows, where hundreds of terms fall;
  - the jobs with some sequences re-drawn so that chosen primes of the
    configuration's own p-window divide chosen candidate terms (oracle.plant
    finds, for a prime p, the n whose k = -c*b^-n mod p is small enough), so
    that the search at the benchmark's p-range must find known factors.

The eliminated-term sets, final bitmaps, prime counts and duplicate counts must
equal the oracle's (bit-exact integer work).
"""
import numpy as np
import pytest

from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu


def _terms(f):
    return set(zip(f["seq"].tolist(), f["n"].tolist()))


def _check_single(sieve, oracle, rs, job, p0, p1, min_factors):
    sieve.load(W.seqs_of(job))
    cnt = sieve.run(p0, p1)
    fac = sieve.factors()
    bm = sieve.bitmap()
    plist = oracle.primes(p0, p1)
    ofac, odups, obm = oracle.brute(oracle_job(oracle, job), plist, ref_skip=True)
    assert len(ofac) >= min_factors, "window too sparse to pin anything"
    assert _terms(fac) == _terms(ofac)
    assert np.array_equal(bm, obm)
    assert cnt["primes"] == len(plist)
    assert cnt["factors"] == len(fac) and cnt["dups"] == odups
    for f in fac[:500]:
        s = int(f["seq"])
        assert rs.verify_factor(int(f["p"]), job["k"][s], int(f["n"]), job["c"][s], job["base"]) == 1
    return fac


def plant_job(oracle, job, p0, p1, nplant, kmax, kparity, seqs=None):
    """A copy of job in which up to nplant sequences get a new k (below kmax,
    of parity kparity, sign unchanged) such that one prime of [p0, p1) divides
    one of the sequence's terms; that term is made a candidate.  Returns the
    new job and the planted (seq, n, p)."""
    job = dict(job)
    job["k"] = list(job["k"])
    job["bitmap"] = job["bitmap"].copy()
    primes = oracle.primes(p0, p1).tolist()
    seqs = list(range(len(job["k"]))) if seqs is None else seqs
    planted = []
    pi = 0
    for s in seqs:
        if len(planted) == nplant or pi >= len(primes):
            break
        found = None
        while found is None and pi < len(primes):
            p = primes[pi]
            pi += 7                                   # spread the planted primes over the window
            r = oracle.plant(p, job["base"], job["c"][s], job["nmin"], job["nmax"] + 1, kmax, kparity)
            if r is not None and r[0] not in job["k"]:
                found = (r[0], r[1], p)
        if found is None:
            break
        k, n, p = found
        job["k"][s] = k
        off = n - job["nmin"]
        job["bitmap"][s, off >> 5] |= np.uint32(1 << (off & 31))
        planted.append((s, n, p))
    return job, planted


def test_config2_job_low_p_windows(sieve, oracle, rs):
    """The unchanged config-2 job over two windows where its terms fall often:
    hundreds of eliminated terms, thousands of duplicates, orders of 2 below
    the n-range length."""
    job = W.config2(2)
    _check_single(sieve, oracle, rs, job, 10 ** 7, 10 ** 7 + 3000, 300)
    _check_single(sieve, oracle, rs, job, 10 ** 8, 10 ** 8 + 6000, 50)


def test_config2_job_planted_at_2_50(sieve, oracle, rs):
    """The config-2 job with 24 sequences re-drawn (k odd < 2^32, same signs) so
    that primes of an 8192-wide window at 2^50 + 2^37 (where the bench runs)
    divide candidate terms; the search must find exactly the oracle's set."""
    p0 = (1 << 50) + (1 << 37)
    p1 = p0 + 8192
    job, planted = plant_job(oracle, W.config2(2), p0, p1, 24, 1 << 32, 1, seqs=list(range(0, 100, 4)))
    assert len(planted) == 24
    fac = _check_single(sieve, oracle, rs, job, p0, p1, 24)
    got = _terms(fac)
    assert all((s, n) in got for s, n, _ in planted)


def test_config2_job_planted_across_2_51_and_at_2_62(sieve, oracle, rs):
    """The config-2 job with sequences re-drawn so that primes on both sides of
    2^51 (the engine splits the window there: FP64 baby and giant steps and chi
    chains below, Shoup steps and lazy Montgomery chains above) and primes of
    a window at 2^62 (Shoup steps; k < 2^40 there, so that small enough k
    exist) divide candidate terms."""
    mid = 1 << 51
    job, lo = plant_job(oracle, W.config2(2), mid - 4096, mid, 6, 1 << 32, 1, seqs=list(range(2, 100, 8)))
    job, hi = plant_job(oracle, job, mid, mid + 4096, 6, 1 << 32, 1, seqs=list(range(6, 100, 8)))
    assert len(lo) >= 4 and len(hi) >= 4
    fac = _check_single(sieve, oracle, rs, job, mid - 4096, mid + 4096, len(lo) + len(hi))
    got = _terms(fac)
    assert all((s, n) in got for s, n, _ in lo + hi)
    p0 = 1 << 62
    job, planted = plant_job(oracle, W.config2(2), p0, p0 + 8192, 8, 1 << 40, 1, seqs=list(range(2, 100, 8)))
    assert len(planted) >= 6
    fac = _check_single(sieve, oracle, rs, job, p0, p0 + 8192, len(planted))
    got = _terms(fac)
    assert all((s, n) in got for s, n, _ in planted)


def test_config2_job_planted_across_3_2_49(sieve, oracle, rs):
    """Planted factors on both sides of 3*2^49, three quarters of the way to
    the 2^51 bound of the FP64 products (chi chains, baby and giant steps)."""
    mid = 3 << 49
    job, lo = plant_job(oracle, W.config2(2), mid - 8192, mid, 6, 1 << 32, 1, seqs=list(range(1, 100, 8)))
    job, hi = plant_job(oracle, job, mid, mid + 8192, 6, 1 << 32, 1, seqs=list(range(5, 100, 8)))
    assert len(lo) >= 4 and len(hi) >= 4
    fac = _check_single(sieve, oracle, rs, job, mid - 8192, mid + 8192, len(lo) + len(hi))
    got = _terms(fac)
    assert all((s, n) in got for s, n, _ in lo + hi)


def test_config4_job_planted_near_2_64(sieve, oracle, rs):
    """The config-4 job (b = 5, 20 sequences, k even < 2^40, c alternating) with
    sequences re-drawn so that primes of the first 2^16 of its p-range, just
    below 2^64 (Montgomery giant steps), divide candidate terms."""
    p0 = (1 << 64) - (1 << 36)
    p1 = p0 + (1 << 16)
    job, planted = plant_job(oracle, W.config4(), p0, p1, 6, 1 << 40, 0)
    assert len(planted) >= 3
    fac = _check_single(sieve, oracle, rs, job, p0, p1, len(planted))
    got = _terms(fac)
    assert all((s, n) in got for s, n, _ in planted)


def _batch_vs_brute(rs, oracle, jobs_windows, min_total):
    b = rs.Batch(0, max_jobs=len(jobs_windows), range_slots=len(jobs_windows) + 8)
    try:
        ids = [b.add(W.seqs_of(j), p0, p1) for j, p0, p1 in jobs_windows]
        assert b.run(0)
        total = 0
        for (job, p0, p1), jid in zip(jobs_windows, ids):
            plist = oracle.primes(p0, p1)
            ofac, _, obm = oracle.brute(oracle_job(oracle, job), plist, ref_skip=True)
            f = b.factors(jid)
            assert _terms(f) == _terms(ofac), job["name"]
            assert np.array_equal(b.bitmap(jid), obm), job["name"]
            q, primes, done = b.job_info(jid)
            assert done and primes == len(plist), job["name"]
            total += len(ofac)
        assert total >= min_total
    finally:
        b.close()


def test_config3_jobs_in_one_batch_low_p(rs, oracle):
    """All 48 config-3 jobs (1-100 sequences, b in {2,3,5,6,10}, n-ranges of
    1e5-1e7) in one batch, each over its own low p-window with many factors."""
    jobs = W.config3(3, njobs=48)
    jw = [(j, 2_000_000 + 5000 * i, 2_000_000 + 5000 * i + 600) for i, j in enumerate(jobs)]
    _batch_vs_brute(rs, oracle, jw, 500)


def test_config3_jobs_in_one_batch_planted_at_own_p_range(rs, oracle):
    """The config-3 jobs at the start of their own p-ranges (2^44..2^60), with
    a sequence of each re-drawn (k < 2^31 of the parity that keeps terms odd)
    so that a prime of the window divides a candidate term, where one exists."""
    jobs = W.config3(3, njobs=48)
    jw, planted = [], 0
    for j in jobs:
        p0 = j["prange"][0]
        p1 = p0 + 4096
        kpar = 0 if j["base"] & 1 else 1
        pj, pl = plant_job(oracle, j, p0, p1, 1, 1 << 31, kpar, seqs=[0])
        planted += len(pl)
        jw.append((pj, p0, p1))
    assert planted >= 12
    _batch_vs_brute(rs, oracle, jw, planted)
