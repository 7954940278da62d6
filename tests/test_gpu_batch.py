"""Batched form: independent jobs advanced together in one rs_batch.

Each job's eliminated terms and final bitmap must equal the brute-force oracle
over its own p-range, and equal what the single-job path (rs_run_range) gives
for the same job and range.  The jobs mix bases, sequence counts, n-ranges and
p-ranges -- one straddles 2^63 and so runs as two ranges (Shoup and
Montgomery giant steps) -- and several need more than one round, so rounds
replayed from the captured graph are covered.
"""
import numpy as np
import pytest

from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu

# seed, kcount, base, nmin, nmax, keep, kmax, p0, p1
JOBS = [
    (51, 12, 2, 1000, 9000, 0.4, 1 << 24, 3, 300_000),
    (52, 30, 3, 20000, 80000, 0.1, 1 << 30, 1_000_000, 1_300_000),
    (53, 8, 5, 100000, 140000, 0.2, 1 << 20, 10 ** 9, 10 ** 9 + 1_000_000),
    (54, 100, 2, 1_000_000, 1_999_999, 0.05, 1 << 28, 3_000_000, 3_002_000),
    (55, 5, 10, 5000, 60000, 0.3, 1 << 20, 50_000, 400_000),
    (56, 20, 6, 1000, 50000, 0.2, 1 << 31, (1 << 63) - (1 << 20), (1 << 63) + (1 << 20)),
    (57, 4, 7, 2000, 10000, 0.5, 1 << 20, 10 ** 7, 10 ** 7 + 3_000_000),
]


def _jobs():
    return [(W.small_job(sd, kcount=kc, base=b, nmin=n0, nmax=n1, keep=kp, kmax=km), p0, p1)
            for sd, kc, b, n0, n1, kp, km, p0, p1 in JOBS]


def _terms(f):
    return set(zip(f["seq"].tolist(), f["n"].tolist()))


def _run_batch(rs, jobs, q=0, rounds_first=1):
    b = rs.Batch(0)
    ids = [b.add(W.seqs_of(job), p0, p1, q) for job, p0, p1 in jobs]
    done = b.run(rounds_first)
    if not done:
        done = b.run(0)
    assert done
    return b, ids


def test_batch_matches_brute_force_oracle(rs, oracle):
    jobs = _jobs()
    b, ids = _run_batch(rs, jobs)
    try:
        for (job, p0, p1), j in zip(jobs, ids):
            plist = oracle.primes(p0, p1)
            ofac, _, obm = oracle.brute(oracle_job(oracle, job), plist, ref_skip=True)
            f = b.factors(j)
            assert _terms(f) == _terms(ofac), (j, job["name"])
            assert np.array_equal(b.bitmap(j), obm), (j, job["name"])
            q, primes, done = b.job_info(j)
            assert done and primes == len(plist) and q in rs.BABY_STEPS
            for row in f[:500]:
                s = int(row["seq"])
                assert rs.verify_factor(int(row["p"]), job["k"][s], int(row["n"]), job["c"][s], job["base"]) == 1
        c = b.counters()
        assert c["primes"] == sum(len(oracle.primes(p0, p1)) for _, p0, p1 in jobs)
    finally:
        b.close()


@pytest.mark.parametrize("q", [1024, 16384])
def test_batch_with_fixed_geometry_matches_single_job_path(rs, sieve, q):
    """All jobs forced to one geometry (one BSGS group per side of 2^63), against
    rs_run_range on the same jobs and ranges."""
    jobs = _jobs()
    b, ids = _run_batch(rs, jobs, q=q, rounds_first=2)
    try:
        for (job, p0, p1), j in zip(jobs, ids):
            sieve.set_baby_steps(q)
            sieve.load(W.seqs_of(job))
            cnt = sieve.run(p0, p1)
            assert _terms(b.factors(j)) == _terms(sieve.factors()), (j, job["name"])
            assert np.array_equal(b.bitmap(j), sieve.bitmap()), (j, job["name"])
            assert b.job_info(j)[1] == cnt["primes"]
    finally:
        sieve.set_baby_steps(0)
        b.close()


def test_batch_config3_shapes_match_single_job_path(rs, sieve):
    """Config-3-shaped jobs (1-100 sequences, bases 2/3/5/6/10, n from 10^6,
    p from 2^44 to 2^60) on narrow windows: batch == single-job path."""
    jobs = W.config3(7, njobs=6)
    wins = [(job["prange"][0], job["prange"][0] + (1 << 22)) for job in jobs]
    b = rs.Batch(0)
    try:
        ids = [b.add(W.seqs_of(job), p0, p1) for job, (p0, p1) in zip(jobs, wins)]
        assert b.run(0)
        for job, j, (p0, p1) in zip(jobs, ids, wins):
            sieve.load(W.seqs_of(job))
            cnt = sieve.run(p0, p1)
            assert _terms(b.factors(j)) == _terms(sieve.factors())
            assert np.array_equal(b.bitmap(j), sieve.bitmap())
            assert b.job_info(j)[1] == cnt["primes"]
    finally:
        b.close()


def test_clone_split_over_range_slots_matches_single_job_path(rs, sieve):
    """A template job cloned over a p-range cut into 7 range slots (one bitmap
    shared by the 7 ranges) gives the single-job path's result."""
    job = W.small_job(58, kcount=16, base=2, nmin=20000, nmax=120000, keep=0.2, kmax=1 << 26)
    seqs = W.seqs_of(job)
    p0, p1 = 2_000_000, 2_600_000
    b = rs.Batch(0, max_jobs=4, range_slots=8)
    try:
        t = b.add(seqs, 3, 3)                       # resident template
        assert b.job_info(t)[1:] == (0, True)
        j = b.add_clone(t, p0, p1, nsplit=7)
        assert b.free_slots() == (2, 1)
        assert b.run(0)
        sieve.load(seqs)
        cnt = sieve.run(p0, p1)
        f = sieve.factors()
        assert len(f) > 0
        assert _terms(b.factors(j)) == _terms(f)
        assert np.array_equal(b.bitmap(j), sieve.bitmap())
        assert b.job_info(j)[1] == cnt["primes"]
        assert np.array_equal(b.bitmap(t), seqs.bitmap)         # the template is untouched
        b.release(j)
        assert b.free_slots() == (3, 8)
    finally:
        b.close()


def test_batch_high_p_edge_matches_oracle(rs, oracle):
    """Config-4 shape in the batch: b = 5, 20 sequences, k even below 2^40, c
    alternating, p just below 2^64 (full-width Montgomery products), the window
    cut over 5 range slots of a clone, beside a small-p job in the same rounds;
    eliminated terms and bitmap equal to the brute-force oracle."""
    job = W.small_job(24, kcount=20, base=5, nmin=1000, nmax=200000, keep=0.05, kmax=1 << 40)
    small = W.small_job(59, kcount=6, base=2, nmin=1000, nmax=9000, keep=0.4, kmax=1 << 24)
    p0, p1 = (1 << 64) - (1 << 22), (1 << 64) - 1
    b = rs.Batch(0, max_jobs=4, range_slots=8)
    try:
        t = b.add(W.seqs_of(job), p0, p0)
        j = b.add_clone(t, p0, p1, nsplit=5)
        s = b.add(W.seqs_of(small), 3, 200_000)
        assert b.run(0)
        for jid, jb, lo, hi in ((j, job, p0, p1), (s, small, 3, 200_000)):
            plist = oracle.primes(lo, hi)
            ofac, _, obm = oracle.brute(oracle_job(oracle, jb), plist, ref_skip=True)
            f = b.factors(jid)
            assert _terms(f) == _terms(ofac), jb["name"]
            assert np.array_equal(b.bitmap(jid), obm), jb["name"]
            assert b.job_info(jid)[1:] == (len(plist), True)
            for row in f[:500]:
                sq = int(row["seq"])
                assert rs.verify_factor(int(row["p"]), jb["k"][sq], int(row["n"]), jb["c"][sq], jb["base"]) == 1
    finally:
        b.close()


def test_batch_config4_job_matches_single_job_path(rs, sieve):
    """The config-4 job itself (n in [10^6, 3*10^6), p from 2^64 - 2^36) on a
    2^24-wide window over 8 range slots: batch == single-job path."""
    job = W.config4()
    seqs = W.seqs_of(job)
    p0 = job["prange"][0]
    p1 = p0 + (1 << 24)
    b = rs.Batch(0, max_jobs=2, range_slots=8)
    try:
        t = b.add(seqs, p0, p0)
        j = b.add_clone(t, p0, p1, nsplit=8)
        assert b.run(0)
        sieve.load(seqs)
        cnt = sieve.run(p0, p1)
        assert _terms(b.factors(j)) == _terms(sieve.factors())
        assert np.array_equal(b.bitmap(j), sieve.bitmap())
        assert b.job_info(j)[1] == cnt["primes"]
    finally:
        b.close()


def test_job_footprint_and_memory_reserve(rs, sieve):
    """A job's footprint is its bitmap plus a 16-byte factor record per candidate
    (and one spare); a reserve of a few footprints maps, and clones admitted
    within it run as usual."""
    job = W.small_job(60, kcount=10, base=2, nmin=1000, nmax=20000, keep=0.3, kmax=1 << 24)
    seqs = W.seqs_of(job)
    b = rs.Batch(0, max_jobs=4, range_slots=4)
    try:
        t = b.add(seqs, 3, 3)
        fb = b.job_bytes(t)
        assert fb == seqs.kcount * seqs.words_per_seq * 4 + (seqs.count() + 1) * 16
        assert b.reserve(4 * fb)
        j1 = b.add_clone(t, 3, 150_000, 2)
        j2 = b.add_clone(t, 150_000, 300_000, 2)
        assert b.job_bytes(j1) == b.job_bytes(j2) == fb
        assert b.run(0)
        sieve.load(seqs)
        sieve.run(3, 300_000)
        assert _terms(b.factors(j1)) | _terms(b.factors(j2)) == _terms(sieve.factors())
    finally:
        b.close()
