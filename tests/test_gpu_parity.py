"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bit-exact integer work: prime sets, eliminated-term sets and final bitmaps
must be identical to the brute-force oracle (which evaluates k*b^n mod p for
every prime and n) on the same seeded inputs.
"""
import numpy as np
import pytest

from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lo,hi", [
    (3, 2_000_000),                                   # exact sieve region, tiny primes
    (4_294_000_000, 4_296_500_000),                   # across 2^32 and 65537^2 (Miller-Rabin starts)
    (1 << 50, (1 << 50) + 30_000_000),                # config 2 region
    (10 ** 12, 10 ** 12 + 20_000_000),                # config 1 region
    ((1 << 64) - (1 << 27), (1 << 64) - 1),           # just below 2^64 (config 4 region)
    (1_000_003, 1_000_004),                           # single odd number, prime
    (1_000_004, 1_000_005),                           # single even number
])
def test_primes_match_oracle(sieve, oracle, lo, hi):
    got = np.sort(sieve.primes(lo, hi))
    want = oracle.primes(lo, hi)
    assert got.dtype == np.uint64
    assert len(got) == len(want)
    assert np.array_equal(got, want)


def _check_job(sieve, oracle, job, p0, p1, rs):
    seqs = W.seqs_of(job)
    sieve.load(seqs)
    cnt = sieve.run(p0, p1)
    fac = sieve.factors()
    bm = sieve.bitmap()
    oj = oracle_job(oracle, job)
    plist = oracle.primes(p0, p1)
    ofac, odups, obm = oracle.brute(oj, plist, ref_skip=True)
    assert oracle.term_set(fac) == oracle.term_set(ofac)
    assert np.array_equal(bm, obm)
    assert cnt["primes"] == len(plist)
    assert cnt["factors"] == len(fac)
    assert cnt["dups"] == odups
    # every reported factor is a real one, by the host verifier
    for f in fac[:2000]:
        seq = int(f["seq"])
        assert rs.verify_factor(int(f["p"]), job["k"][seq], int(f["n"]), job["c"][seq], job["base"]) == 1
    return cnt, fac


@pytest.mark.parametrize("seed,base", [(11, 2), (12, 3), (13, 5), (14, 6), (15, 10), (16, 7)])
def test_small_p_dense_factors(sieve, oracle, rs, seed, base):
    """p from 3: small orders, p dividing k, many duplicates and claims."""
    job = W.small_job(seed, kcount=12, base=base, nmin=1000, nmax=9000, keep=0.4, kmax=1 << 24)
    _check_job(sieve, oracle, job, 3, 300_000, rs)


def test_config1_shape_high_density_window(sieve, oracle, rs):
    job = W.small_job(21, kcount=8, base=2, nmin=100000, nmax=140000, keep=0.06, kmax=1 << 20, signs=-1)
    _check_job(sieve, oracle, job, 10 ** 6, 10 ** 6 + 400_000, rs)


def test_hundred_sequences_mid_p(sieve, oracle, rs):
    job = W.small_job(22, kcount=100, base=2, nmin=20000, nmax=80000, keep=0.05, kmax=1 << 32)
    _check_job(sieve, oracle, job, 5 * 10 ** 7, 5 * 10 ** 7 + 200_000, rs)


def test_odd_nmin_parity_offsets(sieve, oracle, rs):
    job = W.small_job(23, kcount=10, base=2, nmin=3001, nmax=12000, keep=0.5, kmax=1 << 24)
    _check_job(sieve, oracle, job, 1000, 200_000, rs)


def test_large_k_near_2_64(sieve, oracle, rs):
    """config 4 shape on a narrow window: b=5, k < 2^40, p just below 2^64."""
    job = W.small_job(24, kcount=20, base=5, nmin=1000, nmax=200000, keep=0.05, kmax=1 << 40)
    lo = (1 << 64) - (1 << 22)
    _check_job(sieve, oracle, job, lo, (1 << 64) - 1, rs)


@pytest.mark.parametrize("seed,kcount,base", [(31, 100, 2), (32, 12, 2), (33, 40, 3), (34, 24, 7)])
def test_long_n_range_many_giant_chunks(sieve, oracle, rs, seed, kcount, base):
    """n-range of 4*10^6: hundreds of giant steps per target, split into chunks
    whose last one is shorter (a second chain that is empty or one step short),
    against the brute-force oracle over a window with thousands of factors.
    Bases 3 and 7 take the general baby step (b^e added or multiplied)."""
    job = W.small_job(seed, kcount=kcount, base=base, nmin=1_000_000, nmax=4_999_999, keep=0.05, kmax=1 << 28)
    _check_job(sieve, oracle, job, 3_000_000, 3_004_000, rs)


@pytest.mark.parametrize("q", [1024, 2048, 4096, 8192, 16384])
def test_every_baby_step_geometry(sieve, oracle, rs, q):
    """Each BSGS geometry (Q baby steps, its table and block size) against the
    brute-force oracle: dense factors at small p (small orders, table rebuilds)
    and 100 sequences over a long n-range (many giant chunks per target)."""
    sieve.set_baby_steps(q)
    try:
        job = W.small_job(41, kcount=24, base=2, nmin=1000, nmax=30000, keep=0.4, kmax=1 << 24)
        _check_job(sieve, oracle, job, 3, 100_000, rs)
        assert sieve.baby_steps() == (q, False)
        job = W.small_job(42, kcount=100, base=2, nmin=1_000_000, nmax=2_999_999, keep=0.05, kmax=1 << 28)
        _check_job(sieve, oracle, job, 3_000_000, 3_002_000, rs)
    finally:
        sieve.set_baby_steps(0)


def test_tuner_runs_candidates_and_matches_fixed_q(sieve, rs):
    """Automatic Q: the first chunks run the candidate geometries in turn and the
    tuner settles on one; the eliminated terms equal a run with Q fixed."""
    job = W.small_job(43, kcount=8, base=2, nmin=100000, nmax=299999, keep=0.06, kmax=1 << 20, signs=-1)
    p0, p1 = 10 ** 12, 10 ** 12 + 60_000_000          # about 2.2e6 primes, 17 chunks
    sieve.set_baby_steps(0)
    sieve.load(W.seqs_of(job))
    assert sieve.baby_steps()[1]                     # tuning at the start
    cnt_auto = sieve.run(p0, p1)
    q_auto, tuning = sieve.baby_steps()
    assert not tuning and q_auto in rs.BABY_STEPS
    fa, bma = sieve.factors(), sieve.bitmap()
    sieve.set_baby_steps(16384)
    try:
        sieve.load(W.seqs_of(job))
        cnt_fixed = sieve.run(p0, p1)
        ff, bmf = sieve.factors(), sieve.bitmap()
    finally:
        sieve.set_baby_steps(0)
    assert cnt_auto["primes"] == cnt_fixed["primes"]
    assert set(zip(fa["seq"].tolist(), fa["n"].tolist())) == set(zip(ff["seq"].tolist(), ff["n"].tolist()))
    assert np.array_equal(bma, bmf)
    # a batch job of the same shape takes the measured Q, not the cost model's
    b = rs.Batch(0, max_jobs=1, range_slots=1)
    try:
        assert b.job_info(b.add(W.seqs_of(job), p0, p0))[0] == q_auto
    finally:
        b.close()


def _mr7(n):
    """Deterministic 64-bit primality (seven strong bases), for building test inputs."""
    if n < 2:
        return False
    for q in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % q == 0:
            return n == q
    return all(_sprp(n, a) for a in (2, 325, 9375, 28178, 450775, 9780504, 1795265022) if a % n)


def _sprp(n, a):
    d, t = n - 1, 0
    while d % 2 == 0:
        d, t = d // 2, t + 1
    x = pow(a, d, n)
    if x in (1, n - 1):
        return True
    for _ in range(t - 1):
        x = x * x % n
        if x == n - 1:
            return True
    return False


def _base2_strong_pseudoprimes():
    """Composites that pass the base-2 strong test and survive the sieve (no
    factor below 65537): 2^59 - 1 = 179951 * 3203431780337, and products
    p(2p - 1) of two primes near 2^33 and 2^63."""
    out = [(1 << 59) - 1]
    for start in (65537, (1 << 31) + 1):          # odd starts: p steps over odd numbers
        p, found = start, 0
        while found < 6:
            p += 2
            n = p * (2 * p - 1)
            if _mr7(p) and _mr7(2 * p - 1) and _sprp(n, 2):
                out.append(n)
                found += 1
    return out


def test_base2_strong_pseudoprimes_are_rejected(sieve, oracle):
    """The prime generator's test must not stop at base 2: base-2 strong
    pseudoprimes that survive the sieve are composite, the window around
    2^59 - 1 equals the oracle's primes."""
    samples = _base2_strong_pseudoprimes()
    assert len(samples) == 13
    for n in samples:
        assert _sprp(n, 2) and not _mr7(n)
        assert len(sieve.primes(n, n + 1)) == 0, n
    lo = (1 << 59) - 1 - 200_000
    got = np.sort(sieve.primes(lo, lo + 400_000))
    assert np.array_equal(got, oracle.primes(lo, lo + 400_000))
