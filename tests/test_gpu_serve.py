"""Serving loop: units arrive over time and share the device (continuous batching).

Each unit's eliminated terms and final bitmap must equal the brute-force
oracle's over the unit's file and p-range, and be the same in the mix as when
the unit runs alone (the single-job path on the same file and p-range):
units are device-side clones of their file's resident template, each with its
own bitmap.  At most four units run at once, so later arrivals wait for slots
and are admitted while earlier ones are still running.
"""
import numpy as np
import pytest

from rssieve_b200 import serve
from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu


def _files():
    return [W.small_job(61, kcount=10, base=2, nmin=10000, nmax=60000, keep=0.3, kmax=1 << 24),
            W.small_job(62, kcount=25, base=3, nmin=5000, nmax=30000, keep=0.3, kmax=1 << 28),
            W.small_job(63, kcount=6, base=10, nmin=1000, nmax=90000, keep=0.3, kmax=1 << 20)]


def _terms(f):
    return set(zip(f["seq"].tolist(), f["n"].tolist()))


def test_units_same_alone_and_in_the_mix(rs, sieve, oracle):
    files = _files()
    seqs = [W.seqs_of(f) for f in files]
    g = np.random.default_rng(9)
    units = []
    for k in range(12):
        p0 = int(g.integers(1_000_000, 5_000_000))
        units.append(serve.Unit(k, k % 3, p0, p0 + int(g.integers(1 << 16, 1 << 19)), arrival=0.004 * k))
    srv = serve.Server(seqs, max_units=4)
    try:
        done = srv.run(units, collect_bitmaps=True)
    finally:
        srv.close()
    assert all(u.finished is not None and u.admitted >= u.arrival for u in done)
    assert any(u.admitted > u.arrival for u in done)       # some waited for a slot
    for u in done:
        # against the brute-force oracle: the unit's file over its own p-range
        ofac, _, obm = oracle.brute(oracle_job(oracle, files[u.file]), oracle.primes(u.p0, u.p1), ref_skip=True)
        assert _terms(u.factors) == _terms(ofac), u.uid
        assert np.array_equal(u.bitmap, obm), u.uid
        sieve.load(seqs[u.file])
        cnt = sieve.run(u.p0, u.p1)
        f = sieve.factors()
        assert len(f) > 0
        assert _terms(u.factors) == _terms(f), u.uid
        assert np.array_equal(u.bitmap, sieve.bitmap()), u.uid
        assert u.primes == cnt["primes"]
    st = serve.latency_stats(done)
    assert st["units"] == 12 and 0 < st["p50_s"] <= st["p99_s"]
    assert st["primes"] == sum(u.primes for u in done)
