"""The oracle pinned against the golden fixtures (CPU only).

The fixtures come from the reference's own kernels/setup.cl, kernels/sort.cl
and verify_factor.c compiled for the CPU and from the brute-force term
oracle (tests/golden/make_golden.py).  These tests hold the oracle's
restatement to them; the GPU tests then hold the CUDA path to the oracle.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _job(oracle, g, tag, base):
    k = g[tag + "_k"].tolist()
    c = g[tag + "_c"].tolist()
    nmin, nmax = int(g[tag + "_nminmax"][0]), int(g[tag + "_nminmax"][1])
    words = (nmax - nmin + 1 + 31) // 32
    return oracle.Job(base, k, c, nmin, nmax, np.zeros((len(k), words), np.uint32))


@pytest.mark.parametrize("base", [2, 3, 5, 6, 7, 10])
def test_setup_restatement_matches_reference_setup_cl(oracle, base):
    """or_setup (restated setup.cl:89-209) == the reference's setup kernel, value for value."""
    g = np.load(os.path.join(GOLD, "setup_ref.npz"))
    tag = "b%d" % base
    job = _job(oracle, g, tag, base)
    Q = int(g[tag + "_nminmax"][2])
    rows, kd = oracle.setup(job, Q, g[tag + "_primes"])
    assert np.array_equal(rows, g[tag + "_rows"])
    assert np.array_equal(kd["hadj"], g[tag + "_kd_hadj"])
    assert np.array_equal(kd["parity"], g[tag + "_kd_parity"])
    assert np.array_equal(kd["kidx"], g[tag + "_kd_kidx"])


@pytest.mark.parametrize("base", [2, 3, 5, 6, 7, 10])
def test_setup_fixture_against_live_reference(oracle, base):
    """When the compiled reference is present, it still produces the fixture (sort outputs included)."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built here")
    g = np.load(os.path.join(GOLD, "setup_ref.npz"))
    tag = "b%d" % base
    job = _job(oracle, g, tag, base)
    Q = int(g[tag + "_nminmax"][2])
    r = oracle.ref_setup_sort(job, Q, 1024, g[tag + "_primes"])
    assert np.array_equal(r["rows"], g[tag + "_rows"])
    assert np.array_equal(r["counts"], g[tag + "_counts"])
    assert np.array_equal(r["rows_cls"], g[tag + "_rows_cls"])
    assert np.array_equal(r["kcounts"], g[tag + "_kcounts"])


HIGH_TAGS = ["p2e50_b2", "cfg2_b2", "p2e64_b5", "cfg4_b5", "p2e64_b3"]


@pytest.mark.parametrize("tag", HIGH_TAGS)
def test_setup_restatement_at_high_p(oracle, tag):
    """The same value-for-value check where the Montgomery carries matter:
    primes from 2^50 and just below 2^64, including the config-2 and config-4
    n-ranges (the reference's own setup.cl rows and kdata as fixtures)."""
    g = np.load(os.path.join(GOLD, "setup_ref.npz"))
    base = int(g[tag + "_base"][0])
    job = _job(oracle, g, tag, base)
    Q = int(g[tag + "_nminmax"][2])
    pl = g[tag + "_primes"]
    assert int(pl[0]) >= 1 << 50
    rows, kd = oracle.setup(job, Q, pl)
    assert np.array_equal(rows, g[tag + "_rows"])
    assert np.array_equal(kd["hadj"], g[tag + "_kd_hadj"])
    assert np.array_equal(kd["parity"], g[tag + "_kd_parity"])
    assert np.array_equal(kd["kidx"], g[tag + "_kd_kidx"])
    assert int((g[tag + "_rows"][:, 0] != 0).sum()) > 200          # most primes searched, not skipped


@pytest.mark.parametrize("tag", HIGH_TAGS)
def test_high_p_setup_fixture_against_live_reference(oracle, tag):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref not built here")
    g = np.load(os.path.join(GOLD, "setup_ref.npz"))
    job = _job(oracle, g, tag, int(g[tag + "_base"][0]))
    r = oracle.ref_setup_sort(job, int(g[tag + "_nminmax"][2]), 1024, g[tag + "_primes"])
    assert np.array_equal(r["rows"], g[tag + "_rows"])
    assert np.array_equal(r["kd"]["hadj"], g[tag + "_kd_hadj"])
    assert np.array_equal(r["counts"], g[tag + "_counts"])
    assert np.array_equal(r["rows_cls"], g[tag + "_rows_cls"])
    assert np.array_equal(r["kcounts"], g[tag + "_kcounts"])


def test_plant_helper_places_real_factors(oracle):
    """The planted-factor helper used by the GPU tests: every (k, n) it returns
    is a term that p divides, within the asked range and k bound."""
    for p in oracle.primes(1 << 50, (1 << 50) + 3000)[:10].tolist():
        for c in (1, -1):
            r = oracle.plant(p, 2, c, 4000000, 10000000, 1 << 32, 1)
            assert r is not None
            k, n = r
            assert k < 1 << 32 and k & 1 and 4000000 <= n < 10000000
            assert (k * pow(2, n, p) + c) % p == 0
            assert oracle.verify_factor(p, k, n, c, 2) == 1


def test_verify_matches_reference_verify_factor(oracle, rs):
    v = json.load(open(os.path.join(GOLD, "verify_ref.json")))
    for case, want in zip(v["cases"], v["ref_result"]):
        assert oracle.verify_factor(*case) == want, case
        assert rs.verify_factor(*case) == want, case
    assert sum(1 for r in v["ref_result"] if r == 1) >= 100
    assert sum(1 for r in v["ref_result"] if r == -1) >= 8


def test_sprp2_matches_reference(oracle):
    v = json.load(open(os.path.join(GOLD, "sprp2_ref.json")))
    for n, want in zip(v["n"], v["ref_sprp2"]):
        assert oracle.sprp2(n) == want, n
    # the reference's 2-PRP prime set differs from the true primes by exactly
    # the base-2 strong pseudoprimes coprime to 2..113
    diff = sorted(set(oracle.prp2(3, 200000).tolist()) - set(oracle.primes(3, 200000).tolist()))
    assert diff == v["prp2_minus_primes_3_200000"]
    assert diff[:2] == [42799, 49141]


def test_true_primes_against_trial_division(oracle):
    ps = oracle.primes(3, 20000)
    want = [n for n in range(3, 20000, 2) if all(n % d for d in range(3, int(n ** 0.5) + 1, 2))]
    assert ps.tolist() == want
    assert oracle.primes(2 ** 64 - 100, 2 ** 64 - 1).tolist() == [18446744073709551521, 18446744073709551533,
                                                                   18446744073709551557]


def _brute_jobs():
    g = np.load(os.path.join(GOLD, "brute_jobs.npz"))
    seeds = sorted({int(k.split("_")[0][1:]) for k in g.files})
    return g, seeds


@pytest.mark.parametrize("idx", range(5))
def test_brute_force_oracle_reproduces_fixture(oracle, idx):
    g, seeds = _brute_jobs()
    tag = "s%d" % seeds[idx]
    base, kc, nmin, nmax, p0, p1, dups = [int(x) for x in g[tag + "_meta"]]
    job = oracle.Job(base, g[tag + "_k"].tolist(), g[tag + "_c"].tolist(), nmin, nmax, g[tag + "_bitmap"])
    f, d, bm = oracle.brute(job, oracle.primes(p0, p1))
    assert sorted(oracle.term_set(f)) == [tuple(x) for x in g[tag + "_terms"].tolist()]
    assert d == dups
    assert np.array_equal(bm, g[tag + "_bitmap_after"])


@pytest.mark.parametrize("idx", range(5))
def test_bsgs_port_matches_brute_force(oracle, idx):
    """The CPU port of the reference BSGS kernels eliminates exactly the brute-force term set."""
    g, seeds = _brute_jobs()
    tag = "s%d" % seeds[idx]
    base, kc, nmin, nmax, p0, p1, dups = [int(x) for x in g[tag + "_meta"]]
    if nmin % 2:
        pytest.skip("the reference kernels assume an even nmin (read_input rounds it down, inputfile.cpp:405-407)")
    job = oracle.Job(base, g[tag + "_k"].tolist(), g[tag + "_c"].tolist(), nmin, nmax, g[tag + "_bitmap"])
    f, st, bm = oracle.bsgs(job, oracle.primes(p0, p1), nthreads=1)
    assert sorted(oracle.term_set(f)) == [tuple(x) for x in g[tag + "_terms"].tolist()]
    assert np.array_equal(bm, g[tag + "_bitmap_after"])
    assert st["dup_inrange"] == dups


def test_bsgs_port_threads_same_terms(oracle):
    g, seeds = _brute_jobs()
    tag = "s%d" % seeds[3]
    base, kc, nmin, nmax, p0, p1, dups = [int(x) for x in g[tag + "_meta"]]
    job = oracle.Job(base, g[tag + "_k"].tolist(), g[tag + "_c"].tolist(), nmin, nmax, g[tag + "_bitmap"])
    f1, _, bm1 = oracle.bsgs(job, oracle.primes(p0, p1), nthreads=1)
    f4, _, bm4 = oracle.bsgs(job, oracle.primes(p0, p1), nthreads=4)
    assert oracle.term_set(f1) == oracle.term_set(f4)
    assert np.array_equal(bm1, bm4)


def test_ref_params_rule(oracle):
    """build_giant_kernels' Q/M rule, cl_sieve.cpp:893-938, on the benchmark n-ranges."""
    assert oracle.ref_params(100000, 299999) == {"Q": 1024, "hsize": 2048, "m": 196, "QQ": 2048, "mm": 98}
    assert oracle.ref_params(4000000, 9999999) == {"Q": 4096, "hsize": 8192, "m": 1465, "QQ": 8192, "mm": 733}
    assert oracle.ref_params(1000000, 2999999)["Q"] == 2048
    assert oracle.ref_params(1000000, 2999999)["m"] == 977


def test_verify_and_sort_drops_composite_and_flags_false(oracle):
    job = oracle.Job(2, [3, 5], [-1, 1], 10, 40, np.zeros((2, 1), np.uint32))
    f = np.zeros(3, dtype=oracle.FACTOR_DT)
    real = 13                        # 3*2^13-1 = 24575 = 5*4915
    f[0] = (5, real, 0)
    f[1] = (42799, 20, 0)            # composite modulus: dropped like a 2-PRP (cl_sieve.cpp:612-613)
    f[2] = (11, 20, 1)               # 11 does not divide 5*2^20+1 = 5242881 = 11*476625+6
    kept, bad, cs = oracle.verify_and_sort(job, f)
    assert bad
    assert kept.tolist() == [(5, real, 0)]


def test_bench_reference_rule_matches_oracle_restatement(oracle):
    """bench.py's statement of the reference's Q/M rule (cl_sieve.cpp:893-938),
    used to report work per prime against it, agrees with the oracle's own
    restatement on every config's n-range and on the rule's edges."""
    import bench
    ranges = [(100000, 299999), (4000000, 9999999), (1000000, 2999999), (1000, 1000), (1000, 2047),
              (1000, 1000 + 1024 * 1024), (1000, 1000 + 1024 * 1024 + 1), (10 ** 6, 10 ** 6 + 10 ** 7)]
    for nmin, nmax in ranges:
        got = bench.reference_params(nmin, nmax)
        want = oracle.ref_params(nmin, nmax)
        assert (got["Q"], got["M"], got["MM"]) == (want["Q"], want["m"], want["mm"]), (nmin, nmax)
    assert bench.reference_params(4000000, 9999999) == {"Q": 4096, "M": 1465, "MM": 733}
