"""Generate the golden fixtures in this directory.

    python tests/golden/make_golden.py

The reference ships no tests or known-answer vectors, so the fixtures are made
here from the reference's own code where it compiles for the CPU
(oracle/_ref/librsref.so: kernels/setup.cl, kernels/sort.cl and
verify_factor.c built unmodified under oracle/ref_shim.hpp) and from the
brute-force term oracle (oracle/_build/liboracle.so), on seeded inputs:

  setup_ref.npz    per-prime setup rows, kdata and sort outputs of the
                   reference kernels for six small jobs (b = 2,3,5,6,7,10)
                   at p < 4000, and for five jobs at p from 2^50 and just
                   below 2^64 (among them the config-2 and config-4 n-ranges)
  verify_ref.json  verify_factor results (factors, non-factors, composite p)
  sprp2_ref.json   base-2 strong-PRP verdicts, and the composite numbers the
                   reference's 2-PRP generator admits in [3, 2e5)
  brute_jobs.npz   small jobs with their brute-force eliminated terms and
                   final bitmaps
  abcd_sample.txt  an sr2sieve ABCD file with its expected parse in
                   abcd_expected.json
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from rssieve_b200 import workloads as W  # noqa: E402

SETUP_JOBS = [(101, 2, 8), (102, 3, 8), (103, 5, 10), (104, 6, 8), (105, 7, 6), (106, 10, 12)]
# the same rows where the Montgomery carries matter: primes from 2^50 (the
# config-2 p-range) and just below 2^64 (config 4), on small n-ranges and on
# the configurations' own n-ranges.  tag: seed, base, kcount, nmin, nmax, plo, kmax, k parity
SETUP_JOBS_HIGH = {
    "p2e50_b2": (111, 2, 8, 1000, 5000, 1 << 50, 1 << 31, 1),
    "cfg2_b2": (112, 2, 16, 4000000, 9999999, (1 << 50) + (1 << 37), 1 << 31, 1),
    "p2e64_b5": (113, 5, 10, 1000, 5000, (1 << 64) - (1 << 20), 1 << 31, 0),
    "cfg4_b5": (114, 5, 20, 1000000, 2999999, (1 << 64) - (1 << 36), 1 << 31, 0),
    "p2e64_b3": (115, 3, 12, 20000, 80000, (1 << 64) - (1 << 24), 1 << 31, 0),
}
BRUTE_JOBS = [  # seed, base, kcount, nmin, nmax, keep, p0, p1
    (201, 2, 8, 1000, 6000, 0.4, 3, 200000),
    (202, 3, 6, 2000, 5000, 0.5, 3, 150000),
    (203, 5, 10, 500, 4000, 0.3, 1000, 300000),
    (204, 2, 30, 20000, 40000, 0.05, 10 ** 7, 10 ** 7 + 100000),
    (205, 10, 8, 1001, 3000, 0.5, 3, 100000),
]


def job_of(seed, base, kcount, nmin=1000, nmax=5000, keep=0.3):
    j = W.small_job(seed, kcount=kcount, base=base, nmin=nmin, nmax=nmax, keep=keep, kmax=1 << 30)
    return j, O.Job(j["base"], j["k"], j["c"], j["nmin"], j["nmax"], j["bitmap"])


def make_setup():
    out = {}
    for seed, base, kc in SETUP_JOBS:
        j, oj = job_of(seed, base, kc, 1000, 5000)
        pl = O.prp2(3, 4000)[:300]
        Q = O.ref_params(j["nmin"], j["nmax"])["Q"]
        r = O.ref_setup_sort(oj, Q, 1024, pl)
        tag = "b%d" % base
        out[tag + "_k"] = np.array(j["k"], dtype=np.uint64)
        out[tag + "_c"] = np.array(j["c"], dtype=np.int32)
        out[tag + "_nminmax"] = np.array([j["nmin"], j["nmax"], Q], dtype=np.uint32)
        out[tag + "_primes"] = pl
        out[tag + "_rows"] = r["rows"]
        out[tag + "_kd_hadj"] = r["kd"]["hadj"]
        out[tag + "_kd_parity"] = r["kd"]["parity"]
        out[tag + "_kd_kidx"] = r["kd"]["kidx"]
        out[tag + "_counts"] = r["counts"]
        out[tag + "_rows_cls"] = r["rows_cls"]
        out[tag + "_kcounts"] = r["kcounts"]
    for tag, (seed, base, kc, nmin, nmax, plo, kmax, kpar) in SETUP_JOBS_HIGH.items():
        g = W.SplitMix64(seed)
        ks = []
        while len(ks) < kc:
            k = g.uniform(2, kmax)
            k = (k | 1) if kpar else ((k & ~1) or 2)
            if k not in ks:
                ks.append(k)
        cs = [1 if g.next() & 1 else -1 for _ in range(kc)]
        words = (nmax - nmin + 1 + 31) // 32
        oj = O.Job(base, ks, cs, nmin, nmax, np.zeros((kc, words), np.uint32))
        pl = O.prp2(plo, min(plo + 200000, (1 << 64) - 1))[:300]
        Q = O.ref_params(nmin, nmax)["Q"]
        r = O.ref_setup_sort(oj, Q, 1024, pl)
        out[tag + "_base"] = np.array([base], dtype=np.uint32)
        out[tag + "_k"] = np.array(ks, dtype=np.uint64)
        out[tag + "_c"] = np.array(cs, dtype=np.int32)
        out[tag + "_nminmax"] = np.array([nmin, nmax, Q], dtype=np.uint32)
        out[tag + "_primes"] = pl
        out[tag + "_rows"] = r["rows"]
        out[tag + "_kd_hadj"] = r["kd"]["hadj"]
        out[tag + "_kd_parity"] = r["kd"]["parity"]
        out[tag + "_kd_kidx"] = r["kd"]["kidx"]
        out[tag + "_counts"] = r["counts"]
        out[tag + "_rows_cls"] = r["rows_cls"]
        out[tag + "_kcounts"] = r["kcounts"]
    np.savez_compressed(os.path.join(HERE, "setup_ref.npz"), **out)


def make_verify():
    rng = np.random.default_rng(7)
    cases = []
    # true factors found by the brute-force oracle
    j, oj = job_of(301, 2, 8, 1000, 3000, 0.5)
    f, _, _ = O.brute(oj, O.primes(3, 50000))
    for x in f[:120]:
        s = int(x["seq"])
        cases.append((int(x["p"]), j["k"][s], int(x["n"]), j["c"][s], 2))
    # random non-factors, large p, other bases
    for _ in range(120):
        lo = int(rng.integers(1 << 40, 1 << 63))
        pl = O.primes(lo, lo + 2000)
        p = int(pl[0])
        cases.append((p, int(rng.integers(1, 1 << 31)), int(rng.integers(2, 1 << 24)), int(rng.choice([-1, 1])),
                      int(rng.choice([2, 3, 5, 6, 7, 10]))))
    # composite p (base-2 strong pseudoprimes) and near 2^64
    for p in (42799, 49141, 88357, 90751, 104653, 130561, 196093, 4294967297):
        cases.append((p, 3, 100, -1, 2))
    for p in O.primes((1 << 64) - 5000, (1 << 64) - 1)[:20]:
        cases.append((int(p), 5, 12345, 1, 5))
    res = [O.ref_verify_factor(*c) for c in cases]
    with open(os.path.join(HERE, "verify_ref.json"), "w") as fh:
        json.dump({"cases": cases, "ref_result": res}, fh)


def make_sprp2():
    rng = np.random.default_rng(8)
    ns = [int(x) | 1 for x in rng.integers(3, 1 << 62, 300)]
    ns += [42799, 49141, 88357, 90751, 104653, 130561, 196093, 3215031751, 4294967297]
    verdict = [O.ref_sprp2(n) for n in ns]
    diff = sorted(set(O.prp2(3, 200000).tolist()) - set(O.primes(3, 200000).tolist()))
    with open(os.path.join(HERE, "sprp2_ref.json"), "w") as fh:
        json.dump({"n": ns, "ref_sprp2": verdict, "prp2_minus_primes_3_200000": diff}, fh)


def make_brute():
    out = {}
    for seed, base, kc, nmin, nmax, keep, p0, p1 in BRUTE_JOBS:
        j, oj = job_of(seed, base, kc, nmin, nmax, keep)
        f, d, bm = O.brute(oj, O.primes(p0, p1))
        tag = "s%d" % seed
        out[tag + "_meta"] = np.array([base, kc, nmin, nmax, p0, p1, d], dtype=np.uint64)
        out[tag + "_k"] = np.array(j["k"], dtype=np.uint64)
        out[tag + "_c"] = np.array(j["c"], dtype=np.int32)
        out[tag + "_bitmap"] = j["bitmap"]
        out[tag + "_terms"] = np.array(sorted(O.term_set(f)), dtype=np.uint32).reshape(-1, 2)
        out[tag + "_bitmap_after"] = bm
    np.savez_compressed(os.path.join(HERE, "brute_jobs.npz"), **out)


def make_abcd():
    j = W.small_job(401, kcount=5, base=2, nmin=1001, nmax=3000, keep=0.2, kmax=1 << 40)
    text = "# generated by make_golden.py\n\n" + W.to_abcd(j)
    # give the first header the optional '// Sieved to' tail (inputfile.cpp:201-203)
    lines = text.split("\n")
    for i, ln in enumerate(lines):
        if ln.startswith("ABCD"):
            lines[i] = ln + " // Sieved to 1000000"
            break
    text = "\n".join(lines)
    with open(os.path.join(HERE, "abcd_sample.txt"), "w") as fh:
        fh.write(text)
    ns = {}
    for i in range(len(j["k"])):
        row = np.unpackbits(j["bitmap"][i].view(np.uint8), bitorder="little")
        ns[i] = (np.nonzero(row)[0] + j["nmin"]).tolist()
    all_n = [n for v in ns.values() for n in v]
    nmin = min(all_n) & ~1
    exp = {"base": 2, "k": j["k"], "c": j["c"], "nmin": nmin, "nmax": max(all_n),
           "count": len(all_n), "first_n": [v[0] for v in ns.values()]}
    with open(os.path.join(HERE, "abcd_expected.json"), "w") as fh:
        json.dump(exp, fh)


if __name__ == "__main__":
    O.build(os.environ.get("RSSIEVE_REFERENCE_DIR"))
    assert O.ref_available(), "oracle/_ref/librsref.so is needed (build it where the reference tree exists)"
    make_setup()
    make_verify()
    make_sprp2()
    make_brute()
    make_abcd()
    print("fixtures written to", HERE)
