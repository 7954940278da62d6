"""The rssieve command line as a drop-in, end to end on the GPU.

An ABCD file in, `rssieve -p P0 -P P1 -i file -f out` run as a process, and the
factor file read back: every line in the reference's `p | k*b^n+c` format,
sorted by (p, n), every factor real, and the eliminated terms equal to the
brute-force oracle's.  A second run resumes from an A/B checkpoint written at
the middle of the range and must end with the same eliminated terms as one
pass over the whole range.
"""
import re
import subprocess

import pytest

from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu

LINE = re.compile(r"^(\d+) \| (\d+)\*(\d+)\^(\d+)([+-]1)$")


def _job():
    # nmin even: the ABCD reader rounds nmin down to even, as the reference does
    return W.small_job(71, kcount=8, base=2, nmin=1000, nmax=9000, keep=0.4, kmax=1 << 24)


def _read_factors(path):
    lines = [l for l in path.read_text().splitlines() if l.strip()]
    out = []
    for l in lines:
        m = LINE.match(l)
        assert m, l
        out.append(tuple(int(x) for x in m.groups()))
    return out


def _terms(rows):
    return {(k, n, c) for _, k, _, n, c in rows}


def _oracle_terms(oracle, job, p0, p1):
    f, _, _ = oracle.brute(oracle_job(oracle, job), oracle.primes(p0, p1), ref_skip=True)
    return {(job["k"][int(r["seq"])], int(r["n"]), job["c"][int(r["seq"])]) for r in f}


def _run(rs, tmp_path, p0, p1):
    return subprocess.run([rs.CLI_PATH, "-p", str(p0), "-P", str(p1), "-i", "in.abcd", "-f", "out.txt"],
                          capture_output=True, text=True, cwd=tmp_path, timeout=600)


def test_cli_sieves_abcd_file_like_the_oracle(rs, oracle, tmp_path):
    job = _job()
    (tmp_path / "in.abcd").write_text(W.to_abcd(job))
    p0, p1 = 3, 400_000
    r = _run(rs, tmp_path, p0, p1)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = _read_factors(tmp_path / "out.txt")
    assert rows, "expected factors at small p"
    assert [(p, n) for p, _, _, n, _ in rows] == sorted((p, n) for p, _, _, n, _ in rows)
    for p, k, b, n, c in rows[:300]:
        assert b == 2 and rs.verify_factor(p, k, n, c, b) == 1
    assert _terms(rows) == _oracle_terms(oracle, job, p0, p1)
    m = re.search(r"factors (\d+), prime count (\d+)", r.stdout)
    assert m and int(m.group(1)) == len(rows) and int(m.group(2)) == len(oracle.primes(p0, p1))


def test_cli_no_factors_line(rs, tmp_path):
    job = W.small_job(72, kcount=2, base=2, nmin=1000, nmax=1100, keep=0.05, kmax=1 << 20)
    (tmp_path / "in.abcd").write_text(W.to_abcd(job))
    r = _run(rs, tmp_path, 10 ** 15, 10 ** 15 + 100_000)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (tmp_path / "out.txt").read_text() == "no factors\n"


def test_cli_resumes_from_checkpoint(rs, oracle, tmp_path):
    job = _job()
    p0, pm, p1 = 3, 150_000, 400_000
    single = tmp_path / "single"
    single.mkdir()
    (single / "in.abcd").write_text(W.to_abcd(job))
    assert _run(rs, single, p0, p1).returncode == 0
    want = _read_factors(single / "out.txt")

    run = tmp_path / "resume"
    run.mkdir()
    (run / "in.abcd").write_text(W.to_abcd(job))
    r = _run(rs, run, p0, pm)                   # first half: factor file for [p0, pm)
    assert r.returncode == 0, r.stdout + r.stderr
    first = _read_factors(run / "out.txt")
    m = re.search(r"factors (\d+), prime count (\d+), checksum ([0-9A-F]+)", r.stdout)
    assert m
    # a checkpoint of the whole range [p0, p1) stopped at pm, as a 60-second flush would leave it
    seqs = rs.Seqs.from_abcd_file(str(run / "in.abcd"))
    st = rs.State(pmin=p0, pmax=p1, p=pm, checksum=int(m.group(3), 16), primecount=int(m.group(2)),
                  factorcount=len(first), last_trickle=0, dupcount=0)
    st.write(str(run / "stateA.ckp"), seqs)
    (run / "stateB.ckp").unlink(missing_ok=True)
    r = _run(rs, run, p0, p1)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Resuming from checkpoint" in r.stdout
    got = _read_factors(run / "out.txt")
    # the same eliminated terms, each once; which prime reports a term divisible by
    # two primes of one launch is up to the first claimer, as in the reference
    assert _terms(got) == _terms(want)
    assert len(got) == len(_terms(got)) == len(want)
    for p, k, b, n, c in got:
        assert rs.verify_factor(p, k, n, c, b) == 1
    m = re.search(r"prime count (\d+)", r.stdout)
    assert int(m.group(1)) == len(oracle.primes(p0, p1))
