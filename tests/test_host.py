"""Host services of the C ABI (CPU only): ABCD input, verification, factor
file and checkpoints, failure handling, and the library's exported symbols."""
import json
import os
import re
import struct

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(rs):
    hdr = open(os.path.join(ROOT, "include", "rssieve_b200.h")).read()
    declared = set(re.findall(r"\b(rs_[a-z0-9_]+)\s*\(", hdr))
    assert declared == set(rs.EXPORTS)
    L = rs.lib()
    for name in declared:
        assert hasattr(L, name), name
    assert L.rs_version().decode().startswith("rssieve_b200")


def test_device_entry_points_fail_cleanly_without_gpu(rs):
    if rs.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(rs.RSError) as e:
        rs.Sieve(0)
    assert e.value.code == rs.RS_ENODEV


def test_abcd_golden(rs):
    exp = json.load(open(os.path.join(GOLD, "abcd_expected.json")))
    s = rs.Seqs.from_abcd_file(os.path.join(GOLD, "abcd_sample.txt"))
    assert s.base == exp["base"] and s.k == exp["k"] and s.c == exp["c"]
    assert s.nmin == exp["nmin"] and s.nmax == exp["nmax"]
    assert s.count() == exp["count"]
    for i, n0 in enumerate(exp["first_n"]):
        off = n0 - s.nmin
        assert (int(s.bitmap[i, off >> 5]) >> (off & 31)) & 1
        below = [n for n in range(s.nmin, n0)]
        for n in below:
            o = n - s.nmin
            assert not (int(s.bitmap[i, o >> 5]) >> (o & 31)) & 1


def test_abcd_rules(rs):
    # nmin rounded down to even, deltas accumulate, comments and blanks skipped, 64-bit k accepted
    t = "# c\n\nABCD 1099511627791*5^$a-1 [1001]\n2\n10\nABCD 3*5^$a+1 [1004] // Sieved to 12\n1\n"
    s = rs.Seqs.from_abcd_text(t)
    assert (s.base, s.kcount, s.nmin, s.nmax) == (5, 2, 1000, 1013)
    assert s.k == [1099511627791, 3] and s.c == [-1, 1]
    assert s.count() == 5
    for bad, msg in [
        ("12\nABCD 3*2^$a+1 [5]\n", "delta line before"),
        ("ABCD 3*2^$a+1 [5]\nABCD 5*3^$a+1 [5]\n", "mismatched base"),
        ("ABCD 3*2^$a+3 [5]\n", "standard form"),
        ("ABCD 0*2^$a+1 [5]\n", "invalid K"),
        ("ABCD 3*2^$a+1 [0]\n", "invalid N0"),
        ("ABCD 3*1^$a+1 [5]\n", "invalid base"),
        ("hello\n", "unrecognised"),
        ("", "no sequences"),
        ("ABCD 3*2^$a+1 [4294967290]\n10\n", "overflow"),
    ]:
        with pytest.raises(rs.RSError) as e:
            rs.Seqs.from_abcd_text(bad)
        assert msg in str(e.value), (bad, str(e.value))
    many = "".join("ABCD %d*2^$a+1 [5]\n" % (2 * i + 3) for i in range(101))
    with pytest.raises(rs.RSError) as e:
        rs.Seqs.from_abcd_text(many)
    assert "too many sequences" in str(e.value)


def test_seqs_create_validation(rs):
    s = rs.Seqs.create(2, [3, 5], [1, -1], 10, 70)
    assert s.count() == 2 * 61
    with pytest.raises(rs.RSError):
        rs.Seqs.create(2, [0, 5], [1, -1], 10, 70)
    with pytest.raises(rs.RSError):
        rs.Seqs.create(2, [3, 5], [2, -1], 10, 70)
    with pytest.raises(rs.RSError):
        rs.Seqs.create(1, [3], [1], 10, 70)


def test_is_prime(rs, oracle):
    for n in list(range(0, 2000)) + [42799, 4294967297, 2 ** 61 - 1, 18446744073709551557, 18446744073709551559]:
        assert rs.is_prime(n) == oracle.is_prime(n), n


def test_factor_line_format_and_reread(rs, tmp_path):
    # the format example of cl_sieve.cpp:827-828
    s = rs.Seqs.create(2, [91549, 131179], [1, -1], 54378800, 72017300)
    assert s.format_factor(1000133, 54378870, 0) == "1000133 | 91549*2^54378870+1\n"
    assert s.format_factor(1000669, 72017282, 1) == "1000669 | 131179*2^72017282-1\n"
    path = tmp_path / "f.out"
    path.write_text("1000133 | 91549*2^54378870+1\n1000669 | 131179*2^72017282-1\n")
    before = s.count()
    assert s.apply_factor_file(str(path)) == 2
    assert s.count() == before - 2
    path.write_text("1000133 | 91549*3^54378870+1\n")       # wrong base
    with pytest.raises(rs.RSError):
        s.apply_factor_file(str(path))
    path.write_text("garbage\n")
    with pytest.raises(rs.RSError):
        s.apply_factor_file(str(path))


def test_commit_verifies_sorts_and_checksums(rs, tmp_path):
    s = rs.Seqs.create(2, [3, 5], [-1, 1], 10, 40)
    st = rs.State(pmin=3, pmax=100)
    f = np.array([(5, 13, 0), (3, 11, 0)], dtype=rs.FACTOR_DT)   # 3*2^13-1 = 5*4915, 3*2^11-1 = 6143 = 3*...? no
    ok = [x for x in f if rs.verify_factor(int(x["p"]), 3, int(x["n"]), -1, 2) == 1]
    f = np.array(ok, dtype=rs.FACTOR_DT)
    path = tmp_path / "fac.out"
    st.commit(str(path), s, f)
    lines = path.read_text().splitlines()
    assert lines == sorted(lines, key=lambda ln: (int(ln.split()[0]), int(ln.split("^")[1][:-2])))
    assert st.factorcount == len(f)
    assert st.checksum == sum(int(x["p"]) + 3 + int(x["n"]) - 1 for x in f) % 2 ** 64
    bad = np.array([(7, 13, 0)], dtype=rs.FACTOR_DT)
    with pytest.raises(rs.RSError) as e:
        st.commit(str(path), s, bad)
    assert e.value.code == rs.RS_EVERIFY
    assert path.read_text().splitlines() == lines          # nothing appended after a false factor
    comp = np.array([(42799, 13, 0)], dtype=rs.FACTOR_DT)  # composite modulus is dropped, not reported
    st.commit(str(path), s, comp)
    assert path.read_text().splitlines() == lines


def test_finalize(rs, tmp_path):
    path = tmp_path / "fac.out"
    path.write_text("")
    st = rs.State(pmin=3, pmax=100)
    st.finalize(str(path))
    assert path.read_text() == "no factors\n"
    st2 = rs.State(pmin=3, pmax=100, factorcount=3)
    path.write_text("a\nb\n")
    with pytest.raises(rs.RSError) as e:                    # missing factors (cl_sieve.cpp:759-763)
        st2.finalize(str(path))
    assert "Missing factors" in str(e.value)


def _ref_state_bytes(pmin, pmax, p, checksum, primecount, factorcount, last_trickle, dupcount, nmin, nmax, base,
                     klist):
    """The reference's fwrite(&workStatus) bytes (cl_sieve.h:21-26, cl_sieve.cpp:189-192)."""
    kcount = len(klist)
    ssum = (base + pmin + pmax + p + checksum + primecount + factorcount + last_trickle + nmin + nmax + kcount +
            dupcount + sum(klist)) % 2 ** 64
    kl = list(klist) + [0] * (100 - kcount)
    return struct.pack("<9Q3Ii100i", pmin, pmax, p, checksum, primecount, factorcount, last_trickle, ssum, dupcount,
                       nmin, nmax, base, kcount, *kl)


def test_checkpoint_is_byte_compatible_with_reference_layout(rs, tmp_path):
    s = rs.Seqs.create(2, [91549, 131179], [1, -1], 1000, 2000)
    st = rs.State(pmin=3, pmax=10 ** 9, p=123456789, checksum=77, primecount=5000, factorcount=4,
                  last_trickle=1700000000, dupcount=9)
    path = tmp_path / "stateA.ckp"
    st.write(str(path), s)
    want = _ref_state_bytes(3, 10 ** 9, 123456789, 77, 5000, 4, 1700000000, 9, 1000, 2000, 2, [91549, -131179])
    assert path.read_bytes() == want
    back = rs.State.read(str(path), s, 3, 10 ** 9)
    assert (back.p, back.checksum, back.primecount, back.factorcount, back.dupcount) == (123456789, 77, 5000, 4, 9)


def test_checkpoint_rejects_corrupt_truncated_and_foreign(rs, tmp_path):
    s = rs.Seqs.create(2, [91549, 131179], [1, -1], 1000, 2000)
    st = rs.State(pmin=3, pmax=10 ** 9, p=5000)
    path = tmp_path / "s.ckp"
    st.write(str(path), s)
    raw = bytearray(path.read_bytes())
    raw[20] ^= 1                                            # flip a bit in p
    path.write_bytes(bytes(raw))
    with pytest.raises(rs.RSError) as e:
        rs.State.read(str(path), s, 3, 10 ** 9)
    assert e.value.code == rs.RS_ESTATE and "Checksum" in str(e.value)
    st.write(str(path), s)
    path.write_bytes(path.read_bytes()[:100])               # truncated
    with pytest.raises(rs.RSError):
        rs.State.read(str(path), s, 3, 10 ** 9)
    st.write(str(path), s)
    other = rs.Seqs.create(2, [91549, 131179], [1, -1], 1000, 2002)
    with pytest.raises(rs.RSError):                         # another job's checkpoint
        rs.State.read(str(path), other, 3, 10 ** 9)
    with pytest.raises(rs.RSError) as e:                    # another p-range's checkpoint
        rs.State.read(str(path), s, 3, 10 ** 9 + 2)
    assert e.value.code == rs.RS_ESTATE and "Invalid checkpoint" in str(e.value)


def test_checkpoint_v2_for_64bit_k(rs, tmp_path):
    s = rs.Seqs.create(5, [1099511627776, 6], [1, -1], 1000, 2000)
    st = rs.State(pmin=2 ** 63, pmax=2 ** 64 - 1, p=2 ** 63 + 5, dupcount=3)
    path = tmp_path / "s.ckp"
    st.write(str(path), s)
    assert path.read_bytes()[:6] == b"RSB200"
    back = rs.State.read(str(path), s, 2 ** 63, 2 ** 64 - 1)
    assert back.p == 2 ** 63 + 5 and back.dupcount == 3


def test_resume_newest_wins_and_tie_goes_to_b(rs, tmp_path):
    s = rs.Seqs.create(2, [3], [1], 10, 20)
    a, b = str(tmp_path / "stateA.ckp"), str(tmp_path / "stateB.ckp")
    assert rs.State.resume(a, b, s, 3, 1000) == (None, -1)
    rs.State(pmin=3, pmax=1000, p=500).write(a, s)
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 0 and st.p == 500
    rs.State(pmin=3, pmax=1000, p=700).write(b, s)
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 1 and st.p == 700
    rs.State(pmin=3, pmax=1000, p=900).write(a, s)
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 0 and st.p == 900
    rs.State(pmin=3, pmax=1000, p=900).write(b, s)
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 1
    with open(b, "r+b") as fh:                               # corrupt B: A is used
        fh.seek(40)
        fh.write(b"\xff")
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 0 and st.p == 900


def test_resume_ignores_a_newer_file_of_another_p_range(rs, tmp_path):
    """A good A for this run and a stale B of another p-range with a larger p:
    B is invalid before the two are compared, so A is resumed (read_state,
    cl_sieve.cpp:236-242,288-318), not a fresh start that truncates the factors."""
    s = rs.Seqs.create(2, [3], [1], 10, 20)
    a, b = str(tmp_path / "stateA.ckp"), str(tmp_path / "stateB.ckp")
    rs.State(pmin=3, pmax=1000, p=500).write(a, s)
    rs.State(pmin=3, pmax=5000, p=4000).write(b, s)
    st, which = rs.State.resume(a, b, s, 3, 1000)
    assert which == 0 and st.p == 500 and st.pmax == 1000
    assert rs.State.resume(a, b, s, 3, 5000)[1] == 1         # B is the valid one for its own range
    assert rs.State.resume(a, b, s, 7, 1000) == (None, -1)


def test_cli_resumes_from_the_file_of_its_own_range(rs, tmp_path):
    """The command line with a valid A and a stale B of a wider range: it must
    resume from A and keep the factor file (checked before any device work: the
    checkpoint says the range is complete)."""
    import subprocess
    abcd = tmp_path / "in.txt"
    abcd.write_text("ABCD 3*2^$a+1 [11]\n4\n")
    s = rs.Seqs.create(2, [3], [1], 10, 15)
    rs.State(pmin=100, pmax=1000, p=1000).write(str(tmp_path / "stateA.ckp"), s)
    rs.State(pmin=100, pmax=9000, p=5000).write(str(tmp_path / "stateB.ckp"), s)
    (tmp_path / "psp_sr2sieve.out").write_text("kept\n")
    r = subprocess.run([rs.CLI_PATH, "-i", str(abcd), "-p", "100", "-P", "1000"], capture_output=True, text=True,
                       cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Resuming from checkpoint in stateA.ckp" in r.stdout and "Workunit complete" in r.stdout
    assert (tmp_path / "psp_sr2sieve.out").read_text() == "kept\n"


def test_cli_argument_errors(rs, tmp_path):
    import subprocess
    cli = rs.CLI_PATH
    r = subprocess.run([cli, "-h"], capture_output=True, text=True)
    assert r.returncode != 0 and "-p #" in r.stdout
    r = subprocess.run([cli, "-p", "5"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "no input file" in r.stdout
    r = subprocess.run([cli, "-s"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "self test not implemented" in r.stdout
    abcd = tmp_path / "in.txt"
    abcd.write_text("ABCD 3*4^$a+1 [5]\n")
    r = subprocess.run([cli, "-i", str(abcd), "-p", "5", "-P", "100"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "perfect power" in r.stdout
    abcd.write_text("ABCD 3*2^$a+1 [5]\n")
    r = subprocess.run([cli, "-i", str(abcd), "-p", "5"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "-p and -P arguments are required" in r.stdout
    r = subprocess.run([cli, "-i", str(abcd), "-p", "500", "-P", "100"], capture_output=True, text=True, cwd=tmp_path)
    assert r.returncode != 0 and "pmin <= pmax" in r.stdout
