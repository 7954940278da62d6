"""Failure detection on the device: a bounded wait that runs out.

Every wait in the BSGS kernel is bounded.  The test makes the first record
wait of every CTA target a barrier that nothing completes (rs_set_wait_limit's
test switch, with a short bound), so the bound runs out deterministically:
no copy is lost, no GPU fault is raised, and the kernel lets the copy it was
waiting for land before its CTA exits.  The call must return RS_EDEVICE with
the timeout flag (0x10), and the same context must then run a range correctly
(against the brute-force oracle).
"""
import numpy as np
import pytest

from rssieve_b200 import workloads as W
from tests.conftest import oracle_job

pytestmark = pytest.mark.gpu


def test_record_wait_timeout_is_reported_and_context_recovers(rs, oracle):
    job = W.small_job(71, kcount=12, base=2, nmin=1000, nmax=9000, keep=0.4, kmax=1 << 24)
    p0, p1 = 1_000_000, 1_200_000
    with rs.Sieve(0) as s:
        s.set_baby_steps(4096)
        s.load(W.seqs_of(job))
        s.set_wait_limit(64, test_stall=True)
        with pytest.raises(rs.RSError) as e:
            s.run(p0, p1)
        assert e.value.code == rs.RS_EDEVICE
        assert "0x10" in str(e.value)
        # the context stays usable: the default bound, a fresh load, a correct run
        s.set_wait_limit(0)
        s.load(W.seqs_of(job))
        cnt = s.run(p0, p1)
        fac, bm = s.factors(), s.bitmap()
    plist = oracle.primes(p0, p1)
    ofac, odups, obm = oracle.brute(oracle_job(oracle, job), plist, ref_skip=True)
    assert cnt["primes"] == len(plist)
    assert oracle.term_set(fac) == oracle.term_set(ofac)
    assert np.array_equal(bm, obm)
