import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def rs():
    import rssieve_b200
    rssieve_b200.lib()
    return rssieve_b200


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def sieve(rs):
    s = rs.Sieve(0)
    yield s
    s.close()


def oracle_job(oracle, job):
    return oracle.Job(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])
