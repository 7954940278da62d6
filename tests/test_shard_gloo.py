"""Multi-rank path on CPU: two gloo ranks shard the p-range and merge factor sets.

Each rank stands in for one GPU; the per-window sieve here is the CPU oracle
(this tests the sharding and the merge, not the kernels).  The merged result
must equal a single pass over the whole range: same eliminated terms, and for
each term the smallest prime.
"""
import os
import socket

import numpy as np
import pytest

from rssieve_b200 import shard
from rssieve_b200 import workloads as W


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _job():
    return W.small_job(501, kcount=8, base=2, nmin=1000, nmax=4000, keep=0.4, kmax=1 << 24)


def _rank_main(rank, world, port, out_q):
    import torch.distributed as dist
    from oracle import pyoracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    job = _job()
    oj = O.Job(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])

    def sieve_window(a, b):
        f, _, _ = O.brute(oj, O.primes(a, b))     # claims persist in oj's bitmap across windows
        return f.astype(O.FACTOR_DT)

    merged = shard.run_sharded(sieve_window, 3, 120_000, 10_000)
    out_q.put((rank, merged.tobytes()))
    dist.barrier()
    dist.destroy_process_group()


def test_windows_partition():
    ws = [shard.windows(10, 1000, 37, 3, r) for r in range(3)]
    allw = sorted(w for r in ws for w in r)
    assert allw[0][0] == 10 and allw[-1][1] == 1000
    for (a0, b0), (a1, b1) in zip(allw, allw[1:]):
        assert b0 == a1
    assert shard.windows(10, 20, 100, 4, 3) == []


def test_merge_keeps_smallest_p_per_term():
    f = np.array([(7, 100, 1), (5, 100, 1), (11, 3, 0)], dtype=shard.FACTOR_DT)
    g = np.array([(3, 100, 1), (13, 3, 0), (17, 4, 0)], dtype=shard.FACTOR_DT)
    m = shard.merge_factor_sets([f, g])
    assert m.tolist() == [(3, 100, 1), (11, 3, 0), (17, 4, 0)]


def test_two_gloo_ranks_match_single_pass():
    import multiprocessing as mp
    from oracle import pyoracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m0 = np.frombuffer(res[0], dtype=shard.FACTOR_DT)
    m1 = np.frombuffer(res[1], dtype=shard.FACTOR_DT)
    assert np.array_equal(m0, m1)
    job = _job()
    oj = O.Job(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])
    whole, _, _ = O.brute(oj, O.primes(3, 120_000))
    assert O.term_set(m0) == O.term_set(whole)
    # every merged entry is a real factor of its term
    for p, n, sq in m0.tolist():
        assert O.verify_factor(p, job["k"][sq], n, job["c"][sq], job["base"]) == 1
    assert len(set(zip(m0["seq"].tolist(), m0["n"].tolist()))) == len(m0)
