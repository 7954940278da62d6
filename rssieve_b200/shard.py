"""Multi-GPU form: disjoint p-range shards, one process per GPU.

Primes are independent, so the p-range splits across ranks with no exchange
during the sieve.  The only shared state of the reference, the per-term claim
bitmap (giant.cl:21-39), is reconciled on the host at the end: every rank
reports the terms it eliminated with the prime it used, and the merge keeps,
for each term, the smallest prime (what one GPU sieving the windows in
ascending order reports at low factor density).  The merge runs over
torch.distributed (NCCL or gloo) as a gather of small host arrays; it is not
on the data path.
"""
import numpy as np

from . import FACTOR_DT


def windows(p0, p1, width, world, rank):
    """Window i*world + rank of the split of [p0,p1) into width-sized windows (round-robin)."""
    out = []
    i = 0
    while True:
        a = p0 + (i * world + rank) * width
        if a >= p1:
            break
        out.append((a, min(a + width, p1)))
        i += 1
    return out


def merge_factor_sets(parts):
    """Union of per-rank factor arrays: one entry per term (seq, n), smallest p wins."""
    if not parts:
        return np.zeros(0, dtype=FACTOR_DT)
    allf = np.concatenate([np.asarray(p, dtype=FACTOR_DT) for p in parts])
    if len(allf) == 0:
        return allf
    order = np.lexsort((allf["p"], allf["n"], allf["seq"]))
    allf = allf[order]
    key = allf["seq"].astype(np.uint64) << np.uint64(32) | allf["n"].astype(np.uint64)
    first = np.ones(len(allf), dtype=bool)
    first[1:] = key[1:] != key[:-1]
    out = allf[first]
    return out[np.lexsort((out["n"], out["p"]))]


def gather_factors(local, group=None):
    """All ranks' factor arrays merged (every rank receives the merge)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, np.asarray(local, dtype=FACTOR_DT).tobytes(), group=group)
    return merge_factor_sets([np.frombuffer(b, dtype=FACTOR_DT) for b in parts])


def run_sharded(sieve_window, p0, p1, width, group=None):
    """Run sieve_window(a, b) -> factor array over this rank's windows, then merge across ranks."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    local = [sieve_window(a, b) for a, b in windows(p0, p1, width, world, rank)]
    loc = np.concatenate(local) if local else np.zeros(0, dtype=FACTOR_DT)
    return gather_factors(loc, group)
