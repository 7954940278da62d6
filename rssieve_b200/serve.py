"""Serving loop: p-range work units arriving over time, sieved with continuous batching.

A unit is a p-range slice over one of several input files (a job: sequences
and candidate bitmap).  Every file is held on the device once, as a resident
batch template (rs_batch_add with an empty range); a unit is admitted as a
device-side clone of its file's template with its own bitmap, so its result
does not depend on which other units share the device.  Admission is by free
batch slots and device memory: a unit that arrives while others are running
joins at the next round boundary, spread over as many free range slots as
finish it in about one round, runs alongside them (one BSGS launch per
geometry group covers every admitted unit), and leaves when its range is done
-- its factors and bitmap are collected and its slots released for the next
arrival.  Latency is measured from arrival and from admission.
"""
import math
import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch


@dataclass
class Unit:
    uid: int
    file: int            # index into the files given to Server
    p0: int
    p1: int
    arrival: float       # seconds after the start of the run
    admitted: float = None
    finished: float = None
    primes: int = 0
    factors: np.ndarray = field(default=None, repr=False)
    bitmap: np.ndarray = field(default=None, repr=False)


class Server:
    """Continuous-batching sieve server over one device."""

    # primes one range slot covers per round (0.6 of the batch's 65536-prime round capacity)
    PRIMES_PER_SLOT_ROUND = 0.6 * 65536

    def __init__(self, files, device=0, max_units=48, range_slots=64):
        # template slots + unit slots; a unit spreads over one or more range slots
        nf = len(files)
        self.batch = Batch(device, max_jobs=nf + max_units, range_slots=range_slots)
        self.templates = []
        for seqs in files:
            t = self.batch.add(seqs, 3, 3)        # p0 == p1: resident template, never runs
            assert t is not None
            self.templates.append(t)
        self.max_units = max_units

    def close(self):
        self.batch.close()

    def run(self, units, clock=time.perf_counter, collect_bitmaps=False):
        """Serve the units (sorted by arrival time); returns them with timings filled."""
        pending = sorted(units, key=lambda u: u.arrival)
        queue, active = [], {}
        t0 = clock()
        i = 0
        while i < len(pending) or queue or active:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                queue.append(pending[i])
                i += 1
            # admit in arrival order while slots and memory allow; a unit takes as many
            # free range slots as finish it in about one round
            while queue and len(active) < self.max_units:
                u = queue[0]
                free = self.batch.free_slots()[1]
                if free == 0:
                    break
                est = (u.p1 - u.p0) / math.log(max(u.p0, 3))
                nsplit = max(1, min(free, math.ceil(est / self.PRIMES_PER_SLOT_ROUND)))
                slot = self.batch.add_clone(self.templates[u.file], u.p0, u.p1, nsplit)
                if slot is None:
                    break
                u.admitted = clock() - t0
                active[slot] = u
                queue.pop(0)
            if not active:
                if i < len(pending):                 # idle until the next arrival
                    wait = pending[i].arrival - (clock() - t0)
                    if wait > 0:
                        time.sleep(wait)
                continue
            self.batch.run(1)                        # one round for every admitted unit
            for slot in list(active):
                q, primes, done = self.batch.job_info(slot)
                if not done:
                    continue
                u = active.pop(slot)
                u.finished = clock() - t0
                u.primes = primes
                u.factors = self.batch.factors(slot)
                if collect_bitmaps:
                    u.bitmap = self.batch.bitmap(slot)
                self.batch.release(slot)
        return units


def latency_stats(units):
    """p50/p99 completion latency from arrival and from admission (seconds), and throughput."""
    lat = np.array([u.finished - u.arrival for u in units])
    lat_adm = np.array([u.finished - u.admitted for u in units])
    span = max(u.finished for u in units) - min(u.arrival for u in units)
    primes = sum(u.primes for u in units)
    return {"units": len(units), "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "p50_from_admission_s": float(np.percentile(lat_adm, 50)),
            "p99_from_admission_s": float(np.percentile(lat_adm, 99)),
            "primes": int(primes), "span_s": float(span), "primes_per_s": float(primes / span) if span > 0 else 0.0}


def poisson_units(n, rate, files, width_log2=(22, 26), p_log2=(44, 62), seed=5):
    """n units with exponential inter-arrival times at `rate` units/s, widths 2^U{width_log2},
    starts log-uniform in 2^p_log2, each over a uniformly chosen file."""
    g = np.random.default_rng(seed)
    t = np.cumsum(g.exponential(1.0 / rate, size=n))
    out = []
    for k in range(n):
        w = 1 << int(g.integers(width_log2[0], width_log2[1] + 1))
        p0 = int(2.0 ** g.uniform(p_log2[0], p_log2[1]))
        out.append(Unit(k, int(g.integers(0, len(files))), p0, p0 + w, float(t[k])))
    return out

