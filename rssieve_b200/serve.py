"""Serving loop: p-range work units arriving over time, sieved with continuous batching.

A unit is a p-range slice over one of several input files (a job: sequences
and candidate bitmap).  Every file is held on the device once, as a resident
batch template (rs_batch_add with an empty range); a unit is admitted as a
device-side clone of its file's template with its own bitmap, so its result
does not depend on which other units share the device.  Admission is by free
batch slots and HBM footprint: the server maps a memory reserve for unit
buffers once, at start, and admits a unit only while the footprints of the
admitted units (bitmap plus a factor list with room for every candidate) fit
in it, so no admission waits for new device memory.  A unit that arrives while
others are running joins at the next round boundary, spread over a few free
range slots, runs alongside them (one BSGS launch per geometry group covers
every admitted unit), and leaves when its range is done -- its factors and
bitmap are collected and its slots and memory released for the next arrival.
Every round the units share a budget of work, earliest deadline first.
Latency is measured from arrival and from admission.
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


# Relative cost of one prime by the kind of step its p takes in the library:
# FP64 products below 2^51, Shoup products below 2^63, Montgomery products
# above.  Measured on a B200 with config-2-style units served one at a time:
# 4.0e11 model cost units/s below 2^51 against 2.8-3.0e11 for units between
# 2^52 and 2^61, i.e. a prime there costs 1.38 times as much.  Above 2^63 the
# steps and the set-up's chains are full Montgomery products; the factor there
# is the config-4 job's step rate against config 2's (253 against 427 G
# steps/s in the BSGS kernel), an estimate for whole units.
STEP_COST = ((1 << 51, 1.0), (1 << 63, 1.38), (1 << 64, 1.7))


def step_factor(p0):
    """Cost of a prime at p0 relative to one below 2^51 (STEP_COST)."""
    for bound, f in STEP_COST:
        if p0 < bound:
            return f
    return STEP_COST[-1][1]


def cost_per_prime(q, kcount, L):
    """Model cost of one prime in baby-step units for Q baby steps (the library's
    geometry model: Q baby steps plus the giant steps of the surviving targets,
    each over one class of n modulo the prime's split modulus, about 0.15 L/Q
    steps and at least one)."""
    m = max(1.0, 0.15 * L / q + 0.5)
    return 1.15 * q + 1.2 * 0.6 * kcount * m


class Server:
    """Continuous-batching sieve server over one device.

    Each round, units are put in priority order (earliest deadline first by
    default, or least remaining work first; work is primes left times the model
    cost of one prime for the unit's file and step kind) and given primes to cover from a
    round budget of ROUND_S seconds of the measured throughput, so that a short
    unit arriving while long ones run finishes within a round or two.  A unit
    spreads over at most MAX_SPLIT range slots, enough to take a whole round's
    budget, so that slots stay free for arrivals."""

    PRIMES_PER_SLOT_ROUND = 0.6 * 65536    # one range slot's round capacity
    ROUND_S = 0.004                        # target round duration
    MIN_ROUND_S = 0.0015                   # shortest round when a unit is about to finish
    SLOWDOWN = 2.0                         # deadline: arrival + SLOWDOWN x estimated time alone
    MAX_SPLIT = 4                          # range slots per unit: a few absorb a round's budget,
                                           # the rest stay free for new arrivals

    MAX_RESERVE = 64 << 30                 # largest memory reserve for unit buffers (bytes)

    def __init__(self, files, device=0, max_units=48, range_slots=128, round_s=None, short_rounds=False,
                 reserve_bytes=None, policy="edf"):
        nf = len(files)
        self.round_s = round_s or self.ROUND_S
        self.short_rounds = short_rounds
        if policy not in ("edf", "srpt"):
            raise ValueError("policy is 'edf' or 'srpt'")
        self.policy = policy
        self.batch = Batch(device, max_jobs=nf + max_units, range_slots=range_slots)
        self.templates, self.cost, self.footprint = [], {}, {}
        for seqs in files:
            t = self.batch.add(seqs, 3, 3)        # p0 == p1: resident template, never runs
            assert t is not None
            self.templates.append(t)
            self.cost[t] = cost_per_prime(self.batch.job_info(t)[0], seqs.kcount, seqs.nmax - seqs.nmin + 1)
            self.footprint[t] = self.batch.job_bytes(t)
        self.max_units = max_units
        # memory for max_units of the largest footprint, within MAX_RESERVE; halved until the device has it
        want = reserve_bytes or min(max_units * max(self.footprint.values()), self.MAX_RESERVE)
        while not self.batch.reserve(want):
            want //= 2
            if want < max(self.footprint.values()):
                raise MemoryError("no device memory for one unit's buffers")
        self.reserve = want
        self.in_use = 0                           # footprint of the admitted units
        self.rate = None                          # cost units per second, measured
        self.busy_s = 0.0                         # time spent in rounds, over all runs

    def close(self):
        self.batch.close()

    def _unit_cost(self, u):
        """Model cost of one prime of unit u: its file's cost at the unit's step kind."""
        return self.cost[self.templates[u.file]] * step_factor(u.p0)

    def _work(self, u, width):
        """Model cost of sieving `width` of unit u's p-range."""
        return width / math.log(max(u.p0, 3)) * self._unit_cost(u)

    def _budgets(self, active, remaining, given):
        """Primes per unit for the next round, in priority order, from a budget of
        ROUND_S seconds of measured throughput (calls the library only where a
        unit's budget changes).  'srpt': least remaining work first.  'edf':
        earliest deadline first, a unit's deadline being its arrival plus
        SLOWDOWN times its estimated time alone (its work at the measured rate,
        plus a round) -- short units come first, and a long unit that has waited
        overtakes them before its latency reaches SLOWDOWN times its own."""
        def left(slot):
            return self._work(active[slot], remaining[slot])
        if self.policy == "edf" and self.rate is not None:
            def deadline(slot):
                u = active[slot]
                alone = self._work(u, u.p1 - u.p0) / self.rate + self.round_s
                return u.arrival + self.SLOWDOWN * alone
            order = sorted(active, key=deadline)
        else:
            order = sorted(active, key=left)
        budget = None if self.rate is None else self.rate * self.round_s
        if budget is not None and self.short_rounds and order:
            # a unit that finishes this round shares it with at most as much other work
            # as its own, so the round ends within twice the time the unit needs alone
            first = left(order[0])
            if first < budget:
                budget = max(2.0 * first, self.rate * self.MIN_ROUND_S)
        for slot in order:
            if budget is None:                    # first round: full windows
                n = 1 << 40
            else:
                c = self._unit_cost(active[slot])
                give = min(left(slot), budget)
                budget -= give
                n = int(math.ceil(give / c)) if give > 0 else 0
            if given.get(slot) != n:
                self.batch.set_budget(slot, n)
                given[slot] = n

    def run(self, units, clock=time.perf_counter, collect_bitmaps=False, trace=None, sleep=time.sleep):
        """Serve the units (sorted by arrival time); returns them with timings filled.
        trace: an optional list that receives one record per round; clock and sleep
        are the time source and the idle wait (seconds)."""
        pending = sorted(units, key=lambda u: u.arrival)
        queue, active = [], {}
        remaining, given = {}, {}
        primes_seen = {}
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
                need = self.footprint[self.templates[u.file]]
                if self.in_use + need > self.reserve:
                    break
                free = self.batch.free_slots()[1]
                if free == 0:
                    break
                est = (u.p1 - u.p0) / math.log(max(u.p0, 3))
                nsplit = max(1, min(free, self.MAX_SPLIT, math.ceil(est / self.PRIMES_PER_SLOT_ROUND)))
                slot = self.batch.add_clone(self.templates[u.file], u.p0, u.p1, nsplit)
                if slot is None:
                    break
                u.admitted = clock() - t0
                self.in_use += need
                active[slot] = u
                remaining[slot] = u.p1 - u.p0
                primes_seen[slot] = 0
                given.pop(slot, None)
                queue.pop(0)
            if not active:
                if i < len(pending):                 # idle until the next arrival
                    wait = pending[i].arrival - (clock() - t0)
                    if wait > 0:
                        sleep(wait)
                continue
            self._budgets(active, remaining, given)
            r0 = clock()
            self.batch.run(1)                        # one round for every unit with a budget
            done, primes, rem = self.batch.poll()
            dt = clock() - r0
            self.busy_s += dt
            work = sum(float(primes[s] - primes_seen[s]) * self._unit_cost(active[s]) for s in active)
            if trace is not None:
                trace.append({"t": r0 - t0, "dt": dt, "rate": self.rate, "work": work, "queue": len(queue),
                              "free": self.batch.free_slots(),
                              "units": {active[s].uid: (given.get(s), int(primes[s] - primes_seen[s]), int(rem[s]))
                                        for s in active}})
            if dt > 0 and work > 0:
                r = work / dt
                self.rate = r if self.rate is None else 0.7 * self.rate + 0.3 * r
            for slot in list(active):
                remaining[slot] = int(rem[slot])
                primes_seen[slot] = int(primes[slot])
                if not done[slot]:
                    continue
                u = active.pop(slot)
                remaining.pop(slot)
                primes_seen.pop(slot)
                given.pop(slot, None)
                u.finished = clock() - t0
                u.primes = int(primes[slot])
                u.factors = self.batch.factors(slot)
                if collect_bitmaps:
                    u.bitmap = self.batch.bitmap(slot)
                self.batch.release(slot)
                self.in_use -= self.footprint[self.templates[u.file]]
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

