"""The serving loop's host logic on the CPU, against a stand-in for the batch.

The stand-in keeps the batch's bookkeeping (job and range slots, footprints, a
memory reserve, per-job round budgets, one poll per round) and advances each
admitted unit by its budget every round, capped by its range slots' capacity,
on a simulated clock.  What is checked: units are admitted only while their
footprints fit in the reserve, the reserve is halved until the device can map
it, every unit finishes and gives its memory back, and the round budget goes
to units in deadline order (or shortest remaining first).
"""
import math
from types import SimpleNamespace

import numpy as np
import pytest

from rssieve_b200 import serve

SLOT_PRIMES = 39321                 # one range slot's primes per round


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        self.t += 1e-6              # every reading moves time on a little
        return self.t

    def sleep(self, dt):
        self.t += dt


class FakeBatch:
    def __init__(self, clock, max_jobs, range_slots, reserve_limit, round_s=0.004):
        self.clock, self.max_jobs, self.nranges = clock, max_jobs, range_slots
        self.reserve_limit, self.round_s = reserve_limit, round_s
        self.jobs, self.ranges_used = {}, 0
        self.budget_calls, self.max_active = [], 0

    def _new_id(self):
        return next(j for j in range(self.max_jobs) if j not in self.jobs)

    def add(self, seqs, p0, p1, q=0):
        j = self._new_id()
        self.jobs[j] = {"tmpl": True, "bytes": seqs.footprint, "q": 8192}
        return j

    def job_info(self, j):
        return self.jobs[j]["q"], self.jobs[j].get("primes", 0), self.jobs[j].get("rem", 0) == 0

    def job_bytes(self, j):
        return self.jobs[j]["bytes"]

    def reserve(self, nbytes):
        return nbytes <= self.reserve_limit

    def free_slots(self):
        return self.max_jobs - len(self.jobs), self.nranges - self.ranges_used

    def add_clone(self, src, p0, p1, nsplit=1):
        if len(self.jobs) == self.max_jobs or self.nranges - self.ranges_used < nsplit:
            return None
        j = self._new_id()
        self.jobs[j] = {"tmpl": False, "bytes": self.jobs[src]["bytes"], "q": 8192, "p0": p0, "rem": p1 - p0,
                        "primes": 0, "ranges": nsplit, "budget": 1 << 40}
        self.ranges_used += nsplit
        self.max_active = max(self.max_active, sum(1 for v in self.jobs.values() if not v["tmpl"]))
        return j

    def set_budget(self, j, n):
        self.jobs[j]["budget"] = n
        self.budget_calls.append((j, n))

    def run(self, max_rounds=0):
        for v in self.jobs.values():
            if v["tmpl"] or v["rem"] == 0:
                continue
            lnp = math.log(v["p0"])
            n = min(v["budget"], v["ranges"] * SLOT_PRIMES, math.ceil(v["rem"] / lnp))
            v["primes"] += n
            v["rem"] = max(0, v["rem"] - int(n * lnp))
        self.clock.sleep(self.round_s)
        return all(v["tmpl"] or v["rem"] == 0 for v in self.jobs.values())

    def poll(self):
        done = np.zeros(self.max_jobs, dtype=np.uint8)
        primes = np.zeros(self.max_jobs, dtype=np.uint64)
        rem = np.zeros(self.max_jobs, dtype=np.uint64)
        for j, v in self.jobs.items():
            if not v["tmpl"]:
                done[j], primes[j], rem[j] = v["rem"] == 0, v["primes"], v["rem"]
        return done, primes, rem

    def factors(self, j):
        return np.zeros(0, dtype=np.uint64)

    def bitmap(self, j):
        return np.zeros(1, dtype=np.uint32)

    def release(self, j):
        assert not self.jobs[j]["tmpl"]
        self.ranges_used -= self.jobs.pop(j)["ranges"]

    def close(self):
        pass


def _server(monkeypatch, clock, reserve_limit=1 << 40, footprints=(100, 300), **kw):
    made = {}

    def factory(device, max_jobs, range_slots):
        made["b"] = FakeBatch(clock, max_jobs, range_slots, reserve_limit)
        return made["b"]
    monkeypatch.setattr(serve, "Batch", factory)
    files = [SimpleNamespace(kcount=10 * (i + 1), nmin=1000, nmax=200000, footprint=f) for i, f in enumerate(footprints)]
    srv = serve.Server(files, **kw)
    return srv, made["b"]


def _units(n, spacing, width=1 << 24, p0=1 << 44, files=2):
    return [serve.Unit(k, k % files, p0, p0 + width * (1 + k % 3), k * spacing) for k in range(n)]


def test_every_unit_finishes_and_returns_its_memory(monkeypatch):
    clock = Clock()
    srv, b = _server(monkeypatch, clock, max_units=8, range_slots=16)
    out = srv.run(_units(20, 0.003), clock=clock, sleep=clock.sleep)
    assert all(u.arrival <= u.admitted <= u.finished for u in out)
    assert all(u.primes > 0 for u in out)
    assert srv.in_use == 0 and b.ranges_used == 0
    assert sum(1 for v in b.jobs.values() if not v["tmpl"]) == 0
    st = serve.latency_stats(out)
    assert st["units"] == 20 and st["p50_s"] <= st["p99_s"]


def test_admission_stays_within_the_memory_reserve(monkeypatch):
    """Footprints 100 and 300 within a reserve of 450: never more than the
    reserve's worth of units at once, however many arrive together."""
    clock = Clock()
    srv, b = _server(monkeypatch, clock, max_units=8, range_slots=64, reserve_bytes=450)
    assert srv.reserve == 450
    seen = []
    orig = b.add_clone

    def watch(*a, **k):
        j = orig(*a, **k)
        if j is not None:
            seen.append(sum(v["bytes"] for v in b.jobs.values() if not v["tmpl"]))
        return j
    b.add_clone = watch
    srv.run(_units(12, 0.0), clock=clock, sleep=clock.sleep)
    assert seen and max(seen) <= 450
    assert srv.in_use == 0


def test_reserve_is_halved_until_the_device_can_map_it(monkeypatch):
    clock = Clock()
    srv, _ = _server(monkeypatch, clock, reserve_limit=1000, footprints=(100,), max_units=48)
    assert srv.reserve == 600               # 4800 -> 2400 -> 1200 -> 600
    with pytest.raises(MemoryError):
        _server(monkeypatch, clock, reserve_limit=50, footprints=(100,), max_units=4)


def _budget_order(srv, b, units):
    """Budgets of one scheduling pass over the given units, admitted."""
    active, remaining = {}, {}
    for u in units:
        j = b.add_clone(srv.templates[u.file], u.p0, u.p1, 1)
        active[j], remaining[j] = u, u.p1 - u.p0
    b.budget_calls.clear()
    srv._budgets(active, remaining, {})
    return {active[j].uid: n for j, n in b.budget_calls}


def test_deadline_order_lets_a_waiting_long_unit_overtake(monkeypatch):
    """A long unit that arrived long ago has the earlier deadline: EDF gives it
    the round budget first, shortest-remaining-first gives it to the short unit."""
    clock = Clock()
    long_u = serve.Unit(0, 0, 1 << 44, (1 << 44) + (1 << 28), 0.0)
    short_u = serve.Unit(1, 0, 1 << 44, (1 << 44) + (1 << 22), 5.0)
    for policy, first in (("edf", 0), ("srpt", 1)):
        srv, b = _server(monkeypatch, clock, footprints=(100,), policy=policy)
        cost = srv.cost[srv.templates[0]]
        srv.rate = cost * 1e7                # 10^7 primes/s of this file
        got = _budget_order(srv, b, [long_u, short_u])
        other = 1 - first
        assert got[first] > 0
        # the round budget (4 ms at 10^7 primes/s) is smaller than either unit's work
        assert got[first] == math.ceil(srv.rate * srv.round_s / cost)
        assert got[other] == 0


def test_deadlines_price_primes_by_step_kind(monkeypatch):
    """Two units of one file arrive together, one below 2^51 (FP64 steps) and one
    above (integer steps, 1.38 times the cost per prime).  The one below has more
    primes, so a model without the step kind estimated it longer alone and gave
    the round to the other; priced by step kind it is the shorter one and has
    the earlier deadline."""
    clock = Clock()
    lo = serve.Unit(0, 0, 1 << 45, (1 << 45) + (1 << 28), 0.0)
    hi = serve.Unit(1, 0, 1 << 54, (1 << 54) + (1 << 28), 0.1)
    assert serve.step_factor(lo.p0) == 1.0 and serve.step_factor(hi.p0) > 1.3
    srv, b = _server(monkeypatch, clock, footprints=(100,))
    cost = srv.cost[srv.templates[0]]
    srv.rate = cost * 1e7
    assert srv._work(lo, lo.p1 - lo.p0) < srv._work(hi, hi.p1 - hi.p0)
    # without the step kind the unit below 2^51 has the larger work
    assert (lo.p1 - lo.p0) / math.log(lo.p0) > (hi.p1 - hi.p0) / math.log(hi.p0)
    got = _budget_order(srv, b, [lo, hi])
    assert got[0] > 0 and got[1] == 0


def test_policy_must_be_known(monkeypatch):
    clock = Clock()
    with pytest.raises(ValueError):
        _server(monkeypatch, clock, policy="fifo")
