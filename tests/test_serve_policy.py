"""The served request loop's policy on the host, without a GPU: the loop of
highmap_b200.forms.serve driven by a simulated device side and clock.
Requests route by size (large ones to the plain lane, one at a time), small
ones are admitted in arrival order while the batch and the large lane fit
the memory budget, ticks stop at the next completion, every request
completes once, and the throughput counts each request's work."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from highmap_b200 import forms as F  # noqa: E402


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-6)


class FakeLanes:
    """Batch rounds cost 1 ms each; a large solve takes 1 ns per
    cell-update; a job holds 4 bytes per cell."""

    def __init__(self, clock, budget):
        self.clock = clock
        self.budget = budget
        self.jobs = {}        # id -> [request, rounds done, bytes]
        self.next_id = 0
        self.in_use = 0
        self.added = []       # request ids in admission order
        self.large = []       # request ids started on the large lane
        self.large_running = 0
        self.big_bytes_now = 0
        self.violations = 0
        self.max_round_step = 0

    # large lane
    def start_large(self, r):
        self.large.append(r["id"])
        self.large_running += 1
        assert self.large_running == 1, "two large solves at once"
        self.big_bytes_now = self.large_bytes(r)
        return (self.clock.t + r["nx"] * r["ny"] * r["iterations"] * 1e-9, r)

    def large_done(self, handle):
        done = self.clock.t >= handle[0]
        if done:
            self.large_running -= 1
            self.big_bytes_now = 0
        return done

    def large_bytes(self, r):
        return r["nx"] * r["ny"] * 8

    # batch
    def make_job(self, r):
        return (r, r["nx"] * r["ny"] * 4)

    def job_bytes(self, job):
        return job[1]

    def add(self, job):
        r, nbytes = job
        jid = self.next_id
        self.next_id += 1
        self.jobs[jid] = [r, 0, nbytes]
        self.in_use += nbytes
        self.added.append(r["id"])
        if len(self.jobs) > 1 and self.in_use + self.big_bytes_now > self.budget:
            self.violations += 1
        return jid

    def bytes_in_use(self):
        return self.in_use

    def step(self, rounds):
        self.max_round_step = max(self.max_round_step, rounds)
        for j in self.jobs.values():
            j[1] = min(j[0]["iterations"], j[1] + rounds)
        self.clock.t += 1e-3 * rounds

    def status(self, jid):
        r, done, _ = self.jobs[jid]
        return done, done >= r["iterations"]

    def release(self, jid):
        self.in_use -= self.jobs.pop(jid)[2]


def _requests(n=60, rate=50.0, seed=3):
    return F.serve_requests(n, rate, seed, lo=64, hi=1536, it_lo=5, it_hi=300)


@pytest.mark.parametrize("budget", [1 << 40, 12 << 20, 1 << 20])
def test_serve_policy(budget):
    reqs = _requests()
    clock = Clock()
    lanes = FakeLanes(clock, budget)
    large_cells = 512 * 512
    lat, cells, total = F.serve(reqs, None, budget_bytes=budget, rounds_per_tick=16, large_cells=large_cells,
                                lanes=lanes, clock=clock, sleep=clock.sleep)
    # every request completes once, with a non-negative latency
    assert sorted(lat) == [r["id"] for r in reqs]
    assert all(v >= 0 for v in lat.values())
    # routing by size
    big = [r["id"] for r in reqs if r["nx"] * r["ny"] >= large_cells]
    small = [r["id"] for r in reqs if r["nx"] * r["ny"] < large_cells]
    assert big and small
    assert lanes.large == big
    # small requests admitted in arrival order, each once
    assert lanes.added == small
    # the budget holds whenever the batch holds more than one job
    assert lanes.violations == 0
    # a tick is at most rounds_per_tick rounds
    assert 1 <= lanes.max_round_step <= 16
    # work accounting and a drained batch
    assert cells == sum(r["nx"] * r["ny"] * r["iterations"] for r in reqs)
    assert lanes.in_use == 0 and not lanes.jobs
    assert total >= max(r["arrival"] for r in reqs)


def test_tight_budget_serialises_the_batch():
    """With a budget below any two jobs, the batch never holds two at once
    (the first job of an empty batch is always admitted)."""
    reqs = [r for r in _requests() if r["nx"] * r["ny"] < 512 * 512]
    clock = Clock()

    class Single(FakeLanes):
        peak = 0

        def add(self, job):
            jid = super().add(job)
            Single.peak = max(Single.peak, len(self.jobs))
            return jid

    lanes = Single(clock, 1)
    lat, _, _ = F.serve(reqs, None, budget_bytes=1, rounds_per_tick=8, lanes=lanes, clock=clock, sleep=clock.sleep)
    assert len(lat) == len(reqs)
    assert Single.peak == 1
