"""The serve request loop's host logic on CPU, with a host-only stand-in for the device pool: every
request completes and frees its slot, admission waits for the HBM budget (a refused admission is
retried, never an error), a device error flag stops the loop with EXACA_ERR_CUDA, and with a
deadline a request that cannot finish in time is given up (retired while the others run on) and
reported, with its slot freed. The problems are real (host initialisation); only the stepping is
simulated: a slot ends once it has run 250 cycles per 8 z planes."""
import time

import numpy as np
import pytest

import exaca_b200 as ex
from exaca_b200 import serve


class FakeStatus:
    def __init__(self, done, cycle, error=0):
        self.done, self.cycle, self.error = done, cycle, error


class FakePool:
    """Stands in for exaca_b200.Pool in serve.serve (same calls, no device)."""

    instances = []

    def __init__(self, device, budget_bytes, list_capacity, error_after=None):
        self.budget = budget_bytes
        self.used = 0
        self.next_slot = 0
        self.slots = {}  # slot -> [bytes, cycles needed, cycles run]
        self.retired = []
        self.max_resident = 0
        self.max_used = 0
        self.refused = 0
        self.steps = 0
        self.error_after = error_after
        self.closed = False
        FakePool.instances.append(self)

    def admit(self, prob, device_check=True):
        need = prob.slot_bytes()
        if self.used + need > self.budget:
            self.refused += 1
            raise ex.ExacaError(-4, "admission refused: HBM budget exceeded")
        slot = self.next_slot
        self.next_slot += 1
        self.slots[slot] = [need, 250 * ((prob.geometry.nz + 7) // 8), 0]
        self.used += need
        self.max_resident = max(self.max_resident, len(self.slots))
        self.max_used = max(self.max_used, self.used)
        return slot

    def bytes_in_use(self):
        return self.used

    def step(self, n):
        self.steps += 1
        for s in self.slots.values():
            s[2] = min(s[1], s[2] + n)

    def status_many(self, slots):
        err = 8 if self.error_after is not None and self.steps > self.error_after else 0
        return [FakeStatus(self.slots[s][2] >= self.slots[s][1], self.slots[s][2], err) for s in slots]

    def copy_out_concurrent(self, slot):
        return np.full(4, slot, np.int32), np.zeros(4, np.int32)

    def retire(self, slot):
        self.used -= self.slots.pop(slot)[0]
        self.retired.append(slot)

    def close(self):
        self.closed = True


def stream(n, side=(8, 24), rate=2000.0):
    return serve.request_stream(n, rate=rate, seed=7, side=side)


def run(reqs, **kw):
    FakePool.instances.clear()
    out = serve.serve(reqs, pool_factory=FakePool, init_threads=2, keep_results=True, **kw)
    return out, FakePool.instances[-1]


def test_every_request_completes_and_frees_its_slot(lib):
    reqs = stream(10)
    out, pool = run(reqs)
    assert out["timed_out"] == []
    assert all(x is not None and x >= 0 for x in out["latency"])
    assert sorted(pool.retired) == list(range(10)) and pool.used == 0 and pool.closed
    for k, (g, c, cycle) in enumerate(out["results"]):
        assert cycle > 0 and g.dtype == np.int32
    assert out["p50"] <= out["p99"]


def test_admission_waits_for_the_budget(lib):
    reqs = stream(6)
    probs = serve.build_problems([p for _, p in reqs], threads=2)
    budget = max(p.slot_bytes() for p in probs)  # room for the largest request alone
    out, pool = run(reqs, budget_bytes=budget)
    assert out["timed_out"] == [] and all(x is not None for x in out["latency"])
    # never above the budget; smaller requests may share it, so the loop admits fewer than all six at
    # once and waits for retirements
    assert pool.max_used <= budget and pool.max_resident < len(reqs) and pool.used == 0


def test_device_error_stops_the_loop(lib):
    reqs = stream(4)

    def factory(device, budget_bytes, list_capacity):
        return FakePool(device, budget_bytes, list_capacity, error_after=0)

    FakePool.instances.clear()
    with pytest.raises(ex.ExacaError) as e:
        serve.serve(reqs, pool_factory=factory, init_threads=2)
    assert e.value.code == -3 and "device error flags 8" in str(e.value)
    assert FakePool.instances[-1].closed


def test_deadline_zero_gives_every_request_up(lib):
    reqs = stream(8)
    out, pool = run(reqs, deadline_s=0.0)
    assert out["timed_out"] == list(range(8))
    assert all(x is None for x in out["latency"]) and all(r is None for r in out["results"])
    assert pool.used == 0 and pool.closed


def test_running_requests_past_their_deadline_are_retired(lib):
    # domains that never end: each request is admitted within milliseconds of its arrival, then
    # retired as late once 0.2 s have passed, while the others keep running
    class NeverEnding(FakePool):
        def admit(self, prob, device_check=True):
            slot = super().admit(prob, device_check)
            self.slots[slot][1] = 1 << 60
            return slot

        def step(self, n):
            super().step(n)
            time.sleep(0.002)

    reqs = stream(6)
    FakePool.instances.clear()
    out = serve.serve(reqs, pool_factory=NeverEnding, init_threads=2, deadline_s=0.2)
    pool = FakePool.instances[-1]
    assert out["timed_out"] == list(range(6))
    assert sorted(pool.retired) == list(range(6)) and pool.used == 0
    assert out["elapsed"] >= 0.2


def test_a_generous_deadline_changes_nothing(lib):
    reqs = stream(8)
    out, pool = run(reqs, deadline_s=1e9)
    assert out["timed_out"] == [] and all(x is not None for x in out["latency"])
    assert sorted(pool.retired) == list(range(8)) and pool.used == 0
