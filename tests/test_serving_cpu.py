"""Host logic of the continuous-batching loop, on the CPU: a fake engine with
a memory budget and a fixed number of advance calls per case stands in for
the GPU engine (admission runs on a second thread, as with the real one)."""
import threading

import numpy as np

from theseus_b200.serving import Case, SyntheticStream, serve


class FakeEngine:
    def __init__(self, budget, calls_per_case=3):
        self.budget, self.used = budget, 0
        self.calls = calls_per_case
        self.running = {}
        self.next = 1
        self.admitted = []
        self.max_concurrent = 0
        self.lock = threading.Lock()

    def admit(self, case):
        need = case.tag["bytes"]
        with self.lock:
            if self.used + need > self.budget:
                return None
            cid = self.next
            self.next += 1
            self.used += need
            self.running[cid] = [self.calls, case]
            self.admitted.append(case.tag["i"])
            self.max_concurrent = max(self.max_concurrent, len(self.running))
            return cid

    def advance(self):
        with self.lock:
            for v in self.running.values():
                v[0] -= 1

    def poll(self):
        with self.lock:
            return [cid for cid, v in self.running.items() if v[0] <= 0]

    def fetch(self, cid, shape):
        with self.lock:
            _, case = self.running.pop(cid)
            self.used -= case.tag["bytes"]
        return np.full(shape, float(case.tag["i"]))


def make_requests(n, bytes_each, spacing):
    return [Case(mesh=None, u0=np.zeros(3), nsteps=1, dt=1.0, arrival=i * spacing,
                 tag={"i": i, "bytes": bytes_each[i]}) for i in range(n)]


def test_serve_admits_in_order_within_budget():
    reqs = make_requests(12, [3, 1, 2, 2, 1, 3, 1, 1, 2, 2, 1, 1], 0.0)
    eng = FakeEngine(budget=4)
    results, lat, makespan = serve(eng, reqs, idle_sleep=0.0)
    assert eng.admitted == list(range(12))            # first come, first served
    assert eng.max_concurrent >= 2 and eng.used == 0
    for i, r in enumerate(results):
        assert np.all(r == i)
    assert np.all(lat >= 0) and makespan >= lat.max()


def test_serve_waits_for_arrivals():
    reqs = make_requests(4, [1, 1, 1, 1], 0.01)
    eng = FakeEngine(budget=100, calls_per_case=1)
    results, lat, makespan = serve(eng, reqs, idle_sleep=0.0)
    assert makespan >= 0.03
    assert all(r is not None for r in results)


def test_synthetic_stream_is_seeded_and_in_range():
    a = SyntheticStream(64, seed=5)
    b = SyntheticStream(64, seed=5)
    assert a.params == b.params
    arr = np.array([p["arrival"] for p in a.params])
    assert np.all(np.diff(arr) > 0)
    assert all(8 <= p["side"] <= 64 and 2 <= p["order"] <= 5 and 0.1 <= p["mach"] <= 2.0
               for p in a.params)
    assert 0.2 < np.mean([p["inviscid"] for p in a.params]) < 0.8
