"""CPU tests of the serving loop's host logic (micromagnum_b200.serve.Server) with the batch
replaced by a fake that advances every live instance by one accepted step per round: admission
in arrival order within the device-memory budget, the budget never exceeded, requests leaving
when they finish, and the deadline (unfinished requests counted, the steps made on them
recorded).  The byte accounting is the library's own (mm_batch_instance_bytes, host-only)."""
import threading

import numpy as np
import pytest

from micromagnum_b200 import serve
from micromagnum_b200.batch import Instance


class FakeBatch:
    """Stands in for micromagnum_b200.batch.Batch: slots, rounds, results."""
    live_max = 0
    lock = threading.Lock()

    def __init__(self, instances=(), **kw):
        self.slots = {}
        self.next_slot = 0

    def add(self, q, M=None):
        slot = self.next_slot
        self.next_slot += 1
        self.slots[slot] = {"need": q.need, "steps": 0}
        with FakeBatch.lock:
            FakeBatch.live_max = max(FakeBatch.live_max, sum(1 for _ in self.slots))
        return slot

    def remove(self, slot):
        del self.slots[slot]

    def relax(self, max_rounds=1, check_interval=1):
        for s in self.slots.values():
            s["steps"] = min(s["need"], s["steps"] + max_rounds)
        return max_rounds

    def results(self):
        n = self.next_slot
        out = [{"status": -1, "steps": 0, "attempts": 0} for _ in range(n)]
        for slot, s in self.slots.items():
            done = s["steps"] >= s["need"]
            out[slot] = {"status": 1 if done else 0, "steps": s["steps"], "attempts": s["steps"]}
        return out

    def get_M(self, slot):
        raise AssertionError("keep_results is off in these tests")

    def close(self):
        pass


def make_requests(count, dims, need, spacing=0.0):
    out = []
    for i in range(count):
        q = Instance(dims=dims, delta=(4e-9, 4e-9, 4e-9), Ms=8e5, A=1.3e-11, alpha=0.5)
        q.need = need(i)
        out.append(serve.Request(i, q, np.zeros((3, q.n)), i * spacing))
    return out


@pytest.fixture(scope="module", autouse=True)
def library():
    import os
    from micromagnum_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()


@pytest.fixture
def fake(monkeypatch):
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    FakeBatch.live_max = 0
    return FakeBatch


def test_every_request_finishes_within_the_budget(fake):
    reqs = make_requests(8, (32, 32, 1), need=lambda i: 16 * (1 + i % 3))
    res, trans = reqs[0].instance.device_bytes()
    budget = 3 * res + trans  # room for three resident requests
    srv = serve.Server(memory_budget=budget, rounds_per_tick=4)
    st = srv.run(reqs)
    srv.close()
    assert len(st.completed) == len(reqs) and st.unfinished == 0
    assert st.peak_resident <= budget
    assert fake.live_max <= 3
    assert [c.id for c in st.completed] == list(range(len(reqs)))
    for c in st.completed:
        assert c.steps == reqs[c.id].instance.need and c.status == 1
        assert c.arrival <= c.admitted <= c.finished
        assert st.progress[c.id] == c.steps


def test_admission_follows_arrival_order(fake):
    reqs = make_requests(6, (32, 32, 1), need=lambda i: 8)
    res, trans = reqs[0].instance.device_bytes()
    srv = serve.Server(memory_budget=res + trans, rounds_per_tick=2)  # one request at a time
    st = srv.run(reqs)
    srv.close()
    assert fake.live_max == 1
    done = sorted(st.completed, key=lambda c: c.admitted)
    assert [c.id for c in done] == list(range(len(reqs)))
    for a, b in zip(done, done[1:]):
        assert a.finished <= b.admitted + 1e-3


def test_deadline_counts_unfinished_requests_and_their_progress(fake):
    reqs = make_requests(4, (32, 32, 1), need=lambda i: 4 if i < 2 else 10 ** 9)
    srv = serve.Server(memory_budget=1 << 34, rounds_per_tick=1)
    st = srv.run(reqs, deadline=0.3)
    srv.close()
    assert {c.id for c in st.completed} == {0, 1}
    assert st.unfinished == 2
    assert set(st.progress) == {0, 1, 2, 3}
    assert st.progress[2] > 0 and st.progress[3] > 0


def test_request_over_the_budget_is_refused(fake):
    reqs = make_requests(1, (32, 32, 1), need=lambda i: 1)
    res, trans = reqs[0].instance.device_bytes()
    srv = serve.Server(memory_budget=res + trans - 1)
    with pytest.raises(MemoryError):
        srv.run(reqs)
    srv.close()


def test_budget_is_shared_by_all_size_classes(fake):
    # requests of three size classes (class bounds 2^17 and 2^20 cells): the device-memory budget
    # is one pool, so an idle class may not admit past it while the others hold most of it
    small = make_requests(6, (32, 32, 1), need=lambda i: 12)
    mid = make_requests(3, (512, 512, 1), need=lambda i: 8)
    big = make_requests(2, (1024, 1024, 2), need=lambda i: 6)
    reqs = []
    for i, r in enumerate(small + mid + big):
        r.id = i
        r.arrival = 0.0
        reqs.append(r)
    sizes = [sum(r.instance.device_bytes()) for r in reqs]
    budget = max(sizes) + sizes[0]  # the largest request and one small one at a time, at most
    srv = serve.Server(memory_budget=budget, rounds_per_tick=2)
    st = srv.run(reqs)
    srv.close()
    assert len(st.completed) == len(reqs) and st.unfinished == 0
    assert st.peak_resident <= budget


def test_max_live_bounds_each_class(fake):
    # plenty of memory, at most two requests of the class at once; the others wait in arrival order
    reqs = make_requests(7, (32, 32, 1), need=lambda i: 6 + 2 * (i % 3))
    srv = serve.Server(memory_budget=1 << 34, rounds_per_tick=2, max_live=(2, 4, 1))
    st = srv.run(reqs)
    srv.close()
    assert len(st.completed) == len(reqs) and fake.live_max <= 2
    adm = sorted(st.completed, key=lambda c: c.admitted)
    assert [c.id for c in adm] == list(range(len(reqs)))
    with pytest.raises(ValueError):
        serve.Server(memory_budget=1 << 34, max_live=(2, 4))
