"""CPU tests of the served-stream baseline's queue (bench.fifo_queue): one-at-a-time service in
arrival order within the server's makespan, with each solve given up when the window ends."""
from types import SimpleNamespace

import pytest

import bench


def reqs(arrivals):
    return [SimpleNamespace(id=i, arrival=a) for i, a in enumerate(arrivals)]


def test_requests_are_served_in_arrival_order_within_the_window():
    times = {0: 2.0, 1: 3.0, 2: 1.0, 3: 10.0}
    seen = []

    def solve(r, cap):
        seen.append((r.id, cap))
        t = times[r.id]
        return (t, 1, True) if t <= cap else (cap, 1, False)

    # arrivals out of order in the list: the queue sorts them
    rs = reqs([0.0, 0.5, 1.0, 1.5])
    rs = [rs[2], rs[0], rs[3], rs[1]]
    done, lat, spent = bench.fifo_queue(rs, makespan=8.0, solve=solve)
    # 0: 0 -> 2, 1: 2 -> 5, 2: 5 -> 6, 3: starts at 6 with 2 s left and is cut
    assert [i for i, _ in seen] == [0, 1, 2, 3]
    assert [c for _, c in seen] == pytest.approx([8.0, 6.0, 3.0, 2.0])
    assert done == 3
    assert lat == pytest.approx([2.0, 4.5, 5.0])
    assert spent == pytest.approx(2.0 + 3.0 + 1.0 + 2.0)


def test_idle_queue_waits_for_arrivals_and_stops_at_the_makespan():
    def solve(r, cap):
        return (1.0, 1, True)

    done, lat, spent = bench.fifo_queue(reqs([0.0, 5.0, 9.5, 20.0]), makespan=10.0, solve=solve)
    # 0: 0 -> 1; 1: waits to 5 -> 6; 2: 9.5 -> 10.5 is past the window; 3 arrives after it
    assert done == 2 and lat == pytest.approx([1.0, 1.0])
    assert spent == pytest.approx(1.0 + 1.0 + 0.5)


def test_a_long_request_blocks_the_queue():
    def solve(r, cap):
        return (cap, 1, False) if r.id == 1 else (0.1, 1, True)

    done, lat, _ = bench.fifo_queue(reqs([0.0, 0.0, 0.0, 0.0]), makespan=90.0, solve=solve)
    assert done == 1
