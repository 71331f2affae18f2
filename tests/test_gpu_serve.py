"""GPU tests of the serving loop: requests that arrive while others run are admitted as memory
frees up, their work shares the rounds with the running ones, and each result is the same alone
and in the mix (bit for bit: an instance's arithmetic does not depend on the batch around it)."""
import math

import numpy as np
import pytest

from helpers import unit_random

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * math.pi


@pytest.fixture(scope="module")
def mods():
    from micromagnum_b200 import batch, serve
    return batch, serve


def requests(batch, serve, rng, count, rate):
    out, t = [], 0.0
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        nx, ny = (int(v) for v in rng.integers(16, 72, size=2))
        nz = int(rng.choice([1, 2, 4]))
        switching = i % 2 == 1
        if switching:
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            B = rng.uniform(0.01, 0.1)
            kw = dict(H_pulse=tuple(d * B / MU0), pulse_rise=100e-12, t_end=40e-12)
        else:
            kw = {}
        q = batch.Instance(dims=(nx, ny, nz), delta=(4e-9, 4e-9, 4e-9), Ms=float(rng.uniform(6e5, 1.4e6)),
                           A=float(rng.uniform(1e-11, 2e-11)), alpha=0.5, **kw)
        out.append(serve.Request(i, q, unit_random(rng, q.n) * q.Ms, t))
    return out


def test_results_are_the_same_alone_and_in_the_mix(mods):
    batch, serve = mods
    rng = np.random.default_rng(21)
    reqs = requests(batch, serve, rng, 8, rate=200.0)
    srv = serve.Server(memory_budget=8 << 30, max_torque=5e-2, check_every_nth_step=5, rounds_per_tick=4,
                       keep_results=True)
    stats = srv.run(reqs)
    srv.close()
    assert len(stats.completed) == len(reqs)
    assert all(c.status == 1 for c in stats.completed)
    # several requests shared the device at once
    assert any(a.admitted < b.finished and b.admitted < a.finished
               for a in stats.completed for b in stats.completed if a.id != b.id)
    by_id = {c.id: c for c in stats.completed}
    for r in reqs:
        alone = batch.Batch([r.instance], max_torque=5e-2, check_every_nth_step=5)
        alone.set_M(0, r.M0)
        alone.relax(max_rounds=100000)
        res = alone.results()[0]
        M = alone.get_M(0).cpu().numpy()
        alone.close()
        c = by_id[r.id]
        assert res["status"] == 1 and res["steps"] == c.steps and res["attempts"] == c.attempts
        assert np.array_equal(M, c.M), r.id
        if r.instance.t_end > 0:
            assert res["t"] == pytest.approx(r.instance.t_end, rel=1e-12)


def test_admission_waits_for_memory(mods):
    batch, serve = mods
    rng = np.random.default_rng(22)
    reqs = requests(batch, serve, rng, 6, rate=1e6)  # all arrive at once
    need = [sum(r.instance.device_bytes()) for r in reqs]
    budget = max(need) + min(need)  # room for the largest and at most a small one beside it
    srv = serve.Server(memory_budget=budget, max_torque=5e-2, check_every_nth_step=5, rounds_per_tick=4)
    stats = srv.run(reqs)
    srv.close()
    assert len(stats.completed) == len(reqs)
    assert stats.peak_resident <= budget
