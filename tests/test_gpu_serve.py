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


def test_omf_wire_format(mods):
    # requests whose M0 is an OMF file (text for some, binary 8 for others) and results returned as
    # OMF binary-8 files give the same solves as the array path, bit for bit
    from micromagnum_b200 import omf
    batch, serve = mods
    rng = np.random.default_rng(23)
    reqs = requests(batch, serve, rng, 4, rate=500.0)
    import torch
    wire = []
    for r in reqs:
        fmt = omf.TEXT if r.id % 2 else omf.BINARY_8
        data = omf.format(torch.as_tensor(r.M0).cuda(), r.instance.dims, r.instance.delta, fmt)
        # with MAGNUM_OMF_NOSCALE unset the writer divides by max |M|; the round trip is exact for
        # binary 8 only up to the multiplier's 16 digits, so both paths start from the parsed field
        r.M0 = omf.parse(data)[1].cpu().numpy()
        wire.append(serve.Request(r.id, r.instance, data, r.arrival))
    kw = dict(memory_budget=8 << 30, max_torque=5e-2, check_every_nth_step=5, rounds_per_tick=4)
    srv = serve.Server(keep_results=True, **kw)
    plain = {c.id: c for c in srv.run(reqs).completed}
    srv.close()
    srv = serve.Server(keep_results="omf", **kw)
    got = {c.id: c for c in srv.run(wire).completed}
    srv.close()
    assert set(got) == set(plain) == {r.id for r in reqs}
    for r in reqs:
        h, M = omf.parse(got[r.id].M)
        assert (h.xnodes, h.ynodes, h.znodes) == tuple(r.instance.dims) and h.title == f"request {r.id}".encode()
        assert got[r.id].steps == plain[r.id].steps
        assert np.abs(M.cpu().numpy() - plain[r.id].M).max() <= 1e-15 * r.instance.Ms
