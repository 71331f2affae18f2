"""GPU tests of the batched relaxations: every instance of a batch follows the single-instance
solver with the same geometry and controller (to rounding, in FP64, for every tile variant of the
grouped passes), an instance's result does not depend on the batch around it (bit for bit), and
the torque stop criterion holds at the returned states (checked by the FP64 oracle)."""
import numpy as np
import pytest
import torch

from helpers import unit_random

pytestmark = pytest.mark.gpu

POT = 4  # MM_PADDING_ROUND_POT


@pytest.fixture(scope="module")
def bt():
    from micromagnum_b200 import batch
    return batch


@pytest.fixture(scope="module")
def sv():
    from micromagnum_b200 import solver
    return solver


def ellipse(dims, rng):
    nx, ny, nz = dims
    a, b = nx / 2 * rng.uniform(0.5, 1.0), ny / 2 * rng.uniform(0.5, 1.0)
    y, x = np.meshgrid(np.arange(ny) + 0.5 - ny / 2, np.arange(nx) + 0.5 - nx / 2, indexing="ij")
    m2 = ((x / a) ** 2 + (y / b) ** 2 <= 1.0).astype(np.uint8)
    return np.tile(m2.reshape(-1), nz)


def make_instances(bt, rng, shapes):
    out = []
    for dims in shapes:
        out.append(bt.Instance(dims=dims, delta=(4e-9, 4e-9, 4e-9), Ms=float(rng.uniform(6e5, 1.4e6)),
                               A=float(rng.uniform(1e-11, 2e-11)), alpha=0.5, mask=ellipse(dims, rng)))
    return out


def initial(inst, rng):
    return unit_random(rng, inst.n) * inst.Ms


def single(sv, inst, eps, M, prec="f32"):
    mats = [sv.Material(Ms=0.0, A=0.0, alpha=inst.alpha), sv.Material(Ms=inst.Ms, A=inst.A, alpha=inst.alpha)]
    s = sv.Solver(sv.RectangularMesh(inst.dims, inst.delta), mats, regions=inst.mask, terms=("demag", "exchange"),
                  precision=prec, evolver="dp54", eps_abs=eps, eps_rel=eps, h0=1e-13, padding=POT)
    s.M = M
    return s


def smooth(inst):
    # a smooth, non-equilibrium state: rounding differences stay small along its relaxation (a
    # random state's relaxation amplifies them, which says nothing about the batch)
    nx, ny, nz = inst.dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    v = np.stack([np.ones(x.shape), 0.4 * np.sin(2 * np.pi * x / nx), 0.3 * np.cos(2 * np.pi * y / ny)])
    v = v.reshape(3, -1)
    return v / np.linalg.norm(v, axis=0) * inst.Ms


def run_pair(bt, sv, insts, prec, variant, monkeypatch):
    # the grouped passes with a fixed tile variant (MMB200_GROUP_VARIANT), 40 rounds, then each
    # instance alone through the single-instance solver for the same number of accepted steps
    monkeypatch.setenv("MMB200_GROUP_VARIANT", str(variant))
    M0 = [smooth(q) for q in insts]
    b = bt.Batch(insts, precision=prec, eps_abs=1e-4, eps_rel=1e-4, max_torque=0.0)
    for i, M in enumerate(M0):
        b.set_M(i, M)
    assert b.relax(max_rounds=40) == 40
    res = b.results()
    out = []
    for i, q in enumerate(insts):
        r = res[i]
        assert r["status"] == 0 and r["attempts"] == 40 and r["steps"] > 10
        s = single(sv, q, 1e-4, M0[i], prec)
        for _ in range(r["steps"]):
            s.step()
        out.append((r, s.stats, b.get_M(i), s.M))
        s.close()
    b.close()
    return out


def test_batch_instances_follow_the_single_solver(bt, sv, monkeypatch):
    rng = np.random.default_rng(11)
    shapes = [(48, 32, 2), (64, 40, 4), (32, 32, 2), (80, 24, 4)]
    insts = make_instances(bt, rng, shapes)
    # the grouped passes factor the transforms differently from the single-instance passes (tile
    # shapes, radix, and the fused y+z pass of small members): rounding-level differences, checked
    # in FP64 (in FP32 such differences move the adaptive step sizes, so FP32 runs agree at equal
    # times, not at equal step counts)
    for variant in (0, 1, 2, 3):
        for (r, st, got, ref), q in zip(run_pair(bt, sv, insts, "f64", variant, monkeypatch), insts):
            assert st["steps"] == r["steps"] and st["t"] == pytest.approx(r["t"], rel=1e-8)
            assert float((got - ref).abs().max()) / q.Ms < 1e-8


def test_result_is_the_same_alone_and_in_the_mix(bt):
    rng = np.random.default_rng(12)
    shapes = [(40, 36, 1), (64, 64, 2), (24, 56, 4), (100, 20, 1)]
    insts = make_instances(bt, rng, shapes)
    M0 = [initial(q, rng) for q in insts]
    mix = bt.Batch(insts, precision="f32", eps_abs=1e-4, eps_rel=1e-4, max_torque=1e-2, check_every_nth_step=5)
    for i, M in enumerate(M0):
        mix.set_M(i, M)
    mix.relax(max_rounds=20000)
    alone = bt.Batch([insts[2]], precision="f32", eps_abs=1e-4, eps_rel=1e-4, max_torque=1e-2, check_every_nth_step=5)
    alone.set_M(0, M0[2])
    alone.relax(max_rounds=20000)
    r_mix, r_alone = mix.results()[2], alone.results()[0]
    assert r_mix["status"] == r_alone["status"] == 1
    assert r_mix["steps"] == r_alone["steps"] and r_mix["attempts"] == r_alone["attempts"]
    assert torch.equal(mix.get_M(2), alone.get_M(0))


def test_relaxed_states_meet_the_torque_criterion(bt, oracle_mod):
    rng = np.random.default_rng(13)
    shapes = [(32, 24, 1), (40, 40, 2), (20, 36, 4)]
    insts = make_instances(bt, rng, shapes)
    thr = 2e-2
    b = bt.Batch(insts, precision="f32", eps_abs=1e-4, eps_rel=1e-4, max_torque=thr, check_every_nth_step=2)
    for i, q in enumerate(insts):
        b.set_M(i, initial(q, rng))
    b.relax(max_rounds=50000)
    for i, (q, r) in enumerate(zip(insts, b.results())):
        assert r["status"] == 1 and r["steps"] % 2 == 0, (i, r)
        n = q.n
        Ms = q.mask.astype(np.float64) * q.Ms
        orc = oracle_mod.Solver(q.dims, q.delta, Ms, A=np.full(n, q.A), alpha=np.full(n, q.alpha),
                                terms=("demag", "exchange"), tensor=oracle_mod.demag_tensor(*q.dims, *q.delta),
                                float_norm=False)
        orc.M = b.get_M(i).cpu().numpy()
        # FP32 state, FP64 check: the oracle's torque at the returned state is within a few
        # percent of the threshold the FP32 run stopped under
        assert orc.relax_norms()[2] < 1.05 * thr, (i, orc.relax_norms())


def test_fp32_batch_end_states_vs_fp64_oracle(bt, oracle_mod):
    # the batched form as served (FP32 deviation form, grouped passes) relaxes each instance to
    # max |m x H| / Ms < 1e-4; the FP64 oracle relaxes the same instance (same power-of-two padded
    # tensor, dp54 with the same controller, torque checked after every step) from the same state:
    # both take about the same number of steps (an FP32 form whose error estimate had a rounding
    # floor would stall its step size near equilibrium) and reach the same equilibrium, to within
    # what the stop criterion leaves (measured: max |dm| <= 3e-5, |d<m>| <= 8e-6)
    rng = np.random.default_rng(31)
    insts = make_instances(bt, rng, [(24, 20, 1), (20, 16, 2), (32, 12, 1)])
    b = bt.Batch(insts, precision="f32", eps_abs=1e-3, eps_rel=1e-4, max_torque=1e-4, check_every_nth_step=1)
    M0 = [smooth(q) for q in insts]
    for i, M in enumerate(M0):
        b.set_M(i, M)
    b.relax(max_rounds=200000)
    res = b.results()
    got = [b.get_M(i).cpu().numpy() for i in range(len(insts))]
    b.close()
    for q, M, r, Mb in zip(insts, M0, res, got):
        assert r["status"] == 1
        n = q.n
        Ms = q.Ms * q.mask.astype(np.float64)
        tensor = oracle_mod.demag_tensor(*q.dims, *q.delta, padding=POT)
        orc = oracle_mod.Solver(q.dims, q.delta, Ms, A=np.full(n, q.A), alpha=np.full(n, q.alpha),
                                terms=("demag", "exchange"), evolver="dp54", eps_abs=1e-3, eps_rel=1e-4,
                                tensor=tensor, float_norm=False)
        orc.M = M
        steps = 0
        while orc.relax_norms()[2] >= 1e-4 and steps < 200000:
            orc.step()
            steps += 1
        Mo = orc.M
        mask = q.mask.astype(bool)
        dm = np.abs(Mb[:, mask] - Mo[:, mask]).max() / q.Ms
        davg = np.abs(Mb[:, mask].mean(1) - Mo[:, mask].mean(1)).max() / q.Ms
        print(f"{q.dims}: batch {r['steps']} steps, oracle {steps}; max |dm| {dm:.2e}, |d<m>| {davg:.2e}")
        assert abs(r["steps"] - steps) <= 0.1 * steps
        assert davg < 5e-5 and dm < 2e-4


def test_fused_pass_tiles_do_not_change_results(bt):
    # five members of one fused y+z length (py = 512, pz = 4) fill the device with the default
    # tiles; alone, the member takes one kx column per CTA: the same arithmetic, bit for bit
    rng = np.random.default_rng(14)
    insts = make_instances(bt, rng, [(200, 210, 2), (190, 220, 2), (210, 200, 2), (230, 180, 2), (200, 200, 2)])
    M0 = [initial(q, rng) for q in insts]
    mix = bt.Batch(insts, precision="f32", eps_abs=1e-3, eps_rel=1e-4, max_torque=1e-9, check_every_nth_step=1)
    for i, M in enumerate(M0):
        mix.set_M(i, M)
    mix.relax(max_rounds=40, check_interval=40)
    alone = bt.Batch([insts[3]], precision="f32", eps_abs=1e-3, eps_rel=1e-4, max_torque=1e-9,
                     check_every_nth_step=1)
    alone.set_M(0, M0[3])
    alone.relax(max_rounds=40, check_interval=40)
    r_mix, r_alone = mix.results()[3], alone.results()[0]
    assert r_mix["attempts"] == r_alone["attempts"] == 40 and r_mix["steps"] == r_alone["steps"]
    assert torch.equal(mix.get_M(3), alone.get_M(0))
    mix.close()
    alone.close()
