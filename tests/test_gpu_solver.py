"""GPU parity of the fused solver: effective field and dM/dt against the oracle's RHS (reference
tensor injected, <= 1e-12 in FP64), Runge-Kutta trajectories of <M> against the oracle's
restatement of the reference's solve loop (<= 1e-6 FP64, <= 1e-4 FP32 compensated), and the
step-controller semantics (same accepted/rejected counts in FP64)."""
import math

import numpy as np
import pytest
import torch

from helpers import rel_l2, unit_random

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * math.pi


@pytest.fixture(scope="module")
def sv():
    from micromagnum_b200 import solver
    return solver


def film(n=(32, 8, 1), delta=(3.90625e-9, 3.90625e-9, 3e-9)):
    return n, delta


def voronoi(dims, ngrains, rng):
    nx, ny, nz = dims
    pts = rng.random((ngrains, 3)) * np.array(dims)
    z, y, x = np.meshgrid(np.arange(nz) + 0.5, np.arange(ny) + 0.5, np.arange(nx) + 0.5, indexing="ij")
    c = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    d = ((c[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    return d.argmin(1).astype(np.uint8)


def make_pair(sv, oracle_mod, dims, delta, mats, regions, terms, prec, ref_tensor=True, **kw):
    """Our solver and the oracle solver on identical inputs (reference tensor injected)."""
    nx, ny, nz = dims
    n = nx * ny * nz
    reg = np.zeros(n, dtype=np.uint8) if regions is None else regions
    tensor = None
    if "demag" in terms:
        tensor = oracle_mod.demag_tensor(nx, ny, nz, *delta, impl="ref" if ref_tensor else "oracle")
    ours = sv.Solver(sv.RectangularMesh(dims, delta), mats, regions=regions, terms=terms, precision=prec,
                     tensor=None if tensor is None else tensor[0], **kw)

    def per_cell(attr):
        return np.array([getattr(mats[r], attr) for r in reg], dtype=np.float64)

    def per_cell_vec(attr):
        return np.array([getattr(mats[r], attr) for r in reg], dtype=np.float64).T.copy()

    okw = {k: v for k, v in kw.items() if k in ("evolver", "eps_abs", "eps_rel", "h0", "do_precess", "zl_do_precess",
                                                 "H_ext", "H_pulse", "pulse_rise", "fsal_reuse_after_reject")}
    orc = oracle_mod.Solver(dims, delta, per_cell("Ms"), A=per_cell("A"), alpha=per_cell("alpha"),
                            k_uniaxial=per_cell("k_uniaxial"), k_cubic=per_cell("k_cubic"),
                            axis1=per_cell_vec("axis1"), axis2=per_cell_vec("axis2"), P=per_cell("P"),
                            xi=per_cell("xi"), j=per_cell_vec("j"), terms=terms, tensor=tensor,
                            float_norm=False, **okw)
    return ours, orc


def test_eval_film_f64(sv, oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference not built")
    dims, delta = (64, 16, 1), (3.90625e-9, 3.90625e-9, 3e-9)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)]
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, None, ("demag", "exchange"), "f64",
                          H_ext=(1e4, -2e4, 3e3))
    rng = np.random.default_rng(1)
    M = unit_random(rng, int(np.prod(dims))) * 8e5
    ours.M = M
    orc.M = M
    H, dM, Hd = (t.cpu().numpy() for t in ours.eval())
    Hr, dMr, Hdr = orc.eval()
    assert rel_l2(Hd, Hdr) < 1e-12
    assert rel_l2(H, Hr) < 1e-12
    assert rel_l2(dM, dMr) < 1e-12


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_eval_granular_all_terms(sv, oracle_mod, ref_available, prec):
    # grains (uniaxial axes per region), cubic, Zhang-Li, empty cells, applied field
    if not ref_available:
        pytest.skip("reference not built")
    rng = np.random.default_rng(2)
    dims, delta = (24, 20, 4), (2e-9, 2e-9, 2e-9)
    n = int(np.prod(dims))
    mats = [sv.Material()]  # region 0: empty (Ms = 0)
    for g in range(8):
        a1 = unit_random(rng, 1)[:, 0]
        a2 = np.cross(a1, unit_random(rng, 1)[:, 0])
        a2 /= np.linalg.norm(a2)
        mats.append(sv.Material(Ms=1e6, A=1.5e-11, alpha=0.1, k_uniaxial=2e5, k_cubic=-3e4, axis1=tuple(a1),
                                axis2=tuple(a2), P=0.5, xi=0.05, j=(1e12, 0.0, 0.0)))
    reg = voronoi(dims, 8, rng) + 1
    reg[rng.random(n) < 0.05] = 0
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, reg,
                          ("demag", "exchange", "uniaxial", "cubic", "zhangli"), prec, H_ext=(5e3, 0, 1e4))
    M = unit_random(rng, n) * 1e6
    ours.M = M
    orc.M = M
    H, dM, Hd = (t.cpu().numpy() for t in ours.eval())
    Hr, dMr, Hdr = orc.eval()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel_l2(Hd, Hdr) < tol
    assert rel_l2(H, Hr) < tol
    assert rel_l2(dM, dMr) < tol


def granular_materials(sv, rng, ngrains):
    """Region 0 empty (Ms = 0); regions 1..ngrains: grains with their own uniaxial and cubic axes,
    Zhang-Li current along x."""
    mats = [sv.Material()]
    for _ in range(ngrains):
        a1 = unit_random(rng, 1)[:, 0]
        a2 = np.cross(a1, unit_random(rng, 1)[:, 0])
        a2 /= np.linalg.norm(a2)
        mats.append(sv.Material(Ms=1e6, A=1.5e-11, alpha=0.1, k_uniaxial=2e5, k_cubic=-3e4, axis1=tuple(a1),
                                axis2=tuple(a2), P=0.5, xi=0.05, j=(1e12, 0.0, 0.0)))
    return mats


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_staged_kernels_granular_vs_oracle(sv, oracle_mod, ref_available, prec):
    # the kernels the slab benchmark times: the staged stage kernel k_stage_tma with regions
    # (nx % 16 == 0) and the TMA-staged x passes whose forward pass scales by the region's Ms
    # (both x passes take tiles of 2 LPB rows of one plane: ny = 64 is a multiple of that).
    # 64x64x4 cells, 8 grains (uniaxial + cubic), Zhang-Li j = 1e12 A/m^2, 5% empty cells and an
    # applied field: H_eff and dM/dt, the first step's increment, then five more steps
    from micromagnum_b200 import _lib
    if not ref_available:
        pytest.skip("reference not built")
    rng = np.random.default_rng(12)
    dims, delta = (64, 64, 4), (2e-9, 2e-9, 2e-9)
    n = int(np.prod(dims))
    mats = granular_materials(sv, rng, 8)
    reg = voronoi(dims, 8, rng) + 1
    reg[rng.random(n) < 0.05] = 0
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, reg,
                          ("demag", "exchange", "uniaxial", "cubic", "zhangli"), prec, H_ext=(5e3, 0, 1e4),
                          evolver="dp54", eps_abs=1e-3, eps_rel=1e-4)
    M0 = unit_random(rng, n) * 1e6
    ours.M = M0
    orc.M = M0
    M0 = orc.M  # zero in the empty cells
    _lib.profile_reset()
    _lib.profile_enable(True)
    try:
        H, dM, Hd = (t.cpu().numpy() for t in ours.eval())
        ours.step()
        torch.cuda.synchronize()
        ran = set(_lib.profile_read())
    finally:
        _lib.profile_enable(False)
    assert {"k_stage_tma", "k_x_fwd_tma", "k_x_inv_tma"} <= ran, ran
    Hr, dMr, Hdr = orc.eval()
    orc.step()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel_l2(Hd, Hdr) < tol
    assert rel_l2(H, Hr) < tol
    assert rel_l2(dM, dMr) < tol
    # one accepted dp54 step: all seven stages through k_stage_tma; the increment M1 - M0 carries
    # the stage kernel's arithmetic, the step size the controller's
    a, b = ours.stats, orc.stats
    assert a["steps"] == b["steps"] == 1 and a["rejected"] == b["rejected"]
    assert a["t"] == pytest.approx(b["t"], rel=1e-12)
    assert a["h_next"] == pytest.approx(b["h_next"], rel=1e-9 if prec == "f64" else 1e-4)
    assert rel_l2(ours.M.cpu().numpy() - M0, orc.M - M0) < tol
    for _ in range(5):
        ours.step()
        orc.step()
    a, b = ours.stats, orc.stats
    assert a["steps"] == b["steps"] and a["rejected"] == b["rejected"]
    assert a["t"] == pytest.approx(b["t"], rel=1e-10 if prec == "f64" else 1e-4)
    if prec == "f64":
        # rounding differences of the single evaluations (~1e-16) accumulate through the step-size
        # feedback over the steps, as in the other multi-step comparisons
        assert rel_l2(ours.M.cpu().numpy(), orc.M) < 1e-10


@pytest.mark.parametrize("prec,tol", [("f64", 1e-6), ("f32", 1e-4)])
def test_trajectory_film(sv, oracle_mod, ref_available, prec, tol):
    # the thin-film relax/switching problem (3.90625 nm x 3.90625 nm x 3 nm cells, reduced to
    # 32x8 cells so the oracle is quick): dp54, eps 1e-6, <M>/Ms sampled every 1 ps for 0.1 ns
    if not ref_available:
        pytest.skip("reference not built")
    dims, delta = (32, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)]
    kw = dict(evolver="dp54", eps_abs=1e-6, eps_rel=1e-6, H_ext=(2e4, 1e4, 0.0))
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, None, ("demag", "exchange"), prec, **kw)
    rng = np.random.default_rng(3)
    M = unit_random(rng, int(np.prod(dims))) * 8e5
    ours.M = M
    orc.M = M
    t1, m1 = ours.solve(1e-10, sample_dt=1e-12)
    t2, m2 = orc.solve(1e-10, sample_dt=1e-12)
    if prec == "f32":
        # an adaptive step that ends within 1e-16 s short of a sample time is sampled (the
        # reference's tolerance, condition.py:121-133) and followed by a tiny step onto that time,
        # which is sampled again; the FP32 step sequence may meet this where the FP64 one does not,
        # so compare the last sample taken at each sample time
        def last_per_time(t, m):
            keep = np.append(np.abs(np.diff(t)) > 1e-15, True)
            return t[keep], m[keep]
        t1, m1 = last_per_time(t1, m1)
        t2, m2 = last_per_time(t2, m2)
    assert len(t1) == len(t2) == 101
    assert np.allclose(t1, t2, rtol=1e-12, atol=0)
    err = np.abs(m1 - m2).max() / 8e5
    assert err < tol, err
    if prec == "f64":
        s1, s2 = ours.stats, orc.stats
        assert s1["steps"] == s2["steps"] and s1["rejected"] == s2["rejected"]


def test_step_semantics_rejection_and_clamp(sv, oracle_mod, ref_available):
    # a large first step forces rejections; stepping to an explicit t_max exercises the clamp
    # re-apply (runge_kutta.py:75-78) and the reuse of the last stage after a rejection
    if not ref_available:
        pytest.skip("reference not built")
    dims, delta = (16, 8, 1), (4e-9, 4e-9, 3e-9)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.02)]
    kw = dict(evolver="dp54", eps_abs=1e-5, eps_rel=1e-5, h0=1e-12)
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, None, ("demag", "exchange"), "f64", **kw)
    rng = np.random.default_rng(4)
    M = unit_random(rng, int(np.prod(dims))) * 8e5
    ours.M = M
    orc.M = M
    for t_max in (1e-12, 1.5e-12, 7e-12, 1e100, 1e100, 2.2e-11):  # h0 = 1e-12
        ours.step(t_max)
        orc.step(t_max)
        a, b = ours.stats, orc.stats
        assert a["t"] == pytest.approx(b["t"], rel=1e-9)
        assert a["steps"] == b["steps"] and a["rejected"] == b["rejected"]
        assert rel_l2(ours.M.cpu().numpy(), orc.M) < 1e-9
    assert orc.stats["rejected"] > 0


@pytest.mark.parametrize("evolver", ["rkf45", "cc45", "rk23"])
def test_other_tableaus(sv, oracle_mod, ref_available, evolver):
    if not ref_available:
        pytest.skip("reference not built")
    dims, delta = (16, 8, 2), (3e-9, 3e-9, 3e-9)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.3)]
    kw = dict(evolver=evolver, eps_abs=1e-5, eps_rel=1e-5)
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, None, ("demag", "exchange"), "f64", **kw)
    rng = np.random.default_rng(5)
    M = unit_random(rng, int(np.prod(dims))) * 8e5
    ours.M = M
    orc.M = M
    for _ in range(20):
        ours.step()
        orc.step()
    assert ours.stats["t"] == pytest.approx(orc.stats["t"], rel=1e-9)
    assert rel_l2(ours.M.cpu().numpy(), orc.M) < 1e-10


def test_launch_counter_and_native_library(sv):
    from micromagnum_b200 import _lib
    before = _lib.launches()
    s = sv.Solver(sv.RectangularMesh((16, 16, 1), (3e-9, 3e-9, 3e-9)), [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)])
    s.M = (8e5, 0, 0)
    s.step()
    assert _lib.launches() > before


def test_relaxed_condition_matches_oracle(sv, oracle_mod, ref_available):
    # condition.Relaxed(max_degree_per_ns, check_every_nth_step) on the film from a random state:
    # the same check steps, the same decision and the same final <M> as the oracle's restatement
    if not ref_available:
        pytest.skip("reference not built")
    dims, delta = (32, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)]
    kw = dict(evolver="dp54", eps_abs=1e-4, eps_rel=1e-4)
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, None, ("demag", "exchange"), "f64", **kw)
    M = unit_random(np.random.default_rng(5), int(np.prod(dims))) * 8e5
    ours.M = M
    orc.M = M
    # the norms behind deg/ns at the initial state agree with the oracle's
    dmdt, mmax, tq = ours.relax_norms()
    rd, rm, rt = orc.relax_norms()
    assert dmdt == pytest.approx(rd, rel=1e-12) and mmax == pytest.approx(rm, rel=1e-12)
    assert tq == pytest.approx(rt, rel=1e-12)
    ok1 = ours.relax(max_degree_per_ns=2000.0, check_every_nth_step=20, max_steps=3000)
    ok2, deg2 = orc.relax(max_degree_per_ns=2000.0, check_every_nth_step=20, max_steps=3000)
    assert ok1 == ok2
    assert ours.stats["steps"] == orc.stats["steps"]
    assert ours.last_relax_value == pytest.approx(deg2, rel=1e-6)
    assert np.abs(np.array(ours.average_M()) - orc.M.mean(1)).max() / 8e5 < 1e-6


def test_torque_relaxation_criterion(sv, oracle_mod):
    # relax_torque stops at the first checked step with max |m x H| / Ms below the threshold;
    # the oracle's norms at the returned state confirm the value
    dims, delta = (24, 12, 2), (4e-9, 4e-9, 4e-9)
    n = int(np.prod(dims))
    mats = [sv.Material(Ms=1e6, A=1.5e-11, alpha=0.5)]
    s = sv.Solver(sv.RectangularMesh(dims, delta), mats, terms=("demag", "exchange"), precision="f64",
                  evolver="dp54", eps_abs=1e-4, eps_rel=1e-4)
    s.M = unit_random(np.random.default_rng(8), n) * 1e6
    assert s.relax_torque(max_torque=0.05, check_every_nth_step=5, max_steps=20000)
    assert s.last_relax_value < 0.05
    assert s.stats["steps"] % 5 == 0
    orc = oracle_mod.Solver(dims, delta, np.full(n, 1e6), A=np.full(n, 1.5e-11), alpha=np.full(n, 0.5),
                            terms=("demag", "exchange"), tensor=oracle_mod.demag_tensor(*dims, *delta),
                            float_norm=False)
    orc.M = s.M.cpu().numpy()
    assert orc.relax_norms()[2] == pytest.approx(s.last_relax_value, rel=1e-9)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_energies_vs_oracle(sv, oracle_mod, ref_available, prec):
    # E_stray, E_exch, E_aniso (uniaxial + cubic), E_ext and E_tot of a granular box with empty
    # cells against the oracle's fields and energy-returning term functions
    if not ref_available:
        pytest.skip("reference not built")
    rng = np.random.default_rng(21)
    dims, delta = (24, 20, 4), (2e-9, 2e-9, 3e-9)
    n = int(np.prod(dims))
    mats = granular_materials(sv, rng, 6)
    reg = voronoi(dims, 6, rng) + 1
    reg[rng.random(n) < 0.05] = 0
    Hx = (5e3, -2e3, 1e4)
    ours, orc = make_pair(sv, oracle_mod, dims, delta, mats, reg,
                          ("demag", "exchange", "uniaxial", "cubic", "zhangli"), prec, H_ext=Hx)
    M = unit_random(rng, n) * 1e6
    ours.M = M
    orc.M = M
    M = orc.M  # zero in the empty cells
    e = ours.energies()
    _, _, Hd = orc.eval()
    V = float(np.prod(delta))
    Ms = np.array([mats[r].Ms for r in reg])
    A = np.array([mats[r].A for r in reg])
    ku = np.array([mats[r].k_uniaxial for r in reg])
    kc = np.array([mats[r].k_cubic for r in reg])
    a1 = np.array([mats[r].axis1 for r in reg]).T.copy()
    a2 = np.array([mats[r].axis2 for r in reg]).T.copy()
    ref = {"E_stray": -MU0 / 2 * V * float((M * Hd).sum()),
           "E_exch": oracle_mod.exchange(*dims, *delta, Ms, A, M)[1],
           "E_aniso": V * (oracle_mod.uniaxial_anisotropy(a1, ku, Ms, M)[1]
                           + oracle_mod.cubic_anisotropy(a1, a2, kc, Ms, M)[1]),
           "E_ext": -MU0 * V * float((M * np.array(Hx).reshape(3, 1)).sum())}
    ref["E_tot"] = sum(ref.values())
    tol = 1e-12 if prec == "f64" else 1e-5
    for k, v in ref.items():
        assert e[k] == pytest.approx(v, rel=tol), (k, e[k], v)
