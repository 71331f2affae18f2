"""Pins the oracle (CPU restatement) against the reference: its golden OMF fixtures, its
known-answer tests, and its own CPU C++ compiled in place (oracle/_ref/libmmref.so)."""
import math

import numpy as np
import pytest

from helpers import rel_l2, unit_random, vortex

MU0 = 4e-7 * math.pi


# ---- golden fixtures (src/magnum_tests/{exchange,stray_field,anisotropy}_test.py) -------------
def _m1(golden):
    (nx, ny, nz), (dx, dy, dz) = golden["dims"], golden["delta"]
    return int(nx), int(ny), int(nz), float(dx), float(dy), float(dz), golden["M1"]


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_exchange_golden(golden, oracle_mod, ref_available, impl):
    if impl == "ref" and not ref_available:
        pytest.skip("reference not built")
    nx, ny, nz, dx, dy, dz, M = _m1(golden)
    n = nx * ny * nz
    H, _ = oracle_mod.exchange(nx, ny, nz, dx, dy, dz, np.full(n, 8e5), np.full(n, 13e-12), M, impl=impl)
    assert np.abs(H - golden["H1_exch"]).max() < 2.0  # exchange_test.py:52 (eps 2 A/m)


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_uniaxial_golden(golden, oracle_mod, ref_available, impl):
    if impl == "ref" and not ref_available:
        pytest.skip("reference not built")
    nx, ny, nz, dx, dy, dz, M = _m1(golden)
    n = nx * ny * nz
    axis = np.full((3, n), 1 / math.sqrt(3))
    H, _ = oracle_mod.uniaxial_anisotropy(axis, np.full(n, 520e3), np.full(n, 8e5), M, impl=impl)
    assert np.abs(H - golden["H1_unianiso"]).max() < 10.0  # anisotropy_test.py:46 (eps 10 A/m)


@pytest.mark.parametrize("tensor_impl", ["oracle", "ref"])
def test_stray_golden(golden, oracle_mod, ref_available, tensor_impl):
    if tensor_impl == "ref" and not ref_available:
        pytest.skip("reference not built")
    nx, ny, nz, dx, dy, dz, M = _m1(golden)
    N, pd = oracle_mod.demag_tensor(nx, ny, nz, dx, dy, dz, padding=2, impl=tensor_impl)
    assert pd == (400, 100, 1)
    H = oracle_mod.conv(N, (nx, ny, nz), pd, M, method="fft")
    assert np.abs(H - golden["H1_stray"]).max() < 1.0  # stray_field_test.py:48 (eps 1 A/m)


# ---- known-answer tests ------------------------------------------------------------------------
def test_llge_kat(oracle_mod):
    # llge_test.py:26-38
    n = 1000
    dM = oracle_mod.llge(np.full(n, 10.0), np.full(n, 20.0), np.repeat([[5.0], [10.0], [15.0]], n, 1),
                         np.repeat([[20.0], [25.0], [30.0]], n, 1))
    assert np.all(dM.T == np.array([-60750.0, -13500.0, 29250.0]))


def test_scaled_abs_max_kat(oracle_mod):
    # scaled_abs_max_test.py:27-46
    n = 1000
    M = np.repeat([[-8e5], [0.0], [0.0]], n, 1)
    Ms = np.full(n, 8e5)
    assert oracle_mod.scaled_abs_max(M, Ms) == 1.0
    Ms2 = Ms.copy()
    Ms2[0] = 0.0
    assert oracle_mod.scaled_abs_max(M, Ms2) == 1.0


@pytest.mark.parametrize("impl", ["oracle", "ref"])
def test_anisotropy_energy_kats(oracle_mod, ref_available, impl):
    # anisotropy_test.py:52-119: parallel -> E = 0, orthogonal -> E = k V with H = 0
    if impl == "ref" and not ref_available:
        pytest.skip("reference not built")
    n = 40 * 40 * 40
    k, Ms = np.full(n, 520e3), np.full(n, 8e5)

    def uni(axis, m):
        H, e = oracle_mod.uniaxial_anisotropy(np.repeat(np.reshape(axis, (3, 1)), n, 1), k, Ms,
                                              np.repeat(np.reshape(m, (3, 1)), n, 1), impl=impl)
        return H.mean(axis=1), e * 1e-27

    for ax, m in [((1, 0, 0), (8e5, 0, 0)), ((0, 1, 0), (0, -8e5, 0)), ((0, 0, -1), (0, 0, -1))]:
        _, E = uni(ax, m)
        assert E == pytest.approx(0.0, abs=1e-7)
    E_ref = 520e3 * 40e-9 ** 3
    for ax, m in [((0, 0, 1), (8e5, 0, 0)), ((1, 0, 0), (0, -8e5, 0)), ((0, -1, 0), (0, 0, 1))]:
        H, E = uni(ax, m)
        assert E == pytest.approx(E_ref, rel=1e-12)
        assert np.allclose(H, 0.0, atol=1e-7)

    def cub(a1, a2, m):
        H, e = oracle_mod.cubic_anisotropy(np.repeat(np.reshape(a1, (3, 1)), n, 1),
                                           np.repeat(np.reshape(a2, (3, 1)), n, 1), k, Ms,
                                           np.repeat(np.reshape(m, (3, 1)), n, 1), impl=impl)
        return H.mean(axis=1), e * 1e-27

    for a1, a2, m in [((1, 0, 0), (0, 1, 0), (8e5, 0, 0)), ((1, 0, 0), (0, -1, 0), (0, -8e5, 0)),
                      ((0, -1, 0), (0, 0, -1), (0, 0, 8e5))]:
        H, E = cub(a1, a2, m)
        assert E == pytest.approx(0.0, abs=1e-7)
        assert np.allclose(H, 0.0, atol=1e-7)


@pytest.mark.parametrize("impl", ["oracle", "ref"])
@pytest.mark.parametrize("dims", [(100, 100, 1), (100, 100, 20)])
def test_zhangli_vortex_kat(oracle_mod, ref_available, impl, dims):
    # spintorque_test.py:61-94: vortex at (150 nm, 150 nm), 3 nm cells, P = 1, xi = 0.02,
    # j = (1e9, -1e9, 0), alpha = 0.01 -> <dM> = (3.40104691300733e11, 3.37831145947553e11, 7.4e-6)
    if impl == "ref" and not ref_available:
        pytest.skip("reference not built")
    nx, ny, nz = dims
    n = nx * ny * nz
    M = vortex(dims, (3e-9, 3e-9, 3e-9), (150e-9, 150e-9))
    dM = oracle_mod.fdm_zhangli(nx, ny, nz, 3e-9, 3e-9, 3e-9, True, np.full(n, 1.0), np.full(n, 0.02),
                                np.full(n, 8e5), np.full(n, 0.01), np.repeat([[1e9], [-1e9], [0.0]], n, 1),
                                M, impl=impl)
    ref = (340104691300.73352, 337831145947.55255, 7.4024200439453129e-06)
    assert np.all(np.abs(dM.mean(axis=1) - ref) < 1e6)


def test_zhangli_zero_gradient(oracle_mod):
    # spintorque_test.py:49-59: M = 0 everywhere -> zero torque
    nx, ny, nz = 20, 20, 4
    n = nx * ny * nz
    dM = oracle_mod.fdm_zhangli(nx, ny, nz, 3e-9, 3e-9, 3e-9, True, np.ones(n), np.full(n, 0.02),
                                np.full(n, 8e5), np.full(n, 0.01), np.repeat([[1e9], [-1e9], [0.0]], n, 1),
                                np.zeros((3, n)))
    assert np.abs(dM).max() == 0.0


@pytest.mark.parametrize("pbc", [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)])
@pytest.mark.parametrize("dims", [(16 - 5, 16 + 3, 1), (12, 10, 7)])
def test_exchange_uniform_is_zero(oracle_mod, pbc, dims):
    # exchange_test.py:55-77: uniform M gives exactly zero field for every PBC combination
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.default_rng(5)
    M = np.repeat((rng.random(3) - 0.5).reshape(3, 1) * 2e5, n, 1)
    H, _ = oracle_mod.exchange(nx, ny, nz, 1e-9, 1e-9, 1e-9, np.full(n, 8e5), np.full(n, 13e-12), M, pbc=pbc)
    assert np.all(H == 0.0)


# ---- restatement vs the compiled reference on seeded random inputs ----------------------------
@pytest.fixture
def need_ref(ref_available):
    if not ref_available:
        pytest.skip("reference not built")


@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 0, 0), (0, 1, 1), (1, 1, 1)])
def test_exchange_vs_ref(oracle_mod, need_ref, pbc):
    rng = np.random.default_rng(1)
    nx, ny, nz = 13, 9, 5
    n = nx * ny * nz
    Ms = rng.uniform(6e5, 1.4e6, n)
    Ms[rng.random(n) < 0.15] = 0.0
    A = rng.uniform(1e-11, 2e-11, n)
    M = unit_random(rng, n) * Ms
    a, ea = oracle_mod.exchange(nx, ny, nz, 2e-9, 3e-9, 4e-9, Ms, A, M, pbc=pbc)
    b, eb = oracle_mod.exchange(nx, ny, nz, 2e-9, 3e-9, 4e-9, Ms, A, M, pbc=pbc, impl="ref")
    assert rel_l2(a, b) < 1e-14
    assert ea == pytest.approx(eb, rel=1e-12)


def test_terms_vs_ref(oracle_mod, need_ref):
    rng = np.random.default_rng(2)
    nx, ny, nz = 17, 11, 6
    n = nx * ny * nz
    Ms = rng.uniform(6e5, 1.4e6, n)
    Ms[rng.random(n) < 0.1] = 0.0
    M = unit_random(rng, n) * Ms * rng.uniform(0.9, 1.1, n)
    ax1 = unit_random(rng, n)
    ax2 = np.cross(ax1.T, unit_random(rng, n).T).T
    ax2 /= np.linalg.norm(ax2, axis=0)
    k = rng.uniform(-1e5, 5e5, n)
    for fn, args in [(oracle_mod.uniaxial_anisotropy, (ax1, k, Ms, M)),
                     (oracle_mod.cubic_anisotropy, (ax1, ax2, k, Ms, M))]:
        a, ea = fn(*args)
        b, eb = fn(*args, impl="ref")
        assert rel_l2(a, b) < 1e-14
        assert ea == pytest.approx(eb, rel=1e-12)
    f1, f2 = rng.normal(size=n) * 1e5, rng.normal(size=n) * 1e-1
    H = rng.normal(size=(3, n)) * 1e5
    assert rel_l2(oracle_mod.llge(f1, f2, M, H), oracle_mod.llge(f1, f2, M, H, impl="ref")) < 1e-15
    P, xi, al = rng.uniform(0, 1, n), rng.uniform(0, 0.1, n), rng.uniform(0.01, 0.5, n)
    j = rng.normal(size=(3, n)) * 1e11
    for prec in (True, False):
        a = oracle_mod.fdm_zhangli(nx, ny, nz, 2e-9, 3e-9, 4e-9, prec, P, xi, Ms, al, j, M)
        b = oracle_mod.fdm_zhangli(nx, ny, nz, 2e-9, 3e-9, 4e-9, prec, P, xi, Ms, al, j, M, impl="ref")
        assert rel_l2(a, b) < 1e-14
    assert oracle_mod.scaled_abs_max(M, Ms) == pytest.approx(oracle_mod.scaled_abs_max(M, Ms, impl="ref"), rel=1e-15)
    assert np.array_equal(oracle_mod.normalize(Ms, M, float_norm=True), oracle_mod.normalize(Ms, M, impl="ref"))


@pytest.mark.parametrize("case", [((4, 4, 4), (1e-9,) * 3), ((8, 5, 3), (3.90625e-9, 3.90625e-9, 3e-9))])
def test_tensor_near_field_vs_ref(oracle_mod, need_ref, case):
    # tiny grids lie entirely inside the reference's Newell (long double) region: exact match
    (nx, ny, nz), d = case
    a, pa = oracle_mod.demag_tensor(nx, ny, nz, *d)
    b, pb = oracle_mod.demag_tensor(nx, ny, nz, *d, impl="ref")
    assert pa == pb
    assert np.abs(a - b).max() < 1e-15 * np.abs(b).max() * 10


@pytest.mark.parametrize("case", [((12, 7, 1), (2.5e-9, 2.5e-9, 3e-9)), ((6, 6, 9), (2e-9, 5e-9, 1e-9))])
def test_tensor_series_region_vs_ref(oracle_mod, need_ref, case):
    # beyond ~6 cells along an axis the reference uses its axial series (sumf_large_x,
    # tensor_integrals.h:343-368, selected at :387-399); those elements differ from the exact
    # tensor by up to ~1e-5 relative, everything else to rounding
    (nx, ny, nz), d = case
    a, pa = oracle_mod.demag_tensor(nx, ny, nz, *d)
    b, pb = oracle_mod.demag_tensor(nx, ny, nz, *d, impl="ref")
    assert pa == pb
    assert rel_l2(a, b) < 1e-8
    assert np.abs(a - b).max() < 1e-5 * np.abs(b).max()


def test_tensor_far_field_vs_ref(oracle_mod, need_ref):
    # larger grids: the reference switches to truncated asymptotic series; the exact tensor
    # differs by that truncation only (~1e-8 relative in the field)
    nx, ny, nz = 64, 32, 4
    d = (2e-9, 2e-9, 2e-9)
    a, pd = oracle_mod.demag_tensor(nx, ny, nz, *d)
    b, _ = oracle_mod.demag_tensor(nx, ny, nz, *d, impl="ref")
    assert rel_l2(a, b) < 1e-6
    rng = np.random.default_rng(3)
    M = unit_random(rng, nx * ny * nz) * 8e5
    Ha = oracle_mod.conv(a, (nx, ny, nz), pd, M, method="fft")
    Hb = oracle_mod.conv(b, (nx, ny, nz), pd, M, method="fft")
    assert rel_l2(Ha, Hb) < 1e-7


def test_tensor_properties(oracle_mod):
    # trace of the (positive) demag tensor is 1 at the origin and 0 elsewhere; self term of a
    # cube is 1/3
    N, (ex, ey, ez) = oracle_mod.demag_tensor(6, 5, 4, 2e-9, 2e-9, 2e-9)
    T = N.reshape(ez, ey, ex, 6)
    tr = T[..., 0] + T[..., 3] + T[..., 5]
    assert tr[0, 0, 0] == pytest.approx(-1.0, abs=1e-14)
    tr[0, 0, 0] = 0
    assert np.abs(tr).max() < 1e-15
    assert T[0, 0, 0, 0] == pytest.approx(-1 / 3, abs=1e-15)


@pytest.mark.parametrize("dims", [(9, 7, 1), (6, 5, 4), (1, 8, 3)])
def test_conv_methods_agree(oracle_mod, need_ref, dims):
    nx, ny, nz = dims
    N, pd = oracle_mod.demag_tensor(nx, ny, nz, 2e-9, 3e-9, 2.5e-9)
    rng = np.random.default_rng(4)
    M = unit_random(rng, nx * ny * nz) * 8e5
    Hd = oracle_mod.conv(N, dims, pd, M, method="direct")
    Hf = oracle_mod.conv(N, dims, pd, M, method="fft")
    Hr = oracle_mod.conv(N, dims, pd, M, impl="ref")
    assert rel_l2(Hd, Hr) < 1e-14
    assert rel_l2(Hf, Hd) < 1e-13


def test_film_trajectory_fixture_is_the_oracles(oracle_mod, need_ref):
    # tests/golden/film_trajectories.npz (tests/golden/make_trajectories.py) holds the oracle's
    # thin-film runs; re-run the first 20 ps of the relaxation and 5 ps of the dynamics and check
    # the committed samples against them
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    sys.path.insert(0, here)
    import make_trajectories as film
    d = np.load(os.path.join(here, "film_trajectories.npz"))
    s = film.oracle_solver(oracle_mod, 0.5)
    s.M = film.initial_m() * film.MS
    t, m = s.solve(2e-11, sample_dt=film.RELAX_DT)
    assert np.array_equal(t, d["relax_t"][:len(t)])
    assert np.abs(m / film.MS - d["relax_m"][:len(t)]).max() < 1e-13
    s = film.oracle_solver(oracle_mod, 0.02, H_ext=tuple(d["dyn_H_ext"]))
    assert np.allclose(d["dyn_H_ext"], film.applied_field(), rtol=1e-15, atol=0)
    s.M = d["relax_M"]
    t, m = s.solve(5e-12, sample_dt=film.DYN_DT)
    assert np.array_equal(t, d["dyn_t"][:len(t)])
    assert np.abs(m / film.MS - d["dyn_m"][:len(t)]).max() < 1e-13
    assert len(d["dyn_t"]) == 1001 and len(d["relax_t"]) == 201
    for key in ("relax_M", "dyn_M"):
        assert np.allclose(np.linalg.norm(d[key], axis=0), film.MS, rtol=1e-12)
