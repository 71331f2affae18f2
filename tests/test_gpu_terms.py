"""GPU parity of the per-term entry points (the drop-in magneto calls) against the oracle, the
reference's golden fixtures and its known-answer tests.

Tolerances: plain FP64 mode (CUDA_64) <= 1e-12 relative L2 against the FP64 oracle; FP32 mode
(CUDA_32) <= 1e-5 relative L2 (the single-precision form's stated error budget)."""
import math

import numpy as np
import pytest
import torch

from helpers import rel_l2, unit_random, vortex

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


@pytest.fixture(scope="module")
def mg():
    from micromagnum_b200 import magneto
    return magneto


def mode(mg, prec):
    mg.enableCuda(mg.CUDA_64 if prec == "f64" else mg.CUDA_32)


def field(mg, dims, data):
    f = mg.Matrix(dims)
    f.data.copy_(torch.as_tensor(np.asarray(data, dtype=np.float64).reshape(-1)))
    return f


def vfield(mg, dims, data):
    f = mg.VectorMatrix(dims)
    f.data.copy_(torch.as_tensor(np.asarray(data, dtype=np.float64).reshape(-1)))
    return f


def out(f):
    return f.data.view(3, -1).cpu().numpy()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_exchange_golden(mg, golden, prec):
    mode(mg, prec)
    (nx, ny, nz), (dx, dy, dz) = [int(v) for v in golden["dims"]], golden["delta"]
    dims = (nx, ny, nz)
    n = nx * ny * nz
    H = mg.VectorMatrix(dims)
    mg.exchange(nx, ny, nz, dx, dy, dz, False, False, False, field(mg, dims, np.full(n, 8e5)),
                field(mg, dims, np.full(n, 13e-12)), vfield(mg, dims, golden["M1"]), H)
    assert np.abs(out(H) - golden["H1_exch"]).max() < 2.0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_uniaxial_golden(mg, golden, prec):
    mode(mg, prec)
    dims = tuple(int(v) for v in golden["dims"])
    n = int(np.prod(dims))
    H = mg.VectorMatrix(dims)
    mg.uniaxial_anisotropy(vfield(mg, dims, np.full((3, n), 1 / math.sqrt(3))), field(mg, dims, np.full(n, 520e3)),
                           field(mg, dims, np.full(n, 8e5)), vfield(mg, dims, golden["M1"]), H)
    assert np.abs(out(H) - golden["H1_unianiso"]).max() < 10.0


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("pbc", [(0, 0, 0), (1, 0, 0), (0, 1, 1), (1, 1, 1)])
@pytest.mark.parametrize("dims", [(13, 9, 5), (70, 60, 59), (11, 19, 1), (1, 7, 3)])
def test_exchange_vs_oracle(mg, oracle_mod, prec, pbc, dims):
    mode(mg, prec)
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.default_rng(11)
    Ms = rng.uniform(6e5, 1.4e6, n)
    Ms[rng.random(n) < 0.1] = 0.0
    A = rng.uniform(1e-11, 2e-11, n)
    M = unit_random(rng, n) * Ms
    H = mg.VectorMatrix(dims)
    e = mg.exchange(nx, ny, nz, 2e-9, 3e-9, 4e-9, *pbc, field(mg, dims, Ms), field(mg, dims, A), vfield(mg, dims, M), H)
    Hr, _ = oracle_mod.exchange(nx, ny, nz, 2e-9, 3e-9, 4e-9, Ms, A, M, pbc=pbc)
    assert rel_l2(out(H), Hr) < TOL[prec]
    e_ref = -2e-7 * math.pi * 24e-27 * float((M * Hr).sum())
    assert e == pytest.approx(e_ref, rel=1e-9 if prec == "f64" else 1e-4)


@pytest.mark.parametrize("pbc", [(a, b, c) for a in (0, 1) for b in (0, 1) for c in (0, 1)])
@pytest.mark.parametrize("dims", [(64, 64, 64), (64 + 6, 64 - 4, 64 - 5), (16, 16, 1), (16 - 5, 16 + 3, 1)])
def test_exchange_uniform_zero(mg, pbc, dims):
    # exchange_test.py:55-77 (exact zero in FP64)
    mode(mg, "f64")
    n = int(np.prod(dims))
    rng = np.random.default_rng(3)
    M = np.repeat((rng.random(3) - 0.5).reshape(3, 1) * 2e5, n, 1)
    H = mg.VectorMatrix(dims)
    mg.exchange(*dims, 1e-9, 1e-9, 1e-9, *pbc, field(mg, dims, np.full(n, 8e5)), field(mg, dims, np.full(n, 13e-12)),
                vfield(mg, dims, M), H)
    assert float(H.data.abs().max()) == 0.0


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_local_terms_vs_oracle(mg, oracle_mod, prec):
    mode(mg, prec)
    dims = (33, 17, 6)
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.default_rng(12)
    Ms = rng.uniform(6e5, 1.4e6, n)
    Ms[rng.random(n) < 0.1] = 0.0
    M = unit_random(rng, n) * Ms * rng.uniform(0.95, 1.05, n)
    ax1 = unit_random(rng, n)
    ax2 = np.cross(ax1.T, unit_random(rng, n).T).T
    ax2 /= np.linalg.norm(ax2, axis=0)
    k = rng.uniform(-1e5, 5e5, n)
    H = mg.VectorMatrix(dims)
    e = mg.uniaxial_anisotropy(vfield(mg, dims, ax1), field(mg, dims, k), field(mg, dims, Ms), vfield(mg, dims, M), H)
    Hr, er = oracle_mod.uniaxial_anisotropy(ax1, k, Ms, M)
    assert rel_l2(out(H), Hr) < TOL[prec]
    assert e == pytest.approx(er, rel=1e-10 if prec == "f64" else 1e-4)
    e = mg.cubic_anisotropy(vfield(mg, dims, ax1), vfield(mg, dims, ax2), field(mg, dims, k), field(mg, dims, Ms),
                            vfield(mg, dims, M), H)
    Hr, er = oracle_mod.cubic_anisotropy(ax1, ax2, k, Ms, M)
    assert rel_l2(out(H), Hr) < TOL[prec]
    assert e == pytest.approx(er, rel=1e-10 if prec == "f64" else 1e-4)
    f1, f2 = rng.normal(size=n) * 1e5, rng.normal(size=n) * 1e-1
    Hx = rng.normal(size=(3, n)) * 1e5
    dM = mg.VectorMatrix(dims)
    mg.llge(field(mg, dims, f1), field(mg, dims, f2), vfield(mg, dims, M), vfield(mg, dims, Hx), dM)
    assert rel_l2(out(dM), oracle_mod.llge(f1, f2, M, Hx)) < TOL[prec]
    P, xi, al = rng.uniform(0, 1, n), rng.uniform(0, 0.1, n), rng.uniform(0.01, 0.5, n)
    j = rng.normal(size=(3, n)) * 1e12
    for dp in (True, False):
        mg.fdm_zhangli(nx, ny, nz, 2e-9, 3e-9, 4e-9, dp, field(mg, dims, P), field(mg, dims, xi), field(mg, dims, Ms),
                       field(mg, dims, al), vfield(mg, dims, j), vfield(mg, dims, M), dM)
        ref = oracle_mod.fdm_zhangli(nx, ny, nz, 2e-9, 3e-9, 4e-9, dp, P, xi, Ms, al, j, M)
        assert rel_l2(out(dM), ref) < TOL[prec]
    s = mg.scaled_abs_max(vfield(mg, dims, M), field(mg, dims, Ms))
    assert s == pytest.approx(oracle_mod.scaled_abs_max(M, Ms), rel=1e-15 if prec == "f64" else 1e-6)


def test_llge_kat(mg):
    # llge_test.py:26-38 (exact in FP64)
    mode(mg, "f64")
    dims = (10, 10, 10)
    f1, f2, M, H, dM = (mg.Matrix(dims), mg.Matrix(dims), mg.VectorMatrix(dims), mg.VectorMatrix(dims),
                        mg.VectorMatrix(dims))
    f1.fill(10)
    f2.fill(20)
    M.fill((5, 10, 15))
    H.fill((20, 25, 30))
    mg.llge(f1, f2, M, H, dM)
    assert np.all(out(dM).T == np.array([-60750.0, -13500.0, 29250.0]))


def test_scaled_abs_max_kat(mg):
    mode(mg, "f64")
    dims = (10, 10, 10)
    M = mg.VectorMatrix(dims)
    M.fill((-8e5, 0, 0))
    Ms = mg.Matrix(dims)
    Ms.fill(8e5)
    assert mg.scaled_abs_max(M, Ms) == 1.0
    Ms.set(0, 0)
    assert not Ms.isUniform()
    Ms.set(0, 8e5)
    Ms.set(1, 0.0)
    assert mg.scaled_abs_max(M, Ms) == 1.0


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dims", [(100, 100, 1), (100, 100, 20)])
def test_zhangli_vortex_kat(mg, prec, dims):
    # spintorque_test.py:61-94
    mode(mg, prec)
    nx, ny, nz = dims
    n = nx * ny * nz
    M = vortex(dims, (3e-9, 3e-9, 3e-9), (150e-9, 150e-9))
    dM = mg.VectorMatrix(dims)
    mg.fdm_zhangli(nx, ny, nz, 3e-9, 3e-9, 3e-9, True, field(mg, dims, np.ones(n)), field(mg, dims, np.full(n, 0.02)),
                   field(mg, dims, np.full(n, 8e5)), field(mg, dims, np.full(n, 0.01)),
                   vfield(mg, dims, np.repeat([[1e9], [-1e9], [0.0]], n, 1)), vfield(mg, dims, M), dM)
    ref = (340104691300.73352, 337831145947.55255, 7.4024200439453129e-06)
    assert np.all(np.abs(np.asarray(dM.average()) - ref) < 1e6)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_normalize_and_rk_helpers(mg, prec):
    mode(mg, prec)
    dims = (20, 10, 3)
    n = 600
    rng = np.random.default_rng(9)
    Ms = rng.uniform(5e5, 1e6, n)
    M = rng.normal(size=(3, n)) * 1e6
    v = vfield(mg, dims, M)
    v.normalize(field(mg, dims, Ms))
    ref = M / np.linalg.norm(M, axis=0) * Ms
    assert rel_l2(out(v), ref) < TOL[prec]
    # rk_prepare_step / rk_combine_result against numpy for the dp54 tableau
    b = [[], [1 / 5], [3 / 40, 9 / 40], [44 / 45, -56 / 15, 32 / 9]]
    tab = mg.ButcherTableau(6)
    for i, row in enumerate(b):
        for j, x in enumerate(row):
            tab.setB(i, j, x)
    c = [0.1, 0.0, 0.3, 0.2, 0.25, 0.15]
    ec = [0.01, 0.0, -0.02, 0.005, 0.0, 0.005]
    for i in range(6):
        tab.setC(i, c[i])
        tab.setEC(i, ec[i])
    ks = [rng.normal(size=(3, n)) for _ in range(6)]
    kf = [vfield(mg, dims, k) for k in ks]
    y0 = rng.normal(size=(3, n))
    h = 1e-3
    ytmp = mg.VectorMatrix(dims)
    mg.rk_prepare_step(3, h, tab, *kf, vfield(mg, dims, y0), ytmp)
    ref = y0 + h * sum(b[3][j] * ks[j] for j in range(3))
    assert rel_l2(out(ytmp), ref) < TOL[prec]
    y, yerr = vfield(mg, dims, y0), mg.VectorMatrix(dims)
    mg.rk_combine_result(h, tab, *kf, y, yerr)
    assert rel_l2(out(y), y0 + h * sum(c[j] * ks[j] for j in range(6))) < TOL[prec]
    assert rel_l2(out(yerr), h * sum(ec[j] * ks[j] for j in range(6))) < (1e-12 if prec == "f64" else 1e-5)
