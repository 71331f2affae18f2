"""GPU tests of the staged fused stage kernel (bulk-copy pipeline over column tiles marching
through z): its Runge-Kutta steps follow the per-thread-load stage kernel on the same inputs, with
one step per CTA, several column tiles per CTA and ranges that start mid-column."""
import numpy as np
import pytest
import torch

from helpers import unit_random

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sv():
    from micromagnum_b200 import solver
    return solver


def grains(sv, rng, count):
    mats = [sv.Material()]  # region 0: empty (Ms = 0)
    for _ in range(count):
        a1 = unit_random(rng, 1)[:, 0]
        a2 = np.cross(a1, unit_random(rng, 1)[:, 0])
        a2 /= np.linalg.norm(a2)
        mats.append(sv.Material(Ms=1e6, A=1.5e-11, alpha=0.1, k_uniaxial=2e5, k_cubic=-3e4, axis1=tuple(a1),
                                axis2=tuple(a2), P=0.5, xi=0.05, j=(1e12, 3e11, 0.0)))
    return mats


def run(sv, monkeypatch, dims, prec, regions, mats, terms, M, staged, grid_cap, steps=3, H_ext=(5e3, 0, 1e4)):
    monkeypatch.setenv("MMB200_STAGE_TMA", "1" if staged else "0")
    if grid_cap:
        monkeypatch.setenv("MMB200_STAGE_GRID", str(grid_cap))
    else:
        monkeypatch.delenv("MMB200_STAGE_GRID", raising=False)
    s = sv.Solver(sv.RectangularMesh(dims, (2e-9, 2e-9, 2e-9)), mats, regions=regions, terms=terms, precision=prec,
                  evolver="dp54", eps_abs=1e-4, eps_rel=1e-4, H_ext=H_ext)
    s.M = M
    for _ in range(steps):
        s.step()
    out = s.M.clone(), dict(s.stats)
    s.close()
    return out


CASES = [
    # dims, regions, grid cap (None: the resident grid)
    ((64, 16, 1), False, None),
    ((64, 16, 8), False, 3),
    ((128, 24, 5), True, 7),
    ((96, 40, 3), True, 1),
    ((112, 36, 6), True, None),
]


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dims,with_regions,cap", CASES)
def test_staged_stage_follows_plain_stage(sv, monkeypatch, prec, dims, with_regions, cap):
    rng = np.random.default_rng(hash(dims) % 2**32)
    n = int(np.prod(dims))
    if with_regions:
        mats = grains(sv, rng, 6)
        reg = rng.integers(1, len(mats), size=n).astype(np.uint8)
        reg[rng.random(n) < 0.05] = 0
        terms = ("demag", "exchange", "uniaxial", "cubic", "zhangli")
    else:
        mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)]
        reg = None
        terms = ("demag", "exchange")
    M = unit_random(rng, n) * 1e6
    m1, st1 = run(sv, monkeypatch, dims, prec, reg, mats, terms, M, True, cap)
    m0, st0 = run(sv, monkeypatch, dims, prec, reg, mats, terms, M, False, None)
    assert st1["steps"] == st0["steps"] and st1["rejected"] == st0["rejected"]
    assert st1["t"] == pytest.approx(st0["t"], rel=1e-12 if prec == "f64" else 1e-6)
    scale = float(m0.abs().max())
    tol = 1e-12 if prec == "f64" else 1e-6
    assert float((m1 - m0).abs().max()) / scale < tol


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("granular", [False, True])
def test_stage_patterns_follow_the_runtime_stage(sv, monkeypatch, prec, granular):
    # the staged kernels compiled for the Dormand-Prince stage patterns (the granular slab's and
    # the film's term sets) against the same kernels reading the stage structure at run time
    rng = np.random.default_rng(41 + granular)
    dims = (128, 24, 5) if granular else (64, 16, 8)
    n = int(np.prod(dims))
    if granular:
        mats = grains(sv, rng, 6)
        reg = rng.integers(1, len(mats), size=n).astype(np.uint8)
        reg[rng.random(n) < 0.05] = 0
        terms = ("demag", "exchange", "uniaxial", "zhangli")
    else:
        mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.5)]
        reg = None
        terms = ("demag", "exchange")
    M = unit_random(rng, n) * 1e6
    monkeypatch.setenv("MMB200_STAGE_PATTERN", "1")
    m1, st1 = run(sv, monkeypatch, dims, prec, reg, mats, terms, M, True, 5, steps=4, H_ext=(0, 0, 0))
    monkeypatch.setenv("MMB200_STAGE_PATTERN", "0")
    m0, st0 = run(sv, monkeypatch, dims, prec, reg, mats, terms, M, True, 5, steps=4, H_ext=(0, 0, 0))
    assert st1["stage_kernel"] == 3 and st0["stage_kernel"] == 2
    assert st1["steps"] == st0["steps"] and st1["rejected"] == st0["rejected"]
    scale = float(m0.abs().max())
    assert float((m1 - m0).abs().max()) / scale < (1e-14 if prec == "f64" else 1e-7)
