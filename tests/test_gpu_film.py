"""The thin-film problems at their stated sizes against the oracle's trajectories.

tests/golden/film_trajectories.npz holds the oracle's runs (tests/golden/make_trajectories.py):
128x32x1 cells of 3.90625 x 3.90625 x 3 nm, Ms = 8e5 A/m, A = 1.3e-11 J/m, demag + exchange, dp54
at eps_abs = eps_rel = 1e-6, the reference's own demag tensor in both solvers.

  relax    alpha = 0.5 from a seeded random state for 2 ns, <M> every 10 ps: FP64 within 1e-6 of
           the oracle at every sample, H_eff at the oracle's final state within 1e-12
  dynamics alpha = 0.02 from the oracle's relaxed state under a seeded in-plane field for 1 ns,
           <M> every 1 ps (1001 samples): FP64 within 1e-6, FP32 compensated within 1e-4
"""
import os
import sys

import numpy as np
import pytest

from helpers import rel_l2

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_trajectories as film  # noqa: E402  (inputs: sizes, seeds, field)


@pytest.fixture(scope="module")
def traj():
    d = np.load(os.path.join(HERE, "golden", "film_trajectories.npz"))
    return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def ref_tensor(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference not built")
    return oracle_mod.demag_tensor(*film.DIMS, *film.DELTA, impl="ref")


def solver(alpha, prec, tensor, H_ext=(0.0, 0.0, 0.0)):
    from micromagnum_b200 import solver as sv
    return sv.Solver(sv.RectangularMesh(film.DIMS, film.DELTA), [sv.Material(Ms=film.MS, A=film.A, alpha=alpha)],
                     terms=("demag", "exchange"), precision=prec, evolver="dp54", eps_abs=film.TOL,
                     eps_rel=film.TOL, h0=1e-13, H_ext=H_ext, tensor=tensor[0])


def last_per_time(t, m):
    """An adaptive step that ends within 1e-16 s of a sample time is sampled there (the reference's
    tolerance, condition.py:121-133) and followed by a tiny step onto that time, which is sampled
    again; keep the last sample taken at each sample time."""
    keep = np.append(np.abs(np.diff(t)) > 1e-15, True)
    return t[keep], m[keep]


def test_relax_f64(traj, ref_tensor):
    s = solver(0.5, "f64", ref_tensor)
    s.M = film.initial_m() * film.MS
    t, m = s.solve(film.RELAX_T, sample_dt=film.RELAX_DT)
    t, m = last_per_time(t, m / film.MS)
    tr, mr = last_per_time(traj["relax_t"], traj["relax_m"])
    assert len(t) == len(tr) == 201
    assert np.allclose(t, tr, rtol=1e-12, atol=0)
    err = np.abs(m - mr).max()
    assert err < 1e-6, err
    # the final state and the effective field there
    M = s.M.cpu().numpy()
    assert np.abs(M.mean(1) - traj["relax_M"].mean(1)).max() / film.MS < 1e-6
    s.M = traj["relax_M"]
    H = s.eval()[0].cpu().numpy()
    assert rel_l2(H, traj["relax_H"]) < 1e-12


@pytest.mark.parametrize("prec,tol", [("f64", 1e-6), ("f32", 1e-4)])
def test_dynamics(traj, ref_tensor, prec, tol):
    s = solver(0.02, prec, ref_tensor, H_ext=tuple(traj["dyn_H_ext"]))
    s.M = traj["relax_M"]
    t, m = s.solve(film.DYN_T, sample_dt=film.DYN_DT)
    t, m = last_per_time(t, m / film.MS)
    tr, mr = last_per_time(traj["dyn_t"], traj["dyn_m"])
    assert len(t) == len(tr) == 1001
    assert np.allclose(t, tr, rtol=1e-12, atol=0)
    err = np.abs(m - mr).max()
    print(f"{prec}: max |<m> - <m>_oracle| over 1001 samples = {err:.3e}")
    assert err < tol, err
