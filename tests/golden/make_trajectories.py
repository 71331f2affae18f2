"""Oracle trajectories of the thin-film problems, written to tests/golden/film_trajectories.npz.

The film: 128x32x1 cells of 3.90625 x 3.90625 x 3 nm, Ms = 8e5 A/m, A = 1.3e-11 J/m, no
anisotropy, gamma = 2.211e5 m/As, demag (the reference's own tensor, calculateDemagTensor in
oracle/_ref/libmmref.so) + exchange, Dormand-Prince (dp54) with the reference's
MicroMagneticsStepSizeController at eps_abs = eps_rel = 1e-6, h0 = 1e-13.

  relax    alpha = 0.5 from per-cell unit vectors uniform on the sphere (seed RELAX_SEED), 2 ns,
           <M> sampled every 10 ps (EveryNthSecond clamping); the final M and its H_eff
  dynamics alpha = 0.02 from the final M of `relax`, a static in-plane field of angle U[0, 2 pi)
           and |B| U[10, 40] mT (seed DYN_SEED), 1 ns, <M> sampled every 1 ps (1001 samples)

The oracle is the C restatement of the reference's solve loop (oracle.Solver, FP64, full-precision
normalisation like the reference's CUDA normalize).  Run in the build container, where the
reference's CPU sources are compiled into oracle/_ref/libmmref.so:

    python tests/golden/make_trajectories.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

DIMS = (128, 32, 1)
DELTA = (3.90625e-9, 3.90625e-9, 3e-9)
MS, A = 8e5, 1.3e-11
MU0 = 4e-7 * np.pi
RELAX_SEED, DYN_SEED = 1000, 1001
RELAX_T, RELAX_DT = 2e-9, 1e-11
DYN_T, DYN_DT = 1e-9, 1e-12
TOL = 1e-6
OUT = os.path.join(HERE, "film_trajectories.npz")


def initial_m(seed=RELAX_SEED):
    """Per-cell unit vectors uniform on the sphere (normalised Gaussian triples)."""
    n = int(np.prod(DIMS))
    v = np.random.default_rng(seed).normal(size=(3, n))
    return v / np.linalg.norm(v, axis=0)


def applied_field(seed=DYN_SEED):
    """In-plane H = B / mu0 with angle U[0, 2 pi) and |B| U[10, 40] mT."""
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi)
    b = rng.uniform(0.010, 0.040)
    return (b / MU0 * np.cos(phi), b / MU0 * np.sin(phi), 0.0)


def oracle_solver(oracle, alpha, H_ext=(0.0, 0.0, 0.0)):
    tensor = oracle.demag_tensor(*DIMS, *DELTA, impl="ref")
    return oracle.Solver(DIMS, DELTA, MS, A=A, alpha=alpha, terms=("demag", "exchange"), evolver="dp54",
                         eps_abs=TOL, eps_rel=TOL, h0=1e-13, H_ext=H_ext, tensor=tensor, float_norm=False,
                         use_fft=True)


def main():
    import oracle
    if not oracle.have_reference():
        sys.exit("make_trajectories.py needs oracle/_ref/libmmref.so (the reference's tensor)")
    out = {}
    t0 = time.time()
    s = oracle_solver(oracle, 0.5)
    s.M = initial_m() * MS
    ts, ms = s.solve(RELAX_T, sample_dt=RELAX_DT)
    st = s.stats
    M = s.M
    H, _, _ = s.eval()
    out.update(relax_t=ts, relax_m=ms / MS, relax_M=M, relax_H=H,
               relax_stats=np.array([st["t"], st["steps"], st["rejected"]], dtype=np.float64))
    print(f"relax: {st['steps']} steps, {st['rejected']} rejected, {time.time() - t0:.0f} s", flush=True)
    t0 = time.time()
    Hx = applied_field()
    d = oracle_solver(oracle, 0.02, H_ext=Hx)
    d.M = M
    ts, ms = d.solve(DYN_T, sample_dt=DYN_DT)
    st = d.stats
    out.update(dyn_H_ext=np.array(Hx), dyn_t=ts, dyn_m=ms / MS, dyn_M=d.M,
               dyn_stats=np.array([st["t"], st["steps"], st["rejected"]], dtype=np.float64))
    print(f"dynamics: {st['steps']} steps, {st['rejected']} rejected, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
