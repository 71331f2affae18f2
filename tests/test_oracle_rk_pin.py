"""Pins the oracle's Runge-Kutta loop (oracle.Solver, a C restatement of the reference's solve
loop) against the reference itself: the unchanged MicroMagnum Python package (RungeKutta.evolve /
apply, runge_kutta.py:47-137; MicroMagneticsStepSizeController, micro_magnetics_stepsize_
controller.py:35-73; the module system and state caches) runs over oracle/magneto_shim.py, a CPU
``magneto`` whose kernels are the reference's own compiled C++ (oracle/_ref/libmmref.so), with the
oracle's restated FFT convolution for the stray field.  Needs a MicroMagnum checkout named by
MMB200_REFERENCE (the Python package is read from there) and the built reference library.
"""
import os
import sys

import numpy as np
import pytest

DIMS, DELTA = (16, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9)


@pytest.fixture(scope="module")
def magnum_cpu(oracle_mod):
    root = oracle_mod.REF_ROOT
    if not root or not os.path.isdir(os.path.join(root, "src", "magnum")) or not oracle_mod.have_reference():
        pytest.skip("needs a MicroMagnum checkout (MMB200_REFERENCE, or the one the build compiled) and "
                    "oracle/_ref/libmmref.so")
    from oracle import magneto_shim
    saved = {k: v for k, v in sys.modules.items() if k == "magnum" or k.startswith("magnum.")}
    for k in saved:
        del sys.modules[k]
    sys.modules["magnum.magneto_cuda"] = magneto_shim
    argv, path = sys.argv, list(sys.path)
    sys.argv = ["magnum", "-l", "3"]
    sys.path.insert(0, os.path.join(root, "src"))
    try:
        import magnum
        yield magnum, magneto_shim
    finally:
        sys.argv = argv
        sys.path[:] = path
        for k in [k for k in sys.modules if k == "magnum" or k.startswith("magnum.")]:
            del sys.modules[k]
        sys.modules.update(saved)


@pytest.mark.parametrize("evolver,h0", [("dp54", 1e-13), ("rkf45", 1e-13), ("cc45", 1e-13), ("rk23", 1e-13),
                                        ("dp54", 1e-12)])
def test_reference_evolver_matches_the_oracle_loop(magnum_cpu, oracle_mod, evolver, h0):
    m, shim = magnum_cpu
    n = int(np.prod(DIMS))
    mesh = m.RectangularMesh(DIMS, DELTA)
    world = m.World(mesh, m.Body("all", m.Material.Py(alpha=0.5), m.Everywhere()))
    solver = m.create_solver(world, [m.StrayField, m.ExchangeField], log=False, evolver=evolver,
                             eps_abs=1e-6, eps_rel=1e-6)
    v = np.random.default_rng(5).normal(size=(3, n))
    M0 = v / np.linalg.norm(v, axis=0) * 8e5
    F = shim.VectorField(mesh)
    F.from_numpy(M0)
    solver.state.M = F
    solver.state.h = h0  # micro_magnetics.py:38 starts at 1e-13
    tensor = oracle_mod.demag_tensor(*DIMS, *DELTA, impl="ref")
    o = oracle_mod.Solver(DIMS, DELTA, 8e5, A=1.3e-11, alpha=0.5, terms=("demag", "exchange"), evolver=evolver,
                          eps_abs=1e-6, eps_rel=1e-6, h0=h0, tensor=tensor, float_norm=True, use_fft=True)
    o.M = M0
    shim.CALLS.clear()
    for _ in range(30):
        solver.step()
        o.step()
        st = o.stats
        assert solver.state.step == st["steps"]
        assert solver.state.t == pytest.approx(st["t"], rel=1e-10)
        assert solver.state.h == pytest.approx(st["h"], rel=1e-10)
        d = np.abs(solver.state.M.arr.reshape(3, -1) - o.M).max() / 8e5
        assert d < 1e-10, d
    # the reference's own kernels did the work (its FFT convolution needs FFTW: the oracle's)
    assert {"exchange", "llge", "scaled_abs_max", "normalize", "conv_fft"} <= set(shim.CALLS)
    if evolver in ("rkf45", "cc45"):
        assert shim.CALLS["rk_prepare_step"] > 0 and shim.CALLS["rk_combine_result"] > 0
    if h0 >= 1e-12:
        assert st["rejected"] > 0  # the oversized first step was rejected and retried
