"""Periodic boundaries on the GPU against the reference and the oracle.

- the periodic demag tensor (mm_demag_tensor_periodic) against the reference's own
  calculateDemagTensor with the same periodic axes and repetitions (oracle/_ref/libmmref.so), with
  and without the images beyond the repetitions (MAGNUM_DEMAG_NO_INFINITY_CORRECTION): the fields
  the two tensors give, since the reference's own tensor carries the truncation of its far-field
  series (~1e-8 in H, its non-periodic tensor against an exact one);
- the convolution along unpadded (periodic) axes, which takes the generic passes, against the
  oracle's direct circular sum with the reference's periodic tensor;
- the fused solver on periodic meshes (wrapping exchange stencil, periodic tensor) against the
  oracle's solver with the same tensor: H_eff, dM/dt and steps.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from helpers import rel_l2, unit_random

pytestmark = pytest.mark.gpu

CASES = [  # dims, delta, periodic axes, repetitions
    ((24, 12, 1), (3e-9, 3e-9, 4e-9), (1, 0, 0), 15),
    ((16, 16, 2), (2e-9, 2e-9, 3e-9), (1, 1, 0), 3),
    ((8, 6, 10), (2e-9, 3e-9, 2e-9), (0, 0, 1), 15),
    ((8, 8, 4), (3e-9, 3e-9, 3e-9), (1, 1, 1), 2),
]


@pytest.fixture(scope="module")
def need_ref(oracle_mod, ref_available):
    if not ref_available:
        pytest.skip("reference not built")
    return oracle_mod


def gpu_tensor(dims, delta, pbc, repeat):
    from micromagnum_b200 import _lib
    e = [d if p else _lib.lib().mm_round_tensor_dimension(d, 0, 2) for d, p in zip(dims, pbc)]
    T = torch.empty(6 * int(np.prod(e)), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().mm_demag_tensor_periodic(*dims, *delta, *pbc, repeat, *e, ctypes.c_void_p(T.data_ptr()),
                                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    return T.cpu().numpy(), tuple(e)


@pytest.mark.parametrize("dims,delta,pbc,repeat", CASES)
@pytest.mark.parametrize("tails", [True, False])
def test_periodic_tensor_vs_reference(need_ref, monkeypatch, dims, delta, pbc, repeat, tails):
    # The images within the repetitions (tails off) agree with the reference to the truncation of
    # its own far-field series (~1e-8 in H).  With the images beyond them the reference's asymptotic
    # tail formula adds its own error, which grows as the repetitions shrink: against a brute-force
    # image sum it is 7e-4 of the tail at 2 repetitions (the default for three periodic axes),
    # 4e-5 at 3 and 7e-11 at 15; the tails here are checked against brute force in
    # test_periodic_tails_vs_image_sum, and the comparison with the reference is bounded by that.
    oracle = need_ref
    if not tails:
        monkeypatch.setenv("MAGNUM_DEMAG_NO_INFINITY_CORRECTION", "1")  # read by both generators
    ours, e = gpu_tensor(dims, delta, pbc, repeat)
    ref, e2 = oracle.demag_tensor(*dims, *delta, impl="ref", pbc=pbc, repeat=repeat)
    assert e == e2
    n = int(np.prod(dims))
    tol = 1e-4 if tails and repeat < 3 else 1e-6
    M = unit_random(np.random.default_rng(7), n) * 8e5
    H = oracle.conv(ours, dims, e, M, method="direct")
    Hr = oracle.conv(ref, dims, e, M, method="direct")
    err = rel_l2(H, Hr)
    print(f"{dims} pbc={pbc} repeat={repeat} tails={tails}: H relative L2 {err:.2e}, "
          f"tensor max |diff| / max |N| {np.abs(ours - ref).max() / np.abs(ref).max():.2e}")
    assert err < tol, err
    # a uniform state (along the periodic axes its field nearly vanishes: compare absolutely)
    Mu = np.repeat([[8e5], [0.0], [0.0]], n, axis=1)
    Hu = oracle.conv(ours, dims, e, Mu, method="direct")
    Hur = oracle.conv(ref, dims, e, Mu, method="direct")
    assert np.abs(Hu - Hur).max() < tol * 8e5


def brute_line_tail(dims, delta, R, A):
    """Sum over images r >= R along axis A of the point-dipole tensor (V / 4 pi) d_a d_b (1 / r),
    for every source offset (the other two axes non-periodic, offsets on them at zero counting
    half), gathered into the octants like the full tensor; 400000 images (remainder < 1e-11)."""
    n3 = np.array(dims)
    d3 = np.array(delta)
    V4 = np.prod(d3) / (4 * np.pi)
    idx = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    S = np.zeros((dims[2], dims[1], dims[0], 6))
    r = np.arange(400000, dtype=np.float64)
    for k in range(dims[2]):
        for j in range(dims[1]):
            for i in range(dims[0]):
                ijk = np.array([i, j, k], dtype=np.float64)
                P = np.repeat((ijk * d3)[:, None], r.size, axis=1)
                P[A] = (ijk[A] + (R + r) * n3[A]) * d3[A]
                r2 = (P * P).sum(0)
                w = np.prod([0.5 if (ijk[c] == 0 and c != A) else 1.0 for c in range(3)])
                for c, (a, b) in enumerate(idx):
                    S[k, j, i, c] = w * V4 * ((3 * P[a] * P[b] - (a == b) * r2) / r2 ** 2.5).sum()
    return S


def test_periodic_tails_vs_image_sum(need_ref, monkeypatch):
    # one periodic axis with 2 repetitions: (tensor with the images beyond) - (tensor without them)
    # against the brute-force image sum gathered into the octants
    dims, delta, pbc, R = (6, 4, 2), (2e-9, 3e-9, 2.5e-9), (1, 0, 0), 2
    with_t, e = gpu_tensor(dims, delta, pbc, R)
    monkeypatch.setenv("MAGNUM_DEMAG_NO_INFINITY_CORRECTION", "1")
    without, _ = gpu_tensor(dims, delta, pbc, R)
    got = (with_t - without).reshape(e[2], e[1], e[0], 6)
    S = brute_line_tail(dims, delta, R, 0)
    want = np.zeros_like(got)
    for K in range(e[2]):
        for J in range(e[1]):
            for I in range(e[0]):
                for o in (-1, 1):
                    i = (o * I + e[0]) % e[0]
                    for p in (-1, 1):
                        j = (p * J + e[1]) % e[1]
                        for q in (-1, 1):
                            k = (q * K + e[2]) % e[2]
                            if i >= dims[0] or j >= dims[1] or k >= dims[2]:
                                continue
                            s = S[k, j, i]
                            want[K, J, I] += [s[0], o * p * s[1], o * q * s[2], s[3], p * q * s[4], s[5]]
    err = np.abs(got - want).max() / np.abs(want).max()
    print(f"line tail vs brute force: {err:.2e} (of the tail)")
    assert err < 1e-8


@pytest.mark.parametrize("dims,delta,pbc,repeat", CASES)
@pytest.mark.parametrize("prec,tol", [("f64", 1e-12), ("f32", 1e-5)])
def test_periodic_convolution_vs_direct_sum(need_ref, dims, delta, pbc, repeat, prec, tol):
    from micromagnum_b200 import magneto as mg
    oracle = need_ref
    ref, e = oracle.demag_tensor(*dims, *delta, impl="ref", pbc=pbc, repeat=repeat)
    n = int(np.prod(dims))
    M = unit_random(np.random.default_rng(8), n) * 8e5
    Hr = oracle.conv(ref, dims, e, M, method="direct")
    mode = mg._mode
    try:
        mg.enableCuda(mg.CUDA_64 if prec == "f64" else mg.CUDA_32)
        T = mg.Matrix(mg.Shape(6, *e), _fixed_dtype=torch.float64)
        T.data.copy_(torch.from_numpy(ref))
        conv = mg.SymmetricMatrixVectorConvolution_FFT(T, *dims)
        Mv, Hv = mg.VectorMatrix(mg.Shape(*dims)), mg.VectorMatrix(mg.Shape(*dims))
        Mv.from_numpy(M)
        conv.execute(Mv, Hv)
        H = Hv.data.view(3, -1).double().cpu().numpy()
    finally:
        mg._mode = mode
    assert rel_l2(H, Hr) < tol


@pytest.mark.parametrize("dims,delta,pbc,repeat", [CASES[0], CASES[1], CASES[3]])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_periodic_solver_vs_oracle(need_ref, dims, delta, pbc, repeat, prec):
    from micromagnum_b200 import solver as sv
    oracle = need_ref
    n = int(np.prod(dims))
    ref = oracle.demag_tensor(*dims, *delta, impl="ref", pbc=pbc, repeat=repeat)
    axes = "".join(a for a, p in zip("xyz", pbc) if p)
    mesh = sv.RectangularMesh(dims, delta, axes, repeat)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.3)]
    kw = dict(evolver="dp54", eps_abs=1e-5, eps_rel=1e-5, H_ext=(1e4, 0.0, 2e3))
    ours = sv.Solver(mesh, mats, terms=("demag", "exchange"), precision=prec, tensor=ref[0], **kw)
    orc = oracle.Solver(dims, delta, np.full(n, 8e5), A=np.full(n, 1.3e-11), alpha=np.full(n, 0.3),
                        terms=("demag", "exchange"), tensor=ref, float_norm=False, pbc=pbc, **kw)
    if prec == "f64":
        M = unit_random(np.random.default_rng(9), n) * 8e5
    else:
        # FP32 trajectories are compared from a smooth state (a random one starts with violent
        # exchange dynamics whose FP32/FP64 differences exceed 1e-4 within picoseconds)
        v = np.array([[1.0], [0.3], [0.1]]) + 0.2 * np.random.default_rng(9).normal(size=(3, n))
        M = v / np.linalg.norm(v, axis=0) * 8e5
    ours.M = M
    orc.M = M
    H, dM, _ = (t.cpu().numpy() for t in ours.eval())
    Hr, dMr, _ = orc.eval()
    tol = 1e-12 if prec == "f64" else 1e-5
    assert rel_l2(H, Hr) < tol
    assert rel_l2(dM, dMr) < tol
    if prec == "f64":
        # the same step sequence as the oracle
        for _ in range(10):
            ours.step()
            orc.step()
        assert ours.stats["steps"] == orc.stats["steps"]
        assert rel_l2(ours.M.cpu().numpy(), orc.M) < 1e-10
    else:
        # FP32 step sizes differ from FP64 ones after a few steps, so <M> is compared at fixed times
        t, m = ours.solve(2e-12, sample_dt=2e-13)
        tr, mr = orc.solve(2e-12, sample_dt=2e-13)
        keep, keepr = np.append(np.abs(np.diff(t)) > 1e-15, True), np.append(np.abs(np.diff(tr)) > 1e-15, True)
        assert np.allclose(t[keep], tr[keepr], rtol=1e-12, atol=0)
        assert np.abs(m[keep] - mr[keepr]).max() / 8e5 < 1e-4


def test_solver_generates_the_periodic_tensor(need_ref):
    # without a tensor passed in, the solver builds the periodic one on the GPU from the mesh
    from micromagnum_b200 import solver as sv
    oracle = need_ref
    dims, delta, pbc, repeat = CASES[1]
    n = int(np.prod(dims))
    ours_t, e = gpu_tensor(dims, delta, pbc, repeat)
    mats = [sv.Material(Ms=8e5, A=1.3e-11, alpha=0.3)]
    a = sv.Solver(sv.RectangularMesh(dims, delta, "xy", repeat), mats, precision="f64")
    b = sv.Solver(sv.RectangularMesh(dims, delta, "xy", repeat), mats, precision="f64", tensor=ours_t)
    M = unit_random(np.random.default_rng(10), n) * 8e5
    a.M = M
    b.M = M
    assert rel_l2(a.eval()[2].cpu().numpy(), b.eval()[2].cpu().numpy()) < 1e-15
    assert e == (16, 16, oracle.round_tensor_dimension(2, False, 2))
