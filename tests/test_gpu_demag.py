"""GPU parity of the demag path: the FP64 tensor generator against the exact (binary128 Newell)
oracle tensor, and the FFT convolution against the oracle's direct summation with the
reference's own tensor injected (the <= 1e-12 gate of the plain FP64 mode), plus the
reference's H1_stray golden field and full-size (512x512x16) linearity / spot checks."""
import math

import numpy as np
import pytest
import torch

from helpers import rel_l2, unit_random

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mg():
    from micromagnum_b200 import magneto
    return magneto


def mode(mg, prec):
    mg.enableCuda(mg.CUDA_64 if prec == "f64" else mg.CUDA_32)


def vfield(mg, dims, data):
    f = mg.VectorMatrix(dims)
    f.data.copy_(torch.as_tensor(np.asarray(data, dtype=np.float64).reshape(-1)))
    return f


def tensor_matrix(mg, N, pd):
    T = mg.Matrix((6,) + tuple(pd))
    T.data.copy_(torch.as_tensor(np.asarray(N, dtype=np.float64).reshape(-1)))
    return T


@pytest.mark.parametrize("case", [((8, 5, 3), (3.90625e-9, 3.90625e-9, 3e-9)),
                                  ((128, 32, 1), (3.90625e-9, 3.90625e-9, 3e-9)),
                                  ((40, 24, 8), (2e-9, 2e-9, 2e-9)),
                                  ((30, 20, 6), (5e-9, 2e-9, 1e-9)),
                                  ((1, 9, 5), (2e-9, 3e-9, 4e-9))])
def test_gpu_tensor_vs_exact(mg, oracle_mod, case):
    (nx, ny, nz), d = case
    N_ref, pd = oracle_mod.demag_tensor(nx, ny, nz, *d)
    T = mg.GenerateDemagTensor(nx, ny, nz, *d, False, False, False, 1, mg.PADDING_ROUND_4)
    assert T.shape == (6,) + pd
    N = T.data.cpu().numpy()
    # element-wise error relative to the tensor's largest entry, and relative L2
    assert np.abs(N - N_ref).max() < 1e-13 * np.abs(N_ref).max()
    assert rel_l2(N, N_ref) < 1e-12


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("case", [((128, 32, 1), (3.90625e-9, 3.90625e-9, 3e-9)),
                                  ((24, 20, 6), (2e-9, 2e-9, 2e-9)),
                                  ((13, 7, 5), (2e-9, 3e-9, 4e-9)),
                                  ((1, 8, 3), (2e-9, 3e-9, 4e-9)),
                                  ((9, 1, 1), (1e-9, 1e-9, 1e-9)),
                                  ((33, 17, 2), (3e-9, 3e-9, 3e-9))])
def test_conv_reference_tensor_vs_direct(mg, oracle_mod, ref_available, prec, case):
    # the reference's own tensor injected: isolates the convolution error
    if not ref_available:
        pytest.skip("reference not built")
    mode(mg, prec)
    (nx, ny, nz), d = case
    dims = (nx, ny, nz)
    N, pd = oracle_mod.demag_tensor(nx, ny, nz, *d, impl="ref")
    rng = np.random.default_rng(21)
    M = unit_random(rng, nx * ny * nz) * 8e5
    H_ref = oracle_mod.conv(N, dims, pd, M, method="direct")
    conv = mg.SymmetricMatrixVectorConvolution_FFT(tensor_matrix(mg, N, pd), nx, ny, nz)
    H = mg.VectorMatrix(dims)
    conv.execute(vfield(mg, dims, M), H)
    err = rel_l2(H.data.view(3, -1).cpu().numpy(), H_ref)
    assert err < (1e-12 if prec == "f64" else 1e-5), err


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_stray_golden(mg, golden, prec):
    # stray_field_test.py:29-50: M1 -> H1_stray within 1 A/m, tensor generated on the GPU
    mode(mg, prec)
    (nx, ny, nz), (dx, dy, dz) = [int(v) for v in golden["dims"]], golden["delta"]
    dims = (nx, ny, nz)
    T = mg.GenerateDemagTensor(nx, ny, nz, dx, dy, dz, False, False, False, 1, mg.PADDING_ROUND_4)
    conv = mg.SymmetricMatrixVectorConvolution_FFT(T, nx, ny, nz)
    H = mg.VectorMatrix(dims)
    H.fill((1.0, 2.0, 3.0))
    conv.execute(vfield(mg, dims, golden["M1"]), H)
    assert np.abs(H.data.view(3, -1).cpu().numpy() - golden["H1_stray"]).max() < 1.0


def test_spectrum_is_real(mg, oracle_mod):
    # the tensor spectrum's imaginary part is rounding noise (what the real-only storage uses)
    from micromagnum_b200 import _lib
    import ctypes
    mode(mg, "f64")
    nx, ny, nz = 20, 12, 6
    N, pd = oracle_mod.demag_tensor(nx, ny, nz, 2e-9, 2e-9, 2e-9)
    Nh = np.fft.fftn(N.reshape(pd[2], pd[1], pd[0], 6), axes=(0, 1, 2))
    assert np.abs(Nh.imag).max() < 1e-12 * np.abs(Nh.real).max()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_full_size_slab_properties(mg, oracle_mod, prec):
    # 512x512x16 slab of 2 nm cubes (the granular-slab workload): linearity of the convolution
    # and a direct-summation check of the field at sampled cells
    mode(mg, prec)
    nx, ny, nz = 512, 512, 16
    dims = (nx, ny, nz)
    n = nx * ny * nz
    T = mg.GenerateDemagTensor(nx, ny, nz, 2e-9, 2e-9, 2e-9, False, False, False, 1, mg.PADDING_ROUND_4)
    conv = mg.SymmetricMatrixVectorConvolution_FFT(T, nx, ny, nz)
    g = torch.Generator(device="cuda").manual_seed(7)
    M1 = torch.randn(3 * n, generator=g, device="cuda", dtype=torch.float64) * 4e5
    M2 = torch.randn(3 * n, generator=g, device="cuda", dtype=torch.float64) * 4e5
    outs = []
    for data in (M1, M2, 0.3 * M1 - 1.7 * M2):
        v = mg.VectorMatrix(dims)
        v.data.copy_(data)
        H = mg.VectorMatrix(dims)
        conv.execute(v, H)
        outs.append(H.data.clone())
    lin = outs[2] - (0.3 * outs[0] - 1.7 * outs[1])
    assert float(lin.norm() / outs[2].norm()) < (1e-13 if prec == "f64" else 1e-5)
    # direct summation at a few cells: H_i = sum_j N(i - j) M_j (tensor in reference layout)
    ex, ey, ez = T.shape[1:]
    Nt = T.data.view(ez, ey, ex, 6)
    Mv = M1.view(3, nz, ny, nx)
    zz, yy, xx = torch.meshgrid(torch.arange(nz, device="cuda"), torch.arange(ny, device="cuda"),
                                torch.arange(nx, device="cuda"), indexing="ij")
    H1 = outs[0].view(3, nz, ny, nx)
    for (x, y, z) in [(0, 0, 0), (255, 100, 7), (511, 511, 15), (3, 400, 9)]:
        X = (x - xx) % ex
        Y = (y - yy) % ey
        Z = (z - zz) % ez
        Nl = Nt[Z, Y, X]  # (nz, ny, nx, 6)
        hx = (Nl[..., 0] * Mv[0] + Nl[..., 1] * Mv[1] + Nl[..., 2] * Mv[2]).sum()
        hy = (Nl[..., 1] * Mv[0] + Nl[..., 3] * Mv[1] + Nl[..., 4] * Mv[2]).sum()
        hz = (Nl[..., 2] * Mv[0] + Nl[..., 4] * Mv[1] + Nl[..., 5] * Mv[2]).sum()
        ref = torch.stack([hx, hy, hz])
        got = H1[:, z, y, x]
        assert float((got - ref).norm() / ref.norm()) < (1e-11 if prec == "f64" else 1e-4)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dims", [(32, 16, 8), (64, 64, 16), (256, 32, 4), (512, 8, 2), (1024, 4, 2),
                                  (16, 512, 3), (8, 8, 8), (2, 2, 2)])
def test_conv_power_of_two_paths(mg, oracle_mod, prec, dims):
    # padded lengths that are powers of two take the register-FFT passes; checked against the
    # oracle's FFT convolution (itself pinned to direct summation) with the same tensor
    mode(mg, prec)
    nx, ny, nz = dims
    d = (2e-9, 3e-9, 2.5e-9)
    N, pd = oracle_mod.demag_tensor(nx, ny, nz, *d)
    rng = np.random.default_rng(31)
    M = unit_random(rng, nx * ny * nz) * 8e5
    H_ref = oracle_mod.conv(N, dims, pd, M, method="fft")
    conv = mg.SymmetricMatrixVectorConvolution_FFT(tensor_matrix(mg, N, pd), nx, ny, nz)
    H = mg.VectorMatrix(dims)
    conv.execute(vfield(mg, dims, M), H)
    err = rel_l2(H.data.view(3, -1).cpu().numpy(), H_ref)
    assert err < (1e-12 if prec == "f64" else 1e-5), err
