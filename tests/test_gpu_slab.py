"""The granular slab the benchmark times, at its full size, against the oracle.

512x512x16 cells of 2 nm, Ms = 1e6 A/m, A = 1.5e-11 J/m, alpha = 0.1, 64 seeded Voronoi grains with
uniaxial K1 = 2e5 J/m^3 along random easy axes, Zhang-Li j = (1e12, 0, 0) A/m^2, P = 0.5, xi = 0.05,
the benchmark's seeded random initial state (bench.grains, bench.initial_M).  The GPU's FP64
demag tensor (which agrees with the exact Newell tensor to ~1e-13) is given to both solvers, so
the comparison isolates the convolution and the field terms: H_demag, H_eff and dM/dt of the FP32
compensated form within 1e-5 (relative L2) and of the plain FP64 form within 1e-12 of the
oracle's FP64 FFT convolution and field loops.  Full size, because the FP32 error of an FFT
convolution grows with the transform lengths (1024 x 1024 x 32 here).
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def slab(oracle_mod):
    import bench
    from micromagnum_b200 import _lib
    nx, ny, nz = bench.DIMS
    n = nx * ny * nz
    reg, axes = bench.grains(bench.DIMS, bench.NGRAINS, bench.SEED)
    M0 = bench.initial_M(n, bench.SEED)
    ex, ey, ez = oracle_mod.padded(nx, ny, nz)
    T = torch.empty(6 * ex * ey * ez, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().mm_demag_tensor(nx, ny, nz, *bench.DELTA, ex, ey, ez, ctypes.c_void_p(T.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    orc = oracle_mod.Solver(bench.DIMS, bench.DELTA, np.full(n, 1e6), A=np.full(n, 1.5e-11), alpha=np.full(n, 0.1),
                            k_uniaxial=np.full(n, 2e5), axis1=axes[reg].T.copy(), P=np.full(n, 0.5),
                            xi=np.full(n, 0.05), j=(1e12, 0.0, 0.0), terms=("demag", "exchange", "uniaxial", "zhangli"),
                            tensor=(T.cpu().numpy(), (ex, ey, ez)), float_norm=False, use_fft=True)
    orc.M = M0
    H, dM, Hd = orc.eval()
    del orc
    return dict(reg=reg, axes=axes, M0=M0, T=T, H=H, dM=dM, Hd=Hd)


@pytest.mark.parametrize("prec,tol", [("f32", 1e-5), ("f64", 1e-12)])
def test_full_size_fields_vs_oracle(slab, prec, tol):
    import bench
    from micromagnum_b200.solver import RectangularMesh, Solver
    s = Solver(RectangularMesh(bench.DIMS, bench.DELTA), bench.materials(slab["axes"]), regions=slab["reg"],
               terms=("demag", "exchange", "uniaxial", "zhangli"), precision=prec, evolver="dp54", eps_abs=1e-3,
               eps_rel=1e-4, tensor=slab["T"])
    s.M = slab["M0"]
    H, dM, Hd = (t.cpu().numpy() for t in s.eval())
    s.close()
    errs = rel_l2(Hd, slab["Hd"]), rel_l2(H, slab["H"]), rel_l2(dM, slab["dM"])
    print(f"{prec}: relative L2 error of H_demag {errs[0]:.3e}, H_eff {errs[1]:.3e}, dM/dt {errs[2]:.3e}")
    assert max(errs) < tol, errs
