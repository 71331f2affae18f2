"""GPU checks of the drop-in magneto module's containers, OMF files, NR error norm and demag
tensor cache (the per-term field calls are covered in test_gpu_terms.py, the convolution in
test_gpu_demag.py)."""
import os

import numpy as np
import pytest
import torch

from helpers import rel_l2
from test_dropin_host import omf_text

pytestmark = pytest.mark.gpu


@pytest.fixture
def mg():
    from micromagnum_b200 import magneto
    mode = magneto._mode
    magneto.enableCuda(magneto.CUDA_64)
    yield magneto
    magneto._mode = mode


def test_storage_follows_the_precision_mode(mg):
    mesh = mg.RectangularMesh(8, 4, 2, 1e-9, 1e-9, 1e-9)
    M = mg.VectorField(mesh)
    M.fill((1.0, 2.0, 3.0))
    assert M.data.dtype == torch.float64 and not M.isUniform()
    assert torch.equal(M.data.view(3, -1)[:, 5].cpu(), torch.tensor([1.0, 2.0, 3.0], dtype=torch.float64))
    mg.enableCuda(mg.CUDA_32)
    H = mg.VectorField(mesh)
    H.fill((1.0, 0.0, 0.0))
    assert H.data.dtype == torch.float32
    assert M.data.dtype == torch.float32  # converted once on first use in the new mode
    T = mg.GenerateDemagTensor(8, 4, 2, 1e-9, 1e-9, 1e-9, False, False, False, 1, mg.PADDING_ROUND_4)
    assert T.data.dtype == torch.float64  # the tensor stays double in either mode


def test_device_containers(mg):
    mesh = mg.RectangularMesh(5, 4, 3, 1e-9, 2e-9, 3e-9)
    rng = np.random.default_rng(0)
    a = rng.normal(size=(5, 4, 3, 3))
    M = mg.VectorField(mesh)
    M.from_numpy(a)  # [x, y, z, component], the reference's to_numpy layout
    assert np.array_equal(M.to_numpy(), a)
    assert M.get(2, 3, 1) == tuple(a[2, 3, 1])
    assert M.get(2 + 3 * 5 + 1 * 20) == tuple(a[2, 3, 1])
    M.set(1, 1, 1, (7.0, 8.0, 9.0))
    assert M.to_numpy()[1, 1, 1].tolist() == [7.0, 8.0, 9.0]
    b = M.to_numpy()
    assert M.absMax() == pytest.approx(np.sqrt((b ** 2).sum(-1)).max(), rel=1e-15)
    assert M.average() == pytest.approx(tuple(b.reshape(-1, 3).mean(0)), rel=1e-14)
    Ms = mg.Field(mesh)
    ms = rng.uniform(1e5, 1e6, size=(5, 4, 3))
    ms[0, 0, 0] = 0.0
    Ms.from_numpy(ms)
    M.normalize(Ms)
    c = M.to_numpy()
    assert np.allclose(np.linalg.norm(c, axis=-1), ms, rtol=1e-14)
    N = mg.VectorField(mesh)
    N.fill((1.0, -1.0, 0.5))
    assert M.dotSum(N) == pytest.approx((c * np.array([1.0, -1.0, 0.5])).sum(), rel=1e-13)
    N.add(M, 2.0)
    assert np.allclose(N.to_numpy(), 2.0 * c + np.array([1.0, -1.0, 0.5]), rtol=1e-15)
    N.scale_by_vector((1.0, 0.0, 2.0))
    assert np.all(N.to_numpy()[..., 1] == 0.0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("fmt", ["ASCII", "BINARY_4", "BINARY_8"])
def test_omf_round_trip(mg, tmp_path, prec, fmt, golden):
    # the reference's own magnetisation fixture M1 (200x50x1, SP4 state) written and read back
    if prec == "f32":
        mg.enableCuda(mg.CUDA_32)
    nx, ny, nz = (int(v) for v in golden["dims"])
    dx, dy, dz = (float(v) for v in golden["delta"])
    mesh = mg.RectangularMesh(nx, ny, nz, dx, dy, dz)
    M = mg.VectorField(mesh)
    M.from_numpy(golden["M1"])  # (3, N) SoA
    h = mg.OMFHeader()
    h.xnodes, h.ynodes, h.znodes = nx, ny, nz
    h.xstepsize, h.ystepsize, h.zstepsize = dx, dy, dz
    h.meshunit, h.valueunit, h.meshtype, h.Desc = "m", "A/m", "rectangular", ["one", "two"]
    path = str(tmp_path / f"m.{fmt}.omf")
    mg.writeOMF(path, h, M, getattr(mg, "OMF_FORMAT_" + fmt))
    ms = np.sqrt((golden["M1"] ** 2).sum(0))
    assert h.valuemultiplier == pytest.approx(ms.max(), rel=1e-7 if prec == "f32" else 1e-15)
    r = mg.OMFHeader()
    back = mg.readOMF(path, r)
    assert (r.xnodes, r.ynodes, r.znodes, r.Desc, r.valueunit) == (nx, ny, nz, ["one", "two"], "A/m")
    err = np.abs(back.data.view(3, -1).double().cpu().numpy() - M.data.view(3, -1).double().cpu().numpy()).max()
    # text keeps 16 significant digits of the scaled value; binary 4 keeps float32
    # (the header's valuemultiplier carries 16 significant digits)
    tol = {"ASCII": 1e-15, "BINARY_4": 1e-7, "BINARY_8": 1e-15}[fmt] if prec == "f64" else 1e-7
    assert err <= tol * 8e5 + 1e-9
    raw = open(path, "rb").read()
    assert raw.startswith(b"# OOMMF: rectangular mesh v1.0\n# Segment count: 1\n# Begin: Segment\n")
    assert raw.endswith(b"# End: Segment\n")


def test_omf_reads_the_reference_text_layout(mg, monkeypatch):
    # a text file in the reference writer's layout, values scaled by valuemultiplier on reading;
    # unscaled binary 8 (MAGNUM_OMF_NOSCALE, OMFExport.cpp:66) round-trips bit for bit
    monkeypatch.setenv("MAGNUM_OMF_NOSCALE", "1")
    rng = np.random.default_rng(1)
    vals = rng.normal(size=(3 * 2 * 2, 3))
    data = omf_text(3, 2, 2, vals, mult=8e5, newline="\r\n")
    h = mg.OMFHeader()
    M = mg.parseOMF(data, h)
    a = M.to_numpy()  # [x, y, z, c]; file order is x fastest, then y, then z
    assert np.array_equal(a.transpose(2, 1, 0, 3).reshape(-1, 3), vals * 8e5)
    out = mg.formatOMF(h, M, mg.OMF_FORMAT_BINARY_8)
    h2 = mg.OMFHeader()
    assert np.array_equal(mg.parseOMF(out, h2).to_numpy(), a)


def test_nr_error_norm(mg):
    rng = np.random.default_rng(3)
    mesh = mg.RectangularMesh(7, 5, 3, 1e-9, 1e-9, 1e-9)
    y, e = mg.VectorField(mesh), mg.VectorField(mesh)
    yv, ev = rng.normal(size=(3, 105)) * 8e5, rng.normal(size=(3, 105)) * 1e-2
    y.from_numpy(yv)
    e.from_numpy(ev)
    norm = np.sqrt(np.mean((np.abs(ev) / (1e-4 * np.abs(yv) + 1e-3)) ** 2))
    assert mg.rk_adjust_stepsize(5, 1e-12, 1e-3, 1e-4, y, e) == pytest.approx(mg.adjust_from_norm(5, 1e-12, norm),
                                                                             rel=1e-12)


def test_demag_tensor_cache(mg, tmp_path, monkeypatch):
    # a file under the reference's cache name is loaded instead of computing; generations longer
    # than CACHE_AFTER_S are stored (forced here with a zero threshold)
    args = (24, 12, 2, 3e-9, 3e-9, 4e-9, False, False, False, 1, mg.PADDING_ROUND_4)
    monkeypatch.setattr(mg, "CACHE_AFTER_S", 0.0)
    T1 = mg.GenerateDemagTensor(*args, str(tmp_path))
    files = os.listdir(tmp_path)
    assert files == ["Demag--24-12-2--48-24-4--3000-3000-4000.dat"]
    marked = np.fromfile(tmp_path / files[0], dtype=np.float64)
    marked[7] = 12345.0
    marked.tofile(tmp_path / files[0])
    T2 = mg.GenerateDemagTensor(*args, str(tmp_path))
    a, b = T1.data.cpu().numpy(), T2.data.cpu().numpy()
    assert b[7] == 12345.0 and np.array_equal(np.delete(a, 7), np.delete(b, 7))
    monkeypatch.setattr(mg, "CACHE_AFTER_S", 30.0)
    T3 = mg.GenerateDemagTensor(24, 12, 2, 3e-9, 3e-9, 5e-9, False, False, False, 1, mg.PADDING_ROUND_4, str(tmp_path))
    assert len(os.listdir(tmp_path)) == 1 and rel_l2(T3.data.cpu().numpy(), a) > 1e-3
