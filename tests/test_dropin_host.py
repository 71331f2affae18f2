"""CPU checks of the drop-in magneto module (micromagnum_b200.magneto) that need no GPU.

- the containers' uniform state (matty's AbstractMatrix UNIFORM: one value, no storage), which
  serves every operation that needs no per-cell data, and a clear RuntimeError for everything
  that would need the device
- RectangularMesh, Field, VectorField (mesh/RectangularMesh.h, mesh/Field.i, mesh/VectorField.i)
- the demag tensor cache file name (mmm/demag/demag_tensor.cpp:52-73)
- OMF header parsing (mmm/io/OMFImport.cpp), which runs on the host
- the NR step-size rule (evolver/runge_kutta.cpp:98-130)
- the unchanged MicroMagnum package importing and setting up a world and solver over this module
  (when a MicroMagnum checkout is named by MMB200_REFERENCE)
"""
import ctypes
import math
import os
import sys

import numpy as np
import pytest

from micromagnum_b200 import _lib
from micromagnum_b200 import magneto as mg


@pytest.fixture(scope="module", autouse=True)
def library():
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()


def test_uniform_containers_need_no_device():
    mesh = mg.RectangularMesh(4, 3, 2, 1e-9, 2e-9, 3e-9)
    M = mg.VectorField(mesh)
    assert M.isUniform() and M.uniform_value == (0.0, 0.0, 0.0) and M.mesh is mesh
    M.fill((3.0, 0.0, 4.0))
    assert M.absMax() == 5.0
    assert M.average() == (3.0, 0.0, 4.0) and M.sum() == (72.0, 0.0, 96.0)
    M.scale(2.0)
    assert M.uniform_value == (6.0, 0.0, 8.0)
    M.normalize(1.0)
    assert M.uniform_value == pytest.approx((0.6, 0.0, 0.8))
    Ms = mg.Field(mesh)
    Ms.fill(8e5)
    M.normalize(Ms)
    assert M.uniform_value == pytest.approx((4.8e5, 0.0, 6.4e5))
    H = mg.VectorField(mesh)
    H.fill((1.0, 2.0, 3.0))
    assert M.dotSum(H) == pytest.approx(24 * (4.8e5 + 3 * 6.4e5))
    H.add(M, 0.5)
    assert H.uniform_value == pytest.approx((1.0 + 2.4e5, 2.0, 3.0 + 3.2e5))
    a = M.to_numpy()
    assert a.shape == (4, 3, 2, 3) and np.all(a[..., 2] == pytest.approx(6.4e5))
    assert Ms.to_numpy().shape == (4, 3, 2) and Ms.average() == 8e5 and Ms.sum() == 24 * 8e5
    assert M.get(5) == M.uniform_value and Ms.get(1, 2, 1) == 8e5
    Ms.set(3, 8e5)  # same value: stays uniform, as in matty.inc.i set()
    assert Ms.isUniform()
    c = mg.VectorMatrix(M)  # copy constructor
    assert c.uniform_value == M.uniform_value and c.shape == (4, 3, 2)
    assert mg.Shape(4, 3, 2).getLinIdx(1, 2, 1) == 1 + 2 * 4 + 1 * 12
    # anything that needs per-cell storage asks for the device
    with pytest.raises(RuntimeError):
        Ms.set(3, 1.0)


def test_device_calls_raise_when_cuda_is_disabled():
    mode = mg._mode
    try:
        mg.enableCuda(mg.CUDA_DISABLED)
        assert not mg.isCudaEnabled()
        M = mg.VectorMatrix(mg.Shape(4, 4, 1))
        with pytest.raises(RuntimeError, match="no CPU implementation"):
            _ = M.data
        with pytest.raises(RuntimeError, match="no CPU implementation"):
            mg.llge(mg.Matrix(mg.Shape(4, 4, 1)), mg.Matrix(mg.Shape(4, 4, 1)), M, M, M)
    finally:
        mg._mode = mode


def test_rectangular_mesh_api():
    m = mg.RectangularMesh(10, 5, 2, 1e-9, 2e-9, 3e-9)
    assert m.num_nodes == (10, 5, 2) and m.delta == (1e-9, 2e-9, 3e-9) and m.total_nodes == 100
    assert m.cell_volume == pytest.approx(6e-27) and m.volume == pytest.approx(6e-25)
    assert m.size == pytest.approx((1e-8, 1e-8, 6e-9))
    assert m.periodic_bc == ("", 1)
    # linear index 1*(10*5) + 1*10 + 3 -> (x, y, z) = (3, 1, 1): the cell's middle point
    assert m.getPosition(63) == pytest.approx((3.5e-9, 3e-9, 4.5e-9))
    # periodic repetitions default to 1, 15, 3, 2 for 0..3 periodic directions (RectangularMesh.h:10-19)
    assert [mg.RectangularMesh(4, 4, 4, 1, 1, 1, p).periodic_bc[1] for p in ("", "x", "xy", "xyz")] == [1, 15, 3, 2]
    assert mg.RectangularMesh(4, 4, 4, 1, 1, 1, "y", 7).periodic_bc == ("y", 7)
    assert m.isCompatible(mg.RectangularMesh(10, 5, 2, 1e-9, 2e-9, 3e-9))
    assert not m.isCompatible(mg.RectangularMesh(10, 5, 2, 1e-9, 2e-9, 4e-9))
    assert list(m.iterateCellIndices())[:3] == [(0, 0, 0), (0, 0, 1), (0, 1, 0)]
    from micromagnum_b200.solver import RectangularMesh
    s = RectangularMesh((10, 5, 2), (1e-9, 2e-9, 3e-9), "x")
    assert s.num_nodes == (10, 5, 2) and s.periodic_bc == ("x", 15)


def test_demag_cache_file_name():
    # demag_tensor.cpp:52-73: sizes, padded sizes, cell size in whole picometres (truncated), and
    # the periodic directions with their repetitions
    f = mg.demag_cache_file(128, 32, 1, 256, 64, 1, 3.90625e-9, 3.90625e-9, 3e-9, False, False, False, 1, "/c")
    assert f == "/c/Demag--128-32-1--256-64-1--3906-3906-3000.dat"
    g = mg.demag_cache_file(128, 32, 1, 256, 64, 1, 3.9062e-9, 3.90625e-9, 3e-9, False, False, False, 1, "/c")
    assert g == f  # below 1 pm apart: the same file, as in the reference
    p = mg.demag_cache_file(64, 64, 1, 64, 128, 1, 2e-9, 2e-9, 2e-9, True, False, False, 15, "/c")
    assert p == "/c/Demag--64-64-1--64-128-1--2000-2000-2000--p-x-15.dat"


def omf_text(nx, ny, nz, values, mult=1.0, newline="\n", desc=("a", "b")):
    """An OMF 1.0 text file in the layout the reference writes (OMFExport.cpp:83-137)."""
    lines = ["# OOMMF: rectangular mesh v1.0", "# Segment count: 1", "# Begin: Segment", "# Begin: Header",
             "# Title: t"] + [f"# Desc: {d}" for d in desc] + [
        "# meshunit: m", "# valueunit: A/m", f"# valuemultiplier: {mult!r}", "# xmin: 0", "# ymin: 0", "# zmin: 0",
        f"# xmax: {nx * 1e-9!r}", f"# ymax: {ny * 2e-9!r}", f"# zmax: {nz * 3e-9!r}", "# ValueRangeMaxMag: 1",
        "# ValueRangeMinMag: 0", "# meshtype: rectangular", "# xbase: 5e-10", "# ybase: 1e-09", "# zbase: 1.5e-09",
        "# xstepsize: 1e-09", "# ystepsize: 2e-09", "# zstepsize: 3e-09", f"# xnodes: {nx}", f"# ynodes: {ny}",
        f"# znodes: {nz}", "# Unknown: ignored", "# End: Header", "# Begin: Data Text"]
    lines += [" ".join(repr(float(x)) for x in v) for v in values]
    lines += ["# End: Data Text", "# End: Segment"]
    return (newline.join(lines) + newline).encode()


@pytest.mark.parametrize("newline", ["\n", "\r\n", "\r", "\n\r"])
def test_omf_header_is_parsed_on_the_host(newline):
    vals = np.arange(2 * 3 * 1 * 3, dtype=float).reshape(-1, 3)
    data = omf_text(2, 3, 1, vals, mult=800000.0, newline=newline)
    h = _lib.mm_omf_header()
    buf = ctypes.create_string_buffer(data, len(data))
    _lib.check(_lib.lib().mm_omf_parse(buf, len(data), ctypes.byref(h), 0, None, None))
    assert (h.xnodes, h.ynodes, h.znodes) == (2, 3, 1) and h.format == _lib.MM_OMF_TEXT
    assert h.valuemultiplier == 800000.0 and h.zstepsize == 3e-9 and h.xbase == 5e-10
    assert h.title == b"t" and h.desc == b"a\nb" and h.meshunit == b"m" and h.meshtype == b"rectangular"
    hdr = mg.OMFHeader()
    hdr._from_c(h)
    assert hdr.Desc == ["a", "b"] and hdr.xnodes == 2 and hdr.valueunit == "A/m"


def test_omf_malformed_input_is_rejected():
    L = _lib.lib()
    h = _lib.mm_omf_header()
    for bad in (b"", b"# Segment count: 1\n", b"# OOMMF: x\n# Segment count: 1\n# Begin: Segment\n# Begin: Header\n"):
        buf = ctypes.create_string_buffer(bad, max(1, len(bad)))
        assert L.mm_omf_parse(buf, len(bad), ctypes.byref(h), 0, None, None) == 1
    data = omf_text(2, 2, 1, np.zeros((4, 3))).replace(b"Data Text", b"Data Binary 16")
    buf = ctypes.create_string_buffer(data, len(data))
    assert L.mm_omf_parse(buf, len(data), ctypes.byref(h), 0, None, None) == 1
    assert b"Data Text" in L.mm_last_error()


def test_nr_step_size_rule():
    # runge_kutta.cpp:98-130, S = 0.9: shrink above 1.1 (at most 5x), grow below 0.5 (1x..5x)
    assert mg.adjust_from_norm(5, 1.0, 2.0) == pytest.approx(0.9 / 2 ** 0.2)
    assert mg.adjust_from_norm(5, 1.0, 1e9) == pytest.approx(0.2)
    assert mg.adjust_from_norm(5, 1.0, 0.8) == 1.0
    assert mg.adjust_from_norm(5, 1.0, 0.1) == pytest.approx(max(1.0, min(5.0, 0.9 / 0.1 ** (1 / 6))))
    assert mg.adjust_from_norm(5, 1.0, 1e-12) == 5.0
    assert mg.adjust_from_norm(20, 1.0, 0.45) == 1.0  # S / norm^(1/21) < 1: no decrease


@pytest.fixture
def magnum_pkg(monkeypatch):
    """The unchanged MicroMagnum package (src/magnum of the checkout named by MMB200_REFERENCE),
    imported with this module installed as its native backend the way INTEGRATION.md binds it."""
    import oracle
    root = oracle.REF_ROOT
    if not root or not os.path.isdir(os.path.join(root, "src", "magnum")):
        pytest.skip("no MicroMagnum checkout (MMB200_REFERENCE, or the one the build compiled)")
    for name in [k for k in sys.modules if k == "magnum" or k.startswith("magnum.")]:
        monkeypatch.delitem(sys.modules, name)
    monkeypatch.setitem(sys.modules, "magnum.magneto_cuda", mg)
    monkeypatch.syspath_prepend(os.path.join(root, "src"))
    monkeypatch.setattr(sys, "argv", ["magnum"])  # no -g/-G: CUDA disabled
    mode = mg._mode
    import magnum
    yield magnum
    mg._mode = mode


def test_unchanged_magnum_sets_up_over_the_drop_in(magnum_pkg):
    m = magnum_pkg
    assert m.magneto.RectangularMesh is mg.RectangularMesh and m.magneto.llge is mg.llge
    mesh = m.RectangularMesh((32, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9))
    world = m.World(mesh, m.Body("all", m.Material.Py(alpha=0.5), m.Everywhere()))
    solver = m.create_solver(world, [m.ExchangeField], log=False, evolver="rkf45")
    solver.state.M = (8e5, 0, 0)
    assert solver.state.M.isUniform() and solver.state.M.uniform_value == (8e5, 0.0, 0.0)
    assert isinstance(solver.state.M, mg.VectorField) and solver.state.M.mesh.num_nodes == (32, 8, 1)
    # no -g/-G: the first computation asks for CUDA instead of running on the host
    with pytest.raises(RuntimeError, match="CUDA is disabled"):
        solver.step()
