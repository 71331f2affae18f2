"""Helpers shared by the test modules (input generators, comparisons)."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def unit_random(rng, n):
    """Per-cell unit vectors uniform on the sphere (normalised Gaussian triples)."""
    v = rng.normal(size=(3, n))
    return v / np.linalg.norm(v, axis=0)


def vortex(dims, delta, core, Ms=8e5, polarization=1, chirality=1, core_radius=10e-9):
    """magnum/micromagnetics/toolbox/vortex.py magnetizationFunction at the cell midpoints
    (RectangularMesh::getPosition returns the middle of a cell)."""
    nx, ny, nz = dims
    dx, dy, dz = delta
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    px, py = (x.ravel() + 0.5) * dx, (y.ravel() + 0.5) * dy
    Mx = -(py - core[1]) * chirality
    My = +(px - core[0]) * chirality
    Mz = np.full_like(Mx, polarization * core_radius)
    s = Ms / np.sqrt(Mx ** 2 + My ** 2 + Mz ** 2)
    return np.stack([Mx * s, My * s, Mz * s])
