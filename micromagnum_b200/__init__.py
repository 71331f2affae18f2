"""micromagnum_b200: MicroMagnum's effective-field + LLG + Runge-Kutta hot path on B200 GPUs.

Layers
  include/mmb200.h / libmmb200.so  C ABI over hand-written sm_100a CUDA kernels (csrc/)
  micromagnum_b200.magneto         drop-in mirror of the reference's per-term magneto calls
  micromagnum_b200.solver.Solver   the fused solver (state, stages and controller on the GPU)
"""
from ._lib import LIB_PATH, MMError, build, lib, launches  # noqa: F401

__all__ = ["LIB_PATH", "MMError", "build", "lib", "launches"]
