"""hipims_b200 -- B200 (sm_100a) HiPIMS shallow-water step.

Submodules:
  ops        the reference's op surface (flux, friction/update, time step, rain,
             flux mask, Euler update, infiltration) over the C ABI
  solver     ``Godunov``: the reference solver's object API on those ops
  fused      ``FusedSolver``: one fused kernel per step, single or batched
  topology   compaction, neighbour table, boundary coding
  scenarios  seeded synthetic inputs of the benchmark configurations
"""
from ._lib import LIB_PATH, lib  # noqa: F401

__all__ = ["LIB_PATH", "lib"]
