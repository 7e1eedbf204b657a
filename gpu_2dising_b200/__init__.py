"""gasp-b200: a B200-native (sm_100a) engine for GASP's many-replica 2D Ising
Metropolis path.  The compute runs in ``libgasp_b200.so`` (C ABI in
include/gasp.h); this package is its host-side mirror of the reference's
interfaces: ``engine`` (device grids, RNG, driver) and ``gasp`` (the PyGASP
entry points ``run_nucleation_swarm`` / ``run_committor_calc``).
"""
from ._native import GaspError, lib  # noqa: F401

__all__ = ["GaspError", "lib"]
