"""coffee_sim_b200 — B200-native MLS-MPM pour-over step (importable spelling of the
`coffee-sim_b200` package).

The engine is `libcoffee_sim_b200.so`: hand-written sm_100a CUDA kernels behind the C
ABI of include/coffee_sim.h.  This package is its Python host side: a ctypes binding
(`_ffi`), a mirror of the reference's `MpmSim3D` / `MpmSettings` (`sim`), and the
seeded scene generators of the benchmark configurations (`scenes`).
"""
from ._ffi import CsError, CsMetrics, CsSettings, Library  # noqa: F401
from .sim import ENGINE_SO, MpmSettings, MpmSim3D, engine_library  # noqa: F401
