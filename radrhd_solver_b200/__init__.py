"""B200 (sm_100a) implementation of the RadRHD_solver coupled hot path.

Native library: radrhd_solver_b200/librrhd.so (C ABI: include/rrhd.h).
Modules mirror the reference's namespaces: `rhllc` (hydro step, con2prim),
`illum` (scattering integral, moments), `rad_rhd` (radiation 4-force),
`mesh` (synthetic meshes and direction sets).
"""
from . import _lib  # noqa: F401  (fails loudly if librrhd.so is missing)
from . import illum, mesh, rad_rhd, rhllc  # noqa: F401

__all__ = ["illum", "mesh", "rad_rhd", "rhllc"]
