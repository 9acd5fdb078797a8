"""B200 (sm_100a) implementation of the RadRHD_solver coupled hot path.

Native library: radrhd_solver_b200/librrhd.so (C ABI: include/rrhd.h).
Modules mirror the reference's namespaces: `rhllc` (hydro step, con2prim),
`illum` (scattering integral, moments), `rad_rhd` (radiation 4-force),
`mesh` (synthetic meshes and direction sets), `files_sys` (the reference's
binary geometry, initial-state and solution files).

Submodules load on first use, so `radrhd_solver_b200.build` runs on a tree
where the library has not been built yet; every other submodule imports `_lib`,
which raises ImportError when librrhd.so is missing (there is no fallback).
"""
import importlib

__all__ = ["c2p_mlp", "files_sys", "illum", "illum_mpi", "mesh", "rad_rhd", "rad_rhd_mpi", "ray_tracing", "rhllc",
           "rhllc_mpi"]


def __getattr__(name):
    if name in __all__ or name == "_lib":
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
