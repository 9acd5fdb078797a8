"""Relativistic HLLC hydro, mirroring the reference's `rhllc` namespace.

    grid = Grid(mesh, eos=EOS_IDEAL, gamma=4/3)      # grid_t + InitMemory
    grid.set_state_prim(W)                            # HllcPhysToConv
    Hllc3dStab(tau, grid)                             # rhllc::Hllc3dStab
    tau = GetTimeStep(cfl, h_min)                     # rhllc::GetTimeStep

The state lives on the GPU; `grid.get_state()` copies it back.  Functions
raise `RrhdError` where the reference would abort (DIE_IF), e.g. when
con2prim fails in a cell even after PhysPressureFix.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .mesh import Mesh

EOS_IDEAL = L.RRHD_EOS_IDEAL
EOS_TAUB = L.RRHD_EOS_TAUB
BC_TRANSMISSIVE = L.RRHD_BC_TRANSMISSIVE
BC_FIXED = L.RRHD_BC_FIXED
BC_REFLECT = L.RRHD_BC_REFLECT

# rhllc::max_signal_speed (solvers/rhllc/src/rhllc_utils.cpp:13); updated by Hllc3dStab
max_signal_speed = 1.0


class Grid:
    """Device-resident mesh + cell state (grid_t, lib/grids/include/solvers_struct.h:317-387)."""

    def __init__(self, mesh: Mesh, eos: int = EOS_IDEAL, gamma: float = 5.0 / 3.0, device: int = 0,
                 cells_per_block: int = 0, renumber: bool = True):
        self.mesh = mesh
        self.eos = eos
        self.gamma = gamma
        self.size = mesh.n_cells
        self.device = device
        o = L.Opts(eos, gamma, device, cells_per_block, 0 if renumber else -1)
        h = C.c_void_p()
        L.check(L.lib.rrhd_create(C.byref(mesh.desc()), C.byref(o), C.byref(h)), "rrhd_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        return L.lib.rrhd_stream(self._h)

    def close(self):
        if self._h:
            L.lib.rrhd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_boundary(self, code: int, kind: int, W=None):
        w = None if W is None else np.ascontiguousarray(W, dtype=np.float64)
        L.check(L.lib.rrhd_set_boundary(self._h, code, kind, L.ptr(w)), "set_boundary")

    def set_state(self, W=None, U=None):
        where, W, U = _where(W, U)
        L.check(L.lib.rrhd_set_state(self._h, L.ptr(W), L.ptr(U), 5, where), "set_state")
        if where == L.RRHD_HOST:
            self.sync()

    def set_state_prim(self, W):
        where, W, _ = _where(W, None)
        L.check(L.lib.rrhd_set_state_prim(self._h, L.ptr(W), 5, where), "set_state_prim")
        self.sync()

    def get_state(self):
        W = np.zeros((self.size, 5))
        U = np.zeros((self.size, 5))
        L.check(L.lib.rrhd_get_state(self._h, L.ptr(W), L.ptr(U), 5, L.RRHD_HOST), "get_state")
        return W, U

    def keep_face_flux(self, on: bool = True):
        L.check(L.lib.rrhd_keep_face_flux(self._h, 1 if on else 0), "keep_face_flux")

    def face_flux(self) -> np.ndarray:
        F = np.zeros((self.mesh.n_faces, 5))
        L.check(L.lib.rrhd_get_face_flux(self._h, L.ptr(F)), "get_face_flux")
        return F

    def cell_status(self) -> np.ndarray:
        s = np.zeros(self.size, np.uint8)
        L.check(L.lib.rrhd_get_cell_status(self._h, L.ptr(s)), "get_cell_status")
        return s

    def set_time_step(self, cfl: float, h_min: float, initial_max_speed: float = 0.0):
        L.check(L.lib.rrhd_set_time_step(self._h, cfl, h_min, initial_max_speed), "set_time_step")

    def step_info(self):
        t, m = C.c_double(), C.c_double()
        L.check(L.lib.rrhd_get_step_info(self._h, C.byref(t), C.byref(m)), "get_step_info")
        return t.value, m.value

    def sync(self):
        L.check(L.lib.rrhd_sync(self._h), "sync")

    def layout_info(self):
        """The step kernel's layout: cells per CTA, CTA blocks, the length of all CTAs' face
        lists together (faces between two blocks are fluxed by both) and the mesh's faces."""
        cpb, nb, fe, f = C.c_int32(), C.c_int32(), C.c_int64(), C.c_int64()
        L.check(L.lib.rrhd_hydro_layout_info(self._h, C.byref(cpb), C.byref(nb), C.byref(fe), C.byref(f)),
                "rrhd_hydro_layout_info")
        return {"cells_per_block": cpb.value, "blocks": nb.value, "face_entries": fe.value, "faces": f.value}


def _where(W, U):
    t = W if W is not None else U
    if hasattr(t, "is_cuda") and t.is_cuda:
        return L.RRHD_DEVICE, (W.contiguous() if W is not None else None), (U.contiguous() if U is not None else None)
    f = (lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64))
    return L.RRHD_HOST, f(W), f(U)


def Hllc3dStab(tau: float, grid: Grid) -> L.StepStats:
    """One step (solvers/rhllc/src/rhllc_3d_stab.cpp:10-63); sets max_signal_speed."""
    global max_signal_speed
    st = L.StepStats()
    L.check(L.lib.rrhd_hydro_step(grid.handle, tau, C.byref(st)), "Hllc3dStab")
    max_signal_speed = st.max_speed
    return st


def GetTimeStep(cfl: float, h_min: float) -> float:
    """tau = CFL * h_min / max_signal_speed (solvers/rhllc/src/rhllc_utils.cpp:15-23)."""
    t = cfl * h_min / max_signal_speed
    if t < 0:
        raise RuntimeError("negative time step")
    return t


def GetPhysValueStab(U, W, status=None, eos: int = EOS_IDEAL, gamma: float = 5.0 / 3.0,
                     fallback: bool = False, stream=None):
    """Batched con2prim on device tensors [n,5] (rhllc_flux_stab.cpp:123-220);
    with fallback=True also PhysPressureFix (:40-121), which rewrites U[:,4]."""
    n = U.shape[0]
    L.check(L.lib.rrhd_con2prim_batch(eos, gamma, L.ptr(U), L.ptr(W), L.ptr(status), n, 1 if fallback else 0,
                                      stream), "GetPhysValueStab")


def GetPhysValueStabStats(U, W, status=None, eos: int = EOS_IDEAL, gamma: float = 5.0 / 3.0,
                          fallback: bool = True, stream=None) -> L.C2pStats:
    """Batched con2prim with totals (solved, fallbacks, failures, Newton
    iterations); synchronises the stream."""
    st = L.C2pStats()
    L.check(L.lib.rrhd_con2prim_batch_stats(eos, gamma, L.ptr(U), L.ptr(W), L.ptr(status), U.shape[0],
                                            1 if fallback else 0, C.byref(st), stream), "GetPhysValueStabStats")
    return st


def GetConvValueStab(W, U, eos: int = EOS_IDEAL, gamma: float = 5.0 / 3.0, stream=None):
    """Batched prim->cons on device tensors [n,5] (rhllc_flux_stab.cpp:10-38)."""
    L.check(L.lib.rrhd_prim2con_batch(eos, gamma, L.ptr(W), L.ptr(U), W.shape[0], stream), "GetConvValueStab")
