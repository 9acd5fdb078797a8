"""Radiation-hydro coupling, mirroring the reference's `rad_rhd` namespace.

    sw = illum.TransportSweep(grid, dg, groups=4, precision="fp64")
    step = RadRHDStep(sw, absorption=1.0, scattering=0.5, em=emission(1, 1))
    step(tau)                                      # one pass of radRHD_main.cpp:96-139
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def reference_emission() -> L.Emission:
    """The reference's compiled-in CGS emission constants (GetTemperature's gas
    constant, Stefan-Boltzmann, pi, kRadiation; lib/global_consts.h)."""
    return L.lib.rrhd_emission_reference()


def emission(temp_coef: float, sigma_sb: float, pi: float = 3.141592653589793, rad_unit: float = 1.0):
    return L.Emission(temp_coef, sigma_sb, pi, rad_unit)


def GetRadSource(W, alpha, sigma, E, F, T, em=None, G=None, stream=None):
    """Radiation 4-force per cell (solvers/RadRHD/src/radRHD_utils.cpp:44-101).
    All arguments are CUDA float64 tensors: W [n,5], alpha/sigma/E [n], F [n,3],
    T [n,3,3]; returns G [n,4]."""
    import torch
    n = W.shape[0]
    if em is None:
        em = reference_emission()
    if G is None:
        G = torch.empty(n, 4, dtype=torch.float64, device=W.device)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    L.check(L.lib.rrhd_rad_source(C_ref(em), L.ptr(W), L.ptr(alpha), L.ptr(sigma), L.ptr(E), L.ptr(F), L.ptr(T),
                                  L.ptr(G), n, stream), "GetRadSource")
    return G


def C_ref(em):
    import ctypes
    return ctypes.byref(em)


class RadRHDStep:
    """The coupled step of solvers/RadRHD/src/radRHD_main.cpp:96-139 on the Grid
    of a TransportSweep.  scatter: "fp64" (plain form, needs an fp64 sweep), "lowrank"
    (the rank-7 Thomson identity, either sweep precision) or a tensor-core form
    "bf16x3" / "f16x3" / "f16" / "bf16" (fp32 sweep); guess: a
    LearnedGuess for the source con2prim, or None for the reference guess."""

    FORMS = {"fp64": L.RRHD_SCATTER_FP64, "lowrank": L.RRHD_SCATTER_LOWRANK, "bf16x3": L.RRHD_TC_BF16X3,
             "f16x3": L.RRHD_TC_F16X3, "f16": L.RRHD_TC_F16, "bf16": L.RRHD_TC_BF16}

    def __init__(self, sweep, absorption: float = 1.0, scattering: float = 0.5, em=None, scatter: str = "fp64",
                 guess=None, k_stall: int = 0):
        self.sweep = sweep
        self.grid = sweep.grid
        self.guess = guess
        em = em if em is not None else emission(1.0, 1.0)
        self.opts = L.CoupledOpts(self.FORMS[scatter], guess.handle.value if guess is not None else None, k_stall,
                                  absorption, scattering, em)

    def __call__(self, tau: float, stats: bool = False):
        """One coupled step; with stats=True returns (hydro StepStats, source C2pStats).
        Cells where the hydro con2prim failed even after PhysPressureFix are
        counted in the hydro statistics (the step itself completes)."""
        if not stats:
            st = L.lib.rrhd_coupled_step(self.grid.handle, tau, C.byref(self.opts), None, None)
            if st != L.RRHD_ERR_C2P:
                L.check(st, "coupled step")
            return None
        hs, ss = L.StepStats(), L.C2pStats()
        st = L.lib.rrhd_coupled_step(self.grid.handle, tau, C.byref(self.opts), C.byref(hs), C.byref(ss))
        if st != L.RRHD_ERR_C2P:
            L.check(st, "coupled step")
        return hs, ss

    def phase_ms(self):
        """Device ms of the last step's phases: hydro, sweep, source, scattering."""
        ms = (C.c_float * 4)()
        L.check(L.lib.rrhd_coupled_phase_ms(self.grid.handle, ms), "rrhd_coupled_phase_ms")
        return dict(zip(("hydro", "sweep", "source_c2p", "scatter_moments"), list(ms)))

    _KEYS = {"I": L.RRHD_RAD_I, "S": L.RRHD_RAD_S, "G4": L.RRHD_RAD_G4, "MOM": L.RRHD_RAD_MOM}

    def get(self, what: str):
        """Host copy, caller numbering: "I" / "S" [N*G, M], "G4" [N, 4], "MOM" [N*G, 10]
        (E, F0..2, T00, T01, T02, T11, T12, T22 of the last scattering)."""
        n = self.grid.size
        shape = {"G4": (n, 4), "MOM": (n * self.sweep.groups, 10)}.get(what, (n * self.sweep.groups,
                                                                              self.sweep.dg.size))
        out = np.zeros(shape)
        L.check(L.lib.rrhd_rad_get(self.grid.handle, self._KEYS[what], L.ptr(out)), "rrhd_rad_get")
        return out

    def scatter_error(self, sample_cells: int = 65536):
        """Accuracy of this step's reduced-precision scattering (rrhd_coupled_scatter_error):
        (max, rms) relative error of S against FP64 from the same FP32 intensity, and the
        largest moment error (F, T relative to E), on a sample of cells."""
        mx, rms, mm = C.c_double(), C.c_double(), C.c_double()
        L.check(L.lib.rrhd_coupled_scatter_error(self.grid.handle, sample_cells, C.byref(mx), C.byref(rms),
                                                 C.byref(mm)), "rrhd_coupled_scatter_error")
        return mx.value, rms.value, mm.value

    def set(self, what: str, values):
        """Writes "I" or "S" [N*G, M] (caller numbering)."""
        assert what in ("I", "S")
        v = np.ascontiguousarray(values, np.float64)
        assert v.shape == (self.grid.size * self.sweep.groups, self.sweep.dg.size)
        L.check(L.lib.rrhd_rad_set(self.grid.handle, self._KEYS[what], L.ptr(v)), "rrhd_rad_set")
