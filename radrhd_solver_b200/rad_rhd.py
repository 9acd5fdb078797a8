"""Radiation-hydro coupling, mirroring the reference's `rad_rhd` namespace."""
from __future__ import annotations

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
