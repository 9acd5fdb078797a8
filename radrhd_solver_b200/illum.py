"""Radiation scattering integral and moments, mirroring the reference's
`illum` / `cuda::interface::separate_device` calls.

    dg = DirectionGrid(fibonacci_directions(256))          # InitDevice (directions)
    S = CalculateIntScattering(dg, I)                      # GetS_MPI_multi_device
    E, F, T = CalculateAllParam(dg, I)                     # MakeIllumParam
    S, mom = ScatteringLowRank(dg, I)                      # both through the rank-7 Thomson identity
    sw = TransportSweep(grid, dg, groups=1)                # sweep plan (graph/ + make_trace/)
    CalculateIllum(sw, alpha, betta, Q, S, I)              # one sweep of separate_gpu::CalculateIllum

I is a CUDA tensor [rows, M] with rows = cells x groups (cell-major, the
layout of grid.Illum, solvers/illum/src/illum_utils.cpp:362).
"""
from __future__ import annotations

import ctypes as C

from . import _lib as L
from .mesh import Directions


class DirectionGrid:
    def __init__(self, d: Directions, device: int = 0):
        self.directions = d
        self.size = d.size
        self.full_area = d.full_area
        h = C.c_void_p()
        L.check(L.lib.rrhd_dirs_create(d.size, L.ptr(d.dirs), L.ptr(d.areas), d.full_area, device, C.byref(h)),
                "rrhd_dirs_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            L.lib.rrhd_dirs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream(stream):
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return stream


def CalculateIntScattering(dg: DirectionGrid, I, S=None, exact: bool = True, stream=None):
    """FP64 scattering integral (cuda/src/short_characteristics/cuda_scattering.cu:82-105).
    exact=True: the reference's rounding sequence; exact=False: one FMA per term."""
    import torch
    if S is None:
        S = torch.empty_like(I)
    fn = L.lib.rrhd_scatter_fp64 if exact else L.lib.rrhd_scatter_fp64_fma
    L.check(fn(dg.handle, L.ptr(I), L.ptr(S), I.shape[0], _stream(stream)), "CalculateIntScattering")
    return S


def CalculateAllParam(dg: DirectionGrid, I, stream=None):
    """Energy/stream/impulse moments (separate_gpu/cuda_illum_sep_param.cu:9-83)."""
    import torch
    rows = I.shape[0]
    E = torch.empty(rows, dtype=torch.float64, device=I.device)
    F = torch.empty(rows, 3, dtype=torch.float64, device=I.device)
    T = torch.empty(rows, 3, 3, dtype=torch.float64, device=I.device)
    L.check(L.lib.rrhd_moments_fp64(dg.handle, L.ptr(I), L.ptr(E), L.ptr(F), L.ptr(T), rows, _stream(stream)),
            "CalculateAllParam")
    return E, F, T


TC_FORMS = {"bf16x3": L.RRHD_TC_BF16X3, "f16x3": L.RRHD_TC_F16X3, "f16": L.RRHD_TC_F16, "bf16": L.RRHD_TC_BF16}


def ScatteringLowRank(dg: DirectionGrid, I, S=None, moments: bool = True, groups: int = 1, stream=None):
    """Scattering integral and moments through the rank-7 structure of the Thomson
    phase function, S = 3/4 (E + w^T T w), FP64 arithmetic (no counterpart in the
    reference, which sums the O(M^2) form).  I: CUDA float64 or float32 tensor
    [rows, M] (groups = 1) or [cells, M, groups] (groups 2 or 4).  Returns S and the
    [rows, 16] moments {E, F, Txx, Txy, Txz, Tyy, Tyz, Tzz, 0...} in I's dtype."""
    import torch
    assert I.is_cuda and I.is_contiguous() and I.dtype in (torch.float64, torch.float32)
    if S is None:
        S = torch.empty_like(I)
    cells = I.shape[0]
    rows = cells * groups
    mom = torch.empty(rows, 16, dtype=I.dtype, device=I.device) if moments else None
    prec = L.RRHD_RAD_FP64 if I.dtype == torch.float64 else L.RRHD_RAD_FP32
    L.check(L.lib.rrhd_scatter_lowrank(dg.handle, I.data_ptr(), S.data_ptr(), mom.data_ptr() if moments else None,
                                       cells, groups, prec, _stream(stream)), "rrhd_scatter_lowrank")
    return S, mom


def LowRankError(dg: DirectionGrid, I, S_test, groups: int = 1, stream=None):
    """(max, rms) relative error of an FP32 scattering integral against the FP64
    low-rank values, over every row and direction."""
    mx, rms = C.c_double(), C.c_double()
    L.check(L.lib.rrhd_scatter_lowrank_error(dg.handle, I.data_ptr(), S_test.data_ptr(), I.shape[0], groups,
                                             C.byref(mx), C.byref(rms), _stream(stream)), "rrhd_scatter_lowrank_error")
    return mx.value, rms.value


N_FRQ = 100  # spectrum bins of the full-spectrum Compton scattering


def FullSpectrumScattering(dg: DirectionGrid, I, velocity, S=None, dir_disp: int = 0, dir_count: int | None = None,
                           out_stride: int | None = None, stream=None):
    """Frequency-coupled Compton scattering integral over the 100-bin spectrum, the
    reference's CalculateFullSpectrumIntScattering / Get_full_spectrum_multi_device
    (cuda_interface_spectrum.cu:94-140, cuda_scat_full_spectrum.cu:61-118).
    I: CUDA float64 [cells, M, 100]; velocity: CUDA float64 [cells, 3] in units of c.
    Returns S [cells, out_stride, 100] for the output directions dir_disp ..
    dir_disp + dir_count - 1 (all M by default)."""
    import torch
    assert I.is_cuda and I.is_contiguous() and I.dtype == torch.float64 and I.shape[1:] == (dg.size, N_FRQ)
    assert velocity.is_contiguous() and velocity.dtype == torch.float64 and velocity.shape == (I.shape[0], 3)
    dir_count = dg.size - dir_disp if dir_count is None else dir_count
    out_stride = dir_count if out_stride is None else out_stride
    if S is None:
        S = torch.empty(I.shape[0], out_stride, N_FRQ, dtype=torch.float64, device=I.device)
    L.check(L.lib.rrhd_compton_full_spectrum(dg.handle, I.data_ptr(), velocity.data_ptr(), S.data_ptr(), I.shape[0],
                                             dir_disp, dir_count, out_stride, _stream(stream)),
            "rrhd_compton_full_spectrum")
    return S


def SpectrumScattering(dg: DirectionGrid, I, velocity, frq: float, S=None, dir_disp: int = 0,
                       dir_count: int | None = None, out_stride: int | None = None, stream=None):
    """Compton-shifted scattering integral at one frequency frq (Hz), the reference's
    CalculateSpectrumIntScattering / Get_spectrum_multi_device (cuda_interface_spectrum.cu:46-92,
    cuda_scat_spectrum.cu:41-83).  I: CUDA float64 [cells, M] at frq; velocity: CUDA
    float64 [cells, 3] in units of c.  Returns S [cells, out_stride]."""
    import torch
    assert I.is_cuda and I.is_contiguous() and I.dtype == torch.float64 and I.shape[1] == dg.size
    assert velocity.is_contiguous() and velocity.dtype == torch.float64 and velocity.shape == (I.shape[0], 3)
    dir_count = dg.size - dir_disp if dir_count is None else dir_count
    out_stride = dir_count if out_stride is None else out_stride
    if S is None:
        S = torch.empty(I.shape[0], out_stride, dtype=torch.float64, device=I.device)
    L.check(L.lib.rrhd_compton_spectrum(dg.handle, I.data_ptr(), velocity.data_ptr(), S.data_ptr(), I.shape[0], frq,
                                        dir_disp, dir_count, out_stride, _stream(stream)), "rrhd_compton_spectrum")
    return S


class ScatterTC:
    """Tensor-core (tcgen05) scattering integral + moments for one direction set
    and precision form ("bf16x3", "f16x3", "f16", "bf16"); FP32 in/out."""

    def __init__(self, dg: DirectionGrid, form: str = "f16x3"):
        self.dg = dg
        self.form = form
        h = C.c_void_p()
        L.check(L.lib.rrhd_scatter_tc_create(dg.handle, TC_FORMS[form], C.byref(h)), "rrhd_scatter_tc_create")
        self._h = h

    def __call__(self, I, S=None, moments=True, stream=None):
        import torch
        rows = I.shape[0]
        if S is None:
            S = torch.empty_like(I)
        mom = torch.empty(rows, 16, dtype=torch.float32, device=I.device) if moments else None
        L.check(L.lib.rrhd_scatter_tc_run(self._h, L.ptr(I), L.ptr(S), L.ptr(mom), rows, _stream(stream)),
                "rrhd_scatter_tc_run")
        return S, mom

    def check(self, clear=True, stream=None):
        L.check(L.lib.rrhd_scatter_tc_check(self._h, _stream(stream), 1 if clear else 0), "rrhd_scatter_tc_check")

    def close(self):
        if self._h:
            L.lib.rrhd_scatter_tc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def moments_from_tc(mom):
    """Expands the 16-column moment block to E [n], F [n,3], T [n,3,3] (float64)."""
    import torch
    m = mom.to(torch.float64)
    E = m[:, 0].clone()
    F = m[:, 1:4].clone()
    T = torch.stack([m[:, 4], m[:, 5], m[:, 6], m[:, 5], m[:, 7], m[:, 8], m[:, 6], m[:, 8], m[:, 9]], 1).view(-1, 3, 3)
    return E, F, T


class TransportSweep:
    """Device sweep plan for a hydro Grid's mesh and a DirectionGrid: the
    upwind order the reference reads from its offline graph/ and make_trace/
    outputs (sorted_graph, vec_x0), built on the GPU as levels.  precision:
    "fp64" or "fp32" (storage and arithmetic of alpha, betta, Q, S, I), or "mixed"
    (float arrays as "fp32", face values and the transport update in double).
    item_geometry ("fp32" and "mixed"): precompute every (cell, direction) item's
    in/out faces, node choices and in-face distances (float) at setup, 16 bytes per
    item, and stream them in sweep order instead of reading each cell's geometry per
    item."""

    def __init__(self, grid, dg: DirectionGrid, groups: int = 1, precision: str = "fp64", dirs_per_batch: int = 0,
                 boundary_value: float = 0.0, item_geometry: bool = False):
        prec = {"fp64": L.RRHD_RAD_FP64, "fp32": L.RRHD_RAD_FP32, "mixed": L.RRHD_RAD_MIXED}[precision]
        o = L.RadOpts(groups, prec, dirs_per_batch, boundary_value, int(item_geometry))
        L.check(L.lib.rrhd_rad_setup(grid.handle, dg.handle, C.byref(o)), "rrhd_rad_setup")
        self.grid, self.dg, self.groups, self.precision = grid, dg, groups, precision
        self.item_geometry = bool(item_geometry)

    def plan_levels(self):
        """[M, N] (caller numbering): the level in which each (cell, direction) is swept,
        the front index the reference's graph::RunGraphModule gives it."""
        import numpy as np
        out = np.zeros((self.dg.size, self.grid.size), np.int32)
        L.check(L.lib.rrhd_rad_plan_levels(self.grid.handle, L.ptr(out)), "rrhd_rad_plan_levels")
        return out

    def plan_info(self):
        lv, mx = C.c_int64(), C.c_int64()
        L.check(L.lib.rrhd_rad_plan_info(self.grid.handle, C.byref(lv), C.byref(mx)), "rrhd_rad_plan_info")
        return lv.value, mx.value


def CalculateIllum(sw: TransportSweep, alpha, betta, Q, S, I=None):
    """One sweep of all directions and groups (the direction loop of
    solvers/illum/src/mpi/multi_gpu/illum_multi_gpu_face_calc.cpp:91-190) on the
    grid's stream.  CUDA tensors, double for "fp64" and float otherwise, caller cell
    numbering: alpha, betta [N], Q [N, G], S [N*G, M]; returns I [N*G, M]."""
    import torch
    if I is None:
        I = torch.empty_like(S)
    dt = torch.float64 if sw.precision == "fp64" else torch.float32
    for t in (alpha, betta, Q, S, I):
        assert t.is_contiguous() and t.dtype == dt
    L.check(L.lib.rrhd_sweep(sw.grid.handle, L.ptr(alpha), L.ptr(betta), L.ptr(Q), L.ptr(S), L.ptr(I)),
            "CalculateIllum")
    return I
