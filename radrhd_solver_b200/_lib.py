"""ctypes binding of librrhd.so (the C ABI declared in include/rrhd.h).

There is no fallback: if the CUDA library is missing the import fails with
an error that names the build command.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librrhd.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: build it with `python -m radrhd_solver_b200.build` "
                      "(or __graft_entry__.build())")

lib = C.CDLL(LIB_PATH)

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
U64 = C.c_uint64
D = C.c_double

RRHD_OK = 0
RRHD_ERR_INVALID = 1
RRHD_ERR_CUDA = 2
RRHD_ERR_OOM = 3
RRHD_ERR_C2P = 4
RRHD_ERR_STATE = 5
RRHD_ERR_LIMIT = 6
RRHD_HOST = 0
RRHD_DEVICE = 1
RRHD_EOS_IDEAL = 1
RRHD_EOS_TAUB = 2
RRHD_BC_TRANSMISSIVE = 0
RRHD_BC_FIXED = 1
RRHD_BC_REFLECT = 2
RRHD_TC_BF16X3 = 0
RRHD_TC_F16X3 = 1
RRHD_TC_F16 = 2
RRHD_TC_BF16 = 3
STATUS_FALLBACK = 0x10
STATUS_FAILED = 0x20


class MeshDesc(C.Structure):
    _fields_ = [("n_cells", I64), ("n_faces", I64), ("face_id_l", P), ("face_id_r", P), ("face_n", P),
                ("face_area", P), ("cell_faces", P), ("cell_sign", P), ("cell_volume", P),
                ("cell_center", P)]


class Opts(C.Structure):
    _fields_ = [("eos", I32), ("gamma", D), ("device", I32), ("cells_per_block", I32), ("renumber", I32)]


class StepStats(C.Structure):
    _fields_ = [("max_speed", D), ("n_fallback", I64), ("n_failed", I64)]


class C2pStats(C.Structure):
    _fields_ = [("n_ok", I64), ("n_fallback", I64), ("n_failed", I64), ("newton_iters", I64), ("max_iters", I32)]


class KuhnParams(C.Structure):
    _fields_ = [("nx", I32), ("ny", I32), ("nz", I32), ("lo", D * 3), ("hi", D * 3), ("jitter", D),
                ("seed", U64), ("bc_code", I32 * 6), ("inflow_radius", D), ("inflow_code", I32)]


class Emission(C.Structure):
    _fields_ = [("temp_coef", D), ("sigma_sb", D), ("pi", D), ("rad_unit", D)]


RRHD_RAD_FP64 = 0
RRHD_RAD_FP32 = 1
RRHD_RAD_MIXED = 2
RRHD_SCATTER_FP64 = -1
RRHD_SCATTER_LOWRANK = -2
RRHD_RAD_I = 0
RRHD_RAD_S = 1
RRHD_RAD_G4 = 2
RRHD_RAD_MOM = 3


class RadOpts(C.Structure):
    _fields_ = [("groups", I32), ("precision", I32), ("dirs_per_batch", I32), ("boundary_value", D),
                ("item_geometry", I32)]


class CoupledOpts(C.Structure):
    _fields_ = [("scatter", I32), ("guess", P), ("k_stall", I32), ("absorption", D), ("scattering", D),
                ("emission", Emission)]


_SIGS = {
    "rrhd_create": (I32, [P, P, P]),
    "rrhd_destroy": (I32, [P]),
    "rrhd_stream": (P, [P]),
    "rrhd_sync": (I32, [P]),
    "rrhd_set_boundary": (I32, [P, I32, I32, P]),
    "rrhd_set_state": (I32, [P, P, P, I64, I32]),
    "rrhd_get_state": (I32, [P, P, P, I64, I32]),
    "rrhd_set_state_prim": (I32, [P, P, I64, I32]),
    "rrhd_hydro_step": (I32, [P, D, P]),
    "rrhd_set_time_step": (I32, [P, D, D, D]),
    "rrhd_get_step_info": (I32, [P, P, P]),
    "rrhd_hydro_step_host": (I32, [P, D, P, P, I64, P]),
    "rrhd_keep_face_flux": (I32, [P, I32]),
    "rrhd_get_face_flux": (I32, [P, P]),
    "rrhd_get_cell_status": (I32, [P, P]),
    "rrhd_cell_order": (I32, [P, I32, P]),
    "rrhd_part_plan": (I32, [P, P, I32, I32, I32, P, P, P, P, P]),
    "rrhd_hydro_set_part": (I32, [P, I32, I32]),
    "rrhd_hydro_part_info": (I32, [P, P, P, P, P]),
    "rrhd_hydro_layout_info": (I32, [P, P, P, P, P]),
    "rrhd_hydro_pack_halo": (I32, [P, P]),
    "rrhd_hydro_unpack_halo": (I32, [P, P]),
    "rrhd_hydro_max_speed_ptr": (I32, [P, P]),
    "rrhd_con2prim_batch": (I32, [I32, D, P, P, P, I64, I32, P]),
    "rrhd_prim2con_batch": (I32, [I32, D, P, P, I64, P]),
    "rrhd_con2prim_batch_stats": (I32, [I32, D, P, P, P, I64, I32, P, P]),
    "rrhd_dirs_create": (I32, [I32, P, P, D, I32, P]),
    "rrhd_dirs_destroy": (I32, [P]),
    "rrhd_dirs_count": (I32, [P]),
    "rrhd_dirs_device_kernel": (P, [P]),
    "rrhd_scatter_fp64": (I32, [P, P, P, I64, P]),
    "rrhd_scatter_fp64_fma": (I32, [P, P, P, I64, P]),
    "rrhd_moments_fp64": (I32, [P, P, P, P, P, I64, P]),
    "rrhd_scatter_tc_create": (I32, [P, I32, P]),
    "rrhd_scatter_tc_destroy": (I32, [P]),
    "rrhd_scatter_tc_run": (I32, [P, P, P, P, I64, P]),
    "rrhd_scatter_tc_check": (I32, [P, P, I32]),
    "rrhd_emission_reference": (Emission, []),
    "rrhd_rad_source": (I32, [P, P, P, P, P, P, P, P, I64, P]),
    "rrhd_last_error": (C.c_char_p, []),
    "rrhd_version": (C.c_char_p, []),
    "rrhd_mesh_kuhn_sizes": (I32, [P, P, P, P]),
    "rrhd_mesh_kuhn_build": (I32, [P, P, P, P, P, P, P, P, P, P, P, P]),
    "rrhd_directions_fibonacci": (I32, [I32, P, P, P]),
    "rrhd_rng_u01": (D, [U64, U64, U64]),
    "rrhd_fill_intensity_f32": (I32, [P, I64, I32, I32, I32, D, P, U64, P]),
    "rrhd_fill_intensity_f64": (I32, [P, I64, I32, I32, I32, D, P, U64, P]),
    "rrhd_fill_c2p_states": (I32, [P, I64, U64, P]),
    "rrhd_mlp_num_params": (I32, []),
    "rrhd_mlp_create": (I32, [I32, U64, P]),
    "rrhd_mlp_destroy": (I32, [P]),
    "rrhd_mlp_set": (I32, [P, P, P]),
    "rrhd_mlp_get": (I32, [P, P, P]),
    "rrhd_mlp_train": (I32, [P, P, P, I64, I32, I32, C.c_float, U64, I32, P, P]),
    "rrhd_mlp_gradient": (I32, [P, P, P, I64, P, P]),
    "rrhd_con2prim_batch_mlp": (I32, [P, I32, D, P, P, P, I64, I32, I32, P, P, P, P]),
    "rrhd_rad_setup": (I32, [P, P, P]),
    "rrhd_rad_plan_info": (I32, [P, P, P]),
    "rrhd_rad_plan_levels": (I32, [P, P]),
    "rrhd_sweep": (I32, [P, P, P, P, P, P]),
    "rrhd_coupled_step": (I32, [P, D, P, P, P]),
    "rrhd_rad_get": (I32, [P, I32, P]),
    "rrhd_rad_set": (I32, [P, I32, P]),
    "rrhd_coupled_scatter_error": (I32, [P, I64, P, P, P]),
    "rrhd_rad_opacities": (I32, [P, P, I64, I64, D, D, I32, P, P, P, P]),
    "rrhd_rad_source_rows": (I32, [P, P, I64, I64, D, D, I32, P, P, P, P, P]),
    "rrhd_rad_source_con2prim": (I32, [I32, D, P, P, I64, P, D, I64, P, P]),
    "rrhd_coupled_phase_ms": (I32, [P, P]),
    "rrhd_scatter_fp64_cdg": (I32, [P, P, P, I64, I32, I32, P]),
    "rrhd_moments_fp64_cdg": (I32, [P, P, P, P, P, I64, I32, P]),
    "rrhd_scatter_tc_run_cdg": (I32, [P, P, P, P, I64, I32, P]),
    "rrhd_scatter_lowrank": (I32, [P, P, P, P, I64, I32, I32, P]),
    "rrhd_scatter_lowrank_error": (I32, [P, P, P, I64, I32, P, P, P]),
    "rrhd_compton_full_spectrum": (I32, [P, P, P, P, I64, I32, I32, I32, P]),
    "rrhd_compton_spectrum": (I32, [P, P, P, P, I64, D, I32, I32, I32, P]),
    "rrhd_ray_surface_create": (I32, [P, I64, I32, P]),
    "rrhd_ray_surface_destroy": (I32, [P]),
    "rrhd_ray_trace": (I32, [P, P, I64, I32, P, P]),
    "rrhd_ray_make_rays": (I32, [I32, P]),
    "rrhd_ray_image": (I32, [P, I64, P, I32, D, P, P, P, P]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def optional(name: str, restype, argtypes):
    """Binds an entry point that only some builds export (None if absent)."""
    f = getattr(lib, name, None)
    if f is not None:
        f.restype = restype
        f.argtypes = argtypes
    return f


class RrhdError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = lib.rrhd_last_error().decode(errors="replace")
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def check(status: int, where: str = "rrhd") -> int:
    if status != RRHD_OK:
        raise RrhdError(status, where)
    return status


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (None passes through)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def exported_symbols() -> list[str]:
    return sorted(_SIGS)
