"""ctypes wrappers of the oracle libraries (test infrastructure)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "librrhd_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double

_port = None
_refs: dict[str, C.CDLL] = {}


def _p(a):
    return None if a is None else a.ctypes.data


def build_port() -> str:
    if not os.path.exists(PORT_SO) or os.path.getmtime(PORT_SO) < os.path.getmtime(os.path.join(HERE, "rrhd_oracle.c")):
        subprocess.run(["make", "-C", HERE, "port"], check=True, capture_output=True)
    return PORT_SO


class OrcEos(C.Structure):
    _fields_ = [("eos", I32), ("gamma1", D)]


class OrcMesh(C.Structure):
    _fields_ = [("n_cells", I64), ("n_faces", I64), ("face_id_l", P), ("face_id_r", P), ("face_n", P),
                ("face_area", P), ("cell_faces", P), ("cell_sign", P), ("cell_volume", P), ("cell_center", P)]


class OrcBc(C.Structure):
    _fields_ = [("kind", I32 * 8), ("W", (D * 5) * 8), ("U", (D * 5) * 8)]


class OrcSweepMesh(C.Structure):
    _fields_ = [("n_cells", I64), ("n_faces", I64), ("cell_volume", P), ("cell_faces", P), ("cell_nbr", P),
                ("cell_sign", P), ("face_n", P), ("face_area", P)]


class OrcEmission(C.Structure):
    _fields_ = [("temp_coef", D), ("sigma_sb", D), ("pi", D), ("rad_unit", D)]


def port() -> C.CDLL:
    global _port
    if _port is None:
        lib = C.CDLL(build_port())
        sig = {
            "orc_p2c": (None, [P, P, P]), "orc_p2c_plain": (None, [P, P, P]), "orc_c2p": (I32, [P, P, P]),
            "orc_pressure_fix": (I32, [P, P, P]), "orc_rotation": (None, [P, P]),
            "orc_flux": (D, [P, P, P, P, P, P, D, P]),
            "orc_hydro_step": (D, [P, P, P, D, P, P, P, P, C.c_int]),
            "orc_time_step": (D, [D, D, D]),
            "orc_scatter": (None, [I64, I32, P, P, P, D, P, C.c_int]),
            "orc_moments": (None, [I64, I32, P, P, P, D, P, P, P, C.c_int]),
            "orc_rad_source": (None, [I64, P, P, P, P, P, P, P, P]),
            "orc_get_illum": (D, [P, P, D, D]), "orc_get_rhs": (D, [D, D, D, D, P]),
            "orc_recalc_illum": (D, [I64, P, P, P, I32, I32, P]),
            "orc_sweep": (I64, [P, I32, P, I32, P, P, P, P, D, P]),
            "orc_trace_nodes": (None, [P, I32, P, P, P]),
            "orc_compton_full_spectrum": (None, [I32, P, P, D, I64, P, P, I32, I32, I32, P, C.c_int]),
            "orc_compton_frq": (D, [I32]), "orc_compton_frq_idx": (I32, [D]),
            "orc_compton_spectrum": (None, [I32, P, P, D, I64, P, P, D, I32, I32, I32, P, C.c_int]),
            "orc_ray_triangle": (D, [P, P]), "orc_ray_roche": (I32, [P, P]), "orc_ray_sphere_disk": (I32, [P]),
            "orc_ray_trace": (None, [I32, P, I64, P, P, I64, P, C.c_int]), "orc_ray_make_rays": (None, [I32, P]),
        }
        for n, (r, a) in sig.items():
            f = getattr(lib, n)
            f.restype = r
            f.argtypes = a
        _port = lib
    return _port


def have_ref(variant: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"librrhd_ref_{variant}.so"))


def ref(variant: str) -> C.CDLL | None:
    if variant in _refs:
        return _refs[variant]
    path = os.path.join(REF_DIR, f"librrhd_ref_{variant}.so")
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    sig = {
        "ref_kgamma1": (D, []), "ref_c2p": (None, [P, P, P, I64]), "ref_pressure_fix": (None, [P, P, P, I64]),
        "ref_p2c": (None, [P, P, I64]), "ref_p2c_plain": (None, [P, P, I64]),
        "ref_flux": (None, [P, P, P, P, P, P, P, P, I64]),
        "ref_hydro_create": (P, [I64, I64, P, P, P, P, P, P, P, P]), "ref_hydro_destroy": (None, [P]),
        "ref_hydro_set_bc": (None, [P, I32, I32, P, P]), "ref_hydro_set_state": (None, [P, P, P]),
        "ref_hydro_get_state": (None, [P, P, P]), "ref_hydro_get_face_flux": (None, [P, P]),
        "ref_hydro_step": (D, [P, D, C.c_int]), "ref_hydro_step_bc": (D, [P, D, C.c_int, P]),
        "ref_time_step": (D, [D, D, D]),
        "ref_scatter": (None, [I64, I32, P, P, P, D, P, C.c_int]),
        "ref_moments": (None, [I64, I32, P, P, P, D, P, P, P, C.c_int]),
        "ref_rad_source": (None, [I64, P, P, P, P, P, P, P]), "ref_rad_constants": (None, [P]),
        "ref_eos": (C.c_int, []),
        "ref_get_illum": (D, [P, P, D, D]), "ref_get_rhs": (D, [D, D, D, D, P]),
        "ref_recalc_illum": (D, [I64, I64, P, P, P, I32, I32, P]),
        "ref_write_solution": (C.c_int, [P, C.c_char_p]), "ref_write_geo": (C.c_int, [P, C.c_char_p, C.c_char_p]),
        "ref_read_geo": (I64, [C.c_char_p, C.c_char_p, P, P, P, P, P, P, P, P, P]),
        "ref_read_hllc_init": (I64, [C.c_char_p, P]), "ref_record_sizes": (C.c_int, [P]),
        "ref_read_sphere_directions": (I64, [C.c_char_p, P, P, P]),
        "ref_compton_full_spectrum": (C.c_int, [I32, P, P, D, I64, P, P, I32, I32, I32, P, C.c_int]),
        "ref_compton_n_frq": (C.c_int, []), "ref_compton_get_frq": (D, [C.c_int]),
        "ref_compton_get_frq_idx": (C.c_int, [D]), "ref_compton_gamma": (D, [D, D, P, D, D, P, P, P]),
        "ref_compton_spectrum": (C.c_int, [I32, P, P, D, I64, P, P, D, I32, I32, I32, P, C.c_int]),
        "ref_ray_trace": (C.c_int, [I32, P, I32, P, P, I32, P, C.c_int]), "ref_ray_triangle": (D, [P, P]),
        "ref_ray_roche": (C.c_int, [P, P]), "ref_ray_make_rays": (C.c_int, [C.c_int, P]),
    }
    for n, (r, a) in sig.items():
        f = getattr(lib, n, None)
        if f is not None:
            f.restype = r
            f.argtypes = a
    _refs[variant] = lib
    return lib


def ref_variant_for(eos: int, gamma: float, fast: bool = False) -> str:
    if eos == 2:
        return "hydro_taub"
    if abs(gamma - 5.0 / 3.0) < 1e-15:
        v = "hydro_ideal_5_3"
    elif abs(gamma - 4.0 / 3.0) < 1e-15:
        v = "hydro_ideal_4_3"
    else:
        raise ValueError("the reference is compiled for Gamma = 5/3 and 4/3 only")
    return v + ("_fast" if fast else "")


def _eos(eos, gamma):
    return OrcEos(eos, gamma)


def _mesh(m) -> OrcMesh:
    return OrcMesh(m.n_cells, m.n_faces, _p(m.face_id_l), _p(m.face_id_r), _p(m.face_n), _p(m.face_area),
                   _p(m.cell_faces), _p(m.cell_sign), _p(m.cell_volume), _p(m.cell_center))


def _bc(table) -> OrcBc:
    """table: {code: (kind, W5, U5)}"""
    b = OrcBc()
    for k in range(8):
        b.kind[k] = 0
    for code, (kind, W, U) in (table or {}).items():
        k = -code - 1
        b.kind[k] = kind
        for i in range(5):
            b.W[k][i] = W[i] if W is not None else 0.0
            b.U[k][i] = U[i] if U is not None else 0.0
    return b


# ------------------------------------------------------------------ port
def port_c2p(U, eos=1, gamma=5.0 / 3.0, W=None):
    U = np.ascontiguousarray(U, np.float64)
    W = np.zeros_like(U) if W is None else np.array(W, np.float64)
    codes = np.zeros(len(U), np.int32)
    e = _eos(eos, gamma)
    lib = port()
    for i in range(len(U)):
        codes[i] = lib.orc_c2p(C.byref(e), U[i].ctypes.data, W[i].ctypes.data)
    return W, codes


def port_pressure_fix(U, W, eos=1, gamma=5.0 / 3.0):
    U = np.array(U, np.float64)
    W = np.array(W, np.float64)
    codes = np.zeros(len(U), np.int32)
    e = _eos(eos, gamma)
    lib = port()
    for i in range(len(U)):
        codes[i] = lib.orc_pressure_fix(C.byref(e), U[i].ctypes.data, W[i].ctypes.data)
    return U, W, codes


def port_p2c(W, eos=1, gamma=5.0 / 3.0):
    W = np.array(W, np.float64)
    U = np.zeros_like(W)
    e = _eos(eos, gamma)
    lib = port()
    for i in range(len(W)):
        lib.orc_p2c(C.byref(e), W[i].ctypes.data, U[i].ctypes.data)
    return W, U


def port_flux(UL, UR, WL, WR, n, S, eos=1, gamma=5.0 / 3.0):
    k = len(UL)
    F = np.zeros((k, 5))
    sp = np.zeros(k)
    e = _eos(eos, gamma)
    lib = port()
    arrs = [np.ascontiguousarray(a, np.float64) for a in (UL, UR, WL, WR, n)]
    for i in range(k):
        sp[i] = lib.orc_flux(C.byref(e), *(a[i].ctypes.data for a in arrs), float(S[i]), F[i].ctypes.data)
    return F, sp


def port_hydro_step(mesh, U, W, tau, eos=1, gamma=5.0 / 3.0, bc=None, nthreads=1):
    """One step of the restated Hllc3dStab; returns (U, W, face_flux, status, max_speed)."""
    U = np.array(U, np.float64)
    W = np.array(W, np.float64)
    Ff = np.zeros((mesh.n_faces, 5))
    st = np.zeros(mesh.n_cells, np.int32)
    m = _mesh(mesh)
    b = _bc(bc)
    e = _eos(eos, gamma)
    v = port().orc_hydro_step(C.byref(e), C.byref(m), C.byref(b), tau, _p(U), _p(W), _p(Ff), _p(st), nthreads)
    return U, W, Ff, st, v


def port_scatter(I, dirs, areas, full_area, nthreads=1):
    I = np.ascontiguousarray(I, np.float64)
    S = np.zeros_like(I)
    port().orc_scatter(I.shape[0], I.shape[1], _p(I), _p(np.ascontiguousarray(dirs)), _p(np.ascontiguousarray(areas)),
                       full_area, _p(S), nthreads)
    return S


def port_moments(I, dirs, areas, full_area, nthreads=1):
    I = np.ascontiguousarray(I, np.float64)
    N = I.shape[0]
    E, F, T = np.zeros(N), np.zeros((N, 3)), np.zeros((N, 3, 3))
    port().orc_moments(N, I.shape[1], _p(I), _p(np.ascontiguousarray(dirs)), _p(np.ascontiguousarray(areas)),
                       full_area, _p(E), _p(F), _p(T), nthreads)
    return E, F, T


def port_rad_source(W, alpha, sigma, E, F, T, emission):
    N = len(W)
    G = np.zeros((N, 4))
    em = OrcEmission(*emission)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (W, alpha, sigma, E, F, T)]
    port().orc_rad_source(N, C.byref(em), *(_p(a) for a in arrs), _p(G))
    return G


# ------------------------------------------------------------------ reference
def ref_c2p(U, variant, W=None):
    lib = ref(variant)
    U = np.ascontiguousarray(U, np.float64)
    W = np.zeros_like(U) if W is None else np.array(W, np.float64)
    codes = np.zeros(len(U), np.int32)
    lib.ref_c2p(_p(U), _p(W), _p(codes), len(U))
    return W, codes


def ref_pressure_fix(U, W, variant):
    lib = ref(variant)
    U = np.array(U, np.float64)
    W = np.array(W, np.float64)
    codes = np.zeros(len(U), np.int32)
    lib.ref_pressure_fix(_p(U), _p(W), _p(codes), len(U))
    return U, W, codes


def ref_p2c(W, variant):
    lib = ref(variant)
    W = np.array(W, np.float64)
    U = np.zeros_like(W)
    lib.ref_p2c(_p(W), _p(U), len(W))
    return W, U


def ref_flux(UL, UR, WL, WR, n, S, variant):
    lib = ref(variant)
    k = len(UL)
    F = np.zeros((k, 5))
    sp = np.zeros(k)
    arrs = [np.ascontiguousarray(a, np.float64) for a in (UL, UR, WL, WR, n, S)]
    lib.ref_flux(*(_p(a) for a in arrs), _p(F), _p(sp), k)
    return F, sp


class HydroRef:
    """The reference grid_t driven through rhllc::Hllc3dStab (or the same loops
    with a fixed-state inflow boundary)."""

    def __init__(self, mesh, variant):
        self.lib = ref(variant)
        if self.lib is None:
            raise FileNotFoundError(f"reference variant {variant} not built")
        self.mesh = mesh
        self.h = self.lib.ref_hydro_create(mesh.n_cells, mesh.n_faces, _p(mesh.face_id_l), _p(mesh.face_id_r),
                                           _p(mesh.face_n), _p(mesh.face_area), _p(mesh.cell_faces),
                                           _p(mesh.cell_sign), _p(mesh.cell_volume), _p(mesh.cell_center))
        self.custom_bc = False

    def set_bc(self, code, kind, W=None, U=None):
        w = None if W is None else np.ascontiguousarray(W, np.float64)
        u = None if U is None else np.ascontiguousarray(U, np.float64)
        self.lib.ref_hydro_set_bc(self.h, code, kind, _p(w), _p(u))
        self.custom_bc = True

    def set_state(self, W, U):
        W = np.ascontiguousarray(W, np.float64)
        U = np.ascontiguousarray(U, np.float64)
        self.lib.ref_hydro_set_state(self.h, _p(W), _p(U))

    def get_state(self):
        W = np.zeros((self.mesh.n_cells, 5))
        U = np.zeros((self.mesh.n_cells, 5))
        self.lib.ref_hydro_get_state(self.h, _p(W), _p(U))
        return W, U

    def face_flux(self):
        F = np.zeros((self.mesh.n_faces, 5))
        self.lib.ref_hydro_get_face_flux(self.h, _p(F))
        return F

    def step(self, tau, nthreads=0, codes=None):
        if self.custom_bc or codes is not None:
            return self.lib.ref_hydro_step_bc(self.h, tau, nthreads, _p(codes))
        return self.lib.ref_hydro_step(self.h, tau, nthreads)

    def write_solution(self, directory):
        """files_sys::bin::WriteSolution (lib/files_sys/src/writer_bin.cpp:56-114)
        on this grid: density.bin, pressure.bin, velocity.bin under `directory`."""
        d = os.path.join(directory, "")
        os.makedirs(d, exist_ok=True)  # the reference's writer opens files only
        return self.lib.ref_write_solution(self.h, d.encode())

    def write_geo(self, faces_file, cells_file):
        """files_sys::bin::WriteGridGeo of the face and cell records (writer_bin.h)."""
        return self.lib.ref_write_geo(self.h, faces_file.encode(), cells_file.encode())

    def close(self):
        if self.h:
            self.lib.ref_hydro_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_read_geo(faces_file, cells_file, variant="hydro_ideal_5_3"):
    """files_sys::bin::ReadGridGeo of both geometry files
    (lib/files_sys/include/reader_bin.h:113-135); returns a dict of the fields."""
    lib = ref(variant)
    nf = C.c_int64()
    n = lib.ref_read_geo(faces_file.encode(), cells_file.encode(), C.byref(nf), *([None] * 8))
    if n == 0:
        raise OSError("ReadGridGeo failed")
    F = nf.value
    out = dict(face_id_l=np.zeros(F, np.int32), face_id_r=np.zeros(F, np.int32), face_n=np.zeros((F, 3)),
               face_area=np.zeros(F), cell_faces=np.zeros((n, 4), np.int32), cell_sign=np.zeros(n, np.uint8),
               cell_volume=np.zeros(n), cell_center=np.zeros((n, 3)))
    lib.ref_read_geo(faces_file.encode(), cells_file.encode(), C.byref(nf), *(_p(out[k]) for k in
                     ("face_id_l", "face_id_r", "face_n", "face_area", "cell_faces", "cell_sign", "cell_volume",
                      "cell_center")))
    return out


def ref_read_hllc_init(path, variant="hydro_ideal_5_3"):
    """files_sys::bin::ReadHllcInit (reader_bin.h:232-251); returns W [n,5]."""
    lib = ref(variant)
    n = lib.ref_read_hllc_init(path.encode(), None)
    if n == 0:
        raise OSError("ReadHllcInit failed")
    W = np.zeros((n, 5))
    lib.ref_read_hllc_init(path.encode(), _p(W))
    return W


def ref_read_sphere_directions(path, variant="hydro_ideal_5_3"):
    """files_sys::txt::ReadSphereDirectionCartesian (reader_txt.cpp:6-37);
    returns (dirs [M,3], areas [M], full_area)."""
    lib = ref(variant)
    M = lib.ref_read_sphere_directions(path.encode(), None, None, None)
    if M < 0:
        raise OSError("ReadSphereDirectionCartesian failed")
    d, a, fa = np.zeros((M, 3)), np.zeros(M), C.c_double()
    lib.ref_read_sphere_directions(path.encode(), _p(d), _p(a), C.byref(fa))
    return d, a, fa.value


def ref_record_sizes(variant="hydro_ideal_5_3"):
    """sizeof(geo_face_t), sizeof(geo_cell_t), sizeof(flux_t) as compiled."""
    out = np.zeros(3, np.int32)
    ref(variant).ref_record_sizes(_p(out))
    return tuple(int(x) for x in out)


def ref_scatter(I, dirs, areas, full_area, nthreads=0):
    lib = ref("illum")
    I = np.ascontiguousarray(I, np.float64)
    S = np.zeros_like(I)
    lib.ref_scatter(I.shape[0], I.shape[1], _p(I), _p(np.ascontiguousarray(dirs)), _p(np.ascontiguousarray(areas)),
                    full_area, _p(S), nthreads)
    return S


def ref_moments(I, dirs, areas, full_area, nthreads=0):
    lib = ref("illum")
    I = np.ascontiguousarray(I, np.float64)
    N = I.shape[0]
    E, F, T = np.zeros(N), np.zeros((N, 3)), np.zeros((N, 3, 3))
    lib.ref_moments(N, I.shape[1], _p(I), _p(np.ascontiguousarray(dirs)), _p(np.ascontiguousarray(areas)), full_area,
                    _p(E), _p(F), _p(T), nthreads)
    return E, F, T


def ref_rad_source(W, alpha, sigma, E, F, T, variant="rad_ideal_4_3"):
    lib = ref(variant)
    N = len(W)
    G = np.zeros((N, 4))
    arrs = [np.ascontiguousarray(a, np.float64) for a in (W, alpha, sigma, E, F, T)]
    lib.ref_rad_source(N, *(_p(a) for a in arrs), _p(G))
    return G


def port_get_illum(I0, s, k, rhs):
    I0 = np.ascontiguousarray(I0, np.float64)
    s = np.ascontiguousarray(s, np.float64)
    return port().orc_get_illum(_p(I0), _p(s), k, rhs)


def port_get_rhs(alpha, betta, Q, S):
    k = C.c_double()
    r = port().orc_get_rhs(alpha, betta, Q, S, C.byref(k))
    return r, k.value


def port_recalc_illum(cell_faces, face_area, face_values, Illum, direction):
    """Rewrites column `direction` of Illum [N][M] in place; returns the norm."""
    cf = np.ascontiguousarray(cell_faces, np.int32)
    fa = np.ascontiguousarray(face_area, np.float64)
    fv = np.ascontiguousarray(face_values, np.float64)
    assert Illum.flags.c_contiguous and Illum.dtype == np.float64
    return port().orc_recalc_illum(len(cf), _p(cf), _p(fa), _p(fv), Illum.shape[1], direction, _p(Illum))


def sweep_neighbours(mesh):
    """[N][4] neighbour across each local face (-1 on the boundary) of a Mesh."""
    cf = np.asarray(mesh.cell_faces)
    l, r = np.asarray(mesh.face_id_l), np.asarray(mesh.face_id_r)
    own = np.arange(len(cf))[:, None]
    nl, nr = l[cf], r[cf]
    nb = np.where(nl == own, nr, nl)
    return np.where(nb < 0, -1, nb).astype(np.int32)


def _sweep_mesh(mesh):
    keep = [np.ascontiguousarray(mesh.cell_volume, np.float64),
            np.ascontiguousarray(mesh.cell_faces, np.int32), sweep_neighbours(mesh),
            np.ascontiguousarray(mesh.cell_sign, np.uint8), np.ascontiguousarray(mesh.face_n, np.float64),
            np.ascontiguousarray(mesh.face_area, np.float64)]
    return OrcSweepMesh(mesh.n_cells, mesh.n_faces, *(_p(a) for a in keep)), keep


def port_trace_nodes(mesh, dirs):
    """orc_trace_nodes: the sweep's node geometry, in_face and s [M][N][4][3] (in the
    mesh's local faces; node q of face j has weight 2/3 at vertex (j + 1 + q) & 3)."""
    dirs = np.ascontiguousarray(dirs, np.float64)
    M, N = len(dirs), mesh.n_cells
    sm, keep = _sweep_mesh(mesh)
    hf = np.zeros((M, N, 4, 3), np.int32)
    s = np.zeros((M, N, 4, 3))
    port().orc_trace_nodes(C.byref(sm), M, _p(dirs), _p(hf), _p(s))
    return hf, s


_TRACE = None


def ref_trace():
    """The reference's make_trace / graph preprocessing compiled from its sources
    (oracle/_ref/librrhd_ref_trace.so), or None where it was not built."""
    global _TRACE
    if _TRACE is None:
        path = os.path.join(REF_DIR, "librrhd_ref_trace.so")
        if not os.path.exists(path):
            return None
        lib = C.CDLL(path)
        lib.ref_trace_nodes.restype = I64
        lib.ref_trace_nodes.argtypes = [I64, P, P, I32, P, P, P, P, P]
        lib.ref_graph_levels.restype = I32
        lib.ref_graph_levels.argtypes = [I64, P, P, I32, P, P]
        _TRACE = lib
    return _TRACE


def ref_trace_nodes(points, normals, dirs):
    """trace::GetInterpolationNodes + trace::GetLocNodes per direction (make_trace/src/
    trace_main.cpp) on cells given by their points in VTK order [N][4][3] and the outward
    normals of VTK's faces [N][4][3].  Returns (in-face bits [M][N], in_face [M][N][4][3],
    s [M][N][4][3], nodes [N][4][3][3], faces the reference would stop on)."""
    lib = ref_trace()
    pts = np.ascontiguousarray(points, np.float64)
    nrm = np.ascontiguousarray(normals, np.float64)
    dirs = np.ascontiguousarray(dirs, np.float64)
    M, N = len(dirs), len(pts)
    st = np.zeros((M, N), np.int32)
    hf = np.zeros((M, N, 4, 3), np.int32)
    s = np.zeros((M, N, 4, 3))
    nodes = np.zeros((N, 4, 3, 3))
    missed = lib.ref_trace_nodes(N, _p(pts), _p(nrm), M, _p(dirs), _p(st), _p(hf), _p(s), _p(nodes))
    return st, hf, s, nodes, missed


def ref_graph_levels(neighbours, normals, dirs):
    """The front index of every cell per direction in graph::RunGraphModule's sweep order
    (graph/src/graph_by_direction.cpp); neighbours [N][4] = neighbour cell * 4 + its
    local face, < 0 on the boundary.  Returns (levels [M][N], incomplete directions)."""
    lib = ref_trace()
    nb = np.ascontiguousarray(neighbours, np.int32)
    nrm = np.ascontiguousarray(normals, np.float64)
    dirs = np.ascontiguousarray(dirs, np.float64)
    M, N = len(dirs), len(nb)
    lv = np.zeros((M, N), np.int32)
    bad = lib.ref_graph_levels(N, _p(nb), _p(nrm), M, _p(dirs), _p(lv))
    return lv, bad


def port_sweep(mesh, dirs, alpha, betta, Q, S, bc=0.0, I=None):
    """orc_sweep on a Mesh: returns (I [N*G][M], unswept pairs).  I (optional) is the
    previous intensity; only the relative-change norm would read it."""
    N, F = mesh.n_cells, mesh.n_faces
    Q = np.ascontiguousarray(Q, np.float64).reshape(N, -1)
    G = Q.shape[1]
    dirs = np.ascontiguousarray(dirs, np.float64)
    M = len(dirs)
    S = np.ascontiguousarray(S, np.float64).reshape(N * G, M)
    keep = [np.ascontiguousarray(mesh.cell_volume, np.float64),
            np.ascontiguousarray(mesh.cell_faces, np.int32), sweep_neighbours(mesh),
            np.ascontiguousarray(mesh.cell_sign, np.uint8), np.ascontiguousarray(mesh.face_n, np.float64),
            np.ascontiguousarray(mesh.face_area, np.float64)]
    sm = OrcSweepMesh(N, F, *(_p(a) for a in keep))
    a = np.ascontiguousarray(alpha, np.float64)
    b = np.ascontiguousarray(betta, np.float64)
    I = np.zeros((N * G, M)) if I is None else np.array(I, np.float64, order="C")
    missing = port().orc_sweep(C.byref(sm), M, _p(dirs), G, _p(a), _p(b), _p(Q), _p(S), bc, _p(I))
    return I, missing


def ref_get_illum(I0, s, k, rhs, variant="rad_ideal_4_3"):
    I0 = np.ascontiguousarray(I0, np.float64)
    s = np.ascontiguousarray(s, np.float64)
    return ref(variant).ref_get_illum(_p(I0), _p(s), k, rhs)


def ref_get_rhs(alpha, betta, T, S, variant="rad_ideal_4_3"):
    k = C.c_double()
    r = ref(variant).ref_get_rhs(alpha, betta, T, S, C.byref(k))
    return r, k.value


def ref_recalc_illum(cell_faces, face_area, face_values, Illum, direction, variant="rad_ideal_4_3"):
    cf = np.ascontiguousarray(cell_faces, np.int32)
    fa = np.ascontiguousarray(face_area, np.float64)
    fv = np.ascontiguousarray(face_values, np.float64)
    assert Illum.flags.c_contiguous and Illum.dtype == np.float64
    return ref(variant).ref_recalc_illum(len(cf), len(fa), _p(cf), _p(fa), _p(fv), Illum.shape[1], direction,
                                         _p(Illum))


def ref_rad_constants(variant="rad_ideal_4_3"):
    out = np.zeros(4)
    ref(variant).ref_rad_constants(_p(out))
    return out


N_FRQ = 100  # N_Frq of the reference's full-spectrum kernel (cuda_scat_full_spectrum.cu:47)


def _compton_args(I, vel, dirs, areas, dir_disp, dir_count, out_stride):
    I = np.ascontiguousarray(I, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    dirs = np.ascontiguousarray(dirs, dtype=np.float64)
    areas = np.ascontiguousarray(areas, dtype=np.float64)
    cells, M = I.shape[0], dirs.shape[0]
    assert I.shape == (cells, M, N_FRQ) and vel.shape == (cells, 3)
    dir_count = M - dir_disp if dir_count is None else dir_count
    out_stride = dir_count if out_stride is None else out_stride
    S = np.zeros((cells, out_stride, N_FRQ))
    return I, vel, dirs, areas, cells, M, dir_count, out_stride, S


def port_compton(I, vel, dirs, areas, full_area, dir_disp=0, dir_count=None, out_stride=None, nthreads=1):
    """Full-spectrum Compton scattering S [cells][out_stride][100] by the C restatement."""
    I, vel, dirs, areas, cells, M, dir_count, out_stride, S = _compton_args(I, vel, dirs, areas, dir_disp,
                                                                            dir_count, out_stride)
    port().orc_compton_full_spectrum(M, _p(dirs), _p(areas), full_area, cells, _p(I), _p(vel), dir_disp,
                                     dir_count, out_stride, _p(S), nthreads)
    return S


def port_compton_frq(idx):
    return port().orc_compton_frq(idx)


def port_compton_frq_idx(frq):
    return port().orc_compton_frq_idx(frq)


def ref_compton(I, vel, dirs, areas, full_area, dir_disp=0, dir_count=None, out_stride=None, nthreads=0):
    """The same through the reference's own device source compiled for the host."""
    lib = ref("compton")
    if lib is None:
        return None
    I, vel, dirs, areas, cells, M, dir_count, out_stride, S = _compton_args(I, vel, dirs, areas, dir_disp,
                                                                            dir_count, out_stride)
    rc = lib.ref_compton_full_spectrum(M, _p(dirs), _p(areas), full_area, cells, _p(I), _p(vel), dir_disp,
                                       dir_count, out_stride, _p(S), nthreads)
    assert rc == 0
    return S


def ref_compton_get_frq(idx):
    return ref("compton").ref_compton_get_frq(idx)


def ref_compton_get_frq_idx(frq):
    return ref("compton").ref_compton_get_frq_idx(frq)


def _compton_one_args(I, vel, dirs, areas, dir_disp, dir_count, out_stride):
    I = np.ascontiguousarray(I, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    dirs = np.ascontiguousarray(dirs, dtype=np.float64)
    areas = np.ascontiguousarray(areas, dtype=np.float64)
    cells, M = I.shape[0], dirs.shape[0]
    assert I.shape == (cells, M) and vel.shape == (cells, 3)
    dir_count = M - dir_disp if dir_count is None else dir_count
    out_stride = dir_count if out_stride is None else out_stride
    return I, vel, dirs, areas, cells, M, dir_count, out_stride, np.zeros((cells, out_stride))


def port_compton_spectrum(I, vel, dirs, areas, full_area, frq, dir_disp=0, dir_count=None, out_stride=None,
                          nthreads=1):
    """Single-frequency Compton scattering S [cells][out_stride] by the C restatement."""
    I, vel, dirs, areas, cells, M, dir_count, out_stride, S = _compton_one_args(I, vel, dirs, areas, dir_disp,
                                                                                dir_count, out_stride)
    port().orc_compton_spectrum(M, _p(dirs), _p(areas), full_area, cells, _p(I), _p(vel), frq, dir_disp, dir_count,
                                out_stride, _p(S), nthreads)
    return S


def ref_compton_spectrum(I, vel, dirs, areas, full_area, frq, dir_disp=0, dir_count=None, out_stride=None,
                         nthreads=0):
    """The same through the reference's own device source compiled for the host."""
    lib = ref("compton")
    if lib is None:
        return None
    I, vel, dirs, areas, cells, M, dir_count, out_stride, S = _compton_one_args(I, vel, dirs, areas, dir_disp,
                                                                                dir_count, out_stride)
    assert lib.ref_compton_spectrum(M, _p(dirs), _p(areas), full_area, cells, _p(I), _p(vel), frq, dir_disp,
                                    dir_count, out_stride, _p(S), nthreads) == 0
    return S


RAY_PIXELS = (600, 300)  # image plane of solvers/ray_tracing/include/ray_tracing_const.h


def _ray_args(rays, ids, abc):
    rays = np.ascontiguousarray(rays, dtype=np.float64).reshape(-1, 6)
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    abc = np.ascontiguousarray(abc, dtype=np.float64).reshape(-1, 9)
    assert len(ids) == len(abc)
    return rays, ids, abc


def port_ray_trace(mode, rays, ids, abc, nthreads=1):
    """Intersection code per ray (mode 0 RayTracing, 1 RayTracing_Phl1445, 2 InnerRayTracing,
    3 RayTracingGrid) by the C restatement."""
    rays, ids, abc = _ray_args(rays, ids, abc)
    out = np.empty(len(rays), dtype=np.int32)
    port().orc_ray_trace(mode, _p(rays), len(rays), _p(ids), _p(abc), len(ids), _p(out), nthreads)
    return out


def port_ray_make_rays(frame):
    rays = np.empty((RAY_PIXELS[0] * RAY_PIXELS[1], 6))
    port().orc_ray_make_rays(frame, _p(rays))
    return rays


def port_ray_triangle(ray, abc):
    ray, abc = np.ascontiguousarray(ray, dtype=np.float64), np.ascontiguousarray(abc, dtype=np.float64)
    return port().orc_ray_triangle(_p(ray), _p(abc))


def port_ray_roche(ray):
    ray = np.ascontiguousarray(ray, dtype=np.float64)
    d = C.c_double()
    code = port().orc_ray_roche(_p(ray), C.byref(d))
    return code, d.value


def ref_ray(mode, rays, ids, abc, nthreads=0):
    """The same through the reference's own device source compiled for the host."""
    lib = ref("ray")
    if lib is None:
        return None
    rays, ids, abc = _ray_args(rays, ids, abc)
    out = np.empty(len(rays), dtype=np.int32)
    assert lib.ref_ray_trace(mode, _p(rays), len(rays), _p(ids), _p(abc), len(ids), _p(out), nthreads) == 0
    return out


def ref_ray_make_rays(frame):
    lib = ref("ray")
    rays = np.empty((RAY_PIXELS[0] * RAY_PIXELS[1], 6))
    assert lib.ref_ray_make_rays(frame, _p(rays)) == len(rays)
    return rays


def ref_ray_triangle(ray, abc):
    ray, abc = np.ascontiguousarray(ray, dtype=np.float64), np.ascontiguousarray(abc, dtype=np.float64)
    return ref("ray").ref_ray_triangle(_p(ray), _p(abc))


def ref_ray_roche(ray):
    ray = np.ascontiguousarray(ray, dtype=np.float64)
    d = C.c_double()
    code = ref("ray").ref_ray_roche(_p(ray), C.byref(d))
    return code, d.value
