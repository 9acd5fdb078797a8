"""Synthetic meshes and direction sets (include/rrhd_mesh.h).

A `Mesh` holds the arrays of the reference's geo_face_t / geo_cell_t records
(lib/grids/include/solvers_struct.h:87-162) as numpy arrays.  `kuhn_box` builds
an axis-aligned hex grid split into 6 Kuhn tetrahedra per hex with seeded vertex
jitter, faces assembled as ConvertBinToGeo does
(lib/geometry/src/convert_bin_to_geo.cpp:3-48).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class Mesh:
    face_id_l: np.ndarray   # int32 [F]
    face_id_r: np.ndarray   # int32 [F] (negative = boundary code)
    face_n: np.ndarray      # float64 [F,3]
    face_area: np.ndarray   # float64 [F]
    cell_faces: np.ndarray  # int32 [N,4]
    cell_sign: np.ndarray   # uint8 [N]
    cell_volume: np.ndarray  # float64 [N]
    cell_center: np.ndarray  # float64 [N,3]
    h_min: float = 0.0
    vertices: np.ndarray | None = None       # float64 [V,3]
    cell_vertices: np.ndarray | None = None  # int32 [N,4]

    @property
    def n_cells(self) -> int:
        return int(self.cell_volume.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_area.shape[0])

    def desc(self) -> L.MeshDesc:
        for a in (self.face_id_l, self.face_id_r, self.face_n, self.face_area, self.cell_faces,
                  self.cell_sign, self.cell_volume, self.cell_center):
            assert a.flags.c_contiguous
        return L.MeshDesc(self.n_cells, self.n_faces, L.ptr(self.face_id_l), L.ptr(self.face_id_r),
                          L.ptr(self.face_n), L.ptr(self.face_area), L.ptr(self.cell_faces),
                          L.ptr(self.cell_sign), L.ptr(self.cell_volume), L.ptr(self.cell_center))


def kuhn_box(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter: float = 0.15,
             seed: int = 1, bc_codes=(-1, -1, -1, -1, -1, -1), inflow_radius: float = 0.0,
             inflow_code: int = -3, with_vertices: bool = False) -> Mesh:
    p = L.KuhnParams()
    p.nx, p.ny, p.nz = nx, ny, nz
    for a in range(3):
        p.lo[a] = lo[a]
        p.hi[a] = hi[a]
    p.jitter = jitter
    p.seed = seed
    for k in range(6):
        p.bc_code[k] = bc_codes[k]
    p.inflow_radius = inflow_radius
    p.inflow_code = inflow_code
    n, f, v = C.c_int64(), C.c_int64(), C.c_int64()
    L.check(L.lib.rrhd_mesh_kuhn_sizes(C.byref(p), C.byref(n), C.byref(f), C.byref(v)), "kuhn sizes")
    N, F, V = n.value, f.value, v.value
    m = Mesh(np.zeros(F, np.int32), np.zeros(F, np.int32), np.zeros((F, 3)), np.zeros(F),
             np.zeros((N, 4), np.int32), np.zeros(N, np.uint8), np.zeros(N), np.zeros((N, 3)))
    if with_vertices:
        m.vertices = np.zeros((V, 3))
        m.cell_vertices = np.zeros((N, 4), np.int32)
    h = C.c_double()
    L.check(L.lib.rrhd_mesh_kuhn_build(C.byref(p), L.ptr(m.face_id_l), L.ptr(m.face_id_r), L.ptr(m.face_n),
                                       L.ptr(m.face_area), L.ptr(m.cell_faces), L.ptr(m.cell_sign),
                                       L.ptr(m.cell_volume), L.ptr(m.cell_center), C.byref(h),
                                       L.ptr(m.vertices), L.ptr(m.cell_vertices)), "kuhn build")
    m.h_min = h.value
    return m


@dataclass
class Directions:
    """grid_directions_t (lib/geometry/include/geo_types.h:110-127)."""
    dirs: np.ndarray   # [M,3]
    areas: np.ndarray  # [M]
    full_area: float

    @property
    def size(self) -> int:
        return int(self.areas.shape[0])

    def subset(self, first: int, count: int) -> "Directions":
        """Directions first .. first + count - 1 (one rank's share of a direction split),
        with the full sphere's area."""
        return Directions(np.ascontiguousarray(self.dirs[first:first + count]),
                          np.ascontiguousarray(self.areas[first:first + count]), self.full_area)


def fibonacci_directions(M: int) -> Directions:
    d = np.zeros((M, 3))
    a = np.zeros(M)
    fa = C.c_double()
    L.check(L.lib.rrhd_directions_fibonacci(M, L.ptr(d), L.ptr(a), C.byref(fa)), "fibonacci")
    return Directions(d, a, fa.value)


def read_sphere_directions(path: str) -> Directions:
    """Reads the reference's direction-sphere text format: N, then N lines of
    `area x y z`, then full_area (lib/files_sys/src/reader_txt.cpp:6-24).
    A file with fewer values than announced is an error."""
    tok = open(path).read().split()
    if not tok:
        raise OSError(f"{path}: empty direction file")
    n = int(tok[0])
    if n < 0 or len(tok) < 2 + 4 * n:
        raise OSError(f"{path}: {n} directions announced, the file is shorter")
    vals = np.array([float(t) for t in tok[1:1 + 4 * n]]).reshape(n, 4)
    full = float(tok[1 + 4 * n])
    return Directions(np.ascontiguousarray(vals[:, 1:4]), np.ascontiguousarray(vals[:, 0]), full)
