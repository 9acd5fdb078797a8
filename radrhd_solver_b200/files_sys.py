"""The reference's binary file formats (lib/files_sys, `files_sys::bin`).

Every file is little-endian: an `int` element count followed by the raw
records, as the reference's fwrite-based readers and writers produce them.

    geo_faces.bin  int n, n x geo_face_t (40 B)   ReadGridGeo / WriteGridGeo
    geo_cells.bin  int n, n x geo_cell_t (56 B)   (reader_bin.h:113-135, writer_bin.h)
    no.bin         int n, n x flux_t {d, v[3], p}  ReadHllcInit (reader_bin.h:232-251)
    sphere txt     N, N lines `area x y z`, full_area   ReadSphereDirectionCartesian
                   (reader_txt.cpp:6-37)
    Solve<k>/      density.bin, pressure.bin (int n, n doubles), velocity.bin
                   (int n, n x 3 doubles), Illum.bin (int n, direction 0 of each
                   cell), energy.bin / stream.bin / impuls.bin (int n, raw arrays)
                   WriteSolution (writer_bin.cpp:56-114)

Record layouts (lib/grids/include/solvers_struct.h:51-59, 87-162):

    geo_face_t  u32 {id_l:25, id_l_node:6, is_regular:1}, i32 {id_r:26 (signed),
                id_r_node:6}, f64 n[3], f64 S
    geo_cell_t  i32 id_faces[4], f64 V, f64 center[3], u8 sign_n,
                u8 {node:6, is_bound:2}, 6 bytes of padding

Bitfields are allocated from the least significant bit, as gcc does on x86-64.
The node / is_regular / is_bound fields are carried through in `GeoFlags`;
the solver itself does not use them.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from .mesh import Directions, Mesh, read_sphere_directions

F_GEO_FACES = "geo_faces.bin"
F_GEO_CELLS = "geo_cells.bin"
F_INIT_HLLC = "no.bin"
F_DENSITY = "density.bin"
F_PRESSURE = "pressure.bin"
F_VELOCITY = "velocity.bin"
F_ILLUM = "Illum.bin"
F_ENERGY = "energy.bin"
F_STREAM = "stream.bin"
F_IMPULS = "impuls.bin"

GEO_FACE = np.dtype([("w0", "<u4"), ("w1", "<u4"), ("n", "<f8", (3,)), ("S", "<f8")])
GEO_CELL = np.dtype([("id_faces", "<i4", (4,)), ("V", "<f8"), ("center", "<f8", (3,)), ("sign_n", "u1"),
                     ("node_bound", "u1"), ("pad", "V6")])
FLUX = np.dtype([("d", "<f8"), ("v", "<f8", (3,)), ("p", "<f8")])
assert GEO_FACE.itemsize == 40 and GEO_CELL.itemsize == 56 and FLUX.itemsize == 40

_MASK25, _MASK26, _MASK6 = (1 << 25) - 1, (1 << 26) - 1, (1 << 6) - 1


@dataclass
class GeoFlags:
    """The record fields a Mesh does not hold (node numbers of the MPI split,
    regular-face and boundary-cell marks)."""
    face_id_l_node: np.ndarray  # uint8 [F]
    face_id_r_node: np.ndarray  # uint8 [F]
    face_is_regular: np.ndarray  # uint8 [F]
    cell_node: np.ndarray       # uint8 [N]
    cell_is_bound: np.ndarray   # uint8 [N]

    @classmethod
    def defaults(cls, n_faces: int, n_cells: int) -> "GeoFlags":
        """The values of the records' default constructors (is_regular = 1, the rest 0)."""
        return cls(np.zeros(n_faces, np.uint8), np.zeros(n_faces, np.uint8), np.ones(n_faces, np.uint8),
                   np.zeros(n_cells, np.uint8), np.zeros(n_cells, np.uint8))


def _read_count(f, path: str) -> int:
    head = f.read(4)
    if len(head) != 4:
        raise OSError(f"{path}: missing element count")
    n = int(np.frombuffer(head, "<i4")[0])
    if n < 0:
        raise OSError(f"{path}: negative element count {n}")
    return n


def _read_records(path: str, dtype, shape=()) -> np.ndarray:
    """`int n` then n records; a short file is an error, as in the reference readers."""
    with open(path, "rb") as f:
        n = _read_count(f, path)
        count = n * int(np.prod(shape, dtype=np.int64))
        data = np.fromfile(f, dtype=dtype, count=count)
    if data.size != count:
        raise OSError(f"{path}: {n} elements announced, the file is shorter")
    return data.reshape((n,) + tuple(shape)) if shape else data


def _write_records(path: str, n: int, data: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(np.int32(n).astype("<i4").tobytes())
        f.write(np.ascontiguousarray(data).tobytes())


# ------------------------------------------------------------------ geometry
def decode_faces(rec: np.ndarray):
    """geo_face_t records -> (id_l, id_r, n, S, id_l_node, id_r_node, is_regular)."""
    w0 = rec["w0"].astype(np.uint32)
    w1 = rec["w1"].astype(np.uint32)
    id_l = (w0 & _MASK25).astype(np.int32)
    id_l_node = ((w0 >> 25) & _MASK6).astype(np.uint8)
    is_regular = ((w0 >> 31) & 1).astype(np.uint8)
    r = (w1 & _MASK26).astype(np.int64)
    id_r = np.where(r >= (1 << 25), r - (1 << 26), r).astype(np.int32)  # sign-extend the 26-bit field
    id_r_node = ((w1 >> 26) & _MASK6).astype(np.uint8)
    return id_l, id_r, np.ascontiguousarray(rec["n"]), np.ascontiguousarray(rec["S"]), id_l_node, id_r_node, is_regular


def encode_faces(id_l, id_r, n, S, id_l_node=None, id_r_node=None, is_regular=None) -> np.ndarray:
    F = len(S)
    id_l = np.asarray(id_l, np.int64)
    id_r = np.asarray(id_r, np.int64)
    if F and (id_l.min() < 0 or id_l.max() > _MASK25):
        raise ValueError("id_l does not fit the 25-bit field")
    if F and (id_r.min() < -(1 << 25) or id_r.max() >= (1 << 25)):
        raise ValueError("id_r does not fit the signed 26-bit field")
    ln = np.zeros(F, np.uint32) if id_l_node is None else np.asarray(id_l_node, np.uint32) & _MASK6
    rn = np.zeros(F, np.uint32) if id_r_node is None else np.asarray(id_r_node, np.uint32) & _MASK6
    reg = np.ones(F, np.uint32) if is_regular is None else np.asarray(is_regular, np.uint32) & 1
    rec = np.zeros(F, GEO_FACE)
    rec["w0"] = id_l.astype(np.uint32) | (ln << 25) | (reg << 31)
    rec["w1"] = (id_r & _MASK26).astype(np.uint32) | (rn << 26)
    rec["n"] = n
    rec["S"] = S
    return rec


def decode_cells(rec: np.ndarray):
    """geo_cell_t records -> (id_faces, V, center, sign_n, node, is_bound)."""
    nb = rec["node_bound"]
    return (np.ascontiguousarray(rec["id_faces"]), np.ascontiguousarray(rec["V"]),
            np.ascontiguousarray(rec["center"]), np.ascontiguousarray(rec["sign_n"]),
            (nb & _MASK6).astype(np.uint8), (nb >> 6).astype(np.uint8))


def encode_cells(id_faces, V, center, sign_n, node=None, is_bound=None) -> np.ndarray:
    N = len(V)
    rec = np.zeros(N, GEO_CELL)
    rec["id_faces"] = id_faces
    rec["V"] = V
    rec["center"] = center
    rec["sign_n"] = sign_n
    nd = np.zeros(N, np.uint8) if node is None else np.asarray(node, np.uint8) & _MASK6
    bd = np.zeros(N, np.uint8) if is_bound is None else np.asarray(is_bound, np.uint8) & 3
    rec["node_bound"] = nd | (bd << 6)
    return rec


def mesh_h_min(m: Mesh) -> float:
    """min over cells of 3V / (largest face area), the synthetic builders' h_min."""
    if m.n_cells == 0:
        return 0.0
    smax = m.face_area[m.cell_faces].max(axis=1)
    return float((3.0 * m.cell_volume / smax).min())


def read_grid_geo(faces_file: str, cells_file: str, with_flags: bool = False):
    """Both geometry files into a Mesh (ReadGridGeo of grid.faces and grid.cells,
    solvers/rhllc/src/rhllc_main.cpp:21-22).  Face ids must stay within the
    mesh: id_l < n_cells, id_r < n_cells (negative values are boundary codes)."""
    fr = _read_records(faces_file, GEO_FACE)
    cr = _read_records(cells_file, GEO_CELL)
    id_l, id_r, n, S, ln, rn, reg = decode_faces(fr)
    cf, V, c, sg, nd, bd = decode_cells(cr)
    N, F = len(V), len(S)
    if F and (id_l.max() >= N or id_r.max() >= N):
        raise ValueError(f"{faces_file}: a face references a cell >= {N}")
    if N and (cf.min() < 0 or cf.max() >= F):
        raise ValueError(f"{cells_file}: a cell references a face outside [0, {F})")
    m = Mesh(id_l, id_r, n, S, cf, sg, V, c)
    m.h_min = mesh_h_min(m)
    if with_flags:
        return m, GeoFlags(ln, rn, reg, nd, bd)
    return m


def write_grid_geo(m: Mesh, faces_file: str, cells_file: str, flags: GeoFlags | None = None) -> None:
    """WriteGridGeo of the face and the cell records (lib/files_sys/include/writer_bin.h)."""
    fl = flags or GeoFlags.defaults(m.n_faces, m.n_cells)
    _write_records(faces_file, m.n_faces, encode_faces(m.face_id_l, m.face_id_r, m.face_n, m.face_area,
                                                       fl.face_id_l_node, fl.face_id_r_node, fl.face_is_regular))
    _write_records(cells_file, m.n_cells, encode_cells(m.cell_faces, m.cell_volume, m.cell_center, m.cell_sign,
                                                       fl.cell_node, fl.cell_is_bound))


# ------------------------------------------------------------------ direction sphere
def write_sphere_directions(path: str, d: Directions) -> None:
    """The text format read_sphere_directions (and the reference's
    ReadSphereDirectionCartesian) reads; every value is written as its shortest
    round-trip decimal, so the reader gets the same doubles back."""
    with open(path, "w") as f:
        f.write(f"{d.size}\n")
        for i in range(d.size):
            f.write(" ".join(repr(float(v)) for v in (d.areas[i], *d.dirs[i])) + "\n")
        f.write(f"{float(d.full_area)!r}\n")


__all__ = ["read_sphere_directions", "write_sphere_directions", "read_grid_geo", "write_grid_geo",
           "read_hllc_init", "write_hllc_init", "write_solution", "read_solution", "write_simple", "read_simple",
           "illum_direction", "GeoFlags", "mesh_h_min"]


# ------------------------------------------------------------------ hydro state
def read_hllc_init(path: str) -> np.ndarray:
    """no.bin -> primitive states W [n,5] = (rho, vx, vy, vz, p)
    (files_sys::bin::ReadHllcInit, reader_bin.h:232-251)."""
    rec = _read_records(path, FLUX)
    W = np.empty((len(rec), 5))
    W[:, 0] = rec["d"]
    W[:, 1:4] = rec["v"]
    W[:, 4] = rec["p"]
    return W


def write_hllc_init(path: str, W) -> None:
    """Writes W [n,5] in the layout ReadHllcInit reads."""
    W = np.asarray(W, np.float64)
    rec = np.zeros(len(W), FLUX)
    rec["d"] = W[:, 0]
    rec["v"] = W[:, 1:4]
    rec["p"] = W[:, 4]
    _write_records(path, len(W), rec)


# ------------------------------------------------------------------ solutions
def write_simple(path: str, data) -> None:
    """files_sys::bin::WriteSimple: `int n` then the raw array (n = its first dimension)."""
    a = np.ascontiguousarray(data, np.float64)
    _write_records(path, a.shape[0], a)


def read_simple(path: str, shape=()) -> np.ndarray:
    """Reads a WriteSimple / WRITE_FILE_ELEM file of doubles; shape = the trailing
    dimensions of one element ((3,) for velocity.bin, (3, 3) for impuls.bin)."""
    return _read_records(path, "<f8", shape)


def illum_direction(I, n_cells: int, direction: int = 0) -> np.ndarray:
    """The per-cell values WriteSolution puts in Illum.bin:
    GetCellDataBySelectedDirection (lib/geometry/include/convert_face_to_cell.h:51-62)
    takes element j * M + direction of the row-major [rows, M] intensity array for
    j < n_cells."""
    I = np.asarray(I, np.float64)
    return np.ascontiguousarray(I.reshape(-1, I.shape[-1])[:n_cells, direction])


def write_solution(directory: str, W=None, I=None, energy=None, stream=None, impuls=None) -> list[str]:
    """files_sys::bin::WriteSolution (lib/files_sys/src/writer_bin.cpp:56-114): writes
    the files for the fields given and returns their paths.

    W [N,5] primitive states -> density.bin, pressure.bin, velocity.bin;
    I [N*G, M] intensities (caller numbering) -> Illum.bin (direction 0);
    energy [N], stream [N,3], impuls [N,3,3] -> energy.bin, stream.bin, impuls.bin."""
    os.makedirs(directory, exist_ok=True)
    out = []

    def put(name, data):
        p = os.path.join(directory, name)
        write_simple(p, data)
        out.append(p)

    if I is not None:
        n = W.shape[0] if W is not None else (energy.shape[0] if energy is not None else None)
        if n is None:
            raise ValueError("Illum.bin needs the cell count: pass W or energy with I")
        put(F_ILLUM, illum_direction(I, n, 0))
    if energy is not None:
        put(F_ENERGY, energy)
    if stream is not None:
        put(F_STREAM, np.asarray(stream).reshape(-1, 3))
    if impuls is not None:
        put(F_IMPULS, np.asarray(impuls).reshape(-1, 3, 3))
    if W is not None:
        W = np.asarray(W, np.float64)
        put(F_DENSITY, W[:, 0])
        put(F_PRESSURE, W[:, 4])
        put(F_VELOCITY, W[:, 1:4])
    return out


def read_solution(directory: str) -> dict:
    """Reads back whichever WriteSolution files exist under `directory`."""
    shapes = {F_DENSITY: (), F_PRESSURE: (), F_VELOCITY: (3,), F_ILLUM: (), F_ENERGY: (), F_STREAM: (3,),
              F_IMPULS: (3, 3)}
    out = {}
    for name, shape in shapes.items():
        p = os.path.join(directory, name)
        if os.path.exists(p):
            out[name[:-4]] = read_simple(p, shape)
    return out
