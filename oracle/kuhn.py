"""Kuhn tetrahedral box meshes built in numpy (test infrastructure).

An independent restatement of the library's synthetic mesh generator
(`rrhd_mesh_kuhn_build`, radrhd_solver_b200/csrc/mesh.cpp), so that the CPU
reference arm of the benchmark and the oracle tests can build the benchmark
meshes without loading the CUDA library.  `tests/test_oracle_kuhn.py` pins the
two generators to each other array for array, bit for bit.

The mesh: an axis-aligned box of nx x ny x nz hexes, each split into the 6 Kuhn
tetrahedra v000, v000+e_a, v000+e_a+e_b, v111 (one per axis permutation (a, b,
c)); interior vertices jittered by U(-jitter h, +jitter h) per axis from the
counter-based generator (seed, stream 1 + axis, vertex id); faces assembled in
the reference's ConvertBinToGeo order (lib/geometry/src/convert_bin_to_geo.cpp:3-48):
incidences (cell, local face j opposite vertex j) in increasing order, the
first incidence of a face is its left cell (sign bit set, outward normal),
the second its right cell (sign bit cleared); an unmatched incidence gets the
boundary code of its box plane, or the inflow code on the z-low plane inside
the inflow radius.  Every floating-point expression is evaluated in the same
order as the library's, so both give identical doubles.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def u01(seed: int, stream: int, index: np.ndarray) -> np.ndarray:
    """Uniform doubles in [0, 1) with 53 random bits: a pure function of
    (seed, stream, index) (splitmix64 finaliser, as csrc/rng.h)."""
    with np.errstate(over="ignore"):
        s = _mix64(np.array([stream], np.uint64) * np.uint64(0xD1B54A32D192ED03))
        k = _mix64(np.array([seed], np.uint64) ^ s)
        h = _mix64(k ^ np.asarray(index, np.uint64))
    return (h >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


@dataclass
class KuhnMesh:
    face_id_l: np.ndarray
    face_id_r: np.ndarray
    face_n: np.ndarray
    face_area: np.ndarray
    cell_faces: np.ndarray
    cell_sign: np.ndarray
    cell_volume: np.ndarray
    cell_center: np.ndarray
    h_min: float
    vertices: np.ndarray
    cell_vertices: np.ndarray

    @property
    def n_cells(self) -> int:
        return int(self.cell_volume.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.face_area.shape[0])


_PERM = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def _dot(a, b):
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def kuhn_box(nx: int, ny: int, nz: int, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), jitter: float = 0.15,
             seed: int = 1, bc_codes=(-1, -1, -1, -1, -1, -1), inflow_radius: float = 0.0,
             inflow_code: int = -3) -> KuhnMesh:
    if min(nx, ny, nz) <= 0:
        raise ValueError("bad Kuhn mesh size")
    nmax = (nx, ny, nz)
    if (nx + 1) * (ny + 1) * (nz + 1) >= 1 << 21:
        raise ValueError("Kuhn mesh too large (more than 2^21 vertices)")
    h = [(hi[a] - lo[a]) / nmax[a] for a in range(3)]
    V = (nx + 1) * (ny + 1) * (nz + 1)
    vid = np.arange(V, dtype=np.int64)
    gi = [vid % (nx + 1), (vid // (nx + 1)) % (ny + 1), vid // ((nx + 1) * (ny + 1))]
    vx = np.zeros((V, 3))
    for a in range(3):
        x = lo[a] + gi[a].astype(np.float64) * h[a]
        if jitter != 0.0:
            inner = (gi[a] > 0) & (gi[a] < nmax[a])
            u = u01(seed, 1 + a, vid[inner])
            x[inner] += (2.0 * u - 1.0) * jitter * h[a]
        vx[:, a] = x

    # cells: hexes in k, j, i order (i fastest), 6 tets each
    hi_, hj, hk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    hi_, hj, hk = (q.transpose(2, 1, 0).ravel().astype(np.int64) for q in (hi_, hj, hk))
    nh = hi_.size
    N = 6 * nh

    def vof(i, j, k):
        return (k * (ny + 1) + j) * (nx + 1) + i

    tv = np.zeros((nh, 6, 4), np.int64)
    for t, perm in enumerate(_PERM):
        o = [hi_.copy(), hj.copy(), hk.copy()]
        tv[:, t, 0] = vof(*o)
        o[perm[0]] += 1
        tv[:, t, 1] = vof(*o)
        o[perm[1]] += 1
        tv[:, t, 2] = vof(*o)
        tv[:, t, 3] = vof(hi_ + 1, hj + 1, hk + 1)
    tv = tv.reshape(N, 4)
    P = vx[tv]  # [N, 4, 3]
    cr = _cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    vol = np.abs(_dot(cr, P[:, 3] - P[:, 0])) / 6.0
    center = (((P[:, 0] + P[:, 1]) + P[:, 2]) + P[:, 3]) / 4.0
    inc_n = np.zeros((N, 4, 3))
    inc_S = np.zeros((N, 4))
    for fj in range(4):
        A, B, Cc = P[:, (fj + 1) & 3], P[:, (fj + 2) & 3], P[:, (fj + 3) & 3]
        n = _cross(B - A, Cc - A)
        ln = np.sqrt(_dot(n, n))
        inc_S[:, fj] = 0.5 * ln
        n = n / ln[:, None]
        flip = _dot(n, P[:, fj] - A) > 0
        n[flip] = -n[flip]
        inc_n[:, fj] = n
    smax = np.zeros(N)
    for fj in range(4):
        smax = np.maximum(smax, inc_S[:, fj])
    h_min = float(np.min(3.0 * vol / smax))

    # incidences matched by their sorted vertex triple
    q = np.stack([tv[:, [(fj + 1) & 3, (fj + 2) & 3, (fj + 3) & 3]] for fj in range(4)], 1).reshape(4 * N, 3)
    qs = np.sort(q, 1)
    key = (qs[:, 0] << 42) | (qs[:, 1] << 21) | qs[:, 2]
    order = np.lexsort((np.arange(4 * N), key))
    ks = key[order]
    partner = np.full(4 * N, -1, np.int64)
    same = np.nonzero(ks[1:] == ks[:-1])[0]
    # a key occurs at most twice in a conforming mesh: pair each run's first two
    partner[order[same]] = order[same + 1]
    partner[order[same + 1]] = order[same]

    inc = np.arange(4 * N, dtype=np.int64)
    first = (partner < 0) | (inc < partner)
    finc = inc[first]
    F = finc.size
    cell_faces = np.zeros(4 * N, np.int32)
    cell_faces[finc] = np.arange(F, dtype=np.int32)
    pf = partner[finc]
    paired = pf >= 0
    cell_faces[pf[paired]] = np.nonzero(paired)[0].astype(np.int32)
    face_id_l = (finc // 4).astype(np.int32)
    face_id_r = np.where(paired, pf // 4, -1).astype(np.int32)
    face_n = inc_n.reshape(4 * N, 3)[finc]
    face_area = inc_S.reshape(4 * N)[finc]
    sign_bit = np.zeros(4 * N, np.uint8)
    sign_bit[finc] = 1
    cell_sign = (sign_bit.reshape(N, 4) << np.arange(4, dtype=np.uint8)).sum(1).astype(np.uint8)

    # boundary codes of the unmatched incidences: plane of their three vertices
    bidx = np.nonzero(~paired)[0]
    bq = q[finc[bidx]]  # vertex order (fj+1, fj+2, fj+3) & 3
    g = [np.stack([bq % (nx + 1), (bq // (nx + 1)) % (ny + 1), bq // ((nx + 1) * (ny + 1))], -1)]
    g = g[0]  # [nb, 3 vertices, 3 axes]
    plane = np.full(bidx.size, -1, np.int64)
    for ax in range(3):
        lo_ = (plane < 0) & np.all(g[:, :, ax] == 0, 1)
        plane[lo_] = 2 * ax
        hi2 = (plane < 0) & np.all(g[:, :, ax] == nmax[ax], 1)
        plane[hi2] = 2 * ax + 1
    codes = np.full(bidx.size, -1, np.int32)
    bcc = np.asarray(bc_codes, np.int32)
    okp = plane >= 0
    cp = np.where(okp, bcc[np.maximum(plane, 0)], 0)
    codes[okp & (cp != 0)] = cp[okp & (cp != 0)]
    if inflow_radius > 0:
        zl = plane == 4
        cx, cy = 0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1])
        x = np.zeros(bidx.size)
        y = np.zeros(bidx.size)
        for a in range(3):
            x = x + vx[bq[:, a], 0] / 3.0
            y = y + vx[bq[:, a], 1] / 3.0
        inside = zl & ((x - cx) * (x - cx) + (y - cy) * (y - cy) < inflow_radius * inflow_radius)
        codes[inside] = inflow_code
    face_id_r[bidx] = codes
    return KuhnMesh(face_id_l, face_id_r, np.ascontiguousarray(face_n), np.ascontiguousarray(face_area),
                    cell_faces.reshape(N, 4), cell_sign, vol, np.ascontiguousarray(center), h_min, vx,
                    tv.astype(np.int32))
