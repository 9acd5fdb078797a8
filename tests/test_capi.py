"""CPU checks of the native library: it loads, exports every entry point the
public headers declare, and its host-side generators produce valid meshes."""
import os
import re

import numpy as np

from radrhd_solver_b200 import _lib as L
from radrhd_solver_b200 import mesh as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rrhd_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for h in sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")):
        for name in declared(h):
            assert name in exported, f"{h} declares {name} but librrhd.so does not export it"
            assert hasattr(L.lib, name)


def test_errors_are_returned_not_raised():
    st = L.lib.rrhd_create(None, None, None)
    assert st == L.RRHD_ERR_INVALID
    assert b"null" in L.lib.rrhd_last_error()
    assert L.lib.rrhd_version().startswith(b"rrhd")


def test_kuhn_mesh_invariants():
    m = M.kuhn_box(6, 5, 4, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=3, with_vertices=True)
    N, F = m.n_cells, m.n_faces
    assert N == 6 * 6 * 5 * 4
    # each interior face has two cells, boundary faces one
    nb = (m.face_id_r < 0).sum()
    assert nb == 4 * (6 * 5 + 5 * 4 + 6 * 4)
    assert 2 * F - nb == 4 * N
    # every cell's faces close: sum of signed area vectors vanishes
    acc = np.zeros((N, 3))
    for j in range(4):
        f = m.cell_faces[:, j]
        s = np.where((m.cell_sign >> j) & 1, 1.0, -1.0)
        acc += (s * m.face_area[f])[:, None] * m.face_n[f]
    assert np.abs(acc).max() < 1e-14
    assert abs(m.cell_volume.sum() - 8.0) < 1e-12
    # ConvertBinToGeo orientation: id_l's sign bit set, id_r's cleared
    for f in range(0, F, 7):
        l, r = m.face_id_l[f], m.face_id_r[f]
        jl = list(m.cell_faces[l]).index(f)
        assert (m.cell_sign[l] >> jl) & 1
        if r >= 0:
            jr = list(m.cell_faces[r]).index(f)
            assert not (m.cell_sign[r] >> jr) & 1
    # normals point from id_l towards id_r
    inner = m.face_id_r >= 0
    d = m.cell_center[m.face_id_r[inner]] - m.cell_center[m.face_id_l[inner]]
    assert ((d * m.face_n[inner]).sum(1) > 0).all()
    # faces are created in first-incidence order
    first = np.full(F, -1)
    for c in range(N):
        for j in range(4):
            f = m.cell_faces[c, j]
            if first[f] < 0:
                first[f] = 4 * c + j
    assert (np.diff(first) > 0).all()
    assert m.h_min > 0


def test_kuhn_inflow_codes():
    m = M.kuhn_box(10, 10, 4, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.1, seed=1, inflow_radius=0.45,
                   inflow_code=-3)
    codes = set(np.unique(m.face_id_r[m.face_id_r < 0]).tolist())
    assert codes == {-1, -3}
    f = np.where(m.face_id_r == -3)[0]
    assert np.allclose(m.face_n[f], [0, 0, -1])


def test_fibonacci_directions():
    d = M.fibonacci_directions(256)
    assert np.allclose(np.linalg.norm(d.dirs, axis=1), 1.0)
    assert abs(d.areas.sum() - 4 * np.pi) < 1e-12 and d.full_area == 4 * np.pi
    assert np.abs(d.dirs.mean(0)).max() < 1e-2


def test_rng_is_counter_based():
    a = [L.lib.rrhd_rng_u01(5, 1, i) for i in range(1000)]
    assert a == [L.lib.rrhd_rng_u01(5, 1, i) for i in range(1000)]
    assert 0.45 < np.mean(a) < 0.55 and min(a) >= 0 and max(a) < 1
