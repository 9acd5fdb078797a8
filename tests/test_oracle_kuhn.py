"""The oracle's numpy Kuhn mesh generator (oracle/kuhn.py) against the library's
rrhd_mesh_kuhn_build: every array bit for bit.  The benchmark's CPU reference
arm builds its mesh with the oracle generator, so that it never loads the CUDA
library; this pins the two meshes to each other."""
import numpy as np
import pytest

from oracle import kuhn as K
from radrhd_solver_b200 import mesh as M

CASES = [
    dict(nx=5, ny=4, nz=3, jitter=0.15, seed=3),
    dict(nx=6, ny=5, nz=7, lo=(-1, -2, 0.5), hi=(1, 0.5, 2), jitter=0.2, seed=11,
         bc_codes=(-1, -2, -1, -4, -5, -6)),
    dict(nx=12, ny=12, nz=12, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=2024, inflow_radius=0.3,
         inflow_code=-3),
    dict(nx=9, ny=3, nz=2, jitter=0.0, seed=1),
]


@pytest.mark.parametrize("kw", CASES)
def test_kuhn_mesh_identical_to_library(kw):
    a = M.kuhn_box(**kw, with_vertices=True)
    b = K.kuhn_box(**kw)
    assert a.n_cells == b.n_cells and a.n_faces == b.n_faces
    for name in ("face_id_l", "face_id_r", "face_n", "face_area", "cell_faces", "cell_sign", "cell_volume",
                 "cell_center", "vertices", "cell_vertices"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        assert np.array_equal(x, y), name
    assert a.h_min == b.h_min


def test_rng_matches_library():
    from radrhd_solver_b200 import _lib as L
    idx = np.array([0, 1, 2, 12345, 2**40 + 7], np.uint64)
    got = K.u01(2024, 2, idx)
    want = np.array([L.lib.rrhd_rng_u01(2024, 2, int(i)) for i in idx])
    assert np.array_equal(got, want)
