"""Loading of the golden fixtures in tests/golden/ (outputs of the reference
compiled from its own sources, written by tests/golden/make_golden.py)."""
from __future__ import annotations

import os

import numpy as np

from radrhd_solver_b200.mesh import Mesh

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


def mesh(g, prefix="mesh_"):
    return Mesh(g[prefix + "face_id_l"], g[prefix + "face_id_r"], g[prefix + "face_n"], g[prefix + "face_area"],
                g[prefix + "cell_faces"], g[prefix + "cell_sign"], g[prefix + "cell_volume"],
                g[prefix + "cell_center"], float(g[prefix + "h_min"]))
