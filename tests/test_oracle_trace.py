"""The sweep's geometry and order pinned to the reference's own preprocessing.

The reference makes both offline with VTK tools: make_trace (trace::GetInterpolationNodes,
trace::GetLocNodes: per out-face node, the in-face it is traced back to along -w and the
distance s) and graph (graph::RunGraphModule: the fronts the cells are swept in).  Their
sources compile without VTK (oracle/_ref/librrhd_ref_trace.so, ref_trace_shim.cpp); here
they run on the same jittered Kuhn meshes as the oracle (orc_sweep), which the GPU sweep
is tested against to 1e-12:

* every node the reference places is one of the oracle's (barycentric 2/3 at one face
  vertex, 1/6 at the others) to rounding; the in-face of every node is the same and s
  agrees to 1e-12 relative (ray-triangle intersection there, heights over faces here);
* the reference's fronts are the oracle's levels (depth of a cell in the upwind graph);
* a sweep assembled from the reference's geometry, its front order, its GetIllum and its
  ReCalcIllumOpt equals orc_sweep to 1e-12.

The cells are handed to the reference with their points in VTK order (p0, p1, p2, p3) =
(v1, v2, v0, v3), so that VTK's face j ({0,1,3}, {1,2,3}, {2,0,3}, {0,2,1}) is the mesh's
local face j (opposite vertex v_j).
"""
import numpy as np
import pytest

import oracle
from oracle import loader as OL
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box

RAD = "rad_ideal_4_3"
VTK_POINTS = [1, 2, 0, 3]

pytestmark = pytest.mark.skipif(OL.ref_trace() is None, reason="reference trace build not present (make -C oracle ref)")


def _mesh(n=(4, 4, 3), seed=4):
    return kuhn_box(*n, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=seed, with_vertices=True)


def _outward_normals(m):
    sign = np.where((m.cell_sign[:, None] >> np.arange(4)) & 1, 1.0, -1.0)
    return m.face_n[m.cell_faces] * sign[..., None]  # [N][4][3]


def _neighbour_faces(m):
    """[N][4]: neighbour cell * 4 + the neighbour's local index of the shared face, -1 on
    the boundary (the reference's neighbour file layout)."""
    N = m.n_cells
    owner = {}
    for c in range(N):
        for j in range(4):
            owner.setdefault(int(m.cell_faces[c, j]), []).append((c, j))
    nb = np.full((N, 4), -1, np.int32)
    for lst in owner.values():
        if len(lst) == 2:
            (a, ja), (b, jb) = lst
            nb[a, ja] = 4 * b + jb
            nb[b, jb] = 4 * a + ja
    return nb


def _reference_geometry(m, dirs):
    pts = m.vertices[m.cell_vertices[:, VTK_POINTS]]
    return oracle.loader.ref_trace_nodes(pts, _outward_normals(m), dirs)


def test_trace_nodes_match_reference():
    """Every node of every out-face for 24 directions on a jittered 4 x 4 x 3 box.

    One kind of face is left out and counted: a boundary face exactly parallel to a
    direction (the box's faces on the y = +-1 planes and the first Fibonacci direction,
    whose y component is 0).  The reference's FindInAndOutFaces takes any face with
    n.w >= -1e-10 as an out-face and traces its nodes, whose backward rays run inside
    the face's own plane and meet no in-face (the reference stops the program there,
    trace_nodes.cpp:228-231); the sweep here treats such a face as neither in nor out,
    and it keeps the boundary value."""
    m = _mesh()
    dirs = fibonacci_directions(24).dirs
    st, hf_r, s_r, nodes, missed = _reference_geometry(m, dirs)
    hf_o, s_o = OL.port_trace_nodes(m, dirs)
    n = _outward_normals(m)
    cos = np.einsum("cjx,dx->dcj", n, dirs)
    nb = _neighbour_faces(m)
    flat = np.abs(cos) <= 1e-10
    assert np.all(cos[flat] == 0) and np.all(nb[None].repeat(len(dirs), 0)[flat] < 0)
    assert missed <= flat.sum()
    assert np.all(hf_r[~flat] != -2)
    # every other face is classified alike: in-face bit set exactly where n.w < 0
    inb = ((st[..., None] >> np.arange(4)) & 1).astype(bool)
    assert np.array_equal(inb[~flat], (cos < 0)[~flat])
    # node positions: the oracle's node q of face j has weight 2/3 at vertex (j + 1 + q) & 3
    V = m.vertices[m.cell_vertices]  # [N][4][3]
    mine = np.zeros((m.n_cells, 4, 3, 3))
    for j in range(4):
        vi = [(j + 1) & 3, (j + 2) & 3, (j + 3) & 3]  # the vertices of face j
        for q in range(3):
            mine[:, j, q] = (4.0 * V[:, vi[q]] + V[:, vi[(q + 1) % 3]] + V[:, vi[(q + 2) % 3]]) / 6.0
    dist = np.linalg.norm(nodes[:, :, :, None, :] - mine[:, :, None, :, :], axis=-1)  # [N][4][ref n][my q]
    match = dist.argmin(-1)
    assert np.all(np.sort(match, -1) == np.arange(3)), "every reference node is a distinct oracle node"
    assert dist.min(-1).max() < 1e-14 * np.abs(V).max()
    # per (direction, cell, out-face, node): the same in-face, s to 1e-12
    out = (cos > 0) & ~flat
    q_of = np.broadcast_to(match[None], hf_r.shape)
    hf_o_m = np.take_along_axis(hf_o, q_of, -1)
    s_o_m = np.take_along_axis(s_o, q_of, -1)
    assert np.array_equal(hf_r[out], hf_o_m[out])
    rel = np.abs(s_r[out] - s_o_m[out]) / s_r[out]
    print(f"\nnodes {out.sum() * 3}: in-faces identical, s max rel diff {rel.max():.2e}; "
          f"{flat.sum()} boundary faces parallel to a direction left out")
    assert rel.max() <= 1e-12
    assert np.all(hf_r[cos < 0] == -1)


def _depths(m, dirs):
    """Depth of every cell in the upwind graph (0: no upwind neighbour), per direction."""
    n = _outward_normals(m)
    nb = _neighbour_faces(m)
    M, N = len(dirs), m.n_cells
    out = np.full((M, N), -1, np.int32)
    for d in range(M):
        cos = n @ dirs[d]
        up = (cos < 0) & (nb >= 0)
        indeg = up.sum(1)
        cur = list(np.nonzero(indeg == 0)[0])
        lvl = 0
        while cur:
            nxt = []
            for c in cur:
                out[d, c] = lvl
                for j in range(4):
                    if cos[c, j] > 0 and nb[c, j] >= 0:
                        k = nb[c, j] // 4
                        indeg[k] -= 1
                        if indeg[k] == 0:
                            nxt.append(k)
            cur = nxt
            lvl += 1
    return out


def test_graph_fronts_are_the_oracle_levels():
    m = _mesh((5, 4, 4), seed=9)
    dirs = fibonacci_directions(32).dirs
    lv, bad = oracle.loader.ref_graph_levels(_neighbour_faces(m), _outward_normals(m), dirs)
    assert bad == 0 and lv.min() >= 0
    dep = _depths(m, dirs)
    assert np.array_equal(lv, dep)
    print(f"\n{len(dirs)} directions: fronts = levels, up to {lv.max() + 1} per direction")


def test_sweep_on_reference_geometry_and_order():
    """A sweep assembled from the reference's node geometry, its front order, its
    GetIllum and its ReCalcIllumOpt, against orc_sweep."""
    if not oracle.have_ref(RAD):
        pytest.skip(f"reference variant {RAD} not built")
    m = _mesh((3, 3, 3), seed=5)
    M, G = 8, 2
    rng = np.random.default_rng(6)
    # a Fibonacci set turned about the z axis, so that no direction lies in a box plane
    ph = 0.3
    rot = np.array([[np.cos(ph), -np.sin(ph), 0.0], [np.sin(ph), np.cos(ph), 0.0], [0.0, 0.0, 1.0]])
    dirs = np.ascontiguousarray(fibonacci_directions(M).dirs @ rot.T)
    assert np.abs(np.einsum("cjx,dx->dcj", _outward_normals(m), dirs)).min() > 1e-10
    alpha = 10 ** rng.uniform(-1, 1.5, m.n_cells)
    betta = 0.5 * alpha
    Q = 10 ** rng.uniform(-2, 0, (m.n_cells, G))
    S = 10 ** rng.uniform(-3, -1, (m.n_cells * G, M))
    _, hf, s, _, missed = _reference_geometry(m, dirs)
    assert missed == 0
    lv, bad = oracle.loader.ref_graph_levels(_neighbour_faces(m), _outward_normals(m), dirs)
    assert bad == 0
    nb = _neighbour_faces(m)
    cos = np.einsum("cjx,dx->dcj", _outward_normals(m), dirs)
    N, F = m.n_cells, m.n_faces
    I = np.zeros((N * G, M))
    for d in range(M):
        fv = np.zeros((F, G))  # boundary value 0 (illum::BoundaryConditions for free boundaries)
        order = sorted(range(N), key=lambda c: (lv[d, c], c))  # fronts, cells ascending within one
        for c in order:
            for j in range(4):
                if not cos[d, c, j] > 0:
                    continue
                for g in range(G):
                    I0 = [fv[m.cell_faces[c, h], g] if nb[c, h] >= 0 else 0.0 for h in hf[d, c, j]]
                    rhs, k = oracle.port_get_rhs(alpha[c], betta[c], Q[c, g], S[c * G + g, d])
                    fv[m.cell_faces[c, j], g] = oracle.ref_get_illum(I0, s[d, c, j], k, rhs, RAD)
        for g in range(G):
            col = np.ascontiguousarray(I[g::G, :])
            oracle.ref_recalc_illum(m.cell_faces, m.face_area, fv[:, g], col, d, RAD)
            I[g::G, d] = col[:, d]
    Io, missing = oracle.port_sweep(m, dirs, alpha, betta, Q, S)
    assert missing == 0
    err = np.max(np.abs(Io - I) / np.abs(I))
    print(f"\nsweep on the reference's geometry and order vs orc_sweep: max rel diff {err:.2e}")
    assert err <= 1e-12
