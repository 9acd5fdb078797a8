"""Transport-sweep oracle (CPU): the per-face and per-cell arithmetic of
orc_get_illum / orc_get_rhs / orc_recalc_illum bit for bit against the reference
compiled from its own sources (illum::GetIllum, illum::GetRhsOpt,
illum::separate_gpu::ReCalcIllumOpt), and the whole sweep against an independent
pure-Python sweep that traces the characteristics through the cell planes built
from the vertices and evaluates every face and cell with the reference's own
functions."""
import numpy as np
import pytest

import oracle
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box

RAD = "rad_ideal_4_3"


def need(v):
    if not oracle.have_ref(v):
        pytest.skip(f"reference variant {v} not built")


def test_get_illum_bitwise():
    need(RAD)
    rng = np.random.default_rng(1)
    for _ in range(2000):
        I0 = 10 ** rng.uniform(-6, 2, 3)
        s = rng.uniform(0, 0.1, 3)
        k = 10 ** rng.uniform(-3, 3)
        rhs = 10 ** rng.uniform(-6, 2)
        assert oracle.port_get_illum(I0, s, k, rhs) == oracle.ref_get_illum(I0, s, k, rhs, RAD)


def test_get_rhs_bitwise():
    """GetRhsOpt computes Q = B_Plank(T) / kRadiation with B = T^4 sigma / pi
    (lib/physics/src/plunk.cpp:87-90); the port is given Q."""
    need(RAD)
    c = oracle.ref_rad_constants(RAD)
    sigma, pi, rad_unit = c[1], c[2], c[3]
    rng = np.random.default_rng(2)
    for _ in range(2000):
        a, b = 10 ** rng.uniform(-3, 2, 2)
        T = 10 ** rng.uniform(-3, 5)
        S = 10 ** rng.uniform(-6, 1)
        T2 = T * T
        Q = (T2 * T2) * sigma / pi / rad_unit
        assert oracle.port_get_rhs(a, b, Q, S) == oracle.ref_get_rhs(a, b, T, S, RAD)


def test_recalc_illum_bitwise():
    need(RAD)
    m = kuhn_box(4, 3, 2, seed=3)
    rng = np.random.default_rng(3)
    M = 5
    fv = 10 ** rng.uniform(-3, 1, m.n_faces)
    I1 = rng.uniform(0.1, 1, (m.n_cells, M))
    I2 = I1.copy()
    for d in (0, 3):
        n1 = oracle.port_recalc_illum(m.cell_faces, m.face_area, fv, I1, d)
        n2 = oracle.ref_recalc_illum(m.cell_faces, m.face_area, fv, I2, d, RAD)
        assert n1 == n2
        assert np.array_equal(I1, I2)
    # the last cell is a plain mean, every other an area-weighted one
    cf = m.cell_faces
    assert I1[-1, 0] == ((fv[cf[-1, 0]] + fv[cf[-1, 1]]) + fv[cf[-1, 2]] + fv[cf[-1, 3]]) / 4


def _python_sweep(m, dirs, alpha, betta, Q, S, bc):
    """Independent restatement: the out-face nodes (4P + Q + R) / 6 traced back
    along -w through the cell planes n.x = n.V taken from the vertices, each face
    value from the reference's GetIllum and GetRhsOpt-equivalent, each cell value
    from the reference's ReCalcIllumOpt."""
    N, F = m.n_cells, m.n_faces
    G = Q.shape[1]
    M = len(dirs)
    nb = oracle.loader.sweep_neighbours(m)
    V = m.vertices[m.cell_vertices]  # [N][4][3]
    sign = np.where((m.cell_sign[:, None] >> np.arange(4)) & 1, 1.0, -1.0)
    n = m.face_n[m.cell_faces] * sign[..., None]  # [N][4][3]
    d = np.einsum("cjx,cjx->cj", n, V[:, [1, 2, 3, 0]])  # face j holds vertex j+1
    I = np.zeros((N * G, M))
    for dd in range(M):
        w = dirs[dd]
        fv = np.full((F, G), bc)
        cos = n @ w
        indeg = ((cos < 0) & (nb >= 0)).sum(1)
        queue = list(np.nonzero(indeg == 0)[0])
        qh = 0
        while qh < len(queue):
            c = queue[qh]
            qh += 1
            for j in range(4):
                if not cos[c, j] > 0:
                    continue
                vi = [(j + 1) & 3, (j + 2) & 3, (j + 3) & 3]
                hs, ss = [], []
                for q in range(3):
                    x = (V[c, vi[q]] * 4.0 + V[c, vi[(q + 1) % 3]] + V[c, vi[(q + 2) % 3]]) / 6.0
                    best = None
                    for h in range(4):
                        if cos[c, h] < 0:
                            t = (n[c, h] @ x - d[c, h]) / cos[c, h]
                            if best is None or t < best[0]:
                                best = (t, h)
                    hs.append(best[1])
                    ss.append(max(best[0], 0.0))
                for g in range(G):
                    I0 = [fv[m.cell_faces[c, h], g] if nb[c, h] >= 0 else bc for h in hs]
                    rhs, k = oracle.port_get_rhs(alpha[c], betta[c], Q[c, g], S[c * G + g, dd])
                    fv[m.cell_faces[c, j], g] = oracle.ref_get_illum(I0, ss, k, rhs, RAD)
                if nb[c, j] >= 0:
                    indeg[nb[c, j]] -= 1
                    if indeg[nb[c, j]] == 0:
                        queue.append(nb[c, j])
        assert len(queue) == N
        for g in range(G):
            col = np.ascontiguousarray(I[g::G, :])
            oracle.ref_recalc_illum(m.cell_faces, m.face_area, fv[:, g], col, dd, RAD)
            I[g::G, dd] = col[:, dd]
    return I


def _inputs(m, M, G, seed):
    rng = np.random.default_rng(seed)
    dirs = fibonacci_directions(M).dirs
    alpha = 10 ** rng.uniform(-1, 1.5, m.n_cells)
    betta = 0.5 * alpha
    Q = 10 ** rng.uniform(-2, 0, (m.n_cells, G))
    S = 10 ** rng.uniform(-3, -1, (m.n_cells * G, M))
    return dirs, alpha, betta, Q, S


def test_sweep_matches_vertex_traced_sweep():
    need(RAD)
    m = kuhn_box(3, 3, 2, lo=(-1, -1, -1), hi=(1, 1, 1), seed=4, with_vertices=True)
    dirs, alpha, betta, Q, S = _inputs(m, 6, 2, 5)
    Ip, missing = oracle.port_sweep(m, dirs, alpha, betta, Q, S, bc=0.0)
    assert missing == 0
    Ir = _python_sweep(m, dirs, alpha, betta, Q, S, 0.0)
    # same arithmetic except how the node distances are formed (heights vs planes)
    assert np.max(np.abs(Ip - Ir) / np.abs(Ir)) < 1e-12


def test_sweep_physical_limits():
    """Optically thick, no scattering: every cell away from the boundary (whose face
    mean includes the inflow boundary value) tends to the source Q;
    optically thin with zero source and zero inflow: everything stays 0; groups
    are independent."""
    m = kuhn_box(6, 6, 6, lo=(-1, -1, -1), hi=(1, 1, 1), seed=6)
    M, G = 16, 3
    dirs = fibonacci_directions(M).dirs
    Q = np.tile([1.0, 2.0, 3.0], (m.n_cells, 1))
    S = np.zeros((m.n_cells * G, M))
    thick = np.full(m.n_cells, 1e4)
    I, missing = oracle.port_sweep(m, dirs, thick, np.zeros(m.n_cells), Q, S)
    assert missing == 0
    inner = np.all(oracle.sweep_neighbours(m) >= 0, axis=1)
    assert inner.sum() > 100
    assert np.allclose(I.reshape(m.n_cells, G, M)[inner], Q[inner][:, :, None], rtol=1e-12)
    I0, _ = oracle.port_sweep(m, dirs, np.full(m.n_cells, 1e-3), np.full(m.n_cells, 1e-3), 0 * Q, S)
    assert np.all(I0 == 0)
    # a uniform inflow bc through an absorbing-free, source-free medium is carried unchanged
    Ib, _ = oracle.port_sweep(m, dirs, np.full(m.n_cells, 1e-8), np.zeros(m.n_cells), 0 * Q, S, bc=2.0)
    assert np.allclose(Ib, 2.0, rtol=1e-7)


def test_sweep_has_no_cycles_on_jittered_kuhn_mesh():
    m = kuhn_box(10, 10, 10, lo=(-1, -1, -1), hi=(1, 1, 1), seed=7)
    dirs, alpha, betta, Q, S = _inputs(m, 64, 1, 8)
    _, missing = oracle.port_sweep(m, dirs, alpha, betta, Q, S)
    assert missing == 0
