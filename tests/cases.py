"""Seeded synthetic inputs shared by the tests (shapes and value ranges of the
benchmark configurations, at sizes the oracle finishes in seconds)."""
from __future__ import annotations

import numpy as np

from radrhd_solver_b200 import mesh as M

GAMMA_53 = 5.0 / 3
GAMMA_43 = 4.0 / 3


def shock_tube(nx=40, ny=4, nz=4, seed=7):
    """Relativistic shock tube on [0,1] x [0,ny/nx] x [0,nz/nx] (cubic hexes;
    200x10x10 is the [0,1]x[0,0.05]^2 benchmark box): left rho=10, p=13.33;
    right rho=1, p=0.01; v=0 (by cell centroid)."""
    m = M.kuhn_box(nx, ny, nz, hi=(1.0, ny / nx, nz / nx), jitter=0.15, seed=seed)
    xc = m.cell_center[:, 0]
    W = np.zeros((m.n_cells, 5))
    W[:, 0] = np.where(xc < 0.5, 10.0, 1.0)
    W[:, 4] = np.where(xc < 0.5, 13.33, 0.01)
    return m, W


JET_INFLOW = np.array([0.01, 0.0, 0.0, np.sqrt(1.0 - 1.0 / 49.0), 1e-3])  # rho, v (W=7 along +z), p


def jet(n=12, seed=11):
    """Coupled-jet mesh: cube [-1,1]^3, ambient rho=1, p=1e-3, v=0; z=-1 faces
    with centroid radius < 0.1 carry code -3 (fixed inflow state JET_INFLOW).
    For small n the nozzle radius is widened so that some faces are inside."""
    r = max(0.1, 2.5 * 2.0 / n)
    m = M.kuhn_box(n, n, n, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=seed, inflow_radius=r,
                   inflow_code=-3, with_vertices=True)
    W = np.zeros((m.n_cells, 5))
    W[:, 0] = 1.0
    W[:, 4] = 1e-3
    return m, W


def c2p_states(n, gamma=GAMMA_43, seed=5):
    """Config-3 style primitive states: rho log-uniform [1e-4,1e2], p/rho
    log-uniform [1e-6,1e2], Lorentz factor log-uniform [1,50], isotropic v."""
    rng = np.random.default_rng(seed)
    rho = 10 ** rng.uniform(-4, 2, n)
    p = rho * 10 ** rng.uniform(-6, 2, n)
    lor = 10 ** rng.uniform(0, np.log10(50), n)
    v = np.sqrt(1 - 1 / lor ** 2)
    mu = rng.uniform(-1, 1, n)
    ph = rng.uniform(0, 2 * np.pi, n)
    s = np.sqrt(1 - mu ** 2)
    W = np.stack([rho, v * s * np.cos(ph), v * s * np.sin(ph), v * mu, p], axis=1)
    return W


def intensity(N, M_, seed=3, centers=None, groups=1):
    """Config-1 style intensity: lognormal(0, 0.5) * exp(-|x|^2/0.2), cell-major
    [N*groups, M]."""
    rng = np.random.default_rng(seed)
    I = np.exp(rng.normal(0.0, 0.5, (N * groups, M_)))
    if centers is not None:
        r2 = (centers ** 2).sum(1)
        I *= np.repeat(np.exp(-r2 / 0.2), groups)[:, None]
    return I


def split_case(nx=40, ny=8, nz=8, seed=4):
    """Shock tube with perturbed density, pressure and velocity in every cell (so that
    every face carries flux), for the hydro step split over ranks."""
    m, W = shock_tube(nx, ny, nz)
    rng = np.random.default_rng(seed)
    W[:, 0] *= 1 + 0.2 * rng.uniform(-1, 1, m.n_cells)
    W[:, 4] *= 1 + 0.2 * rng.uniform(-1, 1, m.n_cells)
    W[:, 1:4] = 0.3 * rng.uniform(-1, 1, (m.n_cells, 3))
    return m, W


SPLIT_POISON = np.array([2.0, 0.0, 0.0, 0.0, 0.5])  # state of the cells a rank neither owns nor receives

COMPTON_SPEEDS = (0.0, 1e-6, 1e-5, 0.3, 0.9, 0.99)


def compton_case(cells, M_, seed=17, speeds=COMPTON_SPEEDS):
    """Inputs of the full-spectrum Compton scattering: intensity [cells][M][100]
    (lognormal(0, 0.5) times a smooth spectral shape) and velocities [cells][3] in
    units of c whose magnitudes cycle through `speeds`: 0 and 1e-6 take the
    recoil-only branch (v^2 below 1/c in CGS), 1e-5 and above the Doppler branch."""
    rng = np.random.default_rng(seed)
    f = np.arange(100)
    shape = np.exp(-((f - 60.0) / 25.0) ** 2) + 0.05
    I = np.exp(rng.normal(0.0, 0.5, (cells, M_, 100))) * shape
    u = rng.normal(size=(cells, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    vel = u * np.array([speeds[i % len(speeds)] for i in range(cells)])[:, None]
    return I, vel


def ray_surface(n_box=12, n_sphere=16, seed=21):
    """Triangle surface for the image-plane ray tracing: the boundary of the box
    [0.43, 1.33] x [-0.35, 0.35] x [-0.25, 0.25] around the centre of mass (n_box x n_box
    quads per side, two triangles each, shared edges as in a mesh boundary) and a
    latitude-longitude sphere of radius 0.08 around the accretor (1, 0, 0) with jittered
    vertices.  Returns unique shuffled ids [n] and vertices [n][9]."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array([0.43, -0.35, -0.25]), np.array([1.33, 0.35, 0.25])
    tris = []
    g = np.linspace(0.0, 1.0, n_box + 1)
    for ax in range(3):
        u, v = [a for a in range(3) if a != ax]
        for side in (0, 1):
            for i in range(n_box):
                for j in range(n_box):
                    q = []
                    for di, dj in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        p = np.empty(3)
                        p[ax] = lo[ax] if side == 0 else hi[ax]
                        p[u] = lo[u] + (hi[u] - lo[u]) * g[i + di]
                        p[v] = lo[v] + (hi[v] - lo[v]) * g[j + dj]
                        q.append(p)
                    tris.append(np.concatenate([q[0], q[1], q[2]]))
                    tris.append(np.concatenate([q[0], q[2], q[3]]))
    c, r = np.array([1.0, 0.0, 0.0]), 0.08
    th = np.linspace(0, np.pi, n_sphere + 1)
    ph = np.linspace(0, 2 * np.pi, 2 * n_sphere + 1)
    P = np.empty((n_sphere + 1, 2 * n_sphere + 1, 3))
    for a in range(n_sphere + 1):
        for b in range(2 * n_sphere + 1):
            rr = r * (1 + (0.05 * rng.uniform(-1, 1) if 0 < a < n_sphere else 0))
            P[a, b] = c + rr * np.array([np.sin(th[a]) * np.cos(ph[b % (2 * n_sphere)]),
                                         np.sin(th[a]) * np.sin(ph[b % (2 * n_sphere)]), np.cos(th[a])])
    for a in range(n_sphere):
        for b in range(2 * n_sphere):
            tris.append(np.concatenate([P[a, b], P[a + 1, b], P[a + 1, b + 1]]))
            tris.append(np.concatenate([P[a, b], P[a + 1, b + 1], P[a, b + 1]]))
    abc = np.array(tris)
    ids = rng.permutation(4 * len(abc))[:len(abc)].astype(np.int32)
    return ids, abc
