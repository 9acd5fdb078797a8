"""Pins the oracle (C restatement) to the reference compiled from its own
sources (oracle/_ref).  CPU only.  Bar: bit-identical, except where the CPU
reference averages four replicated face values (illum's face layout), whose
summation 0+x+x+x+x can round once: there 2 ulp.

Skipped where oracle/_ref was not built (no reference tree); the committed
golden fixtures (tests/test_golden.py) pin the oracle there.
"""
import numpy as np
import pytest

import oracle
from cases import GAMMA_43, GAMMA_53, JET_INFLOW, c2p_states, intensity, jet, shock_tube
from radrhd_solver_b200.mesh import fibonacci_directions

VARIANTS = [("hydro_ideal_5_3", 1, GAMMA_53), ("hydro_ideal_4_3", 1, GAMMA_43), ("hydro_taub", 2, GAMMA_53)]


def need(v):
    if not oracle.have_ref(v):
        pytest.skip(f"reference variant {v} not built")


@pytest.mark.parametrize("variant,eos,gamma", VARIANTS)
def test_c2p_p2c_pfix(variant, eos, gamma):
    need(variant)
    W = c2p_states(4000, gamma, seed=eos + 10)
    W[:40, 1:4] *= 1.3
    Wp, Up = oracle.port_p2c(W, eos, gamma)
    Wr, Ur = oracle.ref_p2c(W, variant)
    assert np.array_equal(Up, Ur) and np.array_equal(Wp, Wr)
    Wc, cp = oracle.port_c2p(Up, eos, gamma)
    Wcr, cr = oracle.ref_c2p(Up, variant)
    assert np.array_equal(cp, cr)
    assert np.array_equal(Wc[cp == 0], Wcr[cr == 0])
    assert (cp == 0).mean() > 0.9
    U2 = Up.copy()
    U2[:, 4] *= 0.7  # push many states into the fallback
    a = oracle.port_pressure_fix(U2, Wp, eos, gamma)
    b = oracle.ref_pressure_fix(U2, Wp, variant)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("variant,eos,gamma", VARIANTS)
def test_flux_random_faces(variant, eos, gamma):
    need(variant)
    rng = np.random.default_rng(3)
    n = 3000
    WL = c2p_states(n, gamma, seed=1)
    WR = c2p_states(n, gamma, seed=2)
    WL, UL = oracle.port_p2c(WL, eos, gamma)
    WR, UR = oracle.port_p2c(WR, eos, gamma)
    nv = rng.normal(size=(n, 3))
    nv[:30] = [0, 0, 1]
    nv[30:60] = [0, 0, -1]
    nv /= np.linalg.norm(nv, axis=1)[:, None]
    S = rng.uniform(0.1, 2, n)
    Fp, sp = oracle.port_flux(UL, UR, WL, WR, nv, S, eos, gamma)
    Fr, sr = oracle.ref_flux(UL, UR, WL, WR, nv, S, variant)
    assert np.array_equal(Fp, Fr, equal_nan=True) and np.array_equal(sp, sr, equal_nan=True)


def test_hydro_steps_shock_tube():
    need("hydro_ideal_5_3")
    m, W = shock_tube(40, 4, 4)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    h = oracle.HydroRef(m, "hydro_ideal_5_3")
    h.set_state(W, U)
    tau = 0.3 * m.h_min
    for k in range(15):
        U, W, Ff, st, v = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53)
        vr = h.step(tau, 2)
        Wr, Ur = h.get_state()
        assert np.array_equal(U, Ur) and np.array_equal(W, Wr) and v == vr, k
        assert np.array_equal(Ff, h.face_flux())
        tau = oracle.port().orc_time_step(0.3, m.h_min, v)
        assert tau == h.lib.ref_time_step(0.3, m.h_min, vr)


def test_hydro_steps_jet_inflow():
    need("hydro_ideal_4_3")
    m, W = jet(8)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    h = oracle.HydroRef(m, "hydro_ideal_4_3")
    Ubc = np.zeros(5)
    h.lib.ref_p2c_plain(JET_INFLOW.ctypes.data, Ubc.ctypes.data, 1)
    h.set_bc(-3, 1, JET_INFLOW, Ubc)
    h.set_state(W, U)
    bc = {-3: (1, JET_INFLOW, Ubc)}
    # tau = CFL h_min / c: the reference's signed max signal speed
    # (rhllc_flux_stab.cpp:430) misses the inflow's wave travelling against the
    # face normal, and GetTimeStep would then break the CFL condition.
    tau = 0.3 * m.h_min
    codes = np.zeros(m.n_cells, np.int32)
    for k in range(8):
        U, W, _, st, v = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_43, bc=bc)
        vr = h.step(tau, 2, codes)
        Wr, Ur = h.get_state()
        assert np.isfinite(U).all()
        assert np.array_equal(U, Ur) and np.array_equal(W, Wr) and v == vr, k
        assert np.array_equal(st, codes)


def test_scatter_and_moments():
    need("illum")
    M = 96
    d = fibonacci_directions(M)
    I = intensity(300, M, seed=2)
    Sp = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Sr = oracle.ref_scatter(I, d.dirs, d.areas, d.full_area)
    # face-layout average (0+x+x+x+x)/4 of the CPU reference
    assert np.all(np.abs(Sp - Sr) <= 2 * np.spacing(np.abs(Sr)))
    assert (Sp == Sr).mean() > 0.99
    Ep, Fp, Tp = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
    Er, Fr, Tr = oracle.ref_moments(I, d.dirs, d.areas, d.full_area)
    for p, r in ((Ep, Er), (Fp, Fr), (Tp, Tr)):
        assert np.all(np.abs(p - r) <= 2 * np.spacing(np.abs(r)))


def test_scatter_reference_direction_file():
    """The reference's own 26-direction test sphere (full_area 9.99, not 4 pi):
    normalisation by the file's full_area."""
    import os

    from conftest import REFERENCE
    path = os.path.join(REFERENCE, "tests", "data", "surface_26_dir.txt")
    if not os.path.exists(path):
        pytest.skip("reference tree not present")
    need("illum")
    from radrhd_solver_b200.mesh import read_sphere_directions
    d = read_sphere_directions(path)
    assert d.size == 26 and abs(d.full_area - 4 * np.pi) > 1
    I = intensity(50, 26, seed=9)
    Sp = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Sr = oracle.ref_scatter(I, d.dirs, d.areas, d.full_area)
    assert np.all(np.abs(Sp - Sr) <= 2 * np.spacing(np.abs(Sr)))


def test_rad_source_and_constants():
    need("rad_ideal_4_3")
    import ctypes
    from radrhd_solver_b200 import rad_rhd
    c = np.zeros(4)
    oracle.ref("rad_ideal_4_3").ref_rad_constants(c.ctypes.data)
    em = rad_rhd.reference_emission()
    assert (em.temp_coef, em.sigma_sb, em.pi, em.rad_unit) == tuple(c)
    rng = np.random.default_rng(5)
    n = 500
    W = np.stack([10 ** rng.uniform(-2, 1, n), rng.uniform(-.5, .5, n), rng.uniform(-.5, .5, n),
                  rng.uniform(-.5, .5, n), 10 ** rng.uniform(-14, -10, n)], 1)
    alpha, sigma = W[:, 0].copy(), 0.5 * W[:, 0]
    E = 10 ** rng.uniform(-3, 0, n)
    F = rng.uniform(-1, 1, (n, 3)) * E[:, None] * 0.3
    T = rng.uniform(0, 1, (n, 3, 3)) * E[:, None, None]
    Gp = oracle.port_rad_source(W, alpha, sigma, E, F, T, tuple(c))
    Gr = oracle.ref_rad_source(W, alpha, sigma, E, F, T)
    assert np.array_equal(Gp, Gr)
    del ctypes
