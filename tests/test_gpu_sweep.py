"""GPU transport sweep and coupled radiation-hydro step against the oracle.

Bars: the FP64 sweep within 1e-12 relative of orc_sweep per cell, direction and
group (every operation is the oracle's in the oracle's order; only exp comes
from CUDA's libm instead of glibc); the FP32 sweep within 1e-5.  The plain
coupled step (FP64 sweep, FP64 scattering, reference con2prim guess) within
1e-12 of the oracle's composition of the same step; the chosen form (FP32 sweep,
tensor-core scattering, learned con2prim guess) keeps the hydro state within
1e-10 of the plain form.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_43, JET_INFLOW, c2p_states, jet
from radrhd_solver_b200 import _lib as L
from radrhd_solver_b200 import illum, rad_rhd, rhllc
from radrhd_solver_b200.c2p_mlp import LearnedGuess
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box

pytestmark = pytest.mark.gpu


def _inputs(m, M, G, seed):
    rng = np.random.default_rng(seed)
    alpha = 10 ** rng.uniform(-1, 1.5, m.n_cells)
    betta = 0.5 * alpha
    Q = 10 ** rng.uniform(-2, 0, (m.n_cells, G))
    S = 10 ** rng.uniform(-3, -1, (m.n_cells * G, M))
    return alpha, betta, Q, S


def _run_sweep(m, d, G, precision, dirs_per_batch=0, renumber=True, inputs=None, bc=0.0):
    grid = rhllc.Grid(m, gamma=GAMMA_43, renumber=renumber)
    dg = illum.DirectionGrid(d)
    sw = illum.TransportSweep(grid, dg, groups=G, precision=precision, dirs_per_batch=dirs_per_batch,
                              boundary_value=bc)
    dt = torch.float64 if precision == "fp64" else torch.float32
    t = [torch.tensor(a, dtype=dt, device="cuda").contiguous() for a in inputs]
    torch.cuda.synchronize()
    I = illum.CalculateIllum(sw, *t)
    grid.sync()
    out = I.double().cpu().numpy()
    info = sw.plan_info()
    grid.close()
    return out, info


@pytest.mark.parametrize("dirs_per_batch", [0, 4])
def test_sweep_fp64_matches_oracle(dirs_per_batch):
    m = kuhn_box(6, 5, 4, lo=(-1, -1, -1), hi=(1, 1, 1), seed=21)
    d = fibonacci_directions(24)
    G = 3
    inp = _inputs(m, d.size, G, 22)
    Io, missing = oracle.port_sweep(m, d.dirs, *inp)
    assert missing == 0
    Ig, (levels, biggest) = _run_sweep(m, d, G, "fp64", dirs_per_batch, inputs=inp)
    assert levels > 0 and biggest > 0
    err = np.max(np.abs(Ig - Io) / np.abs(Io))
    print(f"\nfp64 sweep: max rel err {err:.2e}, {levels} levels, largest {biggest}")
    assert err <= 1e-12


def test_sweep_fp32_and_boundary_value():
    m = kuhn_box(7, 6, 5, lo=(-1, -1, -1), hi=(1, 1, 1), seed=23)
    d = fibonacci_directions(32)
    G = 2
    inp = _inputs(m, d.size, G, 24)
    Io, _ = oracle.port_sweep(m, d.dirs, *inp, bc=0.25)
    Ig, _ = _run_sweep(m, d, G, "fp32", inputs=inp, bc=0.25)
    err = np.max(np.abs(Ig - Io) / np.abs(Io))
    print(f"\nfp32 sweep: max rel err {err:.2e}")
    assert err <= 1e-5


def test_sweep_independent_of_cell_numbering():
    """The plan is built in the context's own cell order; results in the caller's
    numbering are the same bit for bit with and without renumbering."""
    m = kuhn_box(5, 5, 5, lo=(-1, -1, -1), hi=(1, 1, 1), seed=25)
    d = fibonacci_directions(16)
    inp = _inputs(m, d.size, 1, 26)
    a, _ = _run_sweep(m, d, 1, "fp64", inputs=inp, renumber=True)
    b, _ = _run_sweep(m, d, 1, "fp64", inputs=inp, renumber=False)
    assert np.array_equal(a, b)


def test_sweep_errors():
    m = kuhn_box(3, 3, 3, seed=27)
    grid = rhllc.Grid(m, gamma=GAMMA_43)
    x = torch.zeros(m.n_cells, dtype=torch.float64, device="cuda")
    st = L.lib.rrhd_sweep(grid.handle, L.ptr(x), L.ptr(x), L.ptr(x), L.ptr(x), L.ptr(x))
    assert st == L.RRHD_ERR_STATE
    dg = illum.DirectionGrid(fibonacci_directions(8))
    o = L.RadOpts(1, L.RRHD_RAD_FP64, 3, 0.0)  # not a power of two
    assert L.lib.rrhd_rad_setup(grid.handle, dg.handle, C.byref(o)) == L.RRHD_ERR_INVALID
    sw = illum.TransportSweep(grid, dg, groups=1, precision="fp64")
    step = rad_rhd.RadRHDStep(sw, scatter="f16x3")  # tensor-core scattering needs the fp32 sweep
    st = L.lib.rrhd_coupled_step(grid.handle, 1e-3, C.byref(step.opts), None, None)
    assert st == L.RRHD_ERR_INVALID
    grid.close()


# ------------------------------------------------------------------ coupled step
EM = (1.0, 1.0e4, np.pi, 1.0)  # temp_coef, sigma_sb (a_R), pi, kRadiation: radiation that moves the gas
EM_JET = (1.0, 10.0, np.pi, 1.0)  # the coupled-jet benchmark's constants (a_R = 10 in code units)


def _inflow_bc():
    ubc = np.zeros(5)
    e = oracle.loader.OrcEos(1, GAMMA_43)
    oracle.port().orc_p2c_plain(C.byref(e), np.ascontiguousarray(JET_INFLOW).ctypes.data, ubc.ctypes.data)
    return {-3: (1, JET_INFLOW, ubc)}


def _sum_groups(x, G):
    """Rows cell*G+g summed over g in order, starting from 0 (the kernel's order)."""
    x = x.reshape((-1, G) + x.shape[1:])
    s = np.zeros((x.shape[0],) + x.shape[2:])
    for g in range(G):
        s = s + x[:, g]
    return s


def _oracle_coupled(m, U, W, tau, d, G, S, mom, a=1.0, b=0.5):
    """The oracle's composition of one coupled step (radRHD_main.cpp:96-139)."""
    U, W, _, _, _ = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_43, bc=_inflow_bc())
    rho, p = W[:, 0], W[:, 4]
    alpha, betta = a * rho, b * rho
    T = EM[0] * p / rho
    T2 = T * T
    B = (T2 * T2) * EM[1] / EM[2]
    Q = np.repeat((B / EM[3] / G)[:, None], G, axis=1)
    I, missing = oracle.port_sweep(m, d.dirs, alpha, betta, Q, S)
    assert missing == 0
    E, F, Tm = mom
    G4 = oracle.port_rad_source(W, alpha, betta, E, F, Tm, EM)
    U = U.copy()
    U[:, 4] += tau * G4[:, 0]
    U[:, 1] += tau * G4[:, 1]
    U[:, 2] += tau * G4[:, 2]
    U[:, 3] += tau * G4[:, 3]
    W, _ = oracle.port_c2p(U, 1, GAMMA_43, W=W)
    S = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Er, Fr, Tr = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
    mom = (_sum_groups(Er, G), _sum_groups(Fr, G), _sum_groups(Tr, G))
    return U, W, I, S, mom, G4


def _coupled_grid(m, W, U, d, G, precision):
    g = rhllc.Grid(m, gamma=GAMMA_43)
    g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
    g.set_state(W, U)
    dg = illum.DirectionGrid(d)
    sw = illum.TransportSweep(g, dg, groups=G, precision=precision)
    return g, dg, sw


def test_coupled_plain_matches_oracle():
    m, W = jet(6)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(64)
    G = 2
    g, dg, sw = _coupled_grid(m, W, U, d, G, "fp64")
    step = rad_rhd.RadRHDStep(sw, absorption=1.0, scattering=0.5, em=rad_rhd.emission(*EM), scatter="fp64")
    tau = 0.3 * m.h_min
    S = np.zeros((m.n_cells * G, d.size))
    mom = (np.zeros(m.n_cells), np.zeros((m.n_cells, 3)), np.zeros((m.n_cells, 3, 3)))
    Uo, Wo = U, W
    for k in range(3):
        hs, ss = step(tau, stats=True)
        Uo, Wo, Io, S, mom, G4o = _oracle_coupled(m, Uo, Wo, tau, d, G, S, mom)
        assert ss.n_failed == 0
    Wg, Ug = g.get_state()
    Ig, Sg, G4g = step.get("I"), step.get("S"), step.get("G4")
    assert np.abs(G4o).max() > 0
    rel = lambda a, b: np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
    print(f"\nI {rel(Ig, Io):.2e} S {rel(Sg, S):.2e} G4 {np.max(np.abs(G4g - G4o)) / np.abs(G4o).max():.2e} "
          f"U {np.max(np.abs(Ug - Uo) / np.abs(Uo).max(0)):.2e}")
    assert rel(Ig, Io) <= 1e-12
    assert rel(Sg, S) <= 1e-12
    assert np.max(np.abs(G4g - G4o)) <= 1e-12 * np.abs(G4o).max()
    assert np.all(np.abs(Ug - Uo) <= 1e-12 * np.abs(Uo).max(0))
    assert np.all(np.abs(Wg - Wo) <= 1e-12 * np.abs(Wo).max(0))
    g.close()


def _trained_guess():
    Wc = c2p_states(200_000, GAMMA_43, seed=31)
    Wc, Uc = oracle.port_p2c(Wc, 1, GAMMA_43)
    net = LearnedGuess(seed=3)
    net.train(torch.tensor(Uc, device="cuda"), torch.tensor(Wc[:, 4], device="cuda"), epochs=3, batch=2048,
              lr=2e-3, seed=4)
    return net


def test_coupled_chosen_form_tracks_plain():
    m, W = jet(8)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(64)
    G = 2
    tau = 0.3 * m.h_min
    net = _trained_guess()
    out = {}
    for form in ("plain", "chosen"):
        g, dg, sw = _coupled_grid(m, W, U, d, G, "fp64" if form == "plain" else "fp32")
        step = rad_rhd.RadRHDStep(sw, em=rad_rhd.emission(*EM_JET), scatter="fp64" if form == "plain" else "f16x3",
                                  guess=None if form == "plain" else net)
        stats = [step(tau, stats=True) for _ in range(3)]
        Wg, Ug = g.get_state()
        out[form] = (Ug, Wg, step.get("I"), stats)
        g.close()
    Up, Wp, Ip, sp = out["plain"]
    Uc, Wc, Ic, sc = out["chosen"]
    it_p = sum(s[1].newton_iters for s in sp)
    it_c = sum(s[1].newton_iters for s in sc)
    du = np.max(np.abs(Uc - Up) / np.abs(Up).max(0))
    dI = np.max(np.abs(Ic - Ip) / np.abs(Ip).max())
    print(f"\nchosen vs plain: U {du:.2e}, I {dI:.2e}; source con2prim Newton iterations {it_c} vs {it_p}")
    assert np.all(np.abs(Uc - Up) <= 1e-10 * np.abs(Up).max(0))
    assert np.all(np.abs(Wc - Wp) <= 1e-10 * np.abs(Wp).max(0))
    assert dI <= 1e-4
    assert all(s[1].n_failed == 0 for s in sc)


def test_coupled_chosen_row_scales_from_cell_pass():
    """With one batch of 256 directions the sweep's cell pass hands the FP16 scattering
    its row scales; the step is bit-identical to two batches of 128, where the
    scattering computes them itself."""
    m, W = jet(5)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(256)
    out = []
    for db in (256, 128):
        g = rhllc.Grid(m, gamma=GAMMA_43)
        g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
        g.set_state(W, U)
        dg = illum.DirectionGrid(d)
        sw = illum.TransportSweep(g, dg, groups=4, precision="fp32", dirs_per_batch=db)
        step = rad_rhd.RadRHDStep(sw, em=rad_rhd.emission(*EM_JET), scatter="f16x3")
        for _ in range(2):
            step(0.3 * m.h_min)
        Wg, Ug = g.get_state()
        out.append((Ug, step.get("I"), step.get("S")))
        g.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
