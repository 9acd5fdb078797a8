"""GPU parity of the hydro path (C ABI) against the oracle.

Bar: bit-identical.  The CUDA FP64 kernels are compiled with --fmad=false and
perform the reference's operations in the reference's order, so every field
of every cell equals the oracle exactly (tolerance 0).
"""
import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_43, GAMMA_53, JET_INFLOW, c2p_states, jet, shock_tube
from radrhd_solver_b200 import rhllc

pytestmark = pytest.mark.gpu


def _grid(m, gamma, eos=1, **kw):
    return rhllc.Grid(m, eos=eos, gamma=gamma, **kw)


@pytest.mark.parametrize("eos,gamma", [(1, GAMMA_53), (1, GAMMA_43), (2, GAMMA_53)])
def test_con2prim_batch_bitexact(eos, gamma):
    W0 = c2p_states(20000, gamma, seed=eos)
    W0, U = oracle.port_p2c(W0, eos, gamma)
    Wo, codes = oracle.port_c2p(U, eos, gamma)
    Ud = torch.tensor(U, device="cuda")
    Wd = torch.zeros_like(Ud)
    st = torch.zeros(len(U), dtype=torch.uint8, device="cuda")
    rhllc.GetPhysValueStab(Ud, Wd, st, eos=eos, gamma=gamma, fallback=False,
                           stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ok = codes == 0
    assert np.array_equal(st.cpu().numpy().astype(np.int32), codes)
    assert np.array_equal(Wd.cpu().numpy()[ok], Wo[ok])


def test_con2prim_stats_matches_oracle():
    """Batch con2prim with totals: states, status bytes and the iteration
    statistics equal the oracle's; a batch spanning many CTAs and a ragged tail."""
    W0 = c2p_states(70001, GAMMA_43, seed=21)
    W0, U = oracle.port_p2c(W0, 1, GAMMA_43)
    U[::97, 4] *= 0.6  # some states go to the fallback
    Wo, codes = oracle.port_c2p(U, 1, GAMMA_43, W=W0)
    Uf, Wf, fix = oracle.port_pressure_fix(U, np.where(codes[:, None] == 0, Wo, W0), 1, GAMMA_43)
    Ud = torch.tensor(U, device="cuda")
    Wd = torch.tensor(W0, device="cuda")
    sd = torch.zeros(len(U), dtype=torch.uint8, device="cuda")
    st = rhllc.GetPhysValueStabStats(Ud, Wd, sd, eos=1, gamma=GAMMA_43, fallback=True,
                                     stream=torch.cuda.current_stream().cuda_stream)
    bad = codes != 0
    assert st.n_ok == (~bad).sum() and st.n_fallback == bad.sum() and st.n_failed == ((fix != 0) & bad).sum()
    Wg = Wd.cpu().numpy()
    assert np.array_equal(Wg[~bad], Wo[~bad])
    assert np.array_equal(Wg[bad & (fix == 0)], Wf[bad & (fix == 0)])
    assert 0 < st.newton_iters / len(U) < 40 and 0 < st.max_iters <= 40
    st0 = rhllc.GetPhysValueStabStats(Ud[:0], Wd[:0], None, eos=1, gamma=GAMMA_43,
                                      stream=torch.cuda.current_stream().cuda_stream)
    assert st0.n_ok == 0 and st0.newton_iters == 0


def test_prim2con_batch_bitexact():
    W = c2p_states(5000, GAMMA_43, seed=9)
    W[:50, 1:4] *= 1.5  # |v| >= 1: rescaled by 0.9999 as in GetConvValueStab
    Wo, Uo = oracle.port_p2c(W, 1, GAMMA_43)
    Wd = torch.tensor(W, device="cuda")
    Ud = torch.zeros_like(Wd)
    rhllc.GetConvValueStab(Wd, Ud, eos=1, gamma=GAMMA_43, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(Ud.cpu().numpy(), Uo)
    assert np.array_equal(Wd.cpu().numpy(), Wo)


def test_con2prim_fallback_and_codes():
    """Poisoned states: E below sqrt(m^2+D^2) (code 1) and NaN: the status byte
    and the PhysPressureFix result match the oracle; nothing aborts."""
    W = c2p_states(64, GAMMA_53, seed=2)
    _, U = oracle.port_p2c(W, 1, GAMMA_53)
    U[:16, 4] = np.sqrt((U[:16, 1:4] ** 2).sum(1) + U[:16, 0] ** 2) * 0.999  # no solution
    U[16:20, 4] = np.nan
    Wo, codes = oracle.port_c2p(U, 1, GAMMA_53, W=W)
    Uf, Wf, fix = oracle.port_pressure_fix(U, np.where(codes[:, None] == 0, Wo, W), 1, GAMMA_53)
    Ud = torch.tensor(U, device="cuda")
    Wd = torch.tensor(W, device="cuda")
    st = torch.zeros(len(U), dtype=torch.uint8, device="cuda")
    rhllc.GetPhysValueStab(Ud, Wd, st, eos=1, gamma=GAMMA_53, fallback=True,
                           stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    s = st.cpu().numpy().astype(np.int32)
    exp = np.where(codes != 0, codes | 0x10 | np.where(fix != 0, 0x20, 0), 0)
    assert np.array_equal(s, exp)
    bad = codes != 0
    good_fix = bad & (fix == 0)
    assert np.array_equal(Wd.cpu().numpy()[good_fix], Wf[good_fix])
    assert np.array_equal(Ud.cpu().numpy()[good_fix], Uf[good_fix])


@pytest.mark.parametrize("cpb", [64, 256])
def test_shock_tube_steps_bitexact(cpb):
    """20 steps of the shock tube, tau from the previous step's max speed; state,
    face fluxes and max speed equal the oracle bit for bit every step."""
    m, W = shock_tube(40, 4, 4)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    g = _grid(m, GAMMA_53, cells_per_block=cpb)
    g.set_state(W, U)
    g.keep_face_flux(True)
    tau = 0.3 * m.h_min / 1.0
    for k in range(20):
        st = rhllc.Hllc3dStab(tau, g)
        U, W, Ff, status, vmax = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53)
        Wg, Ug = g.get_state()
        assert np.array_equal(Ug, U), f"step {k}: U differs, max {np.abs(Ug - U).max()}"
        assert np.array_equal(Wg, W), f"step {k}: W differs"
        assert np.array_equal(g.face_flux(), Ff), f"step {k}: face flux differs"
        assert st.max_speed == vmax
        tau = 0.3 * m.h_min / vmax
    g.close()


def test_step_fallback_path_bitexact():
    """Cells whose con2prim fails inside the step take the PhysPressureFix
    fallback pass; state and status bytes equal the oracle's."""
    m, W = shock_tube(24, 3, 3, seed=6)
    W[:, 1] = 0.5
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    bad = np.arange(0, m.n_cells, 17)
    U[bad, 4] = np.sqrt((U[bad, 1:4] ** 2).sum(1) + U[bad, 0] ** 2) * 0.97  # no solution after the update
    g = _grid(m, GAMMA_53)
    g.set_state(W, U)
    tau = 0.1 * m.h_min
    st = rhllc.Hllc3dStab(tau, g)
    U2, W2, _, status, v = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53)
    assert (status & 0x10).sum() > 0 and st.n_fallback == (status & 0x10).astype(bool).sum()
    Wg, Ug = g.get_state()
    assert np.array_equal(Ug, U2) and np.array_equal(Wg, W2)
    assert np.array_equal(g.cell_status().astype(np.int32), status)


def test_taub_eos_steps_bitexact():
    m, W = shock_tube(24, 3, 3, seed=4)
    W[:, 1] = 0.3  # moving gas
    W, U = oracle.port_p2c(W, 2, GAMMA_53)
    g = _grid(m, GAMMA_53, eos=2)
    g.set_state(W, U)
    tau = 0.25 * m.h_min
    for k in range(5):
        rhllc.Hllc3dStab(tau, g)
        U, W, _, _, _ = oracle.port_hydro_step(m, U, W, tau, 2, GAMMA_53)
    Wg, Ug = g.get_state()
    assert np.array_equal(Ug, U) and np.array_equal(Wg, W)


def _inflow_bc():
    import ctypes
    ubc = np.zeros(5)
    e = oracle.loader.OrcEos(1, GAMMA_43)
    oracle.port().orc_p2c_plain(ctypes.byref(e), np.ascontiguousarray(JET_INFLOW).ctypes.data, ubc.ctypes.data)
    return {-3: (1, JET_INFLOW, ubc)}


def test_jet_inflow_bitexact():
    """Jet mesh with the fixed-state nozzle (code -3) and transmissive walls.
    tau = CFL h_min / c (the reference's signed max speed would under-estimate
    the inflow wave and break the CFL condition)."""
    m, W = jet(10)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    g = _grid(m, GAMMA_43)
    g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
    g.set_state(W, U)
    bc = _inflow_bc()
    tau = 0.3 * m.h_min
    for k in range(8):
        st = rhllc.Hllc3dStab(tau, g)
        U, W, _, status, vmax = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_43, bc=bc)
        assert st.max_speed == vmax
    Wg, Ug = g.get_state()
    assert np.isfinite(U).all()
    assert np.array_equal(Ug, U) and np.array_equal(Wg, W)
    assert np.array_equal(g.cell_status().astype(np.int32), status)
    assert (W[:, 3] > 0.1).sum() > 0  # the jet has entered


def test_device_time_step():
    """tau <= 0: tau = CFL h_min / (previous step's max speed) computed on the
    device (rhllc::GetTimeStep), no host round trip."""
    m, W = shock_tube(30, 3, 3, seed=12)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    g = _grid(m, GAMMA_53)
    g.set_state(W, U)
    g.set_time_step(0.3, m.h_min, 1.0)
    vmax = 1.0
    for k in range(6):
        rhllc.Hllc3dStab(0.0, g)
        tau = 0.3 * m.h_min / vmax
        U, W, _, _, vmax = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53)
        t_used, v_dev = g.step_info()
        assert t_used == tau and v_dev == vmax
    Wg, Ug = g.get_state()
    assert np.array_equal(Ug, U) and np.array_equal(Wg, W)


def test_reflecting_wall_bitexact():
    m, W = shock_tube(16, 2, 2, seed=8)
    m.face_id_r[m.face_id_r < 0] = -2
    W[:, 1] = 0.2
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    g = _grid(m, GAMMA_53)
    g.set_boundary(-2, rhllc.BC_REFLECT)
    g.set_state(W, U)
    tau = 0.2 * m.h_min
    for _ in range(3):
        rhllc.Hllc3dStab(tau, g)
        U, W, _, _, _ = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53, bc={-2: (2, None, None)})
    Wg, Ug = g.get_state()
    assert np.array_equal(Ug, U) and np.array_equal(Wg, W)


def test_conservation_to_roundoff():
    """Interior face fluxes enter two cells with opposite signs, so per step
    sum_i U_i V_i changes only by tau * (net boundary flux), to round-off."""
    m, W = shock_tube(30, 3, 3, seed=5)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    g = _grid(m, GAMMA_53)
    g.set_state(W, U)
    g.keep_face_flux(True)
    V = m.cell_volume
    bnd = m.face_id_r < 0
    tau = 0.3 * m.h_min
    _, Ug = g.get_state()
    for _ in range(5):
        tot0 = (Ug * V[:, None]).sum(0)
        rhllc.Hllc3dStab(tau, g)
        _, Ug = g.get_state()
        tot1 = (Ug * V[:, None]).sum(0)
        net = g.face_flux()[bnd].sum(0)
        scale = (np.abs(Ug) * V[:, None]).sum(0) + 1e-300
        assert np.all(np.abs(tot1 - tot0 + tau * net) <= 1e-13 * scale)


def test_host_dropin_matches_device_path():
    m, W = shock_tube(20, 2, 2, seed=9)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    g = _grid(m, GAMMA_53)
    Wh = W.copy()
    Uh = U.copy()
    from radrhd_solver_b200 import _lib as L
    import ctypes
    st = L.StepStats()
    tau = 0.3 * m.h_min
    L.check(L.lib.rrhd_hydro_step_host(g.handle, tau, L.ptr(Wh), L.ptr(Uh), 5, ctypes.byref(st)))
    U2, W2, _, _, v = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53)
    assert np.array_equal(Uh, U2) and np.array_equal(Wh, W2) and st.max_speed == v
    # strided records (elem_t-like stride 17 doubles)
    rec = np.zeros((m.n_cells, 17))
    rec[:, 0:5] = W
    rec[:, 5:10] = U
    Wv = rec[:, 0:5]
    L.check(L.lib.rrhd_set_state(g.handle, L.ptr(rec), L.ptr(rec[:, 5:]), 17, L.RRHD_HOST))
    Wg, Ug = g.get_state()
    assert np.array_equal(Wg, W) and np.array_equal(Ug, U) and Wv.shape == W.shape


def test_config0_shock_tube_200_steps_matches_reference():
    """The plain form's parity case as specified: the relativistic shock tube on
    [0,1] x [0,0.05]^2, 200 x 10 x 10 hexes split into 6 Kuhn tets (120,000 cells, interior
    vertices jittered by +-0.15 h), ideal gas Gamma = 5/3, CFL 0.3, transmissive boundaries,
    200 steps with tau = CFL h_min / (previous step's max signal speed).  Every conserved and
    primitive field of every cell equals the reference's own compiled Hllc3dStab (the oracle
    restatement where that build is absent) after every 20th step and at the end."""
    import os
    m, W = shock_tube(200, 10, 10)
    assert m.n_cells == 120000
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    use_ref = oracle.have_ref("hydro_ideal_5_3")
    ref = oracle.HydroRef(m, "hydro_ideal_5_3") if use_ref else None
    if use_ref:
        ref.set_state(W, U)
    g = _grid(m, GAMMA_53)
    g.set_state(W, U)
    tau = 0.3 * m.h_min / 1.0
    threads = os.cpu_count() or 1
    for k in range(200):
        st = rhllc.Hllc3dStab(tau, g)
        if use_ref:
            vmax = ref.step(tau, nthreads=threads)
        else:
            U, W, _, _, vmax = oracle.port_hydro_step(m, U, W, tau, 1, GAMMA_53, nthreads=threads)
        assert st.max_speed == vmax, f"step {k}: max signal speed differs"
        if k % 20 == 19:
            Wo, Uo = ref.get_state() if use_ref else (W, U)
            Wg, Ug = g.get_state()
            assert np.array_equal(Ug, Uo), f"step {k}: U differs, max {np.abs(Ug - Uo).max()}"
            assert np.array_equal(Wg, Wo), f"step {k}: W differs"
        tau = 0.3 * m.h_min / vmax
    assert st.n_failed == 0
    g.close()
    if use_ref:
        ref.close()


@pytest.mark.parametrize("cpb", [128, 256])
def test_layout_info_counts_the_cta_face_lists(cpb):
    """rrhd_hydro_layout_info: the CTA blocks cover the cells, and the CTAs' face lists hold
    every face at least once and at most twice (a face between two blocks is fluxed by both;
    each list padded to an even length, at most one pad per block)."""
    m, _ = shock_tube(12, 3, 3)
    g = rhllc.Grid(m, gamma=GAMMA_53, cells_per_block=cpb)
    info = g.layout_info()
    g.close()
    assert info["cells_per_block"] == cpb
    assert info["blocks"] == -(-m.n_cells // cpb)
    assert info["faces"] == m.n_faces
    assert m.n_faces <= info["face_entries"] <= 2 * m.n_faces + info["blocks"]
    print(f"\n{cpb} cells per CTA: {info['face_entries'] / m.n_faces:.3f} face flux evaluations per face")
