"""GPU transport sweep and coupled radiation-hydro step against the oracle.

Bars: the FP64 sweep within 1e-12 relative of orc_sweep per cell, direction and
group (every operation is the oracle's in the oracle's order; only exp comes
from CUDA's libm instead of glibc); the FP32 sweep within 1e-5.  The plain
coupled step (FP64 sweep, FP64 scattering, reference con2prim guess) within
1e-12 of the oracle's composition of the same step, per cell; the chosen form
(mixed-precision sweep, tensor-core scattering, learned con2prim guess) keeps the
scattering integral within 1e-6 and the hydro state within 1e-10 of the plain form.
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


@pytest.mark.parametrize("n", [5, 16])
def test_sweep_mixed_matches_oracle(n):
    """Mixed precision: the sweep in double (geometry, records, face values, arithmetic),
    float S in and float I out.  Against the FP64 oracle fed the same (float) inputs the
    error is the one rounding of the output, independent of the mesh size (the all-float
    sweep's stored face values carry their rounding along the characteristics, which the
    larger mesh shows)."""
    m = kuhn_box(n, n, n, lo=(-1, -1, -1), hi=(1, 1, 1), seed=23)
    d = fibonacci_directions(32)
    G = 4
    inp = [a.astype(np.float32).astype(np.float64) for a in _inputs(m, d.size, G, 29)]
    alpha, betta, Q, S = inp
    alpha = alpha / 30.0  # optically thin cells: long characteristics
    betta = (0.5 * alpha).astype(np.float32).astype(np.float64)
    alpha = alpha.astype(np.float32).astype(np.float64)
    Io, missing = oracle.port_sweep(m, d.dirs, alpha, betta, Q, S)
    assert missing == 0
    errs, outs = {}, {}
    for prec, geo in (("mixed", False), ("mixed", True), ("fp32", False), ("fp32", True)):
        grid = rhllc.Grid(m, gamma=GAMMA_43)
        dg = illum.DirectionGrid(d)
        sw = illum.TransportSweep(grid, dg, groups=G, precision=prec, item_geometry=geo)
        t32 = [torch.tensor(a, dtype=torch.float32, device="cuda").contiguous() for a in (alpha, betta, Q, S)]
        I = illum.CalculateIllum(sw, *t32)
        grid.sync()
        outs[prec, geo] = I.cpu().numpy()
        errs[prec, geo] = float(np.max(np.abs(outs[prec, geo].astype(np.float64) - Io) / np.abs(Io)))
        grid.close()
    print(f"\n{m.n_cells} cells: sweep max rel err mixed {errs['mixed', False]:.2e} (item geometry "
          f"{errs['mixed', True]:.2e}), fp32 {errs['fp32', False]:.2e}")
    assert errs["mixed", False] <= 1e-7  # one float rounding of the output: 2^-24 = 6e-8
    # the item-geometry stream holds the in-face distances rounded to float once (every
    # choice made in double): the attenuation moves by k r 2^-24, below the output rounding
    assert errs["mixed", True] <= 1e-7
    # in the all-float sweep the streamed distances are the values it computes anyway
    assert np.array_equal(outs["fp32", True], outs["fp32", False])


@pytest.mark.parametrize("dirs_per_batch", [8, 32])
def test_plan_levels_are_the_reference_fronts(dirs_per_batch):
    """The device plan sweeps every (cell, direction) in the level that the reference's
    graph::RunGraphModule (graph/src/graph_by_direction.cpp, compiled from its sources)
    gives as the cell's front for that direction.  Within a level the order does not
    change any value: each out-face value reads only upwind faces of earlier levels."""
    from oracle import loader as OL
    if OL.ref_trace() is None:
        pytest.skip("reference trace build not present (make -C oracle ref)")
    from test_oracle_trace import _neighbour_faces, _outward_normals
    m = kuhn_box(6, 5, 4, lo=(-1, -1, -1), hi=(1, 1, 1), seed=33, with_vertices=True)
    d = fibonacci_directions(32)
    lv_ref, bad = OL.ref_graph_levels(_neighbour_faces(m), _outward_normals(m), d.dirs)
    assert bad == 0
    grid = rhllc.Grid(m, gamma=GAMMA_43)
    dg = illum.DirectionGrid(d)
    sw = illum.TransportSweep(grid, dg, groups=1, precision="fp64", dirs_per_batch=dirs_per_batch)
    lv = sw.plan_levels()
    grid.close()
    assert np.array_equal(lv, lv_ref)


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
    o = L.RadOpts(1, L.RRHD_RAD_FP64, 0, 0.0, 1)  # the geometry stream holds float distances
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
    rows = np.concatenate([Er[:, None], Fr, Tr[:, [0, 0, 0, 1, 1, 2], [0, 1, 2, 1, 2, 2]]], 1)
    return U, W, I, S, mom, G4, rows


def _state_err(Ug, Wg, Uo, Wo):
    """Largest error of a hydro state, per cell and relative to that cell's own
    scale: D, E, rho and p relative to themselves; the momentum S relative to the
    cell's E (|S| < E); the velocity in units of c."""
    E = np.abs(Uo[:, 4])[:, None]
    eU = max(np.max(np.abs(Ug[:, [0, 4]] - Uo[:, [0, 4]]) / np.abs(Uo[:, [0, 4]])),
             np.max(np.abs(Ug[:, 1:4] - Uo[:, 1:4]) / E))
    eW = max(np.max(np.abs(Wg[:, [0, 4]] - Wo[:, [0, 4]]) / np.abs(Wo[:, [0, 4]])),
             np.max(np.abs(Wg[:, 1:4] - Wo[:, 1:4])))
    return eU, eW


def _moment_err(mg, mo):
    """Per row: E relative to itself, F and T relative to the row's E."""
    E = np.abs(mo[:, :1])
    return max(np.max(np.abs(mg[:, 0] - mo[:, 0]) / E[:, 0]), np.max(np.abs(mg[:, 1:] - mo[:, 1:]) / E))


def _g4_scale(W, mom, G, em, a=1.0, b=0.5):
    """Per-cell magnitude of the terms of the 4-force (rad_rhd::GetRadSource):
    rho gamma (alpha + sigma)(E + |F|) + |q| gamma, q = -alpha rho B / k."""
    rho, v = W[:, 0], W[:, 1:4]
    gamma = 1.0 / np.sqrt(1.0 - np.sum(v * v, 1))
    m = mom.reshape(-1, G, 10).sum(1)
    T = em[0] * W[:, 4] / rho
    B = T ** 4 * em[1] / em[2]
    q = a * rho * rho * B / em[3]
    return rho * gamma * (a + b) * rho * (np.abs(m[:, 0]) + np.linalg.norm(m[:, 1:4], axis=1)) + q * gamma


def _coupled_grid(m, W, U, d, G, precision, item_geometry=False):
    g = rhllc.Grid(m, gamma=GAMMA_43)
    g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
    g.set_state(W, U)
    dg = illum.DirectionGrid(d)
    sw = illum.TransportSweep(g, dg, groups=G, precision=precision, item_geometry=item_geometry)
    return g, dg, sw


def test_coupled_plain_matches_oracle():
    """Three coupled steps of the plain form against the oracle's composition, every
    quantity per cell: I and S per (cell, group, direction) relative to themselves, the
    moments per row, the 4-force per cell against the size of its terms, and the
    hydro state per cell (_state_err), all within 1e-12."""
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
    rows = np.zeros((m.n_cells * G, 10))
    for k in range(3):
        hs, ss = step(tau, stats=True)
        used = rows  # the 4-force of a step reads the moments of the step before
        Uo, Wo, Io, S, mom, G4o, rows = _oracle_coupled(m, Uo, Wo, tau, d, G, S, mom)
        assert ss.n_failed == 0
    Wg, Ug = g.get_state()
    Ig, Sg, G4g, Mg = step.get("I"), step.get("S"), step.get("G4"), step.get("MOM")
    assert np.abs(G4o).max() > 0
    rel = lambda a, b: np.max(np.abs(a - b) / np.abs(b))
    eU, eW = _state_err(Ug, Wg, Uo, Wo)
    eG4 = np.max(np.abs(G4g - G4o) / _g4_scale(Wo, used, G, EM)[:, None])
    print(f"\nper cell: I {rel(Ig, Io):.2e} S {rel(Sg, S):.2e} moments {_moment_err(Mg, rows):.2e} "
          f"G4 {eG4:.2e} U {eU:.2e} W {eW:.2e}")
    assert rel(Ig, Io) <= 1e-12
    assert rel(Sg, S) <= 1e-12
    assert _moment_err(Mg, rows) <= 1e-12
    assert eG4 <= 1e-12
    assert eU <= 1e-12 and eW <= 1e-12
    g.close()


def _trained_guess():
    Wc = c2p_states(200_000, GAMMA_43, seed=31)
    Wc, Uc = oracle.port_p2c(Wc, 1, GAMMA_43)
    net = LearnedGuess(seed=3)
    net.train(torch.tensor(Uc, device="cuda"), torch.tensor(Wc[:, 4], device="cuda"), epochs=3, batch=2048,
              lr=2e-3, seed=4)
    return net


@pytest.mark.parametrize("M", [64, 256])
def test_coupled_chosen_form_tracks_plain(M):
    """Three coupled steps of the chosen form (mixed-precision sweep with the item-geometry
    stream, tensor-core F16X3 scattering, learned con2prim guess) against the FP64 oracle
    and the plain form.

    The scattering integral as an operation: the chosen form's S and moments against the
    FP64 oracle's scattering integral and moments of the chosen form's own intensity,
    per (cell, group, direction) within 1e-6 relative (moments per row, F and T relative
    to E).  The trajectory against the plain form, per cell: the hydro state within 1e-10
    (_state_err), the 4-force within 1e-6 of the size of its terms.  The intensity and the
    scattering integral of the two trajectories differ by more than one operation's error
    (about 1.3e-6 after three steps): each step's scattering error enters the next sweep's
    source and comes back through the next scattering; they are held to 5e-6."""
    m, W = jet(8)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(M)
    G = 2
    tau = 0.3 * m.h_min
    net = _trained_guess()
    out = {}
    lib_err = None
    for form in ("plain", "chosen"):
        g, dg, sw = _coupled_grid(m, W, U, d, G, "fp64" if form == "plain" else "mixed", item_geometry=form != "plain")
        step = rad_rhd.RadRHDStep(sw, em=rad_rhd.emission(*EM_JET), scatter="fp64" if form == "plain" else "f16x3",
                                  guess=None if form == "plain" else net)
        stats = [step(tau, stats=True) for _ in range(3)]
        Wg, Ug = g.get_state()
        out[form] = (Ug, Wg, step.get("I"), step.get("S"), step.get("MOM"), step.get("G4"), stats)
        if form == "chosen":
            lib_err = step.scatter_error(m.n_cells)  # every cell
        g.close()
    Up, Wp, Ip, Sp, Mp, Gp, sp = out["plain"]
    Uc, Wc, Ic, Sc, Mc, Gc, sc = out["chosen"]
    # the operation: FP64 oracle scattering integral and moments of the chosen intensity
    So = oracle.port_scatter(Ic, d.dirs, d.areas, d.full_area)
    Er, Fr, Tr = oracle.port_moments(Ic, d.dirs, d.areas, d.full_area)
    Mo = np.concatenate([Er[:, None], Fr, Tr[:, [0, 0, 0, 1, 1, 2], [0, 1, 2, 1, 2, 2]]], 1)
    eS_op = np.max(np.abs(Sc - So) / np.abs(So))
    eM_op = _moment_err(Mc, Mo)
    # the trajectory
    it_p = sum(s[1].newton_iters for s in sp)
    it_c = sum(s[1].newton_iters for s in sc)
    eU, eW = _state_err(Uc, Wc, Up, Wp)
    eI = np.max(np.abs(Ic - Ip) / np.abs(Ip))
    eS = np.max(np.abs(Sc - Sp) / np.abs(Sp))
    eM = _moment_err(Mc, Mp)
    eG4 = np.max(np.abs(Gc - Gp) / _g4_scale(Wp, Mp, G, EM_JET)[:, None])
    print(f"\nscattering of the chosen intensity vs the FP64 oracle: S {eS_op:.2e} moments {eM_op:.2e}"
          f"\nchosen vs plain after 3 steps, per cell: U {eU:.2e} W {eW:.2e} G4 {eG4:.2e} I {eI:.2e} S {eS:.2e} "
          f"moments {eM:.2e}; source con2prim Newton iterations {it_c} vs {it_p}")
    # the library's own check of the same quantities (FP64 on the device)
    assert abs(lib_err[0] - eS_op) <= 1e-9 and abs(lib_err[2] - eM_op) <= 1e-9
    assert eS_op <= 1e-6
    assert eM_op <= 1e-6
    assert eU <= 1e-10 and eW <= 1e-10
    assert eG4 <= 1e-6
    assert eI <= 5e-6 and eS <= 5e-6 and eM <= 5e-6
    assert all(s[1].n_failed == 0 for s in sc)


@pytest.mark.parametrize("precision,item_geometry", [("fp32", False), ("mixed", False), ("mixed", True)])
def test_coupled_chosen_independent_of_batching(precision, item_geometry):
    """The chosen coupled step with one batch of 256 directions is bit-identical to the
    same step with two batches of 128: the batches change which level launch a
    (cell, direction) item runs in, never its arithmetic (nor its streamed geometry)."""
    m, W = jet(5)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(256)
    out = []
    for db in (256, 128):
        g = rhllc.Grid(m, gamma=GAMMA_43)
        g.set_boundary(-3, rhllc.BC_FIXED, JET_INFLOW)
        g.set_state(W, U)
        dg = illum.DirectionGrid(d)
        sw = illum.TransportSweep(g, dg, groups=4, precision=precision, dirs_per_batch=db,
                                  item_geometry=item_geometry)
        step = rad_rhd.RadRHDStep(sw, em=rad_rhd.emission(*EM_JET), scatter="f16x3")
        for _ in range(2):
            step(0.3 * m.h_min)
        Wg, Ug = g.get_state()
        out.append((Ug, step.get("I"), step.get("S")))
        g.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)
