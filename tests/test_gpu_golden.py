"""The CUDA library against the golden fixtures (outputs of the reference
itself, tests/golden/make_golden.py), through the same entry points a caller
uses.  Bar: bit-identical for con2prim, prim->cons, the hydro step and the
radiation 4-force; 2 ulp for the scattering integral and the moments (the
reference averages four replicated face values there, which can round once)."""
import numpy as np
import pytest
import torch

from golden_io import load, mesh
from radrhd_solver_b200 import illum, rad_rhd, rhllc
from radrhd_solver_b200.mesh import Directions

pytestmark = pytest.mark.gpu

VARIANTS = {"hydro_ideal_5_3": (1, 5.0 / 3.0), "hydro_ideal_4_3": (1, 4.0 / 3.0), "hydro_taub": (2, 5.0 / 3.0)}


def _s():
    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_con2prim_and_prim2con(variant):
    eos, gamma = VARIANTS[variant]
    g = load(variant)
    W = torch.tensor(g["W_in"], device="cuda")
    U = torch.empty_like(W)
    rhllc.GetConvValueStab(W, U, eos=eos, gamma=gamma, stream=_s())
    torch.cuda.synchronize()
    assert np.array_equal(U.cpu().numpy(), g["U_p2c"]) and np.array_equal(W.cpu().numpy(), g["W_p2c"])
    U = torch.tensor(g["U_p2c"], device="cuda")
    Wc = torch.zeros_like(U)
    st = torch.zeros(len(U), dtype=torch.uint8, device="cuda")
    rhllc.GetPhysValueStab(U, Wc, st, eos=eos, gamma=gamma, fallback=False, stream=_s())
    torch.cuda.synchronize()
    codes = st.cpu().numpy().astype(np.int32)
    assert np.array_equal(codes, g["c2p_codes"])
    ok = codes == 0
    assert np.array_equal(Wc.cpu().numpy()[ok], g["W_c2p"][ok])


def test_hydro_steps_shock_tube():
    g = load("step_shock")
    grid = rhllc.Grid(mesh(g), eos=1, gamma=5.0 / 3.0)
    grid.set_state(g["W0"], g["U0"])
    for s in range(len(g["U"])):
        st = rhllc.Hllc3dStab(float(g["tau"]), grid)
        assert st.max_speed == g["speed"][s]
        W, U = grid.get_state()
        assert np.array_equal(U, g["U"][s]) and np.array_equal(W, g["W"][s])
    grid.close()


def test_hydro_steps_jet_inflow():
    g = load("step_jet")
    grid = rhllc.Grid(mesh(g), eos=1, gamma=4.0 / 3.0)
    grid.set_boundary(-3, rhllc.BC_FIXED, [0.01, 0.0, 0.0, np.sqrt(1.0 - 1.0 / 49.0), 1e-3])
    grid.set_state(g["W0"], g["U0"])
    for s in range(len(g["U"])):
        rhllc.Hllc3dStab(float(g["tau"]), grid)
        W, U = grid.get_state()
        assert np.array_equal(U, g["U"][s]) and np.array_equal(W, g["W"][s])
        assert np.array_equal(grid.cell_status().astype(np.int32), g["status"][s])
    grid.close()


def test_scattering_moments_rad_source():
    g = load("radiation")
    dg = illum.DirectionGrid(Directions(g["dirs"], g["areas"], float(g["full_area"])))
    I = torch.tensor(g["I"], device="cuda")
    S = illum.CalculateIntScattering(dg, I, exact=True, stream=_s())
    E, F, T = illum.CalculateAllParam(dg, I, stream=_s())
    torch.cuda.synchronize()
    for a, b in ((S, g["S"]), (E, g["E"]), (F, g["F"]), (T, g["T"])):
        a = a.cpu().numpy()
        assert np.all(np.abs(a - b) <= 2 * np.spacing(np.abs(b)))
    t = {k: torch.tensor(g[k], device="cuda") for k in ("W", "alpha", "sigma", "Er", "Fr", "Tr")}
    G = rad_rhd.GetRadSource(t["W"], t["alpha"], t["sigma"], t["Er"], t["Fr"], t["Tr"],
                             em=rad_rhd.emission(*g["emission"]), stream=_s())
    torch.cuda.synchronize()
    assert np.array_equal(G.cpu().numpy(), g["G"])
    dg.close()


def test_reference_files_into_the_device_state(tmp_path):
    """Geometry and solution files written by the reference's WriteGridGeo /
    WriteSolution, loaded into a device grid, written back out: the device's
    prim->cons matches the reference's and the files come back byte for byte."""
    import os
    from golden_io import GOLDEN
    from radrhd_solver_b200 import files_sys as fs
    g = load("files_sys")
    d = os.path.join(GOLDEN, "files_sys")
    m = fs.read_grid_geo(os.path.join(d, fs.F_GEO_FACES), os.path.join(d, fs.F_GEO_CELLS))
    sol = fs.read_solution(os.path.join(d, "Solve0"))
    W0 = np.concatenate([sol["density"][:, None], sol["velocity"], sol["pressure"][:, None]], 1)
    grid = rhllc.Grid(m, eos=1, gamma=5.0 / 3.0)
    grid.set_state_prim(W0)
    W, U = grid.get_state()
    grid.close()
    assert np.array_equal(W, g["W"]) and np.array_equal(U, g["U"])
    out = fs.write_solution(str(tmp_path), W=W)
    for p in out:
        assert open(p, "rb").read() == open(os.path.join(d, "Solve0", os.path.basename(p)), "rb").read()
