"""Generates the golden fixtures of tests/golden/ by running the reference
RadRHD_solver code compiled from its own sources (oracle/_ref, built by
`make -C oracle ref` where the reference tree is available).

    python tests/golden/make_golden.py

Every array in the .npz files is an input chosen here (seeded) or an output of
the reference's own functions: GetConvValueStab / GetPhysValueStab /
PhysPressureFix, GetFluxStab, Hllc3dStab, the scattering integral and the
energy/stream/impulse moments, GetRadSource, GetIllum, GetRhsOpt and
ReCalcIllumOpt.  tests/golden/files_sys/ holds files written by the reference's
own files_sys::bin::WriteGridGeo and WriteSolution.  The fixtures let the tests pin the oracle and the CUDA
library where the reference tree is absent.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from cases import GAMMA_43, GAMMA_53, JET_INFLOW, c2p_states  # noqa: E402
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box  # noqa: E402

VARIANTS = {"hydro_ideal_5_3": (1, GAMMA_53), "hydro_ideal_4_3": (1, GAMMA_43), "hydro_taub": (2, GAMMA_53)}


def mesh_arrays(m, prefix):
    return {f"{prefix}{k}": np.asarray(getattr(m, k)) for k in
            ("face_id_l", "face_id_r", "face_n", "face_area", "cell_faces", "cell_sign", "cell_volume",
             "cell_center")} | {f"{prefix}h_min": np.float64(m.h_min)}


def hydro_fixtures(out):
    for variant, (eos, gamma) in VARIANTS.items():
        W = c2p_states(200, gamma, seed=eos * 7 + 1)
        W[:10, 1:4] *= 1.3  # |v| >= 1: GetConvValueStab clamps
        Wr, Ur = oracle.ref_p2c(W, variant)
        Wc, codes = oracle.ref_c2p(Ur, variant)
        U2 = Ur.copy()
        U2[:, 4] *= 0.7
        U2f, W2f, fcodes = oracle.ref_pressure_fix(U2, Wr, variant)
        rng = np.random.default_rng(eos + 3)
        WL, UL = oracle.ref_p2c(c2p_states(200, gamma, seed=21), variant)
        WR, UR = oracle.ref_p2c(c2p_states(200, gamma, seed=22), variant)
        nv = rng.normal(size=(200, 3))
        nv[:5] = [0, 0, 1]
        nv[5:10] = [0, 0, -1]
        nv /= np.linalg.norm(nv, axis=1)[:, None]
        S = rng.uniform(0.1, 2, 200)
        F, speed = oracle.ref_flux(UL, UR, WL, WR, nv, S, variant)
        out[variant] = dict(W_in=W, W_p2c=Wr, U_p2c=Ur, W_c2p=Wc, c2p_codes=codes, U_fix_in=U2, U_fix=U2f,
                            W_fix=W2f, fix_codes=fcodes, UL=UL, UR=UR, WL=WL, WR=WR, n=nv, area=S, flux=F,
                            speed=speed)


def step_fixtures(out):
    # shock tube, ideal gas 5/3, transmissive boundaries
    m = kuhn_box(8, 2, 2, hi=(1.0, 0.25, 0.25), jitter=0.15, seed=5)
    W = np.zeros((m.n_cells, 5))
    W[:, 0] = np.where(m.cell_center[:, 0] < 0.5, 10.0, 1.0)
    W[:, 4] = np.where(m.cell_center[:, 0] < 0.5, 13.33, 0.01)
    variant = "hydro_ideal_5_3"
    W, U = oracle.ref_p2c(W, variant)
    h = oracle.HydroRef(m, variant)
    h.set_state(W, U)
    tau = 0.3 * m.h_min
    Us, Ws, speeds = [], [], []
    for _ in range(5):
        speeds.append(h.step(tau, 1))
        w, u = h.get_state()
        Us.append(u)
        Ws.append(w)
    h.close()
    out["step_shock"] = mesh_arrays(m, "mesh_") | dict(W0=W, U0=U, tau=np.float64(tau), U=np.stack(Us),
                                                      W=np.stack(Ws), speed=np.array(speeds))
    # jet nozzle, ideal gas 4/3, fixed inflow state on code -3
    m = kuhn_box(4, 4, 4, lo=(-1, -1, -1), hi=(1, 1, 1), jitter=0.15, seed=6, inflow_radius=0.6, inflow_code=-3)
    variant = "hydro_ideal_4_3"
    W = np.zeros((m.n_cells, 5))
    W[:, 0] = 1.0
    W[:, 4] = 1e-3
    W, U = oracle.ref_p2c(W, variant)
    # inflow boundary state as BoundConditions makes it: rhllc::GetConvValue (rhllc_flux.cpp:7-16)
    win = np.ascontiguousarray(JET_INFLOW[None, :], np.float64)
    ubc = np.zeros_like(win)
    oracle.ref(variant).ref_p2c_plain(win.ctypes.data, ubc.ctypes.data, 1)
    h = oracle.HydroRef(m, variant)
    h.set_bc(-3, 1, JET_INFLOW, ubc[0])
    h.set_state(W, U)
    tau = 0.3 * m.h_min
    Us, Ws, codes = [], [], []
    for _ in range(4):
        c = np.zeros(m.n_cells, np.int32)
        h.step(tau, 1, codes=c)
        w, u = h.get_state()
        Us.append(u)
        Ws.append(w)
        codes.append(c)
    h.close()
    out["step_jet"] = mesh_arrays(m, "mesh_") | dict(W0=W, U0=U, U_inflow=ubc[0], tau=np.float64(tau),
                                                    U=np.stack(Us), W=np.stack(Ws), status=np.stack(codes))


def radiation_fixtures(out):
    d = fibonacci_directions(32)
    rng = np.random.default_rng(9)
    I = np.exp(rng.normal(0, 0.5, (40, 32)))
    S = oracle.ref_scatter(I, d.dirs, d.areas, d.full_area)
    E, F, T = oracle.ref_moments(I, d.dirs, d.areas, d.full_area)
    n = 100
    W = np.stack([10 ** rng.uniform(-2, 1, n), rng.uniform(-.5, .5, n), rng.uniform(-.5, .5, n),
                  rng.uniform(-.5, .5, n), 10 ** rng.uniform(-14, -10, n)], 1)
    alpha, sigma = W[:, 0].copy(), 0.5 * W[:, 0]
    Er = 10 ** rng.uniform(-3, 0, n)
    Fr = rng.uniform(-1, 1, (n, 3)) * Er[:, None] * 0.3
    Tr = rng.uniform(0, 1, (n, 3, 3)) * Er[:, None, None]
    Tr = 0.5 * (Tr + Tr.transpose(0, 2, 1))
    G = oracle.ref_rad_source(W, alpha, sigma, Er, Fr, Tr)
    consts = oracle.ref_rad_constants()
    out["radiation"] = dict(dirs=d.dirs, areas=d.areas, full_area=np.float64(d.full_area), I=I, S=S, E=E, F=F, T=T,
                            W=W, alpha=alpha, sigma=sigma, Er=Er, Fr=Fr, Tr=Tr, G=G, emission=consts)


def sweep_fixtures(out):
    rng = np.random.default_rng(11)
    n = 300
    I0 = 10 ** rng.uniform(-6, 2, (n, 3))
    s = rng.uniform(0, 0.1, (n, 3))
    k = 10 ** rng.uniform(-3, 3, n)
    rhs = 10 ** rng.uniform(-6, 2, n)
    illum = np.array([oracle.ref_get_illum(I0[i], s[i], k[i], rhs[i]) for i in range(n)])
    a, b = 10 ** rng.uniform(-3, 2, (2, n))
    T = 10 ** rng.uniform(-3, 5, n)
    Sg = 10 ** rng.uniform(-6, 1, n)
    rr = np.array([oracle.ref_get_rhs(a[i], b[i], T[i], Sg[i]) for i in range(n)])
    m = kuhn_box(4, 3, 2, seed=3)
    fv = 10 ** rng.uniform(-3, 1, m.n_faces)
    Ill = rng.uniform(0.1, 1, (m.n_cells, 4))
    Ill0 = Ill.copy()
    norms = []
    for dd in (0, 3):
        norms.append(oracle.ref_recalc_illum(m.cell_faces, m.face_area, fv, Ill, dd))
    out["sweep_parts"] = dict(I0=I0, s=s, k=k, rhs=rhs, illum=illum, alpha=a, betta=b, T=T, S=Sg, rhs_out=rr[:, 0],
                              k_out=rr[:, 1], cell_faces=m.cell_faces, face_area=m.face_area, fv=fv,
                              illum_cells_in=Ill0, illum_cells_out=Ill, recalc_norms=np.array(norms), emission=oracle.ref_rad_constants())


def files_fixtures(out):
    # boundary codes -1..-6 on the six box sides, plus an inflow disc (-3)
    m = kuhn_box(2, 2, 2, jitter=0.15, seed=8, bc_codes=(-1, -2, -3, -4, -5, -6), inflow_radius=0.3,
                 inflow_code=-7)
    rng = np.random.default_rng(12)
    W = np.stack([10 ** rng.uniform(-1, 1, m.n_cells), *rng.uniform(-.4, .4, (3, m.n_cells)),
                  10 ** rng.uniform(-2, 0, m.n_cells)], 1)
    W, U = oracle.ref_p2c(W, "hydro_ideal_5_3")
    d = os.path.join(HERE, "files_sys")
    os.makedirs(d, exist_ok=True)
    h = oracle.HydroRef(m, "hydro_ideal_5_3")
    h.set_state(W, U)
    assert h.write_geo(os.path.join(d, "geo_faces.bin"), os.path.join(d, "geo_cells.bin")) == 0
    assert h.write_solution(os.path.join(d, "Solve0")) == 0
    h.close()
    out["files_sys"] = mesh_arrays(m, "mesh_") | dict(W=W, U=U)


def compton_fixtures(out):
    """Full-spectrum Compton scattering by the reference's own device source compiled
    for the host (Get_full_spectrum_multi_device): all directions, and a slice of them
    written into a wider output stride."""
    from cases import compton_case
    d = fibonacci_directions(16)
    I, vel = compton_case(6, 16, seed=23)
    S = oracle.ref_compton(I, vel, d.dirs, d.areas, d.full_area)
    S_part = oracle.ref_compton(I, vel, d.dirs, d.areas, d.full_area, dir_disp=5, dir_count=7, out_stride=9)
    frq = np.array([oracle.loader.ref_compton_get_frq(j) for j in range(101)])
    S_one = np.stack([oracle.ref_compton_spectrum(I[:, :, f], vel, d.dirs, d.areas, d.full_area, nu)
                      for f, nu in ((3, 1e12), (50, 4.2e20), (97, 9e23))])
    out["compton"] = dict(dirs=d.dirs, areas=d.areas, full_area=np.float64(d.full_area), I=I, vel=vel, S=S,
                          S_part=S_part, get_frq=frq, S_one=S_one, one_bins=np.array([3, 50, 97]),
                          one_frq=np.array([1e12, 4.2e20, 9e23]))


def ray_fixtures(out):
    """Image-plane rays of three frames (a sample of pixels) by the reference's MakeRays and
    their intersection codes in the four tracing modes by its own kernels."""
    from cases import ray_surface
    ids, abc = ray_surface(6, 8)
    frames = np.array([3, 40, 88])
    sample = np.arange(0, 600 * 300, 173)
    rays = np.stack([oracle.ref_ray_make_rays(int(f))[sample] for f in frames])
    codes = np.stack([oracle.ref_ray(m, rays.reshape(-1, 6), ids, abc) for m in range(4)])
    out["ray"] = dict(ids=ids, abc=abc, frames=frames, sample=sample, rays=rays, codes=codes)


FIXTURES = {"hydro": hydro_fixtures, "step": step_fixtures, "radiation": radiation_fixtures,
            "sweep": sweep_fixtures, "files": files_fixtures, "compton": compton_fixtures,
            "ray": ray_fixtures}


def main():
    """`make_golden.py` regenerates every fixture; `make_golden.py compton ...` only the named ones."""
    names = sys.argv[1:] or list(FIXTURES)
    need = list(VARIANTS) + ["illum", "rad_ideal_4_3", "compton", "ray"]
    missing = [v for v in need if not oracle.have_ref(v)]
    if missing:
        sys.exit(f"reference variants not built ({', '.join(missing)}): run `make -C oracle ref` first")
    out = {}
    for n in names:
        FIXTURES[n](out)
    for name, arrays in out.items():
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrays)
        size = os.path.getsize(os.path.join(HERE, f"{name}.npz"))
        print(f"{name}.npz: {len(arrays)} arrays, {size / 1024:.1f} KiB")


if __name__ == "__main__":
    main()
