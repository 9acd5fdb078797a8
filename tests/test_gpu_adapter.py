"""The drop-in adapter (adapter/rhllc_3d_stab_b200.cpp) inside the reference's own build.

oracle/_ref/librrhd_ref_adapter_hydro_5_3.so is the reference's hydro sources (ideal gas,
Gamma = 5/3) with the adapter linked in place of solvers/rhllc/src/rhllc_3d_stab.cpp, on the
B200 library -- what a maintainer's build becomes.  Two grid_t objects, one per build, are
stepped through the reference's own entry point rhllc::Hllc3dStab(tau, grid): cell states,
face fluxes left in grid.faces[].f and rhllc::max_signal_speed must agree bit for bit."""
import ctypes

import numpy as np
import pytest

import oracle
from cases import GAMMA_53, shock_tube

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (oracle.have_ref("adapter_hydro_5_3") and oracle.have_ref("hydro_ideal_5_3")),
                                 reason="reference builds not present (make -C oracle ref)")]


def _adapter_controls():
    lib = oracle.ref("adapter_hydro_5_3")
    lib.ref_adapter_keep_face_flux.argtypes = [ctypes.c_int]
    lib.ref_adapter_set_resident.argtypes = [ctypes.c_int]
    lib.ref_adapter_sync_to_host.argtypes = [ctypes.c_void_p]
    return lib


def test_adapter_hllc3dstab_matches_reference_build():
    """Default mode: the state goes both ways every call; with KeepFaceFlux(true) the
    face fluxes are written back into grid.faces[].f as the reference's step leaves them."""
    lib = _adapter_controls()
    m, W = shock_tube(24, 4, 4)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    ref = oracle.HydroRef(m, "hydro_ideal_5_3")
    ada = oracle.HydroRef(m, "adapter_hydro_5_3")
    ref.set_state(W, U)
    ada.set_state(W, U)
    lib.ref_adapter_keep_face_flux(1)
    tau = 0.3 * 0.25 / 24
    for step in range(12):
        s_ref = ref.step(tau, nthreads=4)
        s_ada = ada.step(tau)
        assert s_ada == s_ref, f"max signal speed differs at step {step}"
    Wr, Ur = ref.get_state()
    Wa, Ua = ada.get_state()
    assert np.array_equal(Ua, Ur) and np.array_equal(Wa, Wr)
    assert np.array_equal(ada.face_flux(), ref.face_flux())
    assert np.abs(Ur - U).max() > 0  # the state moved
    lib.ref_adapter_keep_face_flux(0)
    ref.close()
    ada.close()


def test_adapter_resident_mode_matches_reference_build():
    """Resident mode: the state is uploaded by the first call and stays on the device;
    grid.cells keeps the initial state until SyncToHost, which then gives the
    reference build's state bit for bit.  Face fluxes are not downloaded by default."""
    lib = _adapter_controls()
    m, W = shock_tube(24, 4, 4)
    W, U = oracle.port_p2c(W, 1, GAMMA_53)
    ref = oracle.HydroRef(m, "hydro_ideal_5_3")
    ada = oracle.HydroRef(m, "adapter_hydro_5_3")
    ref.set_state(W, U)
    ada.set_state(W, U)
    F0 = ada.face_flux()
    lib.ref_adapter_set_resident(1)
    try:
        tau = 0.3 * 0.25 / 24
        for step in range(10):
            assert ada.step(tau) == ref.step(tau, nthreads=4), f"max signal speed differs at step {step}"
        Wa0, Ua0 = ada.get_state()
        assert np.array_equal(Ua0, U) and np.array_equal(Wa0, W)  # host copy untouched while resident
        assert np.array_equal(ada.face_flux(), F0)
        lib.ref_adapter_sync_to_host(ada.h)
        Wr, Ur = ref.get_state()
        Wa, Ua = ada.get_state()
        assert np.array_equal(Ua, Ur) and np.array_equal(Wa, Wr)
        # stepping on after a sync continues from the device state
        for _ in range(3):
            assert ada.step(tau) == ref.step(tau, nthreads=4)
        lib.ref_adapter_sync_to_host(ada.h)
        assert all(np.array_equal(a, b) for a, b in zip(ada.get_state(), ref.get_state()))
    finally:
        lib.ref_adapter_set_resident(0)
    ref.close()
    ada.close()


def test_adapter_rebuilds_for_a_new_grid():
    """A second grid (other size) through the same process: the adapter notices and
    rebuilds its device copy."""
    for n in (12, 16):
        m, W = shock_tube(n, 2, 2)
        W, U = oracle.port_p2c(W, 1, GAMMA_53)
        ref = oracle.HydroRef(m, "hydro_ideal_5_3")
        ada = oracle.HydroRef(m, "adapter_hydro_5_3")
        ref.set_state(W, U)
        ada.set_state(W, U)
        for _ in range(3):
            assert ada.step(1e-3) == ref.step(1e-3, nthreads=2)
        assert all(np.array_equal(a, b) for a, b in zip(ada.get_state(), ref.get_state()))
        ref.close()
        ada.close()


def test_radiation_adapter_through_the_reference_interface():
    """adapter/cuda_interface_sep_b200.cpp under the reference's headers and types:
    separate_device::InitDevice on a grid_t / grid_directions_t, then
    CalculateIntScatteringAsync as the illum drivers call it.  grid.scattering and the
    energy / stream / impulse moments equal the oracle's restatement of the reference
    kernels bit for bit, for all directions and for a slice of them."""
    import ctypes as C
    import os

    from cases import intensity
    from radrhd_solver_b200.mesh import fibonacci_directions
    path = os.path.join(oracle.loader.REF_DIR, "librrhd_ref_adapter_rad.so")
    if not os.path.exists(path):
        pytest.skip("radiation adapter build not present (make -C oracle ref)")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.radad_create.restype = P
    lib.radad_create.argtypes = [C.c_int64, C.c_int32, P, P, C.c_double]
    lib.radad_scatter.restype = C.c_int
    lib.radad_scatter.argtypes = [P, P, C.c_int32, C.c_int32, P, P, P, P]
    lib.radad_destroy.argtypes = [P]
    N, M = 700, 64
    d = fibonacci_directions(M)
    I = np.ascontiguousarray(intensity(N, M, seed=14))
    h = lib.radad_create(N, M, d.dirs.ctypes.data, d.areas.ctypes.data, d.full_area)
    assert h
    So = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Eo, Fo, To = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
    for start, end in ((0, M), (10, 30)):
        S = np.zeros((N, end - start))
        E, F, T = np.zeros(N), np.zeros((N, 3)), np.zeros((N, 9))
        assert lib.radad_scatter(h, I.ctypes.data, start, end, S.ctypes.data, E.ctypes.data, F.ctypes.data,
                                 T.ctypes.data) == 0
        assert np.array_equal(S, So[:, start:end])
        assert np.array_equal(E, Eo) and np.array_equal(F, Fo)
        assert np.array_equal(T.reshape(N, 3, 3), To.reshape(N, 3, 3))
    lib.radad_destroy(h)


def test_ray_tracing_adapter_through_the_reference_interface():
    """adapter/cuda_ray_interface_b200.cpp under the reference's headers and types: the
    FaceCell / Ray_t vectors of RunRayTracing through InitDevice and the four tracing calls;
    every intersection code equals the reference kernels' (compiled for the host), including
    the reference's call-to-kernel mapping (StartTracing = the Roche-lobe kernel)."""
    import ctypes as C
    import os

    from cases import ray_surface
    path = os.path.join(oracle.loader.REF_DIR, "librrhd_ref_adapter_ray.so")
    if not os.path.exists(path) or not oracle.have_ref("ray"):
        pytest.skip("ray adapter or reference ray build not present (make -C oracle ref)")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.rayad_run.restype = C.c_int
    lib.rayad_run.argtypes = [P, P, C.c_int64, P, C.c_int64, C.c_int, P]
    ids, abc = ray_surface(8, 10)
    ids, abc = np.ascontiguousarray(ids), np.ascontiguousarray(abc)
    rays = np.ascontiguousarray(oracle.port_ray_make_rays(19)[::7])
    for call, mode in ((0, 1), (1, 0), (2, 2), (3, 3)):
        out = np.empty(len(rays), dtype=np.int32)
        assert lib.rayad_run(ids.ctypes.data, abc.ctypes.data, len(ids), rays.ctypes.data, len(rays), call,
                             out.ctypes.data) == 0
        assert np.array_equal(out, oracle.ref_ray(mode, rays, ids, abc))


def test_spectrum_adapter_through_the_reference_interface():
    """The SPECTRUM build of adapter/cuda_interface_sep_b200.cpp: SendVelocity and
    CalculateFullSpectrumIntScattering / CalculateSpectrumIntScattering as the spectrum
    module calls them (grid_t with size_frq = 100, frq_grid, cur_frq_id).  The scattering
    equals the reference's own Compton kernels compiled for the host to within 1e-12."""
    import ctypes as C
    import os

    from cases import compton_case
    from radrhd_solver_b200.mesh import fibonacci_directions
    path = os.path.join(oracle.loader.REF_DIR, "librrhd_ref_adapter_rad_spectrum.so")
    if not os.path.exists(path) or not oracle.have_ref("compton"):
        pytest.skip("spectrum adapter or reference Compton build not present (make -C oracle ref)")
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.radad_create.restype = P
    lib.radad_create.argtypes = [C.c_int64, C.c_int32, P, P, C.c_double]
    lib.radad_full_spectrum.restype = C.c_int
    lib.radad_full_spectrum.argtypes = [P, P, P, C.c_int32, C.c_int32, P]
    lib.radad_spectrum.restype = C.c_int
    lib.radad_spectrum.argtypes = [P, P, P, C.c_double, C.c_double, C.c_int32, C.c_int32, P]
    lib.radad_destroy.argtypes = [P]
    N, M = 9, 32
    d = fibonacci_directions(M)
    I, vel = compton_case(N, M, seed=41)
    I, vel = np.ascontiguousarray(I), np.ascontiguousarray(vel)
    h = lib.radad_create(N, M, d.dirs.ctypes.data, d.areas.ctypes.data, d.full_area)
    assert h

    def rel(a, b):
        assert np.array_equal(a == 0, b == 0)
        nz = b != 0
        return np.max(np.abs(a[nz] - b[nz]) / np.abs(b[nz]))

    for start, end in ((0, M), (4, 20)):
        S = np.zeros((N, end - start, 100))
        assert lib.radad_full_spectrum(h, I.ctypes.data, vel.ctypes.data, start, end, S.ctypes.data) == 0
        want = oracle.ref_compton(I, vel, d.dirs, d.areas, d.full_area, dir_disp=start, dir_count=end - start)
        assert rel(S, want) <= 1e-12
    I1 = np.ascontiguousarray(I[:, :, 55])
    S1 = np.zeros((N, M))
    assert lib.radad_spectrum(h, I1.ctypes.data, vel.ctypes.data, 3e20, 5e20, 0, M, S1.ctypes.data) == 0
    assert rel(S1, oracle.ref_compton_spectrum(I1, vel, d.dirs, d.areas, d.full_area, 0.5 * (3e20 + 5e20))) <= 1e-12
    lib.radad_destroy(h)
