"""Full-spectrum Compton scattering on the GPU (rrhd_compton_full_spectrum) against
the oracle's restatement of Get_full_spectrum_multi_device and the golden fixture
made by the reference's own kernel source.

The single-frequency kernel (rrhd_compton_spectrum, Get_spectrum_multi_device) is
checked the same way.

Bar: every S[i][k][f] within 1e-12 relative of the oracle (all terms are positive,
so the sum is well conditioned; measured differences are a few 1e-16, from the
regrouped arithmetic and FMA).  A shifted frequency within rounding of a bin edge
could select the neighbouring bin; the seeded cases here have none.  Direction
counts above what fits in shared memory (M = 300) run in chunks.
"""
import os

import numpy as np
import pytest
import torch

import oracle
from cases import compton_case
from radrhd_solver_b200 import illum
from radrhd_solver_b200.mesh import fibonacci_directions

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-12


def _rel(S, So):
    assert np.all(np.isfinite(S)) and np.array_equal(S == 0, So == 0)
    nz = So != 0
    return float(np.max(np.abs(S[nz] - So[nz]) / np.abs(So[nz])))


def _run(dg, I, vel, **kw):
    S = illum.FullSpectrumScattering(dg, torch.tensor(I, device="cuda"), torch.tensor(vel, device="cuda"), **kw)
    torch.cuda.synchronize()
    return S.cpu().numpy()


@pytest.mark.parametrize("M,cells,speeds", [(32, 37, None), (64, 13, None), (256, 6, None), (300, 3, None),
                                            (20, 9, (0.0,)), (24, 8, (0.999, 0.5))])
def test_compton_matches_oracle(M, cells, speeds):
    d = fibonacci_directions(M)
    kw = {} if speeds is None else dict(speeds=speeds)
    I, vel = compton_case(cells, M, seed=M + cells, **kw)
    So = oracle.port_compton(I, vel, d.dirs, d.areas, d.full_area, nthreads=os.cpu_count() or 1)
    dg = illum.DirectionGrid(d)
    S = _run(dg, I, vel)
    err = _rel(S, So)
    print(f"\nM={M} cells={cells}: max rel {err:.2e}")
    assert err <= TOL
    dg.close()


def test_compton_matches_reference_golden_fixture():
    g = np.load(os.path.join(HERE, "golden", "compton.npz"))
    d = fibonacci_directions(len(g["areas"]))
    assert np.array_equal(d.dirs, g["dirs"]) and np.array_equal(d.areas, g["areas"])
    dg = illum.DirectionGrid(d)
    assert _rel(_run(dg, g["I"], g["vel"]), g["S"]) <= TOL
    Sp = _run(dg, g["I"], g["vel"], dir_disp=5, dir_count=7, out_stride=9)
    assert _rel(Sp[:, :7], g["S_part"][:, :7]) <= TOL
    dg.close()


def test_compton_direction_slice_and_stride():
    """A slice of output directions into a wider stride gives the same columns bit
    for bit and leaves the padding columns alone; repeated calls are identical."""
    M, cells = 48, 7
    d = fibonacci_directions(M)
    I, vel = compton_case(cells, M, seed=2)
    dg = illum.DirectionGrid(d)
    It, vt = torch.tensor(I, device="cuda"), torch.tensor(vel, device="cuda")
    S = illum.FullSpectrumScattering(dg, It, vt)
    S2 = illum.FullSpectrumScattering(dg, It, vt)
    Sp = torch.full((cells, 20, 100), 7.0, dtype=torch.float64, device="cuda")
    illum.FullSpectrumScattering(dg, It, vt, S=Sp, dir_disp=11, dir_count=17, out_stride=20)
    torch.cuda.synchronize()
    assert torch.equal(S, S2)
    assert torch.equal(Sp[:, :17], S[:, 11:28])
    assert torch.all(Sp[:, 17:] == 7.0)
    dg.close()


@pytest.mark.parametrize("M,cells,frq", [(32, 37, 1e12), (256, 9, 4.2e20), (64, 13, 9e23), (1000, 3, 3e23)])
def test_single_frequency_matches_oracle(M, cells, frq):
    d = fibonacci_directions(M)
    I3, vel = compton_case(cells, M, seed=M)
    I = np.ascontiguousarray(I3[:, :, 40])
    So = oracle.port_compton_spectrum(I, vel, d.dirs, d.areas, d.full_area, frq, nthreads=os.cpu_count() or 1)
    dg = illum.DirectionGrid(d)
    S = illum.SpectrumScattering(dg, torch.tensor(I, device="cuda"), torch.tensor(vel, device="cuda"), frq)
    Sp = torch.full((cells, M + 3), 5.0, dtype=torch.float64, device="cuda")
    illum.SpectrumScattering(dg, torch.tensor(I, device="cuda"), torch.tensor(vel, device="cuda"), frq, S=Sp,
                             dir_disp=2, dir_count=M - 2, out_stride=M + 3)
    torch.cuda.synchronize()
    err = _rel(S.cpu().numpy(), So)
    print(f"\nsingle frequency M={M} frq={frq:.1e}: max rel {err:.2e}")
    assert err <= TOL
    assert torch.equal(Sp[:, :M - 2], S[:, 2:]) and torch.all(Sp[:, M - 2:] == 5.0)
    dg.close()


def test_single_frequency_matches_reference_golden_fixture():
    g = np.load(os.path.join(HERE, "golden", "compton.npz"))
    d = fibonacci_directions(len(g["areas"]))
    dg = illum.DirectionGrid(d)
    vt = torch.tensor(g["vel"], device="cuda")
    for S1, f, nu in zip(g["S_one"], g["one_bins"], g["one_frq"]):
        S = illum.SpectrumScattering(dg, torch.tensor(np.ascontiguousarray(g["I"][:, :, f]), device="cuda"), vt,
                                     float(nu))
        assert _rel(S.cpu().numpy(), S1) <= TOL
    dg.close()


def test_compton_invalid_arguments():
    from radrhd_solver_b200 import _lib as L
    dg = illum.DirectionGrid(fibonacci_directions(16))
    I = torch.zeros(4, 16, 100, dtype=torch.float64, device="cuda")
    v = torch.zeros(4, 3, dtype=torch.float64, device="cuda")
    S = torch.zeros(4 * 16 * 100 + 1, dtype=torch.float64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    f = L.lib.rrhd_compton_full_spectrum
    assert f(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr(), 4, 10, 7, 16, s) == L.RRHD_ERR_INVALID
    assert f(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr(), 4, 0, 16, 15, s) == L.RRHD_ERR_INVALID
    assert f(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr() + 8, 4, 0, 16, 16, s) == L.RRHD_ERR_INVALID
    assert f(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr(), 0, 0, 16, 16, s) == L.RRHD_OK
    g = L.lib.rrhd_compton_spectrum
    assert g(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr(), 4, 0.0, 0, 16, 16, s) == L.RRHD_ERR_INVALID
    assert g(dg.handle, I.data_ptr(), v.data_ptr(), S.data_ptr(), 4, 1e20, 3, 14, 16, s) == L.RRHD_ERR_INVALID
    torch.cuda.synchronize()
    dg.close()
