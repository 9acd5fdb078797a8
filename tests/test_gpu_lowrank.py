"""Low-rank (rank-7 Thomson) scattering integral and moments against the FP64
oracle's direct O(M^2) sum and moments.

Bars: FP64 in/out within 1e-13 relative of the direct sum (different summation
order, all terms positive; measured ~1e-15); FP32 in/out within 2e-7 of the
direct FP64 sum of the same FP32 inputs (the FP32 rounding of S); moments
(relative to E of the row) within 1e-13 in FP64.  The cell-direction-group
layouts give the row layout's values bit for bit, except FP32 with 4 groups (a
vectorised path with another summation order: one FP32 rounding apart).  The
coupled step with the low-rank scattering on the FP64 sweep stays within 1e-12
of the oracle's composition, as the direct-sum form does.
"""
import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_43, intensity, jet
from radrhd_solver_b200 import illum, rad_rhd
from radrhd_solver_b200.mesh import fibonacci_directions
from test_gpu_sweep import EM, _coupled_grid, _oracle_coupled

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.max(np.abs(a - b) / np.abs(b))


def _mom_err(mom, Eo, Fo, To):
    E, F, T = (x.cpu().numpy() for x in illum.moments_from_tc(mom))
    den = Eo[:, None]
    return max(np.max(np.abs(E - Eo) / Eo), np.max(np.abs(F - Fo) / den),
               np.max(np.abs(T - To).reshape(len(Eo), 9) / den))


@pytest.mark.parametrize("M,rows", [(256, 1000), (64, 333), (512, 129), (26, 70)])
def test_lowrank_fp64_matches_direct_sum(M, rows):
    d = fibonacci_directions(M)
    I = intensity(rows, M, seed=M + 3)
    So = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Eo, Fo, To = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
    dg = illum.DirectionGrid(d)
    S, mom = illum.ScatteringLowRank(dg, torch.tensor(I, device="cuda"))
    torch.cuda.synchronize()
    err = _rel(S.cpu().numpy(), So)
    merr = _mom_err(mom, Eo, Fo, To)
    print(f"\nM={M}: S max rel {err:.2e}, moments {merr:.2e}")
    assert err <= 1e-13 and merr <= 1e-13
    assert np.all(mom.cpu().numpy()[:, 10:] == 0)
    dg.close()


@pytest.mark.parametrize("groups", [1, 2, 4])
def test_lowrank_fp32_and_cell_direction_group_layout(groups):
    M, cells = 256, 700
    d = fibonacci_directions(M)
    rows = cells * groups
    I32 = intensity(rows, M, seed=groups).astype(np.float32)
    So = oracle.port_scatter(I32.astype(np.float64), d.dirs, d.areas, d.full_area)
    dg = illum.DirectionGrid(d)
    I = torch.tensor(I32, device="cuda")
    S_rows, mom_rows = illum.ScatteringLowRank(dg, I)
    assert _rel(S_rows.double().cpu().numpy(), So) <= 2e-7
    if groups > 1:
        I_cdg = I.view(cells, groups, M).transpose(1, 2).contiguous()
        S_cdg, mom_cdg = illum.ScatteringLowRank(dg, I_cdg, groups=groups)
        torch.cuda.synchronize()
        S_cdg = S_cdg.transpose(1, 2).reshape(rows, M)
        if groups == 2:
            assert torch.equal(S_cdg, S_rows) and torch.equal(mom_cdg, mom_rows)
        else:
            # the vectorised 4-group path sums each row's directions in another order: the
            # FP64 sums differ in the last bits, the FP32 results by at most one rounding
            assert torch.allclose(S_cdg, S_rows, rtol=1.2e-7, atol=0)
            assert torch.allclose(mom_cdg, mom_rows, rtol=1.2e-7, atol=1e-30)
    dg.close()


def test_lowrank_error_pass_matches_host_errors():
    """The all-rows error pass of a tensor-core result equals the host computation
    against the low-rank FP64 values."""
    M, rows = 256, 2048
    d = fibonacci_directions(M)
    I = torch.tensor(intensity(rows, M, seed=11).astype(np.float32), device="cuda")
    dg = illum.DirectionGrid(d)
    tc = illum.ScatterTC(dg, "f16x3")
    S, _ = tc(I)
    S64, _ = illum.ScatteringLowRank(dg, I.double())
    mx, rms = illum.LowRankError(dg, I, S)
    tc.check()
    rel = (np.abs(S.double().cpu().numpy() - S64.cpu().numpy()) / np.abs(S64.cpu().numpy()))
    print(f"\nf16x3 vs low rank: max {mx:.3e} rms {rms:.3e}")
    assert mx == pytest.approx(rel.max(), rel=1e-9) and rms == pytest.approx(np.sqrt((rel ** 2).mean()), rel=1e-9)
    assert mx <= 1.2e-6
    tc.close()
    dg.close()


def test_lowrank_errors():
    from radrhd_solver_b200 import _lib as L
    dg = illum.DirectionGrid(fibonacci_directions(64))
    I = torch.zeros(10, 64, dtype=torch.float64, device="cuda")
    S = torch.empty_like(I)
    s = torch.cuda.current_stream().cuda_stream
    assert L.lib.rrhd_scatter_lowrank(dg.handle, I.data_ptr(), S.data_ptr(), None, 10, 3, L.RRHD_RAD_FP64, s) \
        == L.RRHD_ERR_INVALID
    assert L.lib.rrhd_scatter_lowrank(dg.handle, I.data_ptr(), S.data_ptr(), None, 10, 1, 7, s) == L.RRHD_ERR_INVALID
    assert L.lib.rrhd_scatter_lowrank(dg.handle, I.data_ptr(), S.data_ptr(), None, 0, 1, L.RRHD_RAD_FP64, s) \
        == L.RRHD_OK
    dg.close()


def test_coupled_lowrank_matches_oracle():
    """The plain coupled step with the low-rank scattering: within 1e-12 of the
    oracle's composition (which sums the scattering directly)."""
    m, W = jet(6)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    d = fibonacci_directions(64)
    G = 2
    g, dg, sw = _coupled_grid(m, W, U, d, G, "fp64")
    step = rad_rhd.RadRHDStep(sw, absorption=1.0, scattering=0.5, em=rad_rhd.emission(*EM), scatter="lowrank")
    tau = 0.3 * m.h_min
    S = np.zeros((m.n_cells * G, d.size))
    mom = (np.zeros(m.n_cells), np.zeros((m.n_cells, 3)), np.zeros((m.n_cells, 3, 3)))
    Uo, Wo = U, W
    for _ in range(3):
        hs, ss = step(tau, stats=True)
        Uo, Wo, Io, S, mom, G4o, _ = _oracle_coupled(m, Uo, Wo, tau, d, G, S, mom)
        assert ss.n_failed == 0
    Wg, Ug = g.get_state()
    Ig, Sg, G4g = step.get("I"), step.get("S"), step.get("G4")
    assert _rel(Ig, Io) <= 1e-12 and _rel(Sg, S) <= 1e-12
    assert np.max(np.abs(G4g - G4o)) <= 1e-12 * np.abs(G4o).max()
    assert np.all(np.abs(Ug - Uo) <= 1e-12 * np.abs(Uo).max(0))
    g.close()
