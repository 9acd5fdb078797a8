"""GPU parity of the FP64 radiation kernels against the oracle.

exact scattering, moments, 4-force: bit-identical (tolerance 0).
FMA scattering: |S - S_oracle| <= 1e-13 * S_oracle (one rounding per term
instead of three).
"""
import numpy as np
import pytest
import torch

import oracle
from cases import intensity, jet
from radrhd_solver_b200 import illum, rad_rhd
from radrhd_solver_b200.mesh import fibonacci_directions

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,M", [(700, 256), (333, 64), (129, 100), (1, 7)])
def test_scatter_and_moments_bitexact(N, M):
    d = fibonacci_directions(M)
    I = intensity(N, M, seed=M)
    dg = illum.DirectionGrid(d)
    Id = torch.tensor(I, device="cuda")
    S = illum.CalculateIntScattering(dg, Id, exact=True)
    E, F, T = illum.CalculateAllParam(dg, Id)
    Sf = illum.CalculateIntScattering(dg, Id, exact=False)
    torch.cuda.synchronize()
    So = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    Eo, Fo, To = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
    assert np.array_equal(S.cpu().numpy(), So)
    assert np.array_equal(E.cpu().numpy(), Eo)
    assert np.array_equal(F.cpu().numpy(), Fo)
    assert np.array_equal(T.cpu().numpy(), To)
    assert np.all(np.abs(Sf.cpu().numpy() - So) <= 1e-13 * np.abs(So))
    dg.close()


def test_thomson_low_rank_identity():
    """S(c,w) = (3/4)(E + w^T T w) for the Thomson phase function with equal
    weights: an independent check of scattering against the moments."""
    M = 128
    d = fibonacci_directions(M)
    I = intensity(400, M, seed=1)
    dg = illum.DirectionGrid(d)
    Id = torch.tensor(I, device="cuda")
    S = illum.CalculateIntScattering(dg, Id).cpu().numpy()
    E, F, T = (x.cpu().numpy() for x in illum.CalculateAllParam(dg, Id))
    pred = 0.75 * (E[:, None] + np.einsum("ki,nij,kj->nk", d.dirs, T, d.dirs))
    assert np.allclose(S, pred, rtol=1e-13, atol=0)


def test_rad_source_bitexact():
    m, W = jet(6)
    n = m.n_cells
    rng = np.random.default_rng(4)
    W = np.stack([10 ** rng.uniform(-2, 1, n), rng.uniform(-.5, .5, n), rng.uniform(-.5, .5, n),
                  rng.uniform(-.5, .5, n), 10 ** rng.uniform(-4, 0, n)], 1)
    alpha = W[:, 0].copy()
    sigma = 0.5 * W[:, 0]
    E = 10 ** rng.uniform(-3, 0, n)
    F = rng.uniform(-1, 1, (n, 3)) * E[:, None] * 0.3
    T = rng.uniform(0, 1, (n, 3, 3)) * E[:, None, None]
    for em in (rad_rhd.reference_emission(), rad_rhd.emission(1.0, 1.0, np.pi, 1.0)):
        G = rad_rhd.GetRadSource(*(torch.tensor(a, device="cuda") for a in (W, alpha, sigma, E, F, T)), em=em)
        torch.cuda.synchronize()
        Go = oracle.port_rad_source(W, alpha, sigma, E, F, T,
                                    (em.temp_coef, em.sigma_sb, em.pi, em.rad_unit))
        assert np.array_equal(G.cpu().numpy(), Go)
