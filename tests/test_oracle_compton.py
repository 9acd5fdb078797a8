"""The full-spectrum Compton scattering oracle (C restatement of
Get_full_spectrum_multi_device, cuda_scat_full_spectrum.cu:61-118) pinned to the
reference's own device source compiled for the host (oracle/_ref, where built) and
to the golden fixture tests/golden/compton.npz made from it, plus the properties
the CUDA kernel's design rests on:

* the reference's bin search get_frq_idx equals a count of bin edges below the
  frequency (the form the kernel evaluates with one exact comparison);
* in the low-frequency, zero-velocity limit the kernel reduces to the Thomson
  scattering integral times 4/3 coef (coef = 2 pi r_e^2);
* a slice of output directions written with a wider stride equals the same
  columns of the full result.
"""
import os

import numpy as np
import pytest

import oracle
from cases import compton_case
from radrhd_solver_b200.mesh import fibonacci_directions

HERE = os.path.dirname(os.path.abspath(__file__))
COEF = 2 * 3.1415926535897932384626433832795 * 2.8179403e-13 * 2.8179403e-13


def _golden():
    return np.load(os.path.join(HERE, "golden", "compton.npz"))


def test_port_matches_golden_fixture_bit_for_bit():
    g = _golden()
    S = oracle.port_compton(g["I"], g["vel"], g["dirs"], g["areas"], float(g["full_area"]), nthreads=2)
    assert np.array_equal(S, g["S"])
    Sp = oracle.port_compton(g["I"], g["vel"], g["dirs"], g["areas"], float(g["full_area"]), dir_disp=5,
                             dir_count=7, out_stride=9)
    assert np.array_equal(Sp, g["S_part"])
    assert np.array_equal(np.array([oracle.port_compton_frq(j) for j in range(101)]), g["get_frq"])
    for S1, f, nu in zip(g["S_one"], g["one_bins"], g["one_frq"]):
        S1p = oracle.port_compton_spectrum(g["I"][:, :, f], g["vel"], g["dirs"], g["areas"], float(g["full_area"]), nu)
        assert np.array_equal(S1p, S1)


@pytest.mark.skipif(not oracle.have_ref("compton"), reason="reference Compton kernel not built (make -C oracle ref)")
@pytest.mark.parametrize("frq", [1e9, 1e12, 3e20, 9e23, 5e24])
def test_single_frequency_port_matches_reference_kernel_bit_for_bit(frq):
    M = 24
    d = fibonacci_directions(M)
    I3, vel = compton_case(12, M, seed=6)
    I = I3[:, :, 30]
    Sr = oracle.ref_compton_spectrum(I, vel, d.dirs, d.areas, d.full_area, frq)
    Sp = oracle.port_compton_spectrum(I, vel, d.dirs, d.areas, d.full_area, frq, nthreads=2)
    assert np.array_equal(Sp, Sr)
    Sr = oracle.ref_compton_spectrum(I, vel, d.dirs, d.areas, d.full_area, frq, dir_disp=4, dir_count=9, out_stride=11)
    Sp = oracle.port_compton_spectrum(I, vel, d.dirs, d.areas, d.full_area, frq, dir_disp=4, dir_count=9, out_stride=11)
    assert np.array_equal(Sp, Sr)


@pytest.mark.skipif(not oracle.have_ref("compton"), reason="reference Compton kernel not built (make -C oracle ref)")
@pytest.mark.parametrize("M,cells,speeds", [(32, 6, None), (20, 12, (0.0, 0.5)), (12, 4, (0.999,))])
def test_port_matches_reference_kernel_bit_for_bit(M, cells, speeds):
    d = fibonacci_directions(M)
    kw = {} if speeds is None else dict(speeds=speeds)
    I, vel = compton_case(cells, M, seed=M, **kw)
    Sr = oracle.ref_compton(I, vel, d.dirs, d.areas, d.full_area)
    Sp = oracle.port_compton(I, vel, d.dirs, d.areas, d.full_area, nthreads=2)
    assert np.array_equal(Sp, Sr)


@pytest.mark.skipif(not oracle.have_ref("compton"), reason="reference Compton kernel not built (make -C oracle ref)")
def test_frequency_grid_and_bin_search_match_reference():
    for j in range(-1, 102):
        assert oracle.port_compton_frq(j) == oracle.loader.ref_compton_get_frq(j)
    rng = np.random.default_rng(4)
    for x in 10 ** rng.uniform(11, 24, 20000):
        assert oracle.port_compton_frq_idx(x) == oracle.loader.ref_compton_get_frq_idx(x)


def test_bin_search_is_a_count_of_edges_below():
    """idx(x) = #{j in 1..99 : get_frq(j) < x} for x below frq0, away from the edges."""
    edges = np.array([oracle.port_compton_frq(j) for j in range(1, 100)])
    rng = np.random.default_rng(5)
    xs = np.concatenate([10 ** rng.uniform(9, 24, 50000), np.sqrt(edges[:-1] * edges[1:]), edges * (1 + 1e-12),
                         edges * (1 - 1e-12)])
    xs = xs[xs < 1e24]
    want = np.searchsorted(edges, xs, side="left")
    got = np.array([oracle.port_compton_frq_idx(x) for x in xs])
    assert np.array_equal(got, want)
    # above frq0 the reference's sqrt of a negative gives idx = N_Frq (that read is cut to zero)
    assert oracle.port_compton_frq_idx(2e24) == 100


def test_low_frequency_rest_frame_limit_is_thomson():
    """v = 0 and a flat spectrum: at the lowest bins the recoil eps = h nu / m c^2 is
    about 1e-8, so S[k][f] = coef sum_d (1 + cos^2) I_d a_d / A = 4/3 coef S_Thomson[k]."""
    M = 24
    d = fibonacci_directions(M)
    rng = np.random.default_rng(8)
    Id = np.exp(rng.normal(0, 0.5, (2, M)))
    I = np.repeat(Id[:, :, None], 100, axis=2)
    vel = np.zeros((2, 3))
    S = oracle.port_compton(I, vel, d.dirs, d.areas, d.full_area)
    St = oracle.port_scatter(Id, d.dirs, d.areas, d.full_area)
    for f in range(1, 5):
        assert np.allclose(S[:, :, f], 4.0 / 3.0 * COEF * St, rtol=1e-6, atol=0)


def test_single_frequency_low_limit_is_quarter_thomson():
    """At rest and low frequency (no shift) the single-frequency kernel is
    0.25 coef sum_d (1 + cos^2) I_d a_d / A = 1/3 coef S_Thomson (cfl = 0.25)."""
    M = 24
    d = fibonacci_directions(M)
    rng = np.random.default_rng(9)
    I = np.exp(rng.normal(0, 0.5, (3, M)))
    S = oracle.port_compton_spectrum(I, np.zeros((3, 3)), d.dirs, d.areas, d.full_area, 1e9)
    St = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
    assert np.allclose(S, COEF / 3.0 * St, rtol=1e-9, atol=0)


def test_direction_slice_equals_columns_of_full_result():
    M = 16
    d = fibonacci_directions(M)
    I, vel = compton_case(5, M, seed=3)
    S = oracle.port_compton(I, vel, d.dirs, d.areas, d.full_area)
    Sp = oracle.port_compton(I, vel, d.dirs, d.areas, d.full_area, dir_disp=3, dir_count=6, out_stride=8)
    assert np.array_equal(Sp[:, :6], S[:, 3:9])
    assert np.all(Sp[:, 6:] == 0)
