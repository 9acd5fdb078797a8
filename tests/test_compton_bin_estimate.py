"""The full-spectrum Compton kernel finds the bin of a shifted frequency x with an FP32
estimate and one exact comparison (radrhd_solver_b200/csrc/compton.cu, frq_slot): it takes x's
exponent and top 20 mantissa bits as a float, t^2 = betta ln2 (log2 frq0 - log2 x) by one FMA,
c = 100 - rint(sqrt(max(t^2, 0))), clamped at 0, and claims c is the true count of edges below x
or one less, so that adding (x > edge[c]) gives the exact count.  This checks that claim on
the CPU with the same FP32 operations, with log2 perturbed by the hardware approximation's
error bound (2^-21.5 absolute, taken as 2^-21) in both directions, over random frequencies
across and beyond the spectrum and at and around every bin edge."""
import numpy as np

import oracle

BETTA, FRQ0 = 350.0, 1e24
kBLn2 = np.float32(BETTA * 0.69314718055994530942)
kBLnF0 = np.float32(BETTA * 55.262042231857095)


def _edges():
    lo = np.nextafter(0.5 * (oracle.port_compton_frq(1) + oracle.port_compton_frq(0)), -np.inf)
    return np.array([lo] + [oracle.port_compton_frq(j) for j in range(1, 100)])


def _estimate(x, dlg):
    bits = x.view(np.uint64)
    hi = (bits >> np.uint64(32)).astype(np.uint32)
    xf = ((hi - np.uint32(896 << 20)) << np.uint32(3)).view(np.float32)
    lg = (np.log2(xf.astype(np.float64)) + dlg).astype(np.float32)
    t2 = np.maximum((np.float64(-kBLn2) * lg.astype(np.float64) + np.float64(kBLnF0)).astype(np.float32),
                    np.float32(0))
    t = np.sqrt(t2.astype(np.float64)).astype(np.float32)
    q = np.rint(t.astype(np.float64))  # t + 1.5 * 2^23 in FP32 rounds to nearest, ties to even
    return np.maximum(100 - q.astype(np.int64), 0)


def test_fp32_bin_estimate_is_exact_or_one_below():
    edges = _edges()
    rng = np.random.default_rng(3)
    xs = np.concatenate([
        10 ** rng.uniform(3, 28, 400000),                       # far below and above the spectrum
        np.concatenate([e * (1 + rng.uniform(-1e-6, 1e-6, 200)) for e in edges]),
        np.nextafter(edges, -np.inf), edges, np.nextafter(edges, np.inf),
        np.array([FRQ0, 2 * FRQ0, 0.5 * oracle.port_compton_frq(1)]),
    ])
    true = np.searchsorted(edges, xs, side="left")  # edges strictly below x
    for dlg in (-2.0 ** -21, 0.0, 2.0 ** -21):
        c = _estimate(xs, dlg)
        assert np.all((c == true) | (c == true - 1)), f"log2 error {dlg}: estimate off by more than one"
        # the kernel's correction with a table edge[0..99], +inf at 100
        edge_pad = np.concatenate([edges, [np.inf]])
        fixed = c + (xs > edge_pad[c])
        assert np.array_equal(fixed, true)
