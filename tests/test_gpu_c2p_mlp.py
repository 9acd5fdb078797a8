"""Learned con2prim guess: gradients of the hand-written backward kernels against
the FP64 numpy oracle, training, and the seeded con2prim against the reference
solve.  Bars: gradient relative L2 error <= 1e-4 (FP32 kernels vs FP64 oracle);
seeded con2prim states within 1e-10 of the reference solve: rho and |v| relative,
p relative to the state's energy E (both solves stop at the reference's test
|dp| < 1e-11 E, rhllc_flux_stab.cpp:182, so for cold fast flows with p/E ~ 1e-10
the pressure itself is only defined to ~1e-11 E); states that fall back to the
reference guess are bit-identical to it."""
import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_43, c2p_states
from oracle import mlp_oracle as MO
from radrhd_solver_b200 import _lib as L
from radrhd_solver_b200 import rhllc
from radrhd_solver_b200.c2p_mlp import LearnedGuess

pytestmark = pytest.mark.gpu


def _labelled(n, seed):
    """Config-3 states made by the solver's own prim->cons; the label is p."""
    W = torch.empty(n, 5, dtype=torch.float64, device="cuda")
    L.check(L.lib.rrhd_fill_c2p_states(W.data_ptr(), n, seed, torch.cuda.current_stream().cuda_stream))
    U = torch.empty_like(W)
    rhllc.GetConvValueStab(W, U, eos=1, gamma=GAMMA_43, stream=torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return U, W, W[:, 4].contiguous()


def test_gradient_matches_fp64_oracle():
    U, W, p = _labelled(1000, 7)
    net = LearnedGuess(seed=5)
    net.train(U, p, epochs=1, batch=128, lr=1e-3, seed=1)  # sets the normalisation, moves off the init
    th, nm = net.params()
    g, loss = net.gradient(U, p)
    f, tau = MO.features(U.cpu().numpy())
    x = (f - nm[:3].astype(np.float64)) / nm[3:6].astype(np.float64)
    t = (np.log(p.cpu().numpy() / tau) - nm[6]) / nm[7]
    lo, go = MO.loss_and_grad(th, x, t)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)


def test_training_and_seeded_con2prim():
    U, W, p = _labelled(400_000, 11)
    net = LearnedGuess(seed=2)
    hist = net.train(U, p, epochs=6, batch=2048, lr=2e-3, seed=4)
    print("\nloss per epoch", hist)
    assert hist[-1] < 0.02 * hist[0], hist
    Ut, Wt, pt = _labelled(200_000, 12)  # held-out states
    s = torch.cuda.current_stream().cuda_stream
    # plain reference solve
    U1, W1 = Ut.clone(), torch.zeros_like(Wt)
    st_plain = rhllc.GetPhysValueStabStats(U1, W1, None, eos=1, gamma=GAMMA_43, stream=s)
    # seeded solve
    U2, W2 = Ut.clone(), torch.zeros_like(Wt)
    guess = torch.zeros(len(Ut), dtype=torch.float64, device="cuda")
    st, n_back = net.con2prim(U2, W2, eos=1, gamma=GAMMA_43, guess=guess, stream=s)
    torch.cuda.synchronize()
    a, b = W1.cpu().numpy(), W2.cpu().numpy()
    E = Ut[:, 4].cpu().numpy()
    assert np.all(np.abs(a[:, 0] - b[:, 0]) <= 1e-10 * a[:, 0])
    dv = np.linalg.norm(a[:, 1:4] - b[:, 1:4], axis=1)
    assert np.all(dv <= 1e-10 * np.linalg.norm(a[:, 1:4], axis=1))
    assert np.all(np.abs(a[:, 4] - b[:, 4]) <= 1e-10 * E)
    gi = guess.cpu().numpy()
    err = np.abs(gi / pt.cpu().numpy() - 1)
    print(f"\nplain: {st_plain.newton_iters / len(Ut):.3f} it/state; learned: {st.newton_iters / len(Ut):.3f} "
          f"it/state, guess fallbacks {n_back}, median guess error {np.median(err):.3e}")
    assert st.newton_iters < st_plain.newton_iters
    assert st.n_failed == 0 and st_plain.n_failed == 0


def test_bad_network_falls_back_to_reference_bitwise():
    U, W, p = _labelled(50_000, 13)
    net = LearnedGuess(seed=3)
    net.train(U, p, epochs=1, batch=4096, seed=5)
    th, nm = net.params()
    th[-1] = 20.0  # guesses exp(20 sigma_t) times too large
    net.set_params(th, nm)
    s = torch.cuda.current_stream().cuda_stream
    U1, W1 = U.clone(), torch.zeros_like(W)
    rhllc.GetPhysValueStabStats(U1, W1, None, eos=1, gamma=GAMMA_43, stream=s)
    U2, W2 = U.clone(), torch.zeros_like(W)
    # one Newton step from a far guess never meets the 1e-11 E stopping test
    st, n_back = net.con2prim(U2, W2, eos=1, gamma=GAMMA_43, k_stall=1, stream=s)
    torch.cuda.synchronize()
    assert n_back == len(U)
    assert torch.equal(W1, W2)
