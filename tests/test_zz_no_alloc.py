"""The allocation-free con2prim entry point, checked against the regular one.

rrhd_con2prim_batch_stats_noalloc serves callers that cannot allocate device
memory (their pool or arena owns the GPU, or cudaMalloc's implicit
synchronisation is not acceptable in their loop): its scratch is a fixed
file-scope device array instead of a cudaMalloc'd buffer.  Two calls in a row
with different batches must give exactly (tolerance 0, as for every FP64 path
here) the states, status bytes and totals of rrhd_con2prim_batch_stats.  This
file is collected last so that a run stopping at the first failure has run
every other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_43, c2p_states
from radrhd_solver_b200 import _lib as L

pytestmark = pytest.mark.gpu

MAX_STATES = 16_777_216


def _noalloc():
    f = L.lib.rrhd_con2prim_batch_stats_noalloc
    f.restype = L.I32
    f.argtypes = [L.I32, L.D, L.P, L.P, L.P, L.I64, L.I32, L.P, L.P]
    return f


def _batch(n, seed):
    W = c2p_states(n, GAMMA_43, seed=seed)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    U[::53, 4] *= 0.6  # some states take the fallback
    return U, W


def _run(fn, U, W):
    s = torch.cuda.current_stream().cuda_stream
    Ud = torch.tensor(U, device="cuda")
    Wd = torch.tensor(W, device="cuda")
    sd = torch.zeros(len(U), dtype=torch.uint8, device="cuda")
    st = L.C2pStats()
    L.check(fn(1, GAMMA_43, Ud.data_ptr(), Wd.data_ptr(), sd.data_ptr(), len(U), 1, ctypes.byref(st), s), fn.__name__)
    torch.cuda.synchronize()
    return Ud.cpu().numpy(), Wd.cpu().numpy(), sd.cpu().numpy(), st


def _same(a, b):
    Ua, Wa, sa, ta = a
    Ub, Wb, sb, tb = b
    assert np.array_equal(Ua, Ub) and np.array_equal(Wa, Wb) and np.array_equal(sa, sb)
    for k in ("n_ok", "n_fallback", "n_failed", "newton_iters", "max_iters"):
        assert getattr(ta, k) == getattr(tb, k), k


def test_noalloc_matches_regular_two_calls():
    f = _noalloc()
    for n, seed in ((50_000, 31), (7_777, 32)):  # the second call reuses the array after a larger one
        U, W = _batch(n, seed)
        ref = _run(L.lib.rrhd_con2prim_batch_stats, U, W)
        got = _run(f, U, W)
        _same(got, ref)
        assert got[3].n_fallback > 0 and got[3].n_ok > 0


def test_noalloc_rejects_oversized_batch():
    f = _noalloc()
    d = torch.zeros(5, dtype=torch.float64, device="cuda")
    st = L.C2pStats()
    r = f(1, GAMMA_43, d.data_ptr(), d.data_ptr(), None, MAX_STATES + 1, 1, ctypes.byref(st),
          torch.cuda.current_stream().cuda_stream)
    assert r == L.RRHD_ERR_LIMIT
    assert b"fixed maximum" in L.lib.rrhd_last_error()


def test_noalloc_empty_batch_gives_zero_totals():
    """n = 0 launches only the reduction, which writes a zero total into the first record."""
    f = _noalloc()
    d = torch.zeros(5, dtype=torch.float64, device="cuda")
    for fn in (f, L.lib.rrhd_con2prim_batch_stats):
        st = L.C2pStats()
        st.n_ok = st.n_fallback = st.n_failed = st.newton_iters = st.max_iters = 7
        L.check(fn(1, GAMMA_43, d.data_ptr(), d.data_ptr(), None, 0, 1, ctypes.byref(st),
                   torch.cuda.current_stream().cuda_stream))
        assert (st.n_ok, st.n_fallback, st.n_failed, st.newton_iters, st.max_iters) == (0, 0, 0, 0, 0)


def test_noalloc_at_the_fixed_maximum():
    """A batch of exactly the maximum uses the last per-CTA record of the array and the
    total right after it; a cheap uniform state, compared with the regular entry point."""
    f = _noalloc()
    U1, W1 = _batch(2, 41)
    s = torch.cuda.current_stream().cuda_stream
    out = []
    for fn in (L.lib.rrhd_con2prim_batch_stats, f):
        Ud = torch.tensor(U1[:1], device="cuda").expand(MAX_STATES, 5).contiguous()
        Wd = torch.zeros_like(Ud)
        sd = torch.zeros(MAX_STATES, dtype=torch.uint8, device="cuda")
        st = L.C2pStats()
        L.check(fn(1, GAMMA_43, Ud.data_ptr(), Wd.data_ptr(), sd.data_ptr(), MAX_STATES, 1, ctypes.byref(st), s))
        torch.cuda.synchronize()
        out.append((Ud, Wd, sd, st))
        del Ud, Wd, sd
    (Ua, Wa, sa, ta), (Ub, Wb, sb, tb) = out
    assert torch.equal(Ua, Ub) and torch.equal(Wa, Wb) and torch.equal(sa, sb)
    for k in ("n_ok", "n_fallback", "n_failed", "newton_iters", "max_iters"):
        assert getattr(ta, k) == getattr(tb, k), k
    assert ta.n_ok + ta.n_fallback == MAX_STATES
