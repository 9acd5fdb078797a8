"""GPU parity of the hydro step split over ranks (C ABI: rrhd_hydro_set_part, the halo pack
and unpack kernels, the step over a rank's CTA blocks, the max-speed address).

The ranks are emulated in one process on one GPU: one context per rank, launched one
after another from the host (no kernel waits on another), with device-to-device copies
standing in for the all-to-all between ranks and a max over the ranks' speeds written back
through rrhd_hydro_max_speed_ptr.  Every cell a rank does not own starts from a poison
state.  Bar: each rank's cells, the time steps and the max signal speed equal the oracle's
(the reference's arithmetic on the CPU, oracle.port_hydro_step) and the whole-mesh step bit
for bit over five device-time-stepped steps.

The torch.distributed path (rhllc_mpi) runs with a one-rank NCCL group in a child
process: it must equal the whole-mesh step too.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

import oracle
from cases import GAMMA_53, SPLIT_POISON, split_case
from radrhd_solver_b200 import _lib as L
from radrhd_solver_b200 import rhllc
from radrhd_solver_b200 import rhllc_mpi as RM

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CFL, H_MIN, STEPS = 0.3, 1.0 / 120, 5


def _max_speed(g):
    p = C.c_void_p()
    L.check(L.lib.rrhd_hydro_max_speed_ptr(g.handle, C.byref(p)))
    return torch.as_tensor(RM._DevicePointer(p.value, 1, "<f8"), device="cuda")


def _whole(m, W0, U0):
    g = rhllc.Grid(m, gamma=GAMMA_53)
    g.set_state(W0, U0)
    g.set_time_step(CFL, H_MIN, 1.0)
    return g


@pytest.mark.parametrize("world", [2, 3, 5])
def test_split_step_bitexact_emulated(world):
    m, W0 = split_case()
    N = m.n_cells
    W0, U0 = oracle.port_p2c(W0, 1, GAMMA_53)
    Wp, Up = oracle.port_p2c(np.tile(SPLIT_POISON, (N, 1)), 1, GAMMA_53)
    whole = _whole(m, W0, U0)
    ranks = []
    for r in range(world):
        g = rhllc.Grid(m, gamma=GAMMA_53)
        L.check(L.lib.rrhd_hydro_set_part(g.handle, world, r))
        rng = np.zeros(2, np.int64)
        sc, rc = np.zeros(world, np.int64), np.zeros(world, np.int64)
        L.check(L.lib.rrhd_hydro_part_info(g.handle, L.ptr(rng), L.ptr(sc), L.ptr(rc), None))
        own = np.zeros(rng[1] - rng[0], np.int32)
        L.check(L.lib.rrhd_hydro_part_info(g.handle, None, None, None, L.ptr(own)))
        W, U = Wp.copy(), Up.copy()
        W[own], U[own] = W0[own], U0[own]
        g.set_state(W, U)
        g.set_time_step(CFL, H_MIN, 1.0)
        send = torch.empty((int(sc.sum()), 10), dtype=torch.float64, device="cuda")
        recv = torch.empty((int(rc.sum()), 10), dtype=torch.float64, device="cuda")
        ranks.append(dict(g=g, own=own, sc=sc, rc=rc, send=send, recv=recv))
    for _ in range(STEPS):
        L.check(L.lib.rrhd_hydro_step(whole.handle, 0.0, None))
        for k in ranks:
            L.check(L.lib.rrhd_hydro_pack_halo(k["g"].handle, k["send"].data_ptr()))
            k["g"].sync()
        for r, k in enumerate(ranks):  # the all-to-all
            at = 0
            for q, kq in enumerate(ranks):
                n = int(k["rc"][q])
                s0 = int(kq["sc"][:r].sum())
                assert n == int(kq["sc"][r])
                k["recv"][at:at + n] = kq["send"][s0:s0 + n]
                at += n
        torch.cuda.synchronize()
        for k in ranks:
            L.check(L.lib.rrhd_hydro_unpack_halo(k["g"].handle, k["recv"].data_ptr()))
            L.check(L.lib.rrhd_hydro_step(k["g"].handle, 0.0, None))
            k["g"].sync()
        speeds = [_max_speed(k["g"]) for k in ranks]
        top = torch.stack(speeds).max()
        for s in speeds:
            s.copy_(top.reshape(1))
        torch.cuda.synchronize()
    tau_w, speed_w = whole.step_info()
    Ww, Uw = whole.get_state()
    # the oracle (the reference's arithmetic on the CPU) over the same device-time-stepped steps
    Uo, Wo, speed_o = U0, W0, 1.0
    for _ in range(STEPS):
        tau_o = (CFL * H_MIN) / speed_o
        Uo, Wo, _, _, speed_o = oracle.port_hydro_step(m, Uo, Wo, tau_o, 1, GAMMA_53)
    assert tau_w == tau_o and speed_w == speed_o
    for k in ranks:
        tau, speed = k["g"].step_info()  # reads the max written through the aliased address
        assert tau == tau_o and speed == speed_o
        W, U = k["g"].get_state()
        assert np.array_equal(W[k["own"]], Wo[k["own"]]) and np.array_equal(U[k["own"]], Uo[k["own"]])
        assert np.array_equal(W[k["own"]], Ww[k["own"]]) and np.array_equal(U[k["own"]], Uw[k["own"]])
    owned = np.concatenate([k["own"] for k in ranks])
    assert np.array_equal(np.sort(owned), np.arange(N))


def test_split_refusals():
    """A split context refuses the host-buffer step; world = 1 restores the whole step."""
    m, W0 = split_case(16, 4, 4)
    W0, U0 = oracle.port_p2c(W0, 1, GAMMA_53)
    g = _whole(m, W0, U0)
    L.check(L.lib.rrhd_hydro_set_part(g.handle, 2, 0))
    W, U = W0.copy(), U0.copy()
    assert L.lib.rrhd_hydro_step_host(g.handle, 1e-3, L.ptr(W), L.ptr(U), 5, None) == L.RRHD_ERR_INVALID
    L.check(L.lib.rrhd_hydro_set_part(g.handle, 1, 0))
    L.check(L.lib.rrhd_hydro_step_host(g.handle, 1e-3, L.ptr(W), L.ptr(U), 5, None))
    Uo, Wo, _, _, _ = oracle.port_hydro_step(m, U0, W0, 1e-3, 1, GAMMA_53)
    assert np.array_equal(U, Uo) and np.array_equal(W, Wo)


def _one_rank_nccl():
    import torch.distributed as dist
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:" + os.environ["SPLIT_PORT"], rank=0,
                            world_size=1)
    try:
        m, W0 = split_case()
        W0, U0 = oracle.port_p2c(W0, 1, GAMMA_53)
        whole = _whole(m, W0, U0)
        g = _whole(m, W0, U0)
        cfg = RM.InitMpiConfig(g)
        assert cfg.cell_range == (0, m.n_cells) and cfg.send.shape[0] == 0
        for s in range(STEPS):
            L.check(L.lib.rrhd_hydro_step(whole.handle, 0.0, None))
            st = RM.Hllc3dStab(0.0, g, stats=(s % 2 == 0))
        tau_w, speed_w = whole.step_info()
        assert g.step_info() == (tau_w, speed_w)
        assert st.max_speed == speed_w and rhllc.max_signal_speed == speed_w
        W, U, ids = RM.local_state(g)
        Ww, Uw = whole.get_state()
        assert np.array_equal(W, Ww[ids]) and np.array_equal(U, Uw[ids])
    finally:
        dist.destroy_process_group()
    print("split-nccl-ok")


def test_split_torch_distributed_one_rank():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    env = dict(os.environ, SPLIT_PORT=str(port), NCCL_NVLS_ENABLE="0")
    code = ("import sys; sys.path[:0] = [%r, %r]; import test_gpu_hydro_split as t; t._one_rank_nccl()"
            % (ROOT, os.path.join(ROOT, "tests")))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "split-nccl-ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
