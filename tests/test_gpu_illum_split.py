"""GPU parity of the radiation split over ranks: the sweep by direction and the scattering
integral by cell rows.

Ranks are emulated in one process on one GPU (one context per rank, launched one after
another; slicing stands in for the two all-to-alls, whose host logic the gloo test covers):
  * each rank's FP64 sweep over its own directions (a DirectionGrid of its subset) equals
    those columns of the whole sweep bit for bit;
  * the FP64 scattering integral of each rank's row range, from all directions of those
    rows, equals those rows of the whole-matrix integral bit for bit.
The torch.distributed layer (illum_mpi) runs on a one-rank NCCL group in a child process.
"""
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from cases import GAMMA_43
from radrhd_solver_b200 import illum, rhllc
from radrhd_solver_b200 import illum_mpi as IM
from radrhd_solver_b200.mesh import fibonacci_directions, kuhn_box

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _inputs(m, M, G, seed=31):
    rng = np.random.default_rng(seed)
    alpha = 10 ** rng.uniform(-1, 1.5, m.n_cells)
    Q = 10 ** rng.uniform(-2, 0, (m.n_cells, G))
    S = 10 ** rng.uniform(-3, -1, (m.n_cells * G, M))
    return alpha, 0.5 * alpha, Q, S


def _sweep(m, d, G, alpha, betta, Q, S):
    grid = rhllc.Grid(m, gamma=GAMMA_43)
    dg = illum.DirectionGrid(d)
    sw = illum.TransportSweep(grid, dg, groups=G, precision="fp64")
    t = [torch.tensor(a, dtype=torch.float64, device="cuda").contiguous() for a in (alpha, betta, Q, S)]
    torch.cuda.synchronize()
    I = illum.CalculateIllum(sw, *t)
    grid.sync()
    out = I.cpu().numpy()
    grid.close()
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_sweep_by_direction_and_scattering_by_rows(world):
    m = kuhn_box(8, 6, 5, lo=(-1, -1, -1), hi=(1, 1, 1), seed=23)
    d = fibonacci_directions(40)
    G = 2
    alpha, betta, Q, S = _inputs(m, d.size, G)
    I_whole = _sweep(m, d, G, alpha, betta, Q, S)
    cnt, disp = IM.GetSend(world, d.size), IM.GetDisp(world, d.size)
    for r in range(world):
        cols = slice(disp[r], disp[r] + cnt[r])
        I_r = _sweep(m, d.subset(disp[r], cnt[r]), G, alpha, betta, Q, np.ascontiguousarray(S[:, cols]))
        assert np.array_equal(I_r, I_whole[:, cols]), f"rank {r}: sweep of directions {cols} differs"

    dg = illum.DirectionGrid(d)
    I = torch.tensor(I_whole, device="cuda")
    S_whole = illum.CalculateIntScattering(dg, I).cpu().numpy()
    rows = I.shape[0]
    rc, rd = IM.GetSend(world, rows), IM.GetDisp(world, rows)
    for r in range(world):
        S_r = illum.CalculateIntScattering(dg, I[rd[r]:rd[r] + rc[r]])  # a row range: no exchange
        torch.cuda.synchronize()
        assert np.array_equal(S_r.cpu().numpy(), S_whole[rd[r]:rd[r] + rc[r]])


def _one_rank_nccl():
    import torch.distributed as dist
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:" + os.environ["SPLIT_PORT"], rank=0,
                            world_size=1)
    try:
        d = fibonacci_directions(24)
        dg = illum.DirectionGrid(d)
        rng = np.random.default_rng(2)
        I = torch.tensor(np.exp(rng.normal(0, 0.5, (50, d.size))), device="cuda")
        sh = IM.DirectionShard(50, d.size)
        assert sh.my_dirs == (0, 24) and sh.my_rows == (0, 50)
        S = IM.CalculateIntScattering(sh, dg, I)
        S_ref = illum.CalculateIntScattering(dg, I)
        E, F, T = IM.CalculateAllParam(sh, dg, I)
        E_ref, F_ref, T_ref = illum.CalculateAllParam(dg, I)
        torch.cuda.synchronize()
        assert torch.equal(S, S_ref) and torch.equal(E, E_ref) and torch.equal(F, F_ref) and torch.equal(T, T_ref)
    finally:
        dist.destroy_process_group()
    print("illum-split-nccl-ok")


def test_illum_split_torch_distributed_one_rank():
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    env = dict(os.environ, SPLIT_PORT=str(port), NCCL_NVLS_ENABLE="0")
    code = ("import sys; sys.path[:0] = [%r, %r]; import test_gpu_illum_split as t; t._one_rank_nccl()"
            % (ROOT, os.path.join(ROOT, "tests")))
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "illum-split-nccl-ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
