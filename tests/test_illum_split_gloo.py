"""Host logic of the radiation split over ranks (illum_mpi), with gloo ranks on CPU.

Each rank holds the intensity of its directions for every row ([rows][M_r], the sweep's
output on a direction split); `to_rows` must give it exactly the rows of its row range with all
directions, `to_dirs` the reverse.  The composition with the oracle's scattering integral on
the rank's rows equals the columns of the oracle's whole-matrix integral bit for bit (its rows
are independent).  Direction and row counts that do not divide by the rank count, and the
reference's GetSend / GetDisp split, are covered."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
ROWS, M = 75, 26  # 25 cells x 3 groups, 26 directions


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, ws, port, out):
    import torch
    import torch.distributed as dist
    sys.path[:0] = [ROOT, HERE]
    import oracle
    from radrhd_solver_b200 import illum_mpi as IM
    from radrhd_solver_b200.mesh import fibonacci_directions
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(9)
        I = np.exp(rng.normal(0, 0.5, (ROWS, M)))
        d = fibonacci_directions(M)
        S = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
        sh = IM.DirectionShard(ROWS, M)
        d0, dn = sh.my_dirs
        r0, rn = sh.my_rows
        I_dir = torch.from_numpy(np.ascontiguousarray(I[:, d0:d0 + dn]))
        I_rows = sh.to_rows(I_dir)
        ok_rows = np.array_equal(I_rows.numpy(), I[r0:r0 + rn])
        S_rows = oracle.port_scatter(I_rows.numpy(), d.dirs, d.areas, d.full_area)
        S_dir = sh.to_dirs(torch.from_numpy(S_rows))
        ok_dirs = np.array_equal(S_dir.numpy(), S[:, d0:d0 + dn])
        out.put((rank, (d0, dn), (r0, rn), ok_rows, ok_dirs))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("ws", [2, 3, 4])
def test_direction_split_transposes(ws):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=240) for _ in range(ws))
    for p in ps:
        p.join(60)
    assert all(p.exitcode == 0 for p in ps)
    assert sum(r[1][1] for r in res) == M and sum(r[2][1] for r in res) == ROWS
    for rank, dirs, rows, ok_rows, ok_dirs in res:
        assert ok_rows, f"rank {rank}: to_rows did not give rows {rows} with all directions"
        assert ok_dirs, f"rank {rank}: scattering integral of directions {dirs} differs from the whole matrix"


def test_get_send_disp():
    """The reference's split: n // np each, the first n % np ranks one more; displacements
    their prefix sums (lib/mpi_extension/src/mpi_shifts.cpp:3-28, e.g. 10 over 4 ranks:
    3, 3, 2, 2 at 0, 3, 6, 8)."""
    sys.path[:0] = [ROOT]
    from radrhd_solver_b200.illum_mpi import GetDisp, GetSend
    assert GetSend(4, 10) == [3, 3, 2, 2] and GetDisp(4, 10) == [0, 3, 6, 8]
    assert GetSend(3, 9) == [3, 3, 3] and GetDisp(3, 9) == [0, 3, 6]
    assert GetSend(5, 3) == [1, 1, 1, 0, 0] and GetDisp(5, 3) == [0, 1, 2, 3, 3]
    for np_ in range(1, 9):
        for n in range(0, 40):
            c, d = GetSend(np_, n), GetDisp(np_, n)
            assert sum(c) == n and d == [sum(c[:i]) for i in range(np_)] and max(c) - min(c) <= 1


def test_direction_subset():
    """A rank's share of the direction set keeps the directions' order, their areas and the
    whole sphere's area (the scattering weights a_d / full_area stay the same)."""
    sys.path[:0] = [ROOT]
    from radrhd_solver_b200.illum_mpi import GetDisp, GetSend
    from radrhd_solver_b200.mesh import fibonacci_directions
    d = fibonacci_directions(26)
    parts = [d.subset(o, c) for o, c in zip(GetDisp(3, 26), GetSend(3, 26))]
    assert [p.size for p in parts] == [9, 9, 8]
    assert np.array_equal(np.concatenate([p.dirs for p in parts]), d.dirs)
    assert np.array_equal(np.concatenate([p.areas for p in parts]), d.areas)
    assert all(p.full_area == d.full_area and p.dirs.flags.c_contiguous for p in parts)
