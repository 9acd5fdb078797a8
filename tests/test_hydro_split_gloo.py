"""Host logic of the hydro step split over ranks (rhllc_mpi), with gloo ranks on CPU.

Each rank holds the whole mesh but only its own cells' states; every other cell holds a
poison state.  Per step the rank exchanges the rows `part_plan` lists with the other ranks
(`exchange_rows`, the all-to-all the GPU path runs over NCCL), steps the whole mesh with
the oracle, keeps its own cells and poisons the rest again.  After three steps a rank's
cells equal the oracle's whole-mesh run bit for bit, which holds only if the exchange
lists hold every face neighbour that another rank updates.  The same loop without the
exchange must differ (the control that the poison reaches the rank's cells)."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))

TAU = 1e-3
STEPS = 3


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
    from cases import SPLIT_POISON as POISON
    from cases import split_case
    from radrhd_solver_b200 import rhllc_mpi as RM
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m, W0 = split_case()
        N = m.n_cells
        W0, U0 = oracle.port_p2c(W0)
        Wp, Up = oracle.port_p2c(np.tile(POISON, (N, 1)))
        Ur, Wr = U0, W0
        for _ in range(STEPS):
            Ur, Wr, _, _, _ = oracle.port_hydro_step(m, Ur, Wr, TAU, nthreads=4)

        order = RM.cell_order(m)
        plan = RM.part_plan(m, order, ws, rank)
        own = order[plan.cell_range[0]:plan.cell_range[1]]
        others = np.ones(N, bool)
        others[own] = False
        send_rows, recv_rows = order[plan.send_ids], order[plan.recv_ids]

        def run(exchange):
            U, W = Up.copy(), Wp.copy()
            U[own], W[own] = U0[own], W0[own]
            for _ in range(STEPS):
                send = torch.from_numpy(np.hstack([U[send_rows], W[send_rows]]))
                recv = torch.empty((len(recv_rows), 10), dtype=torch.float64)
                RM.exchange_rows(send, recv, plan.send_counts, plan.recv_counts)
                if exchange:
                    r = recv.numpy()
                    U[recv_rows], W[recv_rows] = r[:, :5], r[:, 5:]
                U, W, _, _, _ = oracle.port_hydro_step(m, U, W, TAU, nthreads=4)
                U[others], W[others] = Up[others], Wp[others]
            return np.array_equal(U[own], Ur[own]) and np.array_equal(W[own], Wr[own])

        out.put((rank, own.tolist(), plan.send_counts.tolist(), plan.recv_counts.tolist(), run(True), run(False)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("ws", [2, 3])
def test_split_step_equals_whole_mesh(ws):
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
    owned = np.concatenate([np.array(r[1]) for r in res])
    assert np.array_equal(np.sort(owned), np.arange(len(owned)))  # the ranks' cells partition the mesh
    for rank, _, sc, rc, exact, without in res:
        for q_ in range(ws):
            assert sc[q_] == res[q_][3][rank]  # what rank sends to q is what q receives from it
        assert sc[rank] == 0 and sum(sc) > 0
        assert exact, f"rank {rank}: split step differs from the whole-mesh step"
        assert not without, f"rank {rank}: the poisoned cells never reached the rank's cells"


def test_plan_edges():
    """Counts-only calls, world = 1 (nothing to exchange), the world bound (one CTA block a
    rank at most) and a bad rank."""
    sys.path[:0] = [ROOT, HERE]
    from cases import split_case
    from radrhd_solver_b200 import _lib as L
    from radrhd_solver_b200 import rhllc_mpi as RM
    m, _ = split_case(8, 4, 4)
    order = RM.cell_order(m)
    p = RM.part_plan(m, order, 1, 0)
    assert p.cell_range == (0, m.n_cells) and p.send_counts.tolist() == [0] and len(p.recv_ids) == 0
    nb = -(-m.n_cells // 256)
    last = RM.part_plan(m, order, nb, nb - 1)
    assert last.cell_range == ((nb - 1) * 256, m.n_cells)
    with pytest.raises(L.RrhdError):
        RM.part_plan(m, order, nb + 1, 0)
    with pytest.raises(L.RrhdError):
        RM.part_plan(m, order, 2, 2)
    ident = RM.cell_order(m, renumber=False)
    assert np.array_equal(ident, np.arange(m.n_cells))
    bad = order.copy()
    bad[1] = bad[0]  # not a permutation
    with pytest.raises(L.RrhdError):
        RM.part_plan(m, bad, 2, 0)
    # identity order: rank 0 of 2 owns the first half of the caller's cells
    p0 = RM.part_plan(m, ident, 2, 0)
    assert p0.cell_range == (0, 256 * (nb // 2))
    assert np.all(p0.send_ids < p0.cell_range[1]) and np.all(p0.recv_ids >= p0.cell_range[1])
