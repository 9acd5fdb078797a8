"""Host logic of the coupled step over ranks (rad_rhd_mpi.RadRHDStepMPI), with gloo ranks on CPU
and the oracle computing each piece.

Each rank runs the step's host logic as written (its direction and cell-row shares, the
gathers of the cells and of the 4-force, the intensity and scattering all-to-alls, the
one-step lag of the moments); its pieces come from the oracle: the hydro step of the whole
mesh, after which every cell the rank does not own is poisoned (so the gathered state must
come from the other ranks), the sweep of the rank's directions, the scattering integral and
moments of its rows, the 4-force of its row cells, the source update and con2prim.  After
three steps every rank's state equals the oracle's single-process composition of the same
steps bit for bit, for 2 and 3 ranks."""
import contextlib
import ctypes as C
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))

STEPS = 3
G = 2
M = 12
EM = (1.0, 10.0, np.pi, 1.0)  # temp_coef, a_R, pi, kRadiation of the coupled jet
A, B = 1.0, 0.5               # alpha = A rho, betta = B rho
POISON = np.array([7.0, 0.1, -0.2, 0.3, 5.0])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _setup():
    sys.path[:0] = [ROOT, HERE]
    import oracle
    from cases import GAMMA_43, JET_INFLOW, jet
    from radrhd_solver_b200.mesh import fibonacci_directions
    m, W = jet(4)
    W, U = oracle.port_p2c(W, 1, GAMMA_43)
    ubc = np.zeros(5)
    e = oracle.loader.OrcEos(1, GAMMA_43)
    oracle.port().orc_p2c_plain(C.byref(e), np.ascontiguousarray(JET_INFLOW).ctypes.data, ubc.ctypes.data)
    bc = {-3: (1, JET_INFLOW, ubc)}
    return oracle, GAMMA_43, m, W, U, bc, fibonacci_directions(M), 0.3 * m.h_min


def _opacities(W):
    rho, p = W[:, 0], W[:, 4]
    T = EM[0] * p / rho
    T2 = T * T
    Bp = (T2 * T2) * EM[1] / EM[2]
    return A * rho, B * rho, np.repeat((Bp / EM[3] / G)[:, None], G, axis=1)


def _sum_groups(x):
    x = x.reshape((-1, G) + x.shape[1:])
    s = np.zeros((x.shape[0],) + x.shape[2:])
    for g in range(G):
        s = s + x[:, g]
    return s


def _source_c2p(oracle, gamma, U, W, G4, tau):
    U = U.copy()
    U[:, 4] += tau * G4[:, 0]
    U[:, 1] += tau * G4[:, 1]
    U[:, 2] += tau * G4[:, 2]
    U[:, 3] += tau * G4[:, 3]
    W, _ = oracle.port_c2p(U, 1, gamma, W=W)
    return U, W


def _composition(oracle, gamma, m, W, U, bc, d, tau):
    """The oracle's single-process composition of the steps (radRHD_main.cpp:96-139)."""
    S = np.zeros((m.n_cells * G, M))
    mom = (np.zeros(m.n_cells), np.zeros((m.n_cells, 3)), np.zeros((m.n_cells, 3, 3)))
    for _ in range(STEPS):
        U, W, _, _, _ = oracle.port_hydro_step(m, U, W, tau, 1, gamma, bc=bc)
        alpha, betta, Q = _opacities(W)
        I, missing = oracle.port_sweep(m, d.dirs, alpha, betta, Q, S)
        assert missing == 0
        G4 = oracle.port_rad_source(W, alpha, betta, *mom, EM)
        U, W = _source_c2p(oracle, gamma, U, W, G4, tau)
        S = oracle.port_scatter(I, d.dirs, d.areas, d.full_area)
        E, F, T = oracle.port_moments(I, d.dirs, d.areas, d.full_area)
        mom = (_sum_groups(E), _sum_groups(F), _sum_groups(T))
    return U, W


class OracleParts:
    """RadRHDStepMPI's pieces from the oracle, on CPU tensors."""

    def __init__(self, oracle, gamma, m, W, U, bc, d, own, group=None):
        import torch
        from radrhd_solver_b200 import illum_mpi
        self.o, self.gamma, self.m, self.bc, self.d, self.group = oracle, gamma, m, bc, d, group
        self.N, self.G = m.n_cells, G
        self.shard = illum_mpi.DirectionShard(self.N * G, M, group, unit=G)
        d0, dn = self.shard.my_dirs
        self.d_r = d.subset(d0, dn)
        self.own = own
        self.others = np.ones(self.N, bool)
        self.others[own] = False
        self.W, self.U = W.copy(), U.copy()
        self.t = lambda a: torch.from_numpy(np.ascontiguousarray(a))

    def hydro_step(self, tau):
        self.U, self.W, _, _, _ = self.o.port_hydro_step(self.m, self.U, self.W, tau, 1, self.gamma, bc=self.bc)
        Wp, Up = self.o.port_p2c(np.tile(POISON, (self.N, 1)), 1, self.gamma)
        self.W[self.others], self.U[self.others] = Wp[self.others], Up[self.others]

    def own_state(self):
        import torch
        return torch.from_numpy(self.own.astype(np.int64)), self.t(self.W[self.own]), self.t(self.U[self.own])

    def set_state(self, W, U):
        self.W, self.U = W.numpy().copy(), U.numpy().copy()

    def opacities(self, W):
        return tuple(self.t(x) for x in _opacities(W.numpy()))

    def sweep(self, alpha, betta, Q, S_r):
        I, missing = self.o.port_sweep(self.m, self.d_r.dirs, alpha.numpy(), betta.numpy(), Q.numpy(), S_r.numpy())
        assert missing == 0
        return self.t(I)

    def moments_rows(self, I_rows):
        return tuple(self.t(x) for x in self.o.port_moments(I_rows.numpy(), self.d.dirs, self.d.areas, self.d.full_area))

    def scatter_rows(self, I_rows):
        return self.t(self.o.port_scatter(I_rows.numpy(), self.d.dirs, self.d.areas, self.d.full_area))

    def rad_source(self, W_cells, E, F, T):
        Wc = W_cells.numpy()
        alpha, betta, _ = _opacities(Wc)
        mom = (_sum_groups(E.numpy()), _sum_groups(F.numpy()), _sum_groups(T.numpy()))
        return self.t(self.o.port_rad_source(Wc, alpha, betta, *mom, EM))

    def source_c2p(self, U, W, G4, tau):
        U2, W2 = _source_c2p(self.o, self.gamma, U.numpy(), W.numpy(), G4.numpy(), tau)
        return self.t(U2), self.t(W2), None

    def zeros(self, *shape):
        import torch
        return torch.zeros(shape, dtype=torch.float64)

    def ordered(self):
        return contextlib.nullcontext()


def _rank(rank, ws, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws,
                            timeout=datetime.timedelta(seconds=120))
    try:
        oracle, gamma, m, W, U, bc, d, tau = _setup()
        from radrhd_solver_b200 import rad_rhd_mpi, rhllc_mpi
        order = rhllc_mpi.cell_order(m)
        plan = rhllc_mpi.part_plan(m, order, ws, rank, cells_per_block=64)
        own = order[plan.cell_range[0]:plan.cell_range[1]]
        parts = OracleParts(oracle, gamma, m, W, U, bc, d, own)
        step = rad_rhd_mpi.RadRHDStepMPI(parts)
        for _ in range(STEPS):
            step(tau)
        Uo, Wo = _composition(oracle, gamma, m, W, U, bc, d, tau)
        out.put((rank, len(own), np.array_equal(parts.U, Uo), np.array_equal(parts.W, Wo),
                 float(np.max(np.abs(parts.U - Uo)))))
    except Exception as e:  # report instead of leaving the parent waiting
        out.put((rank, -1, False, False, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(600)
@pytest.mark.parametrize("ws", [2, 3])
def test_coupled_step_split_matches_composition(ws):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    res.sort()
    print(f"\n{ws} ranks: own cells {[r[1] for r in res]}, max |dU| {[r[4] for r in res]}")
    assert sum(r[1] for r in res) == 384
    assert all(r[2] and r[3] for r in res)
