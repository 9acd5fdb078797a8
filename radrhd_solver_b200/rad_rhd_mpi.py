"""The coupled radiation-hydro step over ranks, mirroring rad_rhd::RunRadRHDMpiModule
(solvers/RadRHD/src/radRHD_mpi_main.cpp:107-122): the hydro step split by cell blocks, the
radiation split by direction (sweep) and by cell rows (scattering integral and moments).

    dist.init_process_group("nccl", ...)                 # one process per GPU
    grid = rhllc.Grid(mesh, device=local_rank)           # every rank holds the whole mesh
    grid.set_state_prim(W0); rhllc_mpi.InitMpiConfig(grid)
    step = RadRHDStepMPI(GpuParts(grid, directions, groups=G, absorption=1.0, scattering=0.5, em=em))
    step(tau)                                            # one pass of the loop body

Per step, in the order of the single-GPU step (rrhd_coupled_step, radRHD_main.cpp:96-139):

1. hydro (rhllc_mpi::Hllc3dStab): the rank's CTA blocks of cells, halo exchange, the max
   signal speed reduced over ranks;
2. StartPhysCast / SyncAndCalcPhysCast: every rank receives the other ranks' cells (one
   all-gather of (id, W, U) rows), so that each holds the whole state after the step;
3. opacities and emission of every cell (the sweep needs all of them for its directions);
4. the sweep of this rank's directions with the previous scattering integral of those
   directions;
5. the 4-force of the rank's row cells from the previous step's moments (the reference
   computes them at the start of each radiation iteration, so they lag a step), gathered to
   every rank; the source update U += tau G and con2prim of every cell, done identically on
   every rank and written back to the rank's context;
6. the intensity to cell rows (all-to-all), the FP64 scattering integral and moments of the
   rank's rows, the integral back to the rank's directions (all-to-all) for the next sweep.

The compute of each piece comes from a `parts` object: `GpuParts` runs the library's kernels
on the context's stream; the host logic above (splits, collectives, the order and the lag)
is the same whatever computes the pieces.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from . import _lib as L
from . import illum, illum_mpi, rad_rhd, rhllc, rhllc_mpi


def gather_cells(ids: torch.Tensor, rows: torch.Tensor, n_total: int, group=None) -> torch.Tensor:
    """Every rank's (ids, rows) to every rank, placed by id: [n_total][width] (the cells
    nobody owns stay zero).  Each rank's block is padded to the largest block (id -1) and
    gathered with one all-gather, so a rank without cells takes part like the others."""
    world = dist.get_world_size(group)
    width = rows.shape[1]
    n = torch.tensor([rows.shape[0]], dtype=torch.int64, device=rows.device)
    dist.all_reduce(n, op=dist.ReduceOp.MAX, group=group)
    nmax = int(n.item())
    payload = torch.full((max(nmax, 1), width + 1), -1.0, dtype=rows.dtype, device=rows.device)
    payload[:rows.shape[0], 0] = ids.to(rows.dtype)
    payload[:rows.shape[0], 1:] = rows
    recv = torch.empty((world * payload.shape[0], width + 1), dtype=rows.dtype, device=rows.device)
    dist.all_gather_into_tensor(recv, payload, group=group)
    keep = recv[:, 0] >= 0
    out = torch.zeros((n_total, width), dtype=rows.dtype, device=rows.device)
    out[recv[keep, 0].long()] = recv[keep, 1:]
    return out


class GpuParts:
    """The pieces of the step on the library's kernels, for one rank's context `grid` (on
    which rhllc_mpi.InitMpiConfig has run).  The sweep runs this rank's directions in FP64;
    the scattering integral (one FMA per term) and the moments are FP64."""

    def __init__(self, grid: rhllc.Grid, directions, groups: int, absorption: float = 1.0,
                 scattering: float = 0.5, em=None, eos: int = rhllc.EOS_IDEAL, gamma: float = 4.0 / 3.0,
                 group=None):
        self.grid, self.G, self.group = grid, groups, group
        self.a, self.b = absorption, scattering
        self.em = em if em is not None else rad_rhd.emission(1.0, 1.0)
        self.eos, self.gamma = eos, gamma
        self.N, self.M = grid.size, directions.size
        self.shard = illum_mpi.DirectionShard(self.N * groups, self.M, group, unit=groups)
        d0, dn = self.shard.my_dirs
        self.dg = illum.DirectionGrid(directions, grid.device)
        self.dg_r = illum.DirectionGrid(directions.subset(d0, dn), grid.device)
        self.sweep_r = illum.TransportSweep(grid, self.dg_r, groups=groups, precision="fp64")
        self.dev = torch.device("cuda", grid.device)
        cfg = grid.mpi_cfg
        ids = np.zeros(cfg.cell_range[1] - cfg.cell_range[0], np.int32)
        L.check(L.lib.rrhd_hydro_part_info(grid.handle, None, None, None, L.ptr(ids)), "part_info")
        self.ids = torch.as_tensor(ids.astype(np.int64), device=self.dev)  # this rank's cells, caller ids
        self.W = torch.empty((self.N, 5), dtype=torch.float64, device=self.dev)
        self.U = torch.empty_like(self.W)

    def hydro_step(self, tau: float):
        return rhllc_mpi.Hllc3dStab(tau, self.grid, stats=False)

    def own_state(self):
        """(ids, W, U) of this rank's cells, caller ids, on the device."""
        L.check(L.lib.rrhd_get_state(self.grid.handle, L.ptr(self.W), L.ptr(self.U), 5, L.RRHD_DEVICE), "get_state")
        return self.ids, self.W[self.ids], self.U[self.ids]

    def set_state(self, W: torch.Tensor, U: torch.Tensor):
        L.check(L.lib.rrhd_set_state(self.grid.handle, L.ptr(W), L.ptr(U), 5, L.RRHD_DEVICE), "set_state")

    def opacities(self, W: torch.Tensor):
        n = W.shape[0]
        alpha = torch.empty(n, dtype=torch.float64, device=self.dev)
        betta = torch.empty_like(alpha)
        Q = torch.empty((n, self.G), dtype=torch.float64, device=self.dev)
        L.check(L.lib.rrhd_rad_opacities(C.byref(self.em), L.ptr(W), 5, n, self.a, self.b, self.G, L.ptr(alpha),
                                         L.ptr(betta), L.ptr(Q), self.grid.stream), "rrhd_rad_opacities")
        return alpha, betta, Q

    def sweep(self, alpha, betta, Q, S_r):
        return illum.CalculateIllum(self.sweep_r, alpha, betta, Q, S_r)

    def moments_rows(self, I_rows):
        return illum.CalculateAllParam(self.dg, I_rows, stream=self.grid.stream)

    def scatter_rows(self, I_rows):
        return illum.CalculateIntScattering(self.dg, I_rows, exact=False, stream=self.grid.stream)

    def rad_source(self, W_cells, E, F, T):
        n = W_cells.shape[0]
        G4 = torch.empty((n, 4), dtype=torch.float64, device=self.dev)
        L.check(L.lib.rrhd_rad_source_rows(C.byref(self.em), L.ptr(W_cells), 5, n, self.a, self.b, self.G,
                                           L.ptr(E), L.ptr(F), L.ptr(T), L.ptr(G4), self.grid.stream),
                "rrhd_rad_source_rows")
        return G4

    def source_c2p(self, U, W, G4, tau):
        st = L.C2pStats()
        L.check(L.lib.rrhd_rad_source_con2prim(self.eos, self.gamma, L.ptr(U), L.ptr(W), 5, L.ptr(G4), tau,
                                               U.shape[0], C.byref(st), self.grid.stream), "source con2prim")
        return U, W, st

    def zeros(self, *shape):
        return torch.zeros(shape, dtype=torch.float64, device=self.dev)

    def ordered(self):
        """Torch work and collectives on the context's stream, after the library's kernels."""
        return _StreamScope(self.dev, torch.cuda.ExternalStream(self.grid.stream, device=self.dev))


class _StreamScope:
    def __init__(self, dev, stream):
        self.dev, self.stream = dev, stream

    def __enter__(self):
        self._d = torch.cuda.device(self.dev)
        self._s = torch.cuda.stream(self.stream)
        self._d.__enter__()
        self._s.__enter__()

    def __exit__(self, *a):
        self._s.__exit__(*a)
        self._d.__exit__(*a)


class RadRHDStepMPI:
    """One rank's side of the coupled step over the ranks of the parts' group; every rank
    calls it with the same tau."""

    def __init__(self, parts):
        self.p = parts
        sh = parts.shard
        self.r0, self.rn = sh.my_rows
        self.c0, self.cn = self.r0 // parts.G, self.rn // parts.G
        G = parts.G
        self.S_r = parts.zeros(parts.N * G, sh.dir_counts[sh.rank])
        self.mom = (parts.zeros(self.rn), parts.zeros(self.rn, 3), parts.zeros(self.rn, 3, 3))

    def __call__(self, tau: float):
        """Returns the source con2prim statistics of every cell (the same on every rank)."""
        with self.p.ordered():
            return self._step(tau)

    def _step(self, tau: float):
        p, sh, grp = self.p, self.p.shard, self.p.group
        p.hydro_step(tau)
        ids, W_own, U_own = p.own_state()
        full = gather_cells(ids, torch.cat([W_own, U_own], 1), p.N, grp)
        W, U = full[:, :5].contiguous(), full[:, 5:].contiguous()
        alpha, betta, Q = p.opacities(W)
        I_r = p.sweep(alpha, betta, Q, self.S_r)
        G4_own = p.rad_source(W[self.c0:self.c0 + self.cn].contiguous(), *self.mom)
        cell_ids = torch.arange(self.c0, self.c0 + self.cn, device=G4_own.device)
        G4 = gather_cells(cell_ids, G4_own, p.N, grp)
        U, W, st = p.source_c2p(U, W, G4, tau)
        p.set_state(W, U)
        I_rows = sh.to_rows(I_r)
        E, F, T = p.moments_rows(I_rows)
        self.mom = (E.contiguous(), F.contiguous(), T.contiguous())
        self.S_r = sh.to_dirs(p.scatter_rows(I_rows).contiguous())
        return st
