"""Hydro step split over ranks, mirroring the reference's `rhllc_mpi` namespace
(solvers/rhllc/include/rhllc_mpi.h, solvers/rhllc/src/rhllc_3d_mpi.cpp).

    dist.init_process_group("nccl", ...)              # one process per GPU
    grid = rhllc.Grid(mesh, device=local_rank)        # every rank holds the whole mesh
    grid.set_state_prim(W0)
    InitMpiConfig(grid)                               # rhllc_mpi::InitMpiConfig
    Hllc3dStab(tau, grid)                             # rhllc_mpi::Hllc3dStab
    W, U, ids = local_state(grid)                     # this rank's cells (caller ids)

A rank updates a contiguous range of the context's Morton-ordered CTA blocks
(`rrhd_part_plan`).  Each step: the states that other ranks need are packed by the
library's kernel, exchanged as one all-to-all of 80-byte rows (NCCL over NVLink /
NVSwitch), unpacked, the fused step runs over the rank's blocks, and the max signal speed
is max-reduced over ranks in place on the device, so that the next step's
device-computed time step is the same on every rank.  Everything is ordered on the
context's stream; nothing synchronises the host unless statistics are asked for.

Deviation from the reference: the partition is the Morton block split, not a caller's
METIS map, and a rank may have any number of neighbour ranks (the reference allows two,
rhllc_mpi.h:70).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from . import _lib as L
from .mesh import Mesh
from . import rhllc


def cell_order(mesh: Mesh, renumber: bool = True) -> np.ndarray:
    """order[k] = caller id of the k-th cell of a context built on `mesh` (host only)."""
    order = np.empty(mesh.n_cells, np.int32)
    L.check(L.lib.rrhd_cell_order(C.byref(mesh.desc()), 0 if renumber else -1, L.ptr(order)), "cell_order")
    return order


@dataclass
class PartPlan:
    """One rank's share of the split step; ids in context order (see `cell_order`)."""
    cell_range: tuple
    send_counts: np.ndarray
    recv_counts: np.ndarray
    send_ids: np.ndarray
    recv_ids: np.ndarray


def part_plan(mesh: Mesh, order: np.ndarray, world: int, rank: int, cells_per_block: int = 0) -> PartPlan:
    """The cells of `rank` and its exchange lists (host only): InitMpiConfig's geometry part
    (solvers/rhllc/src/rhllc_3d_mpi.cpp:86-369)."""
    order = np.ascontiguousarray(order, np.int32)
    rng = np.zeros(2, np.int64)
    sc = np.zeros(world, np.int64)
    rc = np.zeros(world, np.int64)
    d = mesh.desc()
    L.check(L.lib.rrhd_part_plan(C.byref(d), L.ptr(order), cells_per_block, world, rank, L.ptr(rng), L.ptr(sc),
                                 L.ptr(rc), None, None), "part_plan")
    sid = np.zeros(int(sc.sum()), np.int32)
    rid = np.zeros(int(rc.sum()), np.int32)
    L.check(L.lib.rrhd_part_plan(C.byref(d), L.ptr(order), cells_per_block, world, rank, L.ptr(rng), L.ptr(sc),
                                 L.ptr(rc), L.ptr(sid), L.ptr(rid)), "part_plan")
    return PartPlan((int(rng[0]), int(rng[1])), sc, rc, sid, rid)


def exchange_rows(send: torch.Tensor, recv: torch.Tensor, send_counts, recv_counts, group=None):
    """All-to-all of row blocks: send rows [sum(send_counts[:q]), +send_counts[q]) go to
    rank q, which receives them at its recv rows [sum(recv_counts[:p]), +recv_counts[p])
    for this rank p.  The transfer of StartExchangeBoundaryCells / SyncExchangeBoundaryCells
    (rhllc_3d_mpi.cpp:69-85)."""
    dist.all_to_all_single(recv, send, output_split_sizes=[int(x) for x in recv_counts],
                           input_split_sizes=[int(x) for x in send_counts], group=group)


class _DevicePointer:
    """A device address as a 1-D array that torch can alias without a copy."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False), "strides": None,
                                         "version": 2}


@dataclass
class MpiConfig:
    """mpi_hd_t of the reference (solvers/rhllc/include/rhllc_mpi.h): the split and its buffers."""
    world: int
    rank: int
    group: object
    device: torch.device
    stream: torch.cuda.ExternalStream
    cell_range: tuple
    send_counts: np.ndarray
    recv_counts: np.ndarray
    send: torch.Tensor  # [n_send][10] U(5), W(5)
    recv: torch.Tensor  # [n_recv][10]


def InitMpiConfig(grid: rhllc.Grid, group=None) -> MpiConfig:
    """Splits `grid`'s hydro step over the ranks of `group` (rhllc_mpi::InitMpiConfig,
    rhllc_3d_mpi.cpp:86-369).  Every rank calls it with the same mesh and options."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    L.check(L.lib.rrhd_hydro_set_part(grid.handle, world, rank), "InitMpiConfig")
    rng = np.zeros(2, np.int64)
    sc = np.zeros(world, np.int64)
    rc = np.zeros(world, np.int64)
    L.check(L.lib.rrhd_hydro_part_info(grid.handle, L.ptr(rng), L.ptr(sc), L.ptr(rc), None), "part_info")
    dev = torch.device("cuda", grid.device)
    cfg = MpiConfig(world, rank, group, dev, torch.cuda.ExternalStream(grid.stream, device=dev),
                    (int(rng[0]), int(rng[1])), sc, rc,
                    torch.empty((int(sc.sum()), 10), dtype=torch.float64, device=dev),
                    torch.empty((int(rc.sum()), 10), dtype=torch.float64, device=dev))
    grid.mpi_cfg = cfg
    return cfg


def ExchangeBoundaryCells(grid: rhllc.Grid):
    """Brings the states of the neighbour cells that other ranks update into this rank's
    context (StartExchangeBoundaryCells + SyncExchangeBoundaryCells, rhllc_3d_mpi.cpp:69-85),
    ordered on the context's stream."""
    cfg: MpiConfig = grid.mpi_cfg
    with torch.cuda.device(cfg.device), torch.cuda.stream(cfg.stream):
        L.check(L.lib.rrhd_hydro_pack_halo(grid.handle, cfg.send.data_ptr()), "pack_halo")
        exchange_rows(cfg.send, cfg.recv, cfg.send_counts, cfg.recv_counts, cfg.group)
        L.check(L.lib.rrhd_hydro_unpack_halo(grid.handle, cfg.recv.data_ptr()), "unpack_halo")


def Hllc3dStab(tau: float, grid: rhllc.Grid, stats: bool = True):
    """One split step (rhllc_mpi::Hllc3dStab, rhllc_3d_mpi.cpp:371-486): exchange, the
    fused step over this rank's blocks, max-reduction of the signal speed.  tau <= 0 uses
    the device-computed CFL step (same on every rank).  With stats, synchronises and
    returns the totals over ranks (StepStats), setting rhllc.max_signal_speed; raises
    RrhdError on every rank when con2prim failed in some cell after the fallback (the
    reference's DIE_IF), after all ranks have taken the same collective steps."""
    cfg: MpiConfig = grid.mpi_cfg
    ExchangeBoundaryCells(grid)
    st = L.StepStats()
    with torch.cuda.device(cfg.device), torch.cuda.stream(cfg.stream):
        code = L.lib.rrhd_hydro_step(grid.handle, tau, C.byref(st) if stats else None)
        if code not in (0, L.RRHD_ERR_C2P):
            L.check(code, "Hllc3dStab")
        p = C.c_void_p()
        L.check(L.lib.rrhd_hydro_max_speed_ptr(grid.handle, C.byref(p)), "max_speed_ptr")
        speed = torch.as_tensor(_DevicePointer(p.value, 1, "<f8"), device=cfg.device)
        dist.all_reduce(speed, op=dist.ReduceOp.MAX, group=cfg.group)
        if not stats:
            return None
        counts = torch.tensor([st.n_fallback, st.n_failed], dtype=torch.int64, device=cfg.device)
        dist.all_reduce(counts, op=dist.ReduceOp.SUM, group=cfg.group)
        host = counts.cpu()
        st.max_speed = float(speed.cpu()[0])
    st.n_fallback, st.n_failed = int(host[0]), int(host[1])
    rhllc.max_signal_speed = st.max_speed
    if st.n_failed:
        raise L.RrhdError(L.RRHD_ERR_C2P, f"Hllc3dStab: con2prim failed in {st.n_failed} cells after the fallback")
    return st


def local_state(grid: rhllc.Grid):
    """(W, U, ids): the states of this rank's cells and their caller ids (synchronises)."""
    cfg: MpiConfig = grid.mpi_cfg
    n = cfg.cell_range[1] - cfg.cell_range[0]
    ids = np.zeros(n, np.int32)
    L.check(L.lib.rrhd_hydro_part_info(grid.handle, None, None, None, L.ptr(ids)), "part_info")
    W, U = grid.get_state()
    return W[ids], U[ids], ids
