"""Radiation over several ranks: the sweep split by direction, the scattering integral by
cell rows, mirroring the reference's MPI radiation drivers
(solvers/illum/src/mpi/illum_mpi_sender.cpp:10-59, lib/mpi_extension/src/mpi_shifts.cpp:3-28).

    shard = DirectionShard(rows=N * G, M=M)               # InitSender
    dg_r = illum.DirectionGrid(directions.subset(*shard.my_dirs))
    sw_r = illum.TransportSweep(grid, dg_r, groups=G)     # this rank's directions only
    I_r = illum.CalculateIllum(sw_r, alpha, betta, Q, S_r)        # [N*G][M_r]
    S_r = CalculateIntScattering(shard, dg, I_r)                 # [N*G][M_r] for the next sweep

The reference sweeps each rank's directions and then sends every direction's intensity
column to every other rank (one persistent MPI send per direction and peer), so that every
rank holds the whole intensity and computes the scattering integral for its own directions.
Here the intensity moves once by an all-to-all to a split by cell rows ([rows_r][M] on rank
r, all directions of its rows), the scattering integral runs on those rows (its rows are
independent, so no exchange is needed there), and a second all-to-all returns each rank's
directions of it ([rows][M_r]).  A rank receives 2 rows M (R-1)/R^2 values per iteration
instead of the reference's rows (M - M_r) ~ rows M (R-1)/R: R/2 times less NVLink traffic.
Both all-to-alls are NCCL collectives on the caller's stream; the direction and row counts
per rank are the reference's GetSend / GetDisp split.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from . import illum


def GetSend(np_: int, n: int) -> list:
    """Items per rank: n // np_ each, one more for the first n % np_ ranks
    (lib/mpi_extension/src/mpi_shifts.cpp:3-13)."""
    return [n // np_ + (1 if i < n % np_ else 0) for i in range(np_)]


def GetDisp(np_: int, n: int) -> list:
    """First item of each rank: the exclusive prefix sum of GetSend (mpi_shifts.cpp:15-28)."""
    c = GetSend(np_, n)
    return [int(x) for x in np.concatenate([[0], np.cumsum(c)[:-1]])]


class DirectionShard:
    """Direction split of M directions and row split of `rows` rows (cell * G + g) over the
    ranks of `group`; the two transposes between them."""

    def __init__(self, rows: int, M: int, group=None, unit: int = 1):
        """unit: rows are split in whole blocks of `unit` (the G group rows of one cell, so
        that a rank's rows are whole cells)."""
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        if rows % unit:
            raise ValueError(f"{rows} rows are not whole blocks of {unit}")
        if self.world > M or self.world > rows // unit:
            raise ValueError(f"{self.world} ranks for {M} directions and {rows} rows")
        self.rows, self.M, self.unit = rows, M, unit
        self.dir_counts, self.dir_disp = GetSend(self.world, M), GetDisp(self.world, M)
        self.row_counts = [c * unit for c in GetSend(self.world, rows // unit)]
        self.row_disp = [c * unit for c in GetDisp(self.world, rows // unit)]

    @property
    def my_dirs(self):
        """(first direction, count) of this rank."""
        return self.dir_disp[self.rank], self.dir_counts[self.rank]

    @property
    def my_rows(self):
        """(first row, count) of this rank."""
        return self.row_disp[self.rank], self.row_counts[self.rank]

    def to_rows(self, I_dir: torch.Tensor) -> torch.Tensor:
        """[rows][M_r] of this rank's directions -> [rows_r][M] of this rank's rows.  Row block q
        of the input is contiguous and goes to rank q as it is; the blocks received (one per
        direction range) are placed side by side."""
        r, R = self.rank, self.world
        mr = self.dir_counts[r]
        assert I_dir.shape == (self.rows, mr) and I_dir.is_contiguous()
        nr = self.row_counts[r]
        recv = torch.empty(nr * self.M, dtype=I_dir.dtype, device=I_dir.device)
        dist.all_to_all_single(recv, I_dir.reshape(-1),
                               output_split_sizes=[nr * self.dir_counts[q] for q in range(R)],
                               input_split_sizes=[self.row_counts[q] * mr for q in range(R)], group=self.group)
        out = torch.empty((nr, self.M), dtype=I_dir.dtype, device=I_dir.device)
        at = 0
        for q in range(R):
            n = nr * self.dir_counts[q]
            out[:, self.dir_disp[q]:self.dir_disp[q] + self.dir_counts[q]] = recv[at:at + n].view(nr, -1)
            at += n
        return out

    def to_dirs(self, S_rows: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """[rows_r][M] of this rank's rows -> [rows][M_r] of this rank's directions.  Direction
        range q of the input is packed for rank q; the blocks received are the row blocks of
        the result in rank order, so they land in place."""
        r, R = self.rank, self.world
        nr, mr = self.row_counts[r], self.dir_counts[r]
        assert S_rows.shape == (nr, self.M)
        send = torch.cat([S_rows[:, self.dir_disp[q]:self.dir_disp[q] + self.dir_counts[q]].reshape(-1)
                          for q in range(R)])
        if out is None:
            out = torch.empty((self.rows, mr), dtype=S_rows.dtype, device=S_rows.device)
        assert out.shape == (self.rows, mr) and out.is_contiguous()
        dist.all_to_all_single(out.view(-1), send,
                               output_split_sizes=[self.row_counts[q] * mr for q in range(R)],
                               input_split_sizes=[nr * self.dir_counts[q] for q in range(R)], group=self.group)
        return out


def CalculateIntScattering(shard: DirectionShard, dg: illum.DirectionGrid, I_dir: torch.Tensor,
                           S_dir: torch.Tensor | None = None, exact: bool = True) -> torch.Tensor:
    """Scattering integral of this rank's directions from its sweep output, FP64
    (the reference's SEPARATE_GPU MPI path: exchange, then CalculateIntScatteringAsync for
    directions start_dir .. end_dir, cuda_interface_sep_solve.cu:43-88).  `dg` holds all M
    directions."""
    I_rows = shard.to_rows(I_dir)
    S_rows = illum.CalculateIntScattering(dg, I_rows, exact=exact,
                                          stream=torch.cuda.current_stream().cuda_stream)
    return shard.to_dirs(S_rows, S_dir)


def CalculateAllParam(shard: DirectionShard, dg: illum.DirectionGrid, I_dir: torch.Tensor):
    """Energy, stream and impulse of this rank's rows (E [rows_r], F [rows_r][3], T [rows_r][3][3])
    from its sweep output (cuda_illum_sep_param.cu:9-83 on the rank's share of the cells)."""
    I_rows = shard.to_rows(I_dir)
    return illum.CalculateAllParam(dg, I_rows, stream=torch.cuda.current_stream().cuda_stream)
