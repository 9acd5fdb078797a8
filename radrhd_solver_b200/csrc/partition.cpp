// Cell order of a context and the split of the hydro step over ranks (host only).
//
// The reference splits the hydro cells over MPI ranks by a METIS partition that the caller
// has already grouped into contiguous ranges (rhllc_mpi::InitMpiConfig,
// solvers/rhllc/src/rhllc_3d_mpi.cpp:86-369): each rank computes the faces touching its
// cells, updates them, exchanges the boundary cells with its neighbours at the start of
// every step (StartExchangeBoundaryCells / SyncExchangeBoundaryCells, :69-85) and reduces
// the max signal speed over ranks (:461-485).  Here a rank owns a contiguous range of the
// context's CTA blocks in Morton order, which is a space-filling-curve partition; the
// cells to exchange are the face neighbours of a rank's cells that another rank owns.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <utility>
#include <vector>

#include "rrhd.h"
#include "rrhd_internal.h"

namespace {

uint64_t spread3(uint64_t x) {
  x &= 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

}  // namespace

extern "C" rrhd_status rrhd_cell_order(const rrhd_mesh_desc *m, int32_t renumber, int32_t *order) {
  RRHD_CHECK_ARG(m && order, "null argument");
  RRHD_CHECK_ARG(m->n_cells > 0 && m->n_cells < (int64_t(1) << 30), "bad mesh sizes");
  const int64_t N = m->n_cells;
  std::iota(order, order + N, 0);
  if (renumber < 0) return RRHD_OK;
  RRHD_CHECK_ARG(m->cell_center, "null cell centres");
  // Morton key of the cell centre, 21 bits per axis over the bounding box
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < N; i++)
    for (int a = 0; a < 3; a++) {
      lo[a] = std::min(lo[a], m->cell_center[3 * i + a]);
      hi[a] = std::max(hi[a], m->cell_center[3 * i + a]);
    }
  std::vector<uint64_t> key(N);
  for (int64_t i = 0; i < N; i++) {
    uint64_t code = 0;
    for (int a = 0; a < 3; a++) {
      const double ext = hi[a] - lo[a];
      const double t = ext > 0 ? (m->cell_center[3 * i + a] - lo[a]) / ext : 0.0;
      const uint64_t q = (uint64_t)std::min(2097151.0, std::max(0.0, t * 2097151.0));
      code |= spread3(q) << a;
    }
    key[i] = code;
  }
  std::stable_sort(order, order + N, [&](int32_t a, int32_t b) { return key[a] < key[b]; });
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_part_plan(const rrhd_mesh_desc *m, const int32_t *order, int32_t cells_per_block,
                                      int32_t world, int32_t rank, int64_t *cell_range, int64_t *send_counts,
                                      int64_t *recv_counts, int32_t *send_ids, int32_t *recv_ids) {
  RRHD_CHECK_ARG(m && order && cell_range && send_counts && recv_counts, "null argument");
  RRHD_CHECK_ARG(m->face_id_l && m->face_id_r, "null mesh array");
  const int64_t N = m->n_cells, F = m->n_faces;
  RRHD_CHECK_ARG(N > 0 && F >= 0 && N < (int64_t(1) << 30), "bad mesh sizes");
  const int cpb = cells_per_block > 0 ? cells_per_block : 256;
  RRHD_CHECK_ARG(cpb >= 32 && cpb <= 1024, "cells_per_block out of [32,1024]");
  const int64_t nb = (N + cpb - 1) / cpb;
  RRHD_CHECK_ARG(world >= 1 && world <= nb, "world must be in [1, number of CTA blocks = %lld]", (long long)nb);
  RRHD_CHECK_ARG(rank >= 0 && rank < world, "rank out of [0, world)");

  // rank q owns the blocks [nb q / world, nb (q+1) / world)
  auto first_block = [&](int64_t q) { return nb * q / world; };
  std::vector<int32_t> block_owner(nb);
  for (int q = 0; q < world; q++)
    for (int64_t b = first_block(q); b < first_block(q + 1); b++) block_owner[b] = q;
  cell_range[0] = std::min<int64_t>(N, first_block(rank) * cpb);
  cell_range[1] = std::min<int64_t>(N, first_block(rank + 1) * cpb);

  std::vector<int32_t> iperm(N, -1);
  for (int64_t k = 0; k < N; k++) {
    RRHD_CHECK_ARG(order[k] >= 0 && order[k] < N && iperm[order[k]] < 0, "order is not a permutation");
    iperm[order[k]] = (int32_t)k;
  }
  // (peer, cell) pairs in context numbering
  std::vector<std::pair<int32_t, int32_t>> snd, rcv;
  for (int64_t f = 0; f < F; f++) {
    const int32_t l = m->face_id_l[f], r = m->face_id_r[f];
    RRHD_CHECK_ARG(l >= 0 && l < N && r < N, "face %lld: bad neighbour", (long long)f);
    if (r < 0) continue;
    const int32_t a = iperm[l], b = iperm[r];
    const int32_t pa = block_owner[a / cpb], pb = block_owner[b / cpb];
    if (pa == pb) continue;
    if (pa == rank) {
      snd.emplace_back(pb, a);
      rcv.emplace_back(pb, b);
    } else if (pb == rank) {
      snd.emplace_back(pa, b);
      rcv.emplace_back(pa, a);
    }
  }
  for (auto *v : {&snd, &rcv}) {
    std::sort(v->begin(), v->end());
    v->erase(std::unique(v->begin(), v->end()), v->end());
  }
  std::fill(send_counts, send_counts + world, 0);
  std::fill(recv_counts, recv_counts + world, 0);
  for (size_t i = 0; i < snd.size(); i++) {
    send_counts[snd[i].first]++;
    if (send_ids) send_ids[i] = snd[i].second;
  }
  for (size_t i = 0; i < rcv.size(); i++) {
    recv_counts[rcv[i].first]++;
    if (recv_ids) recv_ids[i] = rcv[i].second;
  }
  return RRHD_OK;
}
