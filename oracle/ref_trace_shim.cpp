// Test infrastructure, not product code: the reference's own preprocessing of the
// transport sweep, compiled from its sources (make_trace/src/trace_nodes.cpp,
// make_trace/src/trace_transitions.cpp, lib/geometry/src/intersections.cpp,
// graph/src/graph_calc.cpp, graph/src/graph_init_state.cpp) without VTK, driven on a
// mesh given as arrays:
//   ref_trace_nodes   the short-characteristic geometry of every (direction, cell,
//                     out-face, node): trace::GetInterpolationNodes places the nodes,
//                     trace::GetLocNodes traces each back along -w to the in-face it
//                     comes through and the distance s, as make_trace/src/trace_main.cpp
//                     runs them per direction;
//   ref_graph_levels  the sweep order of graph::RunGraphModule
//                     (graph/src/graph_by_direction.cpp): fronts of cells whose in-faces
//                     are all defined, from graph::FindNumberOfAllInAndDefFaces,
//                     graph::FindCurFrontWithHole and graph::NewStep; the front index of
//                     every cell is returned.
// The reference builds its inputs from VTK files: the vertex matrix of a cell has the
// cell's points as columns (GetVertexMatrix, lib/geometry/src/convert_vtk_geo.cpp:399-415)
// and its faces are VTK's tetra faces {0,1,3}, {1,2,3}, {2,0,3}, {0,2,1}
// (GetFacesPoints, :9-25); the caller passes the points in that order.
#include <cstdint>
#include <map>
#include <set>
#include <vector>

#include "global_types.h"
#include "graph_calc.h"
#include "graph_init_state.h"
#include "graph_struct.h"
#include "intersections.h"
#include "trace_nodes.h"

// The reference defines this global beside its graph driver (graph/src/graph_main.cpp:22),
// which is not linked here.
std::vector<graph::boundary_trace_t> graph::bound_trace;

namespace {
const int kVtkFace[4][3] = {{0, 1, 3}, {1, 2, 3}, {2, 0, 3}, {0, 2, 1}};

void make_cells(int64_t N, const double *vert, const double *nrm, std::vector<Eigen::Matrix4d> &vertexs,
                std::vector<Face> &grid, std::vector<Normals> &normals) {
  vertexs.resize(N);
  grid.resize(4 * N);
  normals.resize(N);
  for (int64_t c = 0; c < N; c++) {
    const double *P = vert + 12 * c;
    Eigen::Matrix4d &V = vertexs[c];
    for (int j = 0; j < 3; j++)
      for (int p = 0; p < 4; p++) V(j, p) = P[3 * p + j];
    for (int p = 0; p < 4; p++) V(3, p) = 1;
    for (int f = 0; f < 4; f++) {
      Face &F = grid[4 * c + f];
      F.A = Vector3(P[3 * kVtkFace[f][0]], P[3 * kVtkFace[f][0] + 1], P[3 * kVtkFace[f][0] + 2]);
      F.B = Vector3(P[3 * kVtkFace[f][1]], P[3 * kVtkFace[f][1] + 1], P[3 * kVtkFace[f][1] + 2]);
      F.C = Vector3(P[3 * kVtkFace[f][2]], P[3 * kVtkFace[f][2] + 1], P[3 * kVtkFace[f][2] + 2]);
      normals[c].n[f] = Vector3(nrm[12 * c + 3 * f], nrm[12 * c + 3 * f + 1], nrm[12 * c + 3 * f + 2]);
    }
  }
}
}  // namespace

extern "C" {

// vert [N][4][3] points in VTK order, nrm [N][4][3] outward unit normals of the VTK faces,
// dirs [M][3].  Out: state [M][N] the in/out bits of intersection::FindInAndOutFaces
// (bit j set: face j is an in-face), in_face [M][N][4][3] and s [M][N][4][3] per out-face
// and node (-1 / 0 for in-faces); nodes (may be NULL) [N][4][3][3] the node positions of
// trace::GetInterpolationNodes.  A face whose three nodes do not all meet an in-face is
// reported with in_face -2 and is not passed to trace::GetLocNodes (the reference stops
// the program there, trace_nodes.cpp:228-231).  Returns the number of such faces.
int64_t ref_trace_nodes(int64_t N, const double *vert, const double *nrm, int32_t M, const double *dirs,
                        int32_t *state, int32_t *in_face, double *s, double *nodes) {
  std::vector<Eigen::Matrix4d> vertexs;
  std::vector<Face> grid;
  std::vector<Normals> normals;
  make_cells(N, vert, nrm, vertexs, grid, normals);
  std::vector<BasePointTetra> vec_x(N);
  trace::GetInterpolationNodes(vertexs, vec_x);
  if (nodes)
    for (int64_t c = 0; c < N; c++)
      for (int j = 0; j < 4; j++)
        for (int q = 0; q < 3; q++)
          for (int x = 0; x < 3; x++) nodes[((c * 4 + j) * 3 + q) * 3 + x] = vec_x[c].x[j][q][x];
  std::vector<IntId> neighbours(4 * N, -1);  // read only with INTERPOLATION_ON_FACES
  std::vector<cell_local> vec_x0;
  int64_t missed = 0;
  for (int32_t d = 0; d < M; d++) {
    const Vector3 dir(dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2]);
    for (int64_t c = 0; c < N; c++) {
      bits_flag_t fs = 0;
      intersection::FindInAndOutFaces(dir, normals[c], fs);
      state[(int64_t)d * N + c] = (int32_t)fs;
      for (int j = 0; j < 4; j++) {
        int32_t *hf = in_face + (((int64_t)d * N + c) * 4 + j) * 3;
        double *sd = s + (((int64_t)d * N + c) * 4 + j) * 3;
        for (int q = 0; q < 3; q++) {
          hf[q] = -1;
          sd[q] = 0;
        }
        if (CHECK_BIT(fs, j) != e_face_type_out) continue;
        bool all = true;
        for (int q = 0; q < 3 && all; q++) {
          bool hit = false;
          for (int f = 0; f < 4 && !hit; f++) {
            if (CHECK_BIT(fs, f) == e_face_type_out) continue;
            Vector3 x0;
            hit = intersection::RayIntersectsTriangle(vec_x[c].x[j][q], -dir, grid[4 * c + f], x0) > 0;
          }
          all = hit;
        }
        if (!all) {
          for (int q = 0; q < 3; q++) hf[q] = -2;
          missed++;
          continue;
        }
        vec_x0.clear();
        trace::GetLocNodes((int)c, (ShortId)j, grid, vertexs[c], fs, dir, normals[c], neighbours, vec_x[c], vec_x0);
        for (int q = 0; q < 3; q++) {
          hf[q] = vec_x0[q].in_face_id;
          sd[q] = vec_x0[q].s;
        }
      }
    }
  }
  return missed;
}

// nbr [N][4]: neighbour cell * 4 + its local face index, or < 0 on the boundary;
// nrm [N][4][3] as above.  Out: level [M][N] the front index of every cell (-1: never
// reached).  Returns the number of directions whose graph misses some cell.
int32_t ref_graph_levels(int64_t N, const int32_t *nbr, const double *nrm, int32_t M, const double *dirs,
                         int32_t *level) {
  std::vector<IntId> neighbours(nbr, nbr + 4 * N);
  std::vector<Normals> normals(N);
  for (int64_t c = 0; c < N; c++)
    for (int f = 0; f < 4; f++)
      normals[c].n[f] = Vector3(nrm[12 * c + 3 * f], nrm[12 * c + 3 * f + 1], nrm[12 * c + 3 * f + 2]);
  const std::map<IntId, FaceCell> inter_faces;  // no inner boundary
  const std::set<IntId> inter_boundary_face_id;
  int32_t bad = 0;
  for (int32_t d = 0; d < M; d++) {
    const Vector3 dir(dirs[3 * d], dirs[3 * d + 1], dirs[3 * d + 2]);
    int32_t *lv = level + (int64_t)d * N;
    for (int64_t c = 0; c < N; c++) lv[c] = -1;
    std::vector<State> count_in_face, count_def_face, faces_state;
    std::set<IntId> inner_part, outer_part, next_step_el;
    std::vector<IntId> cur_el;
    graph::InitFacesState(neighbours, inter_faces, faces_state);
    graph::DivideInnerBoundary(dir, normals, inter_boundary_face_id, inner_part, outer_part);
    graph::bound_trace.clear();
    graph::FindNumberOfAllInAndDefFaces(dir, normals, faces_state, count_in_face, count_def_face, next_step_el);
    int64_t count = 0;
    int32_t front = 0;
    while (next_step_el.size()) {
      const int ret = graph::FindCurFrontWithHole(dir, normals, inter_faces, next_step_el, count_in_face, inner_part,
                                                  cur_el, count_def_face, outer_part);
      graph::NewStep(neighbours, count_in_face, cur_el, count_def_face, next_step_el);
      for (IntId el : cur_el) lv[el] = front;
      count += (int64_t)cur_el.size();
      front++;
      if ((count != N && next_step_el.size() == 0) || ret != e_completion_success) break;
    }
    if (count != N) bad++;
  }
  return bad;
}

}  // extern "C"
