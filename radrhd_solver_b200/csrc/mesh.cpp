// Synthetic Kuhn tetrahedral meshes, Fibonacci direction sets, error strings.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "rng.h"
#include "rrhd_internal.h"
#include "rrhd_mesh.h"

static thread_local std::string g_last_error;

rrhd_status rrhd_fail(rrhd_status st, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return st;
}

extern "C" const char *rrhd_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *rrhd_version(void) { return "rrhd-b200 0.1 (sm_100a)"; }

extern "C" double rrhd_rng_u01(uint64_t seed, uint64_t stream, uint64_t index) {
  return rrhd_u01(seed, stream, index);
}

namespace {

struct Kuhn {
  int nx, ny, nz;
  int64_t vid(int i, int j, int k) const { return ((int64_t)k * (ny + 1) + j) * (nx + 1) + i; }
};

// The 6 Kuhn tetrahedra of a unit hex: for an axis permutation (a, b, c) the
// tet is v000, v000+e_a, v000+e_a+e_b, v111.
const int kPerm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};

inline void sub3(const double *a, const double *b, double *r) {
  r[0] = a[0] - b[0];
  r[1] = a[1] - b[1];
  r[2] = a[2] - b[2];
}
inline void cross3(const double *a, const double *b, double *r) {
  r[0] = a[1] * b[2] - a[2] * b[1];
  r[1] = a[2] * b[0] - a[0] * b[2];
  r[2] = a[0] * b[1] - a[1] * b[0];
}
inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

}  // namespace

extern "C" rrhd_status rrhd_mesh_kuhn_sizes(const rrhd_kuhn_params *p, int64_t *n_cells,
                                            int64_t *n_faces, int64_t *n_vertices) {
  RRHD_CHECK_ARG(p && p->nx > 0 && p->ny > 0 && p->nz > 0, "bad Kuhn mesh size");
  const int64_t nx = p->nx, ny = p->ny, nz = p->nz;
  RRHD_CHECK_ARG((nx + 1) < (1 << 21) && (ny + 1) < (1 << 21) && (nz + 1) < (1 << 21) &&
                     (nx + 1) * (ny + 1) * (nz + 1) < (int64_t(1) << 21),
                 "Kuhn mesh too large for the face hash (more than 2^21 vertices)");
  const int64_t N = 6 * nx * ny * nz;
  const int64_t nb = 4 * (nx * ny + ny * nz + nx * nz);  // boundary triangles
  if (n_cells) *n_cells = N;
  if (n_faces) *n_faces = (4 * N + nb) / 2;
  if (n_vertices) *n_vertices = (nx + 1) * (ny + 1) * (nz + 1);
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_mesh_kuhn_build(const rrhd_kuhn_params *p, int32_t *face_id_l,
                                            int32_t *face_id_r, double *face_n, double *face_area,
                                            int32_t *cell_faces, uint8_t *cell_sign,
                                            double *cell_volume, double *cell_center,
                                            double *h_min, double *vertices_out,
                                            int32_t *cell_vertices_out) {
  int64_t N, F, V;
  rrhd_status st = rrhd_mesh_kuhn_sizes(p, &N, &F, &V);
  if (st) return st;
  RRHD_CHECK_ARG(face_id_l && face_id_r && face_n && face_area && cell_faces && cell_sign &&
                     cell_volume && cell_center,
                 "null output array");
  const Kuhn K{p->nx, p->ny, p->nz};
  double h[3];
  for (int a = 0; a < 3; a++) h[a] = (p->hi[a] - p->lo[a]) / (a == 0 ? p->nx : a == 1 ? p->ny : p->nz);
  const int nmax[3] = {p->nx, p->ny, p->nz};

  // vertices: boundary vertices move only tangentially (stay on their planes)
  std::vector<double> vx((size_t)V * 3);
  for (int k = 0; k <= p->nz; k++)
    for (int j = 0; j <= p->ny; j++)
      for (int i = 0; i <= p->nx; i++) {
        const int64_t v = K.vid(i, j, k);
        const int idx[3] = {i, j, k};
        for (int a = 0; a < 3; a++) {
          double x = p->lo[a] + idx[a] * h[a];
          if (idx[a] > 0 && idx[a] < nmax[a] && p->jitter != 0.0) {
            const double u = rrhd_u01(p->seed, 1 + a, (uint64_t)v);
            x += (2.0 * u - 1.0) * p->jitter * h[a];
          }
          vx[3 * v + a] = x;
        }
      }

  // cells: hex order k, j, i (i fastest), 6 tets per hex
  std::vector<int32_t> tv((size_t)N * 4);
  std::vector<double> inc_n((size_t)N * 12), inc_S((size_t)N * 4);
  double hmin = 1e300;
  for (int k = 0; k < p->nz; k++)
    for (int j = 0; j < p->ny; j++)
      for (int i = 0; i < p->nx; i++) {
        const int64_t hex = ((int64_t)k * p->ny + j) * p->nx + i;
        for (int t = 0; t < 6; t++) {
          const int64_t c = 6 * hex + t;
          int o[3] = {i, j, k};
          int32_t q[4];
          q[0] = (int32_t)K.vid(o[0], o[1], o[2]);
          o[kPerm[t][0]]++;
          q[1] = (int32_t)K.vid(o[0], o[1], o[2]);
          o[kPerm[t][1]]++;
          q[2] = (int32_t)K.vid(o[0], o[1], o[2]);
          q[3] = (int32_t)K.vid(i + 1, j + 1, k + 1);
          for (int a = 0; a < 4; a++) tv[4 * c + a] = q[a];
          const double *P[4] = {&vx[3 * q[0]], &vx[3 * q[1]], &vx[3 * q[2]], &vx[3 * q[3]]};
          double e1[3], e2[3], e3[3], cr[3];
          sub3(P[1], P[0], e1);
          sub3(P[2], P[0], e2);
          sub3(P[3], P[0], e3);
          cross3(e1, e2, cr);
          const double vol = std::fabs(dot3(cr, e3)) / 6.0;
          cell_volume[c] = vol;
          for (int a = 0; a < 3; a++)
            cell_center[3 * c + a] = (P[0][a] + P[1][a] + P[2][a] + P[3][a]) / 4.0;
          double smax = 0;
          // local face j is opposite vertex j
          for (int fj = 0; fj < 4; fj++) {
            const double *A = P[(fj + 1) & 3], *B = P[(fj + 2) & 3], *C = P[(fj + 3) & 3];
            double ab[3], ac[3], n[3], ad[3];
            sub3(B, A, ab);
            sub3(C, A, ac);
            cross3(ab, ac, n);
            const double len = std::sqrt(dot3(n, n));
            const double S = 0.5 * len;
            for (int a = 0; a < 3; a++) n[a] /= len;
            sub3(P[fj], A, ad);
            if (dot3(n, ad) > 0)
              for (int a = 0; a < 3; a++) n[a] = -n[a];
            for (int a = 0; a < 3; a++) inc_n[12 * c + 3 * fj + a] = n[a];
            inc_S[4 * c + fj] = S;
            smax = std::max(smax, S);
          }
          hmin = std::min(hmin, 3.0 * vol / smax);
        }
      }

  // match incidences by their sorted vertex triple
  std::vector<std::pair<uint64_t, int64_t>> keys((size_t)N * 4);
  for (int64_t c = 0; c < N; c++)
    for (int fj = 0; fj < 4; fj++) {
      uint64_t a = tv[4 * c + ((fj + 1) & 3)], b = tv[4 * c + ((fj + 2) & 3)],
               d = tv[4 * c + ((fj + 3) & 3)];
      if (a > b) std::swap(a, b);
      if (b > d) std::swap(b, d);
      if (a > b) std::swap(a, b);
      keys[4 * c + fj] = {(a << 42) | (b << 21) | d, 4 * c + fj};
    }
  std::sort(keys.begin(), keys.end());
  std::vector<int64_t> partner((size_t)N * 4, -1);
  for (size_t s = 0; s + 1 < keys.size(); s++)
    if (keys[s].first == keys[s + 1].first) {
      partner[keys[s].second] = keys[s + 1].second;
      partner[keys[s + 1].second] = keys[s].second;
      s++;
    }
  keys.clear();
  keys.shrink_to_fit();

  // boundary code of an unmatched incidence: plane of its three vertices
  auto plane_code = [&](int64_t inc) -> int32_t {
    const int64_t c = inc / 4;
    const int fj = (int)(inc % 4);
    int64_t q[3] = {tv[4 * c + ((fj + 1) & 3)], tv[4 * c + ((fj + 2) & 3)], tv[4 * c + ((fj + 3) & 3)]};
    int g[3][3];
    for (int a = 0; a < 3; a++) {
      int64_t v = q[a];
      g[a][0] = (int)(v % (p->nx + 1));
      v /= (p->nx + 1);
      g[a][1] = (int)(v % (p->ny + 1));
      g[a][2] = (int)(v / (p->ny + 1));
    }
    int plane = -1;
    for (int ax = 0; ax < 3 && plane < 0; ax++) {
      if (g[0][ax] == 0 && g[1][ax] == 0 && g[2][ax] == 0) plane = 2 * ax;
      else if (g[0][ax] == nmax[ax] && g[1][ax] == nmax[ax] && g[2][ax] == nmax[ax]) plane = 2 * ax + 1;
    }
    int32_t code = (plane >= 0 && p->bc_code[plane] != 0) ? p->bc_code[plane] : -1;
    if (plane == 4 && p->inflow_radius > 0) {
      const double cx = 0.5 * (p->lo[0] + p->hi[0]), cy = 0.5 * (p->lo[1] + p->hi[1]);
      double x = 0, y = 0;
      for (int a = 0; a < 3; a++) {
        x += vx[3 * q[a]] / 3.0;
        y += vx[3 * q[a] + 1] / 3.0;
      }
      if ((x - cx) * (x - cx) + (y - cy) * (y - cy) < p->inflow_radius * p->inflow_radius)
        code = p->inflow_code;
    }
    return code;
  };

  // face assembly in ConvertBinToGeo order
  std::vector<char> done((size_t)N * 4, 0);
  int64_t cc = 0;
  for (int64_t inc = 0; inc < 4 * N; inc++) {
    if (done[inc]) continue;
    const int64_t c = inc / 4;
    const int fj = (int)(inc % 4);
    face_id_l[cc] = (int32_t)c;
    for (int a = 0; a < 3; a++) face_n[3 * cc + a] = inc_n[3 * inc + a];
    face_area[cc] = inc_S[inc];
    cell_sign[c] = (uint8_t)(cell_sign[c] | (1u << fj));
    cell_faces[4 * c + fj] = (int32_t)cc;
    done[inc] = 1;
    const int64_t o = partner[inc];
    if (o >= 0) {
      face_id_r[cc] = (int32_t)(o / 4);
      cell_sign[o / 4] = (uint8_t)(cell_sign[o / 4] & ~(1u << (o % 4)));
      cell_faces[o] = (int32_t)cc;
      done[o] = 1;
    } else {
      face_id_r[cc] = plane_code(inc);
    }
    cc++;
  }
  if (cc != F) return rrhd_fail(RRHD_ERR_STATE, "face count %lld != expected %lld", (long long)cc, (long long)F);
  if (h_min) *h_min = hmin;
  if (vertices_out) std::memcpy(vertices_out, vx.data(), sizeof(double) * 3 * V);
  if (cell_vertices_out) std::memcpy(cell_vertices_out, tv.data(), sizeof(int32_t) * 4 * N);
  return RRHD_OK;
}

extern "C" rrhd_status rrhd_directions_fibonacci(int32_t M, double *dirs, double *areas,
                                                 double *full_area) {
  RRHD_CHECK_ARG(M > 0 && dirs && areas && full_area, "bad direction-set arguments");
  const double pi = 3.14159265358979323846;
  const double ga = pi * (3.0 - std::sqrt(5.0));
  for (int k = 0; k < M; k++) {
    const double z = 1.0 - (2.0 * k + 1.0) / M;
    const double r = std::sqrt(std::max(0.0, 1.0 - z * z));
    const double ph = ga * k;
    dirs[3 * k + 0] = r * std::cos(ph);
    dirs[3 * k + 1] = r * std::sin(ph);
    dirs[3 * k + 2] = z;
    areas[k] = 4.0 * pi / M;
  }
  *full_area = 4.0 * pi;
  return RRHD_OK;
}
