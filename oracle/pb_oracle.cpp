// CPU oracle of the PB path — test infrastructure only (see pb_oracle.h).
//
// Restatement notes.  The reference's own code (src/pb_class.cpp) fixes the
// markers, edge fractions, charge projection, Dirichlet data and the energy; the
// arithmetic of the bimpp operators it calls (bim3a_rhs, bim3a_laplacian_frac,
// bim3a_reaction_frac, bim3a_reaction, bim3a_dirichlet_bc) lives in bimpp
// (tag NextGenPB-v0.0.01), which is not available.  They are restated as the
// box method the reference's energy code itself evaluates (src/pb_class.cpp:
// 2880, 2896-2898, 2690-2693):
//   * per octant, each of the 12 edges couples its end nodes with conductance
//     wha(eps1, eps2, f) * area_h[axis], wha = 1 / (f/eps1 + (1-f)/eps2),
//     area_h = (h_b h_c / h_a) / 4, f the edge fraction (0.5 off the surface);
//   * the reaction term is mass-lumped: corner c of an octant of volume V gets
//     kappa_c * V/8 * w_c, where w_c = prod over the 3 edges at c of the share
//     of the half-edge at c on c's side of the interface: min(1, 2f) at the
//     edge's first node, min(1, 2(1-f)) at its second (w_c = 1 off the surface);
//   * right-hand sides are V/8 * g_c per corner (bim3a_rhs);
//   * a hanging corner takes the mean of its parents' nodal values and passes
//     its rows and columns to its parents with weight 1/num_parents (A = P^T K P);
//   * Dirichlet nodes (on the 6 faces of the root) get identity rows and are
//     eliminated from the other rows into the right-hand side (same solution as
//     row replacement; keeps A symmetric for CG).
#include "pb_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <parallel/algorithm>
#include <vector>

#include "mc_tri_table.h"

namespace {

const double kPi = 3.14159265358979323846;
// include/pb_class.h:47-54
const double e_0 = 8.85418781762e-12, kb = 1.380649e-23, e_ch = 1.602176634e-19, N_av = 6.022e23, Angs = 1e-10;
const int kRoot = 1 << 19;

// edge2nodes / edge_axis (include/pb_class.h:190-207): the 12 octant edges in
// p8est corner order, x in bit 0
const int E2N[24] = {0, 1, 1, 3, 2, 3, 0, 2, 4, 5, 5, 7, 6, 7, 4, 6, 0, 4, 1, 5, 3, 7, 2, 6};
const int EAX[12] = {0, 1, 0, 1, 0, 1, 0, 1, 2, 2, 2, 2};
// p8est corner of marching-cubes vertex v (src/pb_class.cpp:2579-2581)
const int MC_CORNER[8] = {0, 1, 3, 2, 4, 5, 7, 6};

// Edges whose two end vertices lie on different sides in marching-cubes case k
// (bit v of k: vertex v inside).
int mc_cut_edges(int k) {
  int vertex_of_corner[8];
  for (int v = 0; v < 8; ++v) vertex_of_corner[MC_CORNER[v]] = v;
  int m = 0;
  for (int e = 0; e < 12; ++e)
    if (((k >> vertex_of_corner[E2N[2 * e]]) ^ (k >> vertex_of_corner[E2N[2 * e + 1]])) & 1) m |= 1 << e;
  return m;
}

// The oracle's triangle table (oracle/mc_tri_table.h, from the reference's triTable).
void load_tri_table(signed char tri[256][16]) {
  for (int k = 0; k < 256; ++k)
    for (int j = 0; j < 16; ++j) tri[k][j] = (signed char)oracle_mc::kTriTable[k][j];
}

uint64_t spread3(uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | v << 32) & 0x1f00000000ffffULL;
  v = (v | v << 16) & 0x1f0000ff0000ffULL;
  v = (v | v << 8) & 0x100f00f00f00f00fULL;
  v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
  v = (v | v << 2) & 0x1249249249249249ULL;
  return v;
}
uint64_t morton(uint32_t x, uint32_t y, uint32_t z) { return spread3(x) | spread3(y) << 1 | spread3(z) << 2; }

struct RaySet {
  std::vector<uint64_t> keys;
  std::vector<int64_t> ptr;
  std::vector<double> inters, normals;
  // crossings of ray `key` or n = 0
  int64_t find(uint64_t key, const double** I, const double** N) const {
    auto it = std::lower_bound(keys.begin(), keys.end(), key);
    if (it == keys.end() || *it != key) return 0;
    const int64_t j = it - keys.begin();
    *I = inters.data() + ptr[j];
    *N = normals.data() + 3 * ptr[j];
    return ptr[j + 1] - ptr[j];
  }
};

uint64_t ray_key(int32_t a, int32_t b) { return (uint64_t(uint32_t(a)) << 20) | uint64_t(uint32_t(b)); }

double wha(double eps1, double eps2, double frac) { return 1.0 / (frac / eps1 + (1 - frac) / eps2); }
double phi0(double eps1, double eps2, double phi1, double phi2, double frac) {
  return phi1 + frac * eps2 * (phi2 - phi1) / (eps2 * frac + eps1 * (1 - frac));
}

}  // namespace

struct oracle_state {
  int64_t n_oct = 0, n = 0, nh = 0, na = 0;
  std::vector<int32_t> oct_xyz, oct_nodes, node_xyz, hang_par;
  std::vector<int8_t> level, hang_np;
  std::vector<uint64_t> oct_keys;
  double lo[3], hi[3], len[3], tol;
  RaySet rays[3];
  std::vector<double> pos, q;
  pbgpu_model model;
  double eps_in = 0, eps_out = 0, k2 = 0, k = 0;
  // stage results
  bool have_markers = false, have_density = false, have_system = false, have_phi = false;
  std::vector<double> eps, react, marker, react_cell, frac, rho, vol_patch, rhs, val, phi;
  std::vector<int32_t> border, col;
  std::vector<int64_t> atom_oct, row_ptr;
  std::vector<int8_t> is_border_idx;
  std::vector<int64_t> border_pos;  // octant -> position in border list, -1

  double coord(int a, int32_t i) const {
    const double t = double(i) * 0x1p-19;
    const double p = len[a] * t;
    return lo[a] + p;
  }
  int32_t size_of(int64_t o) const { return 1 << (19 - level[o]); }
  void corner_int(int64_t o, int c, int32_t out[3]) const {
    const int32_t s = size_of(o);
    out[0] = oct_xyz[3 * o] + (c & 1) * s;
    out[1] = oct_xyz[3 * o + 1] + ((c >> 1) & 1) * s;
    out[2] = oct_xyz[3 * o + 2] + ((c >> 2) & 1) * s;
  }
  double corner_coord(int64_t o, int c, int a) const {
    int32_t p[3];
    corner_int(o, c, p);
    return coord(a, p[a]);
  }
  // nodal value at a corner: the node's, or the mean of a hanging node's parents
  double corner_val(const std::vector<double>& v, int32_t node) const {
    if (node < n) return v[node];
    const int64_t h = node - n;
    const int np = hang_np[h];
    double t = 0.0;
    for (int j = 0; j < np; ++j) t += v[hang_par[4 * h + j]] / np;
    return t;
  }
  int parity(int axis, uint64_t key, double x) const {
    const double *I, *N;
    const int64_t m = rays[axis].find(key, &I, &N);
    int i = 0;
    if (m == 0 || x < I[0]) return 0;
    while (i < m && x >= I[i]) ++i;
    return i % 2;
  }
  int parity_stern(int axis, uint64_t key, double x, double stern) const {
    const double *I, *N;
    const int64_t m = rays[axis].find(key, &I, &N);
    int i = 0, sign = 1;
    if (m == 0 || x < (I[0] - stern)) return 0;
    while (i < m && x > (I[i] - stern * sign)) {
      ++i;
      sign *= -1;
    }
    return i % 2;
  }
  // ray along `axis` through corner c of octant o
  uint64_t corner_ray(int64_t o, int c, int axis) const {
    int32_t p[3];
    corner_int(o, c, p);
    const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
    return ray_key(p[t0], p[t1]);
  }
  int64_t find_oct(int32_t x, int32_t y, int32_t z) const {
    const uint64_t key = morton(x, y, z);
    auto it = std::upper_bound(oct_keys.begin(), oct_keys.end(), key);
    return int64_t(it - oct_keys.begin()) - 1;
  }
};

extern "C" {

int oracle_tri_table(int* out) {
  if (!out) return 1;
  for (int k = 0; k < 256; ++k)
    for (int j = 0; j < 16; ++j) out[16 * k + j] = oracle_mc::kTriTable[k][j];
  return 0;
}

oracle_state* oracle_create(const pbgpu_mesh* m, const pbgpu_rays* rays3, int64_t n_atoms, const double* pos,
                            const double* charge, const pbgpu_model* model) {
  if (!m || !rays3 || !model || n_atoms < 0) return nullptr;
  oracle_state* s = new oracle_state();
  s->n_oct = m->n_oct;
  s->n = m->n_nodes;
  s->nh = m->n_hang;
  s->oct_xyz.assign(m->oct_xyz, m->oct_xyz + 3 * m->n_oct);
  s->level.assign(m->oct_level, m->oct_level + m->n_oct);
  s->oct_nodes.assign(m->oct_nodes, m->oct_nodes + 8 * m->n_oct);
  s->node_xyz.assign(m->node_xyz, m->node_xyz + 3 * m->n_nodes);
  if (m->n_hang) {
    s->hang_np.assign(m->hang_np, m->hang_np + m->n_hang);
    s->hang_par.assign(m->hang_par, m->hang_par + 4 * m->n_hang);
  }
  for (int a = 0; a < 3; ++a) {
    s->lo[a] = m->lo[a];
    s->hi[a] = m->hi[a];
    s->len[a] = m->hi[a] - m->lo[a];
  }
  s->tol = m->locate_tol;
  s->oct_keys.resize(s->n_oct);
  for (int64_t o = 0; o < s->n_oct; ++o)
    s->oct_keys[o] = morton(s->oct_xyz[3 * o], s->oct_xyz[3 * o + 1], s->oct_xyz[3 * o + 2]);
  for (int a = 0; a < 3; ++a) {
    const pbgpu_rays& r = rays3[a];
    RaySet& R = s->rays[a];
    R.keys.assign(r.keys, r.keys + r.n_rays);
    R.ptr.assign(r.ptr, r.ptr + r.n_rays + 1);
    const int64_t nc = r.ptr[r.n_rays];
    R.inters.assign(r.inters, r.inters + nc);
    R.normals.assign(r.normals, r.normals + 3 * nc);
  }
  s->na = n_atoms;
  s->pos.assign(pos, pos + 3 * n_atoms);
  s->q.assign(charge, charge + n_atoms);
  s->model = *model;
  const double e_in = model->e_in, e_out = model->e_out, T = model->T, I = model->ionic_strength;
  // src/pb_class.cpp:1800-1806
  s->eps_in = 4.0 * kPi * e_0 * e_in * kb * T * Angs / (e_ch * e_ch);
  s->eps_out = 4.0 * kPi * e_0 * e_out * kb * T * Angs / (e_ch * e_ch);
  const double C_0 = 1.0e3 * N_av * I;
  s->k2 = 2.0 * C_0 * Angs * Angs * e_ch * e_ch / (e_0 * e_out * kb * T);
  s->k = std::sqrt(s->k2);
  return s;
}

void oracle_destroy(oracle_state* s) { delete s; }

// create_markers (src/pb_class.cpp:1793-1941), one process.
int oracle_markers(oracle_state* s) {
  const int64_t n = s->n;
  s->eps.assign(n, s->eps_out);
  s->react.assign(n, s->eps_out * s->k2);
  std::vector<int8_t> inside(n, 0);
  for (int64_t i = 0; i < n; ++i) {
    const int32_t* p = &s->node_xyz[3 * i];
    if (s->parity(2, ray_key(p[0], p[1]), s->coord(2, p[2])) == 1) {
      inside[i] = 1;
      s->eps[i] = s->eps_in;
      s->react[i] = 0.0;
    }
  }
  s->marker.assign(s->n_oct, 0.0);
  s->border.clear();
  s->border_pos.assign(s->n_oct, -1);
  const bool stern = s->model.stern_layer_surf == 1;
  if (stern) s->react_cell.assign(s->n_oct, s->eps_out * s->k2);
  for (int64_t o = 0; o < s->n_oct; ++o) {
    int num_int = 0, num_int_stern = 0, num_hang = 0;
    for (int c = 0; c < 8; ++c) {
      const int32_t nd = s->oct_nodes[8 * o + c];
      if (nd >= s->n) {
        ++num_hang;
        continue;
      }
      if (inside[nd]) {
        ++num_int;
        ++num_int_stern;
      }
      if (stern) {
        const int32_t* p = &s->node_xyz[3 * nd];
        if (s->parity_stern(2, ray_key(p[0], p[1]), s->coord(2, p[2]), s->model.stern_layer) == 1) ++num_int_stern;
      }
    }
    if (num_int == 0)
      s->marker[o] = 1.0;
    else if (num_int < 8 - num_hang) {
      s->marker[o] = 0.5;
      s->border_pos[o] = (int64_t)s->border.size();
      s->border.push_back((int32_t)o);
    }
    if (stern && num_int_stern != 0) s->react_cell[o] = 0.0;
  }
  // cube_fraction_intersection for every border octant (src/pb_class.cpp:2422-2532)
  const int64_t nb = (int64_t)s->border.size();
  s->frac.assign(12 * nb, 0.5);
  for (int64_t b = 0; b < nb; ++b) {
    const int64_t o = s->border[b];
    for (int e = 0; e < 12; ++e) {
      const int axis = EAX[e], i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
      const double x1 = s->corner_coord(o, i1, axis), x2 = s->corner_coord(o, i2, axis);
      const double *I, *N;
      const int64_t m = s->rays[axis].find(s->corner_ray(o, i1, axis), &I, &N);
      for (int64_t t = 0; t < m; ++t)
        if (I[t] >= x1 && I[t] <= x2) s->frac[12 * b + e] = (I[t] - x1) / (x2 - x1);
    }
  }
  s->have_markers = true;
  return PBGPU_OK;
}

static void octant_h(const oracle_state* s, int64_t o, double h[3]) {
  for (int a = 0; a < 3; ++a) h[a] = s->corner_coord(o, 7, a) - s->corner_coord(o, 0, a);
}

// Atom search (src/pb_class.cpp:3633-3729): the octant with
// l - tol < p <= r - tol on every axis.
static int64_t locate_atom(const oracle_state* s, const double* p) {
  int32_t g[3];
  for (int a = 0; a < 3; ++a) {
    double t = (p[a] + s->tol - s->lo[a]) / s->len[a] * double(kRoot);
    if (!(t > -2.0)) t = -2.0;
    if (t > kRoot + 2.0) t = kRoot + 2.0;
    g[a] = (int32_t)std::floor(t);
  }
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int32_t x = g[0] + dx, y = g[1] + dy, z = g[2] + dz;
        if (x < 0 || y < 0 || z < 0 || x >= kRoot || y >= kRoot || z >= kRoot) continue;
        const int64_t o = s->find_oct(x, y, z);
        bool in = true;
        for (int a = 0; a < 3 && in; ++a) {
          const double l = s->corner_coord(o, 0, a), r = s->corner_coord(o, 7, a);
          in = (p[a] > l - s->tol) && (p[a] <= r - s->tol);
        }
        if (in) return o;
      }
  return -1;
}

// trilinear weight of corner c for a point in octant o (src/pb_class.cpp:2018-2021)
static double trilinear_weight(const oracle_state* s, int64_t o, int c, const double* p, double volume) {
  return std::abs((p[0] - s->corner_coord(o, 7 - c, 0)) * (p[1] - s->corner_coord(o, 7 - c, 1)) *
                  (p[2] - s->corner_coord(o, 7 - c, 2))) /
         volume;
}

static double octant_volume(const oracle_state* s, int64_t o) {
  return (s->corner_coord(o, 7, 0) - s->corner_coord(o, 0, 0)) * (s->corner_coord(o, 7, 1) - s->corner_coord(o, 0, 1)) *
         (s->corner_coord(o, 7, 2) - s->corner_coord(o, 0, 2));
}

// create_density_map (src/pb_class.cpp:1944-2050)
int oracle_density(oracle_state* s) {
  const int64_t n = s->n;
  s->vol_patch.assign(n, 0.0);
  for (int64_t o = 0; o < s->n_oct; ++o) {
    double h[3];
    octant_h(s, o, h);
    const double v8 = h[0] * h[1] * h[2] * 0.125;
    for (int c = 0; c < 8; ++c) {
      const int32_t nd = s->oct_nodes[8 * o + c];
      if (nd < n) {
        s->vol_patch[nd] += v8;
      } else {
        const int64_t hh = nd - n;
        const int np = s->hang_np[hh];
        for (int j = 0; j < np; ++j) s->vol_patch[s->hang_par[4 * hh + j]] += v8 / np;
      }
    }
  }
  s->rho.assign(n, 0.0);
  s->atom_oct.assign(s->na, -1);
  for (int64_t a = 0; a < s->na; ++a) {
    const double* p = &s->pos[3 * a];
    const int64_t o = locate_atom(s, p);
    s->atom_oct[a] = o;
    if (o < 0) continue;
    const double volume = octant_volume(s, o);
    for (int c = 0; c < 8; ++c) {
      const double w = trilinear_weight(s, o, c, p, volume);
      const int32_t nd = s->oct_nodes[8 * o + c];
      if (nd < n) {
        s->rho[nd] += s->q[a] * 4.0 * kPi * w / s->vol_patch[nd];
      } else {
        const int64_t hh = nd - n;
        const int np = s->hang_np[hh];
        for (int j = 0; j < np; ++j) {
          const int32_t pj = s->hang_par[4 * hh + j];
          const double denom = np * s->vol_patch[pj];
          s->rho[pj] += s->q[a] * 4.0 * kPi * w / denom;
        }
      }
    }
  }
  s->have_density = true;
  return PBGPU_OK;
}

// Dirichlet value at a boundary node (src/pb_class.cpp:2113-2149, 3531-3571).
static double dirichlet_value(const oracle_state* s, double x, double y, double z) {
  const int bc = s->model.bc_type;
  if (bc == 2) {
    double pot = 0.0;
    for (int64_t a = 0; a < s->na; ++a) {
      const double d = std::hypot(s->pos[3 * a] - x, s->pos[3 * a + 1] - y, s->pos[3 * a + 2] - z);
      pot += s->q[a] * std::exp(-s->k * d) / (d * s->eps_out);
    }
    return pot;
  }
  if (bc == 3) {
    const double rs = 2.0;
    const double pout = s->eps_out * (1.0 + s->k * rs), pin = s->eps_in * rs;
    const double d = std::hypot(x, y, z);
    if (d <= rs) return 1.0 / (pout * rs) + (rs - d) / (pin * d);
    return std::exp(s->k * (rs - d)) / (d * pout);
  }
  return 0.0;
}

struct Trip {
  int64_t row;
  int32_t col;
  double v;
};

// The local box-method matrix K (8x8), right-hand side f and corner expansion
// of octant o (bimpp operators restated as at the top of this file).
struct Local {
  double K[8][8];
  double f[8];
  int32_t g[8][4];
  double gw[8][4];
  int ng[8];
};

static void local_octant(const oracle_state* s, int64_t o, Local& L) {
  const int64_t n = s->n;
  const bool stern = s->model.stern_layer_surf == 1;
  double h[3];
  octant_h(s, o, h);
  const double area_h[3] = {h[1] * h[2] / h[0] * 0.25, h[0] * h[2] / h[1] * 0.25, h[0] * h[1] / h[2] * 0.25};
  const double v8 = h[0] * h[1] * h[2] * 0.125;
  double f[12];
  const int64_t bp = s->border_pos[o];
  for (int e = 0; e < 12; ++e) f[e] = bp >= 0 ? s->frac[12 * bp + e] : 0.5;
  double ec[8], kc[8], rc[8], w[8];
  for (int c = 0; c < 8; ++c) {
    const int32_t nd = s->oct_nodes[8 * o + c];
    ec[c] = s->corner_val(s->eps, nd);
    kc[c] = s->corner_val(s->react, nd);
    rc[c] = s->corner_val(s->rho, nd);
    w[c] = 1.0;
  }
  std::memset(L.K, 0, sizeof(L.K));
  for (int e = 0; e < 12; ++e) {
    const int i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
    const double c = wha(ec[i1], ec[i2], f[e]) * area_h[EAX[e]];
    L.K[i1][i1] += c;
    L.K[i2][i2] += c;
    L.K[i1][i2] -= c;
    L.K[i2][i1] -= c;
    w[i1] *= std::min(1.0, 2.0 * f[e]);
    w[i2] *= std::min(1.0, 2.0 * (1.0 - f[e]));
  }
  for (int c = 0; c < 8; ++c) {
    if (stern)
      L.K[c][c] += s->react_cell[o] * v8;
    else
      L.K[c][c] += kc[c] * v8 * w[c];
    L.f[c] = v8 * rc[c];
  }
  for (int c = 0; c < 8; ++c) {
    const int32_t nd = s->oct_nodes[8 * o + c];
    if (nd < n) {
      L.ng[c] = 1;
      L.g[c][0] = nd;
      L.gw[c][0] = 1.0;
    } else {
      const int64_t hh = nd - n;
      L.ng[c] = s->hang_np[hh];
      for (int j = 0; j < L.ng[c]; ++j) {
        L.g[c][j] = s->hang_par[4 * hh + j];
        L.gw[c][j] = 1.0 / L.ng[c];
      }
    }
  }
}

// Dirichlet nodes: any coordinate on the root boundary; bc_type 0 = none.
static void dirichlet_nodes(const oracle_state* s, std::vector<int8_t>& dir, std::vector<double>& gval) {
  const int64_t n = s->n;
  dir.assign(n, 0);
  gval.assign(n, 0.0);
  if (s->model.bc_type == 0) return;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t* p = &s->node_xyz[3 * i];
    bool onb = false;
    for (int a = 0; a < 3; ++a) onb = onb || p[a] == 0 || p[a] == kRoot;
    if (onb) {
      dir[i] = 1;
      gval[i] = dirichlet_value(s, s->coord(0, p[0]), s->coord(1, p[1]), s->coord(2, p[2]));
    }
  }
}

// Triplet assembly: every octant emits its P^T K P entries in a fixed order
// (diagonal blocks of corners 0..7, then the 12 edges in both directions),
// a stable sort by (row, column) groups them, and equal entries are summed in
// emission order.
static int assemble_triplets(oracle_state* s) {
  const int64_t n = s->n;
  std::vector<Trip> trips;
  trips.reserve(s->n_oct * 40);
  std::vector<double> b(n, 0.0);
  Local L;
  for (int64_t o = 0; o < s->n_oct; ++o) {
    local_octant(s, o, L);
    auto put = [&](int a, int bb) {
      for (int i = 0; i < L.ng[a]; ++i)
        for (int j = 0; j < L.ng[bb]; ++j)
          trips.push_back({L.g[a][i], L.g[bb][j], L.gw[a][i] * L.K[a][bb] * L.gw[bb][j]});
    };
    for (int c = 0; c < 8; ++c) put(c, c);
    for (int e = 0; e < 12; ++e) {
      put(E2N[2 * e], E2N[2 * e + 1]);
      put(E2N[2 * e + 1], E2N[2 * e]);
    }
    for (int c = 0; c < 8; ++c)
      for (int i = 0; i < L.ng[c]; ++i) b[L.g[c][i]] += L.gw[c][i] * L.f[c];
  }
  __gnu_parallel::stable_sort(trips.begin(), trips.end(), [](const Trip& x, const Trip& y) {
    return x.row < y.row || (x.row == y.row && x.col < y.col);
  });
  std::vector<int8_t> dir;
  std::vector<double> gval;
  dirichlet_nodes(s, dir, gval);
  s->row_ptr.assign(n + 1, 0);
  s->col.clear();
  s->val.clear();
  s->rhs = b;
  size_t t = 0;
  for (int64_t r = 0; r < n; ++r) {
    if (dir[r]) {
      while (t < trips.size() && trips[t].row == r) ++t;
      s->col.push_back((int32_t)r);
      s->val.push_back(1.0);
      s->rhs[r] = gval[r];
    } else {
      while (t < trips.size() && trips[t].row == r) {
        const int32_t c = trips[t].col;
        double v = 0.0;
        while (t < trips.size() && trips[t].row == r && trips[t].col == c) v += trips[t++].v;
        if (dir[c])
          s->rhs[r] -= v * gval[c];
        else {
          s->col.push_back(c);
          s->val.push_back(v);
        }
      }
    }
    s->row_ptr[r + 1] = (int64_t)s->col.size();
  }
  s->have_system = true;
  return PBGPU_OK;
}

// Row assembly for large meshes (memory O(nnz)): each row walks its node's
// octant incidences in ascending order and, inside an octant, the same
// emission order as the triplet assembly, so both give identical sums.
static int assemble_rows(oracle_state* s) {
  const int64_t n = s->n, no = s->n_oct;
  // node -> octant incidence lists
  std::vector<int64_t> ptr(n + 1, 0);
  for (int64_t t = 0; t < 8 * no; ++t) {
    const int32_t nd = s->oct_nodes[t];
    if (nd < n)
      ++ptr[nd + 1];
    else
      for (int j = 0; j < s->hang_np[nd - n]; ++j) ++ptr[s->hang_par[4 * (nd - n) + j] + 1];
  }
  for (int64_t i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
  std::vector<int64_t> octs(ptr[n]);
  {
    std::vector<int64_t> cur(ptr.begin(), ptr.end() - 1);
    for (int64_t t = 0; t < 8 * no; ++t) {
      const int32_t nd = s->oct_nodes[t];
      if (nd < n)
        octs[cur[nd]++] = t >> 3;
      else
        for (int j = 0; j < s->hang_np[nd - n]; ++j) octs[cur[s->hang_par[4 * (nd - n) + j]]++] = t >> 3;
    }
  }
  std::vector<int8_t> dir;
  std::vector<double> gval;
  dirichlet_nodes(s, dir, gval);
  const int nt = omp_get_max_threads();
  std::vector<std::vector<int32_t>> tcol(nt);
  std::vector<std::vector<double>> tval(nt);
  std::vector<int64_t> rowlen(n, 0);
  std::vector<double> rhs(n, 0.0);
  const int64_t chunk = (n + nt - 1) / nt;
#pragma omp parallel num_threads(nt)
  {
    const int tid = omp_get_thread_num();
    const int64_t r0 = std::min(n, tid * chunk), r1 = std::min(n, r0 + chunk);
    std::vector<std::pair<int32_t, double>> row;
    Local L;
    for (int64_t r = r0; r < r1; ++r) {
      if (dir[r]) {
        tcol[tid].push_back((int32_t)r);
        tval[tid].push_back(1.0);
        rowlen[r] = 1;
        rhs[r] = gval[r];
        continue;
      }
      row.clear();
      double b = 0.0;
      auto add = [&](int32_t c, double v) {
        auto it = std::lower_bound(row.begin(), row.end(), std::make_pair(c, -1e308),
                                   [](const std::pair<int32_t, double>& x, const std::pair<int32_t, double>& y) {
                                     return x.first < y.first;
                                   });
        if (it != row.end() && it->first == c)
          it->second += v;
        else
          row.insert(it, {c, v});
      };
      // distinct octants of this row, ascending
      int64_t k = ptr[r];
      while (k < ptr[r + 1]) {
        const int64_t o = octs[k];
        while (k < ptr[r + 1] && octs[k] == o) ++k;
        local_octant(s, o, L);
        // row r's weight in each local corner (0 when r is not behind it)
        double wr[8];
        for (int c = 0; c < 8; ++c) {
          wr[c] = 0.0;
          for (int i = 0; i < L.ng[c]; ++i)
            if (L.g[c][i] == r) wr[c] = L.gw[c][i];
        }
        auto put = [&](int a, int bb) {
          if (wr[a] == 0.0) return;
          for (int j = 0; j < L.ng[bb]; ++j) add(L.g[bb][j], wr[a] * L.K[a][bb] * L.gw[bb][j]);
        };
        for (int c = 0; c < 8; ++c) put(c, c);
        for (int e = 0; e < 12; ++e) {
          put(E2N[2 * e], E2N[2 * e + 1]);
          put(E2N[2 * e + 1], E2N[2 * e]);
        }
        for (int c = 0; c < 8; ++c)
          if (wr[c] != 0.0) b += wr[c] * L.f[c];
      }
      int64_t m = 0;
      for (const auto& e : row) {
        if (dir[e.first]) {
          b -= e.second * gval[e.first];
          continue;
        }
        tcol[tid].push_back(e.first);
        tval[tid].push_back(e.second);
        ++m;
      }
      rowlen[r] = m;
      rhs[r] = b;
    }
  }
  s->row_ptr.assign(n + 1, 0);
  for (int64_t r = 0; r < n; ++r) s->row_ptr[r + 1] = s->row_ptr[r] + rowlen[r];
  s->col.clear();
  s->val.clear();
  s->col.reserve(s->row_ptr[n]);
  s->val.reserve(s->row_ptr[n]);
  for (int t = 0; t < nt; ++t) {
    s->col.insert(s->col.end(), tcol[t].begin(), tcol[t].end());
    s->val.insert(s->val.end(), tval[t].begin(), tval[t].end());
  }
  s->rhs = rhs;
  s->have_system = true;
  return PBGPU_OK;
}

// assemple_system_matrix (src/pb_class.cpp:2053-2159) with the bimpp operators
// restated as described at the top of this file.  Meshes above 2M octants use
// the row assembly (same sums, O(nnz) memory).
int oracle_assemble(oracle_state* s) {
  if (!s->have_markers || !s->have_density) return PBGPU_ERR_STATE;
  return s->n_oct > 2000000 ? assemble_rows(s) : assemble_triplets(s);
}

int oracle_assemble_mode(oracle_state* s, int rows) {
  if (!s->have_markers || !s->have_density) return PBGPU_ERR_STATE;
  return rows ? assemble_rows(s) : assemble_triplets(s);
}

static void spmv(const oracle_state* s, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < s->n; ++r) {
    double acc = 0.0;
    for (int64_t k = s->row_ptr[r]; k < s->row_ptr[r + 1]; ++k) acc += s->val[k] * x[s->col[k]];
    y[r] = acc;
  }
}

static double dot(const double* a, const double* b, int64_t n) {
  double t = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : t)
  for (int64_t i = 0; i < n; ++i) t += a[i] * b[i];
  return t;
}

int oracle_spmv(const oracle_state* s, const double* x, double* y, int threads) {
  if (!s->have_system) return PBGPU_ERR_STATE;
  const int prev = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  spmv(s, x, y);
  omp_set_num_threads(prev);
  return PBGPU_OK;
}

static std::vector<double> jacobi_inverse(const oracle_state* s) {
  std::vector<double> d(s->n, 1.0);
  for (int64_t r = 0; r < s->n; ++r)
    for (int64_t k = s->row_ptr[r]; k < s->row_ptr[r + 1]; ++k)
      if (s->col[k] == r) d[r] = 1.0 / s->val[k];
  return d;
}

// The preconditioners of lis_compute_electric_potential's "-p" option as the
// GPU path defines them: none, Jacobi (1 / diag), and block Jacobi over blocks
// of 8 consecutive nodes (node order), each inverted in FP64 by Gauss-Jordan
// elimination and stored symmetrised in FP32.
struct Precond {
  static constexpr int kBlock = 8;
  int kind = PBGPU_PRECOND_JACOBI;
  int64_t n = 0;
  std::vector<double> di;
  std::vector<float> bj;

  Precond(const oracle_state* s, int k) : kind(k), n(s->n) {
    if (kind == PBGPU_PRECOND_NONE) {
      di.assign(n, 1.0);
    } else if (kind == PBGPU_PRECOND_JACOBI) {
      di = jacobi_inverse(s);
    } else {
      const int64_t nb = (n + kBlock - 1) / kBlock;
      bj.assign(nb * kBlock * kBlock, 0.f);
      for (int64_t k0 = 0; k0 < nb * kBlock; k0 += kBlock) {
        double D[kBlock][kBlock] = {}, I[kBlock][kBlock] = {};
        for (int a = 0; a < kBlock; ++a) {
          I[a][a] = 1.0;
          const int64_t r = k0 + a;
          if (r >= n) {
            D[a][a] = 1.0;
            continue;
          }
          for (int64_t q = s->row_ptr[r]; q < s->row_ptr[r + 1]; ++q) {
            const int64_t d = s->col[q] - k0;
            if (d >= 0 && d < kBlock) D[a][d] += s->val[q];
          }
        }
        for (int c = 0; c < kBlock; ++c) {
          const double ip = 1.0 / D[c][c];
          for (int b = 0; b < kBlock; ++b) {
            D[c][b] *= ip;
            I[c][b] *= ip;
          }
          for (int a = 0; a < kBlock; ++a) {
            if (a == c) continue;
            const double f = D[a][c];
            for (int b = 0; b < kBlock; ++b) {
              D[a][b] -= f * D[c][b];
              I[a][b] -= f * I[c][b];
            }
          }
        }
        for (int a = 0; a < kBlock; ++a)
          for (int b = 0; b < kBlock; ++b) bj[(k0 + a) * kBlock + b] = (float)(0.5 * (I[a][b] + I[b][a]));
      }
    }
  }

  // out = M^-1 in
  void apply(const double* in, double* out) const {
    if (kind != PBGPU_PRECOND_BLOCK_JACOBI) {
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < n; ++i) out[i] = di[i] * in[i];
      return;
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      const int64_t k0 = i - i % kBlock;
      double acc = 0.0;
      for (int j = 0; j < kBlock && k0 + j < n; ++j) acc += (double)bj[i * kBlock + j] * in[k0 + j];
      out[i] = acc;
    }
  }
};

static double norm1(const double* a, int64_t n) {
  double t = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : t)
  for (int64_t i = 0; i < n; ++i) t += std::fabs(a[i]);
  return t;
}

int oracle_solve(oracle_state* s, int method, double tol, int max_iter, int threads, double* rel_residual) {
  return oracle_solve_ex(s, method, PBGPU_PRECOND_JACOBI, 0, tol, 1.0, max_iter, threads, rel_residual);
}

int oracle_solve_ex(oracle_state* s, int method, int precond, int conv_cond, double tol, double tol_w, int max_iter,
                    int threads, double* rel_residual) {
  if (!s->have_system) return -PBGPU_ERR_STATE;
  if (precond != PBGPU_PRECOND_NONE && precond != PBGPU_PRECOND_JACOBI && precond != PBGPU_PRECOND_BLOCK_JACOBI)
    return -PBGPU_ERR_ARG;
  if (method != PBGPU_CG && method != PBGPU_BICGSTAB && method != PBGPU_CGS) return -PBGPU_ERR_ARG;
  if (conv_cond < 0 || conv_cond > 2) return -PBGPU_ERR_ARG;
  const int prev = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t n = s->n;
  const Precond M(s, precond);
  std::vector<double> x(n, 0.0), r(s->rhs), z(n), p(n), q(n);
  const double bnorm = std::sqrt(dot(s->rhs.data(), s->rhs.data(), n));
  // LIS conv_cond: 0 / 1 ||r||_2 <= tol ||b||_2 (x0 = 0); 2 ||r||_1 <= tol_w ||b||_1 + tol
  const double lim1 = tol_w * norm1(s->rhs.data(), n) + tol;
  auto converged = [&](const std::vector<double>& res, double rr) {
    return conv_cond == 2 ? norm1(res.data(), n) <= lim1 : std::sqrt(rr) <= tol * bnorm;
  };
  int it = 0;
  if (bnorm == 0.0) {
    s->phi = x;
    s->have_phi = true;
    if (rel_residual) *rel_residual = 0.0;
    omp_set_num_threads(prev);
    return 0;
  }
  if (method == PBGPU_CG) {
    M.apply(r.data(), z.data());
    p = z;
    double rz = dot(r.data(), z.data(), n);
    for (it = 1; it <= max_iter; ++it) {
      spmv(s, p.data(), q.data());
      const double alpha = rz / dot(p.data(), q.data(), n);
      double rr = 0.0;
#pragma omp parallel for reduction(+ : rr)
      for (int64_t i = 0; i < n; ++i) {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
        rr += r[i] * r[i];
      }
      if (converged(r, rr)) break;
      M.apply(r.data(), z.data());
      const double rzn = dot(r.data(), z.data(), n);
      const double beta = rzn / rz;
      rz = rzn;
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
  } else if (method == PBGPU_BICGSTAB) {
    std::vector<double> rh(r), v(n, 0.0), ph(n), sv(n), sh(n), t(n);
    std::fill(p.begin(), p.end(), 0.0);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    for (it = 1; it <= max_iter; ++it) {
      const double rho_n = dot(rh.data(), r.data(), n);
      if (rho_n == 0.0 || !std::isfinite(rho_n)) break;
      const double beta = (rho_n / rho) * (alpha / omega);
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
      M.apply(p.data(), ph.data());
      spmv(s, ph.data(), v.data());
      alpha = rho_n / dot(rh.data(), v.data(), n);
      double ss = 0.0;
#pragma omp parallel for reduction(+ : ss)
      for (int64_t i = 0; i < n; ++i) {
        sv[i] = r[i] - alpha * v[i];
        ss += sv[i] * sv[i];
      }
      if (converged(sv, ss)) {
#pragma omp parallel for
        for (int64_t i = 0; i < n; ++i) x[i] += alpha * ph[i];
        break;
      }
      M.apply(sv.data(), sh.data());
      spmv(s, sh.data(), t.data());
      double ts = 0.0, tt = 0.0;
#pragma omp parallel for reduction(+ : ts, tt)
      for (int64_t i = 0; i < n; ++i) {
        ts += t[i] * sv[i];
        tt += t[i] * t[i];
      }
      omega = ts / tt;
      double rr = 0.0;
#pragma omp parallel for reduction(+ : rr)
      for (int64_t i = 0; i < n; ++i) {
        x[i] += alpha * ph[i] + omega * sh[i];
        r[i] = sv[i] - omega * t[i];
        rr += r[i] * r[i];
      }
      rho = rho_n;
      if (converged(r, rr)) break;
      if (omega == 0.0) break;
    }
  } else {
    // CGS with right preconditioning (the GPU path's k_cgs_* sequence)
    std::vector<double> rh(r), u(n), qc(n, 0.0), v(n), ph(n), w(n), uh(n), t(n);
    std::fill(p.begin(), p.end(), 0.0);
    double rho = dot(rh.data(), r.data(), n), beta = 0.0;
    for (it = 1; it <= max_iter; ++it) {
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i) {
        u[i] = r[i] + beta * qc[i];
        p[i] = u[i] + beta * (qc[i] + beta * p[i]);
      }
      M.apply(p.data(), ph.data());
      spmv(s, ph.data(), v.data());
      const double sigma = dot(rh.data(), v.data(), n);
      if (sigma == 0.0 || !std::isfinite(sigma)) break;
      const double alpha = rho / sigma;
#pragma omp parallel for
      for (int64_t i = 0; i < n; ++i) {
        qc[i] = u[i] - alpha * v[i];
        w[i] = u[i] + qc[i];
      }
      M.apply(w.data(), uh.data());
      spmv(s, uh.data(), t.data());
      double rr = 0.0;
#pragma omp parallel for reduction(+ : rr)
      for (int64_t i = 0; i < n; ++i) {
        x[i] += alpha * uh[i];
        r[i] -= alpha * t[i];
        rr += r[i] * r[i];
      }
      if (converged(r, rr)) break;
      const double rho_n = dot(rh.data(), r.data(), n);
      if (rho_n == 0.0 || !std::isfinite(rho_n)) break;
      beta = rho_n / rho;
      rho = rho_n;
    }
  }
  // true residual
  spmv(s, x.data(), q.data());
  double rr = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const double d = s->rhs[i] - q[i];
    rr += d * d;
  }
  if (rel_residual) *rel_residual = std::sqrt(rr) / bnorm;
  s->phi = x;
  s->have_phi = true;
  omp_set_num_threads(prev);
  return it;
}

double oracle_time_cg_iterations(oracle_state* s, int iters, int threads) {
  if (!s->have_system) return -1.0;
  const int prev = omp_get_max_threads();
  if (threads > 0) omp_set_num_threads(threads);
  const int64_t n = s->n;
  const std::vector<double> Di = jacobi_inverse(s);
  std::vector<double> x(n, 0.0), r(s->rhs), z(n), p(n), q(n);
#pragma omp parallel for
  for (int64_t i = 0; i < n; ++i) p[i] = z[i] = Di[i] * r[i];
  double rz = dot(r.data(), z.data(), n);
  const auto t0 = std::chrono::steady_clock::now();
  for (int it = 0; it < iters; ++it) {
    spmv(s, p.data(), q.data());
    const double alpha = rz / dot(p.data(), q.data(), n);
    double rzn = 0.0;
#pragma omp parallel for reduction(+ : rzn)
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = Di[i] * r[i];
      rzn += r[i] * z[i];
    }
    const double beta = rzn / rz;
    rz = rzn;
#pragma omp parallel for
    for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
  }
  const auto t1 = std::chrono::steady_clock::now();
  omp_set_num_threads(prev);
  return std::chrono::duration<double>(t1 - t0).count();
}

int oracle_set_phi(oracle_state* s, const double* phi) {
  s->phi.assign(phi, phi + s->n);
  s->have_phi = true;
  return PBGPU_OK;
}

int oracle_set_system(oracle_state* s, int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                      const double* rhs) {
  if (n != s->n) return PBGPU_ERR_ARG;
  s->row_ptr.assign(row_ptr, row_ptr + n + 1);
  s->col.assign(col, col + row_ptr[n]);
  s->val.assign(val, val + row_ptr[n]);
  s->rhs.assign(rhs, rhs + n);
  s->have_system = true;
  return PBGPU_OK;
}

// write_potential_on_atoms_fast (src/pb_class.cpp:2333-2417)
int oracle_phi_on_atoms(oracle_state* s, double* out) {
  if (!s->have_phi || !s->have_density) return PBGPU_ERR_STATE;
  for (int64_t a = 0; a < s->na; ++a) {
    const int64_t o = s->atom_oct[a];
    if (o < 0) {
      out[a] = std::numeric_limits<double>::quiet_NaN();
      continue;
    }
    const double* p = &s->pos[3 * a];
    const double volume = octant_volume(s, o);
    double phi = 0.0;
    for (int c = 0; c < 8; ++c) {
      const double w = trilinear_weight(s, o, c, p, volume);
      const int32_t nd = s->oct_nodes[8 * o + c];
      if (nd < s->n)
        phi += s->phi[nd] * w;
      else {
        const int64_t hh = nd - s->n;
        const int np = s->hang_np[hh];
        double ph = 0.0;
        for (int j = 0; j < np; ++j) ph += s->phi[s->hang_par[4 * hh + j]] / np;
        phi += ph * w;
      }
    }
    out[a] = phi;
  }
  return PBGPU_OK;
}

// energy / energy_fast (src/pb_class.cpp:2791-3338).  One deviation, shared with
// the GPU path: the reference keeps the normal N of its last successful
// normal_intersection across octants; here it restarts at (0,0,0) in every
// octant (it matters only for a triangle vertex on an edge without crossing).
int oracle_energy(oracle_state* s, int fast, pbgpu_energy_out* out) {
  if (!s->have_phi || !s->have_markers) return PBGPU_ERR_STATE;
  const double inv_4pi = 1.0 / (4.0 * kPi);
  const double den_in = 1.0 / s->eps_in;
  const double constant_pol = (1.0 / s->eps_out - 1.0 / s->eps_in) * inv_4pi;
  const double constant_react = (1.0 / s->eps_out) * inv_4pi;
  std::vector<double> qa, pa;
  for (int64_t a = 0; a < s->na; ++a)
    if (std::fabs(s->q[a]) > 1.e-5) {
      qa.push_back(s->q[a]);
      pa.insert(pa.end(), &s->pos[3 * a], &s->pos[3 * a] + 3);
    }
  const int64_t m = (int64_t)qa.size();
  double coul = 0.0;
  if (s->model.calc_coulombic == 1) {
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : coul)
    for (int64_t i = 0; i < m; ++i)
      for (int64_t j = i + 1; j < m; ++j) {
        const double dx = pa[3 * i] - pa[3 * j], dy = pa[3 * i + 1] - pa[3 * j + 1], dz = pa[3 * i + 2] - pa[3 * j + 2];
        coul += qa[i] * qa[j] / std::sqrt(dx * dx + dy * dy + dz * dz);
      }
    coul *= den_in;
  }
  const bool ionic = s->model.calc_energy == 2 && s->k > 1.e-5;
  const bool polar = s->model.calc_energy == 1 || (s->model.calc_energy == 2 && s->k < 1.e-5);
  double first_int = 0.0, second_int = 0.0, charge_pol = 0.0;
  signed char tri[256][16];
  load_tri_table(tri);
  const int64_t nb = (int64_t)s->border.size();
  double h0[3] = {0, 0, 0};
  if (fast && nb) octant_h(s, s->border[0], h0);
  if (polar || ionic) {
#pragma omp parallel for schedule(static) reduction(+ : first_int, second_int, charge_pol)
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t o = s->border[b];
      double h[3];
      if (fast)
        for (int a = 0; a < 3; ++a) h[a] = h0[a];
      else
        octant_h(s, o, h);
      const double area_h[3] = {h[1] * h[2] / h[0] * 0.25, h[0] * h[2] / h[1] * 0.25, h[0] * h[1] / h[2] * 0.25};
      double te[8], tp[8];
      for (int c = 0; c < 8; ++c) {
        const int32_t nd = s->oct_nodes[8 * o + c];
        te[c] = s->corner_val(s->eps, nd);
        tp[c] = s->corner_val(s->phi, nd);
      }
      double N[3] = {0, 0, 0};
      auto normal_intersection = [&](int e, double& fract) {
        const int axis = EAX[e], i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
        const double x1 = s->corner_coord(o, i1, axis), x2 = s->corner_coord(o, i2, axis);
        const double *I, *NN;
        const int64_t mr = s->rays[axis].find(s->corner_ray(o, i1, axis), &I, &NN);
        fract = 0.5;
        for (int64_t t = 0; t < mr; ++t)
          if (I[t] >= x1 && I[t] <= x2) {
            N[0] = NN[3 * t];
            N[1] = NN[3 * t + 1];
            N[2] = NN[3 * t + 2];
            fract = (I[t] - x1) / (x2 - x1);
          }
      };
      auto vertex = [&](int e, double fract, double V[3]) {
        const int axis = EAX[e], i1 = E2N[2 * e];
        for (int a = 0; a < 3; ++a) V[a] = s->corner_coord(o, i1, a);
        V[axis] += fract * h[axis];
      };
      for (int e = 0; e < 12; ++e) {
        const int i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
        double dir;
        if (te[i1] < te[i2])
          dir = 1;
        else if (te[i1] > te[i2])
          dir = -1;
        else
          continue;
        double fract;
        normal_intersection(e, fract);
        double V[3];
        vertex(e, fract, V);
        const double tmp_flux = -(tp[i2] - tp[i1]) * wha(te[i1], te[i2], fract) * dir * area_h[EAX[e]];
        charge_pol += tmp_flux;
        double acc = 0.0;
        for (int64_t a = 0; a < m; ++a) {
          const double dx = pa[3 * a] - V[0], dy = pa[3 * a + 1] - V[1], dz = pa[3 * a + 2] - V[2];
          const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
          if (ionic)
            acc += qa[a] * tmp_flux / r;
          else
            acc += qa[a] * (tmp_flux / r);
        }
        first_int += acc;
      }
      if (!ionic) continue;
      int cube = 0;
      for (int v = 0; v < 8; ++v)
        if (te[MC_CORNER[v]] < (s->eps_out - 1e-10)) cube |= 1 << v;
      if (mc_cut_edges(cube) == 0) continue;
      for (int t = 0; tri[cube][3 * t] != -1; ++t) {
        double VT[3][3], NT[3][3], ps[3];
        for (int j = 0; j < 3; ++j) {
          const int e = tri[cube][3 * t + j];
          const int i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
          double fract;
          normal_intersection(e, fract);
          vertex(e, fract, VT[j]);
          for (int a = 0; a < 3; ++a) NT[j][a] = N[a];
          ps[j] = phi0(te[i1], te[i2], tp[i1], tp[i2], fract);
        }
        double ab[3], ac[3];
        for (int a = 0; a < 3; ++a) {
          ab[a] = VT[0][a] - VT[1][a];
          ac[a] = VT[0][a] - VT[2][a];
        }
        const double area = 0.5 * std::hypot(ab[1] * ac[2] - ab[2] * ac[1], ab[0] * ac[2] - ab[2] * ac[0],
                                             ab[1] * ac[0] - ab[0] * ac[1]);
        double acc = 0.0;
        for (int64_t a = 0; a < m; ++a)
          for (int j = 0; j < 3; ++j) {
            const double d0 = VT[j][0] - pa[3 * a], d1 = VT[j][1] - pa[3 * a + 1], d2 = VT[j][2] - pa[3 * a + 2];
            const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
            const double r = std::sqrt(r2);
            const double inv_r3 = 1.0 / (r2 * r);
            const double dt = d0 * NT[j][0] + d1 * NT[j][1] + d2 * NT[j][2];
            acc += qa[a] * ps[j] * dt * inv_r3 * inv_4pi * area / 3.0;
          }
        second_int += acc;
      }
    }
  }
  pbgpu_energy_out e{};
  e.energy_pol = (polar || ionic) ? 0.5 * constant_pol * first_int : 0.0;
  e.energy_react = ionic ? 0.5 * (second_int - first_int * constant_react) : 0.0;
  e.energy_coul = coul;
  e.charge_flux = charge_pol / (4.0 * kPi);
  double net = 0.0;
  for (int64_t a = 0; a < s->na; ++a) net += s->q[a];
  e.net_charge = net;
  e.sum = e.energy_pol + e.energy_react + e.energy_coul;
  *out = e;
  return PBGPU_OK;
}

// pot_field / pot_field_fast (src/pb_class.cpp:3732-5060): the per-atom
// Coulomb, polarisation and ionic potentials and fields.  The surface elements
// are collected in the reference's order (border octants, then each octant's
// flux edges, then its triangles' vertices) and every atom sums over them in
// that order, with the reference's expressions; the Coulomb part is its i < j
// pair loop (:3775-3814).  Same normal deviation as oracle_energy.
int oracle_pot_field(oracle_state* s, int fast, int pt, int ft, double* per_atom, pbgpu_pot_field_out* out) {
  if (!s->have_phi || !s->have_markers) return PBGPU_ERR_STATE;
  if (pt < 0 || pt > 2 || ft < 0 || ft > 2 || !out) return PBGPU_ERR_ARG;
  const double inv_4pi = 1.0 / (4.0 * kPi);
  const double den_in = 1.0 / s->eps_in;
  const double constant_pol = (1.0 / s->eps_out - 1.0 / s->eps_in) * inv_4pi;
  const double constant_react = (1.0 / s->eps_out) * inv_4pi;
  const double k = s->k;
  const int64_t na = s->na;
  const double* pos = s->pos.data();
  const double* q = s->q.data();
  std::vector<double> phi_c(na, 0.0), fcx(na, 0.0), fcy(na, 0.0), fcz(na, 0.0);
  double coul = 0.0;
  for (int64_t i = 0; i < na; ++i)
    for (int64_t j = i + 1; j < na; ++j) {
      const double dx = pos[3 * i] - pos[3 * j], dy = pos[3 * i + 1] - pos[3 * j + 1],
                   dz = pos[3 * i + 2] - pos[3 * j + 2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const double r = std::sqrt(r2);
      const double inv_r3 = 1.0 / (r2 * r);
      coul += (q[i] * q[j]) / r * den_in;
      phi_c[i] += q[j] / r * den_in;
      phi_c[j] += q[i] / r * den_in;
      fcx[i] += dx * inv_r3 * q[j] * den_in;
      fcy[i] += dy * inv_r3 * q[j] * den_in;
      fcz[i] += dz * inv_r3 * q[j] * den_in;
      fcx[j] += -dx * inv_r3 * q[i] * den_in;
      fcy[j] += -dy * inv_r3 * q[i] * den_in;
      fcz[j] += -dz * inv_r3 * q[i] * den_in;
    }
  const bool a1 = (ft == 1 || (ft == 2 && k < 1.e-5)) && pt < 2;
  const bool a2 = !a1 && (pt == 1 || (pt == 2 && k < 1.e-5)) && ft == 0;
  const bool b1 = ft == 2 && k > 1.e-5;
  const bool b2 = !b1 && (pt == 2 && k > 1.e-5) && ft == 0;
  const bool b3 = !b1 && !b2 && (pt == 2 && k > 1.e-5) && ft == 1;
  const bool surface = a1 || a2 || b1 || b2 || b3;
  const bool ionic = b1 || b2 || b3;
  // flux elements (V, F) and triangle vertices (V, N, phi_sup * area / 3 / 4 pi)
  struct Flux {
    double V[3], F;
  };
  struct Vert {
    double V[3], N[3], ps, area;
  };
  std::vector<Flux> flux;
  std::vector<Vert> verts;
  double charge_pol = 0.0;
  signed char tri[256][16];
  load_tri_table(tri);
  const int64_t nb = (int64_t)s->border.size();
  double h0[3] = {0, 0, 0};
  if (fast && nb) octant_h(s, s->border[0], h0);
  if (surface)
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t o = s->border[b];
      double h[3];
      if (fast)
        for (int a = 0; a < 3; ++a) h[a] = h0[a];
      else
        octant_h(s, o, h);
      const double area_h[3] = {h[1] * h[2] / h[0] * 0.25, h[0] * h[2] / h[1] * 0.25, h[0] * h[1] / h[2] * 0.25};
      double te[8], tp[8];
      for (int c = 0; c < 8; ++c) {
        const int32_t nd = s->oct_nodes[8 * o + c];
        te[c] = s->corner_val(s->eps, nd);
        tp[c] = s->corner_val(s->phi, nd);
      }
      double N[3] = {0, 0, 0};
      auto normal_intersection = [&](int e, double& fract) {
        const int axis = EAX[e], i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
        const double x1 = s->corner_coord(o, i1, axis), x2 = s->corner_coord(o, i2, axis);
        const double *I, *NN;
        const int64_t mr = s->rays[axis].find(s->corner_ray(o, i1, axis), &I, &NN);
        fract = 0.5;
        for (int64_t t = 0; t < mr; ++t)
          if (I[t] >= x1 && I[t] <= x2) {
            N[0] = NN[3 * t];
            N[1] = NN[3 * t + 1];
            N[2] = NN[3 * t + 2];
            fract = (I[t] - x1) / (x2 - x1);
          }
      };
      auto vertex = [&](int e, double fract, double V[3]) {
        const int axis = EAX[e], i1 = E2N[2 * e];
        for (int a = 0; a < 3; ++a) V[a] = s->corner_coord(o, i1, a);
        V[axis] += fract * h[axis];
      };
      int cube = 0;
      if (ionic)
        for (int v = 0; v < 8; ++v)
          if (te[MC_CORNER[v]] < (s->eps_out - 1e-10)) cube |= 1 << v;
      for (int e = 0; e < 12; ++e) {
        const int i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
        double dir;
        if (te[i1] < te[i2])
          dir = 1;
        else if (te[i1] > te[i2])
          dir = -1;
        else
          continue;
        double fract;
        normal_intersection(e, fract);
        Flux f;
        vertex(e, fract, f.V);
        f.F = -(tp[i2] - tp[i1]) * wha(te[i1], te[i2], fract) * dir * area_h[EAX[e]];
        charge_pol += f.F;
        flux.push_back(f);
      }
      if (!ionic || mc_cut_edges(cube) == 0) continue;
      for (int t = 0; tri[cube][3 * t] != -1; ++t) {
        Vert T[3];
        for (int j = 0; j < 3; ++j) {
          const int e = tri[cube][3 * t + j];
          const int i1 = E2N[2 * e], i2 = E2N[2 * e + 1];
          double fract;
          normal_intersection(e, fract);
          vertex(e, fract, T[j].V);
          for (int a = 0; a < 3; ++a) T[j].N[a] = N[a];
          T[j].ps = phi0(te[i1], te[i2], tp[i1], tp[i2], fract);
        }
        double ab[3], ac[3];
        for (int a = 0; a < 3; ++a) {
          ab[a] = T[0].V[a] - T[1].V[a];
          ac[a] = T[0].V[a] - T[2].V[a];
        }
        const double area = 0.5 * std::hypot(ab[1] * ac[2] - ab[2] * ac[1], ab[0] * ac[2] - ab[2] * ac[0],
                                             ab[1] * ac[0] - ab[0] * ac[1]);
        for (int j = 0; j < 3; ++j) {
          T[j].area = area;
          verts.push_back(T[j]);
        }
      }
    }
  std::vector<double> pp(na, 0.0), fpx(na, 0.0), fpy(na, 0.0), fpz(na, 0.0);
  std::vector<double> pi(na, 0.0), fix(na, 0.0), fiy(na, 0.0), fiz(na, 0.0);
  std::vector<double> fi_a(na, 0.0), si_a(na, 0.0);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t ia = 0; ia < na; ++ia) {
    const double* ra = &pos[3 * ia];
    double first = 0.0, second = 0.0;
    for (const Flux& f : flux) {
      const double dx = ra[0] - f.V[0], dy = ra[1] - f.V[1], dz = ra[2] - f.V[2];
      const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
      const double inv_r3 = 1.0 / (r * r * r);
      const double qflux = f.F / r;
      first += q[ia] * qflux;
      pp[ia] += qflux * constant_pol;
      fpx[ia] += dx * inv_r3 * f.F * constant_pol;
      fpy[ia] += dy * inv_r3 * f.F * constant_pol;
      fpz[ia] += dz * inv_r3 * f.F * constant_pol;
    }
    for (const Vert& v : verts) {
      const double d0 = v.V[0] - ra[0], d1 = v.V[1] - ra[1], d2 = v.V[2] - ra[2];
      const double r2 = d0 * d0 + d1 * d1 + d2 * d2;
      const double r = std::sqrt(r2);
      const double inv_r3 = 1.0 / (r2 * r);
      const double inv_r5 = inv_r3 / r2;
      const double dot = d0 * v.N[0] + d1 * v.N[1] + d2 * v.N[2];
      const double factor = v.ps * inv_4pi * v.area / 3.0;
      second += q[ia] * v.ps * dot * inv_r3 * inv_4pi * v.area / 3.0;
      pi[ia] += v.ps * dot * inv_r3 * inv_4pi * v.area / 3.0;
      fix[ia] += factor * (-3 * d0 * inv_r5 * dot + v.N[0] * inv_r3);
      fiy[ia] += factor * (-3 * d1 * inv_r5 * dot + v.N[1] * inv_r3);
      fiz[ia] += factor * (-3 * d2 * inv_r5 * dot + v.N[2] * inv_r3);
    }
    fi_a[ia] = first;
    si_a[ia] = second;
  }
  double first_int = 0.0, second_int = 0.0;
  for (int64_t ia = 0; ia < na; ++ia) {
    first_int += fi_a[ia];
    second_int += si_a[ia];
  }
  // print-time correction (:4285-4288) and the written columns (:4281-4375)
  const int kC = (1 << PBGPU_PF_PHI_C) | (7 << PBGPU_PF_EX_C);
  const int kP = 1 << PBGPU_PF_PHI_P, kEP = 7 << PBGPU_PF_EX_P;
  const int kI = 1 << PBGPU_PF_PHI_I, kEI = 7 << PBGPU_PF_EX_I;
  int columns = 0;
  if (b1)
    columns = kC | kP | kEP | kI | kEI;
  else if (b2)
    columns = kC | kP | kI;
  else if (b3)
    columns = kC | kP | kEP | kI;
  else if (a2)
    columns = kC | kP;
  else if (a1)
    columns = kC | kP | kEP;
  if (per_atom)
    for (int64_t i = 0; i < na; ++i) {
      double v[PBGPU_PF_COLUMNS];
      v[PBGPU_PF_PHI_C] = phi_c[i];
      v[PBGPU_PF_EX_C] = fcx[i];
      v[PBGPU_PF_EY_C] = fcy[i];
      v[PBGPU_PF_EZ_C] = fcz[i];
      v[PBGPU_PF_PHI_P] = pp[i];
      v[PBGPU_PF_EX_P] = fpx[i];
      v[PBGPU_PF_EY_P] = fpy[i];
      v[PBGPU_PF_EZ_P] = fpz[i];
      v[PBGPU_PF_PHI_I] = pi[i] - pp[i] / constant_pol * constant_react;
      v[PBGPU_PF_EX_I] = fix[i] - fpx[i] / constant_pol * constant_react;
      v[PBGPU_PF_EY_I] = fiy[i] - fpy[i] / constant_pol * constant_react;
      v[PBGPU_PF_EZ_I] = fiz[i] - fpz[i] / constant_pol * constant_react;
      for (int c = 0; c < PBGPU_PF_COLUMNS; ++c) per_atom[PBGPU_PF_COLUMNS * i + c] = ((columns >> c) & 1) ? v[c] : 0.0;
    }
  pbgpu_pot_field_out o{};
  o.energy_pol = surface ? 0.5 * constant_pol * first_int : 0.0;
  o.energy_react = ionic ? 0.5 * (second_int - first_int * constant_react) : 0.0;
  o.energy_coul = coul;
  o.charge_flux = surface ? charge_pol / (4.0 * kPi) : 0.0;
  o.columns = columns;
  *out = o;
  return PBGPU_OK;
}

int oracle_get_node_coeffs(const oracle_state* s, double* eps, double* react) {
  if (!s->have_markers) return PBGPU_ERR_STATE;
  if (eps) std::copy(s->eps.begin(), s->eps.end(), eps);
  if (react) std::copy(s->react.begin(), s->react.end(), react);
  return PBGPU_OK;
}

int oracle_get_markers(const oracle_state* s, double* marker, int64_t* n_border, int32_t* border) {
  if (!s->have_markers) return PBGPU_ERR_STATE;
  if (marker) std::copy(s->marker.begin(), s->marker.end(), marker);
  if (n_border) *n_border = (int64_t)s->border.size();
  if (border) std::copy(s->border.begin(), s->border.end(), border);
  return PBGPU_OK;
}

int oracle_get_fractions(const oracle_state* s, double* frac) {
  if (!s->have_markers) return PBGPU_ERR_STATE;
  std::copy(s->frac.begin(), s->frac.end(), frac);
  return PBGPU_OK;
}

int oracle_get_density(const oracle_state* s, double* rho, double* vol_patch) {
  if (!s->have_density) return PBGPU_ERR_STATE;
  if (rho) std::copy(s->rho.begin(), s->rho.end(), rho);
  if (vol_patch) std::copy(s->vol_patch.begin(), s->vol_patch.end(), vol_patch);
  return PBGPU_OK;
}

int oracle_get_system(const oracle_state* s, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val, double* rhs) {
  if (!s->have_system) return PBGPU_ERR_STATE;
  if (nnz) *nnz = s->row_ptr[s->n];
  if (row_ptr) std::copy(s->row_ptr.begin(), s->row_ptr.end(), row_ptr);
  if (col) std::copy(s->col.begin(), s->col.end(), col);
  if (val) std::copy(s->val.begin(), s->val.end(), val);
  if (rhs) std::copy(s->rhs.begin(), s->rhs.end(), rhs);
  return PBGPU_OK;
}

int oracle_get_phi(const oracle_state* s, double* phi) {
  if (!s->have_phi) return PBGPU_ERR_STATE;
  std::copy(s->phi.begin(), s->phi.end(), phi);
  return PBGPU_OK;
}

}  // extern "C"
