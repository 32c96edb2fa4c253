// Host-side poisson_boltzmann: configuration, atoms, domain box, octree
// refinement, surface rays, and the GPU path through the pbgpu C ABI.
#include "pb_class.h"
#include "vtu.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <numeric>
#include <parallel/algorithm>
#include <random>
#include <sstream>
#include <stdexcept>

namespace pbh {

// 1 / 2^P8EST_QMAXLEVEL (include/pb_class.h:29)
static const double p4esttol = 1.0 / std::pow(2.0, kQMaxLevel);

poisson_boltzmann::~poisson_boltzmann() {
  if (gpu && own_gpu) pbgpu_ctx_destroy(gpu);
}

// ---------------------------------------------------------------------------
// Options: keys and defaults of src/pb_class.cpp:852-975.
void poisson_boltzmann::apply_options(const OptionFile& g) {
  filetype = g.get("input/filetype", std::string("pqr"));
  pqrfilename = g.get("input/filename", std::string("../../data/1CCM.pqr"));
  const std::string m = "mesh/";
  maxlevel = g.get(m + "maxlevel", 9);
  minlevel = g.get(m + "minlevel", 3);
  unilevel = g.get(m + "unilevel", 5);
  outlevel = g.get(m + "outlevel", 1);
  loc_refinement = g.get(m + "loc_refinement", 0);
  mesh_shape = g.get(m + "mesh_shape", 1);
  refine_box = g.get(m + "refine_box", 0);
  rand_center = g.get(m + "rand_center", 0);
  aligned = g.get(m + "aligned", 0);
  if (mesh_shape < 2 || mesh_shape == 3 || mesh_shape == 4) {
    perfil1 = g.get(m + "perfil1", 0.8);
    perfil2 = g.get(m + "perfil2", 0.2);
  }
  if (mesh_shape < 2 || mesh_shape == 3) scale = g.get(m + "scale", 2.0);
  if (mesh_shape == 2) {
    l_c[0] = g.get(m + "x1", -128.0);
    r_c[0] = g.get(m + "x2", 128.0);
    l_c[1] = g.get(m + "y1", -128.0);
    r_c[1] = g.get(m + "y2", 128.0);
    l_c[2] = g.get(m + "z1", -128.0);
    r_c[2] = g.get(m + "z2", 128.0);
    l_cr[0] = g.get(m + "refine_x1", -64.0);
    r_cr[0] = g.get(m + "refine_x2", 64.0);
    l_cr[1] = g.get(m + "refine_y1", -64.0);
    r_cr[1] = g.get(m + "refine_y2", 64.0);
    l_cr[2] = g.get(m + "refine_z1", -64.0);
    r_cr[2] = g.get(m + "refine_z2", 64.0);
  }
  if (mesh_shape == 3) {
    cc_focusing[0] = g.get(m + "cx_foc", 0.0);
    cc_focusing[1] = g.get(m + "cy_foc", 0.0);
    cc_focusing[2] = g.get(m + "cz_foc", 0.0);
    n_grid = g.get(m + "n_grid", 8);
  }
  if (mesh_shape == 4) {
    scale_min = g.get(m + "scale_min", 0.5);
    scale_max = g.get(m + "scale_max", 2.0);
  }
  if (mesh_shape == 5) {
    len = g.get(m + "lato", 50.0);
    perfil1 = g.get(m + "perfil1", 0.8);
  }
  const std::string md = "model/";
  linearized = g.get(md + "linearized", 1);
  bc = g.get(md + "bc_type", 1);
  ionic_strength = g.get(md + "ionic_strength", 0.145);
  e_in = g.get(md + "molecular_dielectric_constant", 2.0);
  e_out = g.get(md + "solvent_dielectric_constant", 80.0);
  T = g.get(md + "T", 298.15);
  calc_energy = g.get(md + "calc_energy", 2);
  calc_coulombic = g.get(md + "calc_coulombic", 0);
  calc_potential_term = g.get(md + "calc_potential_terms", 0);
  calc_field_term = g.get(md + "calc_field_terms", 0);
  map_type = g.get(md + "map_type", std::string("vtu"));
  potential_map = g.get(md + "potential_map", 0);
  eps_map = g.get(md + "eps_map", 0);
  atoms_write = g.get(md + "atoms_write", 0);
  const std::string s = "surface/";
  surf_type_num = g.get(s + "surface_type", 0);
  surf_param = g.get(s + "surface_parameter", 0.45);
  stern_layer_surf = g.get(s + "stern_layer_surf", 0);
  stern_layer = g.get(s + "stern_layer_thickness", 2.0);
  const std::string a = "algorithm/";
  linear_solver_name = g.get(a + "linear_solver", std::string("lis"));
  linear_solver_options = g.get(a + "solver_options",
                                std::string("-p ssor -ssor_omega 0.51 -i cgs -tol 1.e-6 -print 2 -conv_cond 2 -tol_w 0"));
}

int poisson_boltzmann::parse_options(int argc, char** argv) {
  std::string prm, pqr;
  for (int i = 1; i + 1 < argc; ++i) {
    const std::string k = argv[i];
    if ((k == "--prmfile" || k == "--potfile") && prm.empty()) prm = argv[i + 1];
    if (k == "--pqrfile") pqr = argv[i + 1];
  }
  optionsfilename = prm.empty() ? "../../data/options.prm" : prm;
  OptionFile g;
  if (!g.load_file(optionsfilename)) {
    std::cerr << "Cannot find the options file" << std::endl;
    return 1;
  }
  apply_options(g);
  if (!pqr.empty()) {
    pqrfilename = pqr;
    filetype = "pqr";
  }
  std::ifstream f(pqrfilename);
  if (!f) {
    std::cerr << "Cannot find the pqr file" << std::endl;
    return 1;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// PQR atoms (src/pb_class.cpp:1223-1261): whitespace-separated tokens, optional
// chain identifier, radius < 1e-5 replaced by 1.0; reading stops at the first
// record that does not parse.
static bool read_atom(std::istream& in, Atom& a) {
  std::string field, name, res, token;
  long num;
  if (!(in >> field >> num >> name >> res)) return false;
  if (!(in >> token)) return false;
  const bool is_number = !token.empty() && (std::isdigit((unsigned char)token[0]) || token[0] == '-' || token[0] == '+');
  long resnum;
  if (is_number) {
    std::istringstream t(token);
    if (!(t >> resnum)) return false;
  } else if (!(in >> resnum)) {
    return false;
  }
  if (!(in >> a.pos[0] >> a.pos[1] >> a.pos[2] >> a.charge >> a.radius)) return false;
  if (a.radius < 1.e-5) a.radius = 1.0;
  return true;
}

// Principal-axis alignment applied when [mesh] aligned = 1
// (align_atoms_to_Z, src/pb_class.cpp:1007-1096): centre the atoms, take the
// dominant eigenvector of their second-moment matrix by 20 power iterations,
// and rotate it onto +z with Rodrigues' formula.
static void align_atoms_to_z(std::vector<Atom>& atoms) {
  if (atoms.empty()) return;
  double c[3] = {0, 0, 0};
  for (const Atom& a : atoms)
    for (int k = 0; k < 3; ++k) c[k] += a.pos[k];
  for (int k = 0; k < 3; ++k) c[k] /= double(atoms.size());
  for (Atom& a : atoms)
    for (int k = 0; k < 3; ++k) a.pos[k] -= c[k];
  double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (const Atom& a : atoms)
    for (int i = 0; i < 3; ++i)
      for (int j = i; j < 3; ++j) M[i][j] += a.pos[i] * a.pos[j];
  M[1][0] = M[0][1];
  M[2][0] = M[0][2];
  M[2][1] = M[1][2];
  double v[3] = {1, 0, 0};
  for (int it = 0; it < 20; ++it) {
    double w[3];
    for (int i = 0; i < 3; ++i) w[i] = M[i][0] * v[0] + M[i][1] * v[1] + M[i][2] * v[2];
    const double nrm = std::sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
    if (nrm < 1e-12) break;
    for (int i = 0; i < 3; ++i) v[i] = w[i] / nrm;
  }
  const double vn = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (vn > 1e-12)
    for (double& x : v) x /= vn;
  // axis x (0,0,1)
  const double ax[3] = {v[1], -v[0], 0.0};
  const double s = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
  const double cth = v[2];
  double R[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  if (s >= 1e-8) {
    const double kx = ax[0] / s, ky = ax[1] / s, kz = ax[2] / s, t = 1.0 - cth;
    R[0][0] = cth + kx * kx * t;
    R[0][1] = kx * ky * t - kz * s;
    R[0][2] = kx * kz * t + ky * s;
    R[1][0] = ky * kx * t + kz * s;
    R[1][1] = cth + ky * ky * t;
    R[1][2] = ky * kz * t - kx * s;
    R[2][0] = kz * kx * t - ky * s;
    R[2][1] = kz * ky * t + kx * s;
    R[2][2] = cth + kz * kz * t;
  }
  for (Atom& a : atoms) {
    const double x = a.pos[0], y = a.pos[1], z = a.pos[2];
    for (int i = 0; i < 3; ++i) a.pos[i] = R[i][0] * x + R[i][1] * y + R[i][2] * z;
  }
}

void poisson_boltzmann::read_atoms_from_pqr(std::istream& in) {
  atoms.clear();
  Atom a{};
  while (read_atom(in, a)) atoms.push_back(a);
  if (aligned == 1) align_atoms_to_z(atoms);
  // Fewer than 4 atoms: 6 neutral, zero-radius dummies at +-0.001 A around the
  // largest atom (src/pb_class.cpp:1111-1149).
  if (!atoms.empty() && atoms.size() < 4) {
    auto it = std::max_element(atoms.begin(), atoms.end(),
                               [](const Atom& x, const Atom& y) { return x.radius < y.radius; });
    const double p[3] = {it->pos[0], it->pos[1], it->pos[2]};
    const int dirs[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int d = 0; d < 6; ++d) {
      Atom dm{};
      for (int k = 0; k < 3; ++k) dm.pos[k] = p[k] + 0.001 * dirs[d][k];
      dm.charge = 0.0;
      dm.radius = 0.0;
      atoms.push_back(dm);
    }
  }
}

void poisson_boltzmann::read_atoms_from_class() {
  pos_atoms.clear();
  charge_atoms.clear();
  r_atoms.clear();
  index_atoms.clear();
  int num = 1;
  for (const Atom& a : atoms) {
    pos_atoms.push_back({a.pos[0], a.pos[1], a.pos[2]});
    charge_atoms.push_back(a.charge);
    r_atoms.push_back(a.radius);
    index_atoms.push_back(num++);
  }
}

// ---------------------------------------------------------------------------
// Domain box (create_mesh, src/pb_class.cpp:39-743).  mesh_shape 5 (a forest of
// several trees) is not supported by this single-tree octree.
void poisson_boltzmann::create_mesh() {
  if (pos_atoms.empty()) throw std::runtime_error("create_mesh: no atoms");
  const double eps_out = 4.0 * pi * e_0 * e_out * kb * T * Angs / (e_charge * e_charge);
  const double C_0 = 1.0e3 * N_av * ionic_strength;
  const double k2 = 2.0 * C_0 * Angs * Angs * e_charge * e_charge / (e_0 * e_out * kb * T);
  const double k = std::sqrt(k2);
  double lmax = 0, l[3];
  scale_level = unilevel;
  const double maxradius = *std::max_element(r_atoms.begin(), r_atoms.end());
  double mn[3], mx[3];
  for (int a = 0; a < 3; ++a) {
    mn[a] = 1e300;
    mx[a] = -1e300;
    for (const auto& p : pos_atoms) {
      mn[a] = std::min(mn[a], p[a]);
      mx[a] = std::max(mx[a], p[a]);
    }
  }
  net_charge = std::accumulate(charge_atoms.begin(), charge_atoms.end(), 0.0);
  if (verbose) {
    std::cout << "  Number of atoms    : " << charge_atoms.size() << "\n";
    if (std::fabs(net_charge - std::round(net_charge)) > 1.e-5)
      std::cerr << "  [WARNING] Net charge is not an integer: " << net_charge << '\n';
  }
  if (mesh_shape != 2) {
    for (int a = 0; a < 3; ++a) {
      l_c[a] = mn[a] - maxradius - 2 * prb_radius;
      r_c[a] = mx[a] + maxradius + 2 * prb_radius;
    }
    for (int a = 0; a < 3; ++a) {
      l[a] = r_c[a] - l_c[a];
      cc[a] = (r_c[a] + l_c[a]) * 0.5;
      lmax = l[a] > lmax ? l[a] : lmax;
    }
    if (rand_center == 1) {
      std::random_device rd;
      std::mt19937 gen(rd());
      std::uniform_real_distribution<> dis(-1. / scale * 0.5, 1. / scale * 0.5);
      for (int a = 0; a < 3; ++a) cc[a] = cc[a] + dis(gen);
    }
    for (int a = 0; a < 3; ++a) {
      ll[a] = cc[a] - lmax * 0.5;
      rr[a] = cc[a] + lmax * 0.5;
    }
    for (int a = 0; a < 3; ++a) {
      l_c[a] -= l[a] * 0.5 * (1.0 / perfil1 - 1);
      r_c[a] += l[a] * 0.5 * (1.0 / perfil1 - 1);
    }
    for (int a = 0; a < 3; ++a) {
      ll[a] -= lmax * 0.5 * (1.0 / perfil1 - 1);
      rr[a] += lmax * 0.5 * (1.0 / perfil1 - 1);
    }
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = l_c[a];
      r_cr[a] = r_c[a];
    }
  }
  if (mesh_shape == 0) {
    double size = 1.0 / scale;
    scale_level = 0;
    for (int ii = 0; ii < 29; ++ii) {
      size *= 2;
      scale_level++;
      if (lmax / size < perfil2) break;
    }
    for (int a = 0; a < 3; ++a) {
      ll[a] = cc[a] - size / 2;
      rr[a] = cc[a] + size / 2;
    }
    int nn[3];
    for (int a = 0; a < 3; ++a) nn[a] = (int)((r_cr[a] - cc[a]) * scale + 0.5);
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = cc[a] - nn[a] * 1.0 / scale;
      r_cr[a] = cc[a] + nn[a] * 1.0 / scale;
    }
    const double dist = size / 2 - lmax * 0.5;
    pot_bc = std::exp(-k * dist) / (dist * eps_out);
  } else if (mesh_shape == 1) {
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = ll[a];
      r_cr[a] = rr[a];
    }
    scale = (1 << unilevel) / (rr[0] - ll[0]);
    if (refine_box == 1) {
      for (int a = 0; a < 3; ++a) {
        ll[a] = cc[a] - lmax * 0.5 * 1.0 / perfil2;
        rr[a] = cc[a] + lmax * 0.5 * 1.0 / perfil2;
      }
      const double scale_tmp = (1 << unilevel) / (rr[0] - ll[0]);
      int nn[3];
      for (int a = 0; a < 3; ++a) nn[a] = (int)((r_cr[a] - cc[a]) * scale_tmp + 0.5);
      for (int a = 0; a < 3; ++a) {
        l_cr[a] = cc[a] - nn[a] * 1.0 / scale_tmp;
        r_cr[a] = cc[a] + nn[a] * 1.0 / scale_tmp;
      }
    }
    const double dist = ((rr[0] - ll[0]) - lmax) * 0.5;
    pot_bc = std::exp(-k * dist) / (dist * eps_out);
  } else if (mesh_shape == 2) {
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = l_c[a];
      r_cr[a] = r_c[a];
    }
    scale = (1 << unilevel) / (r_c[0] - l_c[0]);
    const double dist = ((r_cr[0] - l_cr[0]) - lmax) * 0.5;
    pot_bc = std::exp(-k * dist) / (dist * eps_out);
  } else if (mesh_shape == 3) {
    double size = 1.0 / scale;
    const double scale_min_box = 0.5;
    scale_level = 0;
    scale_level_min_box = 0;
    for (int ii = 0; ii < 28; ++ii) {
      size *= 2;
      scale_level++;
      if (lmax / size < perfil2) break;
    }
    for (int ii = 0; ii < scale_level; ++ii) {
      scale_level_min_box++;
      if ((std::pow(2, scale_level_min_box) + 1) / size >= scale_min_box) break;
    }
    for (int a = 0; a < 3; ++a) {
      ll[a] = cc[a] - size / 2;
      rr[a] = cc[a] + size / 2;
    }
    int nn[3];
    for (int a = 0; a < 3; ++a) nn[a] = (int)((r_cr[a] - cc[a]) * scale + 0.5);
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = cc[a] - nn[a] * 1.0 / scale;
      r_cr[a] = cc[a] + nn[a] * 1.0 / scale;
    }
    for (int a = 0; a < 3; ++a) {
      l_box[a] = cc_focusing[a] - std::round(n_grid / 2.) / scale;
      r_box[a] = cc_focusing[a] + std::round(n_grid / 2.) / scale;
      if ((r_box[a] - l_box[a]) >= (r_cr[a] - l_cr[a])) {
        r_box[a] = r_cr[a];
        l_box[a] = l_cr[a];
      } else {
        if (l_box[a] <= l_cr[a]) {
          const double err = l_cr[a] - l_box[a];
          l_box[a] += err;
          r_box[a] += err;
        }
        if (r_box[a] >= r_cr[a]) {
          const double err = r_box[a] - r_cr[a];
          if (a < 2) l_box[a] -= err;  // the reference shifts only r_box on z (:519-522)
          r_box[a] -= err;
        }
      }
    }
    const double len_box_foc = n_grid / scale;
    double len_box = rr[0] - ll[0];
    unsigned ratio = 0;
    for (int ii = 1; ii <= 5; ++ii) {
      len_box /= 2.0;
      if (len_box <= len_box_foc) {
        ratio = ii;
        break;
      }
    }
    outlevel = (int)ratio;
  } else if (mesh_shape == 4) {
    double size = 1.0 / scale_max;
    scale = scale_max;
    maxlevel = 0;
    for (int ii = 0; ii < 28; ++ii) {
      size *= 2;
      maxlevel++;
      if (lmax / size < perfil2) break;
    }
    minlevel = (int)(maxlevel - std::sqrt(scale_max / scale_min));
    unilevel = (int)((maxlevel + minlevel) * 0.5);
    unilevel = unilevel + 1;
    outlevel = minlevel;
    scale_level = maxlevel;
    for (int a = 0; a < 3; ++a) {
      ll[a] = cc[a] - size / 2;
      rr[a] = cc[a] + size / 2;
    }
    int nn[3];
    for (int a = 0; a < 3; ++a) nn[a] = (int)((r_cr[a] - cc[a]) * scale + 0.5);
    for (int a = 0; a < 3; ++a) {
      l_cr[a] = cc[a] - nn[a] * 1.0 / scale;
      r_cr[a] = cc[a] + nn[a] * 1.0 / scale;
    }
  } else if (mesh_shape == 5) {
    throw std::runtime_error("mesh_shape 5 (multi-tree forest) is not supported");
  }
  if (mesh_shape == 2) {
    dom.set(l_c, r_c);
    locate_tol = p4esttol * (r_c[0] - l_c[0]);
  } else {
    dom.set(ll, rr);
    locate_tol = p4esttol * (rr[0] - ll[0]);
  }
  tmsh = Octree();
}

// ---------------------------------------------------------------------------
// Octree initialisation (src/pb_class.cpp:1290-1391).
void poisson_boltzmann::init_tmesh() { tmsh.uniform(unilevel); }

static void refine_in_box(Octree& t, const Domain& dom, const double* bl, const double* br, int scale_level) {
  for (int it = 0; it < scale_level; ++it) {
    const std::vector<uint8_t> hm = t.hanging_masks();
    std::vector<uint8_t> marks(t.size(), 0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < t.size(); ++i) {
      const Octant q = t.leaves[i];
      if (q.level >= scale_level) continue;
      const int32_t s = q.size();
      for (int c = 0; c < 8; ++c) {
        if (hm[i] >> c & 1) continue;
        const double x = dom.coord(0, q.x + (c & 1) * s), y = dom.coord(1, q.y + ((c >> 1) & 1) * s),
                     z = dom.coord(2, q.z + ((c >> 2) & 1) * s);
        if (x >= bl[0] && x <= br[0] && y >= bl[1] && y <= br[1] && z >= bl[2] && z <= br[2]) {
          marks[i] = 1;
          break;
        }
      }
    }
    t.refine(marks);
  }
}

void poisson_boltzmann::init_tmesh_with_refine_scale() {
  tmsh.uniform(outlevel);
  refine_in_box(tmsh, dom, l_c, r_c, scale_level);
}

void poisson_boltzmann::init_tmesh_with_refine_box_scale() {
  tmsh.uniform(outlevel);
  refine_in_box(tmsh, dom, l_box, r_box, scale_level);
}

// z-ray parity of every non-hanging corner of every leaf (is_in_ns_surf with
// dir = 2, the value refine_surface keeps in rcoeff).
std::vector<uint8_t> poisson_boltzmann::corner_inside_z(const std::vector<uint8_t>& hm) {
  const int64_t n = tmsh.size();
  // cast missing z rays
  const int nt = omp_get_max_threads();
  std::vector<std::vector<uint64_t>> miss(nt);
#pragma omp parallel
  {
    std::vector<uint64_t>& mine = miss[omp_get_thread_num()];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      const Octant q = tmsh.leaves[i];
      const int32_t s = q.size();
      for (int col = 0; col < 4; ++col) {  // corners col and col + 4 share the z column
        if ((hm[i] >> col & 1) && (hm[i] >> (col + 4) & 1)) continue;
        const uint64_t key = ray_key(q.x + (col & 1) * s, q.y + ((col >> 1) & 1) * s);
        if (!ray_cache.parity_known(2, key)) mine.push_back(key);
      }
    }
  }
  std::vector<uint64_t> all;
  for (auto& v : miss) all.insert(all.end(), v.begin(), v.end());
  ray_cache.ensure(2, std::move(all));
  std::vector<uint8_t> inside(8 * n, 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const Octant q = tmsh.leaves[i];
    const int32_t s = q.size();
    const double z0 = dom.coord(2, q.z), z1 = dom.coord(2, q.z + s);
    for (int col = 0; col < 4; ++col) {
      int32_t m = 0;
      const double* I = ray_cache.crossings(2, ray_key(q.x + (col & 1) * s, q.y + ((col >> 1) & 1) * s), &m);
      for (int h = 0; h < 2; ++h) {
        const int c = col + 4 * h;
        if (hm[i] >> c & 1) continue;
        const double z = h ? z1 : z0;
        int k = 0;
        while (k < m && z >= I[k]) ++k;
        inside[8 * i + c] = (uint8_t)(k & 1);
      }
    }
  }
  return inside;
}

// Surface refinement / coarsening cycles (src/pb_class.cpp:1468-1745).  The
// reference also refines octants that contain an atom centre and protects them
// from coarsening, by looping over `atoms`; its driver empties that vector
// before refine_surface runs (src/poisson_boltzmann.cpp:115), so those clauses
// never fire and are not reproduced here.
void poisson_boltzmann::refine_surface() {
  const int cycles = (maxlevel - unilevel) > (unilevel - minlevel) ? (maxlevel - unilevel) : (unilevel - minlevel);
  double t_hm = 0, t_in = 0, t_ref = 0, t_crs = 0;
  auto tick = [](double& acc, double t0) { acc += omp_get_wtime() - t0; };
  for (int kk = 0; kk < cycles; ++kk) {
    {
      double t = omp_get_wtime();
      const std::vector<uint8_t> hm = tmsh.hanging_masks();
      tick(t_hm, t);
      t = omp_get_wtime();
      const std::vector<uint8_t> in = corner_inside_z(hm);
      tick(t_in, t);
      t = omp_get_wtime();
      std::vector<uint8_t> marks(tmsh.size(), 0);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < tmsh.size(); ++i) {
        if (tmsh.leaves[i].level >= maxlevel) continue;
        double mn = 2.0, mxv = 0.0;
        for (int c = 0; c < 8; ++c) {
          if (hm[i] >> c & 1) continue;
          const double v = in[8 * i + c];
          mxv = std::max(mxv, v);
          mn = std::min(mn, v);
        }
        if (mxv > 0.5 && mn < 0.5) marks[i] = 1;
      }
      tmsh.refine(marks);
      tick(t_ref, t);
    }
    {
      double t = omp_get_wtime();
      const std::vector<uint8_t> hm = tmsh.hanging_masks();
      tick(t_hm, t);
      t = omp_get_wtime();
      const std::vector<uint8_t> in = corner_inside_z(hm);
      tick(t_in, t);
      t = omp_get_wtime();
      std::vector<uint8_t> marks(tmsh.size(), 0);
#pragma omp parallel for schedule(static)
      for (int64_t i = 0; i < tmsh.size(); ++i) {
        if (tmsh.leaves[i].level <= minlevel) continue;
        double mn = 2.0, mxv = 0.0;
        for (int c = 0; c < 8; ++c) {
          if (hm[i] >> c & 1) continue;
          const double v = in[8 * i + c];
          mxv = std::max(mxv, v);
          mn = std::min(mn, v);
        }
        if (mn > 0.5 || mxv < 0.5) marks[i] = 1;
      }
      tmsh.coarsen(marks);
      tick(t_crs, t);
    }
  }
  if (verbose)
    std::fprintf(stderr, "refine_surface: hanging masks %g s, corner classification %g s, refine %g s, coarsen %g s\n",
                 t_hm, t_in, t_ref, t_crs);
}

void poisson_boltzmann::finalize_mesh() {
  nodes = tmsh.build_nodes();
  const int64_t no = tmsh.size();
  oct_xyz.resize(3 * no);
  oct_level.resize(no);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < no; ++i) {
    oct_xyz[3 * i + 0] = tmsh.leaves[i].x;
    oct_xyz[3 * i + 1] = tmsh.leaves[i].y;
    oct_xyz[3 * i + 2] = tmsh.leaves[i].z;
    oct_level[i] = (int8_t)tmsh.leaves[i].level;
  }
  // every node point (independent and hanging) may start an edge the path
  // queries, on every axis
  const int64_t n = nodes.n_indep, nh = nodes.n_hang;
  for (int axis = 0; axis < 3; ++axis) {
    const int t0 = axis == 0 ? 1 : 0, t1 = axis == 2 ? 1 : 2;
    std::vector<uint64_t> keys(n + nh);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < n; ++j) keys[j] = ray_key(nodes.indep_xyz[3 * j + t0], nodes.indep_xyz[3 * j + t1]);
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < nh; ++j) keys[n + j] = ray_key(nodes.hang_xyz[3 * j + t0], nodes.hang_xyz[3 * j + t1]);
    __gnu_parallel::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    ray_cache.ensure(axis, keys);
    ray_tables[axis] = ray_cache.table(axis, keys);
  }
}

void poisson_boltzmann::build_problem() {
  const double t0 = omp_get_wtime();
  create_mesh();
  surf.build(atoms, 0.0);
  ray_cache.clear();
  ray_cache.surf = &surf;
  ray_cache.dom = &dom;
  if (mesh_shape == 0 || refine_box == 1 || mesh_shape == 4)
    init_tmesh_with_refine_scale();
  else if (mesh_shape == 3)
    init_tmesh_with_refine_box_scale();
  else
    init_tmesh();
  const double t1 = omp_get_wtime();
  if (loc_refinement == 1 || mesh_shape == 4) refine_surface();
  const double t2 = omp_get_wtime();
  finalize_mesh();
  const double t3 = omp_get_wtime();
  if (verbose)
    std::cerr << "build_problem: init " << t1 - t0 << " s, refine_surface " << t2 - t1 << " s, nodes+rays "
              << t3 - t2 << " s, " << tmsh.size() << " octants\n";
}

void poisson_boltzmann::initial_octree(pbgpu_mesh_build* out, bool on_gpu) {
  create_mesh();
  // the init_tmesh* variant of the driver (uniform level, box and its level)
  const bool scale_box = mesh_shape == 0 || refine_box == 1 || mesh_shape == 4;
  const int init_level = (scale_box || mesh_shape == 3) ? outlevel : unilevel;
  const int box_level = (scale_box || mesh_shape == 3) ? scale_level : 0;
  const double* bl = scale_box ? l_c : l_box;
  const double* br = scale_box ? r_c : r_box;
  if (on_gpu && init_level <= 8) {
    tmsh.leaves.clear();
    tmsh.keys.clear();
    gb_xyz.clear();
    gb_level.clear();
  } else if (scale_box) {
    init_tmesh_with_refine_scale();
  } else if (mesh_shape == 3) {
    init_tmesh_with_refine_box_scale();
  } else {
    init_tmesh();
  }
  const int64_t no = (on_gpu && init_level <= 8) ? 0 : tmsh.size();
  gb_xyz.assign(3 * no, 0);
  gb_level.assign(no, 0);
  for (int64_t i = 0; i < no; ++i) {
    gb_xyz[3 * i + 0] = tmsh.leaves[i].x;
    gb_xyz[3 * i + 1] = tmsh.leaves[i].y;
    gb_xyz[3 * i + 2] = tmsh.leaves[i].z;
    gb_level[i] = (int8_t)tmsh.leaves[i].level;
  }
  gb_spheres.assign(4 * atoms.size(), 0.0);
  for (size_t i = 0; i < atoms.size(); ++i) {
    for (int k = 0; k < 3; ++k) gb_spheres[4 * i + k] = atoms[i].pos[k];
    gb_spheres[4 * i + 3] = atoms[i].radius;
  }
  pbgpu_mesh_build& b = *out;
  b = pbgpu_mesh_build{};
  b.n_oct = no;
  b.oct_xyz = gb_xyz.data();
  b.oct_level = gb_level.data();
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = dom.lo[a];
    b.hi[a] = dom.hi[a];
  }
  b.locate_tol = locate_tol;
  b.refine = (loc_refinement == 1 || mesh_shape == 4) ? 1 : 0;
  b.minlevel = minlevel;
  b.maxlevel = maxlevel;
  b.unilevel = unilevel;
  b.n_spheres = (int64_t)atoms.size();
  b.spheres = gb_spheres.data();
  b.init_level = init_level;
  b.box_level = box_level;
  for (int a = 0; a < 3; ++a) {
    b.box_lo[a] = bl[a];
    b.box_hi[a] = br[a];
  }
}

int poisson_boltzmann::build_problem_on_gpu(pbgpu_ctx* ctx) {
  const double t0 = omp_get_wtime();
  pbgpu_mesh_build b{};
  initial_octree(&b, true);
  if (gpu && own_gpu && gpu != ctx) pbgpu_ctx_destroy(gpu);
  gpu = ctx;
  own_gpu = false;
  int st = check(pbgpu_build_mesh(ctx, &b));
  if (st != PBGPU_OK) return st;
  std::vector<double> pos(3 * pos_atoms.size());
  for (size_t i = 0; i < pos_atoms.size(); ++i)
    for (int k = 0; k < 3; ++k) pos[3 * i + k] = pos_atoms[i][k];
  if ((st = check(pbgpu_set_atoms(ctx, (int64_t)pos_atoms.size(), pos.data(), charge_atoms.data()))) != PBGPU_OK)
    return st;
  const pbgpu_model md = model();
  st = check(pbgpu_set_model(ctx, &md));
  if (verbose) std::cerr << "build_problem_on_gpu: " << omp_get_wtime() - t0 << " s\n";
  return st;
}

// ---------------------------------------------------------------------------
// GPU path.
pbgpu_model poisson_boltzmann::model() const {
  pbgpu_model m{};
  m.e_in = e_in;
  m.e_out = e_out;
  m.ionic_strength = ionic_strength;
  m.T = T;
  m.bc_type = bc;
  m.stern_layer_surf = stern_layer_surf;
  m.stern_layer = stern_layer;
  m.calc_energy = calc_energy;
  m.calc_coulombic = calc_coulombic;
  return m;
}

pbgpu_mesh poisson_boltzmann::mesh_view() const {
  pbgpu_mesh m{};
  m.n_oct = (int64_t)oct_level.size();
  m.oct_xyz = oct_xyz.data();
  m.oct_level = oct_level.data();
  m.oct_nodes = nodes.oct_nodes.data();
  m.n_nodes = nodes.n_indep;
  m.node_xyz = nodes.indep_xyz.data();
  m.n_hang = nodes.n_hang;
  m.hang_np = nodes.hang_np.data();
  m.hang_par = nodes.hang_par.data();
  for (int a = 0; a < 3; ++a) {
    m.lo[a] = dom.lo[a];
    m.hi[a] = dom.hi[a];
  }
  m.locate_tol = locate_tol;
  return m;
}

pbgpu_rays poisson_boltzmann::rays_view(int axis) const {
  const RayTable& t = ray_tables[axis];
  pbgpu_rays r{};
  r.n_rays = t.n();
  r.keys = t.keys.data();
  r.ptr = t.ptr.data();
  r.inters = t.inters.data();
  r.normals = t.normals.data();
  return r;
}

int poisson_boltzmann::check(int status) {
  if (status != PBGPU_OK && gpu) last_error = pbgpu_last_error(gpu);
  return status;
}

int poisson_boltzmann::upload() {
  int st = PBGPU_OK;
  if (!gpu) {
    if ((st = pbgpu_ctx_create(&gpu, 0, nullptr)) != PBGPU_OK) {
      last_error = "pbgpu_ctx_create failed";
      return st;
    }
    own_gpu = true;
  }
  const pbgpu_mesh m = mesh_view();
  if ((st = check(pbgpu_set_mesh(gpu, &m))) != PBGPU_OK) return st;
  for (int a = 0; a < 3; ++a) {
    const pbgpu_rays r = rays_view(a);
    if ((st = check(pbgpu_set_rays(gpu, a, &r))) != PBGPU_OK) return st;
  }
  std::vector<double> pos(3 * pos_atoms.size());
  for (size_t i = 0; i < pos_atoms.size(); ++i)
    for (int k = 0; k < 3; ++k) pos[3 * i + k] = pos_atoms[i][k];
  if ((st = check(pbgpu_set_atoms(gpu, (int64_t)pos_atoms.size(), pos.data(), charge_atoms.data()))) != PBGPU_OK)
    return st;
  const pbgpu_model md = model();
  return check(pbgpu_set_model(gpu, &md));
}

int poisson_boltzmann::create_markers() { return check(pbgpu_create_markers(gpu)); }
int poisson_boltzmann::create_density_map() { return check(pbgpu_create_density_map(gpu)); }
int poisson_boltzmann::assemple_system_matrix() { return check(pbgpu_assemble(gpu, nullptr)); }

int poisson_boltzmann::lis_compute_electric_potential() {
  pbgpu_solver_opts o;
  int st = pbgpu_parse_lis_options(linear_solver_options.c_str(), &o);
  if (st != PBGPU_OK) {
    last_error = "bad solver_options";
    return st;
  }
  return check(pbgpu_solve(gpu, &o, &solve_stats));
}

// The reference factorises with MUMPS; here the same system is solved by
// Jacobi-preconditioned BiCGStab to a relative residual of 1e-12.
int poisson_boltzmann::mumps_compute_electric_potential() {
  pbgpu_solver_opts o;
  pbgpu_default_solver_opts(&o);
  o.method = PBGPU_BICGSTAB;
  o.tol = 1e-12;
  o.max_iter = 100000;
  return check(pbgpu_solve(gpu, &o, &solve_stats));
}

// phi_on_atoms.txt in the reference's format (src/pb_class.cpp:2369-2376).
int poisson_boltzmann::write_potential_on_atoms_fast(const std::string& path) {
  phi_on_atoms.assign(pos_atoms.size(), 0.0);
  int st = check(pbgpu_phi_on_atoms(gpu, phi_on_atoms.data()));
  if (st != PBGPU_OK || path.empty()) return st;
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    last_error = "cannot write " + path;
    return PBGPU_ERR_ARG;
  }
  for (size_t i = 0; i < pos_atoms.size(); ++i) {
    if (std::isnan(phi_on_atoms[i])) continue;
    std::fprintf(f, "%8d%8.3f%8.3f%8.3f  %.4f\n", index_atoms[i], pos_atoms[i][0], pos_atoms[i][1], pos_atoms[i][2],
                 phi_on_atoms[i]);
  }
  std::fclose(f);
  return PBGPU_OK;
}

static void print_energy(const pbgpu_energy_out& e, int calc_energy, int calc_coulombic) {
  const int w = 50;
  std::cout << "\n================ [ Electrostatic Energy ] =================\n";
  std::cout << std::left << std::setw(w) << "  Net charge [e]:" << std::setprecision(16) << e.net_charge << "\n";
  std::cout << std::left << std::setw(w) << "  Flux charge [e]:" << std::setprecision(16) << e.charge_flux << "\n";
  std::cout << std::left << std::setw(w) << "  Polarization energy [kT]:" << std::setprecision(16) << e.energy_pol
            << "\n";
  if (calc_energy == 2)
    std::cout << std::left << std::setw(w) << "  Direct ionic energy [kT]:" << std::setprecision(16)
              << e.energy_react << "\n";
  if (calc_coulombic == 1)
    std::cout << std::left << std::setw(w) << "  Coulombic energy [kT]:" << std::setprecision(16) << e.energy_coul
              << "\n";
  std::cout << std::left << std::setw(w) << "  Sum of electrostatic energy contributions [kT]:"
            << std::setprecision(16) << e.sum << "\n";
  std::cout << "===========================================================\n";
}

static int run_energy(poisson_boltzmann& pb, int fast) {
  pbgpu_energy_out e{};
  int st = pbgpu_energy(pb.gpu, fast, &e);
  if (st != PBGPU_OK) {
    pb.last_error = pbgpu_last_error(pb.gpu);
    return st;
  }
  pb.energy_pol = e.energy_pol;
  pb.energy_react = e.energy_react;
  pb.coul_energy = e.energy_coul;
  pb.charge_flux = e.charge_flux;
  if (pb.verbose) print_energy(e, pb.calc_energy, pb.calc_coulombic);
  return PBGPU_OK;
}

int poisson_boltzmann::energy() { return run_energy(*this, 0); }
int poisson_boltzmann::energy_fast() { return run_energy(*this, 1); }

// The heading line of pot_field.dat for each set of written columns
// (src/pb_class.cpp:4279-4363; pot_field adds a space before the newline of the
// phi_i-without-fields heading, :4982).
static const char* pot_field_heading(int columns, int fast) {
  const int kC = (1 << PBGPU_PF_PHI_C) | (7 << PBGPU_PF_EX_C);
  const int kP = 1 << PBGPU_PF_PHI_P, kEP = 7 << PBGPU_PF_EX_P;
  const int kI = 1 << PBGPU_PF_PHI_I, kEI = 7 << PBGPU_PF_EX_I;
  if (columns == (kC | kP | kEP | kI | kEI))
    return "phi_c    phi_p    phi_i    Ex_c    Ey_c    Ez_c   Ex_p    Ey_p    Ez_p   Ex_i    Ey_i    Ez_i\n";
  if (columns == (kC | kP | kI))
    return fast ? "phi_c    phi_p    phi_i    Ex_c    Ey_c    Ez_c\n" : "phi_c    phi_p    phi_i    Ex_c    Ey_c    Ez_c \n";
  if (columns == (kC | kP | kEP | kI)) return "phi_c    phi_p    phi_i    Ex_c    Ey_c    Ez_c   Ex_p    Ey_p    Ez_p\n";
  if (columns == (kC | kP)) return "phi_c    phi_p    Ex_c    Ey_c    Ez_c\n";
  if (columns == (kC | kP | kEP)) return "phi_c    phi_p    Ex_c    Ey_c    Ez_c   Ex_p    Ey_p    Ez_p\n";
  return "";
}

// pot_field / pot_field_fast: the GPU computes the rows; the energies and the
// file follow the reference (:4252-4272 on stdout, :4277-4384 to the file,
// setw(8) in the stream's default 6-significant-digit format).
static int run_pot_field(poisson_boltzmann& pb, int fast, const std::string& path) {
  const size_t na = pb.pos_atoms.size();
  pb.pot_field_rows.assign(na * PBGPU_PF_COLUMNS, 0.0);
  pbgpu_pot_field_out o{};
  int st = pbgpu_pot_field(pb.gpu, fast, pb.calc_potential_term, pb.calc_field_term, pb.pot_field_rows.data(), &o);
  if (st != PBGPU_OK) {
    pb.last_error = pbgpu_last_error(pb.gpu);
    return st;
  }
  pb.pot_field_columns = o.columns;
  pb.energy_pol = o.energy_pol;
  pb.energy_react = o.energy_react;
  pb.coul_energy = o.energy_coul;
  pb.charge_flux = o.charge_flux;
  const int pt = pb.calc_potential_term, ft = pb.calc_field_term;
  if (pb.verbose) {
    const int w = 50;
    std::cout << "\n================ [ Calculating Potential & Field Components ] =================\n";
    if (pt == 1 || ft == 1 || pt == 2 || ft == 2)
      std::cout << std::left << std::setw(w) << "  Polarization energy [kT]:" << std::setprecision(16) << o.energy_pol
                << "\n";
    if (pt == 2 || ft == 2)
      std::cout << std::left << std::setw(w) << "  Direct ionic energy [kT]:" << std::setprecision(16)
                << o.energy_react << "\n";
    std::cout << std::left << std::setw(w) << "  Coulombic energy [kT]:" << std::setprecision(16) << o.energy_coul
              << "\n";
    std::cout << std::left << std::setw(w) << "  Sum of electrostatic energy contributions [kT]:"
              << std::setprecision(16) << (o.energy_pol + o.energy_react + o.energy_coul) << "\n";
    std::cout << "===========================================================\n";
  }
  if (path.empty()) return PBGPU_OK;
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) {
    pb.last_error = "cannot write " + path;
    return PBGPU_ERR_ARG;
  }
  std::fputs("# index    x    y    z    ", f);
  std::fputs(pot_field_heading(o.columns, fast), f);
  if (o.columns)
    for (size_t i = 0; i < na; ++i) {
      std::fprintf(f, "%5d  %8g  %8g  %8g  ", (int)(i + 1), pb.pos_atoms[i][0], pb.pos_atoms[i][1],
                   pb.pos_atoms[i][2]);
      for (int k = 0; k < PBGPU_PF_COLUMNS; ++k)
        if ((o.columns >> k) & 1) std::fprintf(f, "%8g  ", pb.pot_field_rows[i * PBGPU_PF_COLUMNS + k]);
      std::fputs("\n", f);
    }
  std::fclose(f);
  return PBGPU_OK;
}

int poisson_boltzmann::pot_field(const std::string& path) { return run_pot_field(*this, 0, path); }
int poisson_boltzmann::pot_field_fast(const std::string& path) { return run_pot_field(*this, 1, path); }

// The mesh of a field: the host's own tables when the host built the mesh,
// else the context's (built on the GPU), copied back.
int poisson_boltzmann::write_vtu(const std::string& basename, const std::string& fieldname, const double* values) {
  VtuMesh vm;
  std::vector<int32_t> oxyz, onodes, nxyz, hpar;
  std::vector<int8_t> olvl, hnp;
  if (!oct_level.empty()) {
    const pbgpu_mesh m = mesh_view();
    vm.n_oct = m.n_oct;
    vm.oct_xyz = m.oct_xyz;
    vm.oct_level = m.oct_level;
    vm.oct_nodes = m.oct_nodes;
    vm.n_nodes = m.n_nodes;
    vm.node_xyz = m.node_xyz;
    vm.n_hang = m.n_hang;
    vm.hang_np = m.hang_np;
    vm.hang_par = m.hang_par;
    for (int a = 0; a < 3; ++a) {
      vm.lo[a] = m.lo[a];
      vm.extent[a] = m.hi[a] - m.lo[a];
    }
  } else if (gpu) {
    int64_t no = 0, nn = 0, nh = 0, nr[3];
    int st = check(pbgpu_get_mesh_counts(gpu, &no, &nn, &nh, nr));
    if (st != PBGPU_OK) return st;
    oxyz.resize(3 * no);
    olvl.resize(no);
    onodes.resize(8 * no);
    nxyz.resize(3 * nn);
    hnp.resize(nh);
    hpar.resize(4 * nh);
    double box[6];
    st = check(pbgpu_get_mesh(gpu, oxyz.data(), olvl.data(), onodes.data(), nxyz.data(), hnp.data(), hpar.data(), box));
    if (st != PBGPU_OK) return st;
    vm.n_oct = no;
    vm.oct_xyz = oxyz.data();
    vm.oct_level = olvl.data();
    vm.oct_nodes = onodes.data();
    vm.n_nodes = nn;
    vm.node_xyz = nxyz.data();
    vm.n_hang = nh;
    vm.hang_np = hnp.data();
    vm.hang_par = hpar.data();
    for (int a = 0; a < 3; ++a) {
      vm.lo[a] = box[a];
      vm.extent[a] = box[3 + a];
    }
  } else {
    last_error = "write_vtu: no mesh";
    return PBGPU_ERR_STATE;
  }
  if (!pbh::write_vtu(basename, fieldname, vm, values, &last_error)) return PBGPU_ERR_ARG;
  return PBGPU_OK;
}

// map_type = vtu: potential_map_0000.vtu (phi), eps_map_0000.vtu (epsilon at
// the nodes) and their total_*.pvtu.  The octbin format of map_type = oct is
// p4est's own and is not written here.
int poisson_boltzmann::export_maps() {
  if (!potential_map && !eps_map) return PBGPU_OK;
  if (map_type == "oct") {
    last_error = "map_type = oct (p4est octbin) is not supported; use map_type = vtu";
    return PBGPU_ERR_ARG;
  }
  if (map_type != "vtu") {
    last_error = "Wrong type of map output: " + map_type;
    return PBGPU_ERR_ARG;
  }
  int64_t no = 0, nn = 0, nh = 0, nr[3];
  int st = check(pbgpu_get_mesh_counts(gpu, &no, &nn, &nh, nr));
  if (st != PBGPU_OK) return st;
  std::vector<std::string> fields, bases;
  std::vector<double> v(nn);
  if (potential_map) {
    if ((st = check(pbgpu_get_phi(gpu, v.data()))) != PBGPU_OK) return st;
    if ((st = write_vtu("potential_map", "phi", v.data())) != PBGPU_OK) return st;
    fields.push_back("phi");
    bases.push_back("potential_map");
  }
  if (eps_map) {
    if ((st = check(pbgpu_get_node_coeffs(gpu, v.data(), nullptr))) != PBGPU_OK) return st;
    if ((st = write_vtu("eps_map", "eps", v.data())) != PBGPU_OK) return st;
    fields.push_back("eps");
    bases.push_back("eps_map");
  }
  if (!pbh::write_pvtu(fields, bases, 1, &last_error)) return PBGPU_ERR_ARG;
  return PBGPU_OK;
}

// The driver's sequence from create_markers on (src/poisson_boltzmann.cpp:192-299).
int poisson_boltzmann::run_gpu_path() {
  int st;
  if ((st = upload()) != PBGPU_OK) return st;
  if ((st = create_markers()) != PBGPU_OK) return st;
  if ((st = create_density_map()) != PBGPU_OK) return st;
  if ((st = assemple_system_matrix()) != PBGPU_OK) return st;
  if (linear_solver_name == "mumps")
    st = mumps_compute_electric_potential();
  else if (linear_solver_name == "lis")
    st = lis_compute_electric_potential();
  else {
    last_error = "Invalid linear solver selected";
    return PBGPU_ERR_ARG;
  }
  if (st != PBGPU_OK && st != PBGPU_NOT_CONVERGED) return st;
  if (atoms_write == 1) {
    const int s2 = write_potential_on_atoms_fast();
    if (s2 != PBGPU_OK) return s2;
  }
  // :272-296
  if (calc_potential_term > 0 || calc_field_term > 0 || calc_energy > 0) {
    const bool refined = (loc_refinement == 1 || mesh_shape > 2 || (mesh_shape == 2 && refine_box == 1));
    const bool pot_field_bool = (calc_potential_term > 0 || calc_field_term > 0);
    int s3 = PBGPU_OK;
    if (pot_field_bool) {
      s3 = refined ? pot_field() : pot_field_fast();
      if (s3 == PBGPU_OK && calc_energy > calc_potential_term && calc_energy > calc_field_term)
        s3 = refined ? energy() : energy_fast();
    } else {
      s3 = refined ? energy() : energy_fast();
    }
    if (s3 != PBGPU_OK) return s3;
  }
  // :305-351
  const int s4 = export_maps();
  if (s4 != PBGPU_OK) return s4;
  return st;
}

}  // namespace pbh
