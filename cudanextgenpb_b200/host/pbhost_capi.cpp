// C API over the host poisson_boltzmann mirror (include/pbhost.h).
#include "../../include/pbhost.h"

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>

#include "pb_class.h"

struct pbhost {
  pbh::poisson_boltzmann pb;
  pbh::OptionFile opts;
  std::string err;
};

#define PBHOST_TRY(h, body)            \
  try {                                \
    body;                              \
  } catch (const std::exception& ex) { \
    (h)->err = ex.what();              \
    return PBGPU_ERR_ARG;              \
  }

extern "C" {

pbhost* pbhost_create(void) {
  pbhost* h = new pbhost();
  h->pb.apply_options(h->opts);
  return h;
}

void pbhost_destroy(pbhost* h) { delete h; }

const char* pbhost_last_error(const pbhost* h) { return h ? h->err.c_str() : "null handle"; }

int pbhost_load_options_file(pbhost* h, const char* path) {
  if (!h || !path) return PBGPU_ERR_ARG;
  if (!h->opts.load_file(path)) {
    h->err = std::string("cannot read options file ") + path;
    return PBGPU_ERR_ARG;
  }
  PBHOST_TRY(h, h->pb.apply_options(h->opts));
  h->pb.optionsfilename = path;
  return PBGPU_OK;
}

int pbhost_load_options_text(pbhost* h, const char* text) {
  if (!h || !text) return PBGPU_ERR_ARG;
  h->opts.load_text(text);
  PBHOST_TRY(h, h->pb.apply_options(h->opts));
  return PBGPU_OK;
}

int pbhost_set_option(pbhost* h, const char* key, const char* value) {
  if (!h || !key || !value) return PBGPU_ERR_ARG;
  h->opts.set(key, value);
  PBHOST_TRY(h, h->pb.apply_options(h->opts));
  return PBGPU_OK;
}

int pbhost_read_pqr(pbhost* h, const char* path) {
  if (!h || !path) return PBGPU_ERR_ARG;
  std::ifstream f(path);
  if (!f) {
    h->err = std::string("Cannot find the pqr file ") + path;
    return PBGPU_ERR_ARG;
  }
  PBHOST_TRY(h, {
    h->pb.read_atoms_from_pqr(f);
    h->pb.read_atoms_from_class();
  });
  if (h->pb.atoms.empty()) {
    h->err = "no atoms read";
    return PBGPU_ERR_ARG;
  }
  return PBGPU_OK;
}

int pbhost_set_atoms(pbhost* h, int64_t n, const double* pos, const double* charge, const double* radius) {
  if (!h || n <= 0 || !pos || !charge || !radius) return PBGPU_ERR_ARG;
  std::string text;
  h->pb.atoms.clear();
  for (int64_t i = 0; i < n; ++i) {
    pbh::Atom a{};
    for (int k = 0; k < 3; ++k) a.pos[k] = pos[3 * i + k];
    a.charge = charge[i];
    a.radius = radius[i] < 1.e-5 ? 1.0 : radius[i];
    h->pb.atoms.push_back(a);
  }
  if (h->pb.atoms.size() < 4) {
    // same dummy rule as read_atoms_from_pqr
    auto it = std::max_element(h->pb.atoms.begin(), h->pb.atoms.end(),
                               [](const pbh::Atom& x, const pbh::Atom& y) { return x.radius < y.radius; });
    const double p[3] = {it->pos[0], it->pos[1], it->pos[2]};
    const int dirs[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    for (int d = 0; d < 6; ++d) {
      pbh::Atom dm{};
      for (int k = 0; k < 3; ++k) dm.pos[k] = p[k] + 0.001 * dirs[d][k];
      h->pb.atoms.push_back(dm);
    }
  }
  h->pb.read_atoms_from_class();
  return PBGPU_OK;
}

int pbhost_build_problem(pbhost* h) {
  if (!h) return PBGPU_ERR_ARG;
  if (h->pb.atoms.empty()) {
    h->err = "no atoms";
    return PBGPU_ERR_STATE;
  }
  const char* v = std::getenv("PBHOST_VERBOSE");
  h->pb.verbose = (v && *v && *v != '0') ? 1 : 0;
  PBHOST_TRY(h, h->pb.build_problem());
  return PBGPU_OK;
}

int pbhost_build_on_gpu(pbhost* h, pbgpu_ctx* ctx) {
  if (!h || !ctx) return PBGPU_ERR_ARG;
  if (h->pb.atoms.empty()) {
    h->err = "no atoms";
    return PBGPU_ERR_STATE;
  }
  const char* v = std::getenv("PBHOST_VERBOSE");
  h->pb.verbose = (v && *v && *v != '0') ? 1 : 0;
  int st = PBGPU_OK;
  try {
    st = h->pb.build_problem_on_gpu(ctx);
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return PBGPU_ERR_ARG;
  }
  if (st != PBGPU_OK) h->err = h->pb.last_error;
  return st;
}

int pbhost_initial_octree(pbhost* h, int on_gpu, pbgpu_mesh_build* out) {
  if (!h || !out) return PBGPU_ERR_ARG;
  if (h->pb.atoms.empty()) {
    h->err = "no atoms";
    return PBGPU_ERR_STATE;
  }
  try {
    h->pb.initial_octree(out, on_gpu != 0);
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return PBGPU_ERR_ARG;
  }
  return PBGPU_OK;
}

int pbhost_write_vtu(pbhost* h, const char* basename, const char* fieldname, const double* values) {
  if (!h || !basename || !fieldname || !values) return PBGPU_ERR_ARG;
  int st;
  try {
    st = h->pb.write_vtu(basename, fieldname, values);
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return PBGPU_ERR_ARG;
  }
  if (st != PBGPU_OK) h->err = h->pb.last_error;
  return st;
}

int pbhost_get_info(const pbhost* h, pbhost_info* o) {
  if (!h || !o) return PBGPU_ERR_ARG;
  const pbh::poisson_boltzmann& p = h->pb;
  std::memset(o, 0, sizeof(*o));
  o->mesh_shape = p.mesh_shape;
  o->unilevel = p.unilevel;
  o->minlevel = p.minlevel;
  o->maxlevel = p.maxlevel;
  o->outlevel = p.outlevel;
  o->scale_level = p.scale_level;
  o->loc_refinement = p.loc_refinement;
  o->scale = p.scale;
  for (int a = 0; a < 3; ++a) {
    o->lo[a] = p.dom.lo[a];
    o->hi[a] = p.dom.hi[a];
    o->cc[a] = p.cc[a];
    o->l_c[a] = p.l_c[a];
    o->r_c[a] = p.r_c[a];
    o->l_cr[a] = p.l_cr[a];
    o->r_cr[a] = p.r_cr[a];
    o->n_rays[a] = p.ray_tables[a].n();
  }
  o->pot_bc = p.pot_bc;
  o->locate_tol = p.locate_tol;
  o->n_oct = (int64_t)p.oct_level.size();
  o->n_nodes = p.nodes.n_indep;
  o->n_hang = p.nodes.n_hang;
  o->n_atoms = (int64_t)p.pos_atoms.size();
  o->net_charge = p.net_charge;
  return PBGPU_OK;
}

int pbhost_get_mesh(const pbhost* h, pbgpu_mesh* out) {
  if (!h || !out) return PBGPU_ERR_ARG;
  *out = h->pb.mesh_view();
  return PBGPU_OK;
}

int pbhost_get_rays(const pbhost* h, int axis, pbgpu_rays* out) {
  if (!h || !out || axis < 0 || axis > 2) return PBGPU_ERR_ARG;
  *out = h->pb.rays_view(axis);
  return PBGPU_OK;
}

int pbhost_get_atoms(const pbhost* h, double* pos, double* charge, double* radius) {
  if (!h) return PBGPU_ERR_ARG;
  const pbh::poisson_boltzmann& p = h->pb;
  for (size_t i = 0; i < p.pos_atoms.size(); ++i) {
    if (pos)
      for (int k = 0; k < 3; ++k) pos[3 * i + k] = p.pos_atoms[i][k];
    if (charge) charge[i] = p.charge_atoms[i];
    if (radius) radius[i] = p.r_atoms[i];
  }
  return PBGPU_OK;
}

int pbhost_get_model(const pbhost* h, pbgpu_model* out) {
  if (!h || !out) return PBGPU_ERR_ARG;
  *out = h->pb.model();
  return PBGPU_OK;
}

int pbhost_get_solver_opts(const pbhost* h, pbgpu_solver_opts* out) {
  if (!h || !out) return PBGPU_ERR_ARG;
  if (h->pb.linear_solver_name == "mumps") {
    pbgpu_default_solver_opts(out);
    out->method = PBGPU_BICGSTAB;
    out->tol = 1e-12;
    out->max_iter = 100000;
    return PBGPU_OK;
  }
  return pbgpu_parse_lis_options(h->pb.linear_solver_options.c_str(), out);
}

int pbhost_run_gpu(pbhost* h, pbgpu_energy_out* e, pbgpu_solve_stats* st) {
  if (!h) return PBGPU_ERR_ARG;
  int s;
  try {
    s = h->pb.run_gpu_path();
  } catch (const std::exception& ex) {
    h->err = ex.what();
    return PBGPU_ERR_ARG;
  }
  if (s != PBGPU_OK) h->err = h->pb.last_error;
  if (st) *st = h->pb.solve_stats;
  if (e) {
    e->energy_pol = h->pb.energy_pol;
    e->energy_react = h->pb.energy_react;
    e->energy_coul = h->pb.coul_energy;
    e->charge_flux = h->pb.charge_flux;
    e->net_charge = h->pb.net_charge;
    e->sum = h->pb.energy_pol + h->pb.energy_react + h->pb.coul_energy;
  }
  return s;
}

pbgpu_ctx* pbhost_gpu_ctx(pbhost* h) { return h ? h->pb.gpu : nullptr; }

}  // extern "C"
