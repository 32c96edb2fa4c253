// Host-side mirror of the reference's poisson_boltzmann struct (pb_class API,
// include/pb_class.h:57-810), restricted to what the assemble/solve/energy path
// needs.  Member and method names follow the reference so that its driver
// sequence (src/poisson_boltzmann.cpp:58-398) reads the same; the stages from
// create_markers to energy call the pbgpu C ABI (include/pbgpu.h) instead of
// bimpp, LIS and MUMPS.
#pragma once
#include <array>
#include <cstdint>
#include <istream>
#include <string>
#include <vector>

#include "../../include/pbgpu.h"
#include "octree.h"
#include "options.h"
#include "surface.h"

namespace pbh {

// Physical constants of the reference (include/pb_class.h:47-54).
constexpr double e_0 = 8.85418781762e-12;
constexpr double kb = 1.380649e-23;
constexpr double e_charge = 1.602176634e-19;
constexpr double N_av = 6.022e23;
constexpr double Angs = 1e-10;
constexpr double pi = 3.14159265358979323846;

struct poisson_boltzmann {
  // atoms
  std::vector<Atom> atoms;
  std::vector<std::array<double, 3>> pos_atoms;
  std::vector<double> charge_atoms, r_atoms;
  std::vector<int> index_atoms;

  // [input]
  std::string filetype = "pqr", pqrfilename, optionsfilename;
  // domain (src/pb_class.cpp:39-743)
  double cc[3] = {0, 0, 0}, ll[3] = {0, 0, 0}, rr[3] = {0, 0, 0};
  double l_c[3] = {0, 0, 0}, r_c[3] = {0, 0, 0}, l_cr[3] = {0, 0, 0}, r_cr[3] = {0, 0, 0};
  double l_box[3] = {0, 0, 0}, r_box[3] = {0, 0, 0}, cc_focusing[3] = {0, 0, 0};
  double pot_bc = 0.0, len = 50.0;
  int n_grid = 8;
  // [mesh]
  int maxlevel = 9, minlevel = 3, unilevel = 5, outlevel = 1, loc_refinement = 0, mesh_shape = 1;
  int refine_box = 0, rand_center = 0, scale_level = 0, scale_level_min_box = 0, aligned = 0;
  double scale = 2.0, scale_min = 0.5, scale_max = 2.0, perfil1 = 0.8, perfil2 = 0.2;
  // [model]
  int linearized = 1, bc = 1, calc_energy = 2, calc_coulombic = 0, atoms_write = 0;
  int calc_potential_term = 0, calc_field_term = 0;
  std::string map_type = "vtu";
  int potential_map = 0, eps_map = 0;
  double e_in = 2.0, e_out = 80.0, ionic_strength = 0.145, T = 298.15;
  double net_charge = 0.0;
  // [surface]
  int surf_type_num = 0, stern_layer_surf = 0;
  double surf_param = 1.4, prb_radius = 1.4, stern_layer = 2.0;
  // [algorithm]
  std::string linear_solver_name = "lis";
  std::string linear_solver_options = "-p ssor -ssor_omega 0.51 -i cgs -tol 1.e-6 -print 2 -conv_cond 2 -tol_w 0";

  // results (include/pb_class.h:126-128)
  double energy_pol = 0.0, energy_react = 0.0, coul_energy = 0.0, charge_flux = 0.0;
  // pot_field results: one row of PBGPU_PF_COLUMNS values per atom
  std::vector<double> pot_field_rows;
  int pot_field_columns = 0;
  std::vector<double> phi_on_atoms;
  pbgpu_solve_stats solve_stats{};

  // mesh and surface
  Octree tmsh;
  NodeTable nodes;
  std::vector<int32_t> oct_xyz;  // 3 per leaf, filled by finalize_mesh
  std::vector<int8_t> oct_level;
  Domain dom;
  SphereUnion surf;
  RayCache ray_cache;
  RayTable ray_tables[3];
  double locate_tol = 0.0;
  int verbose = 0;

  // GPU context of this problem; destroyed with the problem only when the
  // problem created it (upload), not when a caller lent it (build_problem_on_gpu)
  pbgpu_ctx* gpu = nullptr;
  bool own_gpu = false;
  std::string last_error;

  ~poisson_boltzmann();

  // ---- configuration (src/pb_class.cpp:809-978)
  int parse_options(int argc, char** argv);
  void apply_options(const OptionFile& g);
  // ---- atoms (src/pb_class.cpp:1099-1287)
  void read_atoms_from_pqr(std::istream& in);
  void read_atoms_from_class();
  // ---- mesh (src/pb_class.cpp:39-743, 1290-1391, 1468-1745)
  void create_mesh();
  void init_tmesh();
  void init_tmesh_with_refine_scale();
  void init_tmesh_with_refine_box_scale();
  void refine_surface();
  // Node tables and ray tables for the final mesh (the inputs of the GPU path).
  void finalize_mesh();
  // Standard driver sequence up to finalize_mesh (src/poisson_boltzmann.cpp:112-188).
  void build_problem();
  // The same problem with the surface refinement, nodes and ray tables built on
  // the GPU (pbgpu_build_mesh) into `ctx`, which then also holds the atoms and
  // the model: the domain and the initial octree are built here.
  int build_problem_on_gpu(pbgpu_ctx* ctx);
  // The host half of build_problem_on_gpu: the domain, and the initial
  // octree either built here (arrays in this object until the next call) or,
  // with on_gpu, described for pbgpu_build_mesh to build (n_oct = 0).
  void initial_octree(pbgpu_mesh_build* out, bool on_gpu);
  std::vector<int32_t> gb_xyz;
  std::vector<int8_t> gb_level;
  std::vector<double> gb_spheres;

  // ---- the GPU path (src/poisson_boltzmann.cpp:192-299)
  int upload();
  int create_markers();
  int create_density_map();
  int assemple_system_matrix();
  int lis_compute_electric_potential();
  int mumps_compute_electric_potential();
  int write_potential_on_atoms_fast(const std::string& path = "phi_on_atoms.txt");
  int energy();
  int energy_fast();
  // per-atom potentials and fields, written to `path` (src/pb_class.cpp:3732-5060)
  int pot_field(const std::string& path = "pot_field.dat");
  int pot_field_fast(const std::string& path = "pot_field.dat");
  // potential_map / eps_map output for map_type = vtu (src/poisson_boltzmann.cpp:319-351)
  int export_maps();
  // one node field (values in node order) on the context's mesh to <basename>_0000.vtu
  int write_vtu(const std::string& basename, const std::string& fieldname, const double* values);
  // Whole path in the reference's order; returns a pbgpu status.
  int run_gpu_path();

  pbgpu_model model() const;
  pbgpu_mesh mesh_view() const;
  pbgpu_rays rays_view(int axis) const;

 private:
  std::vector<uint8_t> corner_inside_z(const std::vector<uint8_t>& hmask);
  int check(int status);
};

}  // namespace pbh
