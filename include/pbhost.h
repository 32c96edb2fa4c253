/*
 * pbhost — C API of the host side of the PB path: the poisson_boltzmann
 * mirror (options.prm parsing, PQR reading, domain box, octree construction
 * with surface refinement, surface ray tables) that feeds libpbgpu.
 *
 * It stands where the reference's driver and pb_class set-up stand
 * (src/poisson_boltzmann.cpp:58-188, src/pb_class.cpp:39-1745); the arrays it
 * exposes are exactly the inputs of pbgpu_set_mesh / pbgpu_set_rays /
 * pbgpu_set_atoms.  All pointers returned by the getters stay valid until the
 * next pbhost call that rebuilds the problem, or pbhost_destroy.
 */
#ifndef PBHOST_H
#define PBHOST_H

#include <stdint.h>

#include "pbgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pbhost pbhost;

typedef struct {
  int mesh_shape, unilevel, minlevel, maxlevel, outlevel, scale_level, loc_refinement;
  double scale, lo[3], hi[3], cc[3], l_c[3], r_c[3], l_cr[3], r_cr[3], pot_bc, locate_tol;
  int64_t n_oct, n_nodes, n_hang, n_atoms, n_rays[3];
  double net_charge;
} pbhost_info;

pbhost* pbhost_create(void);
void pbhost_destroy(pbhost* h);
const char* pbhost_last_error(const pbhost* h);

/* parse_options: options.prm file or text (same keys and defaults). */
int pbhost_load_options_file(pbhost* h, const char* path);
int pbhost_load_options_text(pbhost* h, const char* text);
/* Override one "section/key" option (e.g. "mesh/maxlevel", "7"). */
int pbhost_set_option(pbhost* h, const char* key, const char* value);

/* read_atoms_from_pqr + read_atoms_from_class (src/pb_class.cpp:1099-1180). */
int pbhost_read_pqr(pbhost* h, const char* path);
/* Atoms given directly (positions 3n, charges, radii), then the same <4-atom
 * dummy rule as the PQR reader. */
int pbhost_set_atoms(pbhost* h, int64_t n, const double* pos, const double* charge, const double* radius);

/* create_mesh + init_tmesh* + refine_surface + node/ray tables. */
int pbhost_build_problem(pbhost* h);
/* The domain and initial octree on the host, the surface refinement, nodes and
 * ray tables on the GPU (pbgpu_build_mesh) into ctx, which also receives the
 * atoms and the model; the host keeps no mesh (pbhost_get_mesh / _rays then
 * describe nothing). */
int pbhost_build_on_gpu(pbhost* h, pbgpu_ctx* ctx);
/* The host half of pbhost_build_on_gpu alone: the domain (create_mesh) and
 * the initial octree (init_tmesh*) as the input of pbgpu_build_mesh, for a
 * caller that builds the rest on a context of its own or hands it to the
 * server in a pbgpu_request.  on_gpu = 1 leaves the initial octree to
 * pbgpu_build_mesh (n_oct = 0 with its uniform level and box; what
 * pbhost_build_on_gpu does); on_gpu = 0 builds it here.  The arrays `out`
 * points to belong to the handle and stay valid until the next call or
 * pbhost_destroy. */
int pbhost_initial_octree(pbhost* h, int on_gpu, pbgpu_mesh_build* out);
/* One node field (values in node order, n_nodes) on the problem's mesh to
 * <basename>_0000.vtu in the layout of the reference's VTKWriter
 * (src/vtk_class.cpp:20-429): the host's mesh, or the GPU context's when the
 * mesh was built there. */
int pbhost_write_vtu(pbhost* h, const char* basename, const char* fieldname, const double* values);
/* Same with a caller-chosen domain (mesh_shape 2 box) and uniform/surface levels. */
int pbhost_get_info(const pbhost* h, pbhost_info* out);
int pbhost_get_mesh(const pbhost* h, pbgpu_mesh* out);
int pbhost_get_rays(const pbhost* h, int axis, pbgpu_rays* out);
int pbhost_get_atoms(const pbhost* h, double* pos, double* charge, double* radius);
int pbhost_get_model(const pbhost* h, pbgpu_model* out);
int pbhost_get_solver_opts(const pbhost* h, pbgpu_solver_opts* out);

/* The GPU path in the driver's order (markers .. energy) on a context owned by
 * this handle; energies and solve statistics returned. */
int pbhost_run_gpu(pbhost* h, pbgpu_energy_out* energy, pbgpu_solve_stats* stats);
pbgpu_ctx* pbhost_gpu_ctx(pbhost* h);

#ifdef __cplusplus
}
#endif
#endif /* PBHOST_H */
