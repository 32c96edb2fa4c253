/*
 * CPU oracle for the PB assemble/solve/post-process path — TEST
 * INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference arm may load this library, and only as the checker
 * or the timed CPU baseline; the product path never calls it.
 *
 * It restates, in plain sequential-order C++, the reference's hot path on the
 * same inputs the GPU path takes (include/pbgpu.h structures):
 *   markers            src/pb_class.cpp:1793-1941 (+ is_in_ns_surf :769-805,
 *                      is_in_ns_surf_stern :1752-1790)
 *   edge fractions     cube_fraction_intersection :2422-2532
 *   density map        create_density_map :1944-2050, atom search :3633-3729
 *   assembly           assemple_system_matrix :2053-2159 (the bimpp operators
 *                      it calls are restated from their use in this file, see
 *                      pb_oracle.cpp), BCs :3531-3571
 *   Krylov solve       lis_compute_electric_potential :2244-2329 (CG and
 *                      BiCGStab with none / Jacobi / block-Jacobi
 *                      preconditioning), solved tight as MUMPS stand-in
 *   potential at atoms write_potential_on_atoms_fast :2333-2417
 *   energy             energy :2791-3063, energy_fast :3066-3338
 *   per-atom phi / E   pot_field :4390-5060, pot_field_fast :3732-4388
 *
 * PARITY UNPINNED: the reference cannot be built here (bimpp, p4est, LIS, MUMPS
 * and NanoShaper are absent) and ships no tests or golden outputs.  The oracle
 * is anchored instead on the analytic Born / Debye-Hueckel energy of a charged
 * sphere and on the Gauss-law flux check.
 */
#ifndef PB_ORACLE_H
#define PB_ORACLE_H

#include <stdint.h>

#include "../include/pbgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_state oracle_state;

oracle_state* oracle_create(const pbgpu_mesh* mesh, const pbgpu_rays* rays3, int64_t n_atoms, const double* pos,
                            const double* charge, const pbgpu_model* model);
void oracle_destroy(oracle_state* s);

int oracle_markers(oracle_state* s);
int oracle_density(oracle_state* s);
int oracle_assemble(oracle_state* s);
/* rows = 0: triplet assembly (emit, stable sort, sum); rows = 1: per-row
 * gather over node incidences (O(nnz) memory).  Both give identical sums;
 * oracle_assemble picks the row assembly above 2M octants. */
int oracle_assemble_mode(oracle_state* s, int rows);
/* method PBGPU_CG / PBGPU_BICGSTAB, Jacobi preconditioner, x0 = 0, stop on
 * ||b - A x||_2 <= tol ||b||_2 (recursive residual, checked against the true
 * residual at exit).  threads <= 0: all cores.  Returns iterations (<0 error). */
int oracle_solve(oracle_state* s, int method, double tol, int max_iter, int threads, double* rel_residual);
/* the same for method PBGPU_CG / _BICGSTAB / _CGS, preconditioner
 * PBGPU_PRECOND_NONE / _JACOBI / _BLOCK_JACOBI (blocks of 8 consecutive nodes,
 * inverses stored symmetrised in FP32) and LIS's conv_cond: 0 or 1 stop on
 * ||r||_2 <= tol ||b||_2, 2 on ||r||_1 <= tol_w ||b||_1 + tol */
int oracle_solve_ex(oracle_state* s, int method, int precond, int conv_cond, double tol, double tol_w, int max_iter,
                    int threads, double* rel_residual);
int oracle_phi_on_atoms(oracle_state* s, double* out);
int oracle_energy(oracle_state* s, int fast, pbgpu_energy_out* out);
/* pot_field (fast = 0) / pot_field_fast (fast = 1): per-atom rows of
 * PBGPU_PF_COLUMNS values (may be NULL), energies and the written columns */
int oracle_pot_field(oracle_state* s, int fast, int calc_potential_term, int calc_field_term, double* per_atom,
                     pbgpu_pot_field_out* out);

/* getters, same layouts as the pbgpu_get_* calls */
int oracle_get_node_coeffs(const oracle_state* s, double* eps, double* react);
int oracle_get_markers(const oracle_state* s, double* marker, int64_t* n_border, int32_t* border);
int oracle_get_fractions(const oracle_state* s, double* frac);
int oracle_get_density(const oracle_state* s, double* rho, double* vol_patch);
int oracle_get_system(const oracle_state* s, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val, double* rhs);
int oracle_get_phi(const oracle_state* s, double* phi);
/* install a potential (e.g. one computed elsewhere) for phi_on_atoms/energy */
int oracle_set_phi(oracle_state* s, const double* phi);
/* install a system (CSR, node order) in place of oracle_assemble's */
int oracle_set_system(oracle_state* s, int64_t n, const int64_t* row_ptr, const int32_t* col, const double* val,
                      const double* rhs);
/* y = A x with the assembled system (threads <= 0: all cores) */
int oracle_spmv(const oracle_state* s, const double* x, double* y, int threads);
/* Time `iters` Jacobi-CG iterations on the assembled system (CPU baseline). */
double oracle_time_cg_iterations(oracle_state* s, int iters, int threads);
/* the oracle's marching-cubes triangle table, 256 x 16 edge ids (-1 padded) */
int oracle_tri_table(int* out);

#ifdef __cplusplus
}
#endif
#endif
