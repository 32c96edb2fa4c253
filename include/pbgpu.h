/*
 * pbgpu — C ABI of the B200 (sm_100a) assemble/solve/post-process path for the
 * linearized Poisson–Boltzmann equation on a 2:1-balanced octree with hanging
 * nodes (NextGenPB's box-method discretisation).
 *
 * The calls replace, one for one, the pb_class member functions on the
 * reference's hot path (reference paths relative to the NextGenPB tree):
 *
 *   pbgpu_create_markers      poisson_boltzmann::create_markers          src/pb_class.cpp:1793-1941
 *   pbgpu_create_density_map  poisson_boltzmann::create_density_map      src/pb_class.cpp:1944-2050
 *   pbgpu_assemble            poisson_boltzmann::assemple_system_matrix  src/pb_class.cpp:2053-2159
 *                             (bimpp bim3a_rhs / bim3a_laplacian_frac / bim3a_reaction_frac /
 *                              bim3a_dirichlet_bc and cube_fraction_intersection :2422-2532)
 *   pbgpu_solve               poisson_boltzmann::lis_compute_electric_potential   :2244-2329
 *                             poisson_boltzmann::mumps_compute_electric_potential :2200-2239
 *   pbgpu_phi_on_atoms        poisson_boltzmann::write_potential_on_atoms_fast    :2333-2417
 *   pbgpu_energy              poisson_boltzmann::energy / energy_fast              :2791-3338
 *   pbgpu_pot_field           poisson_boltzmann::pot_field / pot_field_fast        :3732-5060
 *
 * Conventions (all plain C types; no framework types cross this boundary):
 *   - Every call returns an int status (PBGPU_OK = 0).  On failure
 *     pbgpu_last_error(ctx) holds a one-line message.
 *   - Host arrays are owned by the caller and copied during the call; device
 *     memory is owned by the context.
 *   - A context is bound to one device and one CUDA stream.  Calls on one context
 *     must be serialised by the caller; distinct contexts are independent.
 *   - Node indices: 0 .. n_nodes-1 are independent nodes (the unknowns);
 *     n_nodes + h names hanging node h, whose value is the mean of its 2
 *     (edge-hanging) or 4 (face-hanging) independent parents.
 *   - Integer coordinates are in units of 2^-19 of the root octant (p4est's
 *     P8EST_ROOT_LEN), corner c of an octant at lower + bits(c) * size with
 *     x in bit 0, y in bit 1, z in bit 2.  Physical coordinates are
 *     lo[a] + (hi[a] - lo[a]) * (i * 2^-19), evaluated without fused multiply-add.
 */
#ifndef PBGPU_H
#define PBGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  PBGPU_OK = 0,
  PBGPU_ERR_ARG = 1,          /* bad argument / size */
  PBGPU_ERR_CUDA = 2,         /* CUDA runtime error */
  PBGPU_ERR_OOM = 3,          /* device allocation failed */
  PBGPU_ERR_STATE = 4,        /* call order: a prerequisite stage has not run */
  PBGPU_ERR_CAPACITY = 5,     /* a fixed-size structure overflowed (row too long, ...) */
  PBGPU_NOT_CONVERGED = 10,   /* Krylov iteration hit max_iter (result kept) */
  PBGPU_BREAKDOWN = 11,       /* Krylov breakdown (rho or omega ~ 0) or non-finite value */
  PBGPU_TIMEOUT = 12,         /* a bounded device-side wait gave up */
  PBGPU_REJECTED = 13         /* server: the request's device-memory estimate exceeds the whole HBM budget */
};

enum { PBGPU_CG = 0, PBGPU_BICGSTAB = 1, PBGPU_CGS = 2 };
enum { PBGPU_PRECOND_NONE = 0, PBGPU_PRECOND_JACOBI = 1, PBGPU_PRECOND_BLOCK_JACOBI = 2 };
enum { PBGPU_FP64 = 0, PBGPU_MIXED = 1 };

typedef struct pbgpu_ctx pbgpu_ctx;

/* Octree mesh (the tmesh_3d the reference builds with p4est). Octants in Morton order. */
typedef struct {
  int64_t n_oct;
  const int32_t* oct_xyz;    /* 3*n_oct: lower corner, integer coordinates */
  const int8_t* oct_level;   /* n_oct */
  const int32_t* oct_nodes;  /* 8*n_oct: node of each corner (>= n_nodes: hanging) */
  int64_t n_nodes;           /* independent nodes = unknowns */
  const int32_t* node_xyz;   /* 3*n_nodes */
  int64_t n_hang;
  const int8_t* hang_np;     /* n_hang: 2 or 4 */
  const int32_t* hang_par;   /* 4*n_hang: parents (ascending, -1 padded) */
  double lo[3], hi[3];       /* domain box: tree vertices 0 and 7 */
  double locate_tol;         /* p4esttol * box edge, atom search tolerance (src/pb_class.cpp:3636-3640) */
} pbgpu_mesh;

/* Crossings of the axis-aligned rays of one axis (NanoShaper's crossings_t).
 * Only rays with at least one crossing are listed; a missing ray has none.
 * key = (a << 20) | b with (a, b) the integer coordinates of the two transverse
 * axes in ascending axis order.  keys ascending. */
typedef struct {
  int64_t n_rays;
  const uint64_t* keys;      /* n_rays */
  const int64_t* ptr;        /* n_rays + 1 */
  const double* inters;      /* ptr[n_rays], ascending within a ray */
  const double* normals;     /* 3*ptr[n_rays], outward unit normals (x, y, z) */
} pbgpu_rays;

/* Model parameters ([model] and [surface] sections of options.prm). */
typedef struct {
  double e_in, e_out;        /* molecular / solvent dielectric constants */
  double ionic_strength;     /* mol/L */
  double T;                  /* K */
  int bc_type;               /* 1: phi = 0; 2: Coulomb/Debye sum; 3: analytic Born sphere */
  int stern_layer_surf;      /* 1: ion-free Stern layer of thickness stern_layer */
  double stern_layer;
  int calc_energy;           /* 0 none, 1 polarisation, 2 polarisation + ionic */
  int calc_coulombic;        /* 1: Coulomb energy */
} pbgpu_model;

typedef struct {
  int chunk;                 /* SELL slice height C (multiple of 32; 0 = default 32) */
  int sigma;                 /* sorting window in rows (1 or a multiple of chunk; 0 = default 2048) */
  int group;                 /* columns stored contiguously per row: 1, 2 or 4 (0 = default 4);
                                a thread loads `group` values with one load instruction;
                                with chunk 32, group 1 selects the SpMV that stages slices
                                through shared memory by bulk async copies */
} pbgpu_sell_opts;

typedef struct {
  int method;                /* PBGPU_CG, PBGPU_BICGSTAB or PBGPU_CGS */
  int precond;               /* PBGPU_PRECOND_* */
  int precision;             /* PBGPU_FP64 or PBGPU_MIXED */
  double tol;                /* stopping tolerance, see conv_cond */
  int max_iter;              /* inner iteration cap */
  double inner_tol;          /* PBGPU_MIXED: residual reduction per fp32 inner solve */
  int max_outer;             /* PBGPU_MIXED: refinement steps cap */
  int check_every;           /* iterations between host polls of the device convergence flag */
  int conv_cond;             /* LIS -conv_cond: 0 or 1 stop when ||r||_2 <= tol ||b||_2 (x0 = 0, so
                                r0 = b); 2 stop when ||r||_1 <= tol_w ||b||_1 + tol */
  double tol_w;              /* LIS -tol_w (conv_cond 2) */
} pbgpu_solver_opts;

typedef struct {
  int status;
  int iterations;            /* inner iterations (all refinement steps) */
  int outer;                 /* fp64 refinement steps (PBGPU_MIXED) */
  double rel_residual;       /* ||b - A x||_2 / ||b||_2 recomputed in fp64 at exit */
  double device_ms;          /* device time of the solve (CUDA events on the context stream) */
} pbgpu_solve_stats;

typedef struct {
  double energy_pol;         /* polarisation energy [kT] */
  double energy_react;       /* direct ionic energy [kT] (calc_energy == 2) */
  double energy_coul;        /* Coulomb energy [kT] (calc_coulombic == 1) */
  double charge_flux;        /* flux charge [e], Gauss-law check */
  double net_charge;         /* sum of atomic charges [e] */
  double sum;                /* energy_pol + energy_react + energy_coul */
} pbgpu_energy_out;

/* Per-atom columns of pbgpu_pot_field, in the order of the reference's
 * pot_field.dat (src/pb_class.cpp:4282-4300): potentials phi_c (Coulomb),
 * phi_p (polarisation), phi_i (ionic), then the field components of each. */
enum {
  PBGPU_PF_PHI_C = 0, PBGPU_PF_PHI_P = 1, PBGPU_PF_PHI_I = 2,
  PBGPU_PF_EX_C = 3, PBGPU_PF_EY_C = 4, PBGPU_PF_EZ_C = 5,
  PBGPU_PF_EX_P = 6, PBGPU_PF_EY_P = 7, PBGPU_PF_EZ_P = 8,
  PBGPU_PF_EX_I = 9, PBGPU_PF_EY_I = 10, PBGPU_PF_EZ_I = 11,
  PBGPU_PF_COLUMNS = 12
};

typedef struct {
  double energy_pol;         /* polarisation energy [kT] (0 when the options compute none) */
  double energy_react;       /* direct ionic energy [kT] (0 when the options compute none) */
  double energy_coul;        /* Coulomb energy over all atom pairs [kT] */
  double charge_flux;        /* sum of the flux elements / 4 pi [e] */
  int columns;               /* bit k set: column k is written to pot_field.dat under these options */
  int reserved;
} pbgpu_pot_field_out;

/* ---- context ---------------------------------------------------------- */
int pbgpu_ctx_create(pbgpu_ctx** out, int device, void* cuda_stream /* NULL: own stream */);
void pbgpu_ctx_destroy(pbgpu_ctx* ctx);
const char* pbgpu_last_error(const pbgpu_ctx* ctx);
int pbgpu_version(void);
/* The CUDA stream the context runs on (cudaStream_t), so a caller can order
 * its own work after the path's.  No counterpart in the reference. */
void* pbgpu_ctx_stream(const pbgpu_ctx* ctx);

/* ---- inputs ------------------------------------------------------------ */
/* Mesh of tmesh_3d after refine_surface (src/poisson_boltzmann.cpp:181-186). */
int pbgpu_set_mesh(pbgpu_ctx* ctx, const pbgpu_mesh* mesh);
/* Ray crossings of one axis (0, 1, 2): ray_cache_t::rays (include/raytracer.h:37-85). */
int pbgpu_set_rays(pbgpu_ctx* ctx, int axis, const pbgpu_rays* rays);
/* Atoms: pos_atoms / charge_atoms (include/pb_class.h:68-72). */
int pbgpu_set_atoms(pbgpu_ctx* ctx, int64_t n_atoms, const double* pos /* 3n */, const double* charge);
int pbgpu_set_model(pbgpu_ctx* ctx, const pbgpu_model* model);

/* ---- the path ------------------------------------------------------------ */
/* create_markers (src/pb_class.cpp:1793-1941): node in/out by z-ray parity,
 * epsilon_nodes / reaction_nodes, octant marker 0 / 0.5 / 1, border_quad. */
int pbgpu_create_markers(pbgpu_ctx* ctx);
/* create_density_map (src/pb_class.cpp:1944-2050): patch volumes, atom search,
 * trilinear charge projection to rho_fixed. */
int pbgpu_create_density_map(pbgpu_ctx* ctx);
/* assemple_system_matrix (src/pb_class.cpp:2053-2159): edge fractions of border
 * octants, box-method Laplacian with harmonic edge coefficients, kappa^2
 * reaction, hanging-node elimination, Dirichlet conditions -> SELL-C-sigma
 * matrix and right-hand side on the device.  opts may be NULL. */
int pbgpu_assemble(pbgpu_ctx* ctx, const pbgpu_sell_opts* opts);
/* lis_/mumps_compute_electric_potential: Krylov solve of the assembled system,
 * x0 = 0.  stats may be NULL. Returns PBGPU_NOT_CONVERGED / PBGPU_BREAKDOWN with
 * the last iterate kept. */
int pbgpu_solve(pbgpu_ctx* ctx, const pbgpu_solver_opts* opts, pbgpu_solve_stats* stats);
/* write_potential_on_atoms_fast (src/pb_class.cpp:2333-2417): phi at every atom
 * found in the mesh (trilinear in its octant); NaN for atoms outside. */
int pbgpu_phi_on_atoms(pbgpu_ctx* ctx, double* phi_atoms /* n_atoms */);
/* energy (fast = 0, src/pb_class.cpp:2791-3063) or energy_fast (fast = 1, :3066-3338). */
int pbgpu_energy(pbgpu_ctx* ctx, int fast, pbgpu_energy_out* out);
/* pot_field (fast = 0, src/pb_class.cpp:4390-5060) or pot_field_fast (fast = 1,
 * :3732-4388): the potential and field at every atom, split into Coulomb,
 * polarisation and ionic parts, for the model options calc_potential_terms and
 * calc_field_terms (0, 1 or 2; src/pb_class.cpp:947-948).  per_atom (may be
 * NULL) receives n_atoms rows of PBGPU_PF_COLUMNS doubles; columns that the
 * options do not compute are 0, and out->columns names those the reference
 * writes.  Every atom counts, charged or not, as in the reference. */
int pbgpu_pot_field(pbgpu_ctx* ctx, int fast, int calc_potential_term, int calc_field_term, double* per_atom,
                    pbgpu_pot_field_out* out);

/* Parse a LIS option string ("-i bicgstab -p jacobi -tol 1.e-8 ...") into
 * solver options, the way lis_solver_set_option is fed at src/pb_class.cpp:2313.
 * Unsupported LIS solvers map to the nearest supported one (cgs, bicg, bicgsafe,
 * gmres -> bicgstab; cr -> cg); ssor/ilu/sainv map to block Jacobi. */
int pbgpu_parse_lis_options(const char* options, pbgpu_solver_opts* out);
void pbgpu_default_solver_opts(pbgpu_solver_opts* out);

/* ---- read-back (parity checks and downstream output) -------------------- */
int pbgpu_get_node_coeffs(pbgpu_ctx* ctx, double* epsilon_nodes, double* reaction_nodes);
/* marker per octant (0, 0.5, 1); border octants ascending. */
int pbgpu_get_markers(pbgpu_ctx* ctx, double* marker, int64_t* n_border, int32_t* border /* may be NULL */);
/* 12 edge fractions per border octant, in border order (reference edge order). */
int pbgpu_get_fractions(pbgpu_ctx* ctx, double* frac);
int pbgpu_get_density(pbgpu_ctx* ctx, double* rho_fixed, double* vol_patch);
/* Assembled system in CSR, node order, columns ascending.  Call with col = NULL
 * to get nnz only. */
int pbgpu_get_system(pbgpu_ctx* ctx, int64_t* nnz, int64_t* row_ptr, int32_t* col, double* val, double* rhs);
int pbgpu_get_phi(pbgpu_ctx* ctx, double* phi);
/* Device time of the last call of each stage (ms): markers, density, assemble,
 * solve, phi_on_atoms, energy. */
int pbgpu_get_stage_ms(pbgpu_ctx* ctx, double ms[6]);

/* Measurement counters (no counterpart in the reference, which has no GPU
 * path): kernels launched by this context, and — while profiling is on — the
 * SpMV launches of the Krylov solves with their summed device time from CUDA
 * events recorded around each launch, and the algorithmic bytes one SpMV moves
 * (nnz * (value + index) + 2 * n * value). */
typedef struct {
  int64_t launches;
  int64_t spmv_launches;
  double spmv_ms;
  double spmv_bytes;
  int64_t krylov_iterations;
  int64_t energy_points;     /* distinct surface points of the last energy call */
  int64_t energy_pairs;      /* surface point x charged atom pairs evaluated */
  int64_t device_bytes;      /* device memory the context holds now */
} pbgpu_counters;
int pbgpu_set_profiling(pbgpu_ctx* ctx, int on);
/* Upper bound in seconds (0 .. 60, default 1) on each bounded device-side wait
 * of this context's kernels: the staged SpMV's waits for its bulk copies.  A
 * wait that reaches it ends the solve with PBGPU_TIMEOUT, after the kernel has
 * waited for its own copies in flight, and the context stays usable.  0 makes
 * every such wait give up at once: tests drive the timeout path with it.  No
 * counterpart in the reference. */
int pbgpu_set_wait_limit(pbgpu_ctx* ctx, double seconds);
int pbgpu_get_counters(pbgpu_ctx* ctx, pbgpu_counters* out);
int pbgpu_reset_counters(pbgpu_ctx* ctx);

/* Coulomb energy sum_{i<j} q_i q_j / r_ij / eps_in [kT] that allocates no
 * device memory.  It has no counterpart in the reference; it is the Coulomb
 * term of pbgpu_energy (energy_coul) for callers that cannot call cudaMalloc:
 * code running inside another library's enqueue or plugin callback, where
 * allocating is not permitted, or a process whose device memory is owned by a
 * pool allocator.  Needs no context.
 *   atoms       device pointer, n_atoms x 4 doubles (x, y, z, q); charges with
 *               |q| <= 1e-5 are left out, as in the reference
 *   e_in, T     molecular dielectric constant and temperature (eps_in is
 *               formed in the reference's units)
 *   out_energy  device pointer to one double, written on `cuda_stream`
 *               (NULL: the legacy default stream); read it after the stream
 *               has reached the call
 * Scratch lives in fixed device arrays of this library (4 MiB, held by every
 * GPU that loads it until the process exits): at most 131072 atoms
 * (PBGPU_ERR_CAPACITY beyond).  The first call on a device looks up the
 * arrays' device addresses (cudaGetSymbolAddress) with that device current;
 * make that first call before any stream capture.  The addresses are those of
 * the device's primary context and stay cached for the life of the process:
 * do not call it after cudaDeviceReset or from a non-primary context.  With
 * fewer than 2 atoms the energy (0) is written by a memset on the stream; the
 * call never waits for the stream.  All calls share the arrays: calls whose
 * work overlaps on the GPU race and must be serialised. */
int pbgpu_coulomb_energy_static(const double* atoms, int64_t n_atoms, double e_in, double T, double* out_energy,
                                void* cuda_stream);

/* ---- mesh construction on the GPU ----------------------------------------
 * refine_surface (src/pb_class.cpp:1468-1745), the node numbering with hanging
 * nodes (p8est_nodes / tmesh_3d) and the ray crossing tables of the three axes
 * (NanoShaper's ray cache, src/raytracer.cpp:379-467; here the van der Waals
 * union of the spheres), on the device.  Input: the initial octree that
 * init_tmesh* builds (Morton order), the domain box, the refinement levels and
 * the spheres (x, y, z, radius; radius <= 0 skipped).  The initial octree is
 * the caller's (n_oct > 0) or, with n_oct = 0, built here as init_tmesh*
 * builds it (src/pb_class.cpp:1290-1391): uniform at init_level, then
 * box_level passes that split every leaf below box_level with a non-hanging
 * corner inside [box_lo, box_hi], each followed by 2:1 balance.  Afterwards
 * the context holds the mesh and rays as after pbgpu_set_mesh /
 * pbgpu_set_rays, identical to the host build of the same problem. */
typedef struct {
  int64_t n_oct;             /* 0: build the initial octree from init_level / box_* */
  const int32_t* oct_xyz;    /* 3*n_oct */
  const int8_t* oct_level;   /* n_oct */
  double lo[3], hi[3];
  double locate_tol;
  int refine;                /* 1: run the surface refinement (loc_refinement == 1 or mesh_shape 4) */
  int minlevel, maxlevel, unilevel;
  int64_t n_spheres;
  const double* spheres;     /* 4*n_spheres */
  int init_level;            /* n_oct == 0: uniform level (outlevel, or unilevel for init_tmesh), 0..8 */
  int box_level;             /* n_oct == 0: scale_level of init_tmesh_with_refine_(box_)scale; 0: none */
  double box_lo[3], box_hi[3];  /* the box: l_c / r_c (mesh_shape 0, 4, refine_box) or l_box / r_box (3) */
} pbgpu_mesh_build;
int pbgpu_build_mesh(pbgpu_ctx* ctx, const pbgpu_mesh_build* build);
/* sizes of the context's mesh; n_rays: 3 entries (rays with crossings per axis) */
int pbgpu_get_mesh_counts(pbgpu_ctx* ctx, int64_t* n_oct, int64_t* n_nodes, int64_t* n_hang, int64_t* n_rays);
/* The context's mesh (set or built) copied to host arrays in the layout of
 * pbgpu_mesh, any of them NULL to skip, sized by pbgpu_get_mesh_counts;
 * hang_par takes 4 per hanging node.  box (may be NULL) receives lo[3] and the
 * extents hi - lo [3]: a corner at integer coordinate i sits at
 * lo + extent * (i * 2^-19).  No reference counterpart (tmesh accessors). */
int pbgpu_get_mesh(pbgpu_ctx* ctx, int32_t* oct_xyz, int8_t* oct_level, int32_t* oct_nodes, int32_t* node_xyz,
                   int8_t* hang_np, int32_t* hang_par, double* box);

/* ---- SELL layout autotuner ----------------------------------------------
 * No counterpart in the reference.  Assembles the context's system (markers
 * and density map must be current) in each candidate layout (chunk 32 / 64,
 * sigma 256 / 2048 / 16384, group 1 / 2 / 4, and for chunk 32 group 1 the
 * staged SpMV's chunk width 12 / 16), times the CG SpMV over `iterations`
 * Jacobi-CG iterations (0: 24) with CUDA events, and leaves the fastest layout
 * assembled.  The choice is remembered per matrix size class (log2 of the
 * row count) for later pbgpu_assemble(ctx, NULL) calls in this process.
 * best_cols is 0 unless the staged kernel won. */
int pbgpu_autotune(pbgpu_ctx* ctx, int iterations, pbgpu_sell_opts* best, int* best_cols, double* best_spmv_ms);

/* ---- many charge vectors on one system ----------------------------------
 * No counterpart in the reference (one charge set per run).  The context's
 * assembled matrix is shared by k <= 64 charge vectors (charges: k x n_atoms,
 * same atom positions): each gets its density map and right-hand side, the k
 * systems are solved by k Jacobi-CG recurrences sharing every SpMV (FP64,
 * relative 2-norm tolerance), and energies[j] / stats[j] are those of charge
 * vector j (either may be NULL).  Afterwards the context holds its own charges
 * again and the potential of the last vector. */
int pbgpu_solve_charges(pbgpu_ctx* ctx, int k, const double* charges, const pbgpu_solver_opts* opts, int fast,
                        pbgpu_energy_out* energies, pbgpu_solve_stats* stats);

/* ---- batches: many systems, one persistent launch ------------------------
 * No counterpart in the reference, which solves one system per process
 * (lis_compute_electric_potential, src/pb_class.cpp:2244-2329).  A batch holds
 * contexts whose systems are assembled (pbgpu_assemble with chunk 32 and
 * group 4) and solves them together: one persistent cooperative kernel per
 * chunk of check_every iterations advances every member (Jacobi CG, FP64 or
 * FP32-inner / FP64-refined, per-member scalars, convergence and
 * deterministic reductions).  After pbgpu_batch_solve every member context
 * holds its potential, so pbgpu_phi_on_atoms / pbgpu_energy run on it as
 * after pbgpu_solve.  A member context must not be used by other calls while
 * a batch call runs.  Results equal the member's own pbgpu_solve within the
 * solve tolerance. */
typedef struct pbgpu_batch pbgpu_batch;
int pbgpu_batch_create(pbgpu_batch** out, int device, void* cuda_stream);
void pbgpu_batch_destroy(pbgpu_batch* batch);
const char* pbgpu_batch_last_error(const pbgpu_batch* batch);
/* adds an assembled context; *slot receives its index (the lowest free one) */
int pbgpu_batch_add(pbgpu_batch* batch, pbgpu_ctx* ctx, int* slot);
int pbgpu_batch_remove(pbgpu_batch* batch, int slot);
int pbgpu_batch_size(const pbgpu_batch* batch);
/* opts: method PBGPU_CG, precond PBGPU_PRECOND_JACOBI, conv_cond 0 or 1;
 * stats: NULL or one entry per slot index (members only are written) */
int pbgpu_batch_solve(pbgpu_batch* batch, const pbgpu_solver_opts* opts, pbgpu_solve_stats* stats);
/* Incremental use (continuous batching): begin fixes the options and starts
 * every member afresh; each step call runs one persistent launch of up to
 * `steps` steps (a step is one inner CG iteration of every member in its inner
 * phase) and reports the members not yet done.  Members added after begin
 * start at the next step; a member reported done by pbgpu_batch_member has its
 * potential in its context and can be removed. */
int pbgpu_batch_begin(pbgpu_batch* batch, const pbgpu_solver_opts* opts);
int pbgpu_batch_step(pbgpu_batch* batch, int steps, int* n_active);
int pbgpu_batch_member(pbgpu_batch* batch, int slot, int* done, pbgpu_solve_stats* stats);
/* pbgpu_batch_step in two halves: launch returns once the persistent kernel
 * is queued (other contexts' work can be issued meanwhile); wait completes it.
 * Between them members may be added but not removed or queried. */
int pbgpu_batch_launch(pbgpu_batch* batch, int steps);
int pbgpu_batch_wait(pbgpu_batch* batch, int* n_active);
/* resident blocks per SM of the persistent kernel (0: as many as fit); fewer
 * leave room for other streams' kernels to run beside it */
int pbgpu_batch_set_blocks_per_sm(pbgpu_batch* batch, int blocks);
/* Upper bound in seconds (0 .. 60, default 2) on each wait of a member's CTAs
 * at the member's barrier inside the persistent kernel.  A wait that reaches
 * it makes every CTA of the launch return at its next barrier, and the call
 * returns PBGPU_TIMEOUT; the batch stays usable (the next begin or solve
 * restarts its members).  0 makes every such wait give up at once: tests
 * drive the timeout path with it. */
int pbgpu_batch_set_wait_limit(pbgpu_batch* batch, double seconds);

/* ---- server: continuous batching of PB solves ----------------------------
 * No counterpart in the reference.  Requests (one molecule each: mesh, rays,
 * atoms, model) are queued by pbgpu_server_submit; every
 * pbgpu_server_progress call admits queued requests FIFO while max_members and
 * the HBM budget allow (device bytes held by all contexts plus an estimate for
 * the request), builds their systems on their own contexts, advances all
 * member systems with one persistent multi-system launch, and returns the
 * requests that finished (energies, solve statistics, latency).  A request
 * whose estimate alone exceeds the budget can never be admitted: it leaves the
 * queue at once and comes back as a result with status PBGPU_REJECTED.  The
 * arrays a request points to must stay valid until its result is returned. */
typedef struct {
  const pbgpu_mesh* mesh;    /* the molecule's mesh, or NULL to build it from `build` */
  pbgpu_rays rays[3];        /* with `mesh`; ignored when the mesh is built */
  int64_t n_atoms;
  const double* pos;         /* 3 n_atoms */
  const double* charge;      /* n_atoms */
  const pbgpu_model* model;
  int64_t user_tag;
  const pbgpu_mesh_build* build;  /* used when mesh is NULL: the server runs pbgpu_build_mesh (surface
                                     refinement, nodes, hanging nodes, ray tables) on the request's
                                     context as the first step of serving it */
} pbgpu_request;

typedef struct {
  int64_t id;                /* from pbgpu_server_submit */
  int64_t user_tag;
  int status;
  pbgpu_energy_out energy;
  pbgpu_solve_stats stats;
  double latency_ms;         /* submit to completion (host wall clock) */
  double queue_ms;           /* submit to admission */
} pbgpu_result;

typedef struct {
  double hbm_budget_bytes;   /* device memory all server contexts may hold (default 160e9) */
  int max_members;           /* systems solved at once (default 64) */
  int steps_per_tick;        /* persistent-kernel steps per progress call (default 32) */
  int blocks_per_sm;         /* persistent kernel residency (default 2; 0: as many as fit) */
  pbgpu_solver_opts solver;  /* CG + Jacobi; PBGPU_MIXED by default (FP32 inner, FP64 refined) */
  int energy_fast;           /* 1: energy_fast, 0: energy */
  int admit_per_tick;        /* requests set up per progress call (default 16; 0: no cap) */
  int mode;                  /* 0: members advance together in the persistent multi-system kernel;
                                1: `workers` host threads each run whole requests on their own
                                context and stream, overlapping on the device */
  int workers;               /* host threads (default 8): mode 1 runs whole requests on them; mode 0
                                sets up admitted requests and computes energies on them */
} pbgpu_server_opts;

typedef struct pbgpu_server pbgpu_server;
void pbgpu_default_server_opts(pbgpu_server_opts* opts);
int pbgpu_server_create(pbgpu_server** out, int device, const pbgpu_server_opts* opts);
void pbgpu_server_destroy(pbgpu_server* server);
const char* pbgpu_server_last_error(const pbgpu_server* server);
int pbgpu_server_submit(pbgpu_server* server, const pbgpu_request* request, int64_t* id);
/* one tick; writes up to `cap` finished requests to out[0 .. *n_out) */
int pbgpu_server_progress(pbgpu_server* server, pbgpu_result* out, int cap, int* n_out);
int pbgpu_server_pending(const pbgpu_server* server, int* queued, int* running, int64_t* device_bytes);
/* Requests admitted, completed and rejected so far, and the kernels the
 * server's contexts and persistent batch have launched (any may be NULL). */
int pbgpu_server_stats(const pbgpu_server* server, int64_t* admitted, int64_t* completed, int64_t* rejected,
                       int64_t* launches);
/* device bytes the server plans for a request before it holds any; for a
 * request that carries a mesh build, from the initial octree and the number of
 * refinement levels above it (an upper bound of the refined mesh's size) */
int64_t pbgpu_request_bytes_estimate(const pbgpu_request* request);

#ifdef __cplusplus
}
#endif
#endif /* PBGPU_H */
