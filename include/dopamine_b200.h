/*
 * dopamine_b200 — C ABI of the sm_100a RK3W fractional-step hot path.
 *
 * Two groups of entry points:
 *
 *  1. fvm_petsc_*  — the pressure-solve seam the reference already has.  Same symbol names,
 *     argument order and meaning as src/solver/pressure_backend_petsc.c (declared for Fortran in
 *     src/solver/mod_pressure_solver.f90:23-74), implemented here with device-resident Krylov
 *     solves instead of PETSc/hypre: Jacobi-preconditioned conjugate gradients ("jacobi") or
 *     flexible CG preconditioned by an aggregation-multigrid V-cycle ("boomeramg" / "gamg", the
 *     reference's default selection).  A Fortran host that links this library instead of
 *     pressure_backend_petsc.c needs no source change.
 *
 *  2. dpm_*        — the explicit part of the time step plus the whole-step driver, mirroring the
 *     FVSolver interface (src/solver/mod_fv_solver.f90:270-285: init, advance, project_once,
 *     compute_dt, to_device, sync_host, state_is_finite) and the per-operator Fortran
 *     subroutines, so that one operator at a time can be swapped.
 *
 * Conventions: plain C types only; all arrays are host pointers unless a name says "_dev";
 * cell vectors use the reference's Fortran layout (U(3,n): component fastest; grad(3,3,n):
 * grad(i,j,c) = dU_j/dx_i, i fastest).  Indices are 0-based in dpm_* calls; fvm_petsc_* keeps
 * the reference's 1-based indices.  Every call returns 0 on success or a negative status;
 * nothing throws and nothing calls exit().  One host thread per handle; calls are ordered on
 * the handle's CUDA stream.
 */
#ifndef DOPAMINE_B200_H
#define DOPAMINE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------------------------- */
/* Status codes                                                                              */
/* ---------------------------------------------------------------------------------------- */
#define DPM_OK 0
#define DPM_ERR_ARG (-1)
#define DPM_ERR_CUDA (-2)
#define DPM_ERR_MESH (-3)
#define DPM_ERR_NOT_FINITE (-4)
#define DPM_ERR_DT_COLLAPSE (-5)
#define DPM_ERR_UNSUPPORTED (-6)
#define DPM_ERR_BARRIER_TIMEOUT (-7)  /* a grid-wide wait of a Krylov kernel ran out (see
                                         dpm_set_barrier_spin_limit); the kernel returned and
                                         the handle stays usable                               */
/* Krylov failure after the fallback retry: -(1000 + reason), reason < 0 as in PETSc. */

/* Advection schemes (src/mod_parameters.f90:54-60). */
#define DPM_SCHEME_VANLEER_TVD 1
#define DPM_SCHEME_KOREN_TVD 2
#define DPM_SCHEME_CDS 3
#define DPM_SCHEME_KEP 4
#define DPM_SCHEME_QUICK 5

/* SGS closures (src/solver/mod_fv_solver.f90:1258-1278). */
#define DPM_SGS_NONE 0
#define DPM_SGS_VREMAN 1
#define DPM_SGS_SMAGORINSKY 2
#define DPM_SGS_AMD 3

/* Wall models (src/abl/mod_abl_types.f90 WM_*): log law (Reichardt) or none. */
#define DPM_WM_LOGLAW 0
#define DPM_WM_NONE 1
#define DPM_WM_MOST 2       /* Monin-Obukhov surface layer (src/abl/mod_abl_wall.f90)      */

/* Pressure-solve forms. */
#define DPM_PSOLVER_JACOBI_PCG 0
#define DPM_PSOLVER_TWOLEVEL_FCG 1
#define DPM_PSOLVER_MULTILEVEL_FCG 2  /* FCG + FP32 aggregation-multigrid V-cycle (no reference counterpart) */
#define DPM_PSOLVER_AUTO 3  /* the two-level form when the mesh fits it (<= 4096 cells per SM), else the multilevel form */
#define DPM_GRAD_LEAST_SQUARES 0
#define DPM_GRAD_GREEN_GAUSS 1
#define DPM_CELL_PROJECTION_LS 0
#define DPM_CELL_PROJECTION_EXACT 1
#define DPM_FORM_FP64 0     /* FP64 Krylov iterations                                    */
#define DPM_FORM_MIXED 1    /* with DPM_PSOLVER_TWOLEVEL_FCG: inner iterations on an FP32 copy of
                               the operator and an FP32 preconditioned vector, inside an FP64
                               defect correction (each inner solve ends at 1e-5 of its FP64
                               initial residual; the outer loop stops on the FP64 residual)   */

/* Raw mesh, as a gmsh v4 file holds it (src/mesh/mod_gmsh_reader.f90:build_mesh_from_gmsh). */
typedef struct dpm_raw_mesh {
  int64_t n_nodes;
  const double* xyz;          /* [n_nodes][3]                                                */
  int64_t n_cells;
  const int* cell_type;       /* gmsh codes: 4 tet, 5 hex, 6 prism, 7 pyramid                */
  const int64_t* cell_off;    /* [n_cells+1]                                                 */
  const int* cell_nodes;      /* 0-based node ids, gmsh local ordering                       */
  int64_t n_bfaces;
  const int64_t* bface_off;   /* [n_bfaces+1]                                                */
  const int* bface_nodes;
  const int* bface_patch;     /* [n_bfaces] patch index 0..n_patches-1                       */
  int n_patches;
} dpm_raw_mesh_t;

/* Per-patch boundary configuration (src/bc/mod_bc.f90:BCConfig). */
typedef struct dpm_patch_cfg {
  int bc_id;                  /* BC_* id (src/mod_parameters.f90:41-51)                      */
  double U_val[3];            /* inlet / moving-wall velocity                                */
  double p_val;               /* outlet pressure                                             */
  double T_val;               /* fixed temperature                                           */
  int scalar_mode[4];         /* per passive scalar: 0 zero gradient, 1 Dirichlet (value),    */
  double scalar_value[4];     /* 2 Neumann (value = flux per area, constant in time)          */
  double abl_z0_m, abl_z0_h;  /* MOST roughness lengths of this patch; <= 0: the global
                               * abl_z0_m / abl_z0_h (src/abl/mod_abl_wall.f90:248-257)       */
} dpm_patch_cfg_t;

/* Solver parameters (src/solver/mod_fv_solver.f90:solver_params_t), numerics pinned as the
 * reference's regression inputs pin them. */
typedef struct dpm_params {
  double nu;                  /* molecular kinematic viscosity                               */
  double dt;                  /* requested time step (clamped to the CFL limit)              */
  double cfl_max;
  double p_tol;               /* Poisson relative tolerance                                  */
  int p_max_iter;             /* Krylov iteration cap of one solve; the solve uses at least
                               * 2000 (max(p_max_iter, 2000)) so that the Jacobi-PCG form is
                               * not cut off on large meshes, and a capped solve is retried from
                               * a zero guess with 4x the cap (pressure_backend_petsc.c:878-961) */
  int scheme;                 /* DPM_SCHEME_* for momentum                                   */
  int sgs_model;              /* DPM_SGS_*                                                   */
  int wall_model;             /* DPM_WM_*                                                    */
  int n_nonortho_corr;        /* Jasak correctors per stage (>= 1)                           */
  int rhie_chow_dual;
  int nonortho_check;
  int use_rotational_projection;
  int adapt_dt;
  double pressure_min_cos_theta;
  double f_const[3];          /* constant body force                                         */
  double g[3];                /* gravity, Boussinesq only                                    */
  int boussinesq;
  double beta, T_ref, alpha_T, Pr_t;
  int temperature_scheme;
  int n_scalars;              /* passive scalars, <= 4                                       */
  int scalar_scheme;
  double scalar_diffusivity[4];
  double scalar_pr_t[4];
  double c_amd;
  int amd_wall_gradient;
  double wall_model_height, wall_model_filter_time, wall_model_filter_tf_fac;
  int form;                   /* DPM_FORM_*                                                  */
  /* Pressure solver (no counterpart in the reference's namelists, which select PETSc options):
   * DPM_PSOLVER_JACOBI_PCG mirrors `-pc_type jacobi`; DPM_PSOLVER_TWOLEVEL_FCG is flexible CG
   * with a part-local Chebyshev smoother of degree p_smooth_degree on the interval
   * [p_smooth_lmin, p_smooth_lmax] of D^-1 A plus a one-value-per-part coarse correction.
   * Zero / non-positive smoother settings select the defaults (7, 0.05, 2.0). */
  int p_solver;
  int p_smooth_degree;
  double p_smooth_lmin, p_smooth_lmax;
  /* MOST wall model (src/abl/mod_abl_types.f90:ABLConfig): roughness lengths, surface
   * temperature, initial Obukhov length (0 = neutral) and whether its domain mean is updated. */
  double abl_z0_m, abl_z0_h, abl_T_surface, abl_L_obukhov;
  int abl_compute_L;
  /* DPM_PSOLVER_MULTILEVEL_FCG: Chebyshev steps per smoothing (0: 3), over-correction of the
   * coarse correction (0: 1.6), pairwise-aggregation passes per level (0: 3; at most 3, as an
   * aggregate of up to 3^passes rows must fit the 32 lanes of the restriction). */
  int p_ml_degree;
  double p_ml_overcorrect;
  int p_ml_passes;
  /* Cell gradients (src/solver/mod_fv_solver.f90:85-86 gradient_scheme, gg_iterations):
   * DPM_GRAD_LEAST_SQUARES (default) or DPM_GRAD_GREEN_GAUSS with gg_iterations sweeps (the
   * sweeps after the first add the eps.grad skewness correction; 0 means the reference's 2). */
  int gradient_scheme;
  int gg_iterations;
  /* Stall guard of the flexible-CG forms: when ||r|| is above p_stall_ratio times its value
   * p_stall_window iterations earlier, the solve is handed to plain Jacobi-PCG from its current
   * iterate (dpm_stats_t.p_fallbacks).  Zero / non-positive: 50 iterations, ratio 0.9. */
  int p_stall_window;
  double p_stall_ratio;
  /* DPM_PSOLVER_MULTILEVEL_FCG: storage of the smoother's D^-1-scaled off-diagonal entries, 16
   * (binary16, with a per-row diagonal term that keeps each stored row's sum exact) or 32 (FP32);
   * 0: 32. */
  int p_ml_value_bits;
  /* Cell velocity after the face-flux projection (src/solver/mod_fv_solver.f90:91-92,
   * src/io/mod_input_parser.f90:200-201, 305-306): DPM_CELL_PROJECTION_LS reconstructs it from the
   * pressure gradient; DPM_CELL_PROJECTION_EXACT (the reference's default) projects it
   * V-orthogonally onto zero divergence of the interpolated face flux
   * (src/numerics/mod_cell_projection.f90), by flexible CG preconditioned with a pressure solve
   * to relative tolerance 0.05, stopping when the last step's velocity energy is below
   * cell_projection_tol^2 times the total (<= 0: 0.1; floored at 1e-8 as the reference's parser
   * floors it). */
  int cell_projection;
  double cell_projection_tol;
  /* Body forces besides f_const (src/solver/mod_fv_solver.f90:45-58, :959-983, :1662-1699):
   * constant_mass_flux_forcing replaces f_const by (U_bulk_target - <U>) / dt, recomputed at the
   * start of every step from the volume-mean velocity; use_harmonic_forcing adds
   * forcing_amp cos(forcing_omega t + forcing_phase) along forcing_dir (x when it is zero), t the
   * stage time; use_rotation adds the Coriolis term -2 omega_rot x U. */
  int constant_mass_flux_forcing;
  double U_bulk_target[3];
  int use_harmonic_forcing;
  double forcing_amp, forcing_omega, forcing_phase, forcing_dir[3];
  int use_rotation;
  double omega_rot[3];
  /* Davies nudging of U (and T) towards the profiles given by dpm_set_nudging_profiles
   * (src/abl/mod_abl_weather.f90:233-366): relaxation rate 1/nudging_tau, clamped at 0.5/dt,
   * in cells whose centroid height is at least nudging_z_start, ramped linearly to full strength
   * at nudging_z_full (no ramp when that is not above z_start); the vertical velocity is left
   * alone when nudging_horizontal_only (the reference's default). */
  int use_nudging;
  double nudging_tau, nudging_z_start, nudging_z_full;
  int nudging_horizontal_only;
  /* ABL inlet (BC_ABL_INLET patches; src/bc/mod_bc.f90:352-372, :557-562, src/abl/mod_abl_profiles.f90):
   * the neutral log-law mean U(z) = (u_star / kappa) ln(z / z0_m) along the wind direction
   * (meteorological degrees), u_star = kappa u_ref / ln(z_ref / z0_m), abl_z0_m the roughness; the
   * temperature there follows the log law from abl_T_surface towards abl_T_ref at z_ref with
   * abl_z0_h.  With use_sem the synthetic-eddy fluctuation is added (src/abl/mod_sem_inflow.f90):
   * sem_type DPM_SEM_DFSEM (divergence-free eddies, the reference's default) or DPM_SEM_JARRIN,
   * sem_n_eddies eddies of scale sem_sigma (<= 0: a tenth of the smaller inlet span), seed
   * sem_seed (0: the built-in one); target stresses from Panofsky-Dutton (sem_Iu_ref <= 0) or an
   * intensity law (sem_Iu_ref, sem_Iv_ratio, sem_Iw_ratio, sem_rho_uw); sem_mean_law
   * DPM_SEM_MEAN_LOG or DPM_SEM_MEAN_POWER (exponent sem_alpha). */
  double abl_u_ref, abl_z_ref, abl_T_ref, abl_wind_dir_deg;
  int use_sem, sem_type, sem_n_eddies, sem_seed, sem_mean_law;
  double sem_sigma, sem_alpha, sem_Iu_ref, sem_Iv_ratio, sem_Iw_ratio, sem_rho_uw;
  /* Mesh and static-operator set-up of dpm_create (mod_gmsh_reader.f90:build_faces_from_cells,
   * mod_mesh.f90:437-756, 1336-1461, mod_pressure_solver.f90:100-452): 0 = on the device (face
   * matching by radix sort, per-cell geometry, LS stencil and operators one thread per cell),
   * 1 = the host C++ builder.  Both give the same values; see dpm_setup_compare. */
  int host_setup;
} dpm_params_t;
#define DPM_SEM_DFSEM 0
#define DPM_SEM_JARRIN 1
#define DPM_SEM_MEAN_LOG 0
#define DPM_SEM_MEAN_POWER 1

/* Per-step integral statistics (src/stats/mod_stats.f90:compute_stats_sums and
 * src/solver/mod_fv_solver.f90:solver_divergence_metrics). */
typedef struct dpm_stats {
  double time, E, eps, Umax, Ub, tauw_mean, nu_sgs_mean;
  double max_abs_divU, volavg_abs_divU;
  double dt_used;
  int p_solves, p_iters;
  double p_resid_max;
  int p_fallbacks;            /* pressure solves handed from flexible CG to plain PCG (total)   */
  int p_solver_used;          /* DPM_PSOLVER_* of the pressure solve in use (never AUTO)      */
  double p_bytes_per_iteration;  /* algorithmic bytes one Krylov iteration of that solve moves
                                    (each array read or written once per pass): the roofline
                                    numerator of the pressure solve                           */
  int cp_iters;               /* DPM_CELL_PROJECTION_EXACT: outer iterations of the last step's
                                 cell projections (summed over its stages)                    */
  int cp_precond_iters;       /* and the Krylov iterations of their preconditioning solves      */
  double max_abs_divU_cell, volavg_abs_divU_cell;  /* divergence of the gc-interpolated cell
                                 velocity (src/solver/mod_fv_solver.f90:3582-3607), a different
                                 operator from the projected face flux's, not zeroed by it        */
} dpm_stats_t;

/* Outcome of dpm_learn_train. */
typedef struct dpm_learn_report {
  int samples, val_solves;    /* training samples; held-out solves used to set gamma            */
  double loss_initial, loss_final;  /* A-angle loss over the samples before / after training    */
  float gamma;                /* scale of the learned term kept (0: the term is switched off)   */
  int its_val_base, its_val_learned;  /* held-out iterations with gamma = 0 and with gamma      */
  double train_ms;
} dpm_learn_report_t;

/* ---------------------------------------------------------------------------------------- */
/* 1. Pressure-solve seam (src/solver/pressure_backend_petsc.c)                              */
/* ---------------------------------------------------------------------------------------- */
/* src/solver/mod_pressure_solver.f90:25 — 1 when the backend can be used. */
int fvm_petsc_backend_available(void);
/* src/solver/mod_pressure_solver.f90:29 — creates the CUDA context and stream. */
int fvm_petsc_backend_initialize(void);
/* src/solver/mod_pressure_solver.f90:33 — releases the cached operator and device memory. */
int fvm_petsc_backend_finalize(void);
/* src/solver/mod_pressure_solver.f90:37 — "boomeramg" / "gamg" select flexible CG with this
 * library's FP32 aggregation-multigrid V-cycle (an algebraic multigrid, as hypre's BoomerAMG is
 * in the reference); "jacobi" selects the Jacobi PCG, which is also what runs before any
 * selection. */
void fvm_petsc_set_pressure_solver(const char* solver_name);
/* src/solver/mod_pressure_solver.f90:42 — 1: rhs/solution may be device pointers. */
int fvm_petsc_device_io_supported(void);
/* src/solver/mod_pressure_solver.f90:47 */
void fvm_petsc_set_io_on_device(int on);
/* src/solver/mod_pressure_solver.f90:52 — PETSc option strings; "-pc_type jacobi",
 * "-ksp_max_it N", "-ksp_rtol X" are honoured, others ignored. */
void fvm_petsc_insert_option(const char* opt);
/* src/solver/mod_device.f90:119-126 — device binding of the calling rank. */
void fvm_petsc_set_device_local_rank(int local_rank);
/* src/solver/pressure_backend_petsc.c:648-668 (Fortran interface mod_pressure_solver.f90:60-73).
 * Solves A x = rhs, A = diag - sum_f coeff_f (off-diagonal), with conjugate gradients on the
 * unpreconditioned residual norm, ||r|| <= max(rtol ||b||, atol), nonzero initial guess
 * (solution on entry), constant null space when no Dirichlet rows exist.  Indices 1-based.
 * As in the reference: non-finite entries of rhs and of the initial guess are zeroed; a failed
 * solve is retried from a zero guess with Jacobi PCG and 4x the cap, and a DIVERGED_ITS retry
 * whose residual is below 1e4 rtol or 1e3 atol is accepted; otherwise -(1000 + reason).  The cap
 * is max(max_iterations, 2000) unless "-ksp_max_it N" was inserted, which sets it to N. */
int fvm_petsc_solve_pressure(int n_cells_local, int n_cells_global, int n_faces,
                             const int* local_to_global, const int* face_owner,
                             const int* face_neighbor_local, const int* face_neighbor_global,
                             const int* skip_face, const double* diagonal, const double* rhs,
                             const double* face_coeff, int reference_cell, int max_iterations,
                             double rtol, double atol, const int* dirichlet_rows,
                             const double* dirichlet_values, int n_dirichlet_rows,
                             double* solution, int* iteration_count, double* residual_norm);

/* Mesh ingestion: gmsh v4.1 ASCII files (src/mesh/mod_gmsh_reader.f90:gmsh_read).  Volume
 * elements (first-order tets, hexes, prisms, pyramids; 10-node tets and 20-node hexes by their
 * corner nodes) become cells in file order, triangles and quads become boundary faces, and the
 * 2-D physical groups that hold faces become the patches, in $PhysicalNames order (a file without
 * physical names gets one patch, "boundary").  dpm_gmsh_read returns DPM_ERR_ARG when the file
 * cannot be opened and DPM_ERR_MESH for what the reference refuses (binary or pre-4 files, other
 * element types, a surface element outside every 2-D group), with the reason in errbuf.  The
 * arrays of dpm_gmsh_fill are dpm_raw_mesh_t's, sized by dpm_gmsh_sizes. */
typedef struct dpm_gmsh dpm_gmsh_t;
int dpm_gmsh_read(const char* path, dpm_gmsh_t** out, char* errbuf, int errlen);
int dpm_gmsh_sizes(const dpm_gmsh_t* h, int64_t* n_nodes, int64_t* n_cells, int64_t* n_cell_nodes,
                   int64_t* n_bfaces, int64_t* n_bface_nodes, int* n_patches);
int dpm_gmsh_fill(const dpm_gmsh_t* h, double* xyz, int* cell_type, int64_t* cell_off, int* cell_nodes,
                  int64_t* bface_off, int* bface_nodes, int* bface_patch);
const char* dpm_gmsh_patch_name(const dpm_gmsh_t* h, int k);
int dpm_gmsh_free(dpm_gmsh_t* h);
/* Writes a raw mesh as a gmsh v4.1 ASCII file that dpm_gmsh_read reads back to the same cells,
 * faces and patches: one 2-D physical group per patch (tags 1..n_patches), one 3-D group. */
int dpm_gmsh_write(const char* path, const dpm_raw_mesh_t* mesh, const char* const* patch_names);

/* Mesh ingestion: OpenFOAM polyMesh directories (src/mesh/mod_foam_reader.f90:foam_read): points,
 * faces (faceList or faceCompactList), owner, neighbour and boundary, ASCII or binary (byte order,
 * label and scalar sizes from the header's arch entry).  The arrays of dpm_foam_fill are
 * dpm_poly_mesh_t's, sized by dpm_foam_sizes; each patch's name and OpenFOAM type are kept for
 * the caller's choice of dpm_patch_cfg_t.  DPM_ERR_ARG when a file cannot be opened,
 * DPM_ERR_MESH when one is malformed, with the reason in errbuf. */
typedef struct dpm_foam dpm_foam_t;
int dpm_foam_read(const char* polymesh_dir, dpm_foam_t** out, char* errbuf, int errlen);
int dpm_foam_sizes(const dpm_foam_t* h, int64_t* n_points, int64_t* n_faces, int64_t* n_face_nodes,
                   int64_t* n_int_faces, int* n_patches);
int dpm_foam_fill(const dpm_foam_t* h, double* xyz, int64_t* face_off, int* face_nodes, int* owner,
                  int* neighbour, int64_t* patch_start, int64_t* patch_nfaces);
const char* dpm_foam_patch_name(const dpm_foam_t* h, int k);
const char* dpm_foam_patch_type(const dpm_foam_t* h, int k);
int dpm_foam_free(dpm_foam_t* h);

/* ---------------------------------------------------------------------------------------- */
/* 2. Whole-step solver handle (src/solver/mod_fv_solver.f90 FVSolver)                       */
/* ---------------------------------------------------------------------------------------- */
typedef struct dpm_solver dpm_solver_t;

/* Mesh set-up and solver_init (mod_fv_solver.f90:302-508): builds geometry, periodic pairs,
 * LS stencils and the static projection operators on the device, where they stay (host_setup =
 * 1: on the host, then uploaded; the same values), and the pressure solver's hierarchy. */
int dpm_create(const dpm_raw_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
               int device, dpm_solver_t** out);
/* Face-based (polyhedral) mesh, as an OpenFOAM polyMesh holds it: faces in the file's order
 * (internal faces first with owner < neighbour, then each patch's faces), 0-based indices. */
typedef struct {
  int64_t n_points;
  const double* xyz;            /* [n_points][3] */
  int64_t n_faces;
  const int64_t* face_off;      /* [n_faces+1] into face_nodes */
  const int* face_nodes;
  const int* owner;             /* [n_faces] */
  int64_t n_int_faces;
  const int* neighbour;         /* [n_int_faces] */
  int n_patches;
  const int64_t* patch_start;   /* [n_patches] startFace (absolute face index) */
  const int64_t* patch_nfaces;  /* [n_patches] nFaces */
} dpm_poly_mesh_t;
/* dpm_create for a polyhedral mesh: the reference's OpenFOAM-path geometry (faces kept in the
 * file's order, polygon face geometry, cell moments from the faces; mod_mesh.f90:1336-1461), on
 * the device by default (host_setup = 1: on the host; the same values), then the same static
 * operators and time step as dpm_create.  Patches must cover the boundary faces, periodic
 * patches come in pairs (DPM_ERR_MESH otherwise). */
int dpm_create_poly(const dpm_poly_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                    int device, dpm_solver_t** out);
/* The polyhedral set-up alone, on the host (no device needed): cell centroids (3, n_cells) and
 * volumes of a dpm_poly_mesh_t with the given per-patch bc ids, or DPM_ERR_MESH with the
 * reason in errbuf (corrupt connectivity, owner >= neighbour, patches not covering the boundary,
 * an odd number of periodic patches). */
int dpm_poly_cell_geometry(const dpm_poly_mesh_t* mesh, const int* patch_bc, double* centroid, double* volume,
                           char* errbuf, int errlen);
int dpm_destroy(dpm_solver_t* s);
int dpm_n_cells(const dpm_solver_t* s, int64_t* n_cells, int64_t* n_faces, int64_t* n_bnd_faces);
/* solver_to_device (mod_fv_solver.f90:3286): U(3,nc), p(nc), T(nc) may be NULL. */
int dpm_upload_state(dpm_solver_t* s, const double* U, const double* p, const double* T);
/* solver_sync_host (mod_fv_solver.f90:3326): any output pointer may be NULL. */
int dpm_download_state(dpm_solver_t* s, double* U, double* p, double* T, double* nu_sgs);
/* Divergence-free face flux of the last projection (n_faces, mesh face order). */
int dpm_download_face_flux(dpm_solver_t* s, double* face_flux);
/* Velocity gradient of the last gradient pass, grad_U(3,3,nc). */
int dpm_download_gradient(dpm_solver_t* s, double* grad_U);
/* Cell centroids (3,nc) and volumes (nc) computed by the mesh set-up. */
int dpm_cell_geometry(const dpm_solver_t* s, double* centroid, double* volume);
/* solver_project_once (mod_fv_solver.f90:837-918). */
int dpm_project_once(dpm_solver_t* s, double dt);
/* solver_advance (mod_fv_solver.f90:920-958): CFL clamp of a fixed dt, RK3W, time += dt.
 * Status DPM_ERR_DT_COLLAPSE mirrors solver_compute_dt's stop. */
int dpm_advance(dpm_solver_t* s, double dt);
/* n steps in one call (dpm_advance n times); stats of the last step. */
int dpm_advance_n(dpm_solver_t* s, double dt, int n_steps);
int dpm_stats(dpm_solver_t* s, dpm_stats_t* out);
/* solver_state_is_finite (mod_fv_solver.f90:3925-3945): *ok = 1 when U and p are finite. */
int dpm_state_is_finite(dpm_solver_t* s, int* ok);
/* solver_compute_dt (mod_fv_solver.f90:3872-3899). */
int dpm_compute_dt(dpm_solver_t* s, double* dt);
int dpm_get_time(const dpm_solver_t* s, double* time);
int dpm_set_time(dpm_solver_t* s, double time);
/* Device time (CUDA events) of the last dpm_advance, in ms: whole step and Poisson solves. */
int dpm_last_timing(const dpm_solver_t* s, double* step_ms, double* poisson_ms);
/* Kernel launch count since the handle was created (own kernels only). */
int dpm_kernel_launches(const dpm_solver_t* s, int64_t* n);
/* Wall-clock milliseconds of the handle's set-up (12 values): ms[0] mesh (connectivity, geometry,
 * periodic pairs, LS stencil), ms[1] static operators, ms[2] upload and solver state, ms[3] total
 * of dpm_create; ms[4..10] the device builder's stages (raw upload, cells and face matching, faces
 * and cell lists, periodic pairing on the host, LS stencil, pressure operators, LS/cell operators),
 * zero with host_setup; ms[11] the pressure-solver hierarchy (part of ms[2]). */
int dpm_setup_times(const dpm_solver_t* s, double* ms);
/* Phase times of the two-level flexible-CG kernel (diagnostics).  us (may be NULL) receives what
 * was recorded since the last call: us[0..5] the mean microseconds per iteration that block 0
 * spends in the coarse values, the part-local smoother, publishing z plus the grid barrier,
 * w = A z with the sums, the reduce-and-gather, and the update; us[7] the iterations counted.
 * enable = 1 (re)starts the recording (one globaltimer read per phase in one thread), 0 stops it. */
int dpm_fcg_phase_times(dpm_solver_t* s, int enable, double* us);
/* Builds the mesh and static operators of one configuration with both builders and compares
 * them entry by entry.  mismatches[k] (k < DPM_SETUP_N_ARRAYS, named by dpm_setup_array_name)
 * counts the entries of array k whose bits differ, the SGS filter tensor excepted: its scale is a
 * cube root by pow(), whose last bit may differ between the device and host libraries, so
 * *G_max_rel gets its largest entry difference relative to the cell's |G_11|+|G_22|+|G_33|.  ms: host mesh, host operators, device
 * mesh, device operators. */
#define DPM_SETUP_N_ARRAYS 64
int dpm_setup_compare(const dpm_raw_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                      int device, int64_t* mismatches, double* G_max_rel, double* ms);
const char* dpm_setup_array_name(int k);
/* dpm_setup_compare for a face-based mesh (the builders behind dpm_create_poly). */
int dpm_setup_compare_poly(const dpm_poly_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                           int device, int64_t* mismatches, double* G_max_rel, double* ms);
/* The host builder alone (no device needed): builds the mesh and static operators on the host
 * threads and writes a 64-bit FNV-1a digest of each array's element count and bytes to
 * digests[k], k < *n_arrays, in dpm_setup_array_name order (digests holds DPM_SETUP_N_ARRAYS
 * entries), and the SGS filter tensor's to *G_digest.  A refused mesh returns DPM_ERR_MESH (or DPM_ERR_UNSUPPORTED for an assembled row
 * wider than 16 entries) with the host builder's reason in errbuf. */
int dpm_setup_host_digest(const dpm_raw_mesh_t* mesh, const dpm_patch_cfg_t* patches, const dpm_params_t* params,
                          uint64_t* digests, int* n_arrays, uint64_t* G_digest, char* errbuf, int errlen);
/* dpm_setup_host_digest for a face-based mesh. */
int dpm_setup_host_digest_poly(const dpm_poly_mesh_t* mesh, const dpm_patch_cfg_t* patches,
                               const dpm_params_t* params, uint64_t* digests, int* n_arrays, uint64_t* G_digest,
                               char* errbuf, int errlen);
/* Switches an existing handle's pressure solve: DPM_PSOLVER_JACOBI_PCG (always available) or
 * back to the flexible-CG form it was created with (that form's value, or DPM_PSOLVER_AUTO);
 * any other form returns DPM_ERR_UNSUPPORTED.  Lets the plain FP64 form be timed on the same
 * handle, mesh and state as the chosen form. */
int dpm_select_pressure_solver(dpm_solver_t* s, int p_solver);
/* Failure-detection hook: every grid-wide wait of this handle's Krylov kernels gives up after
 * `spins` polls of its arrival counter (0 restores the default, 2^26 polls, about a second).  A
 * wait that runs out sets the kernel's status word, every block returns, and the call that
 * launched it returns DPM_ERR_BARRIER_TIMEOUT; the handle stays usable.  Tests use a tiny value
 * to exercise that path without hanging or faulting the GPU. */
int dpm_set_barrier_spin_limit(dpm_solver_t* s, long long spins);

/* ---------------------------------------------------------------------------------------- */
/* 3. Per-operator entry points: same arguments as the Fortran subroutines, operating on the */
/*    handle's mesh.  Host arrays in, host arrays out, so a single operator can be compared   */
/*    or swapped in.                                                                          */
/* ---------------------------------------------------------------------------------------- */
/* ls_gradient_vector (src/numerics/mod_gradient.f90:425): grad_U(3,3,nc) from U(3,nc), U_bnd(3,nbnd). */
int dpm_ls_gradient_vector(dpm_solver_t* s, const double* U, const double* U_bnd, double* grad_U);
/* advection_rhs_vector (src/numerics/mod_advection.f90:679) with face_flux(n_faces). */
int dpm_advection_rhs_vector(dpm_solver_t* s, int scheme, const double* U, const double* U_bnd,
                             const double* face_flux, const double* grad_U, double* rhs);
/* viscous_rhs_vector (src/numerics/mod_viscous.f90:37). */
int dpm_viscous_rhs_vector(dpm_solver_t* s, const double* U, double nu, const double* nu_sgs,
                           const double* grad_U, const double* U_bnd, double* rhs);
/* vreman_sgs_viscosity / smagorinsky_sgs / amd_sgs_viscosity (src/sgs/): nu_sgs(nc). */
int dpm_sgs_viscosity(dpm_solver_t* s, int model, const double* U, const double* U_bnd,
                      const double* grad_U, double dt_stab, double* nu_sgs);
/* apply_wall_model_bc (src/sgs/mod_wall_model.f90:176): tau_w(3,nbnd). */
int dpm_wall_model(dpm_solver_t* s, const double* U, double nu, double* tau_w);
/* src/numerics/mod_advection.f90:56 advection_rhs_scalar (SoA fast paths :267-675): rhs[n] of a
 * scalar phi[n] with boundary values phi_bnd[n_bnd], face flux[n_faces] and grad_phi(3, n);
 * scheme CDS, QUICK, VANLEER_TVD or KOREN_TVD. */
int dpm_advection_rhs_scalar(dpm_solver_t* s, int scheme, const double* phi, const double* phi_bnd,
                             const double* face_flux, const double* grad_phi, double* rhs);
/* src/numerics/mod_viscous.f90:286 viscous_rhs_scalar: diffusivity alpha + nu_sgs / Pr_t. */
int dpm_viscous_rhs_scalar(dpm_solver_t* s, const double* phi, double alpha, const double* nu_sgs, double Pr_t,
                           const double* grad_phi, const double* phi_bnd, double* rhs);
/* The exact cell projection's operators (src/numerics/mod_cell_projection.f90), on the
 * handle's pressure faces and outlet faces whatever its cell_projection setting:
 * cp_divergence (:84): out(nc) = B u, the outflow divergence of the gc-interpolated flux of
 * u(3,nc); cp_adjoint_gradient (:129): v(3,nc) = V^-1 B^T chi; cp_project (:192): u <- u - V^-1 B^T
 * chi with (B V^-1 B^T) chi = B u + bconst(nc) by flexible CG, stopping on max|r| <= 1e-12 max|b|
 * or (after 2 iterations) a last step's velocity energy below tol^2 times the total, at most
 * max_it iterations (n_it: those taken); preconditioned by the handle's pressure solve to
 * rtol 0.05 as project_cells_exact does, or by z = r when identity_precond is non-zero (the form
 * of the reference's unit test). */
int dpm_cell_divergence(dpm_solver_t* s, const double* u, double* out);
int dpm_cell_adjoint_gradient(dpm_solver_t* s, const double* chi, double* v);
int dpm_cell_project(dpm_solver_t* s, double* u, const double* bconst, double tol, int max_it, int identity_precond,
                     int* n_it);
/* ---- output on the device (src/io/mod_checkpoint_io.f90, src/stats/mod_sampling.f90) ---- */
/* write_checkpoint / read_checkpoint (mod_checkpoint_io.f90:15-282): the reference's per-rank
 * file <checkpoint_dir>/processor0/checkpoint_<step, 8 digits>.bin as sequential unformatted
 * records (4-byte markers): header(8) = n_cells, n_scalars, 0, solver step, has scalars, 0, face
 * flux present, wall-model mask (1 tau_w, 2 q_w, 4 L, 8 wall-stress filter); time; global ids
 * 1..n_cells (int64); U(3,n); p; T; nu_sgs; C(n_scalars,n); U_face(n_faces); tau_w(3,n_bnd);
 * q_w; L; the filter state (3,n_bnd) - and the manifest <checkpoint_dir>/checkpoint_latest.
 * Fields leave the device one record at a time.  Reading (step < 0: the step the manifest
 * names) restores them, rejects another mesh or partition (DPM_ERR_MESH), skips a synthetic-eddy
 * record, then refreshes boundary values and gradients as solver_refresh_after_restart does and
 * rebuilds a missing face flux (solver_rebuild_face_flux). */
int dpm_write_checkpoint(dpm_solver_t* s, const char* checkpoint_dir, int step);
int dpm_read_checkpoint(dpm_solver_t* s, const char* checkpoint_dir, int step);
/* Sampling (mod_sampling.f90): dpm_sampling_set_points finds each point's owner, the cell with
 * the nearest centroid (cache_object_owners :520-562; owner_cell(n) 0-based, may be NULL);
 * dpm_sample_points fills payload(6, n) = U(3), p, T, nu_sgs at the points, the owner's value plus
 * its Green-Gauss gradient times the offset from its centroid (sample_points_local :493-518), with
 * the gradients taken as sampling_maybe_sample takes them (:171-177).  Only the payload crosses
 * PCIe; the NetCDF files are written by the host (dopamine_b200/sampling.py). */
int dpm_sampling_set_points(dpm_solver_t* s, int n_points, const double* xyz, int* owner_cell);
/* Reference profiles of the Davies nudging (mod_abl_weather.f90: NudgingData): n_times times
 * (ascending), n_levels heights (ascending), U_profile(3, n_levels, n_times) and
 * T_profile(n_levels, n_times) in the Fortran layout; bilinear in (time, height), clamped at the
 * ends (nudging_interpolate, interp_find_indices :289-366). */
int dpm_set_nudging_profiles(dpm_solver_t* s, int n_times, int n_levels, const double* times, const double* z_levels,
                             const double* U_profile, const double* T_profile);
/* Passive-scalar sources (src/mod_scalar.f90:ScalarSourceDef, scalar_source_value_at :133-183,
 * added to the scalar's right-hand side as add_scalar_source_terms does, mod_fv_solver.f90:1764-
 * 1784): each source adds magnitude x time scale (1, or cos(omega t + phase) when harmonic) to
 * every cell whose centroid it covers - a sphere (point, or a volume of shape sphere), the
 * neighbourhood of a segment (line), a slab about a plane optionally within a radius (surface,
 * or a volume of shape plane), a box, or the neighbourhood of tag points (obj).  scalar_id is
 * 1-based as in the namelist. */
typedef struct dpm_scalar_source {
  int enabled, scalar_id, src_kind, shape, time_mode;
  double magnitude, omega, phase;
  double center[3], p0[3], p1[3], normal[3];
  double half_thickness, radius, box_min[3], box_max[3], tag_radius;
  int n_tag_points;
  const double* tag_points;   /* (3, n_tag_points) */
} dpm_scalar_source_t;
#define DPM_SCALAR_SRC_POINT 1
#define DPM_SCALAR_SRC_LINE 2
#define DPM_SCALAR_SRC_SURFACE 3
#define DPM_SCALAR_SRC_VOLUME 4
#define DPM_SCALAR_SRC_OBJ 5
#define DPM_SCALAR_SHAPE_SPHERE 1
#define DPM_SCALAR_SHAPE_BOX 2
#define DPM_SCALAR_SHAPE_PLANE 3
#define DPM_SCALAR_TIME_CONSTANT 1
#define DPM_SCALAR_TIME_HARMONIC 2
int dpm_set_scalar_sources(dpm_solver_t* s, int n_sources, const dpm_scalar_source_t* sources);
int dpm_sample_points(dpm_solver_t* s, double* payload);
/* Passive scalars C(n_scalars, n) in the reference's Fortran layout (src/solver/mod_fv_solver.f90:326,
 * scalar index fastest); the temperature travels with dpm_upload_state / dpm_download_state. */
int dpm_upload_scalars(dpm_solver_t* s, const double* C);

/* ---- learned term of the two-level flexible-CG preconditioner (no counterpart in the
 * reference).  A one-ring message-passing network (BF16 weights on tensor cores, FP32
 * accumulate) maps static per-cell features of the pressure operator to omega_i >= 0, and the
 * preconditioned residual gains gamma * omega .* D^-1 (r - A Z y).  Requires
 * p_solver = DPM_PSOLVER_TWOLEVEL_FCG. */
/* Advances n_steps time steps recording (residual, preconditioned residual, D^-1-scaled
 * deflated residual, error) samples from the pressure solves (up to 32). */
int dpm_learn_collect(dpm_solver_t* s, int n_steps, int* n_samples);
/* Trains the network with Adam for `epochs` steps on all samples but those of the last recorded
 * solve, then sets gamma in {0, 0.5, 1} by the held-out solves' iterations (0 kept on ties). */
int dpm_learn_train(dpm_solver_t* s, int epochs, double lr, dpm_learn_report_t* report);
/* Overrides gamma (0 switches the learned term off). */
int dpm_learn_set_gamma(dpm_solver_t* s, double gamma);
/* sizes[7] = {n_cells, cells per part, local row width, global row width, training samples,
 * features per cell, parameters}. */
int dpm_learn_sizes(dpm_solver_t* s, int* sizes);
/* Copies the training problem to host buffers (renumbered order; any pointer may be NULL):
 * features [F][n], packed local rows [WL][n], operator [WA][n], samples R, Z, U, E [S][n],
 * current parameters [P]. */
int dpm_learn_export(dpm_solver_t* s, float* feat, unsigned* lpk, int* col, double* val, double* R, double* Z,
                     double* U, double* E, float* params);
/* Loss and parameter gradient over the training samples at `params` (NULL: the current ones);
 * the stored parameters are left unchanged. */
int dpm_learn_loss_grad(dpm_solver_t* s, const float* params, double* loss, float* grad);
int dpm_download_scalars(dpm_solver_t* s, double* C);

/* Aggregation hierarchy of DPM_PSOLVER_MULTILEVEL_FCG for an operator in padded ELL [width][n]
 * (host memory, no device needed): rows and non-zeros per level, coarsest last.  Returns the
 * number of levels (<= max_levels) or a negative code. */
int dpm_multilevel_hierarchy(int n, int width, const int* col, const double* val, int nullsp, int passes,
                             int* sizes, long long* nnz, int max_levels);
/* The same hierarchy, reduced to one 64-bit FNV-1a digest of every level's arrays (operator, scaled
 * rows in FP32 and binary16, diagonals, aggregates, members, eigenvalue estimate) and the coarsest
 * level's inverse.  Returns the number of levels or a negative code. */
int dpm_multilevel_digest(int n, int width, const int* col, const double* val, int nullsp, int passes,
                          unsigned long long* digest);

/* ---- allocation-free Jacobi-PCG solve --------------------------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device memory when they
 * solve (hosts whose device memory is owned by their own pool allocator, or latency-bound loops
 * where cudaMalloc's implicit synchronization is unacceptable).  All pointers are DEVICE
 * pointers owned by the caller: the operator in padded ELL form [row_width][n_cells] (col, val;
 * padding entries are (own row, 0.0)), the inverse diagonal, the right-hand side and the
 * solution x (used as the initial guess, overwritten).  Work vectors live in a fixed
 * file-scope device array of DPM_NOALLOC_MAX_CELLS cells (about 5.3 MB); larger systems or rows
 * wider than 16 return DPM_ERR_ARG.
 * First call per device: the CUDA runtime loads the library's device module lazily, so the
 * array and the solve kernels are created on a device by the first call there (which can fail
 * with DPM_ERR_CUDA if the device has no free memory) and are then held until the process
 * exits.  A call with max_iterations == 0 (sizes in range, array pointers may be NULL) does only
 * that set-up and returns 0: make it once per device before the host's pool reserves the
 * device's memory.
 * Stopping rule: the PETSc KSPCG test of fvm_petsc_solve_pressure (unpreconditioned norm,
 * ||r|| <= max(rtol ||b||, atol)); null_space != 0 projects the constant mode out of the
 * right-hand side.  Unlike fvm_petsc_solve_pressure there is no retry from a zero guess, no
 * 2000-iteration floor on max_iterations and no zeroing of non-finite entries: a solve that
 * reaches max_iterations returns -(1000 + KSP_DIVERGED_ITS) = -997.
 * Every call shares the array: calls that overlap on the GPU race and must be serialized by the
 * caller.  Blocks until the solve on `stream` (a cudaStream_t, NULL = legacy default) has
 * finished. */
#define DPM_NOALLOC_MAX_CELLS 131072
int dpm_pcg_solve_noalloc(int n_cells, int row_width, const int* col, const double* val,
                          const double* inv_diag, const double* rhs, double* x, double rtol, double atol,
                          int max_iterations, int null_space, void* stream, int* iteration_count,
                          double* residual_norm);

#ifdef __cplusplus
}
#endif
#endif /* DOPAMINE_B200_H */
