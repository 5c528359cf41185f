/*
 * easyfsi_b200 C ABI -- the drop-in boundary of the B200 implementation of the
 * EasyFsi coupled-step hot path.
 *
 * Every entry point takes plain device pointers (CUDA global memory, C order
 * (nx, ny, nz) with k fastest, vector fields stored as (n, 3) and matrices as
 * (n, 3, 3) rows), plain sizes and a cudaStream_t passed as void*.  Every entry
 * point returns an int status (EFSI_OK on success); a failing status leaves
 * the message in efsi_last_error().  No entry point takes ownership of caller
 * memory.  Plans (efsi_fv_plan, efsi_mpm_plan, efsi_bin_plan) own their
 * derived tables and work buffers.
 *
 * Each declaration names the reference function it replaces as
 * file:line in lizhuoh9/EasyFsi (simulation_core/...).
 */
#ifndef EASYFSI_B200_H
#define EASYFSI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define EFSI_OK 0
#define EFSI_ERR_ARG 1
#define EFSI_ERR_CUDA 2
#define EFSI_ERR_STATE 3

typedef struct efsi_fv_plan efsi_fv_plan;
typedef struct efsi_mpm_plan efsi_mpm_plan;
typedef struct efsi_bin_plan efsi_bin_plan;
typedef struct efsi_ib_search_plan efsi_ib_search_plan;
typedef struct efsi_reach_plan efsi_reach_plan;

/* Last error message of the calling thread (never NULL). */
const char* efsi_last_error(void);
/* Library version string. */
const char* efsi_version(void);
/* Number of kernels this library has launched in the process so far. */
uint64_t efsi_kernel_launch_count(void);

/* Benchmark instrumentation (no counterpart in the reference): bracket every
 * launch of a kernel family with CUDA events on its stream and accumulate the
 * family's algorithmic bytes.  Families: 0 SpMV+direction, 1 level-0 smoother
 * sweeps, 2 CG update, 3 level-0 residual+restriction, 4 CG dots, 5 MPM P2G,
 * 6 predictor.  Enabling resets the family's record; reading synchronises. */
int efsi_kernel_timing_enable(int32_t family, int32_t enable);
int efsi_kernel_timing_read(int32_t family, int64_t* launches, double* total_ms, double* total_bytes);

/* Benchmark helper (no counterpart in the reference): launch one level-0
 * kernel family (0 SpMV+direction, 1 smoother sweep, 2 CG update, 3 residual +
 * restriction, 4 CG dots) `reps` times back to back on the plan's work buffers;
 * returns the mean CUDA-event time per launch and its algorithmic bytes. */
int efsi_fv_kernel_replay(efsi_fv_plan* plan, int32_t family, int32_t reps, double* avg_ms,
                          double* bytes_per_launch, void* stream);

/* Tile autotuner of the V-cycle (no counterpart in the reference): for every
 * level that launches its own kernels, times a unit of its work -- level 0:
 * the PCG's direction SpMV plus a whole V-cycle with the dots fused in; a
 * coarse level: its sweep + restriction -- under each candidate launch shape
 * (plane-marching kernels with 3, 1, 2, 4 or 6 blocks' worth of planes per
 * SM; on levels >= 1 also the tiled / per-cell kernels) and keeps the
 * fastest on the plan.  choice[l] is the blocks-per-SM multiple picked (0:
 * tiled / per-cell kernels, -1: level not tuned) and best_us[l] the time of
 * its unit, for l < max_levels.  Needs the masks; drops the plan's captured PCG graphs
 * (the next solve records the tuned launches; a step graph captured before
 * must be captured again). */
int efsi_fv_autotune(efsi_fv_plan* plan, int32_t reps, int32_t* choice, double* best_us, int32_t max_levels,
                     void* stream);

/* ------------------------------------------------------------------------ */
/* Fluid grid / multigrid hierarchy                                          */
/* ------------------------------------------------------------------------ */

/* One multigrid level: f32 device axis arrays exactly as the reference loads
 * them into cell_width_*_m / center_distance_*_m (fluid.py:1013-1024,
 * 1161-1199; coarse levels fluid.py:692-729). */
typedef struct efsi_level_desc {
  int32_t nx, ny, nz;
  const float* wx;
  const float* wy;
  const float* wz;
  const float* cdx;
  const float* cdy;
  const float* cdz;
} efsi_level_desc;

/* Builds the per-level f64 face-coefficient tables and allocates the solver
 * work vectors for the hierarchy (replaces the field allocation of
 * CartesianFluidSolver.__init__, fluid.py:736-1075). */
int efsi_fv_plan_create(const efsi_level_desc* levels, int32_t n_levels, int32_t uniform_grid, efsi_fv_plan** out);
int efsi_fv_plan_destroy(efsi_fv_plan* plan);

/* Rebuilds the per-cell stencil masks of every level from the obstacle, the
 * velocity-Dirichlet rows and the interface diagonal (the coarse part replaces
 * the obstacle / Dirichlet / interface-diagonal half of
 * _mg_restrict_residual_kernel, fluid.py:5310-5388).  vdir_active, vdir_weight
 * and iface_diag may be NULL (inactive). */
int efsi_fv_set_masks(efsi_fv_plan* plan, const int32_t* obstacle, const int32_t* vdir_active,
                      const float* vdir_weight, const double* iface_diag, void* stream);

/* fluid.py:3451-3486 _compute_divergence_kernel. velocity (n,3) f32 -> div f32. */
int efsi_compute_divergence(efsi_fv_plan* plan, const float* velocity, int32_t outlet, float* divergence,
                            void* stream);

/* fluid.py:5228-5243 _mg_prepare_level0_kernel: rhs = s (div - src) - iface_rhs (f64 out).
 * iface_rhs may be NULL. */
int efsi_mg_prepare_level0(efsi_fv_plan* plan, const float* divergence, const float* volume_source,
                           const double* iface_rhs, float rhs_scale, double* rhs, void* stream);

/* fluid.py:4312-4345 _fv_laplacian_apply_kernel (level 0, f64). */
int efsi_fv_apply(efsi_fv_plan* plan, const double* p, double* out, int32_t outlet, void* stream);

/* fluid.py:4280-4309 _fv_diagonal_kernel. */
int efsi_fv_diagonal(efsi_fv_plan* plan, double* diag, int32_t outlet, void* stream);

/* fluid.py:4503-4516 _apply_jacobi_preconditioner_kernel. */
int efsi_apply_jacobi_preconditioner(efsi_fv_plan* plan, const double* diag, const double* r, double* z,
                                     void* stream);

/* fluid.py:4534-4546 _weighted_dot_kernel: sum over fluid cells of a b V (f64,
 * deterministic order).  Synchronises the stream and writes the host result. */
int efsi_weighted_dot(efsi_fv_plan* plan, const double* a, const double* b, double* result_host, void* stream);

/* No counterpart in the reference: the same fluid-weighted dot (fluid =
 * obstacle == 0, V = wx[i] wy[j] wz[k]) with no plan and no allocation; its
 * reduction scratch is a static device array of the library, so at most
 * 268435456 cells (larger grids return EFSI_ERR_ARG) and calls on one device
 * must not overlap.  Each call clears the scratch's ticket on its stream
 * before the launch.  The first call on a device resolves that scratch (and
 * may load the module): make it before any stream capture.  The resolved
 * address is kept for the life of the process: do not use the library across
 * a cudaDeviceReset of a device it has used.  Writes the total to
 * result_device without synchronising. */
int efsi_weighted_dot_noalloc(int32_t nx, int32_t ny, int32_t nz, const int32_t* obstacle, const float* wx,
                              const float* wy, const float* wz, const double* a, const double* b,
                              double* result_device, void* stream);

/* fluid.py:4224-4273 _pressure_fv_jacobi_kernel, one out-of-place sweep on
 * level `level` (level 0: double arrays, coarse levels: float arrays).  rhs
 * and iface follow the level's storage type. */
int efsi_fv_jacobi_sweep(efsi_fv_plan* plan, int32_t level, const void* p, const void* rhs, void* tmp,
                         int32_t outlet, double omega, void* stream);

/* fluid.py:5262-5307 _mg_compute_residual_kernel on `level`. */
int efsi_fv_residual(efsi_fv_plan* plan, int32_t level, const void* p, const void* rhs, void* residual,
                     int32_t outlet, void* stream);

/* fluid.py:5310-5388 _mg_restrict_residual_kernel: coarse_rhs of level+1
 * (float) from the fine residual of `level`; the optional outputs receive the
 * coarse interface diagonal, obstacle and Dirichlet flag / weight views. */
int efsi_mg_restrict(efsi_fv_plan* plan, int32_t level, const void* fine_residual, float* coarse_rhs,
                     float* coarse_iface, int32_t* coarse_obstacle, int32_t* coarse_vdir_active,
                     float* coarse_vdir_weight, void* stream);

/* fluid.py:5391-5406 _mg_prolongate_add_kernel: fine(level) += s * coarse(level+1). */
int efsi_mg_prolong(efsi_fv_plan* plan, int32_t level, void* fine_p, const float* coarse_p, double scale,
                    void* stream);

/* fluid.py:6085-6262 _apply_fv_multigrid_preconditioner: z = V-cycle(r), zero
 * initial guess. */
int efsi_mg_vcycle(efsi_fv_plan* plan, const double* r, double* z, int32_t outlet, int32_t pre, int32_t coarse,
                   int32_t post, void* stream);

typedef struct efsi_pcg_params {
  int32_t max_iters;
  int32_t precond;      /* 0 jacobi, 1 fv_multigrid (2/24/2), 2 fv_multigrid_light (1/12/1),
                           3 fv_multigrid_mixed: the 2/24/2 V-cycle with FP32 level-0 iterates and
                           arithmetic (no reference counterpart; the CG stays FP64),
                           4 learned: two-level, with the network attached by
                           efsi_fv_set_learned_preconditioner as the coarse correction between two
                           damped-Jacobi sweeps on each side, falling back to the 2/24/2 V-cycle
                           (no reference counterpart),
                           5 the same without the fallback (measurement of the learned preconditioner alone) */
  int32_t remove_mean;  /* closed-domain zero-mean projection */
  int32_t outlet;       /* pressure_outlet_zmin */
  int32_t iface_active; /* interface terms present: MG disabled, restart every 256 */
  int32_t use_graphs;   /* capture the 16-iteration blocks into CUDA graphs */
  double tolerance;
  int32_t device_loop;  /* no host reads: the iterations run as a device-side loop (a CUDA-graph WHILE
                           node) that stops on convergence, a breakdown code or max_iters; the stream
                           must be under stream capture (efsi_step_graph_begin) or the solve builds and
                           launches a graph of its own; stats come from efsi_fv_pcg_device_stats.
                           No reference counterpart (the reference reads the residual every 16
                           iterations on the host). */
} efsi_pcg_params;

typedef struct efsi_cg_stats {
  int32_t iterations;
  int32_t converged;
  int32_t breakdown_code;
  int32_t breakdown_reason; /* 0 none, 1 initial dot, 2 device scalar, 3 restart dot */
  int32_t host_residual_checks;
  int32_t restart_count;
  int32_t mean_projection_count;
  int32_t used_mg;
  int32_t used_graphs; /* the 16-iteration blocks ran as CUDA graphs */
  int32_t learned_iterations; /* iterations preconditioned by the learned network (code 4) before any
                                 fallback to the V-cycle */
  double initial_relative_residual;
  double relative_residual;
  double breakdown_dAd;
  double b_norm;
  double learned_relative_residual; /* relative residual at the last check preconditioned by the learned network */
  int32_t unreached_set_mean_projection_count; /* fluid.py:4965 _subtract_unreached_set_mean_device calls */
} efsi_cg_stats;

/* fluid.py:6535-6811 _solve_pressure_poisson_fv_cg: flexible MG/Jacobi PCG on
 * A p = b in the cell-volume inner product, from the f64 level-0 rhs built by
 * efsi_mg_prepare_level0.  pressure is the warm start and the solution. */
int efsi_fv_pcg_solve(efsi_fv_plan* plan, const double* rhs0, double* pressure, const efsi_pcg_params* params,
                      efsi_cg_stats* stats, void* stream);

/* The PCG's device scalars of a plan (the reference's 0-D cg_rz, cg_rz_new,
 * cg_dAd, cg_beta_numerator, cg_alpha, cg_beta, cg_breakdown_dAd and
 * cg_breakdown_code fields, fluid.py:1098-1112). */
typedef struct efsi_cg_scalar_values {
  double rz, rz_new, dAd, beta_numerator, alpha, beta, breakdown_dAd;
  int32_t breakdown_code;
} efsi_cg_scalar_values;

/* Writes / reads the plan's device scalars (read synchronises the stream). */
int efsi_cg_scalars_write(efsi_fv_plan* plan, const efsi_cg_scalar_values* values, void* stream);
int efsi_cg_scalars_read(efsi_fv_plan* plan, efsi_cg_scalar_values* values, void* stream);

/* fluid.py:4567-4574 _cg_compute_alpha_kernel on the plan's device scalars
 * (the same device step the PCG's SpMV finishers run): alpha = rz / dAd, or
 * breakdown code 1 when dAd <= 0. */
int efsi_cg_compute_alpha(efsi_fv_plan* plan, void* stream);

/* fluid.py:4590-4601 _cg_compute_beta_kernel on the plan's device scalars
 * (the same device step the PCG's dots finishers run): Polak-Ribiere beta
 * clamped at 0 when use_mg, else rz_new / rz; breakdown code 2 when rz <=
 * 1e-300 or rz_new <= 0. */
int efsi_cg_compute_beta(efsi_fv_plan* plan, int32_t use_mg, void* stream);

/* Why CUDA-graph capture was abandoned for this plan ("" when it was not). */
const char* efsi_fv_graph_error(efsi_fv_plan* plan);

/* Statistics of the last efsi_fv_pcg_solve with device_loop under an outer
 * stream capture, read after the captured graph ran (synchronises the
 * stream): iterations, converged, relative residuals, b_norm, breakdown code.
 * No reference counterpart. */
int efsi_fv_pcg_device_stats(efsi_fv_plan* plan, efsi_cg_stats* stats, void* stream);

/* Whole-step CUDA graphs (no reference counterpart: the reference launches
 * every kernel of a step from Python, hibm_mpm.py:10533-10616).  begin starts
 * a stream capture on a created stream (not the legacy default stream); the
 * library calls of one step follow, with device-side PCG loops
 * (efsi_pcg_params::device_loop) and no host reads; end instantiates the
 * graph; launch replays the whole step with one call. */
typedef struct efsi_step_graph efsi_step_graph;
int efsi_step_graph_begin(void* stream);
int efsi_step_graph_end(void* stream, efsi_step_graph** out);
int efsi_step_graph_launch(efsi_step_graph* graph, void* stream);
int efsi_step_graph_destroy(efsi_step_graph* graph);

/* Grid size of the cooperative kernel that runs the V-cycle's levels 1 ..
 * lt-1 and its tail in one launch (0: per-level launches; efsi_last_error()
 * then says why).  No reference counterpart: the reference launches every
 * level's kernels (fluid.py:6085-6262). */
int efsi_fv_coarse_kernel_blocks(efsi_fv_plan* plan, int32_t* blocks);

/* fluid.py:5992-6083 _solve_pressure_poisson_fv_multigrid (standalone cycles). */
int efsi_fv_multigrid_solve(efsi_fv_plan* plan, const double* rhs0, double* pressure, int32_t outlet,
                            int32_t iterations, int32_t cycles, void* stream);

/* fluid.py:5977-5990 _solve_pressure_poisson_fv_jacobi (omega 0.8 sweeps on level 0). */
int efsi_fv_jacobi_solve(efsi_fv_plan* plan, const double* rhs0, double* pressure, int32_t outlet,
                         int32_t iterations, void* stream);

/* fluid.py:3997-4059 _pressure_jacobi_kernel + _copy_pressure_kernel, `iterations`
 * times (the legacy uniform-grid solver "jacobi"); tmp is an f64 scratch field. */
int efsi_legacy_jacobi_solve(efsi_fv_plan* plan, const float* divergence, const float* volume_source,
                             float rhs_scale, float inv_dx2, float inv_dy2, float inv_dz2, int32_t outlet,
                             int32_t iterations, double* pressure, double* tmp, void* stream);

/* fluid.py:5538-5582 _subtract_pressure_gradient_kernel.  vdir_* may be NULL. */
int efsi_subtract_pressure_gradient(efsi_fv_plan* plan, const double* pressure, const int32_t* vdir_active,
                                    const float* vdir_weight, const float* vdir_value, float dt_over_rho,
                                    int32_t outlet, float* velocity, void* stream);

/* fluid.py:5529-5536 _apply_closed_boundary_no_normal_flow_kernel. */
int efsi_apply_closed_boundary(efsi_fv_plan* plan, int32_t outlet, float* velocity, void* stream);

/* fluid.py:5762-5766 _apply_zmin_no_backflow_kernel. */
int efsi_apply_zmin_no_backflow(efsi_fv_plan* plan, float* velocity, void* stream);

/* fluid.py:2549-2593 _apply_velocity_dirichlet_boundary_rows_kernel.
 * report_device (may be NULL): double[6] = cells, delta_sum, delta_max, momentum xyz. */
int efsi_apply_velocity_dirichlet_rows(efsi_fv_plan* plan, const int32_t* vdir_active, const float* vdir_value,
                                       float density, float* velocity, double* report_device, void* stream);

/* Fluid grid faces / centres (device f32) used by the predictor and samplers. */
typedef struct efsi_grid_axes {
  const float* fx;
  const float* fy;
  const float* fz;
  const float* cx;
  const float* cy;
  const float* cz;
} efsi_grid_axes;

/* fluid.py:2447-2527 _predict_kernel (velocity_prev is read, velocity written). */
int efsi_predict(efsi_fv_plan* plan, const efsi_grid_axes* axes, const float* velocity_prev, float dt, float nu,
                 int32_t rk2, float* velocity, void* stream);

/* fluid.py:3574-3663 _divergence_final_report_kernel: out_host[54] = 18 slots
 * of (max_abs, sum_sq, count) over the fluid cells, raw |div + iface_div|
 * then residual |... - source| per pair: all, interior, near / far from a
 * velocity-Dirichlet row (fluid.py:3665-3690), with / without a pressure-
 * correctable face (fluid.py:3717-3768), interior with / without, and the
 * outlet-unreached cells (outlet_reachable == 0; NULL: none), which are kept
 * out of every other slot.  velocity_dirichlet_active may be NULL. */
int efsi_divergence_final_report(efsi_fv_plan* plan, const float* divergence, const double* iface_div,
                                 const float* volume_source, const int32_t* velocity_dirichlet_active,
                                 const int32_t* outlet_reachable, int32_t outlet, double* out_host, void* stream);

/* fluid.py:3494-3565 _divergence_stats_kernel / _divergence_residual_stats_kernel.
 * mode 0 raw, 1 residual (minus volume source).  out_host: max_abs, sum_sq, count. */
int efsi_divergence_stats(efsi_fv_plan* plan, const float* divergence, const double* iface_div,
                          const float* volume_source, int32_t mode, int32_t interior_only, double* out_host,
                          void* stream);

/* fluid.py:3196-3273 _spread_surface_forces_kernel.  report_device: double[6]
 * (surface force xyz, grid force xyz). */
int efsi_spread_surface_forces(efsi_fv_plan* plan, const efsi_grid_axes* axes, const float* position,
                               const float* force, int32_t vertex_count, float cx, float cy, float cz,
                               float force_sign, float* grid_force_density, double* report_device, void* stream);

/* fluid.py:3301-3328 _apply_body_force_kernel.  report_device: double[7]
 * (impulse xyz, momentum xyz, active cells). */
int efsi_apply_body_force(efsi_fv_plan* plan, const float* grid_force_density, float dt, float density,
                          float* velocity, double* report_device, void* stream);

/* ------------------------------------------------------------------------ */
/* Neo-Hookean MLS/APIC-MPM                                                  */
/* ------------------------------------------------------------------------ */

/* Scratch for particle binning on the MPM node grid (replaces nothing in the
 * reference, which scatters with per-particle global atomics). */
int efsi_mpm_plan_create(int32_t particle_capacity, int32_t nx, int32_t ny, int32_t nz, efsi_mpm_plan** out);
int efsi_mpm_plan_destroy(efsi_mpm_plan* plan);

typedef struct efsi_mpm_state {
  int32_t particle_count;
  int32_t nx, ny, nz;
  float bmin[3];
  float dx[3];
  float* x;
  float* v;
  float* C;
  float* F;
  const float* mass;
  const float* volume;
  const float* fext;
  const int32_t* fixed;
  const int32_t* region;
  const float* rest_x;
  float* normal;
  float* area;
  const float* rest_normal;
  const float* rest_area;
  float* grid_mass;
  float* grid_velocity;
  float* grid_force;
} efsi_mpm_state;

/* neo_hookean_mpm.py:696-959 _step_kernel (clear, P2G, grid update, G2P,
 * surface geometry, diagnostics).  report_device: double[34] in the layout of
 * report_host_snapshot (neo_hookean_mpm.py:909-958), or NULL. */
int efsi_mpm_step(efsi_mpm_plan* plan, const efsi_mpm_state* state, float dt, float mu, float lambda_,
                  float velocity_damping, int32_t primary_region, int32_t secondary_region,
                  double* report_device, void* stream);

/* ------------------------------------------------------------------------ */
/* Triangle Mooney-Rivlin membrane MPM                                       */
/* ------------------------------------------------------------------------ */

/* Doubles of caller-provided scratch that efsi_shell_step accumulates its
 * report sums in (cleared by the step itself). */
#define EFSI_SHELL_SCRATCH_DOUBLES 48

/* Device buffers of one membrane (float3 arrays are [n][3]; the node grid is
 * x-major [nx][ny][nz]).  Mirrors the fields of TriMooneyShellMpmState
 * (mooney_shell_mpm.py:179-222). */
typedef struct efsi_shell_state {
  int32_t particle_count, face_count, edge_count;
  int32_t nx, ny, nz;
  float bmin[3];
  float dx[3];
  float* x;
  float* u;
  float* v;
  const float* rest_x;
  const float* mass;
  float* area;
  float* normal;
  float* internal_force;
  float* external_force;
  const int32_t* vertex_region;
  const int32_t* fixed;
  const int32_t* faces;       /* [face_count][3] */
  const int32_t* face_region; /* [face_count] */
  const int32_t* edges;       /* [edge_count][2], unique undirected */
  float* grid_mass;
  float* grid_velocity;
  float* grid_velocity_before;
  float* grid_force;
} efsi_shell_state;

/* Arguments of one step.  region_loads = 0 is step() (uniform pressure on
 * every face, mooney_shell_mpm.py:860-1003, 1179-1202); region_loads = 1 is
 * advance_region_loads() / advance_with_external_forces() (:1005-1292), with
 * the region thicknesses, the area load on area_load_region and the two
 * interface reactions spread by rest area over primary_area / secondary_area. */
typedef struct efsi_shell_params {
  float dt, pressure, velocity_damping, flip_blend;
  float body_acceleration[3];
  float c1, c2, membrane_force_scale;
  float thickness, primary_thickness, secondary_thickness;
  int32_t region_loads;
  int32_t preserve_external_force;
  int32_t primary_region, secondary_region, area_load_region;
  float primary_area_load[3];
  float primary_reaction[3];
  float secondary_reaction[3];
  float primary_area, secondary_area;
} efsi_shell_params;

/* mooney_shell_mpm.py:480-540 _init_mass_kernel: zero the particle state,
 * rest-area mass and area shares, vertex regions (minimum of the faces'),
 * fixed vertices; region_totals (float[4] or NULL) = primary area, primary
 * mass, secondary area, secondary mass; then the current-shape normals. */
int efsi_shell_init(const efsi_shell_state* state, float* mass, int32_t* vertex_region, int32_t* fixed,
                    float density, float thickness, float primary_thickness, float secondary_thickness,
                    int32_t primary_region, int32_t secondary_region, int32_t fixed_region, float* region_totals,
                    void* stream);

/* mooney_shell_mpm.py:449-461 _update_particle_surface_normals (used after
 * restore_state, :1301-1309). */
int efsi_shell_update_normals(const efsi_shell_state* state, void* stream);

/* mooney_shell_mpm.py:710-728 _add_region_area_load_kernel. */
int efsi_shell_add_region_area_load(const efsi_shell_state* state, int32_t region_id, const float* area_load_npm2,
                                    void* stream);

/* mooney_shell_mpm.py:860-1003 _step_kernel and :1005-1177
 * _step_region_kernel.  scratch: EFSI_SHELL_SCRATCH_DOUBLES doubles of device
 * memory; report_device: double[37] in the layout of report_host_snapshot
 * (:337-391), or NULL. */
int efsi_shell_step(const efsi_shell_state* state, const efsi_shell_params* params, double* scratch,
                    double* report_device, void* stream);

/* ------------------------------------------------------------------------ */
/* HIBM surface markers                                                      */
/* ------------------------------------------------------------------------ */

/* hibm_mpm.py:2253-2432 _sample_pressure_only_marker_tractions_kernel.
 * report_device: double[5] = valid, invalid, two_sided, one_sided, max |t|. */
int efsi_sample_pressure_tractions(int32_t nx, int32_t ny, int32_t nz, const efsi_grid_axes* axes,
                                   const float* wx, const float* wy, const float* wz, const int32_t* obstacle,
                                   const double* pressure, int32_t marker_count, const float* x_gamma,
                                   const float* n_gamma, const int32_t* region, int32_t two_sided,
                                   int32_t one_sided_region, float one_sided_reference, double* t_gamma,
                                   int32_t* valid, double* report_device, void* stream);

/* hibm_mpm.py:903-909 _compute_marker_forces_kernel: F = t A. */
int efsi_compute_marker_forces(int32_t marker_count, const double* t_gamma, const float* area, double* f_gamma,
                               void* stream);

/* hibm_mpm.py:4861-4878 _clear_mpm_external_forces_kernel.
 * report_device: double[2] = cleared count, max |f| before. */
int efsi_clear_external_forces(int32_t particle_count, float* external_force, double* report_device,
                               void* stream);

/* Uniform binning of particles with bin edge = support radius over a box;
 * used by the spreading and feedback entry points below. */
int efsi_bin_plan_create(int32_t particle_capacity, const float* box_min, const float* box_max,
                         float support_radius, efsi_bin_plan** out);
int efsi_bin_plan_destroy(efsi_bin_plan* plan);
/* Sorts particle indices into bins (stable: particle order within a bin). */
int efsi_bin_particles(efsi_bin_plan* plan, const float* particle_x, int32_t particle_count, void* stream);

/* hibm_mpm.py:4899-4959 _scatter_marker_forces_to_mpm_particles_kernel over the
 * binned particles (the reference loops over all particles per marker).
 * report_device: double[9] = active markers, invalid markers, active
 * contributions, marker force xyz, external force xyz. */
int efsi_scatter_marker_forces(efsi_bin_plan* plan, int32_t marker_count, const float* x_gamma,
                               const double* f_gamma, const float* particle_x, float* external_force,
                               double* report_device, void* stream);

/* hibm_mpm.py:5097-5180 _update_surface_feedback_from_mpm_surface_particles_kernel
 * (particle_normal / particle_area NULL: velocity-only variant hibm_mpm.py:5012-5053).
 * report_device: double[8] = updated, invalid, geometry updated, geometry
 * invalid, max displacement, max speed, max normal change, max area change. */
int efsi_surface_feedback(efsi_bin_plan* plan, int32_t marker_count, float* x_gamma, float* v_gamma,
                          float* n_gamma, float* area_gamma, const float* particle_x, const float* particle_v,
                          const float* particle_normal, const float* particle_area, float dt,
                          double* report_device, void* stream);

/* Immersed-boundary node search (hibm_mpm.py:5385-6220 HibmMpmIbNodeSearch). */
typedef struct efsi_ib_search_params {
  int32_t nx, ny, nz;            /* nodes */
  int32_t marker_count;
  int32_t triangle_count;        /* projection triangles; 0: search the markers */
  int32_t classify_far_internal_nodes;
  float search_radius_m, interior_probe_distance_m, sign_tolerance_m;
  /* node positions: the three centre arrays (nx, ny, nz floats) when given
     (search_and_classify_grid_fields), else bounds_min + (i + 0.5) * spacing
     per axis in f32 (search_and_classify) */
  const float* cell_center_x_m;
  const float* cell_center_y_m;
  const float* cell_center_z_m;
  float bounds_min_m[3];
  float spacing_m[3];
  float box_min_m[3], box_max_m[3]; /* box of the node positions, for the triangle bins */
  const float* marker_x;         /* marker positions, 3 floats each */
  const float* marker_n;         /* marker normals */
  const int32_t* triangles;      /* 3 marker indices each */
} efsi_ib_search_params;

/* Per-node output fields (hibm_mpm.py:5418-5436), C order over (nx, ny, nz):
   node kind (0 none, 1 external IB, 2 internal), nearest marker, signed
   distance, boundary point (3), interior fluid point (3), projection marker
   indices (3) and weights (3); report: int32[4] = near-boundary, external IB,
   internal and invalid-projection node counts (written on the device). */
typedef struct efsi_ib_search_fields {
  int32_t* node_kind;
  int32_t* nearest_marker;
  float* signed_distance_m;
  float* boundary_point_m;
  float* interior_fluid_point_m;
  int32_t* projection_marker_indices;
  float* projection_marker_weights;
  int32_t* report;
} efsi_ib_search_fields;

/* Work buffers of the node search (triangle bins), grown on demand. */
int efsi_ib_search_plan_create(efsi_ib_search_plan** out);
int efsi_ib_search_plan_destroy(efsi_ib_search_plan* plan);

/* hibm_mpm.py:5601-5835 _search_and_classify_kernel and 5837-6068
 * _search_and_classify_grid_fields_kernel (argument checks of
 * hibm_mpm.py:6069-6094).  Same fields and counts as the reference's
 * all-pairs loop; the triangles are binned by their box widened by the
 * search radius, so a near node visits only its bin.  Synchronises the
 * stream once (the bin entry total). */
int efsi_ib_node_search(efsi_ib_search_plan* plan, const efsi_ib_search_params* params,
                        const efsi_ib_search_fields* fields, void* stream);

/* Report of efsi_ib_build_boundary_conditions (HibmMpmIbBoundaryConditionReport). */
typedef struct efsi_ib_bc_report {
  int32_t no_slip_dirichlet_count;
  int32_t pressure_neumann_count;
  int32_t inactive_internal_node_count;
  float max_abs_velocity_mps;
} efsi_ib_bc_report;

/* hibm_mpm.py:6499-6577 HibmMpmIbBoundaryConditions._build_from_search_kernel:
 * per external IB node of the search, the no-slip velocity, Neumann normal
 * and Neumann gradient targets interpolated from the projection markers
 * (3 floats per node for velocity and normal).  report_device is written on
 * the device. */
int efsi_ib_build_boundary_conditions(int64_t node_count, const int32_t* node_kind, const int32_t* nearest_marker,
                                      const int32_t* projection_marker_indices,
                                      const float* projection_marker_weights, const float* marker_velocity,
                                      const float* marker_normal, const float* marker_gradient, int32_t marker_count,
                                      int32_t* active, float* velocity, float* normal, float* gradient,
                                      efsi_ib_bc_report* report_device, void* stream);

/* Inputs of efsi_ib_velocity_dirichlet_rows: the fluid grid (faces n + 1 and
   centres n per axis, f32), the boundary targets (active IB flag, target
   velocity and normal), the node search's boundary / interior points and
   nearest markers, the obstacle and cell velocity (3 floats per cell), and
   optionally the markers' region ids for the region stamp. */
typedef struct efsi_ib_vd_params {
  int32_t nx, ny, nz;
  const float* face_x_m;
  const float* face_y_m;
  const float* face_z_m;
  const float* center_x_m;
  const float* center_y_m;
  const float* center_z_m;
  const int32_t* active_ib_node;
  const float* target_velocity;
  const float* target_normal;
  const float* boundary_point_m;
  const float* interior_fluid_point_m;
  const int32_t* nearest_marker;
  const int32_t* obstacle;
  const float* velocity;
  const int32_t* marker_region_id; /* NULL: no region stamp */
  int32_t marker_count;
} efsi_ib_vd_params;

/* Report of the velocity-Dirichlet rows (HibmMpmVelocityDirichletBoundaryReport;
   blocked_rows is both its inactive_obstacle_rows and relocation_blocked_row_count). */
typedef struct efsi_ib_vd_report {
  int32_t active_rows;
  int32_t blocked_rows;
  int32_t invalid_rows;
  int32_t invalid_no_fluid_sample_rows;
  int32_t invalid_nonpositive_gap_rows;
  int32_t invalid_node_behind_boundary_rows;
  int32_t invalid_node_beyond_interior_rows;
  int32_t narrow_gap_rows;
  int32_t relocated_rows;
  int32_t merged_rows;
  float max_abs_velocity_mps;
  float min_projection_weight; /* 1e30 when no row was written */
  float max_projection_weight;
} efsi_ib_vd_report;

/* Outputs: the fluid's row fields (active, value 3 per cell, projection
   weight), the search's anchor cells (3 int32 per node), the region ids (in
   place) and the report (device). */
typedef struct efsi_ib_vd_fields {
  int32_t* active;
  float* value_mps;
  float* projection_weight;
  int32_t* anchor_cell;
  int32_t* marker_region_id;
  efsi_ib_vd_report* report;
} efsi_ib_vd_fields;

/* reconstruct = 0: hibm_mpm.py:6649-6688 _assemble_velocity_dirichlet_boundary_rows_kernel
 * (the target velocity on every unmasked active IB node; only the active and
 * value fields are written).  reconstruct = 1: hibm_mpm.py:7655-7800
 * assemble_velocity_dirichlet_reconstructed_boundary_rows: anchor prefill
 * (7551-7616), row reconstruction along the normal with its fallbacks
 * (6904-7335), relocation of masked rows (7337-7549) and the region stamp
 * (7618-7653).  Where the reference's parallel loops race (relocation claims,
 * region writes), the node visited first in C order claims a cell and the
 * one visited last stamps it. */
int efsi_ib_velocity_dirichlet_rows(efsi_ib_search_plan* plan, const efsi_ib_vd_params* params,
                                    const efsi_ib_vd_fields* fields, int32_t reconstruct, void* stream);

/* hibm_mpm.py:5463-5475 _reset_node_anchor_cells_kernel: every node's
 * anchor cell (3 int32 each) to (-1, -1, -1). */
int efsi_ib_reset_anchor_cells(int32_t* anchor_cells, int64_t node_count, void* stream);

/* fluid.py:6264-6533 _continue_pressure_poisson_fv_bicgstab: the BiCGSTAB
 * fallback (right Jacobi preconditioning) of the level-0 system A p = rhs
 * from the pressure in `pressure`, relative to b_norm; remove_mean applies
 * the zero-mean projection where the reference does, and with an outlet the
 * unreached-component anchoring of efsi_fv_set_unreached_components.  Host loop with one host read per inner product; allocates
 * nine work vectors for the call.  stats: int64[4] = iterations, converged,
 * restarts, breakdown code (0 none, 1 shadow dot, 2 recurrence scalar,
 * 3 beta, 4 alpha denominator, 5 alpha, 6 omega denominator, 7 omega,
 * 8 not converged). */
int efsi_fv_bicgstab(efsi_fv_plan* plan, const double* rhs, double* pressure, int32_t outlet, int32_t max_iters,
                     double tolerance, double b_norm, int32_t remove_mean, int64_t* stats, double* relative_residual,
                     void* stream);

/* The unreached components of an outlet solve (fluid.py:4729-4981): comp[c]
 * (device int32 per level-0 cell) is the component of an outlet-unreached
 * fluid cell that the PCG anchors, -1 elsewhere; at most 256 components
 * (ncomp 0 clears them).  With an outlet, efsi_fv_pcg_solve and
 * efsi_fv_bicgstab then subtract each component's volume-weighted mean from
 * the residual, the preconditioned residual and the pressure where the
 * reference calls _subtract_unreached_set_mean_device.  Copies comp into the
 * plan; synchronises. */
int efsi_fv_set_unreached_components(efsi_fv_plan* plan, const int32_t* comp, int32_t ncomp, void* stream);

/* fluid.py:4965-4981 _subtract_unreached_set_mean_device on a level-0 f64
 * field with the components set by efsi_fv_set_unreached_components; with
 * sums_host / volumes_host (double[ncomp], either may be NULL) also returns
 * each component's volume-weighted integral and volume before the subtraction
 * (fluid.py:4985-5020 measures the rhs incompatibility from them). */
int efsi_fv_subtract_unreached_means(efsi_fv_plan* plan, double* field, double* sums_host, double* volumes_host,
                                     void* stream);

/* Report of efsi_outlet_reachability. */
typedef struct efsi_reach_report {
  int64_t unreached_cells;
  int32_t components; /* ranked components, at most 256 */
  int32_t overflow;   /* more than 256 components */
} efsi_reach_report;

int efsi_reach_plan_create(efsi_reach_plan** out);
int efsi_reach_plan_destroy(efsi_reach_plan* plan);

/* fluid.py:1614-1876 mark_hibm_pressure_outlet_disconnected_nonprojectable_cells
 * (reachability part) with fluid.py:4764-4910 (unreached component labels):
 * the z-min outlet reachability of every fluid, non-barrier cell, and the
 * unreached components' labels (-(rank + 1) by smallest cell index, up to
 * 256; 1 << 30 for reached and non-fluid cells).  With update_barrier the
 * barrier field is first set from node_kind == barrier_code (node_kind NULL:
 * cleared), fluid.py:1618-1647.  One union-find over the open faces instead
 * of the reference's Jacobi sweeps; synchronises the stream twice. */
int efsi_outlet_reachability(efsi_reach_plan* plan, int32_t nx, int32_t ny, int32_t nz, const int32_t* obstacle,
                             const int32_t* velocity_dirichlet_active, int32_t* barrier, const int32_t* node_kind,
                             int32_t barrier_code, int32_t update_barrier, int32_t* reachable, int32_t* label,
                             efsi_reach_report* report, void* stream);

/* Zeroes `count` (<= 64) device buffers of bytes[q] bytes (multiples of 4)
 * in one launch: the per-solve clears of the multigrid work fields of
 * fluid.py:5228-5260 _prepare_fv_multigrid_rhs.  ptrs and bytes are host
 * arrays. */
int efsi_zero_buffers(int32_t count, void* const* ptrs, const int64_t* bytes, void* stream);

/* fluid.py:4345-4456, the interface-coupling terms of _fv_laplacian_apply_kernel
 * (row list, or per-cell slots when the row count is 0): installs them in the
 * plan's level-0 operator (efsi_fv_apply, the PCG and the BiCGSTAB fallback).
 * They arrive as rows: for receiving cell rows[r] (distinct, increasing
 * linear indices), entries row_ptr[r] .. row_ptr[r + 1] of (src, coef) add
 * -(coef * p[src]) in entry order, coef = T / V_receiver.  Device arrays,
 * validated on the host (synchronises); nrows = 0 removes them. */
int efsi_fv_set_interface_coupling(efsi_fv_plan* plan, int32_t nrows, const int32_t* rows, const int32_t* row_ptr,
                                   const int32_t* src, const double* coef, void* stream);

/* The positive right-hand side b of the last efsi_fv_pcg_solve (the reference's
 * cg_rhs, fluid.py:6589-6603), copied to out (f64, level 0). */
int efsi_fv_copy_rhs(efsi_fv_plan* plan, double* out, void* stream);

/* ------------------------------------------------------------------------
 * Learned preconditioner (no counterpart in the reference: a new
 * preconditioner for the reference's flexible PCG, fluid.py:6535-6811, whose
 * multigrid V-cycle stays the fallback).  A 3-D convolutional U-Net (4
 * levels, 16/32/48/64 channels, 15 convolutions of 3x3x3, about 0.69 M
 * parameters) on channels-last BF16 volumes; convolutions on the tensor cores
 * (tcgen05, FP32 accumulation), weight gradients and Adam in FP32.
 * ------------------------------------------------------------------------ */
typedef struct efsi_unet efsi_unet;

/* One 3x3x3 convolution, zero padded, of x (BF16 [n][cin]) with w (BF16
 * [cout][27][cin], tap t = (di + 1) * 9 + (dj + 1) * 3 + (dk + 1)), plus the
 * bias and an optional ReLU; writes BF16 y [n][cout] and/or FP32 yf.  cin and
 * cout are multiples of 16.  A pipeline wait that gives up sets
 * *error_device. */
int efsi_conv3d_bf16(int32_t nx, int32_t ny, int32_t nz, int32_t cin, int32_t cout, const void* x, const void* w,
                     const float* bias, int32_t relu, void* y, float* yf, int32_t* error_device, void* stream);

/* Weight gradient of that convolution: dw[co][t][ci] += sum_v dy[v][co]
 * x[v + off(t)][ci] (FP32 accumulation into dw). */
int efsi_conv3d_wgrad(int32_t nx, int32_t ny, int32_t nz, int32_t cin, int32_t cout, const void* x,
                      const void* dy, float* dw, void* stream);

/* The network: He-normal weights from `seed`, zero biases. */
int efsi_unet_create(int32_t seed, efsi_unet** out);
int efsi_unet_destroy(efsi_unet* net);
int efsi_unet_param_count(efsi_unet* net, int64_t* count);
/* Per layer (15): weight and bias offsets in the packed parameter vector, and
 * (level, cin, cout, relu). */
int efsi_unet_layer_offsets(efsi_unet* net, int64_t* weight_offsets, int64_t* bias_offsets, int32_t* shapes);
/* FP32 parameters and accumulated gradients to the host (either may be NULL). */
int efsi_unet_get_params(efsi_unet* net, float* host_params, float* host_grads);
/* Loads FP32 parameters from the host and resets the Adam state. */
int efsi_unet_set_params(efsi_unet* net, const float* host_params);
/* Forward pass of a volume: input BF16 [n][16]; output FP32 [n][16]
 * (channel 0 is the network output) or NULL.  Synchronises the stream. */
int efsi_unet_forward(efsi_unet* net, int32_t nx, int32_t ny, int32_t nz, const void* input, float* output,
                      void* stream);
/* Forward, masked mean-square loss of output channel 0 against target (FP32
 * [n]; mask FP32 [n]) and backward; gradients are accumulated.  Writes the
 * loss to *loss_host and synchronises the stream. */
int efsi_unet_accumulate_gradient(efsi_unet* net, int32_t nx, int32_t ny, int32_t nz, const void* input,
                                  const float* target, const float* mask, double* loss_host, void* stream);
/* Forward and backward from a given output gradient dout (FP32 [n][16]);
 * gradients are accumulated (gradient checks). */
int efsi_unet_backward_from(efsi_unet* net, int32_t nx, int32_t ny, int32_t nz, const void* input,
                            const float* dout, void* stream);
int efsi_unet_zero_grad(efsi_unet* net, void* stream);
/* One Adam step on the accumulated gradients (which it clears). */
int efsi_unet_adam_step(efsi_unet* net, float lr, float beta1, float beta2, float eps, void* stream);

/* Attaches a network to a solver plan as preconditioner codes 4 and 5 of
 * efsi_fv_pcg_solve (NULL detaches).  Inside the flexible PCG, z is: z_pre =
 * two damped-Jacobi sweeps (the V-cycle's level-0 smoother) on A z = r from
 * zero; r' = r - A z_pre; n = RMS(r') net(r')[0]; z_c = z_pre + s n with
 * s = <r', n>_V / <n, A n>_V (the energy-minimising scale; 0 when <n, A n>_V
 * is not positive); z = two more sweeps from z_c.  With code 4 the multigrid
 * V-cycle takes over when a 16-iteration block does not halve the residual.
 * Allocates the network's workspace for level 0 (call before any stream
 * capture); synchronises. */
int efsi_fv_set_learned_preconditioner(efsi_fv_plan* plan, efsi_unet* net, void* stream);

/* The network input of the plan's level 0 for residual r (f64): channel 0 r
 * scaled to unit volume-weighted RMS over the fluid cells, 1 the fluid mask,
 * 2-4 log2 of the cell widths over the finest width of each axis (BF16 [n][16]). */
int efsi_fv_learned_input(efsi_fv_plan* plan, const double* r, void* input, void* stream);

/* z = the learned preconditioner's pre-smoothing of r: two damped-Jacobi
 * sweeps of the plan's level 0 on A z = r from zero (training pairs are
 * formed from the residual and error that remain after it).  No reference
 * counterpart. */
int efsi_fv_learned_presmooth(efsi_fv_plan* plan, const double* r, double* z, int32_t outlet, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* EASYFSI_B200_H */
