/*
 * netflux_b200.h — C ABI of the B200 implementation of NetFlux's explicit
 * second-order Euler step.
 *
 * Plain C types only (pointers, sizes, ints, doubles); no CUDA or torch types
 * cross this boundary. Every function returns 0 (NF_OK) on success or an
 * NF_ERR_* code; the text of the last error of a solver is available from
 * nf_last_error(), of a failed mesh or solver creation from nf_last_error(NULL).
 *
 * Each entry point replaces one piece of the reference's C++ call path
 * (file:line in andersresell/NetFlux):
 *
 *   nf_mesh_from_su2 / nf_mesh_from_arrays
 *       geometry::PrimalGrid(config) + geometry::FV_Grid(config, primal)
 *       (PrimalGrid.cpp:140-244, FV_Grid.cpp:21-205)
 *   nf_create          EulerSolver::EulerSolver (Solver.cpp:135-142)
 *   nf_set_state / nf_get_state
 *                      SolverData::get_solution (SolverData.hpp:46-47) — the
 *                      AoS double[N][5] the reference's Output reads
 *   nf_calc_timestep   EulerSolver::calc_timestep (Solver.cpp:232-274)
 *   nf_set_timestep    Config::set_delta_time (Config.hpp:146)
 *   nf_step            Solver::step (Solver.cpp:34-52): TVD_RK3 (103-133) or
 *                      explicit_euler (83-101)
 *   nf_advance         n iterations of Driver::solve's loop body
 *                      (Driver.cpp:38-47) without host round trips
 *   nf_get_field       the SolverData accessors get_primvars / _gradient /
 *                      _limiter / get_flux_balance (SolverData.hpp:52-68)
 *   nf_destroy         ~Solver
 *
 * Threading: a solver handle is bound to the CUDA device that was current
 * when it was created and to its own stream; it is not re-entrant.
 */
#ifndef NETFLUX_B200_H
#define NETFLUX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define NF_OK 0
#define NF_ERR_ARG 1          /* invalid argument or size mismatch */
#define NF_ERR_MESH 2         /* unreadable or invalid mesh */
#define NF_ERR_CUDA 3         /* a CUDA call failed */
#define NF_ERR_NONPHYSICAL 4  /* non-finite values or rho <= 0 / p <= 0 */
#define NF_ERR_DT 5           /* invalid time step (not finite or <= 0) */
#define NF_ERR_UNSUPPORTED 6  /* option not implemented */

/* ---- enums (same meaning and order as the reference's, Utilities.hpp) ---- */
#define NF_BC_NO_SLIP_WALL 0  /* BoundaryType::NoSlipWall */
#define NF_BC_SLIP_WALL 1     /* BoundaryType::SlipWall */
#define NF_BC_FAR_FIELD 2     /* BoundaryType::FarField */

#define NF_EXPLICIT_EULER 0   /* TimeScheme::ExplicitEuler */
#define NF_TVD_RK3 1          /* TimeScheme::TVD_RK3 */

#define NF_FIRST_ORDER 0      /* SpatialOrder::First */
#define NF_SECOND_ORDER 1     /* SpatialOrder::Second */

#define NF_LIMITER_NONE 0     /* Limiter::NONE */
#define NF_LIMITER_BARTH 1    /* Limiter::Barth */

#define NF_FLUX_RUSANOV 0     /* InviscidFluxScheme::Rusanov */

/* Arithmetic of the step. */
#define NF_PREC_FP64_REF 0    /* FP64 in the reference's operation order, no FMA
                                 contraction, true divisions: reproduces the
                                 reference to the last bit except pow() */
#define NF_PREC_FP64 1        /* FP64 throughout, FMA and reciprocals allowed */
#define NF_PREC_MIXED 2       /* FP64 state / RK combine / dt / norms; FP32
                                 gradient, limiter, reconstruction and flux in
                                 differences to the cell's FP64 primitives
                                 (converges to steady residuals like FP64) */
#define NF_PREC_MIXED32 3     /* FP64 state / RK combine / dt / norms; FP32
                                 copies of the primitives, FP32 gradient,
                                 limiter, reconstruction and flux (faster;
                                 its steady residual stops near a 1e-5 drop).
                                 Not for split meshes (nf_split_*, halos) */

/* nf_get_field selectors */
#define NF_FIELD_SOLUTION 0   /* U  [N][5] */
#define NF_FIELD_PRIMVARS 1   /* V of the last evaluated stage [N][5] (interior) */
#define NF_FIELD_GRADIENT 2   /* grad V [N][15], entry (k,d) at 5*d+k as in the reference */
#define NF_FIELD_LIMITER 3    /* Barth limiter [N][5] */
#define NF_FIELD_FLUX_BALANCE 4 /* R of the last stage [N][5] */
/* GRADIENT, LIMITER and FLUX_BALANCE need nf_params.keep_stage_fields */
#define NF_FIELD_LOCAL_DT 5   /* per-cell dt [N] (local time stepping) */

typedef struct nf_mesh nf_mesh;
typedef struct nf_solver nf_solver;

typedef struct {
  int64_t n_nodes;
  int64_t n_interior_cells;  /* Config::get_N_INTERIOR_CELLS */
  int64_t n_ghost_cells;     /* = boundary faces */
  int64_t n_interior_faces;  /* Config::get_N_INTERIOR_FACES */
  int64_t n_total_faces;     /* Config::get_N_TOTAL_FACES */
  int32_t n_patches;
  int32_t max_faces_per_cell;
  int64_t n_uncovered_boundary_faces; /* tet faces on the boundary that no
                                         marker lists; the reference drops them
                                         (FV_Grid.cpp:79-85) and so does this */
  int32_t n_cases;           /* concatenated cases (1 unless batched) */
  int32_t reserved;
} nf_mesh_info;

/* Build the face-based grid from an SU2 file. patch_names/patch_types give
 * the boundary type of every marker, like input.yml's "patches:" list; a
 * marker missing from the list is an error (PrimalGrid.cpp:216-217). Only
 * tetrahedral volume elements are accepted. */
nf_mesh* nf_mesh_from_su2(const char* path, int n_patch_types, const char* const* patch_names,
                          const int* patch_types);

/* The same from arrays: nodes [n_nodes][3]; tets [n_cells][4] node ids in the
 * order an SU2 file lists them; markers: n_markers names, marker_tris
 * [sum][3] with marker_offsets[n_markers+1] delimiting each marker. */
nf_mesh* nf_mesh_from_arrays(int64_t n_nodes, const double* nodes, int64_t n_cells, const int64_t* tets,
                             int n_markers, const char* const* marker_names, const int* marker_types,
                             const int64_t* marker_offsets, const int64_t* marker_tris);
/* The same grid built on a CUDA device (device < 0: the current one): face
 * matching by sorting on the GPU instead of FV_Grid's std::map
 * (FV_Grid.cpp:38-64), the reference's face order (Faces::sort,
 * GeometryUtilities.cpp:484-513), the geometry of FV_Grid.cpp:154-205 and
 * GeometryUtilities.cpp:289-325, calc_Delta_S (Solver.cpp:276-298) and the
 * Hilbert renumbering, all as kernels with the host builder's rounding. The
 * resulting mesh equals nf_mesh_from_arrays's bit for bit, and invalid input
 * gives the same error text. */
nf_mesh* nf_mesh_from_arrays_device(int64_t n_nodes, const double* nodes, int64_t n_cells, const int64_t* tets,
                                    int n_markers, const char* const* marker_names, const int* marker_types,
                                    const int64_t* marker_offsets, const int64_t* marker_tris, int device);

/* Concatenate meshes into one batched mesh (cells, faces and patches of case
 * b follow those of case b-1). Every case keeps its own patches. */
nf_mesh* nf_mesh_concat(int n, const nf_mesh* const* meshes);

int nf_mesh_get_info(const nf_mesh* m, nf_mesh_info* out);
/* Patch p: boundary type, first face, number of faces, owning case, name. */
int nf_mesh_get_patch(const nf_mesh* m, int p, int* type, int64_t* first_face, int64_t* n_faces,
                      int* case_index, char* name, size_t name_len);
/* Face-based grid in the reference's order (FV_Grid accessors): face_ij
 * [F][2] (ghost j >= n_interior_cells), S/ri/rj [F][3], vol and centroid for
 * all cells incl. ghosts [Nt], [Nt][3], dS [Nc][3]. Any pointer may be NULL. */
int nf_mesh_export(const nf_mesh* m, uint32_t* face_ij, double* S, double* ri, double* rj, double* vol,
                   double* centroid, double* dS);
/* Device cell index of every reference cell (the space-filling-curve
 * renumbering), [Nc]. */
int nf_mesh_get_permutation(const nf_mesh* m, int64_t* device_of_ref);
/* First cell of each case, [n_cases+1]. */
int nf_mesh_get_case_offsets(const nf_mesh* m, int64_t* cell_offsets);
void nf_mesh_destroy(nf_mesh* m);

typedef struct {
  int type;             /* NF_BC_* */
  double farfield[5];   /* freestream primitives (rho,u,v,w,p) seen by a far-field patch */
} nf_patch_bc;

typedef struct {
  int time_scheme;      /* NF_EXPLICIT_EULER / NF_TVD_RK3 */
  int spatial_order;    /* NF_FIRST_ORDER / NF_SECOND_ORDER */
  int limiter;          /* NF_LIMITER_NONE / NF_LIMITER_BARTH */
  int flux_scheme;      /* NF_FLUX_RUSANOV */
  int precision;        /* NF_PREC_* */
  int local_time_stepping; /* 0: one global dt (reference); 1: per-cell dt */
  int dt_from_current_state; /* 0: dt from the primitives of the last
                                evaluated stage, as the reference does
                                (Solver.cpp:250); 1: from the current state */
  int keep_stage_fields;     /* keep the gradient, limiter and flux balance of
                                the last stage for nf_get_field */
  double cfl;
  double t_end;         /* > 0: nf_advance clips dt so time never passes t_end */
  /* Boundary conditions per patch of the mesh, in patch order. NULL: every
   * patch uses the mesh's type and the far-field state below. */
  const nf_patch_bc* patches;
  int n_patches;
  double freestream[5]; /* Config::get_primvars_inf (rho,u,v,w,p) */
  int block_size;       /* 0: library default; > 0: fixed block size of the
                           gradient and flux kernels (no tuning) */
  int kernel_variant;   /* with block_size > 0: fast-kernel variant (see nf_tune) */
  /* Limiter ratchet (extension; the reference's Barth limiter is always live,
   * Numerics.hpp:148-250, and its residual stalls near a 1e-3 drop on steady
   * problems). Once a case's ratchet is on, every stage's limiter value of a
   * cell and variable is the minimum of the live value and the value kept so
   * far, and is kept; it can only tighten, so it stops changing and the
   * residual converges. It turns on for every case at step
   * limiter_ratchet_step (> 0; steps counted from nf_set_state), and in
   * nf_solve_steady for a case whose residual drop reaches
   * limiter_ratchet_drop (> 0). Both 0: off. */
  int64_t limiter_ratchet_step;
  double limiter_ratchet_drop;
  /* Extension: 1 gives far-field ghosts the isentropic density
   * (c_b^2 / (gamma s_b))^(1/(gamma-1)); 0 (default) keeps the reference's
   * inverted form (Numerics.cpp:149), which is exact only for a free-stream
   * density of 1. */
  int farfield_density_fix;
  int device;           /* CUDA device of the solver; -1 (default): the calling thread's current device */
} nf_params;

void nf_params_default(nf_params* p);

/* One solver takes at most 107,374,080 cells (its kernels use 32-bit row
 * offsets); a larger mesh is refused with a message (nf_last_error(NULL)) and
 * is split across solvers instead. */
nf_solver* nf_create(const nf_mesh* m, const nf_params* params);
/* U in reference cell order, AoS [n_cells][5]. Setting the state also sets
 * the primitives the next nf_calc_timestep reads. */
int nf_set_state(nf_solver* s, const double* U, int64_t n_cells);
int nf_get_state(nf_solver* s, double* U, int64_t n_cells);
/* Start copying the conserved state (reference cell order, [n_cells][5]) to
 * host memory U without waiting: the copy runs on a side stream and overlaps
 * the steps queued after this call, which do not change what is copied. U
 * must stay valid, and unread, until nf_snapshot_wait returns; with pinned
 * memory (cudaHostAlloc, cudaHostRegister) the copy is asynchronous, with
 * pageable memory the driver may complete it before returning. Snapshots may
 * overlap one another and the host never waits here: two device staging
 * buffers are used in turn, and a gather waits on the device for the copy out
 * of its buffer two snapshots back; the copies land in the order begun.
 * Replaces the synchronous solution read of Output::write_vtk_ascii
 * (Output.cpp:17-45) with one the step loop need not wait for. */
int nf_snapshot_begin(nf_solver* s, double* U, int64_t n_cells);
/* Wait until every snapshot begun so far is in host memory (NF_OK at once
 * when none is in flight). */
int nf_snapshot_wait(nf_solver* s);
/* The other direction: start copying a conserved state (reference cell
 * order, [n_cells][5]) from host memory U to the device on a side stream,
 * overlapping the work already queued, which it does not change; U must stay
 * valid and unchanged until nf_upload_wait returns (pinned memory makes the
 * copy asynchronous). One upload per solver between begin and commit: a
 * second begin before the commit is NF_ERR_ARG. nf_upload_commit then makes
 * that state the solver's state exactly as nf_set_state does, queued on the
 * device after the work already queued and after the copy, and returns
 * without waiting; NF_ERR_ARG without a begin. The next begin may follow at
 * once: uploads use two device staging buffers in turn, so its copy waits on
 * the device only for the state committed two uploads back to have been
 * taken. nf_upload_wait blocks until every upload's copy has landed, after
 * which their host buffers may change.
 * Together with the snapshots this streams independent states through one
 * solver with both copies overlapping the steps and the host never waiting
 * on a copy. No counterpart in the reference (it has no device memory). */
int nf_upload_begin(nf_solver* s, const double* U, int64_t n_cells);
int nf_upload_commit(nf_solver* s);
int nf_upload_wait(nf_solver* s);
/* U^n of the next step's TVD-RK3 combination (the reference's solution_old,
 * Solver.cpp:127-132), AoS [n_cells][5] in reference cell order; applies to
 * the next step only (afterwards U^n is the state, Solver.cpp:51).
 * nf_set_state makes U^n the state itself. NetFlux's own free-stream start
 * writes only solution (set_freestream_values, SolverData.cpp:50-58), so its
 * first RK3 step combines with a zero solution_old; the drop-in passes that
 * array through here to reproduce the reference program exactly. */
int nf_set_state_old(nf_solver* s, const double* U_old, int64_t n_cells);
/* Global dt = min_i CFL*vol_i/sum_d (|u_d|+c) dS_i,d (or the per-cell dt
 * with local time stepping, then *dt_out is its minimum). */
int nf_calc_timestep(nf_solver* s, double* dt_out);
int nf_set_timestep(nf_solver* s, double dt);
int nf_step(nf_solver* s);
/* One stage of a step (0, 1, 2 for TVD-RK3; 0 for explicit Euler), in order;
 * the last stage ends the step as nf_step does. Between stages the caller may
 * exchange halo primitives (nf_halo_pack / nf_halo_unpack) with the solvers
 * of the other parts of a mesh split across solvers. NF_ERR_ARG out of
 * order; nf_step and nf_advance refuse while a step begun here is open.
 * Stage-wise time integration has no counterpart in the reference, which
 * runs TVD_RK3 as one call (Solver.cpp:103-133). */
int nf_stage(nf_solver* s, int stage);
/* Halo exchange of a mesh split across solvers (one per part, each part with
 * two layers of halo cells; netflux_b200/partition.py builds the parts and
 * the exchange plan): nf_halo_pack gathers what the next stage (nf_stage)
 * reads of the n cells listed (device numbering, int64 on the device) into
 * the device buffer buf [10][n]: rows 0-4 the primitives, rows 5-9 the
 * conserved stage input (U, or the RK stage for stages 1 and 2);
 * nf_halo_unpack writes such a buffer into the listed cells. Both run on the
 * solver's stream and return when done. No counterpart in the reference (its
 * MPI decomposition is a commented-out sketch, Decomposition.cpp:3-51). */
int nf_halo_pack(nf_solver* s, const int64_t* cells, int64_t n, double* buf);
int nf_halo_unpack(nf_solver* s, const int64_t* cells, int64_t n, const double* buf);
/* The same split stepped on the device without host waits: nf_split_create
 * takes the parts' solvers (same parameters; each on its own device or
 * sharing one; peer access is enabled between their devices), nf_split_link
 * one direction of the exchange plan (the owner part `from`, the receiving
 * part `to`, n device cell indices on each side, host arrays).
 * nf_split_advance queues n steps: each step's dt on every part (with a
 * global dt, the minimum over the parts, reduced on the device into every
 * part), then per stage every halo (primitives and conserved stage input)
 * written by a kernel on the receiver's stream that reads the owner's (its
 * own GPU, or a peer GPU over NVLink), the parts' streams ordered by events,
 * then the stage on every part. nf_split_synchronize waits for the parts and returns the first
 * failing part's status. A part must not be stepped on its own while it is in
 * a split, and the split is destroyed before its parts (nf_split_destroy
 * waits for their streams). NULL from nf_split_create:
 * nf_split_last_error(NULL). No
 * counterpart in the reference (Decomposition.cpp:3-51 is a commented-out
 * sketch). */
typedef struct nf_split nf_split;
nf_split* nf_split_create(nf_solver* const* parts, int n_parts);
int nf_split_link(nf_split* sp, int from, int to, const int64_t* from_cells, const int64_t* to_cells, int64_t n);
int nf_split_advance(nf_split* sp, int64_t n_steps);
int nf_split_synchronize(nf_split* sp);
const char* nf_split_last_error(const nf_split* sp);
void nf_split_destroy(nf_split* sp);
/* n_steps x (calc_timestep + step) on the device; time (may be NULL) returns
 * the accumulated time. Uses a CUDA graph after the first call. */
int nf_advance(nf_solver* s, int64_t n_steps, double* time_out);
/* Steady solve with local time stepping (and the limiter ratchet of
 * nf_params when set): run steps until every case's
 * density residual (RMS of R_rho/vol over its cells, first stage of a step)
 * is at most tol times its value at the first step, or until max_steps. The
 * residuals are checked every check_every steps (CUDA graph replays in
 * between); a converged case is frozen (its cells keep their state exactly)
 * while the others continue. Per case (arrays of n_cases, any may be NULL):
 * steps to convergence (minus the steps run if it did not converge), the
 * first and last residual, and the device time until it converged. The
 * reference has no steady driver (it runs n_timesteps global steps,
 * Driver.cpp:31-57). */
int nf_solve_steady(nf_solver* s, double tol, int64_t max_steps, int check_every, int64_t* steps_per_case,
                    double* res0_per_case, double* res_per_case, double* ms_per_case);
/* The same with an absolute density-residual target per case
 * (res_target[n_cases]), e.g. the tolerance times the residual of a
 * free-stream start, so that a warm-started solve stops at the same residual
 * as the plain one. A case already at its target after the first step stops
 * there. */
int nf_solve_steady_to(nf_solver* s, const double* res_target, int64_t max_steps, int check_every,
                       int64_t* steps_per_case, double* res0_per_case, double* res_per_case, double* ms_per_case);

/* Density residual of the first stage of the last step: RMS and max of
 * R_rho,i / vol_i over all cells (per case: n_cases pairs). */
int nf_get_residual(nf_solver* s, double* rms_and_max, int n_cases);
int nf_get_field(nf_solver* s, int which, double* out, int64_t n_values);
/* Wait for queued work; report a device-side validity failure. */
int nf_synchronize(nf_solver* s);

/* Time the launch shapes of the gradient and flux kernels on the current
 * state and keep the fastest: block size (64 or 128 threads), whether each
 * thread issues its next variable's / face's loads before the current
 * arithmetic (variants 1, 3, 5), all of its loads before any arithmetic
 * (variants 6, 7), or L2 prefetches of its own rows first (variants 8, 9),
 * and a register cap for occupancy (none, variants 0-1 and 6; 6 / 8 resident
 * 128-thread blocks for FP64 / FP32, variants 2-3 and 8; 7 / 9, variants 4-5
 * and 9; 4 / 5, variant 7). config (may be NULL) receives {gradient block, gradient
 * variant, flux block, flux variant}. The state is unchanged. The reference
 * has no counterpart (it runs on one CPU thread). */
int nf_tune(nf_solver* s, int* config);
/* Fix the launch shapes instead of timing them: config = {gradient block,
 * gradient variant, flux block, flux variant} as nf_tune reports them (block
 * 32..128 in steps of 32, variant 0..9); NF_ERR_ARG otherwise. Used to
 * profile a given shape. No counterpart in the reference. */
int nf_set_launch_shapes(nf_solver* s, const int* config);

/* Kernel classes reported by nf_time_steps. */
#define NF_KERNEL_TIMESTEP 0
#define NF_KERNEL_GRADIENT 1
#define NF_KERNEL_FLUX 2
#define NF_KERNEL_OTHER 3
#define NF_KERNEL_COUNT 4

/* Run n_steps (calc_timestep + step each) and time them with CUDA events on
 * the solver's stream. per_kernel = 0: the steps run as in nf_advance (CUDA
 * graph) and *ms_total is their device time. per_kernel = 1: every kernel is
 * bracketed by events; kernel_ms[NF_KERNEL_COUNT] and
 * kernel_launches[NF_KERNEL_COUNT] receive the summed time and launch count
 * per kernel class. No counterpart in the reference (it has no timers beyond
 * a wall clock around Driver::solve, Driver.cpp:27,59-60). */
int nf_time_steps(nf_solver* s, int64_t n_steps, int per_kernel, double* ms_total, double* kernel_ms,
                  int64_t* kernel_launches);
const char* nf_last_error(const nf_solver* s);
void nf_destroy(nf_solver* s);

/* Residual norms without any device allocation: out[0] = sqrt(sum v^2 / n),
 * out[1] = max |v| over the n doubles at the device pointer `values`; `out`
 * is a device pointer to 2 doubles; work is queued on `stream` (a
 * cudaStream_t, NULL for the default stream) and is complete when the stream
 * reaches it. For callers that cannot allocate device memory when they need
 * the reduction (a host that gives the library a fixed memory pool and
 * forbids allocation after start-up, or a real-time loop that must not block
 * on the allocator). Its per-block partial sums live in a fixed 128 KiB array
 * in the library, so n is limited to 134,217,728; larger n returns
 * NF_ERR_ARG. The first call on a device looks up that array's address and
 * should come before any stream capture; calls that overlap on the GPU share
 * the array and race. It has no counterpart in the reference, which computes
 * no residual norms. */
int nf_residual_norms_noalloc(const double* values, int64_t n, double* out, void* stream);


/* Cap on the host threads one mesh build (nf_mesh_from_su2 / _from_arrays /
 * _concat) uses: 0 restores the default (the hardware's threads, at most 16),
 * n in 1..64 bounds it. For callers that build several meshes at once on
 * their own threads, so that builds times builder threads do not oversubscribe
 * the host. Process-wide; the environment variable NETFLUX_B200_HOST_THREADS,
 * when set, takes precedence. No reference counterpart (its grid builder is
 * single-threaded). */
int nf_set_host_threads(int n);

/* Whether one solver can take a mesh of n_cells interior cells and n_faces
 * faces: NF_OK, or NF_ERR_MESH with the reason in nf_last_error(NULL).
 * nf_create applies the same check. The stage kernels address the 20 rows of
 * the [20][stride] face-state arrays with 32-bit offsets (stride = n_cells
 * rounded up to 64), so at most 107,374,080 cells fit one solver; larger
 * meshes are split across solvers. No reference counterpart (the reference's
 * arrays are 64-bit indexed). */
int nf_check_mesh_size(int64_t n_cells, int64_t n_faces);

/* Self-test of the fast forms' reciprocal and reciprocal square root (a
 * single-precision estimate refined by two Newton-Raphson steps) on n
 * positive inputs; no reference counterpart. */
int nf_fastmath_selftest(const double* x, int64_t n, double* rcp_out, double* rsqrt_out);

/* ------------------------------------------------------------------------
 * Surrogate MLP for warm starts (extension; the reference has no learned
 * part). 7 inputs (cell centroid x, y, z, wall distance, Mach, bump height,
 * each normalised by the caller) -> 4 hidden layers of 128 SiLU units -> 5
 * outputs (the caller's normalised conserved variables). BF16 weights and
 * activations with FP32 accumulation on the tensor cores; FP32 master weights
 * and Adam (beta 0.9/0.999, eps 1e-8). Parameters (FP32, nf_mlp_param_count
 * values, padded shapes): W0 [128][16] (columns 0..6 inputs, column 7 bias),
 * W1, W2, W3 [128][128], b1, b2, b3 [128], W4 [16][128] (rows 0..4), b4 [16].
 * ------------------------------------------------------------------------ */
typedef struct nf_mlp nf_mlp;
int nf_mlp_param_count(void);
nf_mlp* nf_mlp_create(uint64_t seed);
const char* nf_mlp_last_error(const nf_mlp* m);
void nf_mlp_destroy(nf_mlp* m);
int nf_mlp_get_params(nf_mlp* m, float* out);
int nf_mlp_set_params(nf_mlp* m, const float* in);
/* Training set: features [n][7], targets [n][5] (copied to the device). */
int nf_mlp_set_data(nf_mlp* m, const float* features, const float* targets, int64_t n);
/* steps of Adam on uniformly drawn batches of `batch` samples (mean squared
 * error over the 5 outputs); loss_report[n_report]: the loss of the last step
 * of each of n_report equal segments; *ms_out the device time. */
int nf_mlp_train(nf_mlp* m, int64_t steps, int64_t batch, float lr, uint64_t seed, int n_report,
                 double* loss_report, double* ms_out);
/* Gradient of the mean squared error over the given samples (no update). */
int nf_mlp_gradients(nf_mlp* m, const float* features, const float* targets, int64_t n, float* grad_out,
                     double* loss_out);
/* Forward pass: out [n][5]; *ms_out the device time of the kernel. */
int nf_mlp_predict(nf_mlp* m, const float* features, int64_t n, float* out, double* ms_out);
/* Distance from each of n points [n][3] to the nearest of m wall points
 * [m][3] (the surrogate's wall-distance input), out [n]; FP32. */
int nf_wall_distance(const float* points, int64_t n, const float* wall, int64_t m, float* out);
/* D[128][N] = A[128][K] B[N][K]^T through the library's tcgen05 path
 * (A, B as BF16 bit patterns, row-major); 16 <= N, K <= 256, multiples of 16. */
int nf_mlp_gemm_selftest(const uint16_t* A, const uint16_t* B, int N, int K, float* D);

#ifdef __cplusplus
}
#endif
#endif /* NETFLUX_B200_H */
