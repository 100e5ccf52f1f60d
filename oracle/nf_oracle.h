/*
 * CPU restatement of NetFlux's explicit Euler step — ORACLE-ONLY TEST
 * INFRASTRUCTURE. Used by tests/ and bench.py's CPU baseline as the checker,
 * never by the product path.
 *
 * It runs the reference's face loops in the reference's cell and face
 * numbering (Solver.cpp:54-298, Numerics.hpp:86-292, Numerics.cpp:10-171,
 * SolverData.hpp:165-262, SolverData.cpp:37-58) on a face-based grid given as
 * arrays (the FV_Grid accessors). Compiled with -ffp-contract=off so it rounds
 * like the reference's x86-64 build. Pinned against the reference itself
 * (oracle/_ref, built from the unmodified sources) by tests/test_oracle.py.
 */
#ifndef NF_ORACLE_H
#define NF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int64_t n_cells;           /* interior cells */
  int64_t n_faces;           /* all faces */
  int64_t n_interior_faces;
  const uint32_t* face_ij;   /* [F][2]; j >= n_cells is a ghost */
  const double* S;           /* [F][3] */
  const double* ri;          /* [F][3] */
  const double* rj;          /* [F][3] */
  const double* vol;         /* [n_cells] (at least) */
  const double* dS;          /* [n_cells][3] */
  int n_patches;
  const int* patch_type;     /* 0 no-slip, 1 slip, 2 far field */
  const int64_t* patch_first;
  const int64_t* patch_n;
  const double* patch_fs;    /* [n_patches][5] free-stream primitives per patch */
} nfo_mesh;

typedef struct {
  int time_scheme;           /* 0 explicit Euler, 1 TVD-RK3 */
  int spatial_order;         /* 0 first, 1 second */
  int limiter;               /* 0 none, 1 Barth */
  int local_time_stepping;   /* extension: per-cell dt */
  int dt_from_current_state; /* extension: dt from V(U^n) instead of the last stage's primitives */
  double cfl;
  double t_end;              /* extension: > 0 clips dt at t_end */
  int64_t limiter_ratchet_step; /* extension: > 0 ratchets the Barth limiter from that step on (0-based):
                                   every stage takes the minimum of its live value and the value
                                   it kept, and keeps that; 0 keeps the limiter live */
  int farfield_density_fix;      /* extension: 1 = isentropic far-field ghost density instead of the
                                    reference's inverted form (Numerics.cpp:149) */
  const double* U_old_first;     /* U^n of the first step's RK3 combination ([n_cells][5]); NULL = the
                                    initial state. The reference's free-stream start leaves its
                                    solution_old at zero (SolverData.cpp:50-58, Solver.cpp:127-132) */
} nfo_params;

/* Advance U (AoS [n_cells][5], in/out) by n_steps of calc_timestep + step.
 * Optional outputs (NULL to skip): dt per step, the last evaluated stage's
 * primitives incl. ghosts [n_cells+n_ghost][5], gradient [n_cells][15]
 * (column-major 5x3), limiter [n_cells][5], flux balance [n_cells][5], and per
 * step the RMS and max of R_rho/vol of the first stage [n_steps][2].
 * Returns 0, or 5 when a dt is invalid (the reference throws), 2 on bad input. */
int nfo_run(const nfo_mesh* m, const nfo_params* p, double* U, int64_t n_steps, double* dt_hist, double* V_out,
            double* grad_out, double* lim_out, double* R_out, double* res_out, double* time_out);

/* Pieces of a step, for tests that split a step across ranks and exchange
 * halo states between stages (extension; same arithmetic as nfo_run):
 * nfo_timestep_of computes calc_timestep from the primitives of U (the
 * dt_from_current_state form): the minimum in dt_out and, when dtl is not
 * NULL, the per-cell values. nfo_stage runs stage `stage` (0..2; 0 only for
 * explicit Euler) on U (stage input in, stage output out) with Un the step's
 * starting state and the step's dt, or the per-cell dtl when not NULL. The
 * limiter ratchet is not supported there (2). Both return 0, 5 for an
 * invalid dt, 2 on bad input. */
int nfo_timestep_of(const nfo_mesh* m, const nfo_params* p, const double* U, double* dt_out, double* dtl);
int nfo_stage(const nfo_mesh* m, const nfo_params* p, double* U, const double* Un, int stage, double dt,
              const double* dtl);

#ifdef __cplusplus
}
#endif
#endif
