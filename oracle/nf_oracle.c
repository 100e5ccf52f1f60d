/*
 * CPU restatement of NetFlux's explicit Euler step — ORACLE-ONLY TEST
 * INFRASTRUCTURE (see nf_oracle.h). Each function names the reference lines
 * it restates; expressions keep the reference's operand order.
 */
#include "nf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* EulerEqs constants (SolverData.hpp:129-131) */
static const double GAMMA = 1.4;
#define G1 (GAMMA - 1.0)
#define G1_INV (1.0 / (GAMMA - 1.0))

static inline double dmax(double a, double b) { return (a < b) ? b : a; } /* std::max */
static inline double dmin(double a, double b) { return (b < a) ? b : a; } /* std::min */
static inline int isign(double v) { return (v > 0.0) ? 1 : ((v < 0.0) ? -1 : 0); } /* Includes.hpp:100-104 */

/* EulerEqs::prim_to_cons (SolverData.hpp:165-177) */
static void prim_to_cons(const double* V, double* U) {
  U[0] = V[0];
  U[1] = V[0] * V[1];
  U[2] = V[0] * V[2];
  U[3] = V[0] * V[3];
  U[4] = G1_INV * V[4] + 0.5 * V[0] * (V[1] * V[1] + V[2] * V[2] + V[3] * V[3]);
}

/* EulerEqs::pressure (SolverData.hpp:194-201) */
static double pressure(const double* U) { return G1 * (U[4] - 0.5 / U[0] * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3])); }

/* EulerEqs::cons_to_prim (SolverData.hpp:179-192) */
static void cons_to_prim(const double* U, double* V) {
  V[0] = U[0];
  V[1] = U[1] / U[0];
  V[2] = U[2] / U[0];
  V[3] = U[3] / U[0];
  V[4] = pressure(U);
}

/* Vec3::normalized() and norm(): v / sqrt(v.v), sqrt(v.v) */
static void normalize(const double* S, double* n, double* area) {
  const double z = S[0] * S[0] + S[1] * S[1] + S[2] * S[2];
  const double a = sqrt(z);
  for (int d = 0; d < 3; d++) n[d] = z > 0.0 ? S[d] / a : S[d];
  if (area) *area = a;
}

/* EulerEqs::inviscid_flux (SolverData.hpp:239-255) */
static void inviscid_flux(const double* U, const double* n, double* F) {
  const double rho = U[0];
  const double p = pressure(U);
  const double vn = (U[1] * n[0] + U[2] * n[1] + U[3] * n[2]) / rho;
  F[0] = vn * rho;
  F[1] = vn * U[1] + p * n[0];
  F[2] = vn * U[2] + p * n[1];
  F[3] = vn * U[3] + p * n[2];
  F[4] = vn * (U[4] + p);
}

/* EulerEqs::conv_spectral_radii (SolverData.hpp:230-237) */
static double spectral_radius(const double* U, const double* n) {
  const double vn = (U[1] * n[0] + U[2] * n[1] + U[3] * n[2]) / U[0];
  return fabs(vn) + sqrt(GAMMA * pressure(U) / U[0]);
}

/* NumericalFlux::rusanov (Numerics.cpp:10-18) */
static void rusanov(const double* UL, const double* UR, const double* S, double* F) {
  double n[3], area;
  normalize(S, n, &area);
  const double sL = spectral_radius(UL, n), sR = spectral_radius(UR, n);
  double FR[5], FL[5];
  inviscid_flux(UR, n, FR);
  inviscid_flux(UL, n, FL);
  const double smax = dmax(sR, sL);
  const double a = area * 0.5;
  for (int k = 0; k < 5; k++) F[k] = a * (FR[k] + FL[k] - smax * (UR[k] - UL[k]));
}

/* BoundaryCondition::calc_ghost_val (Numerics.cpp:59-171) */
static int g_density_fix = 0; /* farfield_density_fix of the current run */

static void ghost(int type, const double* fs, const double* Vd, const double* S, double* Vg) {
  double n[3];
  normalize(S, n, NULL);
  if (type == 1) { /* BC_SlipWall */
    const double vn = Vd[1] * n[0] + Vd[2] * n[1] + Vd[3] * n[2];
    Vg[0] = Vd[0];
    for (int d = 0; d < 3; d++) Vg[d + 1] = Vd[d + 1] - 2 * vn * n[d];
    Vg[4] = Vd[4];
  } else if (type == 2) { /* BC_FarField, incl. its density and tangential-velocity quirks */
    const double c_fs = sqrt(GAMMA * fs[4] / fs[0]);
    const double s_fs = fs[4] * pow(fs[0], -GAMMA);
    const double vn_fs = n[0] * fs[1] + n[1] * fs[2] + n[2] * fs[3];
    const double vn_d = n[0] * Vd[1] + n[1] * Vd[2] + n[2] * Vd[3];
    const double c_d = sqrt(GAMMA * Vd[4] / Vd[0]);
    const double Rp = (vn_fs + c_fs > 0.0) ? vn_d + 2 * c_d / G1 : vn_fs + 2 * c_fs / G1;
    const double Rm = (vn_fs - c_fs > 0.0) ? vn_d - 2 * c_d / G1 : vn_fs - 2 * c_fs / G1;
    const double vn_b = 0.5 * (Rp + Rm);
    const double c_b = G1 / 4 * (Rp - Rm);
    double s_b;
    if (vn_fs > 0.0) {
      for (int d = 0; d < 3; d++) Vg[d + 1] = Vd[d + 1] + (vn_b - vn_d) * n[d];
      s_b = Vd[4] * pow(Vd[0], -GAMMA);
    } else {
      for (int d = 0; d < 3; d++) Vg[d + 1] = fs[d + 1] + (vn_fs - vn_b) * n[d];
      s_b = s_fs;
    }
    const double rho_b = g_density_fix ? pow(c_b * c_b / (GAMMA * s_b), G1_INV)
                                       : pow(GAMMA * s_b / (c_b * c_b), G1_INV);
    Vg[0] = rho_b;
    Vg[4] = c_b * c_b * rho_b / GAMMA;
  } else { /* BC_NoSlipWall */
    Vg[0] = Vd[0];
    Vg[1] = -Vd[1];
    Vg[2] = -Vd[2];
    Vg[3] = -Vd[3];
    Vg[4] = Vd[4];
  }
}

typedef struct {
  int64_t NC, NT, NF, NIF;
  double *V, *G, *L, *Vmax, *Vmin, *R;
  int* face_patch;
  int ratchet; /* limiter-ratchet extension: phi = min(live phi, Lf), kept in Lf */
  double* Lf;   /* starts at DBL_MAX */
} work_t;

/* Solver::evaluate_flux_balance (Solver.cpp:54-81) and what it calls. */
static void flux_balance(const nfo_mesh* m, const nfo_params* p, work_t* w, const double* U) {
  const int64_t NC = w->NC, NF = w->NF, NIF = w->NIF;
  memset(w->R, 0, sizeof(double) * 5 * NC);
  /* set_primvars (SolverData.cpp:37-48) */
  for (int64_t i = 0; i < NC; i++) cons_to_prim(U + 5 * i, w->V + 5 * i);
  /* set_constant_ghost_values (Solver.cpp:300-330) */
  for (int64_t f = NIF; f < NF; f++) {
    const int q = w->face_patch[f];
    const uint32_t i = m->face_ij[2 * f], j = m->face_ij[2 * f + 1];
    ghost(m->patch_type[q], m->patch_fs + 5 * q, w->V + 5 * (int64_t)i, m->S + 3 * f, w->V + 5 * (int64_t)j);
  }
  if (p->spatial_order == 1) {
    /* calc_green_gauss_gradient (Numerics.hpp:86-128); (k,d) at 5*d+k */
    memset(w->G, 0, sizeof(double) * 15 * NC);
    for (int64_t f = 0; f < NF; f++) {
      const int64_t i = m->face_ij[2 * f], j = m->face_ij[2 * f + 1];
      const double* S = m->S + 3 * f;
      for (int k = 0; k < 5; k++) {
        const double uf = 0.5 * (w->V[5 * i + k] + w->V[5 * j + k]);
        for (int d = 0; d < 3; d++) {
          const double t = uf * S[d];
          w->G[15 * i + 5 * d + k] += t / m->vol[i];
          if (j < NC) w->G[15 * j + 5 * d + k] -= t / m->vol[j];
        }
      }
    }
    if (p->limiter == 1) {
      /* calc_max_and_min_values (Numerics.hpp:253-292) */
      for (int64_t x = 0; x < 5 * NC; x++) {
        w->Vmax[x] = -DBL_MAX;
        w->Vmin[x] = DBL_MAX;
      }
      for (int64_t f = 0; f < NF; f++) {
        const int64_t i = m->face_ij[2 * f], j = m->face_ij[2 * f + 1];
        for (int k = 0; k < 5; k++) {
          const double a = w->V[5 * i + k], b = w->V[5 * j + k];
          w->Vmax[5 * i + k] = dmax(w->Vmax[5 * i + k], dmax(a, b));
          if (j < NC) w->Vmax[5 * j + k] = dmax(w->Vmax[5 * j + k], dmax(a, b));
          w->Vmin[5 * i + k] = dmin(w->Vmin[5 * i + k], dmin(a, b));
          if (j < NC) w->Vmin[5 * j + k] = dmin(w->Vmin[5 * j + k], dmin(a, b));
        }
      }
      /* calc_barth_limiter (Numerics.hpp:148-250) */
      const double EPS = DBL_EPSILON;
      for (int64_t x = 0; x < 5 * NC; x++) w->L[x] = DBL_MAX;
      for (int64_t f = 0; f < NF; f++) {
        const int64_t i = m->face_ij[2 * f], j = m->face_ij[2 * f + 1];
        for (int side = 0; side < 2; side++) {
          const int64_t c = side ? j : i;
          if (side && j >= NC) break;
          const double* r = side ? m->rj + 3 * f : m->ri + 3 * f;
          const double* g = w->G + 15 * c;
          for (int k = 0; k < 5; k++) {
            double d2 = g[k] * r[0] + g[5 + k] * r[1] + g[10 + k] * r[2];
            d2 = isign(d2) * (fabs(d2) + EPS);
            double fc;
            if (d2 > 0.0) fc = dmin(1.0, (w->Vmax[5 * c + k] - w->V[5 * c + k]) / d2);
            else if (d2 < 0.0) fc = dmin(1.0, (w->Vmin[5 * c + k] - w->V[5 * c + k]) / d2);
            else fc = 1.0;
            w->L[5 * c + k] = dmin(w->L[5 * c + k], fc);
          }
        }
      }
      if (w->ratchet)
        for (int64_t x = 0; x < 5 * NC; x++) w->Lf[x] = w->L[x] = dmin(w->L[x], w->Lf[x]);
    } else {
      for (int64_t x = 0; x < 5 * NC; x++) w->L[x] = 1.0; /* SolverData.cpp:331 */
    }
  }
  /* EulerSolver::evaluate_inviscid_fluxes (Solver.cpp:144-230) with
   * calc_reconstructed_value (Solver.hpp:81-112) */
  for (int64_t f = 0; f < NF; f++) {
    const int64_t i = m->face_ij[2 * f], j = m->face_ij[2 * f + 1];
    double VL[5], VR[5], UL[5], UR[5], F[5];
    for (int side = 0; side < 2; side++) {
      const int64_t c = side ? j : i;
      double* out = side ? VR : VL;
      if (side && j >= NC) break;
      const double* r = side ? m->rj + 3 * f : m->ri + 3 * f;
      for (int k = 0; k < 5; k++) {
        if (p->spatial_order == 1) {
          const double* g = w->G + 15 * c;
          out[k] = w->V[5 * c + k] + w->L[5 * c + k] * (g[k] * r[0] + g[5 + k] * r[1] + g[10 + k] * r[2]);
        } else {
          out[k] = w->V[5 * c + k];
        }
      }
    }
    if (j >= NC) {
      const int q = w->face_patch[f];
      ghost(m->patch_type[q], m->patch_fs + 5 * q, VL, m->S + 3 * f, VR); /* Solver.cpp:212 */
    }
    prim_to_cons(VL, UL);
    prim_to_cons(VR, UR);
    rusanov(UL, UR, m->S + 3 * f, F);
    for (int k = 0; k < 5; k++) {
      w->R[5 * i + k] -= F[k];
      if (j < NC) w->R[5 * j + k] += F[k];
    }
  }
}

/* EulerSolver::calc_timestep (Solver.cpp:232-274) from the primitives in V;
 * with local time stepping the per-cell values go to dtl. */
static int timestep(const nfo_mesh* m, const nfo_params* p, const double* V, double* dt_out, double* dtl) {
  double dt = DBL_MAX;
  for (int64_t i = 0; i < m->n_cells; i++) {
    const double* v = V + 5 * i;
    const double c = sqrt(GAMMA * v[4] / v[0]);
    const double sx = (fabs(v[1]) + c) * m->dS[3 * i];
    const double sy = (fabs(v[2]) + c) * m->dS[3 * i + 1];
    const double sz = (fabs(v[3]) + c) * m->dS[3 * i + 2];
    const double d = p->cfl * m->vol[i] / (sx + sy + sz);
    if (dtl) dtl[i] = d;
    dt = dmin(dt, d);
  }
  *dt_out = dt;
  if (!(isfinite(dt) && dt > 0.0)) return 5;
  return 0;
}

/* Stage s of explicit Euler / TVD-RK3 from the flux balance in w->R
 * (Solver.cpp:83-133): U is the stage input and receives the output. */
static void stage_update(const nfo_mesh* m, const nfo_params* p, const work_t* w, double* U, const double* Un, int s,
                         double dt, const double* dtl) {
  for (int64_t i = 0; i < w->NC; i++) {
    const double h = dtl ? dtl[i] : dt;
    for (int k = 0; k < 5; k++) {
      double* u = U + 5 * i + k;
      const double r = w->R[5 * i + k];
      if (p->time_scheme == 0 || s == 0) /* Solver.cpp:97-98, 123-124 */
        *u += h / m->vol[i] * r;
      else if (s == 1) /* Solver.cpp:127-128 */
        *u = 3.0 / 4.0 * Un[5 * i + k] + 1.0 / 4.0 * *u + 1.0 / 4.0 * h / m->vol[i] * r;
      else /* Solver.cpp:131-132 */
        *u = 1.0 / 3.0 * Un[5 * i + k] + 2.0 / 3.0 * *u + 2.0 / 3.0 * h / m->vol[i] * r;
    }
  }
}

static void free_work(work_t* w) {
  free(w->V);
  free(w->G);
  free(w->L);
  free(w->Vmax);
  free(w->Vmin);
  free(w->R);
  free(w->face_patch);
  free(w->Lf);
}

int nfo_timestep_of(const nfo_mesh* m, const nfo_params* p, const double* U, double* dt_out, double* dtl) {
  if (!m || !p || !U || !dt_out || m->n_cells <= 0) return 2;
  double* V = (double*)malloc(sizeof(double) * 5 * m->n_cells);
  if (!V) return 2;
  for (int64_t i = 0; i < m->n_cells; i++) cons_to_prim(U + 5 * i, V + 5 * i);
  const int rc = timestep(m, p, V, dt_out, dtl);
  free(V);
  return rc;
}

int nfo_stage(const nfo_mesh* m, const nfo_params* p, double* U, const double* Un, int stage, double dt,
              const double* dtl) {
  if (!m || !p || !U || !Un || m->n_cells <= 0 || m->n_faces < m->n_interior_faces || stage < 0 || stage > 2 ||
      p->limiter_ratchet_step > 0)
    return 2;
  work_t w;
  memset(&w, 0, sizeof w);
  w.NC = m->n_cells;
  w.NF = m->n_faces;
  w.NIF = m->n_interior_faces;
  w.NT = w.NC + (w.NF - w.NIF);
  w.V = (double*)calloc((size_t)(5 * w.NT), sizeof(double));
  w.G = (double*)calloc((size_t)(15 * w.NC), sizeof(double));
  w.L = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.Vmax = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.Vmin = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.R = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.face_patch = (int*)calloc((size_t)w.NF, sizeof(int));
  int rc = 0;
  if (!w.V || !w.G || !w.L || !w.Vmax || !w.Vmin || !w.R || !w.face_patch) {
    rc = 2;
  } else {
    g_density_fix = p->farfield_density_fix;
    for (int q = 0; q < m->n_patches; q++)
      for (int64_t f = m->patch_first[q]; f < m->patch_first[q] + m->patch_n[q]; f++) w.face_patch[f] = q;
    flux_balance(m, p, &w, U);
    stage_update(m, p, &w, U, Un, stage, dt, dtl);
  }
  free_work(&w);
  return rc;
}

int nfo_run(const nfo_mesh* m, const nfo_params* p, double* U, int64_t n_steps, double* dt_hist, double* V_out,
            double* grad_out, double* lim_out, double* R_out, double* res_out, double* time_out) {
  if (!m || !p || !U || m->n_cells <= 0 || m->n_faces < m->n_interior_faces) return 2;
  work_t w;
  w.NC = m->n_cells;
  w.NF = m->n_faces;
  w.NIF = m->n_interior_faces;
  w.NT = w.NC + (w.NF - w.NIF);
  w.V = (double*)calloc((size_t)(5 * w.NT), sizeof(double));
  w.G = (double*)calloc((size_t)(15 * w.NC), sizeof(double));
  w.L = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.Vmax = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.Vmin = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.R = (double*)calloc((size_t)(5 * w.NC), sizeof(double));
  w.face_patch = (int*)calloc((size_t)w.NF, sizeof(int));
  g_density_fix = p->farfield_density_fix;
  w.ratchet = 0;
  w.Lf = p->limiter_ratchet_step > 0 ? (double*)malloc(sizeof(double) * 5 * w.NC) : NULL;
  if (w.Lf)
    for (int64_t x = 0; x < 5 * w.NC; x++) w.Lf[x] = DBL_MAX;
  double* Un = (double*)malloc(sizeof(double) * 5 * w.NC);
  double* dtl = p->local_time_stepping ? (double*)malloc(sizeof(double) * w.NC) : NULL;
  double* Vdt = (double*)malloc(sizeof(double) * 5 * w.NC);
  int rc = 0;
  double time = 0.0;
  const int n_stages = p->time_scheme == 1 ? 3 : 1;
  if (!w.V || !w.G || !w.L || !w.Vmax || !w.Vmin || !w.R || !w.face_patch || !Un || !Vdt ||
      (p->local_time_stepping && !dtl) || (p->limiter_ratchet_step > 0 && !w.Lf)) {
    rc = 2;
    goto done;
  }
  for (int q = 0; q < m->n_patches; q++)
    for (int64_t f = m->patch_first[q]; f < m->patch_first[q] + m->patch_n[q]; f++) w.face_patch[f] = q;
  for (int64_t i = 0; i < w.NC; i++) cons_to_prim(U + 5 * i, w.V + 5 * i);
  memcpy(Un, p->U_old_first ? p->U_old_first : U, sizeof(double) * 5 * w.NC);
  for (int64_t n = 0; n < n_steps; n++) {
    /* Driver::solve: calc_timestep then step. The primitives are those of the
     * last evaluated stage (Solver.cpp:250) unless the extension asks for
     * the current state's. */
    double dt;
    if (p->dt_from_current_state) {
      for (int64_t i = 0; i < w.NC; i++) cons_to_prim(U + 5 * i, Vdt + 5 * i);
      rc = timestep(m, p, Vdt, &dt, dtl);
    } else {
      rc = timestep(m, p, w.V, &dt, dtl);
    }
    if (rc) goto done;
    if (p->t_end > 0.0) {
      const double left = p->t_end - time;
      dt = (left < dt) ? left : dt;
    }
    if (dt_hist) dt_hist[n] = dt;
    for (int s = 0; s < n_stages; s++) {
      w.ratchet = p->limiter_ratchet_step > 0 && n >= p->limiter_ratchet_step;
      flux_balance(m, p, &w, U);
      if (s == 0 && res_out) {
        double ss = 0.0, mx = 0.0;
        for (int64_t i = 0; i < w.NC; i++) {
          const double r = w.R[5 * i] / m->vol[i];
          ss += r * r;
          mx = fmax(mx, fabs(r));
        }
        res_out[2 * n] = sqrt(ss / (double)w.NC);
        res_out[2 * n + 1] = mx;
      }
      stage_update(m, p, &w, U, Un, s, dt, dtl);
    }
    memcpy(Un, U, sizeof(double) * 5 * w.NC); /* solution_old = solution (Solver.cpp:51) */
    time += dt;
  }
  if (time_out) *time_out = time;
  if (V_out) memcpy(V_out, w.V, sizeof(double) * 5 * w.NT);
  if (grad_out) memcpy(grad_out, w.G, sizeof(double) * 15 * w.NC);
  if (lim_out) memcpy(lim_out, w.L, sizeof(double) * 5 * w.NC);
  if (R_out) memcpy(R_out, w.R, sizeof(double) * 5 * w.NC);
done:
  free(w.V);
  free(w.G);
  free(w.L);
  free(w.Vmax);
  free(w.Vmin);
  free(w.R);
  free(w.face_patch);
  free(w.Lf);
  free(Un);
  free(dtl);
  free(Vdt);
  return rc;
}
