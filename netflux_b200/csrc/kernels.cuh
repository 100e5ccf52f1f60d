// Per-cell gather kernels of one explicit step on the device mesh.
//
// Layout (all arrays resident in HBM for the whole run; cell c is the c-th
// cell along the Hilbert curve):
//   cell SoA    U, W, V[2], phi : [5][stride], grad : [15][stride] (k*3+d)
//               vol, dt_local   : [stride], dS : [3][stride]
//   cell slots  slot : [4][stride] = face << 1 | side (side 0: the cell is the
//               face's owner i, side 1: its neighbour j), -1 = no face. The 4
//               slots of a cell list its faces in the reference's global face
//               order, which is the order the reference accumulates the
//               gradient and the flux balance of that cell in
//               (FV_Grid.cpp:135-137, 207-227), so every per-cell sum below
//               adds the same terms in the same order as the face loops of
//               Numerics.hpp:112-127 and Solver.cpp:171-229.
//   face SoA    fi, fj : [F] owner / neighbour cell (fj < 0: boundary face of
//               patch -fj-1); S, nhat, ri, rj : [3][F]; area : [F]
// Each face's flux is evaluated by both of its cells with the owner on the
// left, so both see bit-identical values; no atomics, deterministic results.
#pragma once

#include <cuda_runtime.h>

#include "euler.cuh"

namespace nf {

// Geometry and topology of the device mesh (T: double, or float for the
// mixed-precision face work).
template <typename T>
struct MeshView {
  int n;          // interior cells
  int stride;     // SoA stride of cell arrays
  int n_faces;
  const int* __restrict__ slot;
  const int* __restrict__ fi;
  const int* __restrict__ fj;
  const T* __restrict__ S;
  const T* __restrict__ nhat;
  const T* __restrict__ area;
  const T* __restrict__ ri;
  const T* __restrict__ rj;
  const double* __restrict__ vol;
  const double* __restrict__ dS;
  const PatchBC* __restrict__ patches;
};

struct StageArgs {
  int second_order;      // SpatialOrder::Second
  int barth;             // Limiter::Barth
  int scheme;            // 0 explicit Euler, 1 TVD-RK3
  int stage;             // 0, 1, 2
  int local_dt;
  const double* Vin;     // primitives of the stage input [5][stride]
  double* grad;          // [15][stride]
  double* phi;           // [5][stride]
  const double* Uin;     // stage input state (own cell)
  const double* Un;      // U^n (stages 1, 2)
  double* Uout;          // may alias Uin
  double* Vout;          // primitives of Uout
  double* R;             // optional flux-balance dump [5][stride]
  double* res_cell;      // optional R_rho / vol per cell (first stage)
  const double* dt_local;
  const double* scal;    // device scalars: [0] dt (min target), [1] time, [2] t_end
  unsigned* status;
  // mixed precision: FP32 copies of the primitives and gradients
  const float* Vin32;
  float* Vout32;
  float* grad32;
  float* phi32;
};

enum : int { kScalDtMin = 0, kScalTime = 1, kScalTEnd = 2, kScalDtUsed = 3, kScalCount = 8 };

__device__ __forceinline__ double stage_dt(const double* scal) {
  double dt = scal[kScalDtMin];
  const double t_end = scal[kScalTEnd];
  if (t_end > 0.0) {
    const double left = t_end - scal[kScalTime];
    dt = (left < dt) ? left : dt;
  }
  return dt;
}

// ---------------------------------------------------------------------------
// Green-Gauss gradient + min/max + Barth limiter of one cell
// (calc_green_gauss_gradient, calc_max_and_min_values, calc_barth_limiter,
//  Numerics.hpp:86-292). Ghost states at boundary faces are the cell-centre
// ghosts of set_constant_ghost_values (Solver.cpp:300-330).
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) gradient_limiter_kernel(MeshView<T> m, StageArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.n) return;
  const int st = m.stride;
  T Vc[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if constexpr (sizeof(T) == 8) Vc[k] = T(a.Vin[k * st + c]);
    else Vc[k] = a.Vin32[k * st + c];
  }
  const T vol = T(m.vol[c]);
  T g[5][3];
  T vmax[5], vmin[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    g[k][0] = g[k][1] = g[k][2] = T(0);
    vmax[k] = -std::numeric_limits<T>::max();
    vmin[k] = std::numeric_limits<T>::max();
  }
  T gsum[5][3];  // fast form: sum the face terms, divide once
  if constexpr (!kRef) {
#pragma unroll
    for (int k = 0; k < 5; k++) gsum[k][0] = gsum[k][1] = gsum[k][2] = T(0);
  }
  int slots[4];
#pragma unroll
  for (int s = 0; s < 4; s++) slots[s] = m.slot[s * st + c];
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const int sl = slots[s];
    if (sl < 0) continue;
    const int f = sl >> 1;
    const bool own = (sl & 1) == 0;
    const T S[3] = {m.S[f], m.S[m.n_faces + f], m.S[2 * m.n_faces + f]};
    const int o = own ? m.fj[f] : m.fi[f];
    T Vo[5];
    if (o >= 0) {
#pragma unroll
      for (int k = 0; k < 5; k++) {
        if constexpr (sizeof(T) == 8) Vo[k] = T(a.Vin[k * st + o]);
        else Vo[k] = a.Vin32[k * st + o];
      }
    } else {
      const T nh[3] = {m.nhat[f], m.nhat[m.n_faces + f], m.nhat[2 * m.n_faces + f]};
      ghost_state<T>(m.patches[-o - 1], Vc, nh, Vo);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
      // U_face = 0.5 * (V_i + V_j); the sum commutes exactly
      const T uf = T(0.5) * (Vc[k] + Vo[k]);
#pragma unroll
      for (int d = 0; d < 3; d++) {
        const T t = uf * S[d];
        if constexpr (kRef) {
          g[k][d] = own ? g[k][d] + t / vol : g[k][d] - t / vol;
        } else {
          gsum[k][d] = own ? gsum[k][d] + t : gsum[k][d] - t;
        }
      }
      // max(V_i, V_j) / min(V_i, V_j) with the face's own operand order
      const T vi = own ? Vc[k] : Vo[k], vj = own ? Vo[k] : Vc[k];
      vmax[k] = rmax(vmax[k], rmax(vi, vj));
      vmin[k] = rmin(vmin[k], rmin(vi, vj));
    }
  }
  if constexpr (!kRef) {
    const T iv = T(1) / vol;
#pragma unroll
    for (int k = 0; k < 5; k++)
#pragma unroll
      for (int d = 0; d < 3; d++) g[k][d] = gsum[k][d] * iv;
  }
  T phi[5];
  if (a.barth) {
#pragma unroll
    for (int k = 0; k < 5; k++) phi[k] = std::numeric_limits<T>::max();
#pragma unroll
    for (int s = 0; s < 4; s++) {
      const int sl = slots[s];
      if (sl < 0) continue;
      const int f = sl >> 1;
      const T* rr = (sl & 1) ? m.rj : m.ri;
      const T r[3] = {rr[f], rr[m.n_faces + f], rr[2 * m.n_faces + f]};
#pragma unroll
      for (int k = 0; k < 5; k++) {
        T d2 = (g[k][0] * r[0] + g[k][1] * r[1]) + g[k][2] * r[2];
        const T sg = (d2 > T(0)) ? T(1) : ((d2 < T(0)) ? T(-1) : T(0));
        d2 = sg * (fabs(d2) + Gas<T>::eps);
        T fc;
        if (d2 > T(0)) fc = rmin(T(1), (vmax[k] - Vc[k]) / d2);
        else if (d2 < T(0)) fc = rmin(T(1), (vmin[k] - Vc[k]) / d2);
        else fc = T(1);
        phi[k] = rmin(phi[k], fc);
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 5; k++) phi[k] = T(1);
  }
#pragma unroll
  for (int k = 0; k < 5; k++) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if constexpr (sizeof(T) == 8) a.grad[(k * 3 + d) * st + c] = g[k][d];
      else a.grad32[(k * 3 + d) * st + c] = g[k][d];
    }
    if constexpr (sizeof(T) == 8) a.phi[k * st + c] = phi[k];
    else a.phi32[k * st + c] = phi[k];
  }
}

// Limited reconstruction V_face = V + phi (.) (grad V . r) (Numerics.hpp:135-145).
template <typename T>
__device__ __forceinline__ void reconstruct(const T V[5], const T g[5][3], const T phi[5], const T r[3], T out[5]) {
#pragma unroll
  for (int k = 0; k < 5; k++) out[k] = V[k] + phi[k] * ((g[k][0] * r[0] + g[k][1] * r[1]) + g[k][2] * r[2]);
}

template <typename T>
__device__ __forceinline__ void load_cell(const StageArgs& a, int st, int c, bool second, T V[5], T g[5][3], T phi[5]) {
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if constexpr (sizeof(T) == 8) V[k] = a.Vin[k * st + c];
    else V[k] = a.Vin32[k * st + c];
  }
  if (second) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if constexpr (sizeof(T) == 8) g[k][d] = a.grad[(k * 3 + d) * st + c];
        else g[k][d] = a.grad32[(k * 3 + d) * st + c];
      }
      if constexpr (sizeof(T) == 8) phi[k] = a.phi[k * st + c];
      else phi[k] = a.phi32[k * st + c];
    }
  }
}

// ---------------------------------------------------------------------------
// Face fluxes, flux balance R and the stage update of one cell
// (evaluate_inviscid_fluxes Solver.cpp:144-230, rusanov Numerics.cpp:10-18,
//  TVD_RK3 Solver.cpp:103-133, explicit_euler 83-101), then the primitives of
// the new state for the next stage (set_primvars, SolverData.cpp:37-48).
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) flux_update_kernel(MeshView<T> m, StageArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.n) return;
  const int st = m.stride;
  const bool second = a.second_order != 0;
  T Vc[5], gc[5][3], phic[5];
  load_cell<T>(a, st, c, second, Vc, gc, phic);
  double R[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int s = 0; s < 4; s++) {
    const int sl = m.slot[s * st + c];
    if (sl < 0) continue;
    const int f = sl >> 1;
    const bool own = (sl & 1) == 0;
    const T nh[3] = {m.nhat[f], m.nhat[m.n_faces + f], m.nhat[2 * m.n_faces + f]};
    const T area = m.area[f];
    T VL[5], VR[5];
    const T* rc = own ? m.ri : m.rj;  // this cell's centroid-to-face vector
    const T r_own[3] = {rc[f], rc[m.n_faces + f], rc[2 * m.n_faces + f]};
    T* Vown = own ? VL : VR;
    T* Voth = own ? VR : VL;
    if (second) reconstruct<T>(Vc, gc, phic, r_own, Vown);
    else {
#pragma unroll
      for (int k = 0; k < 5; k++) Vown[k] = Vc[k];
    }
    const int o = own ? m.fj[f] : m.fi[f];
    if (o >= 0) {
      T Vo[5], go[5][3], phio[5];
      load_cell<T>(a, st, o, second, Vo, go, phio);
      if (second) {
        const T* ro = own ? m.rj : m.ri;
        const T r_oth[3] = {ro[f], ro[m.n_faces + f], ro[2 * m.n_faces + f]};
        reconstruct<T>(Vo, go, phio, r_oth, Voth);
      } else {
#pragma unroll
        for (int k = 0; k < 5; k++) Voth[k] = Vo[k];
      }
    } else {
      // boundary face: ghost from the reconstructed face value (Solver.cpp:212)
      ghost_state<T>(m.patches[-o - 1], VL, nh, VR);
    }
    T F[5];
    if constexpr (kRef) {
      T UL[5], UR[5];
      prim_to_cons<T, kRef>(VL, UL);
      prim_to_cons<T, kRef>(VR, UR);
      rusanov_ref<T>(UL, UR, nh, area, F);
    } else {
      rusanov_fast<T>(VL, VR, nh, area, F);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) R[k] = own ? R[k] - double(F[k]) : R[k] + double(F[k]);
  }

  // ---- stage update (FP64) ----
  const double vol = m.vol[c];
  const double dt = a.local_dt ? a.dt_local[c] : stage_dt(a.scal);
  double U[5], Uo[5];
#pragma unroll
  for (int k = 0; k < 5; k++) U[k] = a.Uin[k * st + c];
  if (a.scheme == 1 && a.stage > 0) {
#pragma unroll
    for (int k = 0; k < 5; k++) Uo[k] = a.Un[k * st + c];
  }
  double Unew[5];
  if (a.scheme == 0 || a.stage == 0) {
    const double q = dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = U[k] + q * R[k];
  } else if (a.stage == 1) {
    const double q = 1.0 / 4.0 * dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 3.0 / 4.0 * Uo[k] + 1.0 / 4.0 * U[k] + q * R[k];
  } else {
    const double q = 2.0 / 3.0 * dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 1.0 / 3.0 * Uo[k] + 2.0 / 3.0 * U[k] + q * R[k];
  }
  double Vn[5];
  cons_to_prim<double, kRef>(Unew, Vn);
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    a.Uout[k * st + c] = Unew[k];
    a.Vout[k * st + c] = Vn[k];
    if (a.Vout32) a.Vout32[k * st + c] = float(Vn[k]);
    finite = finite && isfinite(R[k]) && isfinite(Unew[k]);
  }
  if (a.R) {
#pragma unroll
    for (int k = 0; k < 5; k++) a.R[k * st + c] = R[k];
  }
  if (a.res_cell) a.res_cell[c] = R[0] / vol;
  if (!finite) atomicOr(a.status, kErrNonFinite);
  else if (!(Vn[0] > 0.0) || !(Vn[4] > 0.0)) atomicOr(a.status, kErrNonPhysical);
}

// ---------------------------------------------------------------------------
// Time step (EulerSolver::calc_timestep, Solver.cpp:232-274): per cell
// CFL*vol / sum_d (|u_d| + c) dS_d from the given primitives; the global dt
// is their minimum (atomicMin on the bit pattern, exact and order-free for
// positive doubles).
// ---------------------------------------------------------------------------
struct DtArgs {
  const double* V;
  double cfl;
  double* dt_local;  // per-cell dt, or nullptr
  unsigned long long* dt_min_bits;
  unsigned* status;
};

template <bool kRef>
__global__ void __launch_bounds__(256) timestep_kernel(MeshView<double> m, DtArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = DBL_MAX;
  if (c < m.n) {
    const int st = m.stride;
    const double V0 = a.V[c], V1 = a.V[st + c], V2 = a.V[2 * st + c], V3 = a.V[3 * st + c], V4 = a.V[4 * st + c];
    const double cs = sqrt(Gas<double>::gamma * V4 / V0);
    const double sx = (fabs(V1) + cs) * m.dS[c];
    const double sy = (fabs(V2) + cs) * m.dS[st + c];
    const double sz = (fabs(V3) + cs) * m.dS[2 * st + c];
    const double d = a.cfl * m.vol[c] / (sx + sy + sz);
    if (a.dt_local) a.dt_local[c] = d;
    if (!(d > 0.0) && !isnan(d)) atomicOr(a.status, kErrDt);
    if (d > 0.0) dtc = d;  // std::min skips NaN (comparisons with NaN are false)
  }
  // warp then block minimum, one atomic per block
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, off));
  __shared__ double wmin[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wmin[warp] = dtc;
  __syncthreads();
  if (warp == 0) {
    dtc = (lane < (blockDim.x + 31) / 32) ? wmin[lane] : DBL_MAX;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dtc = fmin(dtc, __shfl_xor_sync(0xffffffffu, dtc, off));
    if (lane == 0) atomicMin(a.dt_min_bits, (unsigned long long)__double_as_longlong(dtc));
  }
}

}  // namespace nf
