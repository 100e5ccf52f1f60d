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
//               nbslot : [4][stride] = neighbour << 2 | the neighbour's slot
//               of the same face, or -(1 + patch) at a boundary face
//   face states fs : [4][5][stride], the limited reconstruction of the cell's
//               primitives at each of its faces (written by the gradient
//               kernel, read by the flux kernel of both adjacent cells)
//   face SoA    S, nhat, ri, rj : [3][F]; area : [F]
// Each face's flux is evaluated by both of its cells with the owner on the
// left, so both see bit-identical values; no atomics, deterministic results.
// The gradient and flux kernels run four threads per cell (one per face slot).
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
  const int* __restrict__ slot;    // [4][stride] face << 1 | side
  const int* __restrict__ nbslot;  // [4][stride] neighbour << 2 | its slot, or -(1 + patch)
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
  double* fs;            // reconstructed face states [4 slots][5][stride]
  double* grad;          // optional copy of the gradient [15][stride] (k*3+d)
  double* phi;           // optional copy of the limiter [5][stride]
  const double* Uin;     // stage input state (own cell)
  const double* Un;      // U^n (stages 1, 2)
  double* Uout;          // may alias Uin
  double* Vout;          // primitives of Uout
  double* R;             // optional flux-balance dump [5][stride]
  double* res_cell;      // optional R_rho / vol per cell (first stage)
  const double* dt_local;
  const double* scal;    // device scalars: [0] dt (min target), [1] time, [2] t_end
  unsigned* status;
  // mixed precision: FP32 copies of the primitives, face states and fields
  const float* Vin32;
  float* Vout32;
  float* fs32;
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

template <typename T>
__device__ __forceinline__ T ld_v(const StageArgs& a, int idx) {
  if constexpr (sizeof(T) == 8) return a.Vin[idx];
  else return a.Vin32[idx];
}

// Four threads per cell: lane q of a quad owns the cell's face slot q. A
// cell's per-face terms are combined across its quad with shuffles, folded in
// slot order q = 0, 1, 2, 3, so sums keep the reference's order. A missing
// slot contributes -0.0, which leaves any IEEE sum unchanged.
constexpr unsigned kFull = 0xffffffffu;

template <typename T>
__device__ __forceinline__ T quad_sum_ordered(T v) {
  T s = T(0);
#pragma unroll
  for (int p = 0; p < 4; p++) s = s + __shfl_sync(kFull, v, p, 4);
  return s;
}
template <typename T>
__device__ __forceinline__ T quad_max_ordered(T init, T v) {
#pragma unroll
  for (int p = 0; p < 4; p++) init = rmax(init, __shfl_sync(kFull, v, p, 4));
  return init;
}
template <typename T>
__device__ __forceinline__ T quad_min_ordered(T init, T v) {
#pragma unroll
  for (int p = 0; p < 4; p++) init = rmin(init, __shfl_sync(kFull, v, p, 4));
  return init;
}
template <typename T>
__device__ __forceinline__ T quad_sum_tree(T v) {
  v = v + __shfl_xor_sync(kFull, v, 1, 4);
  return v + __shfl_xor_sync(kFull, v, 2, 4);
}
template <typename T>
__device__ __forceinline__ T quad_min_tree(T v) {
  v = fmin(v, __shfl_xor_sync(kFull, v, 1, 4));
  return fmin(v, __shfl_xor_sync(kFull, v, 2, 4));
}
template <typename T>
__device__ __forceinline__ T quad_max_tree(T v) {
  v = fmax(v, __shfl_xor_sync(kFull, v, 1, 4));
  return fmax(v, __shfl_xor_sync(kFull, v, 2, 4));
}

// ---------------------------------------------------------------------------
// Green-Gauss gradient + min/max + Barth limiter of one cell
// (calc_green_gauss_gradient, calc_max_and_min_values, calc_barth_limiter,
//  Numerics.hpp:86-292), then the limited reconstruction at each of its faces
// (calc_limited_reconstruction, Numerics.hpp:135-145), which is what the flux
// kernel consumes. Ghost states at boundary faces are the cell-centre ghosts
// of set_constant_ghost_values (Solver.cpp:300-330).
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) gradient_limiter_kernel(MeshView<T> m, StageArgs a) {
  const int q = threadIdx.x & 3;
  int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 2;
  const bool valid = c < m.n;
  if (!valid) c = m.n - 1;  // every lane takes part in the quad shuffles
  const int st = m.stride;
  const int F = m.n_faces;
  T Vc[5];
#pragma unroll
  for (int k = 0; k < 5; k++) Vc[k] = ld_v<T>(a, k * st + c);
  const T vol = T(m.vol[c]);
  const int sl = m.slot[q * st + c];
  const int ns = m.nbslot[q * st + c];
  const bool has = sl >= 0;
  const int f = has ? (sl >> 1) : 0;
  const bool own = (sl & 1) == 0;

  // this face's Green-Gauss term (reference: already divided by the volume)
  // and its max/min candidates
  T t[5][3], mx[5], mn[5];
  if (has) {
    const T S[3] = {m.S[f], m.S[F + f], m.S[2 * F + f]};
    // the neighbour side of a face subtracts its term: (-x)/v == -(x/v) and
    // g + (-y) == g - y exactly, so a signed normal reproduces both branches
    const T Sg[3] = {own ? S[0] : -S[0], own ? S[1] : -S[1], own ? S[2] : -S[2]};
    T Vo[5];
    if (ns >= 0) {
      const int o = ns >> 2;
#pragma unroll
      for (int k = 0; k < 5; k++) Vo[k] = ld_v<T>(a, k * st + o);
    } else {
      const T nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
      ghost_state<T>(m.patches[-ns - 1], Vc, nh, Vo);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const T uf = T(0.5) * (Vc[k] + Vo[k]);  // 0.5 (V_i + V_j); the sum commutes
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if constexpr (kRef) t[k][d] = uf * Sg[d] / vol;
        else t[k][d] = uf * Sg[d];
      }
      if constexpr (kRef) {
        const T vi = own ? Vc[k] : Vo[k], vj = own ? Vo[k] : Vc[k];
        mx[k] = rmax(vi, vj);
        mn[k] = rmin(vi, vj);
      } else {
        mx[k] = Vo[k];
        mn[k] = Vo[k];
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      t[k][0] = t[k][1] = t[k][2] = T(-0.0);
      mx[k] = -std::numeric_limits<T>::max();
      mn[k] = std::numeric_limits<T>::max();
    }
  }
  // gradient of the cell: sum of the quad's terms
  T g[5][3];
  T vmax[5], vmin[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if constexpr (kRef) g[k][d] = quad_sum_ordered(t[k][d]);
      else g[k][d] = quad_sum_tree(t[k][d]);
    }
    if constexpr (kRef) {
      vmax[k] = quad_max_ordered(-std::numeric_limits<T>::max(), mx[k]);
      vmin[k] = quad_min_ordered(std::numeric_limits<T>::max(), mn[k]);
    } else {
      vmax[k] = fmax(Vc[k], quad_max_tree(mx[k]));
      vmin[k] = fmin(Vc[k], quad_min_tree(mn[k]));
    }
  }
  if constexpr (!kRef) {
    const T iv = T(1) / vol;
#pragma unroll
    for (int k = 0; k < 5; k++)
#pragma unroll
      for (int d = 0; d < 3; d++) g[k][d] *= iv;
  }
  // grad V . r at this lane's face: the limiter's Delta_2 before its
  // sign/epsilon adjustment, and the increment of the reconstruction
  T gr[5];
  {
    const T* rr = own ? m.ri : m.rj;
    const T r[3] = {rr[f], rr[F + f], rr[2 * F + f]};
#pragma unroll
    for (int k = 0; k < 5; k++) gr[k] = (g[k][0] * r[0] + g[k][1] * r[1]) + g[k][2] * r[2];
  }
  T phi[5];
  if (a.barth) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      T fc = std::numeric_limits<T>::max();  // identity of the min for an empty slot
      if (has) {
        T d2 = gr[k];
        const T sg = (d2 > T(0)) ? T(1) : ((d2 < T(0)) ? T(-1) : T(0));
        d2 = sg * (fabs(d2) + Gas<T>::eps);
        if (d2 != T(0)) {
          const T num = (d2 > T(0)) ? vmax[k] - Vc[k] : vmin[k] - Vc[k];
          fc = rmin(T(1), num / d2);
        } else {
          fc = T(1);
        }
      }
      if constexpr (kRef) phi[k] = quad_min_ordered(std::numeric_limits<T>::max(), fc);
      else phi[k] = quad_min_tree(fc);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 5; k++) phi[k] = T(1);
  }
  if (valid && has) {
#pragma unroll
    for (int k = 0; k < 5; k++) {
      const T v = Vc[k] + phi[k] * gr[k];
      if constexpr (sizeof(T) == 8) a.fs[(q * 5 + k) * st + c] = v;
      else a.fs32[(q * 5 + k) * st + c] = v;
    }
  }
  if (valid && q == 0) {
    if constexpr (sizeof(T) == 8) {
      if (a.grad) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
#pragma unroll
          for (int d = 0; d < 3; d++) a.grad[(k * 3 + d) * st + c] = g[k][d];
          a.phi[k * st + c] = phi[k];
        }
      }
    } else {
      if (a.grad32) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
#pragma unroll
          for (int d = 0; d < 3; d++) a.grad32[(k * 3 + d) * st + c] = g[k][d];
          a.phi32[k * st + c] = phi[k];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Face fluxes, flux balance R and the stage update of one cell
// (evaluate_inviscid_fluxes Solver.cpp:144-230, rusanov Numerics.cpp:10-18,
//  TVD_RK3 Solver.cpp:103-133, explicit_euler 83-101), then the primitives of
// the new state for the next stage (set_primvars, SolverData.cpp:37-48).
// The face states come from gradient_limiter_kernel (second order) or are the
// cell primitives (first order). Lane q evaluates the flux of face slot q.
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) flux_update_kernel(MeshView<T> m, StageArgs a) {
  const int q = threadIdx.x & 3;
  int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 2;
  const bool valid = c < m.n;
  if (!valid) c = m.n - 1;
  const int st = m.stride;
  const int F = m.n_faces;
  const bool second = a.second_order != 0;
  const int sl = m.slot[q * st + c];
  const int ns = m.nbslot[q * st + c];
  const bool has = sl >= 0;
  const bool own = (sl & 1) == 0;
  // this face's contribution to R: -F on the owner side, +F on the other
  double contrib[5] = {-0.0, -0.0, -0.0, -0.0, -0.0};
  if (has) {
    const int f = sl >> 1;
    const T nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
    const T area = m.area[f];
    T Vs[5], Vx[5];  // this cell's face state, the other side's
#pragma unroll
    for (int k = 0; k < 5; k++) {
      if (second) {
        if constexpr (sizeof(T) == 8) Vs[k] = a.fs[(q * 5 + k) * st + c];
        else Vs[k] = a.fs32[(q * 5 + k) * st + c];
      } else {
        Vs[k] = ld_v<T>(a, k * st + c);
      }
    }
    if (ns >= 0) {
      const int o = ns >> 2, q2 = ns & 3;
#pragma unroll
      for (int k = 0; k < 5; k++) {
        if (second) {
          if constexpr (sizeof(T) == 8) Vx[k] = a.fs[(q2 * 5 + k) * st + o];
          else Vx[k] = a.fs32[(q2 * 5 + k) * st + o];
        } else {
          Vx[k] = ld_v<T>(a, k * st + o);
        }
      }
    } else {
      // boundary face (this cell is its owner): ghost from the reconstructed
      // face value (Solver.cpp:212)
      ghost_state<T>(m.patches[-ns - 1], Vs, nh, Vx);
    }
    const T* VL = own ? Vs : Vx;
    const T* VR = own ? Vx : Vs;
    T Fl[5];
    if constexpr (kRef) {
      T UL[5], UR[5];
      prim_to_cons<T, kRef>(VL, UL);
      prim_to_cons<T, kRef>(VR, UR);
      rusanov_ref<T>(UL, UR, nh, area, Fl);
    } else {
      rusanov_fast<T>(VL, VR, nh, area, Fl);
    }
#pragma unroll
    for (int k = 0; k < 5; k++) contrib[k] = own ? -double(Fl[k]) : double(Fl[k]);
  }
  // flux balance, accumulated in face-slot order: ((0 + c0) + c1) + ...
  double R[5];
#pragma unroll
  for (int k = 0; k < 5; k++) R[k] = quad_sum_ordered(contrib[k]);

  // ---- stage update (FP64); every lane computes it, lanes store by component ----
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
    const double qf = dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = U[k] + qf * R[k];
  } else if (a.stage == 1) {
    const double qf = 1.0 / 4.0 * dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 3.0 / 4.0 * Uo[k] + 1.0 / 4.0 * U[k] + qf * R[k];
  } else {
    const double qf = 2.0 / 3.0 * dt / vol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 1.0 / 3.0 * Uo[k] + 2.0 / 3.0 * U[k] + qf * R[k];
  }
  double Vn[5];
  cons_to_prim<double, kRef>(Unew, Vn);
  if (!valid) return;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if (k == q || (k == 4 && q == 0)) {
      a.Uout[k * st + c] = Unew[k];
      a.Vout[k * st + c] = Vn[k];
      if (a.Vout32) a.Vout32[k * st + c] = float(Vn[k]);
      if (a.R) a.R[k * st + c] = R[k];
    }
  }
  if (q == 0) {
    if (a.res_cell) a.res_cell[c] = R[0] / vol;
    bool finite = true;
#pragma unroll
    for (int k = 0; k < 5; k++) finite = finite && isfinite(R[k]) && isfinite(Unew[k]);
    if (!finite) atomicOr(a.status, kErrNonFinite);
    else if (!(Vn[0] > 0.0) || !(Vn[4] > 0.0)) atomicOr(a.status, kErrNonPhysical);
  }
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
