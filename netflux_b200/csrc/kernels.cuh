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
//   face SoA    S, nhat : [3][F]; area : [F]
//   slot SoA    rs : [3][4][stride], the vector from the cell centroid to the
//               centroid of each of its faces (r_i or r_j of the face)
//   boundary    b_cell, b_slot, b_face, b_patch : [nb]; ghost states vg and
//               boundary fluxes fb : [5][bstride]
// Each face's flux is evaluated by both of its cells with the owner on the
// left, so both see bit-identical values; no atomics, deterministic results.
// The gradient kernel runs one thread per (cell, variable), the flux kernel
// four threads per cell (one per face slot).
#pragma once

#include <type_traits>

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
  const int* __restrict__ nbslot;  // [4][stride] neighbour << 2 | its slot, or -(1 + boundary face)
  const T* __restrict__ S;         // [3][F]
  const T* __restrict__ nhat;      // [3][F]
  const T* __restrict__ area;      // [F]
  const T* __restrict__ rs;        // [3][4][stride] centroid-to-face vector of each slot
  // node-based geometry of the fast forms (face m = the face opposite vertex m)
  const T* __restrict__ nodes;     // [n_nodes][4] x, y, z, 0
  const int* __restrict__ cnode;   // [4][stride] vertices of each cell, ascending node id
  const int* __restrict__ gcode;   // [stride] per face m, bits 3m..3m+2: present, outward flip, neighbour side
  const int* __restrict__ nbvf;    // [4][stride] neighbour cell of face m, -(1 + boundary face), or the cell itself
  const int* __restrict__ nbsf;    // [4][stride] neighbour << 2 | its face index, or -(1 + boundary face)
  const double* __restrict__ vol;
  const double* __restrict__ dS;
  const PatchBC* __restrict__ patches;
  // boundary faces, ordered by owner cell
  int nb;                          // number of boundary faces
  int bstride;                     // SoA stride of boundary arrays
  const int* __restrict__ b_cell;  // owner cell
  const int* __restrict__ b_slot;  // owner's slot of the face
  const int* __restrict__ b_face;  // face id (geometry)
  const int* __restrict__ b_patch; // patch
  const int* __restrict__ b_fs;    // face-state slot of the owner (slot order of the kernels in use)
  int n_nodes;                     // for the index checks of NF_DEBUG builds
  int n_patches;
};

// Index checks of NF_DEBUG builds (make debug): every index a kernel reads
// from the mesh arrays is checked before it is used; an index out of range
// sets kErrIndex in the status word and is replaced by a valid one (0, or the
// cell itself), so the access stays in bounds and the host reports the error.
// In the release build these are the identity.
__device__ __forceinline__ int checked(int idx, int limit, unsigned* status) {
#ifdef NF_DEBUG
  if (idx < 0 || idx >= limit) {
    atomicOr(status, kErrIndex);
    return 0;
  }
#endif
  return idx;
}
// a neighbour code: cell << shift (| slot) below n cells, or -(1 + boundary face) below nb
__device__ __forceinline__ int checked_nb(int code, int shift, int n, int nb, int self, unsigned* status) {
#ifdef NF_DEBUG
  const bool ok = code >= 0 ? (code >> shift) < n : (-code - 1) < nb;
  if (!ok) {
    atomicOr(status, kErrIndex);
    return self;
  }
#endif
  return code;
}

struct StageArgs {
  int second_order;      // SpatialOrder::Second
  int barth;             // Limiter::Barth
  int scheme;            // 0 explicit Euler, 1 TVD-RK3
  int stage;             // 0, 1, 2
  int local_dt;
  int freeze;            // a cell with dt == 0 keeps its state exactly (converged case)
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
  // mixed form: FP32 reconstruction increments and fields
  float* fs32;
  float* grad32;
  float* phi32;
  // boundary faces: cell-centre ghost states [5][bstride] and boundary fluxes
  // [5][bstride] (mixed form: FP32 differences to the owner's physical flux)
  double* vg;
  double* fb;
  float* fb32;
  // mixed form with FP32 copies (NF_PREC_MIXED32): the FP32 primitives of
  // the stage input and of its result, and FP32 ghost states [5][bstride];
  // the face states go to fs32 and the boundary fluxes to fb32. Vout (FP64)
  // is written only where a later time step reads it (null otherwise).
  const float* Vin32;
  float* Vout32;
  float* vg32;
  // mixed forms, TVD-RK3: the stage whose result is the last stage's input
  // (stage 2 of 3) also computes the next step's time step from the FP64
  // primitives of that result, the ones the reference's calc_timestep reads
  // (Solver.cpp:250): per cell into dt_next (local time stepping, else null)
  // and the minimum into *dt_next_min (null: not this stage)
  double* dt_next;
  unsigned long long* dt_next_min;
  const double* dS;  // [3][stride] projected areas (calc_Delta_S)
  double cfl;
  // converged cases of a steady solve (null: none); their cells are skipped
  // by the fast kernels (cases share no faces, and U is left untouched)
  const int* case_frozen;
  // limiter ratchet (extension): per-cell case, per-case switch (null: off)
  // and the kept limiter values [5][stride] (FP64 or FP32 with the state form)
  const int* cell_case;
  const int* lim_ratchet;
  double* phi_keep;
  float* phi_keep32;
};

// Programmatic dependent launch (the fast forms' stage kernels are launched
// with programmatic stream serialization, solver.cu): a kernel lets the next
// one in the stream launch once all of its blocks have started, and waits for
// the previous one to complete (its writes visible) before reading anything
// that kernel wrote. The next kernel's launch and block set-up then overlap
// this one's last wave. Launched without the attribute, both are no-ops.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;"); }
__device__ __forceinline__ void pdl_wait_previous() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Once a case's ratchet is on, a cell's limiter value is the minimum of the
// live value and the kept one, and is kept: it only tightens, so it settles
// and the steady residual can converge (the live Barth limiter makes it stall).
__device__ __forceinline__ bool frozen_cell(const StageArgs& a, int c) {
  return a.case_frozen != nullptr && a.case_frozen[a.cell_case[c]] != 0;
}
__device__ __forceinline__ bool ratchet_on(const StageArgs& a, int c) {
  return a.lim_ratchet != nullptr && a.lim_ratchet[a.cell_case[c]] != 0;
}
template <typename T>
__device__ __forceinline__ T ratchet(const StageArgs& a, size_t at, T phi) {
  T* keep;
  if constexpr (sizeof(T) == 8) keep = a.phi_keep;
  else keep = a.phi_keep32;
  const T v = (keep[at] < phi) ? keep[at] : phi;  // std::min(phi, kept)
  keep[at] = v;
  return v;
}

// The arrays the node kernels read and write, by arithmetic type: FP64 for
// the FP64 form, the FP32 copies for the mixed form with FP32 copies
// (primitives, ghosts, face states, boundary fluxes, optional dumps).
template <typename T>
struct StageIO;
template <>
struct StageIO<double> {
  static __device__ __forceinline__ const double* vin(const StageArgs& a) { return a.Vin; }
  static __device__ __forceinline__ const double* vg(const StageArgs& a) { return a.vg; }
  static __device__ __forceinline__ double* fs(const StageArgs& a) { return a.fs; }
  static __device__ __forceinline__ const double* fb(const StageArgs& a) { return a.fb; }
  static __device__ __forceinline__ double* grad(const StageArgs& a) { return a.grad; }
  static __device__ __forceinline__ double* phi(const StageArgs& a) { return a.phi; }
};
template <>
struct StageIO<float> {
  static __device__ __forceinline__ const float* vin(const StageArgs& a) { return a.Vin32; }
  static __device__ __forceinline__ const float* vg(const StageArgs& a) { return a.vg32; }
  static __device__ __forceinline__ float* fs(const StageArgs& a) { return a.fs32; }
  static __device__ __forceinline__ const float* fb(const StageArgs& a) { return a.fb32; }
  static __device__ __forceinline__ float* grad(const StageArgs& a) { return a.grad32; }
  static __device__ __forceinline__ float* phi(const StageArgs& a) { return a.phi32; }
};

// device scalars: the step's dt (minimum), the time, t_end, the dt last used,
// and the next step's dt while the last stage computes it
enum : int { kScalDtMin = 0, kScalTime = 1, kScalTEnd = 2, kScalDtUsed = 3, kScalDtNext = 4, kScalCount = 8 };

__device__ __forceinline__ double stage_dt(const double* scal) {
  double dt = scal[kScalDtMin];
  const double t_end = scal[kScalTEnd];
  if (t_end > 0.0) {
    const double left = t_end - scal[kScalTime];
    dt = (left < dt) ? left : dt;
  }
  return dt;
}

// The templated kernels below run in FP64 (T = double); the mixed form has
// its own kernels (kernels_mixed.cuh).
template <typename T>
__device__ __forceinline__ T ld_v(const StageArgs& a, int idx) {
  static_assert(sizeof(T) == 8, "FP64 kernels");
  return a.Vin[idx];
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
// Green-Gauss gradient + min/max + Barth limiter
// (calc_green_gauss_gradient, calc_max_and_min_values, calc_barth_limiter,
//  Numerics.hpp:86-292), then the limited reconstruction at each face
// (calc_limited_reconstruction, Numerics.hpp:135-145), which is what the flux
// kernel consumes. Ghost states at boundary faces are the cell-centre ghosts
// of set_constant_ghost_values (Solver.cpp:300-330).
//
// One thread per (cell, primitive variable k): every step of this kernel acts
// on one variable at a time, so the five threads of a cell share nothing but
// the cell's geometry (same addresses, served once per warp). Each thread
// folds its cell's faces in slot order, exactly as the reference's face loops
// reach that cell.
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) gradient_limiter_kernel(MeshView<T> m, StageArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = t / 5;
  const int k = t - 5 * c;
  if (c >= m.n) return;
  const int st = m.stride;
  const int F = m.n_faces;
  int sl[4], ns[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    sl[q] = m.slot[q * st + c];
    sl[q] = sl[q] < 0 ? -1 : (checked(sl[q] >> 1, F, a.status) << 1 | (sl[q] & 1));
    ns[q] = checked_nb(m.nbslot[q * st + c], 2, m.n, m.nb, c << 2, a.status);
  }
  const T vc = ld_v<T>(a, k * st + c);
  const T vol = T(m.vol[c]);
  T g[3] = {T(0), T(0), T(0)};
  T vmax = -std::numeric_limits<T>::max(), vmin = std::numeric_limits<T>::max();
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (sl[q] < 0) continue;
    const int f = sl[q] >> 1;
    const bool own = (sl[q] & 1) == 0;
    T vo;
    if (ns[q] >= 0) vo = ld_v<T>(a, k * st + (ns[q] >> 2));
    else vo = a.vg[k * m.bstride + (-ns[q] - 1)];
    // the neighbour side subtracts its term: (-x)/v == -(x/v) and
    // g + (-y) == g - y exactly, so a signed normal reproduces both branches
    const T s0 = m.S[f], s1 = m.S[F + f], s2 = m.S[2 * F + f];
    const T Sg[3] = {own ? s0 : -s0, own ? s1 : -s1, own ? s2 : -s2};
    const T uf = T(0.5) * (vc + vo);  // 0.5 (V_i + V_j); the sum commutes exactly
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if constexpr (kRef) g[d] = g[d] + uf * Sg[d] / vol;
      else g[d] = fma(uf, Sg[d], g[d]);
    }
    if constexpr (kRef) {
      const T vi = own ? vc : vo, vj = own ? vo : vc;  // max(V_i, V_j) in the face's operand order
      vmax = rmax(vmax, rmax(vi, vj));
      vmin = rmin(vmin, rmin(vi, vj));
    } else {
      vmax = fmax(vmax, vo);
      vmin = fmin(vmin, vo);
    }
  }
  if constexpr (!kRef) {
    const T iv = T(1) / vol;
    g[0] *= iv;
    g[1] *= iv;
    g[2] *= iv;
    vmax = fmax(vmax, vc);
    vmin = fmin(vmin, vc);
  }
  // grad V_k . r at each face: the limiter's Delta_2 before its sign/epsilon
  // adjustment, and the increment of the reconstruction
  T gr[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const T* r = m.rs + q * st + c;  // [d][q][cell]
    gr[q] = (g[0] * r[0] + g[1] * r[4 * st]) + g[2] * r[8 * st];
  }
  T phi = T(1);
  if (a.barth) {
    phi = std::numeric_limits<T>::max();
#pragma unroll
    for (int q = 0; q < 4; q++) {
      if (sl[q] < 0) continue;
      T d2 = gr[q];
      const T sg = (d2 > T(0)) ? T(1) : ((d2 < T(0)) ? T(-1) : T(0));
      d2 = sg * (fabs(d2) + Gas<T>::eps);
      T fc = T(1);
      if (d2 != T(0)) {
        const T num = (d2 > T(0)) ? vmax - vc : vmin - vc;
        fc = rmin(T(1), num / d2);
      }
      phi = rmin(phi, fc);
    }
    if (ratchet_on(a, c)) phi = ratchet(a, size_t(k) * st + c, phi);
  }
#pragma unroll
  for (int q = 0; q < 4; q++) {
    if (sl[q] < 0) continue;
    a.fs[(q * 5 + k) * st + c] = vc + phi * gr[q];
  }
  if (a.grad) {
#pragma unroll
    for (int d = 0; d < 3; d++) a.grad[(k * 3 + d) * st + c] = g[d];
    a.phi[k * st + c] = phi;
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
  int sl = m.slot[q * st + c];
  sl = sl < 0 ? -1 : (checked(sl >> 1, F, a.status) << 1 | (sl & 1));
  const int ns = checked_nb(m.nbslot[q * st + c], 2, m.n, m.nb, c << 2 | q, a.status);
  const bool has = sl >= 0;
  const bool own = (sl & 1) == 0;
  // this face's contribution to R: -F on the owner side, +F on the other
  double contrib[5] = {-0.0, -0.0, -0.0, -0.0, -0.0};
  if (has && ns < 0) {
    // boundary face (this cell is its owner): flux from boundary_flux_kernel
    const int b = -ns - 1;
#pragma unroll
    for (int k = 0; k < 5; k++) contrib[k] = -a.fb[k * m.bstride + b];
  } else if (has) {
    const int f = sl >> 1;
    const T nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
    const T area = m.area[f];
    T Vs[5], Vx[5];  // this cell's face state, the other side's
    const int o = ns >> 2, q2 = ns & 3;
#pragma unroll
    for (int k = 0; k < 5; k++) {
      if (second) {
        Vs[k] = a.fs[(q * 5 + k) * st + c];
        Vx[k] = a.fs[(q2 * 5 + k) * st + o];
      } else {
        Vs[k] = ld_v<T>(a, k * st + c);
        Vx[k] = ld_v<T>(a, k * st + o);
      }
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
  for (int k = 0; k < 5; k++) {
    if constexpr (kRef) R[k] = quad_sum_ordered(contrib[k]);
    else R[k] = quad_sum_tree(contrib[k]);
  }

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
  if (a.freeze && dt == 0.0) {
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = U[k];
  }
  double Vn[5];
  cons_to_prim<double, kRef>(Unew, Vn);
  if (!valid) return;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if (k == q || (k == 4 && q == 0)) {
      a.Uout[k * st + c] = Unew[k];
      a.Vout[k * st + c] = Vn[k];
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

// Per-cell CFL time step of EulerSolver::calc_timestep (Solver.cpp:232-274) on
// one cell's primitives, every operation rounded on its own (no contraction)
// in the reference's order, so the result is the reference's bit for bit in
// every translation unit.
__device__ __forceinline__ double dt_of_cell(const double V[5], double dS0, double dS1, double dS2, double vol,
                                             double cfl) {
  const double cs = __dsqrt_rn(__ddiv_rn(__dmul_rn(Gas<double>::gamma, V[4]), V[0]));
  const double sx = __dmul_rn(__dadd_rn(fabs(V[1]), cs), dS0);
  const double sy = __dmul_rn(__dadd_rn(fabs(V[2]), cs), dS1);
  const double sz = __dmul_rn(__dadd_rn(fabs(V[3]), cs), dS2);
  return __ddiv_rn(__dmul_rn(cfl, vol), __dadd_rn(__dadd_rn(sx, sy), sz));
}

// Minimum of v over the warp, then one atomicMin on the bit pattern (exact
// and order-free for positive doubles), skipped when the warp's minimum is not
// below the current one (the value only decreases, so the result is the same
// exact minimum); no block barrier. Every lane of the warp calls it.
__device__ __forceinline__ void warp_min_to(double v, unsigned long long* target) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, off));
  if ((threadIdx.x & 31) == 0 && v < DBL_MAX &&
      v < __longlong_as_double(static_cast<long long>(*reinterpret_cast<volatile unsigned long long*>(target))))
    atomicMin(target, (unsigned long long)__double_as_longlong(v));
}

// The next step's time step, computed by the FP64 form's last-stage gradient
// kernel from the primitives it reads: those of the last stage input, which
// the reference's calc_timestep reads (Solver.cpp:250).
struct DtFuse {
  double cfl;
  double* dt_next;                  // per-cell dt of the next step (local time stepping) or null
  unsigned long long* dt_min_bits;  // minimum over the cells (global time step)
};

// ---------------------------------------------------------------------------
// Fast forms (FP64 with contraction, and mixed FP32): one thread per cell, the
// cell's faces indexed by the vertex they face, geometry rebuilt from the
// vertices (the node array stays in L2):
//   * the vertices of a cell are stored sorted by node id, so face m's three
//     vertices, taken in that order, are the same ordered triple in both cells
//     of the face and give bit-identical normals S = 0.5 (B - A) x (C - A);
//     a per-face bit turns S outward;
//   * the vector from the centroid to the centroid of face m is
//     (centroid - P_m) / 3.
// gradient_node_kernel computes the same Green-Gauss gradient, min/max, Barth
// limiter and reconstruction as the reference form, rearranged for fewer
// instructions (agreement to round-off):
//   grad V = 0.5/vol (sum_m V_m S_m + V_c sum_m S_m);
//   phi = min(1, min_m A_m / D_m) with A_m = (V_max - V_c) or (V_c - V_min)
//   and D_m = |grad V . r_m| + eps, the minimising face found by
//   cross-multiplication, then one division per variable.
// A missing face (a boundary face no marker lists) has S = r = 0 and points
// at the cell itself, so it changes nothing.
// ---------------------------------------------------------------------------
// Ask the memory system to bring a line into L2 without holding a register;
// the later load of the same address then waits on an L2 hit, not on DRAM.
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// The own-cell rows the stage update reads (Uin, Un, the local dt).
__device__ __forceinline__ void prefetch_update_rows(const StageArgs& a, int c, int st) {
#pragma unroll
  for (int k = 0; k < 5; k++) prefetch_l2(a.Uin + size_t(k) * st + c);
  if (a.scheme != 0 && a.stage != 0) {
#pragma unroll
    for (int k = 0; k < 5; k++) prefetch_l2(a.Un + size_t(k) * st + c);
  }
  if (a.local_dt) prefetch_l2(a.dt_local + c);
}

// Node records are 4 values (x, y, z, pad) from a 256-byte aligned buffer, so
// a record starts on 32 bytes (FP64) or 16 bytes (FP32): x and y come in one
// 16-byte load (FP64), or the whole record in one (FP32).
template <typename T>
__device__ __forceinline__ void load_vertices(const MeshView<T>& m, int c, T P[4][3], unsigned* status) {
#pragma unroll
  for (int v = 0; v < 4; v++) {
    const int id = checked(m.cnode[v * m.stride + c], m.n_nodes, status);
    const T* p = m.nodes + 4 * size_t(id);
    if constexpr (sizeof(T) == 8) {
      const double2 xy = *reinterpret_cast<const double2*>(p);
      P[v][0] = xy.x;
      P[v][1] = xy.y;
      P[v][2] = p[2];
    } else {
      const float4 r = *reinterpret_cast<const float4*>(p);
      P[v][0] = r.x;
      P[v][1] = r.y;
      P[v][2] = r.z;
    }
  }
}

// normal of face fm (opposite vertex fm) from its vertices in ascending order
template <typename T, int fm>
__device__ __forceinline__ void face_normal(const T P[4][3], T S[3]) {
  constexpr int a = fm == 0 ? 1 : 0;
  constexpr int b = fm <= 1 ? 2 : 1;
  constexpr int cc = fm == 3 ? 2 : 3;
  const T e1[3] = {P[b][0] - P[a][0], P[b][1] - P[a][1], P[b][2] - P[a][2]};
  const T e2[3] = {P[cc][0] - P[a][0], P[cc][1] - P[a][1], P[cc][2] - P[a][2]};
  S[0] = T(0.5) * (e1[1] * e2[2] - e1[2] * e2[1]);
  S[1] = T(0.5) * (e1[2] * e2[0] - e1[0] * e2[2]);
  S[2] = T(0.5) * (e1[0] * e2[1] - e1[1] * e2[0]);
}

template <typename T>
__device__ __forceinline__ void face_normals(const T P[4][3], T S[4][3]) {
  face_normal<T, 0>(P, S[0]);
  face_normal<T, 1>(P, S[1]);
  face_normal<T, 2>(P, S[2]);
  face_normal<T, 3>(P, S[3]);
}

// kPipe: 0 one variable's loads at a time; 1 the next variable's loads in
// flight during this one's arithmetic; 2 all five variables' loads issued
// together before any arithmetic (one exposed memory latency instead of five,
// at the cost of registers); 3 as 0, with the cell's own rows prefetched
// into L2 first.
// The body for one cell; vown receives the cell's own primitives.
// CFL time step of one cell from its primitives with the fast forms'
// reciprocal and reciprocal square root (within 2 ulp of dt_of_cell).
__device__ __forceinline__ double dt_of_cell_fast(const double V[5], double dS0, double dS1, double dS2, double vol,
                                                  double cfl) {
  const double g = Gas<double>::gamma * V[4];
  const double cs = g * nr_rsqrt(g * V[0]);  // sqrt(gamma p / rho)
  const double sum = fma(fabs(V[3]) + cs, dS2, fma(fabs(V[2]) + cs, dS1, (fabs(V[1]) + cs) * dS0));
  return cfl * vol * nr_rcp(sum);
}

template <typename T, int kPipe, bool kDS = false>
__device__ __forceinline__ void gradient_node_cell(const MeshView<T>& m, const StageArgs& a, int c, T vown[5],
                                                   T* dS_out = nullptr) {
  const int st = m.stride;
  const T* __restrict__ Vin = StageIO<T>::vin(a);
  const T* __restrict__ Vg = StageIO<T>::vg(a);
  T* __restrict__ fsc = StageIO<T>::fs(a) + c;  // this cell's column of the face states
  int nb[4];
#pragma unroll
  for (int q = 0; q < 4; q++) nb[q] = checked_nb(m.nbvf[q * st + c], 0, m.n, m.nb, c, a.status);
  // each face's row base and row stride (a cell's or a ghost's) chosen once,
  // so a variable's neighbour load is one address computation
  const T* qb[4];
  int qs[4];
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const bool cell = nb[q] >= 0;
    qb[q] = cell ? Vin + nb[q] : Vg + (-nb[q] - 1);
    qs[q] = cell ? st : m.bstride;
  }
  auto fetch = [&](int k, T& vc, T vo[4]) {
    vc = Vin[size_t(k) * st + c];
#pragma unroll
    for (int q = 0; q < 4; q++) vo[q] = qb[q][k * qs[q]];
  };
  if constexpr (kPipe == 3) {
#pragma unroll
    for (int k = 0; k < 5; k++) prefetch_l2(Vin + size_t(k) * st + c);
  }
  [[maybe_unused]] T vcN, voN[4];
  [[maybe_unused]] T vcA[5], voA[5][4];
  if constexpr (kPipe == 2) {
    // the same loads as fetch(), all five variables' at once
#pragma unroll
    for (int k = 0; k < 5; k++) vcA[k] = Vin[size_t(k) * st + c];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const bool cell = nb[q] >= 0;
      const auto* p = cell ? Vin + nb[q] : Vg + (-nb[q] - 1);
      const size_t rs = cell ? size_t(st) : size_t(m.bstride);
#pragma unroll
      for (int k = 0; k < 5; k++) voA[k][q] = p[k * rs];
    }
  } else if (kPipe == 1) {
    fetch(0, vcN, voN);
  }
  const int code = m.gcode[c];
  T S[4][3], d[4][3];  // outward normals; (centroid - P_m) / 3
  {
    T P[4][3];
    load_vertices(m, c, P, a.status);
    face_normals(P, S);
    const T cen[3] = {T(0.25) * ((P[0][0] + P[1][0]) + (P[2][0] + P[3][0])),
                      T(0.25) * ((P[0][1] + P[1][1]) + (P[2][1] + P[3][1])),
                      T(0.25) * ((P[0][2] + P[1][2]) + (P[2][2] + P[3][2]))};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int bits = code >> (3 * q);
      const T sgn = (bits & 1) == 0 ? T(0) : ((bits & 2) ? T(-1) : T(1));  // 0: no face
#pragma unroll
      for (int e = 0; e < 3; e++) {
        S[q][e] *= sgn;
        d[q][e] = (bits & 1) ? (cen[e] - P[q][e]) * T(1.0 / 3.0) : T(0);
      }
    }
  }
  const T ssum[3] = {(S[0][0] + S[1][0]) + (S[2][0] + S[3][0]), (S[0][1] + S[1][1]) + (S[2][1] + S[3][1]),
                     (S[0][2] + S[1][2]) + (S[2][2] + S[3][2])};
  if constexpr (kDS) {
    // projected areas of calc_Delta_S (Solver.cpp:276-298): half the sum of
    // |S_d| over the cell's interior faces, from the normals in registers
#pragma unroll
    for (int e = 0; e < 3; e++) {
      T acc = T(0);
#pragma unroll
      for (int q = 0; q < 4; q++) acc += nb[q] >= 0 ? fabs(S[q][e]) : T(0);
      dS_out[e] = T(0.5) * acc;
    }
  }
  const T hv = T(0.5) * nr_rcp(T(m.vol[c]));
  const bool rat = a.barth && ratchet_on(a, c);
  auto variable = [&](int k, T vc, const T vo[4]) {
    vown[k] = vc;
    T acc[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      acc[e] = vc * ssum[e];
#pragma unroll
      for (int q = 0; q < 4; q++) acc[e] = fma(vo[q], S[q][e], acc[e]);
    }
    const T g[3] = {hv * acc[0], hv * acc[1], hv * acc[2]};
    const T vmax = fmax(fmax(fmax(vc, vo[0]), fmax(vo[1], vo[2])), vo[3]);
    const T vmin = fmin(fmin(fmin(vc, vo[0]), fmin(vo[1], vo[2])), vo[3]);
    T gr[4];
#pragma unroll
    for (int q = 0; q < 4; q++) gr[q] = fma(g[2], d[q][2], fma(g[1], d[q][1], g[0] * d[q][0]));
    T phi = T(1);
    if (a.barth) {
      T An = T(1), Dn = T(1);  // best ratio so far, starting at 1
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const T d2 = gr[q];
        const T A = d2 > T(0) ? vmax - vc : vc - vmin;
        const T D = fabs(d2) + Gas<T>::eps;
        const bool better = (d2 != T(0)) && (A * Dn < An * D);
        An = better ? A : An;
        Dn = better ? D : Dn;
      }
      phi = An * nr_rcp(Dn);
      if (rat) phi = ratchet(a, size_t(k) * st + c, phi);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) fsc[size_t(q * 5 + k) * st] = fma(phi, gr[q], vc);
    if (T* gdump = StageIO<T>::grad(a)) {
#pragma unroll
      for (int e = 0; e < 3; e++) gdump[(k * 3 + e) * st + c] = g[e];
      StageIO<T>::phi(a)[k * st + c] = phi;
    }
  };
  if constexpr (kPipe == 2) {
#pragma unroll
    for (int k = 0; k < 5; k++) variable(k, vcA[k], voA[k]);
  } else {
#pragma unroll 1
    for (int k = 0; k < 5; k++) {
      T vc, vo[4];
      if (kPipe == 1) {
        vc = vcN;
#pragma unroll
        for (int q = 0; q < 4; q++) vo[q] = voN[q];
        if (k < 4) fetch(k + 1, vcN, voN);  // next variable's loads overlap this one's arithmetic
      } else {
        fetch(k, vc, vo);
      }
      variable(k, vc, vo);
    }
  }
}


// kDt: also the next step's time step from the cell's own primitives, after
// the gradient work (the FP64 form's last stage; the primitives are those of
// the last stage input, which the reference's calc_timestep reads,
// Solver.cpp:250; every thread reaches the block minimum).
template <typename T, int kPipe, int kMinBlocks, bool kDt = false>
__global__ void __launch_bounds__(128, kMinBlocks) gradient_node_kernel(MeshView<T> m, StageArgs a, DtFuse dtf) {
  static_assert(!kDt || sizeof(T) == 8, "the fused time step is the FP64 form's");
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  const bool in = c < m.n;
  const bool active = in && !frozen_cell(a, c);
  T vown[5], dS[3];
  if (active) gradient_node_cell<T, kPipe, kDt>(m, a, c, vown, dS);
  if constexpr (kDt) {
    double dtc = DBL_MAX;
    if (in) {
      if (!active) {
        if (dtf.dt_next) dtf.dt_next[c] = 0.0;  // a converged case keeps its state
      } else {
        const double d = dt_of_cell_fast(vown, dS[0], dS[1], dS[2], m.vol[c], dtf.cfl);
        if (dtf.dt_next) dtf.dt_next[c] = d;
        if (!(d > 0.0) && !isnan(d)) atomicOr(a.status, kErrDt);
        if (d > 0.0) dtc = d;  // std::min skips NaN (comparisons with NaN are false)
      }
    }
    warp_min_to(dtc, dtf.dt_min_bits);
  }
}

// flux_node_kernel: flux balance and stage update of one cell per thread.
// Each interior face's flux is evaluated with the reference's owner on the
// left and the owner-to-neighbour unit normal, which both cells rebuild to the
// same bits, so both add exactly opposite contributions; boundary faces add
// the flux boundary_flux_kernel computed.
template <typename T>
struct FaceIn {
  T s[5];      // this cell's face state, or the boundary flux
  T x[5];      // the other side's face state
  int kind;    // 0 no face, 1 interior (owner), 2 interior (neighbour side), 3 boundary
};

// Stage update of one cell from its flux balance R (TVD_RK3 Solver.cpp:103-133,
// explicit_euler 83-101) in FP64, then the primitives of the new state
// (set_primvars, SolverData.cpp:37-48), the optional dumps and the status.
__device__ __forceinline__ void stage_update(const StageArgs& a, int c, int st, const double R[5], double vol) {
  const double dt = a.local_dt ? a.dt_local[c] : stage_dt(a.scal);
  double Unew[5];
  const double ivol = nr_rcp(vol);
  if (a.scheme == 0 || a.stage == 0) {
    const double qf = dt * ivol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = fma(qf, R[k], a.Uin[k * st + c]);
  } else if (a.stage == 1) {
    const double qf = 0.25 * dt * ivol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 0.75 * a.Un[k * st + c] + 0.25 * a.Uin[k * st + c] + qf * R[k];
  } else {
    const double qf = 2.0 / 3.0 * dt * ivol;
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = 1.0 / 3.0 * a.Un[k * st + c] + 2.0 / 3.0 * a.Uin[k * st + c] + qf * R[k];
  }
  if (a.freeze && dt == 0.0) {
#pragma unroll
    for (int k = 0; k < 5; k++) Unew[k] = a.Uin[k * st + c];
  }
  double Vn[5];
  cons_to_prim<double, false>(Unew, Vn);
  bool finite = true;
#pragma unroll
  for (int k = 0; k < 5; k++) {
    a.Uout[k * st + c] = Unew[k];
    if (a.Vout) a.Vout[k * st + c] = Vn[k];
    if (a.Vout32) a.Vout32[k * st + c] = float(Vn[k]);
    if (a.R) a.R[k * st + c] = R[k];
    finite = finite && isfinite(R[k]) && isfinite(Unew[k]);
  }
  if (a.res_cell) a.res_cell[c] = R[0] * ivol;
  if (!finite) atomicOr(a.status, kErrNonFinite);
  else if (!(Vn[0] > 0.0) || !(Vn[4] > 0.0)) atomicOr(a.status, kErrNonPhysical);
  if (a.dt_next_min) {
    // the next step's time step from this result's primitives; the minimum
    // by one atomicMin on the bit pattern (exact for positive doubles),
    // skipped when the value is not below the current minimum
    const double d = (a.freeze && dt == 0.0) ? 0.0 : dt_of_cell_fast(Vn, a.dS[c], a.dS[st + c], a.dS[2 * st + c], vol, a.cfl);
    if (a.dt_next) a.dt_next[c] = d;
    if (!(a.freeze && dt == 0.0)) {
      if (!(d > 0.0) && !isnan(d)) atomicOr(a.status, kErrDt);
      if (d > 0.0 &&
          d < __longlong_as_double(static_cast<long long>(*reinterpret_cast<volatile unsigned long long*>(a.dt_next_min))))
        atomicMin(a.dt_next_min, (unsigned long long)__double_as_longlong(d));
    }
  }
}

// kPipe: 0 one face's loads at a time, 1 the next face's loads in flight
// during this face's flux, 2 all four faces' loads issued together, 3 as 0
// with the cell's own face states and update rows prefetched into L2 first.
template <typename T, int kPipe, int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) flux_node_kernel(MeshView<T> m, StageArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (c >= m.n) return;
  if (frozen_cell(a, c)) {
    if (a.dt_next_min && a.dt_next) a.dt_next[c] = 0.0;  // a converged case keeps its state
    return;
  }
  const int st = m.stride;
  const bool second = a.second_order != 0;
  const T* __restrict__ fsb = StageIO<T>::fs(a);
  const T* __restrict__ Vin = StageIO<T>::vin(a);
  const T* __restrict__ fb = StageIO<T>::fb(a);
  const int code = m.gcode[c];
  int ns[4];
#pragma unroll
  for (int q = 0; q < 4; q++) ns[q] = checked_nb(m.nbsf[q * st + c], 2, m.n, m.nb, c << 2 | q, a.status);
  auto fetch = [&](int q, FaceIn<T>& in) {
    const int bits = code >> (3 * q);
    if ((bits & 1) == 0) {
      in.kind = 0;
    } else if (ns[q] < 0) {
      in.kind = 3;
      const int b = -ns[q] - 1;
#pragma unroll
      for (int k = 0; k < 5; k++) in.s[k] = fb[k * m.bstride + b];
    } else {
      const int o = ns[q] >> 2, q2 = ns[q] & 3;
      in.kind = (bits & 4) ? 2 : 1;
#pragma unroll
      for (int k = 0; k < 5; k++) {
        in.s[k] = second ? fsb[(q * 5 + k) * st + c] : Vin[k * st + c];
        in.x[k] = second ? fsb[(q2 * 5 + k) * st + o] : Vin[k * st + o];
      }
    }
  };
  if constexpr (kPipe == 3) {
    if (second) {
#pragma unroll
      for (int r = 0; r < 20; r++) prefetch_l2(fsb + size_t(r) * st + c);
    }
    prefetch_update_rows(a, c, st);
  }
  [[maybe_unused]] FaceIn<T> nxt;
  [[maybe_unused]] FaceIn<T> all[4];
  if constexpr (kPipe == 2) {
#pragma unroll
    for (int q = 0; q < 4; q++) fetch(q, all[q]);
  } else if (kPipe == 1) {
    fetch(0, nxt);
  }
  T S[4][3];
  {
    T P[4][3];
    load_vertices(m, c, P, a.status);
    face_normals(P, S);
  }
  // the flux balance in FP64 (FP64 form); the FP32 form sums its FP32 fluxes
  // in FP32 and hands the sum to the FP64 update
  using Acc = typename std::conditional<sizeof(T) == 8, double, float>::type;
  Acc R[5] = {Acc(0), Acc(0), Acc(0), Acc(0), Acc(0)};
#pragma unroll
  for (int q = 0; q < 4; q++) {
    FaceIn<T> cur;
    if constexpr (kPipe == 2) {
      cur = all[q];
    } else if (kPipe == 1) {
      cur = nxt;
      if (q < 3) fetch(q + 1, nxt);  // next face's loads overlap this face's flux
    } else {
      fetch(q, cur);
    }
    if (cur.kind == 3) {
#pragma unroll
      for (int k = 0; k < 5; k++) R[k] -= Acc(cur.s[k]);
    } else if (cur.kind != 0) {
      const int bits = code >> (3 * q);
      const bool own = cur.kind == 1;
      // owner-to-neighbour normal: this cell's outward normal on the owner side
      const bool flip = own ? (bits & 2) != 0 : (bits & 2) == 0;
      const T a2 = (S[q][0] * S[q][0] + S[q][1] * S[q][1]) + S[q][2] * S[q][2];
      const T inv = nr_rsqrt(a2);  // 1 / |S|
      const T area = a2 * inv;
      const T sg = flip ? -inv : inv;
      const T nh[3] = {S[q][0] * sg, S[q][1] * sg, S[q][2] * sg};
      T Fl[5];
      if (own) rusanov_fast<T>(cur.s, cur.x, nh, area, Fl);
      else rusanov_fast<T>(cur.x, cur.s, nh, area, Fl);
#pragma unroll
      for (int k = 0; k < 5; k++) R[k] = own ? R[k] - Acc(Fl[k]) : R[k] + Acc(Fl[k]);
    }
  }
  const double Rd[5] = {double(R[0]), double(R[1]), double(R[2]), double(R[3]), double(R[4])};
  stage_update(a, c, st, Rd, m.vol[c]);
}

// ---------------------------------------------------------------------------
// Boundary faces. ghost_kernel: the cell-centre ghost state of every boundary
// face (set_constant_ghost_values, Solver.cpp:300-330), read by the gradient
// kernel like a neighbour's primitives. boundary_flux_kernel: the flux through
// every boundary face, from the owner's reconstructed face state and the ghost
// built from that state (Solver.cpp:197-229), read by the flux kernel at the
// face's slot. One thread per boundary face; the hot kernels carry no
// boundary-condition code.
// ---------------------------------------------------------------------------
template <typename T, bool kRef>
__global__ void __launch_bounds__(256) ghost_kernel(MeshView<T> m, StageArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (b >= m.nb) return;
  const int c = checked(m.b_cell[b], m.n, a.status), f = checked(m.b_face[b], m.n_faces, a.status);
  const int F = m.n_faces, st = m.stride;
  T V[5], G[5];
#pragma unroll
  for (int k = 0; k < 5; k++) V[k] = ld_v<T>(a, k * st + c);
  const T nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
  ghost_state<T>(m.patches[checked(m.b_patch[b], m.n_patches, a.status)], V, nh, G);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    a.vg[k * m.bstride + b] = G[k];
  }
}

template <typename T, bool kRef>
__global__ void __launch_bounds__(256) boundary_flux_kernel(MeshView<T> m, StageArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (b >= m.nb) return;
  const int c = checked(m.b_cell[b], m.n, a.status), q = checked(m.b_fs[b], 4, a.status),
            f = checked(m.b_face[b], m.n_faces, a.status);
  const int F = m.n_faces, st = m.stride;
  T VL[5], VR[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    if (a.second_order) {
      VL[k] = a.fs[(q * 5 + k) * st + c];
    } else {
      VL[k] = ld_v<T>(a, k * st + c);
    }
  }
  const T nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
  ghost_state<T>(m.patches[checked(m.b_patch[b], m.n_patches, a.status)], VL, nh, VR);
  T Fl[5];
  if constexpr (kRef) {
    T UL[5], UR[5];
    prim_to_cons<T, kRef>(VL, UL);
    prim_to_cons<T, kRef>(VR, UR);
    rusanov_ref<T>(UL, UR, nh, m.area[f], Fl);
  } else {
    rusanov_fast<T>(VL, VR, nh, m.area[f], Fl);
  }
#pragma unroll
  for (int k = 0; k < 5; k++) a.fb[k * m.bstride + b] = Fl[k];
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
  const int* cell_case;    // case of each cell (batched meshes)
  const int* case_frozen;  // nonzero: the case has converged; its cells get dt = 0
};

template <bool kRef>
__global__ void __launch_bounds__(256) timestep_kernel(MeshView<double> m, DtArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = DBL_MAX;
  if (c < m.n) {
    const int st = m.stride;
    double V[5];
#pragma unroll
    for (int k = 0; k < 5; k++) V[k] = a.V[k * st + c];
    const double d = dt_of_cell(V, m.dS[c], m.dS[st + c], m.dS[2 * st + c], m.vol[c], a.cfl);
    const bool frozen = a.case_frozen && a.case_frozen[a.cell_case[c]];
    if (a.dt_local) a.dt_local[c] = frozen ? 0.0 : d;
    if (!frozen) {
      if (!(d > 0.0) && !isnan(d)) atomicOr(a.status, kErrDt);
      if (d > 0.0) dtc = d;  // std::min skips NaN (comparisons with NaN are false)
    }
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
