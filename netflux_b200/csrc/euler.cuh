// Compressible Euler physics for one cell-centred finite-volume face, as
// device functions. Two arithmetic forms share this file:
//
//  * Ref (kRef = true): every expression in the reference's operand order
//    (SolverData.hpp:165-262, Numerics.cpp:10-171, Numerics.hpp:135-250) with
//    true divisions. The translation unit that instantiates it is compiled
//    with -fmad=false, so results round exactly as the reference's x86-64
//    build (which has no FMA), pow() excepted.
//  * Fast (kRef = false): the same mathematics with reciprocals, fused
//    multiply-adds and the primitive face state used directly in the flux
//    (no primitive -> conservative -> primitive round trip).
//
// Real is the arithmetic type of the face work: double, or float in the
// mixed-precision form.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

namespace nf {

// Error bits of the device status word.
enum : unsigned {
  kErrNonFinite = 1u,     // a non-finite residual or state
  kErrNonPhysical = 2u,   // rho <= 0 or p <= 0 after an update
  kErrDt = 4u,            // a cell produced dt <= 0
  kErrIndex = 8u,         // NF_DEBUG builds: a mesh index out of range (the access was redirected)
};

template <typename T>
struct Gas {
  // EulerEqs::GAMMA etc. (SolverData.hpp:129-131), evaluated in T.
  static constexpr T gamma = T(1.4);
  static constexpr T g1 = gamma - T(1);
  static constexpr T g1_inv = T(1) / g1;
  static constexpr T eps = std::numeric_limits<T>::epsilon();
};

enum : int { kBcNoSlip = 0, kBcSlip = 1, kBcFarField = 2 };

// Boundary condition of one patch. The far-field constants are computed on
// the host with the reference's expressions (BC_FarField ctor,
// Numerics.cpp:76-84).
struct PatchBC {
  int type;
  int case_index;
  double fs[5];     // rho, u, v, w, p of the free stream
  double c_fs;      // sqrt(gamma * p / rho)
  double s_fs;      // p * rho^-gamma
  int density_fix;  // extension: 1 = physical far-field density (the reference inverts it)
  int pad;
};

// Reciprocal and reciprocal square root for the fast forms, by the
// Newton-Raphson method from a single-precision hardware estimate: each
// iteration roughly doubles the number of correct bits (about 2^-22 after the
// estimate, 2^-44 after one step, beyond double precision after two), so the
// FP64 results are within about 1 ulp; FP32 uses the hardware estimate
// directly (within about 1 ulp of the correctly rounded value). The FP64
// forms start from the correctly rounded FP32 reciprocal: with the bare
// estimate there the FP64 gradient kernel measured 17 % slower at 3.1M tets.
// Operands are positive, normal and within single-precision range (densities,
// pressures, |S|^2, volumes).
// the hardware's single-precision reciprocal estimate (PTX rcp.approx.ftz.f32,
// relative error below 2^-23 for the normal operands used here)
__device__ __forceinline__ float rcp_estimate(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ double nr_rcp(double b) {
  double r = double(__frcp_rn(float(b)));
  double e = fma(-b, r, 1.0);
  r = fma(r, e, r);
  e = fma(-b, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ double nr_rsqrt(double x) {
  double r = double(rsqrtf(float(x)));
  const double h = 0.5 * x;
  double e = fma(-h * r, r, 0.5);  // r <- r (3/2 - x r^2 / 2)
  r = fma(r, e, r);
  e = fma(-h * r, r, 0.5);
  return fma(r, e, r);
}
__device__ __forceinline__ float nr_rcp(float b) { return rcp_estimate(b); }
__device__ __forceinline__ float nr_rsqrt(float x) { return rsqrtf(x); }

// speed of sound sqrt(gamma p / rho) = gamma p / sqrt(gamma p rho): no division
template <typename T>
__device__ __forceinline__ T sound_speed_fast(T rho, T p) {
  const T g = Gas<T>::gamma * p;
  return g * nr_rsqrt(g * rho);
}

template <typename T>
__device__ __forceinline__ T rmax(T a, T b) { return (a < b) ? b : a; }  // std::max
template <typename T>
__device__ __forceinline__ T rmin(T a, T b) { return (b < a) ? b : a; }  // std::min

// ---- EulerEqs (SolverData.hpp:165-262) ----
template <typename T, bool kRef>
__device__ __forceinline__ void prim_to_cons(const T V[5], T U[5]) {
  U[0] = V[0];
  U[1] = V[0] * V[1];
  U[2] = V[0] * V[2];
  U[3] = V[0] * V[3];
  U[4] = Gas<T>::g1_inv * V[4] + T(0.5) * V[0] * ((V[1] * V[1] + V[2] * V[2]) + V[3] * V[3]);
}

template <typename T, bool kRef>
__device__ __forceinline__ T pressure(const T U[5]) {
  return Gas<T>::g1 * (U[4] - T(0.5) / U[0] * ((U[1] * U[1] + U[2] * U[2]) + U[3] * U[3]));
}

template <typename T, bool kRef>
__device__ __forceinline__ void cons_to_prim(const T U[5], T V[5]) {
  if constexpr (kRef) {
    V[0] = U[0];
    V[1] = U[1] / U[0];
    V[2] = U[2] / U[0];
    V[3] = U[3] / U[0];
    V[4] = pressure<T, kRef>(U);
  } else {
    const T ir = nr_rcp(U[0]);
    V[0] = U[0];
    V[1] = U[1] * ir;
    V[2] = U[2] * ir;
    V[3] = U[3] * ir;
    V[4] = Gas<T>::g1 * (U[4] - T(0.5) * ir * ((U[1] * U[1] + U[2] * U[2]) + U[3] * U[3]));
  }
}

// NumericalFlux::rusanov (Numerics.cpp:10-18) on conservative states, with the
// unit normal and area precomputed per face (same IEEE operations as
// S.normalized() / S.norm()).
template <typename T>
__device__ __forceinline__ void rusanov_ref(const T UL[5], const T UR[5], const T n[3], T area, T F[5]) {
  // conv_spectral_radii = |projected_velocity| + sound_speed_conservative
  const T pL = pressure<T, true>(UL), pR = pressure<T, true>(UR);
  const T vnL = ((UL[1] * n[0] + UL[2] * n[1]) + UL[3] * n[2]) / UL[0];
  const T vnR = ((UR[1] * n[0] + UR[2] * n[1]) + UR[3] * n[2]) / UR[0];
  const T sL = fabs(vnL) + sqrt(Gas<T>::gamma * pL / UL[0]);
  const T sR = fabs(vnR) + sqrt(Gas<T>::gamma * pR / UR[0]);
  const T smax = rmax(sR, sL);
  // inviscid_flux (SolverData.hpp:239-255)
  T FL[5], FR[5];
  FL[0] = vnL * UL[0];
  FL[1] = vnL * UL[1] + pL * n[0];
  FL[2] = vnL * UL[2] + pL * n[1];
  FL[3] = vnL * UL[3] + pL * n[2];
  FL[4] = vnL * (UL[4] + pL);
  FR[0] = vnR * UR[0];
  FR[1] = vnR * UR[1] + pR * n[0];
  FR[2] = vnR * UR[2] + pR * n[1];
  FR[3] = vnR * UR[3] + pR * n[2];
  FR[4] = vnR * (UR[4] + pR);
  const T a = area * T(0.5);
#pragma unroll
  for (int k = 0; k < 5; k++) F[k] = a * ((FR[k] + FL[k]) - smax * (UR[k] - UL[k]));
}

// The same flux evaluated from the primitive face states: pressure and
// velocity come straight from V, one reciprocal per side.
template <typename T>
__device__ __forceinline__ void rusanov_fast(const T VL[5], const T VR[5], const T n[3], T area, T F[5]) {
  const T vnL = (VL[1] * n[0] + VL[2] * n[1]) + VL[3] * n[2];
  const T vnR = (VR[1] * n[0] + VR[2] * n[1]) + VR[3] * n[2];
  const T sL = fabs(vnL) + sound_speed_fast(VL[0], VL[4]);
  const T sR = fabs(vnR) + sound_speed_fast(VR[0], VR[4]);
  const T smax = rmax(sR, sL);
  const T keL = T(0.5) * VL[0] * ((VL[1] * VL[1] + VL[2] * VL[2]) + VL[3] * VL[3]);
  const T keR = T(0.5) * VR[0] * ((VR[1] * VR[1] + VR[2] * VR[2]) + VR[3] * VR[3]);
  const T EL = Gas<T>::g1_inv * VL[4] + keL, ER = Gas<T>::g1_inv * VR[4] + keR;
  const T mL = VL[0] * vnL, mR = VR[0] * vnR;
  const T a = area * T(0.5);
  F[0] = a * ((mR + mL) - smax * (VR[0] - VL[0]));
  F[1] = a * ((mR * VR[1] + VR[4] * n[0] + mL * VL[1] + VL[4] * n[0]) - smax * (VR[0] * VR[1] - VL[0] * VL[1]));
  F[2] = a * ((mR * VR[2] + VR[4] * n[1] + mL * VL[2] + VL[4] * n[1]) - smax * (VR[0] * VR[2] - VL[0] * VL[2]));
  F[3] = a * ((mR * VR[3] + VR[4] * n[2] + mL * VL[3] + VL[4] * n[2]) - smax * (VR[0] * VR[3] - VL[0] * VL[3]));
  F[4] = a * ((vnR * (ER + VR[4]) + vnL * (EL + VL[4])) - smax * (ER - EL));
}

// ---- boundary conditions (Numerics.cpp:59-171) on primitive states ----
// n is S.normalized() of the face (S points out of the domain).
template <typename T>
__device__ __forceinline__ void ghost_state(const PatchBC& bc, const T V[5], const T n[3], T G[5]) {
  if (bc.type == kBcSlip) {  // BC_SlipWall
    const T vn = (V[1] * n[0] + V[2] * n[1]) + V[3] * n[2];
    G[0] = V[0];
    G[1] = V[1] - T(2) * vn * n[0];
    G[2] = V[2] - T(2) * vn * n[1];
    G[3] = V[3] - T(2) * vn * n[2];
    G[4] = V[4];
  } else if (bc.type == kBcFarField) {  // BC_FarField, incl. its quirks
    const T gam = Gas<T>::gamma, g1 = Gas<T>::g1;
    const T vfs[3] = {T(bc.fs[1]), T(bc.fs[2]), T(bc.fs[3])};
    const T c_fs = T(bc.c_fs);
    const T vn_fs = (n[0] * vfs[0] + n[1] * vfs[1]) + n[2] * vfs[2];
    const T vn_d = (n[0] * V[1] + n[1] * V[2]) + n[2] * V[3];
    const T c_d = sqrt(gam * V[4] / V[0]);
    const T Rp = (vn_fs + c_fs > T(0)) ? vn_d + T(2) * c_d / g1 : vn_fs + T(2) * c_fs / g1;
    const T Rm = (vn_fs - c_fs > T(0)) ? vn_d - T(2) * c_d / g1 : vn_fs - T(2) * c_fs / g1;
    const T vn_b = T(0.5) * (Rp + Rm);
    const T c_b = g1 / T(4) * (Rp - Rm);
    T s_b;
    if (vn_fs > T(0)) {
      G[1] = V[1] + (vn_b - vn_d) * n[0];
      G[2] = V[2] + (vn_b - vn_d) * n[1];
      G[3] = V[3] + (vn_b - vn_d) * n[2];
      s_b = V[4] * pow(V[0], -gam);
    } else {
      G[1] = vfs[0] + (vn_fs - vn_b) * n[0];
      G[2] = vfs[1] + (vn_fs - vn_b) * n[1];
      G[3] = vfs[2] + (vn_fs - vn_b) * n[2];
      s_b = T(bc.s_fs);
    }
    // Numerics.cpp:149 computes (gamma s / c^2)^(1/(gamma-1)), the inverse of
    // the isentropic density; it is exact only for rho = 1 (kept by default)
    const T rho_b = bc.density_fix ? pow(c_b * c_b / (gam * s_b), Gas<T>::g1_inv)
                                   : pow(gam * s_b / (c_b * c_b), Gas<T>::g1_inv);
    G[0] = rho_b;
    G[4] = c_b * c_b * rho_b / gam;
  } else {  // BC_NoSlipWall
    G[0] = V[0];
    G[1] = -V[1];
    G[2] = -V[2];
    G[3] = -V[3];
    G[4] = V[4];
  }
}

}  // namespace nf
