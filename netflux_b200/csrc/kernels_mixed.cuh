// Mixed-precision form in difference variables: FP64 state, primitives,
// ghosts, boundary fluxes and update; FP32 gradient, limiter, reconstruction
// and interior Rusanov fluxes, computed from differences to the cell's own
// FP64 primitives so that FP32 rounding is relative to those differences.
//
// With the face normals of a closed cell summing to zero,
//   grad V_c = 1/vol sum_f 0.5 (V_c + V_f) S_f = 0.5/vol sum_f (V_f - V_c) S_f
//   R_c = -sum_f F(V_L, V_R; S_f) = -sum_f [F(V_L, V_R; S_f) - F(V_c) . S_f]
// (calc_green_gauss_gradient Numerics.hpp:86-128, evaluate_inviscid_fluxes
// Solver.cpp:144-230): the same operator as the FP64 forms in exact
// arithmetic. Storing FP32 copies of V and of the face states instead rounds
// at |V| * 2^-24, which puts a floor under the steady residual (near a 1e-5
// drop); here everything FP32 carries is small near a steady state: V_f - V_c,
// the reconstruction increments phi grad V . r and the flux differences
// F - F(V_c), so the residual keeps converging.
#pragma once

#include "kernels.cuh"

namespace nf {

// F(V_c + dL, V_c + dR; n, area) - area F(V_c) . n for the Rusanov flux
// (rusanov Numerics.cpp:10-18, inviscid_flux SolverData.hpp:239-255), expanded
// so every term is a difference times an O(1) factor:
//   rho_X q_X - rho_c q_c            = d_rho q_c + rho_X dq
//   rho_X u_X q_X - rho_c u_c q_c    = (d_rho u_c + rho_X du) q_c + rho_X u_X dq
//   H_X q_X - H_c q_c                = (dE + dp) q_c + H_X dq
//   E_X - E_c = dp/(g-1) + 0.5 (d_rho |u_c|^2 + rho_X (2 u_c . du + |du|^2))
struct DeltaSide {
  float dU[5];  // U(V_c + d) - U(V_c)
  float dF[5];  // (F(V_c + d) - F(V_c)) . n
  float s;      // |q| + c of the state
};

__device__ __forceinline__ DeltaSide delta_side(const float vc[5], float q_c, float uu_c, const float d[5],
                                                const float n[3]) {
  constexpr float g1i = Gas<float>::g1_inv;
  DeltaSide o;
  const float rho = vc[0] + d[0], p = vc[4] + d[4];
  const float u[3] = {vc[1] + d[1], vc[2] + d[2], vc[3] + d[3]};
  const float dq = fmaf(d[3], n[2], fmaf(d[2], n[1], d[1] * n[0]));
  const float udu = fmaf(vc[3], d[3], fmaf(vc[2], d[2], vc[1] * d[1]));
  const float dudu = fmaf(d[3], d[3], fmaf(d[2], d[2], d[1] * d[1]));
  const float dE = fmaf(d[4], g1i, 0.5f * fmaf(d[0], uu_c, rho * fmaf(2.0f, udu, dudu)));
  o.dU[0] = d[0];
  o.dF[0] = fmaf(d[0], q_c, rho * dq);
#pragma unroll
  for (int e = 0; e < 3; e++) {
    o.dU[e + 1] = fmaf(d[0], vc[e + 1], rho * d[e + 1]);
    o.dF[e + 1] = fmaf(o.dU[e + 1], q_c, fmaf(rho * u[e], dq, d[4] * n[e]));
  }
  const float uu = fmaf(u[2], u[2], fmaf(u[1], u[1], u[0] * u[0]));
  const float H = fmaf(p, g1i, fmaf(0.5f * rho, uu, p));  // E + p
  o.dU[4] = dE;
  o.dF[4] = fmaf(dE + d[4], q_c, H * dq);
  o.s = fabsf(q_c + dq) + sound_speed_fast(rho, p);
  return o;
}

__device__ __forceinline__ void rusanov_delta(const float vc[5], const float dL[5], const float dR[5],
                                              const float n[3], float area, float F[5]) {
  const float q_c = fmaf(vc[3], n[2], fmaf(vc[2], n[1], vc[1] * n[0]));
  const float uu_c = fmaf(vc[3], vc[3], fmaf(vc[2], vc[2], vc[1] * vc[1]));
  const DeltaSide L = delta_side(vc, q_c, uu_c, dL, n);
  const DeltaSide R = delta_side(vc, q_c, uu_c, dR, n);
  const float smax = fmaxf(R.s, L.s);
  const float h = 0.5f * area;
#pragma unroll
  for (int k = 0; k < 5; k++) F[k] = h * fmaf(-smax, R.dU[k] - L.dU[k], L.dF[k] + R.dF[k]);
}

// Gradient, min/max, Barth limiter (FLT_EPSILON, as the reference's
// single-precision build, Numerics.hpp:171) and the reconstruction increments
// phi grad V . r_m, one thread per cell, from FP64 primitives and ghosts.
template <int kPipe, int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) gradient_delta_kernel(MeshView<float> m, StageArgs a) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (c >= m.n || frozen_cell(a, c)) return;
  const int st = m.stride;
  const double* __restrict__ V = a.Vin;
  const double* __restrict__ Vg = a.vg;
  float* __restrict__ inc_c = a.fs32 + c;  // this cell's column of the increments
  int nb[4];
#pragma unroll
  for (int q = 0; q < 4; q++) nb[q] = checked_nb(m.nbvf[q * st + c], 0, m.n, m.nb, c, a.status);
  auto fetch = [&](int k, double& vc, double vo[4]) {
    const double* Vk = V + size_t(k) * st;
    vc = Vk[c];
#pragma unroll
    for (int q = 0; q < 4; q++) vo[q] = nb[q] >= 0 ? Vk[nb[q]] : Vg[k * m.bstride + (-nb[q] - 1)];
  };
  if constexpr (kPipe == 3) {
#pragma unroll
    for (int k = 0; k < 5; k++) prefetch_l2(V + size_t(k) * st + c);
  }
  [[maybe_unused]] double vcN, voN[4];
  [[maybe_unused]] double vcA[5], voA[5][4];
  if constexpr (kPipe == 2) {
    // the same loads as fetch(), with each face's row base and row stride
    // chosen once (cell row or ghost row) instead of per variable
#pragma unroll
    for (int k = 0; k < 5; k++) vcA[k] = V[size_t(k) * st + c];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const bool cell = nb[q] >= 0;
      const auto* p = cell ? V + nb[q] : Vg + (-nb[q] - 1);
      const size_t rs = cell ? size_t(st) : size_t(m.bstride);
#pragma unroll
      for (int k = 0; k < 5; k++) voA[k][q] = p[k * rs];
    }
  } else if (kPipe == 1) {
    fetch(0, vcN, voN);
  }
  const int code = m.gcode[c];
  float S[4][3], d[4][3];  // outward normals; (centroid - P_m) / 3
  {
    float P[4][3];
    load_vertices(m, c, P, a.status);
    face_normals(P, S);
    const float cen[3] = {0.25f * ((P[0][0] + P[1][0]) + (P[2][0] + P[3][0])),
                          0.25f * ((P[0][1] + P[1][1]) + (P[2][1] + P[3][1])),
                          0.25f * ((P[0][2] + P[1][2]) + (P[2][2] + P[3][2]))};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int bits = code >> (3 * q);
      const float sgn = (bits & 1) == 0 ? 0.f : ((bits & 2) ? -1.f : 1.f);  // 0: no face
#pragma unroll
      for (int e = 0; e < 3; e++) {
        S[q][e] *= sgn;
        d[q][e] = (bits & 1) ? (cen[e] - P[q][e]) * (1.0f / 3.0f) : 0.f;
      }
    }
  }
  const float hv = float(0.5 / m.vol[c]);
  const bool rat = a.barth && ratchet_on(a, c);
  auto variable = [&](int k, double vc, const double vo[4]) {
    float dv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) dv[q] = float(vo[q] - vc);
    float acc[3];
#pragma unroll
    for (int e = 0; e < 3; e++) {
      acc[e] = dv[0] * S[0][e];
#pragma unroll
      for (int q = 1; q < 4; q++) acc[e] = fmaf(dv[q], S[q][e], acc[e]);
    }
    float g[3] = {hv * acc[0], hv * acc[1], hv * acc[2]};
    if ((code & 0x249) != 0x249) {
      // a dropped boundary face (FV_Grid.cpp:79-85): the listed normals do not
      // sum to zero, grad = grad_diff + V_c sum_listed S / vol
#pragma unroll
      for (int e = 0; e < 3; e++)
        g[e] += float(vc * double((S[0][e] + S[1][e]) + (S[2][e] + S[3][e])) / m.vol[c]);
    }
    const float up = fmaxf(fmaxf(fmaxf(0.f, dv[0]), fmaxf(dv[1], dv[2])), dv[3]);   // V_max - V_c
    const float dn = fminf(fminf(fminf(0.f, dv[0]), fminf(dv[1], dv[2])), dv[3]);   // V_min - V_c
    float gr[4];
#pragma unroll
    for (int q = 0; q < 4; q++) gr[q] = fmaf(g[2], d[q][2], fmaf(g[1], d[q][1], g[0] * d[q][0]));
    float phi = 1.f;
    if (a.barth) {
      float An = 1.f, Dn = 1.f;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const float d2 = gr[q];
        const float A = d2 > 0.f ? up : -dn;
        const float D = fabsf(d2) + Gas<float>::eps;
        const bool better = (d2 != 0.f) && (A * Dn < An * D);
        An = better ? A : An;
        Dn = better ? D : Dn;
      }
      phi = An * nr_rcp(Dn);
      if (rat) phi = ratchet(a, size_t(k) * st + c, phi);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) inc_c[size_t(q * 5 + k) * st] = phi * gr[q];
    if (a.grad32) {
#pragma unroll
      for (int e = 0; e < 3; e++) a.grad32[(k * 3 + e) * st + c] = g[e];
      a.phi32[k * st + c] = phi;
    }
  };
  if constexpr (kPipe == 2) {
#pragma unroll
    for (int k = 0; k < 5; k++) variable(k, vcA[k], voA[k]);
  } else {
#pragma unroll 1
    for (int k = 0; k < 5; k++) {
      double vc, vo[4];
      if (kPipe == 1) {
        vc = vcN;
#pragma unroll
        for (int q = 0; q < 4; q++) vo[q] = voN[q];
        if (k < 4) fetch(k + 1, vcN, voN);
      } else {
        fetch(k, vc, vo);
      }
      variable(k, vc, vo);
    }
  }
}

// Flux balance from the difference form and the FP64 stage update, one
// thread per cell; boundary faces add boundary_flux_delta_kernel's values.
template <int kPipe, int kMinBlocks>
__global__ void __launch_bounds__(128, kMinBlocks) flux_delta_kernel(MeshView<float> m, StageArgs a) {
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
  const double* __restrict__ V = a.Vin;
  const float* __restrict__ inc = a.fs32;
  const float* __restrict__ fbd = a.fb32;
  const int code = m.gcode[c];
  double vcd[5];
  float vc[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    vcd[k] = V[k * st + c];
    vc[k] = float(vcd[k]);
  }
  int ns[4];
#pragma unroll
  for (int q = 0; q < 4; q++) ns[q] = checked_nb(m.nbsf[q * st + c], 2, m.n, m.nb, c << 2 | q, a.status);
  // kind 0 no face, 1 interior, 3 boundary; s: own increments or the
  // boundary flux difference; x: the other side's state minus V_c
  auto fetch = [&](int q, FaceIn<float>& in) {
    const int bits = code >> (3 * q);
    if ((bits & 1) == 0) {
      in.kind = 0;
    } else if (ns[q] < 0) {
      in.kind = 3;
      const int b = -ns[q] - 1;
#pragma unroll
      for (int k = 0; k < 5; k++) in.s[k] = fbd[k * m.bstride + b];
    } else {
      const int o = ns[q] >> 2, q2 = ns[q] & 3;
      in.kind = 1;
      // row bases chosen once per face
      const double* pv = V + o;
      const float* ps = inc + size_t(q * 5) * st + c;
      const float* px = inc + size_t(q2 * 5) * st + o;
#pragma unroll
      for (int k = 0; k < 5; k++) {
        const float dvo = float(pv[size_t(k) * st] - vcd[k]);
        in.s[k] = second ? ps[size_t(k) * st] : 0.f;
        in.x[k] = second ? dvo + px[size_t(k) * st] : dvo;
      }
    }
  };
  if constexpr (kPipe == 3) {
    if (second) {
#pragma unroll
      for (int r = 0; r < 20; r++) prefetch_l2(inc + size_t(r) * st + c);
    }
    prefetch_update_rows(a, c, st);
  }
  [[maybe_unused]] FaceIn<float> nxt;
  [[maybe_unused]] FaceIn<float> all[4];
  if constexpr (kPipe == 2) {
#pragma unroll
    for (int q = 0; q < 4; q++) fetch(q, all[q]);
  } else if (kPipe == 1) {
    fetch(0, nxt);
  }
  float S[4][3];
  {
    float P[4][3];
    load_vertices(m, c, P, a.status);
    face_normals(P, S);
  }
  double R[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  float slist[3] = {0.f, 0.f, 0.f};  // sum of the listed faces' outward normals
#pragma unroll
  for (int q = 0; q < 4; q++) {
    FaceIn<float> cur;
    if constexpr (kPipe == 2) {
      cur = all[q];
    } else if (kPipe == 1) {
      cur = nxt;
      if (q < 3) fetch(q + 1, nxt);
    } else {
      fetch(q, cur);
    }
    if (cur.kind != 0) {
      const float sgn = ((code >> (3 * q)) & 2) ? -1.f : 1.f;
#pragma unroll
      for (int e = 0; e < 3; e++) slist[e] = fmaf(sgn, S[q][e], slist[e]);
    }
    if (cur.kind == 3) {
#pragma unroll
      for (int k = 0; k < 5; k++) R[k] -= double(cur.s[k]);
    } else if (cur.kind == 1) {
      const int bits = code >> (3 * q);
      const float a2 = fmaf(S[q][2], S[q][2], fmaf(S[q][1], S[q][1], S[q][0] * S[q][0]));
      const float inv = nr_rsqrt(a2);  // 1 / |S|
      const float area = a2 * inv;
      const float sg = (bits & 2) ? -inv : inv;  // outward unit normal
      const float nh[3] = {S[q][0] * sg, S[q][1] * sg, S[q][2] * sg};
      float Fl[5];
      rusanov_delta(vc, cur.s, cur.x, nh, area, Fl);
#pragma unroll
      for (int k = 0; k < 5; k++) R[k] -= double(Fl[k]);
    }
  }
  if ((code & 0x249) != 0x249) {
    // A boundary face that no marker lists is dropped (FV_Grid.cpp:79-85), so
    // the listed normals do not sum to zero: R = R_diff - F(V_c) . sum_listed S.
    const double sx = slist[0], sy = slist[1], sz = slist[2];
    const double qs = (vcd[1] * sx + vcd[2] * sy) + vcd[3] * sz;
    const double m0 = vcd[0] * qs;
    const double E = Gas<double>::g1_inv * vcd[4] + 0.5 * vcd[0] * ((vcd[1] * vcd[1] + vcd[2] * vcd[2]) + vcd[3] * vcd[3]);
    R[0] -= m0;
    R[1] -= m0 * vcd[1] + vcd[4] * sx;
    R[2] -= m0 * vcd[2] + vcd[4] * sy;
    R[3] -= m0 * vcd[3] + vcd[4] * sz;
    R[4] -= qs * (E + vcd[4]);
  }
  stage_update(a, c, st, R, m.vol[c]);
}

// Boundary faces in FP64: the owner's reconstructed state V_c + increment, its
// ghost (Solver.cpp:212), the Rusanov flux, minus the owner's physical flux
// through the face; stored as FP32 difference.
__global__ void __launch_bounds__(256) boundary_flux_delta_kernel(MeshView<double> m, StageArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (b >= m.nb) return;
  const int c = checked(m.b_cell[b], m.n, a.status), q = checked(m.b_fs[b], 4, a.status),
            f = checked(m.b_face[b], m.n_faces, a.status);
  const int F = m.n_faces, st = m.stride;
  double Vc[5], VL[5], VR[5];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    Vc[k] = a.Vin[k * st + c];
    VL[k] = a.second_order ? Vc[k] + double(a.fs32[(q * 5 + k) * st + c]) : Vc[k];
  }
  const double nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
  const double area = m.area[f];
  ghost_state<double>(m.patches[checked(m.b_patch[b], m.n_patches, a.status)], VL, nh, VR);
  double Fl[5];
  rusanov_fast<double>(VL, VR, nh, area, Fl);
  // area F(V_c) . n
  const double qn = (Vc[1] * nh[0] + Vc[2] * nh[1]) + Vc[3] * nh[2];
  const double m0 = Vc[0] * qn;
  const double E = Gas<double>::g1_inv * Vc[4] + 0.5 * Vc[0] * ((Vc[1] * Vc[1] + Vc[2] * Vc[2]) + Vc[3] * Vc[3]);
  const double Fc[5] = {m0, m0 * Vc[1] + Vc[4] * nh[0], m0 * Vc[2] + Vc[4] * nh[1], m0 * Vc[3] + Vc[4] * nh[2],
                        qn * (E + Vc[4])};
#pragma unroll
  for (int k = 0; k < 5; k++) a.fb32[k * m.bstride + b] = float(Fl[k] - area * Fc[k]);
}

}  // namespace nf
