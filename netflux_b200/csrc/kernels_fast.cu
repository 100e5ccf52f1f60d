// Kernels with reciprocals and fused multiply-adds (FP64), and the
// mixed-precision form (FP32 face work in difference variables, FP64 state,
// primitives, ghosts, boundary fluxes and update).
#include <utility>

#include "kernels_mixed.cuh"
#include "launch.hpp"

namespace nf {

template <bool kRef>
__global__ void __launch_bounds__(256) prim_kernel_fast(int n, int st, const double* __restrict__ U,
                                                       double* __restrict__ V, float* __restrict__ V32) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  double u[5], v[5];
#pragma unroll
  for (int k = 0; k < 5; k++) u[k] = U[k * st + c];
  cons_to_prim<double, kRef>(u, v);
#pragma unroll
  for (int k = 0; k < 5; k++) {
    V[k * st + c] = v[k];
    if (V32) V32[k * st + c] = float(v[k]);
  }
}

static inline int grid_for(int n, int block) { return (n + block - 1) / block; }

// Launch with programmatic stream serialization: the kernel may start while
// the previous kernel in the stream finishes (it waits for it on the device
// before reading its results, pdl_wait_previous). Captured into the step's
// CUDA graph as a programmatic dependency.
template <typename... P, typename... A>
static void launch_pdl(void (*kernel)(P...), int grid, int block, cudaStream_t stream, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(unsigned(grid));
  cfg.blockDim = dim3(unsigned(block));
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// one thread per cell, at most 128 threads per block (the kernels' launch bounds)
static inline int fast_block(int b) { return b > 128 ? 128 : b; }

// Variants (the tuner times them): 0 plain, 1 software-pipelined, 2 plain
// with registers capped for at least kCap resident 128-thread blocks per SM
// (6 for FP64, 8 for FP32), 3 pipelined with the same cap, 4 and 5 the same
// with a tighter cap (7 / 9 blocks), 6 and 7 with every load issued before the
// arithmetic (kPipe 2), uncapped and capped for kCap3 blocks (4 / 5), 8 and 9
// plain with the cell's own rows prefetched into L2 (kPipe 3), capped as 2
// and 4. (Prefetching the neighbours' rows as well measured slower.)
template <typename T>
constexpr int kCap = sizeof(T) == 8 ? 6 : 8;
template <typename T>
constexpr int kCap2 = sizeof(T) == 8 ? 7 : 9;
template <typename T>
constexpr int kCap3 = sizeof(T) == 8 ? 4 : 5;
#define NF_NODE_DISPATCH(KERNEL, T, m, a, l)                                                       \
  do {                                                                                              \
    const int b = fast_block(l.block);                                                             \
    const int g = grid_for(m.n, b);                                                                \
    switch (l.variant) {                                                                            \
      case 1: launch_pdl(KERNEL<T, 1, 1>, g, b, l.stream, m, a); break;                                 \
      case 2: launch_pdl(KERNEL<T, 0, kCap<T>>, g, b, l.stream, m, a); break;                           \
      case 3: launch_pdl(KERNEL<T, 1, kCap<T>>, g, b, l.stream, m, a); break;                           \
      case 4: launch_pdl(KERNEL<T, 0, kCap2<T>>, g, b, l.stream, m, a); break;                          \
      case 5: launch_pdl(KERNEL<T, 1, kCap2<T>>, g, b, l.stream, m, a); break;                          \
      case 6: launch_pdl(KERNEL<T, 2, 1>, g, b, l.stream, m, a); break;                                 \
      case 7: launch_pdl(KERNEL<T, 2, kCap3<T>>, g, b, l.stream, m, a); break;                          \
      case 8: launch_pdl(KERNEL<T, 3, kCap<T>>, g, b, l.stream, m, a); break;                           \
      case 9: launch_pdl(KERNEL<T, 3, kCap2<T>>, g, b, l.stream, m, a); break;                          \
      default: launch_pdl(KERNEL<T, 0, 1>, g, b, l.stream, m, a); break;                                \
    }                                                                                               \
  } while (0)

// the gradient kernel's variants, with and without the next step's time step
#define NF_GRAD_DISPATCH(KDT)                                                                       \
  do {                                                                                              \
    const int b = fast_block(l.block);                                                             \
    const int g = grid_for(m.n, b);                                                                \
    switch (l.variant) {                                                                            \
      case 1: launch_pdl(gradient_node_kernel<double, 1, 1, KDT>, g, b, l.stream, m, a, d); break;       \
      case 2: launch_pdl(gradient_node_kernel<double, 0, kCap<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 3: launch_pdl(gradient_node_kernel<double, 1, kCap<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 4: launch_pdl(gradient_node_kernel<double, 0, kCap2<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 5: launch_pdl(gradient_node_kernel<double, 1, kCap2<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 6: launch_pdl(gradient_node_kernel<double, 2, 1, KDT>, g, b, l.stream, m, a, d); break;       \
      case 7: launch_pdl(gradient_node_kernel<double, 2, kCap3<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 8: launch_pdl(gradient_node_kernel<double, 3, kCap<double>, KDT>, g, b, l.stream, m, a, d); break; \
      case 9: launch_pdl(gradient_node_kernel<double, 3, kCap2<double>, KDT>, g, b, l.stream, m, a, d); break; \
      default: launch_pdl(gradient_node_kernel<double, 0, 1, KDT>, g, b, l.stream, m, a, d); break;      \
    }                                                                                               \
  } while (0)

void launch_gradient_fast(const MeshView<double>& m, const StageArgs& a, const DtFuse* dt, Launch l) {
  const DtFuse d = dt ? *dt : DtFuse{0.0, nullptr, nullptr};
  if (dt) NF_GRAD_DISPATCH(true);
  else NF_GRAD_DISPATCH(false);
}
#undef NF_GRAD_DISPATCH
void launch_flux_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  NF_NODE_DISPATCH(flux_node_kernel, double, m, a, l);
}
// mixed form (difference variables, kernels_mixed.cuh)
#define NF_DELTA_DISPATCH(KERNEL, m, a, l)                                                         \
  do {                                                                                              \
    const int b = fast_block(l.block);                                                             \
    const int g = grid_for(m.n, b);                                                                \
    switch (l.variant) {                                                                            \
      case 1: launch_pdl(KERNEL<1, 1>, g, b, l.stream, m, a); break;                                    \
      case 2: launch_pdl(KERNEL<0, kCap<float>>, g, b, l.stream, m, a); break;                          \
      case 3: launch_pdl(KERNEL<1, kCap<float>>, g, b, l.stream, m, a); break;                          \
      case 4: launch_pdl(KERNEL<0, kCap2<float>>, g, b, l.stream, m, a); break;                         \
      case 5: launch_pdl(KERNEL<1, kCap2<float>>, g, b, l.stream, m, a); break;                         \
      case 6: launch_pdl(KERNEL<2, 1>, g, b, l.stream, m, a); break;                                    \
      case 7: launch_pdl(KERNEL<2, kCap3<float>>, g, b, l.stream, m, a); break;                         \
      case 8: launch_pdl(KERNEL<3, kCap<float>>, g, b, l.stream, m, a); break;                          \
      case 9: launch_pdl(KERNEL<3, kCap2<float>>, g, b, l.stream, m, a); break;                         \
      default: launch_pdl(KERNEL<0, 1>, g, b, l.stream, m, a); break;                                   \
    }                                                                                               \
  } while (0)

void launch_gradient_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  NF_DELTA_DISPATCH(gradient_delta_kernel, m, a, l);
}
void launch_flux_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  NF_DELTA_DISPATCH(flux_delta_kernel, m, a, l);
}
// The mixed form with FP32 copies: ghost states and boundary fluxes computed
// in FP64 from the FP32 primitives or face states (boundary faces are a few
// percent of the faces) and stored in FP32 for the FP32 node kernels.
__global__ void __launch_bounds__(256) ghost32_kernel(MeshView<double> m, StageArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (b >= m.nb) return;
  const int c = checked(m.b_cell[b], m.n, a.status), f = checked(m.b_face[b], m.n_faces, a.status);
  const int F = m.n_faces, st = m.stride;
  double V[5], G[5];
#pragma unroll
  for (int k = 0; k < 5; k++) V[k] = double(a.Vin32[k * st + c]);
  const double nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
  ghost_state<double>(m.patches[checked(m.b_patch[b], m.n_patches, a.status)], V, nh, G);
#pragma unroll
  for (int k = 0; k < 5; k++) a.vg32[k * m.bstride + b] = float(G[k]);
}

__global__ void __launch_bounds__(256) boundary_flux32_kernel(MeshView<double> m, StageArgs a) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  pdl_launch_dependents();
  pdl_wait_previous();
  if (b >= m.nb) return;
  const int c = checked(m.b_cell[b], m.n, a.status), q = checked(m.b_fs[b], 4, a.status),
            f = checked(m.b_face[b], m.n_faces, a.status);
  const int F = m.n_faces, st = m.stride;
  double VL[5], VR[5];
#pragma unroll
  for (int k = 0; k < 5; k++) VL[k] = double(a.second_order ? a.fs32[(q * 5 + k) * st + c] : a.Vin32[k * st + c]);
  const double nh[3] = {m.nhat[f], m.nhat[F + f], m.nhat[2 * F + f]};
  ghost_state<double>(m.patches[checked(m.b_patch[b], m.n_patches, a.status)], VL, nh, VR);
  double Fl[5];
  rusanov_fast<double>(VL, VR, nh, m.area[f], Fl);
#pragma unroll
  for (int k = 0; k < 5; k++) a.fb32[k * m.bstride + b] = float(Fl[k]);
}

// mixed form with FP32 copies: the node kernels in FP32 (no fused time step)
void launch_gradient_m32(const MeshView<float>& m, const StageArgs& a, Launch l) {
  const DtFuse d{0.0, nullptr, nullptr};
  const int b = fast_block(l.block);
  const int g = grid_for(m.n, b);
  switch (l.variant) {
    case 1: launch_pdl(gradient_node_kernel<float, 1, 1, false>, g, b, l.stream, m, a, d); break;
    case 2: launch_pdl(gradient_node_kernel<float, 0, kCap<float>, false>, g, b, l.stream, m, a, d); break;
    case 3: launch_pdl(gradient_node_kernel<float, 1, kCap<float>, false>, g, b, l.stream, m, a, d); break;
    case 4: launch_pdl(gradient_node_kernel<float, 0, kCap2<float>, false>, g, b, l.stream, m, a, d); break;
    case 5: launch_pdl(gradient_node_kernel<float, 1, kCap2<float>, false>, g, b, l.stream, m, a, d); break;
    case 6: launch_pdl(gradient_node_kernel<float, 2, 1, false>, g, b, l.stream, m, a, d); break;
    case 7: launch_pdl(gradient_node_kernel<float, 2, kCap3<float>, false>, g, b, l.stream, m, a, d); break;
    case 8: launch_pdl(gradient_node_kernel<float, 3, kCap<float>, false>, g, b, l.stream, m, a, d); break;
    case 9: launch_pdl(gradient_node_kernel<float, 3, kCap2<float>, false>, g, b, l.stream, m, a, d); break;
    default: launch_pdl(gradient_node_kernel<float, 0, 1, false>, g, b, l.stream, m, a, d); break;
  }
}
void launch_flux_m32(const MeshView<float>& m, const StageArgs& a, Launch l) {
  NF_NODE_DISPATCH(flux_node_kernel, float, m, a, l);
}
void launch_ghost_m32(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) launch_pdl(ghost32_kernel, grid_for(m.nb, l.block), l.block, l.stream, m, a);
}
void launch_bflux_m32(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) launch_pdl(boundary_flux32_kernel, grid_for(m.nb, l.block), l.block, l.stream, m, a);
}
void launch_ghost_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) launch_pdl(ghost_kernel<double, false>, grid_for(m.nb, l.block), l.block, l.stream, m, a);
}
void launch_bflux_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) launch_pdl(boundary_flux_kernel<double, false>, grid_for(m.nb, l.block), l.block, l.stream, m, a);
}
void launch_bflux_mixed(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) launch_pdl(boundary_flux_delta_kernel, grid_for(m.nb, l.block), l.block, l.stream, m, a);
}
__global__ void fastmath_kernel(const double* x, int n, double* rcp, double* rsq) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rcp[i] = nr_rcp(x[i]);
  rsq[i] = nr_rsqrt(x[i]);
}
void launch_fastmath(const double* x, int n, double* rcp, double* rsq, Launch l) {
  fastmath_kernel<<<grid_for(n, l.block), l.block, 0, l.stream>>>(x, n, rcp, rsq);
}

void launch_prim_fast(int n, int stride, const double* U, double* V, float* V32, Launch l) {
  prim_kernel_fast<false><<<grid_for(n, l.block), l.block, 0, l.stream>>>(n, stride, U, V, V32);
}

}  // namespace nf
