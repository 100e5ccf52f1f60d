// Kernels with reciprocals and fused multiply-adds (FP64), and the
// mixed-precision form (FP32 face work, FP64 state and update).
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

// one thread per cell, at most 128 threads per block (the kernels' launch bounds)
static inline int fast_block(int b) { return b > 128 ? 128 : b; }

void launch_gradient_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  const int b = fast_block(l.block);
  if (l.variant == 1) gradient_fast_kernel<double, true><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
  else gradient_fast_kernel<double, false><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
}
void launch_flux_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  const int b = fast_block(l.block);
  if (l.variant == 1) flux_fast_kernel<double, true><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
  else flux_fast_kernel<double, false><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
}
void launch_gradient_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  const int b = fast_block(l.block);
  if (l.variant == 1) gradient_fast_kernel<float, true><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
  else gradient_fast_kernel<float, false><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
}
void launch_flux_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  const int b = fast_block(l.block);
  if (l.variant == 1) flux_fast_kernel<float, true><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
  else flux_fast_kernel<float, false><<<grid_for(m.n, b), b, 0, l.stream>>>(m, a);
}
void launch_ghost_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) ghost_kernel<double, false><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_bflux_fast(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) boundary_flux_kernel<double, false><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_ghost_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) ghost_kernel<float, false><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_bflux_mixed(const MeshView<float>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) boundary_flux_kernel<float, false><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_prim_fast(int n, int stride, const double* U, double* V, float* V32, Launch l) {
  prim_kernel_fast<false><<<grid_for(n, l.block), l.block, 0, l.stream>>>(n, stride, U, V, V32);
}

}  // namespace nf
