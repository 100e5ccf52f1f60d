// Kernels in the reference's operation order. Compiled with -fmad=false so
// no multiply-add is contracted: every operation rounds as in the reference.
#include "launch.hpp"

namespace nf {

template <bool kRef>
__global__ void __launch_bounds__(256) prim_kernel(int n, int st, const double* __restrict__ U, double* __restrict__ V,
                                                  float* __restrict__ V32) {
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

void launch_gradient_ref(const MeshView<double>& m, const StageArgs& a, Launch l) {
  gradient_limiter_kernel<double, true><<<grid_for(5 * m.n, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_flux_ref(const MeshView<double>& m, const StageArgs& a, Launch l) {
  flux_update_kernel<double, true><<<grid_for(4 * m.n, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_ghost_ref(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) ghost_kernel<double, true><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_bflux_ref(const MeshView<double>& m, const StageArgs& a, Launch l) {
  if (m.nb > 0) boundary_flux_kernel<double, true><<<grid_for(m.nb, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_timestep(const MeshView<double>& m, const DtArgs& a, Launch l) {
  timestep_kernel<true><<<grid_for(m.n, l.block), l.block, 0, l.stream>>>(m, a);
}
void launch_prim_ref(int n, int stride, const double* U, double* V, float* V32, Launch l) {
  prim_kernel<true><<<grid_for(n, l.block), l.block, 0, l.stream>>>(n, stride, U, V, V32);
}

}  // namespace nf
