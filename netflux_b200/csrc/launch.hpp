// Host-callable launchers of the device kernels. Each arithmetic form lives
// in its own translation unit: kernels_ref.cu is compiled with -fmad=false
// (reference rounding), kernels_fast.cu with contraction on.
#pragma once

#include <cuda_runtime.h>

#include "kernels.cuh"

namespace nf {

struct Launch {
  int block;
  cudaStream_t stream;
  int variant = 0;  // fast kernels: bit 0 software-pipelined, bit 1 registers capped for occupancy
};

// reference-order FP64 (kernels_ref.cu)
void launch_gradient_ref(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_flux_ref(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_ghost_ref(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_bflux_ref(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_timestep(const MeshView<double>& m, const DtArgs& a, Launch l);
void launch_prim_ref(int n, int stride, const double* U, double* V, float* V32, Launch l);

// fast FP64 and mixed FP32/FP64 (kernels_fast.cu)
// dt, when not null, makes the gradient kernel compute the next step's time
// step too (the last stage)
void launch_gradient_fast(const MeshView<double>& m, const StageArgs& a, const DtFuse* dt, Launch l);
void launch_flux_fast(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_gradient_mixed(const MeshView<float>& m, const StageArgs& a, Launch l);
void launch_flux_mixed(const MeshView<float>& m, const StageArgs& a, Launch l);
void launch_ghost_fast(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_bflux_fast(const MeshView<double>& m, const StageArgs& a, Launch l);
// mixed: ghosts come from launch_ghost_fast (FP64); boundary fluxes are
// stored as FP32 differences to the owner's physical flux
void launch_bflux_mixed(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_prim_fast(int n, int stride, const double* U, double* V, float* V32, Launch l);
// mixed with FP32 copies: the FP32 node kernels and the boundary kernels that
// read and write the FP32 copies (kernels_fast.cu)
void launch_gradient_m32(const MeshView<float>& m, const StageArgs& a, Launch l);
void launch_flux_m32(const MeshView<float>& m, const StageArgs& a, Launch l);
void launch_ghost_m32(const MeshView<double>& m, const StageArgs& a, Launch l);
void launch_bflux_m32(const MeshView<double>& m, const StageArgs& a, Launch l);
// the fast forms' reciprocal and reciprocal square root, elementwise (self-test)
void launch_fastmath(const double* x, int n, double* rcp, double* rsq, Launch l);

}  // namespace nf
