// Solver context and the C ABI declared in include/netflux_b200.h.
//
// The context uploads the mesh once (device numbering, see kernels.cuh), owns
// every device buffer, one stream and the CUDA graphs of the step, and
// enqueues per step:
//   [dt reset + timestep kernel]   EulerSolver::calc_timestep
//   per stage: gradient_limiter, flux_update
//   [end-of-step kernel]           time += dt (Driver.cpp:47), validity of dt
// The primitives of successive stage inputs alternate between two buffers, so
// the buffer that fed the last stage still holds them when the next
// calc_timestep runs; the reference reads exactly those (Solver.cpp:250).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/netflux_b200.h"
#include "launch.hpp"
#include "mesh.hpp"


namespace {

thread_local std::string g_create_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    release();
    n = count;
    if (count) ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
  }
  void upload(const std::vector<T>& h, cudaStream_t s) {
    alloc(h.size());
    if (n) ck(cudaMemcpyAsync(p, h.data(), n * sizeof(T), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
  }
  void zero(cudaStream_t s) {
    if (n) ck(cudaMemsetAsync(p, 0, n * sizeof(T), s), "cudaMemsetAsync");
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
};

__global__ void scal_kernel(double* scal, int op, unsigned* status) {
  using namespace nf;
  if (op == 0) {  // reset the dt minima before the timestep kernel
    scal[kScalDtMin] = DBL_MAX;
    scal[kScalDtNext] = DBL_MAX;
  } else {  // end of step: time += dt actually used
    // the computed dt must be valid (Solver.cpp:267-268); the dt clipped at
    // t_end may be 0 once the end time is reached
    const double raw = scal[kScalDtMin];
    if (!(raw > 0.0) || !isfinite(raw)) atomicOr(status, kErrDt);
    const double dt = stage_dt(scal);
    scal[kScalDtUsed] = dt;
    scal[kScalTime] = scal[kScalTime] + dt;
    if (op == 2) {  // the last stage computed the next step's dt
      scal[kScalDtMin] = scal[kScalDtNext];
      scal[kScalDtNext] = DBL_MAX;
    }
  }
}

// Copy the status word and the device scalars into host-mapped memory. The
// host reads them after synchronising the solver stream; done by a kernel
// rather than a device-to-host memcpy, so the read-back never queues on a
// copy engine behind a large snapshot copy running on a side stream.
__global__ void report_kernel(const unsigned* status, const double* scal, unsigned* h_status, double* h_scal) {
  if (threadIdx.x == 0) *h_status = *status;
  if (threadIdx.x < nf::kScalCount) h_scal[threadIdx.x] = scal[threadIdx.x];
}

// max(a, b) that keeps a NaN from either operand (fmax would drop it, and a
// non-finite residual must not vanish from the L-infinity norm).
__device__ __forceinline__ double max_keep_nan(double a, double b) { return (a != a || a > b) ? a : b; }

// Per-case RMS and max of the per-cell density residual (deterministic: fixed
// chunking, fixed summation order).
__global__ void residual_partials_kernel(const double* __restrict__ r, const long long* __restrict__ chunk_begin,
                                         const long long* __restrict__ chunk_end, double* __restrict__ part) {
  const int b = blockIdx.x;
  const long long beg = chunk_begin[b], end = chunk_end[b];
  double s = 0.0, mx = 0.0;
  for (long long c = beg + threadIdx.x; c < end; c += blockDim.x) {
    const double v = r[c];
    s += v * v;
    mx = max_keep_nan(mx, fabs(v));
  }
  __shared__ double ss[256], sm[256];
  ss[threadIdx.x] = s;
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      ss[threadIdx.x] += ss[threadIdx.x + w];
      sm[threadIdx.x] = max_keep_nan(sm[threadIdx.x], sm[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * b] = ss[0];
    part[2 * b + 1] = sm[0];
  }
}

__global__ void residual_finalize_kernel(const double* __restrict__ part, const int* __restrict__ case_chunk0,
                                         const long long* __restrict__ case_cells, int n_cases,
                                         double* __restrict__ out) {
  const int cs = blockIdx.x * blockDim.x + threadIdx.x;
  if (cs >= n_cases) return;
  double s = 0.0, mx = 0.0;
  for (int b = case_chunk0[cs]; b < case_chunk0[cs + 1]; b++) {
    s += part[2 * b];
    mx = max_keep_nan(mx, part[2 * b + 1]);
  }
  const long long n = case_cells[cs];
  out[2 * cs] = n > 0 ? sqrt(s / double(n)) : 0.0;
  out[2 * cs + 1] = mx;
}

// Halo exchange of a mesh split across solvers: the stage-input primitives of
// listed cells (device order) gathered into / scattered from [5][n] rows.
// Halo rows of a mesh split across solvers: the primitives V and the conserved
// state U the next stage reads (its stage input; the stage update of a halo
// cell starts from it), 10 rows of [n] in buf.
__global__ void halo_pack_kernel(int64_t n, int st, const int64_t* __restrict__ cells, const double* __restrict__ V,
                                 const double* __restrict__ U, double* __restrict__ buf) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cells[i];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    buf[k * n + i] = V[size_t(k) * st + c];
    buf[(5 + k) * n + i] = U[size_t(k) * st + c];
  }
}
__global__ void halo_unpack_kernel(int64_t n, int st, const int64_t* __restrict__ cells,
                                   const double* __restrict__ buf, double* __restrict__ V, double* __restrict__ U) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cells[i];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    V[size_t(k) * st + c] = buf[k * n + i];
    U[size_t(k) * st + c] = buf[(5 + k) * n + i];
  }
}
// One link of a split mesh: the receiver's halo rows (V and the stage input U)
// take the sender's (V_from / U_from on this device or, with peer access, on
// another GPU: plain loads over NVLink).
__global__ void halo_copy_kernel(int64_t n, int st_from, const int64_t* __restrict__ from_cells,
                                 const double* __restrict__ V_from, const double* __restrict__ U_from, int st_to,
                                 const int64_t* __restrict__ to_cells, double* __restrict__ V_to,
                                 double* __restrict__ U_to) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t a = from_cells[i], b = to_cells[i];
#pragma unroll
  for (int k = 0; k < 5; k++) {
    V_to[size_t(k) * st_to + b] = V_from[size_t(k) * st_from + a];
    U_to[size_t(k) * st_to + b] = U_from[size_t(k) * st_from + a];
  }
}

// The global time step of a split mesh: every part's minimum replaced by the
// minimum over the parts (peer loads and stores across GPUs); a NaN wins, so
// every part's end-of-step check reports it.
__global__ void split_dt_min_kernel(double* const* __restrict__ scal, int n_parts) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = scal[0][nf::kScalDtMin];
  for (int i = 1; i < n_parts && !isnan(m); i++) {
    const double v = scal[i][nf::kScalDtMin];
    if (isnan(v) || v < m) m = v;
  }
  for (int i = 0; i < n_parts; i++) scal[i][nf::kScalDtMin] = m;
}

// AoS state in reference cell order <-> SoA in device order.
__global__ void scatter_state_kernel(int n, int st, const long long* __restrict__ dev_of_ref,
                                     const double* __restrict__ aos, double* __restrict__ soa) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long long d = dev_of_ref[c];
#pragma unroll
  for (int k = 0; k < 5; k++) soa[k * st + d] = aos[5 * (long long)c + k];
}

__global__ void gather_state_kernel(int n, int st, const long long* __restrict__ dev_of_ref,
                                    const double* __restrict__ soa, double* __restrict__ aos) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long long d = dev_of_ref[c];
#pragma unroll
  for (int k = 0; k < 5; k++) aos[5 * (long long)c + k] = soa[k * st + d];
}

}  // namespace

namespace nf {
// Error text returned by nf_last_error(NULL) for calls that have no solver.
void set_last_error_text(const std::string& msg) { g_create_error = msg; }
}  // namespace nf

// Largest cell count one solver takes: 20 rows of (N rounded up to 64) int
// offsets must stay below 2^31 (107,374,080 cells).
constexpr int64_t kMaxCells = (int64_t(INT32_MAX) / 20) / 64 * 64 - 64;
static_assert(20 * ((kMaxCells + 63) / 64 * 64) <= int64_t(INT32_MAX), "face-state rows of the largest mesh");

extern "C" int nf_check_mesh_size(int64_t n_cells, int64_t n_faces) {
  if (n_cells <= 0 || n_faces < 0) {
    g_create_error = "mesh has no cells";
    return NF_ERR_MESH;
  }
  // The stage kernels index the 20 face-state rows of [20][stride] arrays
  // with 32-bit products, so 20 * stride must stay below 2^31; faces are
  // numbered in 32-bit ints as well.
  if (n_cells > kMaxCells) {
    g_create_error = "mesh too large for one solver: " + std::to_string(n_cells) + " cells, at most " +
                     std::to_string(kMaxCells) + " (split larger meshes across solvers)";
    return NF_ERR_MESH;
  }
  if (n_faces >= (int64_t(1) << 30)) {
    g_create_error = "mesh too large for one solver: " + std::to_string(n_faces) + " faces, at most 2^30 - 1";
    return NF_ERR_MESH;
  }
  return NF_OK;
}

struct nf_solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  nf_params p{};
  int n = 0, stride = 0, n_faces = 0, n_cases = 1;
  int64_t n_nodes = 0;
  int block = 256;
  std::vector<int64_t> dev_of_ref;
  std::vector<int64_t> case_offsets;
  std::string err;

  // mesh
  DevBuf<int> slot, nbslot, b_cell, b_slot, b_face, b_patch, b_slotf;
  DevBuf<int> cnode, gcode, nbvf, nbsf;  // node-based layout of the fast forms
  DevBuf<double> S, nhat, area, rs, vol, dS, nodes4;
  DevBuf<float> nodes4_32;
  int nb = 0, bstride = 0;
  DevBuf<nf::PatchBC> patches;
  // state
  DevBuf<double> U, W, V0, V1, fs, grad, phi, R, dt_local, res_cell, scal, part, res_out, vg, fb;
  // FP64 form: the last stage also computes the next step's dt, into the
  // other per-cell dt buffer (dtl_cur names the one the next step uses);
  // dt_ready says the next step's dt is already on the device
  DevBuf<double> dt_local2;
  int dtl_cur = 0;
  bool dt_ready = false;
  DevBuf<double> Uold;       // U^n of the next step when set apart from U (nf_set_state_old)
  bool old_pending = false;
  DevBuf<float> fs32, grad32, phi32, fb32;  // mixed: increments, fields, boundary flux differences
  // mixed with FP32 copies: FP32 primitives of successive stage inputs (the
  // same double-buffering as V0/V1) and FP32 ghost states; fs32 and fb32
  // hold its face states and boundary fluxes
  DevBuf<float> V32a, V32b, vg32;
  DevBuf<unsigned> status;
  DevBuf<long long> chunk_begin, chunk_end, case_cells;
  DevBuf<int> case_chunk0;
  DevBuf<int> cell_case, case_frozen;  // per-cell case; per-case convergence freeze
  bool freeze = false;
  // limiter ratchet (extension): per-case switch and the kept limiter values
  bool ratchet_alloc = false, ratchet_step_done = false;
  int64_t steps_done = 0;  // steps since nf_set_state
  DevBuf<int> case_ratchet;
  DevBuf<double> phi_keep;
  DevBuf<float> phi_keep32;
  std::vector<int> h_ratchet;
  int n_chunks = 0;
  double* h_scal = nullptr;  // pinned
  // host-mapped copies of the status word and the scalars (report_kernel)
  unsigned* h_rep_status = nullptr;
  double* h_rep_scal = nullptr;
  unsigned* d_rep_status = nullptr;
  double* d_rep_scal = nullptr;
  // status and scalars into the mapped buffers, then wait for the stream
  void report() {
    report_kernel<<<1, 32, 0, stream>>>(status.p, scal.p, d_rep_status, d_rep_scal);
    ck(cudaGetLastError(), "report launch");
    ck(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
  }
  int vcur = 0;              // V buffer holding the primitives of the current state
  bool stepped = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // two steps from vcur = 0 / 1
  // launch configuration of the gradient and flux kernels (fast forms)
  struct KCfg {
    int block = 128;
    int variant = 0;
  };
  KCfg kgrad, kflux;
  bool tuned = false;
  DevBuf<double> stage;           // AoS staging for state transfers [N][5]
  // asynchronous state snapshots (nf_snapshot_begin / nf_snapshot_wait): a
  // second AoS staging buffer, copied to the host on its own stream
  // Two staging buffers, used in turn: a snapshot's gather waits (on the
  // device) only for the copy out of its buffer two snapshots back, so the
  // host never blocks in nf_snapshot_begin.
  DevBuf<double> snap[2];
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_ready = nullptr, snap_done[2] = {nullptr, nullptr};
  bool snap_used[2] = {false, false};
  int snap_k = 0;
  bool snap_pending = false;
  // asynchronous state uploads (nf_upload_begin / nf_upload_commit): two
  // more AoS staging buffers, used in turn and filled from the host on their
  // own stream, so the next state's copy never waits for the scatter of the
  // one before it (only for the scatter two uploads back)
  DevBuf<double> up[2];
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_done[2] = {nullptr, nullptr};  // copy into up[k] landed
  cudaEvent_t up_free[2] = {nullptr, nullptr};  // the scatter of up[k] is done reading it
  bool up_used[2] = {false, false};
  int up_k = 0;    // staging buffer of the next upload
  int up_cur = 0;  // staging buffer of the upload in flight
  bool up_pending = false;
  bool up_reading = false;  // copies may still read the caller's buffers (until nf_upload_wait)
  DevBuf<long long> d_dev_of_ref;  // [N]

  // per-kernel timing: events around every launch while prof_on
  bool prof_on = false;
  std::vector<cudaEvent_t> prof_ev;
  std::vector<int> prof_cls;
  size_t prof_used = 0;
  void prof_begin(int cls) {
    if (!prof_on) return;
    if (2 * prof_used + 2 > prof_ev.size()) {
      for (int k = 0; k < 64; k++) {
        cudaEvent_t e;
        ck(cudaEventCreate(&e), "cudaEventCreate");
        prof_ev.push_back(e);
      }
    }
    if (prof_cls.size() <= prof_used) prof_cls.resize(prof_used + 1);
    prof_cls[prof_used] = cls;
    ck(cudaEventRecord(prof_ev[2 * prof_used], stream), "cudaEventRecord");
  }
  void prof_end() {
    if (!prof_on) return;
    ck(cudaEventRecord(prof_ev[2 * prof_used + 1], stream), "cudaEventRecord");
    prof_used++;
  }

  double* Vbuf(int i) { return i ? V1.p : V0.p; }
  float* V32buf(int i) { return i ? V32b.p : V32a.p; }
  // the conserved state stage s reads (Solver.cpp:103-133: U, then the RK
  // stage W)
  double* stage_input(int s) { return (p.time_scheme == NF_TVD_RK3 && s > 0) ? W.p : U.p; }
  double* dtl(int i) { return i ? dt_local2.p : dt_local.p; }
  // the FP64 form's last stage computes the next step's dt (second order:
  // its gradient kernel reads the primitives the reference's dt reads)
  bool fuse_dt() const {
    return p.precision == NF_PREC_FP64 && p.spatial_order == NF_SECOND_ORDER && !p.dt_from_current_state;
  }
  // the mixed forms (TVD-RK3): the stage-2 flux kernel computes the next
  // step's dt from the primitives of its result, the last stage's input
  bool fuse_dt_flux() const {
    return (p.precision == NF_PREC_MIXED || p.precision == NF_PREC_MIXED32) && p.time_scheme == NF_TVD_RK3 &&
           !p.dt_from_current_state;
  }
  // primitives of Usrc into primitive buffer b (and its FP32 copy in the
  // mixed form with FP32 copies)
  void launch_prim(const double* Usrc, int b) {
    float* v32 = p.precision == NF_PREC_MIXED32 ? V32buf(b) : nullptr;
    if (p.precision == NF_PREC_FP64_REF) nf::launch_prim_ref(n, stride, Usrc, Vbuf(b), nullptr, launch());
    else nf::launch_prim_fast(n, stride, Usrc, Vbuf(b), v32, launch());
  }
  nf::Launch launch() const { return nf::Launch{block, stream}; }

  nf::MeshView<double> view64() const {
    const bool fast = p.precision != NF_PREC_FP64_REF;
    return nf::MeshView<double>{n, stride, n_faces, slot.p, nbslot.p, S.p, nhat.p, area.p, rs.p,
                                nodes4.p, cnode.p, gcode.p, nbvf.p, nbsf.p, vol.p, dS.p, patches.p, nb,
                                bstride, b_cell.p, b_slot.p, b_face.p, b_patch.p, fast ? b_slotf.p : b_slot.p,
                                int(n_nodes), int(patches.n)};
  }
  nf::MeshView<float> view32() const {
    return nf::MeshView<float>{n, stride, n_faces, slot.p, nbslot.p, nullptr, nullptr, nullptr, nullptr,
                               nodes4_32.p, cnode.p, gcode.p, nbvf.p, nbsf.p, vol.p, dS.p, patches.p, nb,
                               bstride, b_cell.p, b_slot.p, b_face.p, b_patch.p, b_slotf.p, int(n_nodes),
                               int(patches.n)};
  }

  void enqueue_dt() {
    if (dt_ready) return;  // the previous step's last stage computed it
    prof_begin(NF_KERNEL_OTHER);
    scal_kernel<<<1, 1, 0, stream>>>(scal.p, 0, status.p);
    prof_end();
    nf::DtArgs a;
    const int vb = p.dt_from_current_state ? vcur : (stepped ? 1 - vcur : vcur);
    a.V = Vbuf(vb);
    a.cfl = p.cfl;
    a.dt_local = p.local_time_stepping ? dtl(dtl_cur) : nullptr;
    a.dt_min_bits = reinterpret_cast<unsigned long long*>(scal.p + nf::kScalDtMin);
    a.status = status.p;
    a.cell_case = cell_case.p;
    a.case_frozen = freeze ? case_frozen.p : nullptr;
    prof_begin(NF_KERNEL_TIMESTEP);
    nf::launch_timestep(view64(), a, launch());
    prof_end();
  }

  // primitives of U in both V buffers (as after nf_set_state)
  void refresh_primitives() {
    for (int b = 0; b < 2; b++) launch_prim(U.p, b);
  }

  void ratchet_reset() {
    ratchet_step_done = false;
    if (!ratchet_alloc) return;
    std::fill(h_ratchet.begin(), h_ratchet.end(), 0);
    ck(cudaMemsetAsync(case_ratchet.p, 0, size_t(n_cases) * sizeof(int), stream), "ratchet reset");
    // bytes 0x7f: a value above every limiter value (<= 1) in FP64 and FP32
    if (phi_keep.p) ck(cudaMemsetAsync(phi_keep.p, 0x7f, size_t(5) * stride * sizeof(double), stream), "ratchet reset");
    if (phi_keep32.p)
      ck(cudaMemsetAsync(phi_keep32.p, 0x7f, size_t(5) * stride * sizeof(float), stream), "ratchet reset");
  }
  void ratchet_start(int cs) {  // cs < 0: every case
    if (!ratchet_alloc) return;
    for (int k = 0; k < n_cases; k++)
      if (cs < 0 || k == cs) h_ratchet[size_t(k)] = 1;
    // pageable source: the call returns once the values are staged
    ck(cudaMemcpyAsync(case_ratchet.p, h_ratchet.data(), size_t(n_cases) * sizeof(int), cudaMemcpyHostToDevice,
                       stream),
       "ratchet H2D");
  }
  // steps before the ratchet's start step, or all of n once it has started
  int64_t ratchet_due(int64_t n) {
    if (!ratchet_alloc || p.limiter_ratchet_step <= 0 || ratchet_step_done) return n;
    if (steps_done >= p.limiter_ratchet_step) {
      ratchet_start(-1);
      ratchet_step_done = true;
      return n;
    }
    return std::min<int64_t>(n, p.limiter_ratchet_step - steps_done);
  }

  // n x (calc_timestep + step), replays of a two-step CUDA graph where
  // possible; the ratchet starts at its step.
  void run_steps(int64_t n) {
    if (n > 0 && old_pending) {  // this step's U^n is not U: outside the graphs
      ratchet_due(1);
      enqueue_dt();
      enqueue_step();
      steps_done++;
      n--;
    }
    while (n > 0) {
      int64_t left = ratchet_due(n);
      n -= left;
      steps_done += left;
      if (left >= 2 && stepped) {
        const int v0 = vcur;
        if (!graph[v0]) {
          // capture two steps: the V buffers return to their roles afterwards
          cudaGraph_t g = nullptr;
          ck(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "begin capture");
          for (int k = 0; k < 2; k++) {
            enqueue_dt();
            enqueue_step();
          }
          ck(cudaStreamEndCapture(stream, &g), "end capture");
          ck(cudaGraphInstantiate(&graph[v0], g, 0), "graph instantiate");
          cudaGraphDestroy(g);
          vcur = v0;
        }
        while (left >= 2) {
          ck(cudaGraphLaunch(graph[v0], stream), "graph launch");
          left -= 2;
        }
      }
      while (left > 0) {
        enqueue_dt();
        enqueue_step();
        left--;
      }
    }
  }

  void launch_gradient(const nf::StageArgs& a, const KCfg& k, const nf::DtFuse* dtf = nullptr) {
    const nf::Launch l{k.block, stream, k.variant};
    if (p.precision == NF_PREC_MIXED) nf::launch_gradient_mixed(view32(), a, l);
    else if (p.precision == NF_PREC_MIXED32) nf::launch_gradient_m32(view32(), a, l);
    else if (p.precision == NF_PREC_FP64) nf::launch_gradient_fast(view64(), a, dtf, l);
    else nf::launch_gradient_ref(view64(), a, launch());
  }
  void launch_flux(const nf::StageArgs& a, const KCfg& k) {
    const nf::Launch l{k.block, stream, k.variant};
    if (p.precision == NF_PREC_MIXED) nf::launch_flux_mixed(view32(), a, l);
    else if (p.precision == NF_PREC_MIXED32) nf::launch_flux_m32(view32(), a, l);
    else if (p.precision == NF_PREC_FP64) nf::launch_flux_fast(view64(), a, l);
    else nf::launch_flux_ref(view64(), a, launch());
  }
  // ghost states and boundary fluxes of the stage, in each form's precision
  void launch_ghost(const nf::StageArgs& a) {
    if (p.precision == NF_PREC_FP64_REF) nf::launch_ghost_ref(view64(), a, launch());
    else if (p.precision == NF_PREC_MIXED32) nf::launch_ghost_m32(view64(), a, launch());
    else nf::launch_ghost_fast(view64(), a, launch());
  }
  void launch_bflux(const nf::StageArgs& a) {
    if (p.precision == NF_PREC_MIXED) nf::launch_bflux_mixed(view64(), a, launch());
    else if (p.precision == NF_PREC_MIXED32) nf::launch_bflux_m32(view64(), a, launch());
    else if (p.precision == NF_PREC_FP64) nf::launch_bflux_fast(view64(), a, launch());
    else nf::launch_bflux_ref(view64(), a, launch());
  }
  // launch variants the tuner may pick (gradient, flux)
  int grad_variants() const { return 10; }
  int flux_variants() const { return 10; }

  // Arguments of the first stage of a step from the current state, writing
  // only scratch (face states, W, the other primitive buffer).
  nf::StageArgs first_stage_args() {
    nf::StageArgs a{};
    a.second_order = p.spatial_order == NF_SECOND_ORDER;
    a.barth = p.limiter == NF_LIMITER_BARTH;
    a.scheme = p.time_scheme == NF_TVD_RK3 ? 1 : 0;
    a.stage = 0;
    a.local_dt = p.local_time_stepping;
    a.Vin = Vbuf(vcur);
    a.Vout = Vbuf(1 - vcur);
    a.fs = fs.p;
    a.vg = vg.p;
    a.fb = fb.p;
    a.fb32 = fb32.p;
    if (p.precision == NF_PREC_MIXED32) {
      a.Vin32 = V32buf(vcur);
      a.Vout32 = V32buf(1 - vcur);
      a.vg32 = vg32.p;
    }
    a.dt_local = dtl(dtl_cur);
    a.scal = scal.p;
    a.status = status.p;
    a.Uin = U.p;
    a.Uout = W.p;
    a.fs32 = fs32.p;
    return a;
  }

  // Pick block size and variant of the gradient and flux kernels by timing
  // each candidate on the current state (CUDA events on this stream).
  void tune() {
    tuned = true;
    if (p.precision == NF_PREC_FP64_REF) return;  // reference form: fixed shape
    const int other = 1 - vcur;
    std::vector<double> keep(size_t(5) * stride);
    std::vector<float> keep32(p.precision == NF_PREC_MIXED32 ? size_t(5) * stride : 0);
    ck(cudaMemcpyAsync(keep.data(), Vbuf(other), keep.size() * sizeof(double), cudaMemcpyDeviceToHost, stream),
       "tune save");
    if (!keep32.empty())
      ck(cudaMemcpyAsync(keep32.data(), V32buf(other), keep32.size() * sizeof(float), cudaMemcpyDeviceToHost,
                         stream),
         "tune save");
    ck(cudaStreamSynchronize(stream), "tune sync");
    nf::StageArgs a = first_stage_args();
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    auto time_it = [&](auto&& fn) {
      fn();  // warm
      ck(cudaEventRecord(e0, stream), "cudaEventRecord");
      for (int r = 0; r < 3; r++) fn();
      ck(cudaEventRecord(e1, stream), "cudaEventRecord");
      ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0.f;
      ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      return ms;
    };
    auto cands = [](int n_variants) {
      std::vector<KCfg> c;
      for (int b : {128, 64})
        for (int v = 0; v < n_variants; v++) c.push_back(KCfg{b, v});
      return c;
    };
    if (a.second_order) {
      launch_ghost(a);
      float best = 1e30f;
      for (const KCfg& k : cands(grad_variants())) {
        const float t = time_it([&] { launch_gradient(a, k); });
        if (t < best) {
          best = t;
          kgrad = k;
        }
      }
      launch_gradient(a, kgrad);
    }
    launch_bflux(a);
    float best = 1e30f;
    for (const KCfg& k : cands(flux_variants())) {
      const float t = time_it([&] { launch_flux(a, k); });
      if (t < best) {
        best = t;
        kflux = k;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ck(cudaMemcpyAsync(Vbuf(other), keep.data(), keep.size() * sizeof(double), cudaMemcpyHostToDevice, stream),
       "tune restore");
    if (!keep32.empty())
      ck(cudaMemcpyAsync(V32buf(other), keep32.data(), keep32.size() * sizeof(float), cudaMemcpyHostToDevice,
                         stream),
         "tune restore");
    ck(cudaMemsetAsync(status.p, 0, sizeof(unsigned), stream), "status reset");
    ck(cudaStreamSynchronize(stream), "tune sync");
    for (auto& g : graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  }

  int n_stages() const { return p.time_scheme == NF_TVD_RK3 ? 3 : 1; }
  int stage_next = 0;  // the next stage nf_stage may enqueue

  void enqueue_step() {
    for (int s = 0; s < n_stages(); s++) enqueue_stage(s);
    stage_next = 0;
  }

  // One stage of the step; the last one also ends the step.
  void enqueue_stage(int s) {
    const int n_stages = this->n_stages();
    const bool fuse = fuse_dt() || fuse_dt_flux();
    nf::DtFuse dtf{p.cfl, p.local_time_stepping ? dtl(1 - dtl_cur) : nullptr,
                   reinterpret_cast<unsigned long long*>(scal.p + nf::kScalDtNext)};
    {
      nf::StageArgs a{};
      a.second_order = p.spatial_order == NF_SECOND_ORDER;
      a.barth = p.limiter == NF_LIMITER_BARTH;
      a.scheme = p.time_scheme == NF_TVD_RK3 ? 1 : 0;
      a.stage = s;
      a.local_dt = p.local_time_stepping;
      a.freeze = freeze && p.local_time_stepping;
      a.cell_case = cell_case.p;
      if (a.freeze && p.precision != NF_PREC_FP64_REF) a.case_frozen = case_frozen.p;
      a.Vin = Vbuf(vcur);
      a.Vout = Vbuf(1 - vcur);
      a.fs = fs.p;
      a.vg = vg.p;
      a.fb = fb.p;
      a.fb32 = fb32.p;
      a.grad = p.keep_stage_fields ? grad.p : nullptr;
      a.phi = p.keep_stage_fields ? phi.p : nullptr;
      a.R = p.keep_stage_fields ? R.p : nullptr;
      a.res_cell = s == 0 ? res_cell.p : nullptr;
      a.dt_local = dtl(dtl_cur);
      a.scal = scal.p;
      a.status = status.p;
      if (ratchet_alloc) {
        a.lim_ratchet = case_ratchet.p;
        a.phi_keep = phi_keep.p;
        a.phi_keep32 = phi_keep32.p;
      }
      if (a.scheme == 0) {
        a.Uin = U.p;
        a.Uout = U.p;
      } else if (s == 0) {
        a.Uin = U.p;
        a.Uout = W.p;
      } else if (s == 1) {
        a.Uin = W.p;
        a.Un = old_pending ? Uold.p : U.p;
        a.Uout = W.p;
      } else {
        a.Uin = W.p;
        a.Un = old_pending ? Uold.p : U.p;
        a.Uout = U.p;
      }
      if (p.precision == NF_PREC_MIXED32) {
        a.Vin32 = V32buf(vcur);
        a.Vout32 = V32buf(1 - vcur);
        a.vg32 = vg32.p;
        // the FP64 primitives only where a time-step kernel reads them: the
        // state the next time step reads (the last stage's input, Q3, or with
        // dt_from_current_state the step's result), unless the stage-2 flux
        // kernel computes that time step itself from its FP64 result
        const int dt_stage = p.dt_from_current_state ? n_stages - 1 : std::max(n_stages - 2, 0);
        if (s != dt_stage || fuse_dt_flux()) a.Vout = nullptr;
      }
      if (fuse_dt_flux() && s == n_stages - 2) {
        a.dt_next = dtf.dt_next;
        a.dt_next_min = dtf.dt_min_bits;
        a.dS = dS.p;
        a.cfl = p.cfl;
      }
      if (p.precision == NF_PREC_MIXED || p.precision == NF_PREC_MIXED32) {
        a.fs32 = fs32.p;
        a.grad32 = p.keep_stage_fields ? grad32.p : nullptr;
        a.phi32 = p.keep_stage_fields ? phi32.p : nullptr;
      }
      if (a.second_order) {
        prof_begin(NF_KERNEL_OTHER);
        launch_ghost(a);
        prof_end();
        prof_begin(NF_KERNEL_GRADIENT);
        launch_gradient(a, kgrad, (fuse_dt() && s == n_stages - 1) ? &dtf : nullptr);
        prof_end();
      }
      prof_begin(NF_KERNEL_OTHER);
      launch_bflux(a);
      prof_end();
      prof_begin(NF_KERNEL_FLUX);
      launch_flux(a, kflux);
      prof_end();
      vcur = 1 - vcur;
    }
    if (s < n_stages - 1) return;
    prof_begin(NF_KERNEL_OTHER);
    scal_kernel<<<1, 1, 0, stream>>>(scal.p, fuse ? 2 : 1, status.p);
    prof_end();
    if (fuse) {
      dtl_cur = 1 - dtl_cur;
      dt_ready = true;
    }
    stepped = true;
    old_pending = false;  // solution_old = solution (Solver.cpp:51)
  }

  // Report a device-side failure as the reference would have (exceptions in
  // calc_timestep / check_flux_balance_validity become status codes).
  int check_status() {
    report();
    const unsigned st = *h_rep_status;
    if (st & nf::kErrNonFinite) {
      err = "unphysical values detected in the flux_balance field of the Euler solver (non-finite)";
      return NF_ERR_NONPHYSICAL;
    }
    if (st & nf::kErrNonPhysical) {
      err = "unphysical state: density or pressure <= 0 after an update";
      return NF_ERR_NONPHYSICAL;
    }
    if (st & nf::kErrDt) {
      err = "Invalid dt calculated";
      return NF_ERR_DT;
    }
    if (st & nf::kErrIndex) {
      err = "a mesh index read by a kernel is out of range (checked in the NF_DEBUG build)";
      return NF_ERR_MESH;
    }
    return NF_OK;
  }

  // Make the AoS state in device memory (reference cell order) the solver's
  // state: permute it into U, primitives of it in both V buffers (the first
  // calc_timestep reads them, like the harness-initialised reference), and
  // the step bookkeeping of a fresh start. Queued on the solver stream.
  void adopt_state(const double* aos) {
    const int st = stride;
    scatter_state_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, st, d_dev_of_ref.p, aos, U.p);
    for (int b = 0; b < 2; b++) launch_prim(U.p, b);
    vcur = 0;
    dtl_cur = 0;
    dt_ready = false;
    stage_next = 0;
    stepped = false;
    old_pending = false;
    steps_done = 0;
    ratchet_reset();
    ck(cudaMemsetAsync(status.p, 0, sizeof(unsigned), stream), "status reset");
  }

  ~nf_solver() {
    if (snap_stream) cudaStreamSynchronize(snap_stream);  // copies may still write the caller's memory
    if (snap_ready) cudaEventDestroy(snap_ready);
    for (auto e : snap_done)
      if (e) cudaEventDestroy(e);
    if (snap_stream) cudaStreamDestroy(snap_stream);
    if (up_stream) cudaStreamSynchronize(up_stream);  // copies may still read the caller's memory
    for (int k = 0; k < 2; k++) {
      if (up_done[k]) cudaEventDestroy(up_done[k]);
      if (up_free[k]) cudaEventDestroy(up_free[k]);
    }
    if (up_stream) cudaStreamDestroy(up_stream);
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    for (auto e : prof_ev) cudaEventDestroy(e);
    if (h_scal) cudaFreeHost(h_scal);
    if (h_rep_status) cudaFreeHost(h_rep_status);
    if (h_rep_scal) cudaFreeHost(h_rep_scal);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <typename F>
int guarded(nf_solver* s, F&& fn) {
  if (!s) return NF_ERR_ARG;
  try {
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != s->device) ck(cudaSetDevice(s->device), "cudaSetDevice");
    return fn();
  } catch (const CudaError& e) {
    s->err = e.what();
    return NF_ERR_CUDA;
  } catch (const std::exception& e) {
    s->err = e.what();
    return NF_ERR_ARG;
  }
}

nf_mesh* wrap_mesh(nf::Mesh&& m) {
  auto* h = new nf_mesh;
  h->m = std::move(m);
  return h;
}

}  // namespace

// One mesh split across solvers (partition.py's parts): the owner of every
// halo cell writes its primitives into the receiving part before each stage,
// by a kernel on the receiver's stream that reads the owner's buffer (same
// GPU, or a peer GPU over NVLink with plain loads). Events order the parts'
// streams; the host waits on nothing inside a step.
struct nf_split {
  struct Link {
    int from = 0, to = 0;
    int64_t n = 0;
    DevBuf<int64_t> from_cells, to_cells;  // both on the receiver's device
  };
  std::vector<nf_solver*> parts;
  std::vector<std::unique_ptr<Link>> links;
  std::vector<cudaEvent_t> ready, copied;  // per part: stage input ready; its incoming halos written
  cudaEvent_t dt_done = nullptr;           // the global dt written into every part
  DevBuf<double*> scal_ptrs;               // on part 0's device
  std::string err;
  bool global_dt = false;

  void set_dev(int d) { ck(cudaSetDevice(d), "cudaSetDevice"); }
  // every part's halo rows from their owners, before stage k of every part
  void exchange(int k) {
    for (size_t i = 0; i < parts.size(); i++) {
      set_dev(parts[i]->device);
      ck(cudaEventRecord(ready[i], parts[i]->stream), "cudaEventRecord");
    }
    for (auto& lk : links) {
      nf_solver* a = parts[size_t(lk->from)];
      nf_solver* b = parts[size_t(lk->to)];
      set_dev(b->device);
      ck(cudaStreamWaitEvent(b->stream, ready[size_t(lk->from)], 0), "cudaStreamWaitEvent");
      halo_copy_kernel<<<int((lk->n + 255) / 256), 256, 0, b->stream>>>(
          lk->n, a->stride, lk->from_cells.p, a->Vbuf(a->vcur), a->stage_input(k), b->stride, lk->to_cells.p,
          b->Vbuf(b->vcur), b->stage_input(k));
      ck(cudaGetLastError(), "halo copy launch");
    }
    for (size_t i = 0; i < parts.size(); i++) {
      set_dev(parts[i]->device);
      ck(cudaEventRecord(copied[i], parts[i]->stream), "cudaEventRecord");
    }
    // stage k of a sender updates in place what the receivers have just read
    // (the RK stage W at stage 1, U under explicit Euler): it waits for their
    // copies
    for (auto& lk : links) {
      nf_solver* a = parts[size_t(lk->from)];
      set_dev(a->device);
      ck(cudaStreamWaitEvent(a->stream, copied[size_t(lk->to)], 0), "cudaStreamWaitEvent");
    }
  }
  // with a global dt: the minimum over the parts into every part
  void reduce_dt() {
    for (size_t i = 0; i < parts.size(); i++) {
      set_dev(parts[i]->device);
      ck(cudaEventRecord(ready[i], parts[i]->stream), "cudaEventRecord");
    }
    nf_solver* p0 = parts[0];
    set_dev(p0->device);
    for (size_t i = 1; i < parts.size(); i++)
      ck(cudaStreamWaitEvent(p0->stream, ready[i], 0), "cudaStreamWaitEvent");
    split_dt_min_kernel<<<1, 32, 0, p0->stream>>>(scal_ptrs.p, int(parts.size()));
    ck(cudaGetLastError(), "dt min launch");
    ck(cudaEventRecord(dt_done, p0->stream), "cudaEventRecord");
    for (size_t i = 1; i < parts.size(); i++) {
      set_dev(parts[i]->device);
      ck(cudaStreamWaitEvent(parts[i]->stream, dt_done, 0), "cudaStreamWaitEvent");
    }
  }
  void step() {
    for (nf_solver* s : parts) {
      set_dev(s->device);
      s->ratchet_due(1);
      s->enqueue_dt();
    }
    if (global_dt) reduce_dt();
    const int ns = parts[0]->n_stages();
    for (int k = 0; k < ns; k++) {
      exchange(k);
      for (nf_solver* s : parts) {
        set_dev(s->device);
        s->enqueue_stage(k);
      }
    }
    for (nf_solver* s : parts) s->steps_done++;
  }
  ~nf_split() {
    for (size_t i = 0; i < parts.size(); i++) {
      cudaSetDevice(parts[i]->device);
      cudaStreamSynchronize(parts[i]->stream);
    }
    for (auto e : ready)
      if (e) cudaEventDestroy(e);
    for (auto e : copied)
      if (e) cudaEventDestroy(e);
    if (dt_done) cudaEventDestroy(dt_done);
  }
};

// calls on a split mesh: the device is restored, exceptions become status codes
template <typename F>
int split_guarded(nf_split* sp, F&& fn) {
  if (!sp) return NF_ERR_ARG;
  int dev = 0;
  cudaGetDevice(&dev);
  int rc;
  try {
    rc = fn();
  } catch (const CudaError& e) {
    sp->err = e.what();
    rc = NF_ERR_CUDA;
  } catch (const std::exception& e) {
    sp->err = e.what();
    rc = NF_ERR_ARG;
  }
  cudaSetDevice(dev);
  return rc;
}

extern "C" {

// ---------------------------------------------------------------------------
// mesh
// ---------------------------------------------------------------------------
nf_mesh* nf_mesh_from_su2(const char* path, int n_patch_types, const char* const* patch_names,
                          const int* patch_types) {
  try {
    if (!path || n_patch_types < 0 || (n_patch_types && (!patch_names || !patch_types)))
      throw nf::MeshError("invalid arguments");
    std::vector<std::string> names;
    std::vector<int> types;
    for (int i = 0; i < n_patch_types; i++) {
      names.emplace_back(patch_names[i]);
      types.push_back(patch_types[i]);
    }
    return wrap_mesh(nf::read_su2(path, names, types));
  } catch (const std::exception& e) {
    g_create_error = std::string("Error reading su2 mesh '") + (path ? path : "") + "', " + e.what();
    return nullptr;
  }
}

nf_mesh* nf_mesh_from_arrays(int64_t n_nodes, const double* nodes, int64_t n_cells, const int64_t* tets,
                             int n_markers, const char* const* marker_names, const int* marker_types,
                             const int64_t* marker_offsets, const int64_t* marker_tris) {
  try {
    if (n_nodes <= 0 || n_cells <= 0 || !nodes || !tets || n_markers < 0 ||
        (n_markers && (!marker_names || !marker_types || !marker_offsets || !marker_tris)))
      throw nf::MeshError("invalid arguments");
    std::vector<double> nd(nodes, nodes + 3 * n_nodes);
    std::vector<int64_t> tt(tets, tets + 4 * n_cells);
    std::vector<nf::MarkerInput> mk(static_cast<size_t>(n_markers));
    for (int i = 0; i < n_markers; i++) {
      mk[size_t(i)].name = marker_names[i];
      mk[size_t(i)].type = marker_types[i];
      const int64_t b = marker_offsets[i], e = marker_offsets[i + 1];
      if (e < b) throw nf::MeshError("marker offsets must be non-decreasing");
      mk[size_t(i)].tris.assign(marker_tris + 3 * b, marker_tris + 3 * e);
    }
    return wrap_mesh(nf::build_mesh(nd, tt, mk));
  } catch (const std::exception& e) {
    g_create_error = std::string("Error creating grid:\n") + e.what();
    return nullptr;
  }
}

nf_mesh* nf_mesh_concat(int n, const nf_mesh* const* meshes) {
  try {
    if (n <= 0 || !meshes) throw nf::MeshError("invalid arguments");
    std::vector<const nf::Mesh*> parts;
    for (int i = 0; i < n; i++) {
      if (!meshes[i]) throw nf::MeshError("null mesh");
      parts.push_back(&meshes[i]->m);
    }
    return wrap_mesh(nf::concat_meshes(parts));
  } catch (const std::exception& e) {
    g_create_error = std::string("Error concatenating meshes: ") + e.what();
    return nullptr;
  }
}

int nf_mesh_get_info(const nf_mesh* h, nf_mesh_info* out) {
  if (!h || !out) return NF_ERR_ARG;
  const nf::Mesh& m = h->m;
  std::memset(out, 0, sizeof(*out));
  out->n_nodes = m.n_nodes;
  out->n_interior_cells = m.n_cells;
  out->n_ghost_cells = m.n_ghost();
  out->n_interior_faces = m.n_interior_faces;
  out->n_total_faces = m.n_faces;
  out->n_patches = int32_t(m.patches.size());
  out->max_faces_per_cell = 4;
  out->n_uncovered_boundary_faces = m.n_uncovered;
  out->n_cases = m.n_cases();
  return NF_OK;
}

int nf_mesh_get_patch(const nf_mesh* h, int p, int* type, int64_t* first_face, int64_t* n_faces, int* case_index,
                      char* name, size_t name_len) {
  if (!h || p < 0 || p >= int(h->m.patches.size())) return NF_ERR_ARG;
  const nf::Patch& P = h->m.patches[size_t(p)];
  if (type) *type = P.type;
  if (first_face) *first_face = P.first_face;
  if (n_faces) *n_faces = P.n_faces;
  if (case_index) *case_index = P.case_index;
  if (name && name_len) {
    std::strncpy(name, P.name.c_str(), name_len - 1);
    name[name_len - 1] = '\0';
  }
  return NF_OK;
}

int nf_mesh_export(const nf_mesh* h, uint32_t* face_ij, double* S, double* ri, double* rj, double* vol,
                   double* centroid, double* dS) {
  if (!h) return NF_ERR_ARG;
  const nf::Mesh& m = h->m;
  if (face_ij)
    for (int64_t f = 0; f < m.n_faces; f++) {
      face_ij[2 * f] = m.face_i[size_t(f)];
      face_ij[2 * f + 1] = m.face_j[size_t(f)];
    }
  if (S) std::memcpy(S, m.S.data(), m.S.size() * sizeof(double));
  if (ri) std::memcpy(ri, m.ri.data(), m.ri.size() * sizeof(double));
  if (rj) std::memcpy(rj, m.rj.data(), m.rj.size() * sizeof(double));
  if (vol) std::memcpy(vol, m.vol.data(), m.vol.size() * sizeof(double));
  if (centroid) std::memcpy(centroid, m.centroid.data(), m.centroid.size() * sizeof(double));
  if (dS) std::memcpy(dS, m.dS.data(), m.dS.size() * sizeof(double));
  return NF_OK;
}

int nf_mesh_get_permutation(const nf_mesh* h, int64_t* device_of_ref) {
  if (!h || !device_of_ref) return NF_ERR_ARG;
  std::memcpy(device_of_ref, h->m.dev_of_ref.data(), h->m.dev_of_ref.size() * sizeof(int64_t));
  return NF_OK;
}

int nf_mesh_get_case_offsets(const nf_mesh* h, int64_t* cell_offsets) {
  if (!h || !cell_offsets) return NF_ERR_ARG;
  std::memcpy(cell_offsets, h->m.case_offsets.data(), h->m.case_offsets.size() * sizeof(int64_t));
  return NF_OK;
}

void nf_mesh_destroy(nf_mesh* h) { delete h; }

// ---------------------------------------------------------------------------
// solver
// ---------------------------------------------------------------------------
void nf_params_default(nf_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->time_scheme = NF_TVD_RK3;
  p->spatial_order = NF_SECOND_ORDER;
  p->limiter = NF_LIMITER_BARTH;
  p->flux_scheme = NF_FLUX_RUSANOV;
  p->precision = NF_PREC_FP64;
  p->cfl = 0.8;
  p->device = -1;
  p->freestream[0] = 1.225;   // standard air (Utilities.hpp:100-107)
  p->freestream[4] = 101325.0;
}

nf_solver* nf_create(const nf_mesh* h, const nf_params* params) {
  if (!h || !params) {
    g_create_error = "nf_create: null mesh or params";
    return nullptr;
  }
  auto s = std::make_unique<nf_solver>();
  try {
    const nf::Mesh& m = h->m;
    const nf_params& p = *params;
    if (p.time_scheme != NF_EXPLICIT_EULER && p.time_scheme != NF_TVD_RK3) throw std::runtime_error("bad time_scheme");
    if (p.spatial_order != NF_FIRST_ORDER && p.spatial_order != NF_SECOND_ORDER)
      throw std::runtime_error("bad spatial_order");
    if (p.limiter != NF_LIMITER_NONE && p.limiter != NF_LIMITER_BARTH) throw std::runtime_error("bad limiter");
    if (p.flux_scheme != NF_FLUX_RUSANOV)
      throw std::runtime_error("only the Rusanov flux is implemented (the reference's HLLC is a stub)");
    if (p.precision < NF_PREC_FP64_REF || p.precision > NF_PREC_MIXED32) throw std::runtime_error("bad precision");
    if (p.patches && p.n_patches != int(m.patches.size()))
      throw std::runtime_error("params.n_patches does not match the mesh's patch count");
    s->p = p;
    s->p.patches = nullptr;  // copied below
    s->block = p.block_size > 0 ? p.block_size : 256;
    if (p.block_size > 0) {
      s->kgrad.block = s->kflux.block = std::min(p.block_size, 128);
      s->kgrad.variant = std::max(0, std::min(p.kernel_variant, s->grad_variants() - 1));
      s->kflux.variant = std::max(0, std::min(p.kernel_variant, s->flux_variants() - 1));
      s->tuned = true;  // a caller-fixed shape is not tuned
    }
    if (s->block % 32 || s->block > 256) throw std::runtime_error("block_size must be a multiple of 32, <= 256");
    if (p.device >= 0) ck(cudaSetDevice(p.device), "cudaSetDevice");
    ck(cudaGetDevice(&s->device), "cudaGetDevice");
    ck(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaStream_t st = s->stream;

    const int64_t N = m.n_cells, F = m.n_faces;
    if (nf_check_mesh_size(N, F) != NF_OK) throw std::runtime_error(g_create_error);
    s->n = int(N);
    s->stride = int((N + 63) / 64 * 64);
    s->n_faces = int(F);
    s->n_nodes = m.n_nodes;
    s->dev_of_ref = m.dev_of_ref;
    s->case_offsets = m.case_offsets;
    s->n_cases = m.n_cases();
    const int stride = s->stride;

    // device face order: by the first device cell that touches the face
    std::vector<int64_t> key(static_cast<size_t>(F));
    for (int64_t f = 0; f < F; f++) {
      const int64_t di = m.dev_of_ref[m.face_i[size_t(f)]];
      const bool interior = m.face_j[size_t(f)] < uint32_t(N);
      key[size_t(f)] = interior ? std::min(di, m.dev_of_ref[m.face_j[size_t(f)]]) : di;
    }
    std::vector<int64_t> dev_face_order(static_cast<size_t>(F));
    std::iota(dev_face_order.begin(), dev_face_order.end(), 0);
    std::stable_sort(dev_face_order.begin(), dev_face_order.end(),
                     [&](int64_t a, int64_t b) { return key[size_t(a)] < key[size_t(b)]; });
    std::vector<int64_t> fdev(static_cast<size_t>(F));
    for (int64_t k = 0; k < F; k++) fdev[size_t(dev_face_order[size_t(k)])] = k;

    std::vector<double> h_S(size_t(3 * F)), h_n(size_t(3 * F)), h_a(static_cast<size_t>(F));
    for (int64_t f = 0; f < F; f++) {
      const int64_t d = fdev[size_t(f)];
      h_a[size_t(d)] = m.area[size_t(f)];
      for (int c = 0; c < 3; c++) {
        h_S[size_t(c * F + d)] = m.S[size_t(3 * f + c)];
        h_n[size_t(c * F + d)] = m.nhat[size_t(3 * f + c)];
      }
    }
    // slots in reference face order; nbslot names the other side of each face
    std::vector<int> h_slot(size_t(4) * stride, -1), h_nb(size_t(4) * stride, 0);
    std::vector<double> h_rs(size_t(12) * stride, 0.0);  // [d][q][cell]
    struct BFace {
      int64_t cell;
      int q, face, patch;
    };
    std::vector<BFace> bfaces;
    std::vector<int> fill(static_cast<size_t>(stride), 0);
    auto add_slot = [&](int64_t cell_dev, int value) {
      int& k = fill[size_t(cell_dev)];
      if (k >= 4) throw std::runtime_error("a cell has more than 4 faces (only tetrahedra are supported)");
      h_slot[size_t(k) * stride + size_t(cell_dev)] = value;
      return k++;
    };
    for (int64_t f = 0; f < F; f++) {
      const int fd = int(fdev[size_t(f)]);
      const int64_t di = m.dev_of_ref[m.face_i[size_t(f)]];
      const int qi = add_slot(di, fd << 1);
      for (int c = 0; c < 3; c++) h_rs[(size_t(c) * 4 + qi) * stride + size_t(di)] = m.ri[size_t(3 * f + c)];
      const uint32_t j = m.face_j[size_t(f)];
      if (j < uint32_t(N)) {
        const int64_t dj = m.dev_of_ref[j];
        const int qj = add_slot(dj, (fd << 1) | 1);
        for (int c = 0; c < 3; c++) h_rs[(size_t(c) * 4 + qj) * stride + size_t(dj)] = m.rj[size_t(3 * f + c)];
        h_nb[size_t(qi) * stride + size_t(di)] = int(dj << 2) | qj;
        h_nb[size_t(qj) * stride + size_t(dj)] = int(di << 2) | qi;
      } else {
        bfaces.push_back({di, qi, fd, int(m.face_patch[size_t(f)])});
      }
    }
    // boundary faces in owner-cell order; the owner's slot names its index
    std::stable_sort(bfaces.begin(), bfaces.end(), [](const BFace& x, const BFace& y) { return x.cell < y.cell; });
    const int nbf = int(bfaces.size());
    std::vector<int> hb_cell(static_cast<size_t>(nbf)), hb_slot(static_cast<size_t>(nbf)), hb_face(static_cast<size_t>(nbf)), hb_patch(static_cast<size_t>(nbf));
    for (int b = 0; b < nbf; b++) {
      hb_cell[size_t(b)] = int(bfaces[size_t(b)].cell);
      hb_slot[size_t(b)] = bfaces[size_t(b)].q;
      hb_face[size_t(b)] = bfaces[size_t(b)].face;
      hb_patch[size_t(b)] = bfaces[size_t(b)].patch;
      h_nb[size_t(bfaces[size_t(b)].q) * stride + size_t(bfaces[size_t(b)].cell)] = -(1 + b);
    }
    // node-based layout of the fast forms: a cell's vertices sorted by node
    // id; face m is the face opposite vertex m
    const bool fast = p.precision != NF_PREC_FP64_REF;
    std::vector<int> h_cnode, h_gcode, h_nbvf, h_nbsf, hb_slotf;
    if (fast) {
      h_cnode.assign(size_t(4) * stride, 0);
      h_gcode.assign(size_t(stride), 0);
      h_nbvf.assign(size_t(4) * stride, 0);
      h_nbsf.assign(size_t(4) * stride, 0);
      for (int64_t c = 0; c < stride; c++)
        for (int q = 0; q < 4; q++) h_nbvf[size_t(q) * stride + size_t(c)] = int(std::min<int64_t>(c, N - 1));
      std::vector<uint32_t> sorted(size_t(4) * N);
      for (int64_t c = 0; c < N; c++) {
        uint32_t v[4] = {m.tet[size_t(4 * c)], m.tet[size_t(4 * c + 1)], m.tet[size_t(4 * c + 2)],
                         m.tet[size_t(4 * c + 3)]};
        std::sort(v, v + 4);
        const int64_t d = m.dev_of_ref[size_t(c)];
        for (int q = 0; q < 4; q++) {
          sorted[size_t(4 * c + q)] = v[q];
          h_cnode[size_t(q) * stride + size_t(d)] = int(v[q]);
        }
      }
      auto P = [&](uint32_t id, int e) { return m.nodes[size_t(3) * id + size_t(e)]; };
      // index of the vertex of ref cell c that face f does not contain, and
      // whether the normal from the ascending triple points into the cell
      auto face_of = [&](int64_t c, int64_t f, int* mface, bool* inward) {
        const uint32_t* fn = &m.face_nodes[size_t(3 * f)];
        int om = -1;
        for (int q = 0; q < 4; q++) {
          const uint32_t v = sorted[size_t(4 * c + q)];
          if (v != fn[0] && v != fn[1] && v != fn[2]) om = q;
        }
        if (om < 0) throw std::runtime_error("face nodes do not match its cell");
        uint32_t t[3];
        int k = 0;
        for (int q = 0; q < 4; q++)
          if (q != om) t[k++] = sorted[size_t(4 * c + q)];
        double e1[3], e2[3], S[3], cen[3], fc[3];
        for (int e = 0; e < 3; e++) {
          e1[e] = P(t[1], e) - P(t[0], e);
          e2[e] = P(t[2], e) - P(t[0], e);
          fc[e] = (P(t[0], e) + P(t[1], e) + P(t[2], e)) / 3.0;
          cen[e] = 0.25 * (P(sorted[size_t(4 * c)], e) + P(sorted[size_t(4 * c + 1)], e) +
                           P(sorted[size_t(4 * c + 2)], e) + P(sorted[size_t(4 * c + 3)], e));
        }
        S[0] = e1[1] * e2[2] - e1[2] * e2[1];
        S[1] = e1[2] * e2[0] - e1[0] * e2[2];
        S[2] = e1[0] * e2[1] - e1[1] * e2[0];
        const double dd = S[0] * (fc[0] - cen[0]) + S[1] * (fc[1] - cen[1]) + S[2] * (fc[2] - cen[2]);
        *mface = om;
        *inward = dd < 0.0;
      };
      hb_slotf.assign(size_t(nbf), 0);
      std::vector<int> bindex(static_cast<size_t>(F), -1);  // boundary index of a device face
      for (int b = 0; b < nbf; b++) bindex[size_t(bfaces[size_t(b)].face)] = b;
      for (int64_t f = 0; f < F; f++) {
        const int64_t ci = m.face_i[size_t(f)];
        const int64_t di = m.dev_of_ref[size_t(ci)];
        int mi;
        bool ini;
        face_of(ci, f, &mi, &ini);
        int& gi = h_gcode[size_t(di)];
        gi |= (1 | (ini ? 2 : 0)) << (3 * mi);  // owner side: bit 2 clear
        const uint32_t j = m.face_j[size_t(f)];
        if (j < uint32_t(N)) {
          const int64_t dj = m.dev_of_ref[j];
          int mj;
          bool inj;
          face_of(j, f, &mj, &inj);
          h_gcode[size_t(dj)] |= (1 | (inj ? 2 : 0) | 4) << (3 * mj);
          h_nbvf[size_t(mi) * stride + size_t(di)] = int(dj);
          h_nbvf[size_t(mj) * stride + size_t(dj)] = int(di);
          h_nbsf[size_t(mi) * stride + size_t(di)] = int(dj << 2) | mj;
          h_nbsf[size_t(mj) * stride + size_t(dj)] = int(di << 2) | mi;
        } else {
          const int b = bindex[size_t(fdev[size_t(f)])];
          h_nbvf[size_t(mi) * stride + size_t(di)] = -(1 + b);
          h_nbsf[size_t(mi) * stride + size_t(di)] = -(1 + b);
          hb_slotf[size_t(b)] = mi;
        }
      }
    }
    s->nb = nbf;
    s->bstride = std::max(64, (nbf + 63) / 64 * 64);
    std::vector<double> h_vol(size_t(stride), 1.0), h_dS(size_t(3) * stride, 0.0);
    for (int64_t c = 0; c < N; c++) {
      const int64_t d = m.dev_of_ref[size_t(c)];
      h_vol[size_t(d)] = m.vol[size_t(c)];
      for (int k = 0; k < 3; k++) h_dS[size_t(k) * stride + size_t(d)] = m.dS[size_t(3 * c + k)];
    }
    // boundary conditions per patch
    std::vector<nf::PatchBC> h_pb(m.patches.size());
    for (size_t q = 0; q < m.patches.size(); q++) {
      nf::PatchBC& b = h_pb[q];
      b.type = params->patches ? params->patches[q].type : m.patches[q].type;
      b.case_index = m.patches[q].case_index;
      const double* fs = params->patches ? params->patches[q].farfield : p.freestream;
      for (int k = 0; k < 5; k++) b.fs[k] = fs[k];
      // BC_FarField::BC_FarField (Numerics.cpp:76-84)
      b.c_fs = std::sqrt(nf::Gas<double>::gamma * fs[4] / fs[0]);
      b.s_fs = fs[4] * std::pow(fs[0], -nf::Gas<double>::gamma);
      b.density_fix = p.farfield_density_fix ? 1 : 0;
      b.pad = 0;
      if (b.type < 0 || b.type > 2) throw std::runtime_error("bad boundary type");
    }

    s->slot.upload(h_slot, st);
    s->nbslot.upload(h_nb, st);
    s->b_cell.upload(hb_cell, st);
    s->b_slot.upload(hb_slot, st);
    s->b_face.upload(hb_face, st);
    s->b_patch.upload(hb_patch, st);
    s->rs.upload(h_rs, st);
    if (fast) {
      s->gcode.upload(h_gcode, st);
      s->b_slotf.upload(hb_slotf, st);
      s->cnode.upload(h_cnode, st);
      s->nbvf.upload(h_nbvf, st);
      s->nbsf.upload(h_nbsf, st);
      std::vector<double> n4(size_t(4) * m.n_nodes, 0.0);
      for (int64_t v = 0; v < m.n_nodes; v++)
        for (int e = 0; e < 3; e++) n4[size_t(4 * v + e)] = m.nodes[size_t(3 * v + e)];
      s->nodes4.upload(n4, st);
      if (p.precision == NF_PREC_MIXED || p.precision == NF_PREC_MIXED32) {
        std::vector<float> n4f(n4.size());
        for (size_t i = 0; i < n4.size(); i++) n4f[i] = float(n4[i]);
        s->nodes4_32.upload(n4f, st);
      }
    }
    s->S.upload(h_S, st);
    s->nhat.upload(h_n, st);
    s->area.upload(h_a, st);
    s->vol.upload(h_vol, st);
    s->dS.upload(h_dS, st);
    s->patches.upload(h_pb, st);
    const bool fp32_fields = p.precision == NF_PREC_MIXED || p.precision == NF_PREC_MIXED32;
    if (p.precision == NF_PREC_MIXED32) {
      s->V32a.alloc(size_t(5) * stride);
      s->V32b.alloc(size_t(5) * stride);
      s->vg32.alloc(size_t(5) * s->bstride);
      s->vg32.zero(st);
    }
    if (fp32_fields) {
      s->fb32.alloc(size_t(5) * s->bstride);
      s->fb32.zero(st);
      s->fs32.alloc(size_t(20) * stride);
      s->fs32.zero(st);
      if (p.keep_stage_fields) {
        s->grad32.alloc(size_t(15) * stride);
        s->phi32.alloc(size_t(5) * stride);
        s->grad32.zero(st);
        s->phi32.zero(st);
      }
    }
    s->U.alloc(size_t(5) * stride);
    s->W.alloc(size_t(5) * stride);
    s->V0.alloc(size_t(5) * stride);
    s->V1.alloc(size_t(5) * stride);
    s->vg.alloc(size_t(5) * s->bstride);  // FP64 ghosts in every form
    s->vg.zero(st);
    if (!fp32_fields) {
      s->fs.alloc(size_t(20) * stride);
      s->fs.zero(st);
      s->fb.alloc(size_t(5) * s->bstride);
      s->fb.zero(st);
    }
    if (p.keep_stage_fields) {
      s->R.alloc(size_t(5) * stride);
      s->R.zero(st);
      if (!fp32_fields) {
        s->grad.alloc(size_t(15) * stride);
        s->phi.alloc(size_t(5) * stride);
        s->grad.zero(st);
        s->phi.zero(st);
      }
    }
    s->dt_local.alloc(static_cast<size_t>(stride));
    s->dt_local2.alloc(static_cast<size_t>(stride));
    s->dt_local2.zero(st);
    s->res_cell.alloc(static_cast<size_t>(stride));
    s->scal.alloc(nf::kScalCount);
    s->status.alloc(1);
    for (auto* b : {&s->U, &s->W, &s->V0, &s->V1, &s->dt_local, &s->res_cell, &s->scal})
      b->zero(st);
    s->status.zero(st);
    // residual chunks: fixed-size pieces of each case's cell range
    std::vector<long long> cb, ce, cc;
    std::vector<int> c0{0};
    const long long chunk = 16384;
    for (int cs = 0; cs < s->n_cases; cs++) {
      const long long b0 = m.case_offsets[size_t(cs)], e0 = m.case_offsets[size_t(cs + 1)];
      for (long long b = b0; b < e0; b += chunk) {
        cb.push_back(b);
        ce.push_back(std::min(e0, b + chunk));
      }
      if (e0 == b0) {
        cb.push_back(b0);
        ce.push_back(b0);
      }
      c0.push_back(int(cb.size()));
      cc.push_back(e0 - b0);
    }
    s->n_chunks = int(cb.size());
    s->chunk_begin.upload(cb, st);
    s->chunk_end.upload(ce, st);
    s->case_cells.upload(cc, st);
    s->case_chunk0.upload(c0, st);
    s->part.alloc(size_t(2) * s->n_chunks);
    {
      std::vector<int> cc2(static_cast<size_t>(stride), 0);
      for (int cs = 0; cs < s->n_cases; cs++)
        for (int64_t c = m.case_offsets[size_t(cs)]; c < m.case_offsets[size_t(cs + 1)]; c++) cc2[size_t(c)] = cs;
      s->cell_case.upload(cc2, st);
      s->case_frozen.alloc(size_t(s->n_cases));
      s->case_frozen.zero(st);
    }
    if (p.spatial_order == NF_SECOND_ORDER && p.limiter == NF_LIMITER_BARTH &&
        (p.limiter_ratchet_step > 0 || p.limiter_ratchet_drop > 0.0)) {
      s->ratchet_alloc = true;
      s->case_ratchet.alloc(size_t(s->n_cases));
      s->h_ratchet.assign(size_t(s->n_cases), 0);
      if (p.precision == NF_PREC_MIXED || p.precision == NF_PREC_MIXED32) s->phi_keep32.alloc(size_t(5) * stride);
      else s->phi_keep.alloc(size_t(5) * stride);
      s->ratchet_reset();
    }
    s->stage.alloc(size_t(5) * N);
    {
      std::vector<long long> dor(m.dev_of_ref.begin(), m.dev_of_ref.end());
      s->d_dev_of_ref.upload(dor, st);
    }
    s->res_out.alloc(size_t(2) * s->n_cases);
    ck(cudaMallocHost(&s->h_scal, nf::kScalCount * sizeof(double)), "cudaMallocHost");
    ck(cudaHostAlloc(&s->h_rep_status, sizeof(unsigned), cudaHostAllocMapped), "cudaHostAlloc");
    ck(cudaHostAlloc(&s->h_rep_scal, nf::kScalCount * sizeof(double), cudaHostAllocMapped), "cudaHostAlloc");
    ck(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_rep_status), s->h_rep_status, 0),
       "cudaHostGetDevicePointer");
    ck(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->d_rep_scal), s->h_rep_scal, 0),
       "cudaHostGetDevicePointer");
    std::fill(s->h_scal, s->h_scal + nf::kScalCount, 0.0);
    s->h_scal[nf::kScalTEnd] = p.t_end;
    ck(cudaMemcpyAsync(s->scal.p, s->h_scal, nf::kScalCount * sizeof(double), cudaMemcpyHostToDevice, st),
       "scal H2D");
    ck(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    ck(cudaGetLastError(), "nf_create");
  } catch (const std::exception& e) {
    g_create_error = std::string("nf_create: ") + e.what();
    return nullptr;
  }
  return s.release();
}

int nf_set_state(nf_solver* s, const double* U, int64_t n_cells) {
  return guarded(s, [&]() -> int {
    if (!U || n_cells != s->n) {
      s->err = "nf_set_state: state size does not match the mesh";
      return NF_ERR_ARG;
    }
    // one copy of the caller's AoS array, then a permutation kernel into SoA
    ck(cudaMemcpyAsync(s->stage.p, U, size_t(5) * s->n * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "U H2D");
    s->adopt_state(s->stage.p);
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    ck(cudaGetLastError(), "nf_set_state");
    return NF_OK;
  });
}

int nf_set_state_old(nf_solver* s, const double* U_old, int64_t n_cells) {
  return guarded(s, [&]() -> int {
    if (!U_old || n_cells != s->n) {
      s->err = "nf_set_state_old: state size does not match the mesh";
      return NF_ERR_ARG;
    }
    if (!s->Uold.p) s->Uold.alloc(size_t(5) * s->stride);
    ck(cudaMemcpyAsync(s->stage.p, U_old, size_t(5) * s->n * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "U_old H2D");
    scatter_state_kernel<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->stride, s->d_dev_of_ref.p, s->stage.p,
                                                                   s->Uold.p);
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    ck(cudaGetLastError(), "nf_set_state_old");
    s->old_pending = true;
    return NF_OK;
  });
}

int nf_get_state(nf_solver* s, double* U, int64_t n_cells) {
  return guarded(s, [&]() -> int {
    if (!U || n_cells != s->n) {
      s->err = "nf_get_state: state size does not match the mesh";
      return NF_ERR_ARG;
    }
    gather_state_kernel<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->stride, s->d_dev_of_ref.p, s->U.p,
                                                                   s->stage.p);
    ck(cudaMemcpyAsync(U, s->stage.p, size_t(5) * s->n * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
       "U D2H");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    return s->check_status();
  });
}

int nf_snapshot_begin(nf_solver* s, double* U, int64_t n_cells) {
  return guarded(s, [&]() -> int {
    if (!U || n_cells != s->n) {
      s->err = "nf_snapshot_begin: state size does not match the mesh";
      return NF_ERR_ARG;
    }
    if (!s->snap_stream) {
      ck(cudaStreamCreateWithFlags(&s->snap_stream, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&s->snap_ready, cudaEventDisableTiming), "cudaEventCreate");
      for (auto& e : s->snap_done) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    }
    const int k = s->snap_k;
    if (s->snap[k].n != size_t(5) * s->n) s->snap[k].alloc(size_t(5) * s->n);
    // the copy out of this staging buffer two snapshots back must be done
    // before the gather overwrites it (a device-side wait, usually long met)
    if (s->snap_used[k]) ck(cudaStreamWaitEvent(s->stream, s->snap_done[k], 0), "cudaStreamWaitEvent");
    // the gather is ordered after the queued steps and before the later ones
    gather_state_kernel<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->n, s->stride, s->d_dev_of_ref.p, s->U.p,
                                                                   s->snap[k].p);
    ck(cudaGetLastError(), "snapshot gather");
    ck(cudaEventRecord(s->snap_ready, s->stream), "cudaEventRecord");
    ck(cudaStreamWaitEvent(s->snap_stream, s->snap_ready, 0), "cudaStreamWaitEvent");
    ck(cudaMemcpyAsync(U, s->snap[k].p, size_t(5) * s->n * sizeof(double), cudaMemcpyDeviceToHost,
                       s->snap_stream),
       "snapshot D2H");
    ck(cudaEventRecord(s->snap_done[k], s->snap_stream), "cudaEventRecord");
    s->snap_used[k] = true;
    s->snap_k = 1 - k;
    s->snap_pending = true;
    return NF_OK;
  });
}

int nf_snapshot_wait(nf_solver* s) {
  return guarded(s, [&]() -> int {
    if (!s->snap_pending) return NF_OK;
    // the copies run in order on one stream: the last one done means all are
    ck(cudaStreamSynchronize(s->snap_stream), "snapshot wait");
    s->snap_pending = false;
    return NF_OK;
  });
}

int nf_upload_begin(nf_solver* s, const double* U, int64_t n_cells) {
  return guarded(s, [&]() -> int {
    if (!U || n_cells != s->n) {
      s->err = "nf_upload_begin: state size does not match the mesh";
      return NF_ERR_ARG;
    }
    if (s->up_pending) {
      s->err = "nf_upload_begin: an upload is already in flight (commit it first)";
      return NF_ERR_ARG;
    }
    if (!s->up_stream) {
      ck(cudaStreamCreateWithFlags(&s->up_stream, cudaStreamNonBlocking), "cudaStreamCreate");
      for (int k = 0; k < 2; k++) {
        ck(cudaEventCreateWithFlags(&s->up_done[k], cudaEventDisableTiming), "cudaEventCreate");
        ck(cudaEventCreateWithFlags(&s->up_free[k], cudaEventDisableTiming), "cudaEventCreate");
      }
    }
    const int k = s->up_k;
    if (s->up[k].n != size_t(5) * s->n) s->up[k].alloc(size_t(5) * s->n);
    // the scatter of this staging buffer's previous state may still be reading it
    if (s->up_used[k]) ck(cudaStreamWaitEvent(s->up_stream, s->up_free[k], 0), "cudaStreamWaitEvent");
    ck(cudaMemcpyAsync(s->up[k].p, U, size_t(5) * s->n * sizeof(double), cudaMemcpyHostToDevice, s->up_stream),
       "upload H2D");
    ck(cudaEventRecord(s->up_done[k], s->up_stream), "cudaEventRecord");
    s->up_cur = k;
    s->up_k = 1 - k;
    s->up_pending = true;
    return NF_OK;
  });
}

int nf_upload_commit(nf_solver* s) {
  return guarded(s, [&]() -> int {
    if (!s->up_pending) {
      s->err = "nf_upload_commit: no upload in flight";
      return NF_ERR_ARG;
    }
    // the solver stream takes the state once the copy has landed; work
    // queued before this call runs first and is not affected
    const int k = s->up_cur;
    ck(cudaStreamWaitEvent(s->stream, s->up_done[k], 0), "cudaStreamWaitEvent");
    s->adopt_state(s->up[k].p);
    ck(cudaGetLastError(), "nf_upload_commit");
    ck(cudaEventRecord(s->up_free[k], s->stream), "cudaEventRecord");
    s->up_used[k] = true;
    s->up_pending = false;
    s->up_reading = true;  // until nf_upload_wait: the copy may still read the caller's buffer
    return NF_OK;
  });
}

int nf_upload_wait(nf_solver* s) {
  return guarded(s, [&]() -> int {
    if ((s->up_pending || s->up_reading) && s->up_stream) ck(cudaStreamSynchronize(s->up_stream), "upload wait");
    s->up_reading = false;
    return NF_OK;
  });
}

int nf_calc_timestep(nf_solver* s, double* dt_out) {
  return guarded(s, [&]() -> int {
    s->enqueue_dt();
    ck(cudaGetLastError(), "timestep launch");
    int rc = s->check_status();  // also brings the scalars into h_rep_scal
    const double dt = s->h_rep_scal[nf::kScalDtMin];
    if (dt_out) *dt_out = dt;
    if (rc == NF_OK && !(std::isfinite(dt) && dt > 0.0)) rc = NF_ERR_DT;
    if (rc == NF_ERR_DT) {
      char buf[96];
      std::snprintf(buf, sizeof(buf), "Invalid dt calculated (dt = %f)", dt);
      s->err = buf;
    }
    return rc;
  });
}

int nf_set_timestep(nf_solver* s, double dt) {
  return guarded(s, [&]() -> int {
    if (!(dt > 0.0) || !std::isfinite(dt)) {
      s->err = "nf_set_timestep: dt must be positive and finite";
      return NF_ERR_ARG;
    }
    s->h_scal[nf::kScalCount - 1] = dt;
    ck(cudaMemcpyAsync(s->scal.p + nf::kScalDtMin, s->h_scal + nf::kScalCount - 1, sizeof(double),
                       cudaMemcpyHostToDevice, s->stream),
       "dt H2D");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    return NF_OK;
  });
}

int nf_step(nf_solver* s) {
  return guarded(s, [&]() -> int {
    if (s->stage_next != 0) {
      s->err = "nf_step: a step begun with nf_stage is not finished";
      return NF_ERR_ARG;
    }
    s->ratchet_due(1);
    s->enqueue_step();
    s->steps_done++;
    ck(cudaGetLastError(), "step launch");
    return NF_OK;
  });
}

int nf_stage(nf_solver* s, int stage) {
  return guarded(s, [&]() -> int {
    if (stage != s->stage_next) {
      s->err = "nf_stage: stage " + std::to_string(stage) + " out of order (next is " +
               std::to_string(s->stage_next) + ")";
      return NF_ERR_ARG;
    }
    if (stage == 0) s->ratchet_due(1);
    s->enqueue_stage(stage);
    s->stage_next = (stage + 1) % s->n_stages();
    if (s->stage_next == 0) s->steps_done++;
    ck(cudaGetLastError(), "stage launch");
    return NF_OK;
  });
}

static int halo_args(nf_solver* s, const int64_t* cells, int64_t n, const double* buf, const char* what) {
  if (n < 0 || (n > 0 && (!cells || !buf))) {
    s->err = std::string(what) + ": null pointer or negative count";
    return NF_ERR_ARG;
  }
  if (s->p.precision == NF_PREC_MIXED32) {
    s->err = std::string(what) + ": the mixed form with FP32 copies keeps its stage primitives in FP32 only";
    return NF_ERR_UNSUPPORTED;
  }
  return NF_OK;
}

int nf_halo_pack(nf_solver* s, const int64_t* cells, int64_t n, double* buf) {
  return guarded(s, [&]() -> int {
    int rc = halo_args(s, cells, n, buf, "nf_halo_pack");
    if (rc != NF_OK || n == 0) return rc;
    halo_pack_kernel<<<int((n + 255) / 256), 256, 0, s->stream>>>(n, s->stride, cells, s->Vbuf(s->vcur),
                                                                   s->stage_input(s->stage_next), buf);
    ck(cudaGetLastError(), "halo pack");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    return NF_OK;
  });
}

int nf_halo_unpack(nf_solver* s, const int64_t* cells, int64_t n, const double* buf) {
  return guarded(s, [&]() -> int {
    int rc = halo_args(s, cells, n, buf, "nf_halo_unpack");
    if (rc != NF_OK || n == 0) return rc;
    halo_unpack_kernel<<<int((n + 255) / 256), 256, 0, s->stream>>>(n, s->stride, cells, buf, s->Vbuf(s->vcur),
                                                                     s->stage_input(s->stage_next));
    ck(cudaGetLastError(), "halo unpack");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    return NF_OK;
  });
}

int nf_advance(nf_solver* s, int64_t n_steps, double* time_out) {
  return guarded(s, [&]() -> int {
    if (n_steps < 0) return NF_ERR_ARG;
    if (s->stage_next != 0) {
      s->err = "nf_advance: a step begun with nf_stage is not finished";
      return NF_ERR_ARG;
    }
    s->run_steps(n_steps);
    ck(cudaGetLastError(), "advance launch");
    int rc = s->check_status();
    if (time_out) *time_out = s->h_rep_scal[nf::kScalTime];
    return rc;
  });
}

static void enqueue_residual(nf_solver* s) {
  residual_partials_kernel<<<s->n_chunks, 256, 0, s->stream>>>(s->res_cell.p, s->chunk_begin.p, s->chunk_end.p,
                                                               s->part.p);
  residual_finalize_kernel<<<(s->n_cases + 127) / 128, 128, 0, s->stream>>>(s->part.p, s->case_chunk0.p,
                                                                          s->case_cells.p, s->n_cases,
                                                                          s->res_out.p);
}

namespace {

// tol > 0: relative to each case's first residual; else abs_target[case].
int solve_steady_impl(nf_solver* s, double tol, const double* abs_target, int64_t max_steps, int check_every,
                      int64_t* steps_per_case, double* res0_per_case, double* res_per_case, double* ms_per_case) {
  return guarded(s, [&]() -> int {
    if (!s->p.local_time_stepping) {
      s->err = "nf_solve_steady needs local time stepping";
      return NF_ERR_ARG;
    }
    if (!(tol > 0.0) && !abs_target) return NF_ERR_ARG;
    if (max_steps < 1 || check_every < 1) return NF_ERR_ARG;
    const int nc = s->n_cases;
    std::vector<int> frozen(size_t(nc), 0);
    std::vector<int64_t> steps(size_t(nc), -1);
    std::vector<double> r0(size_t(nc), 0.0), rl(size_t(nc), 0.0), ms(size_t(nc), 0.0), h(size_t(2) * nc);
    // Graphs bake the freeze argument into their launches, so they are dropped
    // when it is switched on and again when it is switched off; the guard
    // restores the unfrozen solver on every exit, error paths included.
    auto drop_graphs = [s]() {
      for (auto& g : s->graph)
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    struct Restore {
      nf_solver* s;
      int nc;
      cudaEvent_t *e0, *e1;
      std::function<void()> drop;
      ~Restore() {
        if (*e0) cudaEventDestroy(*e0);
        if (*e1) cudaEventDestroy(*e1);
        s->freeze = false;
        drop();
        cudaMemsetAsync(s->case_frozen.p, 0, size_t(nc) * sizeof(int), s->stream);
        // frozen cells were skipped: both primitive buffers from U again
        s->refresh_primitives();
      }
    } restore{s, nc, &e0, &e1, drop_graphs};
    ck(cudaMemsetAsync(s->case_frozen.p, 0, size_t(nc) * sizeof(int), s->stream), "freeze reset");
    s->freeze = true;
    drop_graphs();
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    ck(cudaEventRecord(e0, s->stream), "cudaEventRecord");
    auto read_res = [&]() {
      enqueue_residual(s);
      ck(cudaMemcpyAsync(h.data(), s->res_out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
         "residual D2H");
      ck(cudaEventRecord(e1, s->stream), "cudaEventRecord");
      ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
    };
    // first step: the reference residual of every case
    s->run_steps(1);
    read_res();
    int64_t done = 1, left = nc;
    std::vector<double> target(size_t(nc), 0.0);
    for (int cs = 0; cs < nc; cs++) {
      r0[size_t(cs)] = h[size_t(2 * cs)];
      rl[size_t(cs)] = r0[size_t(cs)];
      target[size_t(cs)] = abs_target ? abs_target[cs] : tol * r0[size_t(cs)];
      if (!(r0[size_t(cs)] > 0.0) || r0[size_t(cs)] <= target[size_t(cs)]) {  // already steady
        steps[size_t(cs)] = 1;
        frozen[size_t(cs)] = 1;
        left--;
      }
    }
    while (left > 0 && done < max_steps) {
      const int64_t k = std::min<int64_t>(check_every, max_steps - done);
      ck(cudaMemcpyAsync(s->case_frozen.p, frozen.data(), size_t(nc) * sizeof(int), cudaMemcpyHostToDevice,
                         s->stream),
         "freeze H2D");
      s->run_steps(k);
      done += k;
      read_res();
      float t = 0.f;
      ck(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
      for (int cs = 0; cs < nc; cs++) {
        if (frozen[size_t(cs)]) continue;
        rl[size_t(cs)] = h[size_t(2 * cs)];
        if (!std::isfinite(rl[size_t(cs)])) {
          s->err = "residual is not finite";
          return NF_ERR_NONPHYSICAL;
        }
        if (s->ratchet_alloc && s->p.limiter_ratchet_drop > 0.0 && !s->h_ratchet[size_t(cs)] &&
            rl[size_t(cs)] <= s->p.limiter_ratchet_drop * r0[size_t(cs)])
          s->ratchet_start(cs);
        if (rl[size_t(cs)] <= target[size_t(cs)]) {
          frozen[size_t(cs)] = 1;
          steps[size_t(cs)] = done;
          ms[size_t(cs)] = t;
          left--;
        }
      }
    }
    float t = 0.f;
    ck(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
    for (int cs = 0; cs < nc; cs++)
      if (steps[size_t(cs)] < 0) ms[size_t(cs)] = t;  // not converged: report the time spent
    for (int cs = 0; cs < nc; cs++) {
      if (steps_per_case) steps_per_case[cs] = steps[size_t(cs)] < 0 ? -done : steps[size_t(cs)];
      if (res0_per_case) res0_per_case[cs] = r0[size_t(cs)];
      if (res_per_case) res_per_case[cs] = rl[size_t(cs)];
      if (ms_per_case) ms_per_case[cs] = ms[size_t(cs)];
    }
    return s->check_status();
  });
}

}  // namespace

int nf_solve_steady(nf_solver* s, double tol, int64_t max_steps, int check_every, int64_t* steps_per_case,
                    double* res0_per_case, double* res_per_case, double* ms_per_case) {
  if (!(tol > 0.0)) return NF_ERR_ARG;
  return solve_steady_impl(s, tol, nullptr, max_steps, check_every, steps_per_case, res0_per_case, res_per_case,
                           ms_per_case);
}

int nf_solve_steady_to(nf_solver* s, const double* res_target, int64_t max_steps, int check_every,
                       int64_t* steps_per_case, double* res0_per_case, double* res_per_case, double* ms_per_case) {
  if (!res_target) return NF_ERR_ARG;
  return solve_steady_impl(s, 0.0, res_target, max_steps, check_every, steps_per_case, res0_per_case, res_per_case,
                           ms_per_case);
}

int nf_get_residual(nf_solver* s, double* out, int n_cases) {
  return guarded(s, [&]() -> int {
    if (!out || n_cases != s->n_cases) {
      s->err = "nf_get_residual: n_cases does not match the mesh";
      return NF_ERR_ARG;
    }
    enqueue_residual(s);
    ck(cudaGetLastError(), "residual launch");
    std::vector<double> h(size_t(2) * s->n_cases);
    ck(cudaMemcpyAsync(h.data(), s->res_out.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
       "residual D2H");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    std::copy(h.begin(), h.end(), out);
    return NF_OK;
  });
}

int nf_get_field(nf_solver* s, int which, double* out, int64_t n_values) {
  return guarded(s, [&]() -> int {
    const int st = s->stride;
    const double* src = nullptr;
    int comps = 5;
    switch (which) {
      case NF_FIELD_SOLUTION: src = s->U.p; break;
      case NF_FIELD_PRIMVARS: src = s->Vbuf(s->stepped ? 1 - s->vcur : s->vcur); break;
      case NF_FIELD_GRADIENT: src = s->grad.p; comps = 15; break;
      case NF_FIELD_LIMITER: src = s->phi.p; break;
      case NF_FIELD_FLUX_BALANCE: src = s->R.p; break;
      case NF_FIELD_LOCAL_DT: src = s->dtl(s->dtl_cur); comps = 1; break;
      default: s->err = "nf_get_field: unknown field"; return NF_ERR_ARG;
    }
    if (!src) {
      s->err = "nf_get_field: field not kept (set keep_stage_fields)";
      return NF_ERR_ARG;
    }
    if (!out || n_values != int64_t(comps) * s->n) {
      s->err = "nf_get_field: output size does not match";
      return NF_ERR_ARG;
    }
    std::vector<double> h(size_t(comps) * st);
    const bool m32_prim = s->p.precision == NF_PREC_MIXED32 && which == NF_FIELD_PRIMVARS && s->stepped;
    if (((s->p.precision == NF_PREC_MIXED || s->p.precision == NF_PREC_MIXED32) &&
         (which == NF_FIELD_GRADIENT || which == NF_FIELD_LIMITER)) ||
        m32_prim) {
      if (!m32_prim && !s->grad32.p) {
        s->err = "nf_get_field: field not kept (set keep_stage_fields)";
        return NF_ERR_ARG;
      }
      // the mixed form with FP32 copies keeps the stage primitives in FP32
      std::vector<float> hf(size_t(comps) * st);
      const float* src32 = m32_prim ? s->V32buf(1 - s->vcur) : which == NF_FIELD_GRADIENT ? s->grad32.p : s->phi32.p;
      ck(cudaMemcpyAsync(hf.data(), src32, hf.size() * sizeof(float), cudaMemcpyDeviceToHost, s->stream), "D2H");
      ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
      for (size_t i = 0; i < hf.size(); i++) h[i] = hf[i];
    } else {
      ck(cudaMemcpyAsync(h.data(), src, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "D2H");
      ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    }
    for (int64_t c = 0; c < s->n; c++) {
      const int64_t d = s->dev_of_ref[size_t(c)];
      if (which == NF_FIELD_GRADIENT) {
        // reference layout: Eigen column-major 5x3, entry (k, dim) at 5*dim + k
        for (int k = 0; k < 5; k++)
          for (int dm = 0; dm < 3; dm++) out[15 * c + 5 * dm + k] = h[size_t(k * 3 + dm) * st + size_t(d)];
      } else {
        for (int k = 0; k < comps; k++) out[comps * c + k] = h[size_t(k) * st + size_t(d)];
      }
    }
    return NF_OK;
  });
}

int nf_time_steps(nf_solver* s, int64_t n_steps, int per_kernel, double* ms_total, double* kernel_ms,
                  int64_t* kernel_launches) {
  return guarded(s, [&]() -> int {
    if (n_steps <= 0 || !ms_total) return NF_ERR_ARG;
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
    if (per_kernel) {
      s->prof_on = true;
      s->prof_used = 0;
    }
    ck(cudaEventRecord(e0, s->stream), "cudaEventRecord");
    int64_t left = n_steps;
    if (!per_kernel && left >= 2 && s->stepped) {
      const int v0 = s->vcur;
      if (!s->graph[v0]) {
        cudaGraph_t g = nullptr;
        ck(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        for (int k = 0; k < 2; k++) {
          s->enqueue_dt();
          s->enqueue_step();
        }
        ck(cudaStreamEndCapture(s->stream, &g), "end capture");
        ck(cudaGraphInstantiate(&s->graph[v0], g, 0), "graph instantiate");
        cudaGraphDestroy(g);
        s->vcur = v0;
        // instantiation happened inside the timed region: upload the graph
        // (which a first launch would otherwise do while the stream waits),
        // then restart the clock
        ck(cudaGraphUpload(s->graph[v0], s->stream), "graph upload");
        ck(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
        ck(cudaEventRecord(e0, s->stream), "cudaEventRecord");
      }
      while (left >= 2) {
        ck(cudaGraphLaunch(s->graph[v0], s->stream), "graph launch");
        left -= 2;
      }
    }
    while (left > 0) {
      s->enqueue_dt();
      s->enqueue_step();
      left--;
    }
    s->steps_done += n_steps;  // timing runs count as steps but do not start the ratchet
    ck(cudaEventRecord(e1, s->stream), "cudaEventRecord");
    ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    *ms_total = ms;
    if (per_kernel) {
      s->prof_on = false;
      if (kernel_ms)
        for (int k = 0; k < NF_KERNEL_COUNT; k++) kernel_ms[k] = 0.0;
      if (kernel_launches)
        for (int k = 0; k < NF_KERNEL_COUNT; k++) kernel_launches[k] = 0;
      for (size_t i = 0; i < s->prof_used; i++) {
        float t = 0.f;
        ck(cudaEventElapsedTime(&t, s->prof_ev[2 * i], s->prof_ev[2 * i + 1]), "cudaEventElapsedTime");
        if (kernel_ms) kernel_ms[s->prof_cls[i]] += t;
        if (kernel_launches) kernel_launches[s->prof_cls[i]] += 1;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s->check_status();
  });
}

int nf_tune(nf_solver* s, int* config) {
  return guarded(s, [&]() -> int {
    s->tune();
    if (config) {
      config[0] = s->kgrad.block;
      config[1] = s->kgrad.variant;
      config[2] = s->kflux.block;
      config[3] = s->kflux.variant;
    }
    return s->check_status();
  });
}

int nf_set_launch_shapes(nf_solver* s, const int* config) {
  if (!s) return NF_ERR_ARG;
  return guarded(s, [&]() -> int {
    if (!config) return NF_ERR_ARG;
    for (int i = 0; i < 4; i += 2) {
      const int b = config[i], v = config[i + 1];
      const int nv = i == 0 ? s->grad_variants() : s->flux_variants();
      if (b < 32 || b > 128 || b % 32 || v < 0 || v >= nv) {
        s->err = "launch shapes: block must be 32..128 in steps of 32, variant 0.." + std::to_string(nv - 1) +
                 (i == 0 ? " (gradient)" : " (flux)");
        return NF_ERR_ARG;
      }
    }
    s->kgrad.block = config[0];
    s->kgrad.variant = config[1];
    s->kflux.block = config[2];
    s->kflux.variant = config[3];
    s->tuned = true;
    for (auto& g : s->graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    return NF_OK;
  });
}

int nf_fastmath_selftest(const double* x, int64_t n, double* rcp_out, double* rsqrt_out) {
  if (!x || !rcp_out || !rsqrt_out || n <= 0 || n > (int64_t(1) << 26)) return NF_ERR_ARG;
  try {
    DevBuf<double> dx, dr, ds;
    dx.alloc(size_t(n));
    dr.alloc(size_t(n));
    ds.alloc(size_t(n));
    ck(cudaMemcpy(dx.p, x, size_t(n) * sizeof(double), cudaMemcpyHostToDevice), "H2D");
    nf::launch_fastmath(dx.p, int(n), dr.p, ds.p, nf::Launch{256, nullptr});
    ck(cudaGetLastError(), "fastmath launch");
    ck(cudaMemcpy(rcp_out, dr.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
    ck(cudaMemcpy(rsqrt_out, ds.p, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
  } catch (const std::exception& e) {
    nf::set_last_error_text(e.what());
    return NF_ERR_CUDA;
  }
  return NF_OK;
}

int nf_synchronize(nf_solver* s) {
  return guarded(s, [&]() -> int { return s->check_status(); });
}

const char* nf_last_error(const nf_solver* s) { return s ? s->err.c_str() : g_create_error.c_str(); }

void nf_destroy(nf_solver* s) {
  if (!s) return;
  int dev = 0;
  cudaGetDevice(&dev);
  const int own = s->device;
  if (dev != own) cudaSetDevice(own);
  cudaStreamSynchronize(s->stream);
  delete s;
  if (dev != own) cudaSetDevice(dev);
}

// ---------------------------------------------------------------------------
// a mesh split across solvers
// ---------------------------------------------------------------------------
nf_split* nf_split_create(nf_solver* const* parts, int n_parts) {
  if (!parts || n_parts < 1) {
    g_create_error = "nf_split_create: no parts";
    return nullptr;
  }
  auto sp = std::make_unique<nf_split>();
  int dev = 0;
  cudaGetDevice(&dev);
  try {
    const nf_params& p0 = parts[0] ? parts[0]->p : nf_params{};
    for (int i = 0; i < n_parts; i++) {
      nf_solver* s = parts[i];
      if (!s) throw std::invalid_argument("nf_split_create: null part");
      if (s->p.precision != p0.precision || s->p.time_scheme != p0.time_scheme ||
          s->p.spatial_order != p0.spatial_order || s->p.local_time_stepping != p0.local_time_stepping ||
          s->p.dt_from_current_state != p0.dt_from_current_state)
        throw std::invalid_argument("nf_split_create: the parts' solver parameters differ");
      if (s->stage_next != 0) throw std::invalid_argument("nf_split_create: a part is inside a step");
      if (s->p.precision == NF_PREC_MIXED32)
        throw std::invalid_argument("nf_split_create: the mixed form with FP32 copies is not split (its halo would "
                                    "need the FP32 primitives exchanged)");
      for (int j = 0; j < i; j++)
        if (parts[j] == s) throw std::invalid_argument("nf_split_create: a part is listed twice");
      sp->parts.push_back(s);
    }
    sp->global_dt = !p0.local_time_stepping;
    for (int i = 0; i < n_parts; i++) {
      sp->set_dev(parts[i]->device);
      cudaEvent_t a, b;
      ck(cudaEventCreateWithFlags(&a, cudaEventDisableTiming), "cudaEventCreate");
      sp->ready.push_back(a);
      ck(cudaEventCreateWithFlags(&b, cudaEventDisableTiming), "cudaEventCreate");
      sp->copied.push_back(b);
      // peer access between every pair of devices the parts use
      for (int j = 0; j < n_parts; j++) {
        const int d = parts[j]->device;
        if (d == parts[i]->device) continue;
        int ok = 0;
        ck(cudaDeviceCanAccessPeer(&ok, parts[i]->device, d), "cudaDeviceCanAccessPeer");
        if (!ok) throw std::invalid_argument("nf_split_create: devices without peer access");
        const cudaError_t e = cudaDeviceEnablePeerAccess(d, 0);
        if (e == cudaErrorPeerAccessAlreadyEnabled) cudaGetLastError();
        else ck(e, "cudaDeviceEnablePeerAccess");
      }
    }
    sp->set_dev(parts[0]->device);
    ck(cudaEventCreateWithFlags(&sp->dt_done, cudaEventDisableTiming), "cudaEventCreate");
    std::vector<double*> sc;
    for (int i = 0; i < n_parts; i++) sc.push_back(parts[i]->scal.p);
    sp->scal_ptrs.alloc(sc.size());
    ck(cudaMemcpy(sp->scal_ptrs.p, sc.data(), sc.size() * sizeof(double*), cudaMemcpyHostToDevice), "H2D");
  } catch (const std::exception& e) {
    g_create_error = e.what();
    cudaSetDevice(dev);
    return nullptr;
  }
  cudaSetDevice(dev);
  return sp.release();
}

int nf_split_link(nf_split* sp, int from, int to, const int64_t* from_cells, const int64_t* to_cells, int64_t n) {
  return split_guarded(sp, [&]() -> int {
    const int np = int(sp->parts.size());
    if (from < 0 || from >= np || to < 0 || to >= np || from == to || n < 0 || (n > 0 && (!from_cells || !to_cells))) {
      sp->err = "nf_split_link: bad part index, count or null cell list";
      return NF_ERR_ARG;
    }
    const int64_t na = sp->parts[size_t(from)]->n, nb = sp->parts[size_t(to)]->n;
    for (int64_t i = 0; i < n; i++)
      if (from_cells[i] < 0 || from_cells[i] >= na || to_cells[i] < 0 || to_cells[i] >= nb) {
        sp->err = "nf_split_link: cell index out of range at entry " + std::to_string(i);
        return NF_ERR_ARG;
      }
    if (n == 0) return NF_OK;
    auto lk = std::make_unique<nf_split::Link>();
    lk->from = from;
    lk->to = to;
    lk->n = n;
    nf_solver* b = sp->parts[size_t(to)];
    sp->set_dev(b->device);
    lk->from_cells.alloc(size_t(n));
    lk->to_cells.alloc(size_t(n));
    ck(cudaMemcpy(lk->from_cells.p, from_cells, size_t(n) * sizeof(int64_t), cudaMemcpyHostToDevice), "H2D");
    ck(cudaMemcpy(lk->to_cells.p, to_cells, size_t(n) * sizeof(int64_t), cudaMemcpyHostToDevice), "H2D");
    sp->links.push_back(std::move(lk));
    return NF_OK;
  });
}

int nf_split_advance(nf_split* sp, int64_t n_steps) {
  return split_guarded(sp, [&]() -> int {
    if (n_steps < 0) return NF_ERR_ARG;
    for (nf_solver* s : sp->parts)
      if (s->stage_next != 0) {
        sp->err = "nf_split_advance: a part is inside a step";
        return NF_ERR_ARG;
      }
    for (int64_t k = 0; k < n_steps; k++) sp->step();
    return NF_OK;
  });
}

int nf_split_synchronize(nf_split* sp) {
  return split_guarded(sp, [&]() -> int {
    for (nf_solver* s : sp->parts) {
      sp->set_dev(s->device);
      const int rc = s->check_status();
      if (rc != NF_OK) {
        sp->err = s->err;
        return rc;
      }
    }
    return NF_OK;
  });
}

const char* nf_split_last_error(const nf_split* sp) { return sp ? sp->err.c_str() : g_create_error.c_str(); }

void nf_split_destroy(nf_split* sp) {
  if (!sp) return;
  int dev = 0;
  cudaGetDevice(&dev);
  delete sp;
  cudaSetDevice(dev);
}

}  // extern "C"
