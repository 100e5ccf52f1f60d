// Residual norms with no device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need this
// reduction: hosts that hand the library a fixed memory pool and forbid
// allocation after start-up, and real-time drivers that must not block on the
// allocator (cudaMalloc can synchronise the device). nf_residual_norms_noalloc serves them: the caller
// passes the input and output device buffers, and the per-block partial sums
// live in a fixed array compiled into this library.
//
// The array below is a file-scope __device__ variable: every GPU that loads the
// library holds it (128 KiB) until the process exits. In host code its name is
// only a host-side stand-in, not a device address, so the device address is
// looked up with cudaGetSymbolAddress once per device, with that device
// current, the first time the entry point runs on it; that first call should
// therefore come before any stream capture. Every call shares the array and
// overwrites the partials it uses before reading them (nothing needs to start
// at zero); two calls whose kernels overlap on the GPU, e.g. on two unordered
// streams, race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/netflux_b200.h"

namespace nf {
void set_last_error_text(const std::string& msg);  // defined in solver.cu
}

namespace {

constexpr int kThreads = 256;
constexpr long long kChunk = 16384;      // values reduced by one block
constexpr int kMaxBlocks = 8192;         // capacity of the scratch array
constexpr long long kMaxValues = kChunk * kMaxBlocks;  // 134,217,728

// per-block (sum of squares, max |v|)
static __device__ __align__(256) double g_partials[2 * kMaxBlocks];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_addr[kMaxDevices] = {};

// max(a, b) that keeps a NaN from either operand (fmax would drop it: a
// non-finite value must show in the max norm).
__device__ __forceinline__ double max_keep_nan(double a, double b) { return (a != a || a > b) ? a : b; }

__global__ void __launch_bounds__(kThreads) partials_kernel(const double* __restrict__ v, long long n,
                                                            double* __restrict__ part) {
  const long long beg = blockIdx.x * kChunk;
  const long long end = beg + kChunk < n ? beg + kChunk : n;
  double s = 0.0, mx = 0.0;
  for (long long i = beg + threadIdx.x; i < end; i += kThreads) {
    const double x = v[i];
    s += x * x;
    mx = max_keep_nan(mx, fabs(x));
  }
  __shared__ double ss[kThreads], sm[kThreads];
  ss[threadIdx.x] = s;
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int w = kThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      ss[threadIdx.x] += ss[threadIdx.x + w];
      sm[threadIdx.x] = max_keep_nan(sm[threadIdx.x], sm[threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ss[0];
    part[2 * blockIdx.x + 1] = sm[0];
  }
}

__global__ void finalize_kernel(const double* __restrict__ part, int n_blocks, long long n, double* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0, mx = 0.0;
  for (int b = 0; b < n_blocks; b++) {  // fixed order: deterministic
    s += part[2 * b];
    mx = max_keep_nan(mx, part[2 * b + 1]);
  }
  out[0] = n > 0 ? sqrt(s / double(n)) : 0.0;
  out[1] = mx;
}

// Device address of g_partials on the current device (looked up once).
int partials_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    nf::set_last_error_text(std::string("nf_residual_norms_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return NF_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    nf::set_last_error_text("nf_residual_norms_noalloc: device ordinal out of range");
    return NF_ERR_CUDA;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_partials_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_partials);
    if (e != cudaSuccess || !p) {
      nf::set_last_error_text(std::string("nf_residual_norms_noalloc: cudaGetSymbolAddress: ") +
                              cudaGetErrorString(e));
      return NF_ERR_CUDA;
    }
    g_partials_addr[dev] = static_cast<double*>(p);
  }
  *out = g_partials_addr[dev];
  return NF_OK;
}

}  // namespace

extern "C" int nf_residual_norms_noalloc(const double* values, int64_t n, double* out, void* stream) {
  if (n < 0 || n > kMaxValues) {
    char buf[160];
    std::snprintf(buf, sizeof(buf),
                  "nf_residual_norms_noalloc: n = %lld is outside [0, %lld], the capacity of its fixed scratch",
                  static_cast<long long>(n), kMaxValues);
    nf::set_last_error_text(buf);
    return NF_ERR_ARG;
  }
  if (!out || (n > 0 && !values)) {
    nf::set_last_error_text("nf_residual_norms_noalloc: null device pointer");
    return NF_ERR_ARG;
  }
  double* part = nullptr;
  int rc = partials_address(&part);
  if (rc != NF_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int blocks = int((n + kChunk - 1) / kChunk);
  if (blocks > 0) partials_kernel<<<blocks, kThreads, 0, st>>>(values, n, part);
  finalize_kernel<<<1, 32, 0, st>>>(part, blocks, n, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    nf::set_last_error_text(std::string("nf_residual_norms_noalloc: launch: ") + cudaGetErrorString(e));
    return NF_ERR_CUDA;
  }
  return NF_OK;
}
