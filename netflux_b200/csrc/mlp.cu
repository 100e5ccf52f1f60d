// Surrogate MLP for warm starts (extension; the reference has no learned
// part): 7 inputs (cell centroid, wall distance, Mach, bump height) ->
// 4 hidden layers of 128 SiLU units -> 5 outputs (conserved variables
// normalised by the free stream). BF16 weights and activations, FP32
// accumulation in tensor memory, hand-written tcgen05 kernels:
//   mlp_forward_kernel     all five layers of a 128-sample tile, weights
//                          resident in shared memory, the TMEM accumulator
//                          turned into the next layer's operand by the SiLU
//                          epilogue; two tiles in flight per CTA (one
//                          warpgroup, operand buffer and accumulator each), so
//                          one tile's MMAs overlap the other's epilogue;
//                          optionally saves activations and the loss gradient
//   mlp_backward_kernel    the same structure backwards (transposed weights,
//                          SiLU derivative in the epilogue) -> dZ of each layer
//   mlp_wgrad_kernel       dW = dZ^T H over the batch (split over CTAs), batch
//                          chunks transposed while staged into one of two
//                          operand buffers as the other's MMAs run, five
//                          accumulators in TMEM, bias gradients through a
//                          column of ones
//   mlp_adam_kernel        sums the per-CTA partial gradients, Adam update of
//                          the FP32 master weights, BF16 operand images
// Parameters in FP32 (padded shapes): W0 [128][16] (inputs 0..6, bias in
// column 7), W1..W3 [128][128], b1..b3 [128], W4 [16][128] (rows 0..4 used),
// b4 [16].
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstring>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/netflux_b200.h"
#include "umma.cuh"

namespace nf {
namespace mlp {

constexpr int H = 128;    // hidden width
constexpr int KIN = 16;   // 7 inputs, a constant 1 (bias) and padding
constexpr int NOUT = 16;  // 5 outputs and padding
constexpr int NIN = 7;
constexpr int NO = 5;
constexpr int TILE = 128;  // samples per tile (MMA M)
constexpr int KC = 32;     // batch rows per weight-gradient chunk
constexpr int NAUG = H + 16;  // H columns, a column of ones, padding
constexpr long long kWaitCycles = 4000000000LL;  // about 2 s

constexpr int OFF_W0 = 0;
constexpr int OFF_W1 = OFF_W0 + H * KIN;
constexpr int OFF_W2 = OFF_W1 + H * H;
constexpr int OFF_W3 = OFF_W2 + H * H;
constexpr int OFF_B1 = OFF_W3 + H * H;
constexpr int OFF_B2 = OFF_B1 + H;
constexpr int OFF_B3 = OFF_B2 + H;
constexpr int OFF_W4 = OFF_B3 + H;
constexpr int OFF_B4 = OFF_W4 + NOUT * H;
constexpr int N_PARAM = OFF_B4 + NOUT;

// BF16 operand images, byte offsets; each is a K-major tile as it sits in
// shared memory. Forward: W_l as [out][in]; backward: W_l^T as [in][out].
constexpr int IMG_W0 = 0;
constexpr int IMG_W1 = IMG_W0 + H * KIN * 2;
constexpr int IMG_W2 = IMG_W1 + H * H * 2;
constexpr int IMG_W3 = IMG_W2 + H * H * 2;
constexpr int IMG_W4 = IMG_W3 + H * H * 2;
constexpr int IMG_FWD = IMG_W4 + NOUT * H * 2;
constexpr int IMG_T1 = 0;
constexpr int IMG_T2 = IMG_T1 + H * H * 2;
constexpr int IMG_T3 = IMG_T2 + H * H * 2;
constexpr int IMG_T4 = IMG_T3 + H * H * 2;
constexpr int IMG_BWD = IMG_T4 + H * NOUT * 2;

// saved activations, element offsets in units of BF16 for B samples
__host__ __device__ inline int64_t save_x0(int64_t) { return 0; }
__host__ __device__ inline int64_t save_z(int64_t B, int l) { return B * KIN + (2 * l) * B * H; }
__host__ __device__ inline int64_t save_h(int64_t B, int l) { return B * KIN + (2 * l + 1) * B * H; }
__host__ __device__ inline int64_t save_size(int64_t B) { return B * KIN + 8 * B * H; }

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

// pack 8 floats to 8 BF16 (round to nearest even) in a 16-byte vector
__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 r;
  uint32_t* w = reinterpret_cast<uint32_t*>(&r);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<const uint32_t*>(&p);
  }
  return r;
}
__device__ __forceinline__ void unpack8(uint4 r, float* v) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(&r);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const __nv_bfloat162 p = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    const float2 f = __bfloat1622float2(p);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// Tiles in flight per CTA in the forward and backward kernels: each has its
// own 128 threads (one warpgroup), operand buffers, mbarrier and TMEM
// accumulator, so one tile's MMAs run while another's epilogue does.
constexpr int NSLOT = 2;
// CTAs that give every slot at least one tile of B samples
inline int tile_ctas(int64_t B) { return int(((B + TILE - 1) / TILE + NSLOT - 1) / NSLOT); }

// Barrier among the 128 threads of one slot (named barriers 1..NSLOT; 0 is
// __syncthreads), optionally AND-reducing a predicate over them.
__device__ __forceinline__ void slot_sync(int slot) { asm volatile("bar.sync %0, 128;" ::"r"(slot + 1) : "memory"); }
__device__ __forceinline__ bool slot_sync_and(int slot, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t"
      ".reg .pred p, q;\n\t"
      "setp.ne.u32 q, %1, 0;\n\t"
      "bar.red.and.pred p, %2, 128, q;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(r)
      : "r"(uint32_t(v)), "r"(slot + 1)
      : "memory");
  return r != 0;
}

struct TileSync {
  uint32_t mbar;
  uint32_t phase = 0;
  unsigned* status;
  int slot = -1;  // -1: the whole CTA takes part; else the slot's 128 threads
  // wait for the MMAs committed to mbar; every participating thread agrees on
  // the outcome
  __device__ bool wait() {
    const bool ok = umma::mbar_wait(mbar, phase, kWaitCycles);
    phase ^= 1u;
    const bool all_ok = slot < 0 ? __syncthreads_and(ok ? 1 : 0) != 0 : slot_sync_and(slot, ok);
    if (!all_ok && (threadIdx.x & 127) == 0) atomicOr(status, 1u);
    umma::fence_after_sync();
    return all_ok;
  }
};

// Common prologue: n mbarriers, TMEM columns; returns the TMEM base address.
__device__ uint32_t setup(uint64_t* mbar, int n, uint32_t* tslot, uint32_t ncols) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < n; i++) umma::mbar_init(umma::smem_addr(mbar + i), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) umma::tmem_alloc(umma::smem_addr(tslot), ncols);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  return *tslot;
}
__device__ void teardown(uint32_t tbase, uint32_t ncols) {
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  if (threadIdx.x < 32) umma::tmem_dealloc(tbase, ncols);
}

// ---------------------------------------------------------------------------
// Forward
// ---------------------------------------------------------------------------
struct FwdArgs {
  const uint8_t* img;     // forward BF16 image
  const float* params;    // FP32 master (biases b1..b4)
  const float* feat;      // [n_all][7] normalised inputs
  const float* target;    // [n_all][5] or null
  const int64_t* idx;     // [B] sample of each row, or null (row b is sample b)
  int64_t B;
  float* out;             // [B][5] or null
  __nv_bfloat16* save;    // saved activations (save_size(B)) or null
  __nv_bfloat16* dz4;     // [B][16] loss gradient or null
  double* loss;           // sum of squared errors (with target)
  float loss_scale;       // d loss / d y = loss_scale * (y - t)
  unsigned* status;
};

constexpr int FWD_SLOT = TILE * H * 2 + TILE * KIN * 2;  // one tile's activations and inputs
constexpr int FWD_SMEM = IMG_FWD + NSLOT * FWD_SLOT + (3 * H + NOUT) * 4 + 64;

__global__ void __launch_bounds__(128 * NSLOT, 1) mlp_forward_kernel(FwdArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int slot = threadIdx.x >> 7, t = threadIdx.x & 127, w = t >> 5;
  uint8_t* s_img = sm;
  uint8_t* s_act = sm + IMG_FWD + slot * FWD_SLOT;  // [128 x K128] activations of this slot's tile
  uint8_t* s_x0 = s_act + TILE * H * 2;             // [128 x K16] inputs
  float* s_bias = reinterpret_cast<float*>(sm + IMG_FWD + NSLOT * FWD_SLOT);  // b1, b2, b3, b4
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(s_bias + 3 * H + NOUT);    // one per slot
  uint32_t* s_tslot = reinterpret_cast<uint32_t*>(s_mbar + NSLOT);
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.img);
    uint4* dst = reinterpret_cast<uint4*>(s_img);
    for (int i = threadIdx.x; i < IMG_FWD / 16; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < 3 * H + NOUT; i += blockDim.x)
      s_bias[i] = i < 3 * H ? a.params[OFF_B1 + i] : a.params[OFF_B4 + i - 3 * H];
  }
  const uint32_t tbase = setup(s_mbar, NSLOT, s_tslot, 128 * NSLOT);
  TileSync sync{umma::smem_addr(s_mbar + slot), 0u, a.status, slot};
  const uint32_t tacc = tbase + uint32_t(slot * 128);  // this slot's 128 accumulator columns
  const uint32_t lane_addr = tacc + (uint32_t(w * 32) << 16);
  const uint32_t a_act = umma::smem_addr(s_act), a_x0 = umma::smem_addr(s_x0), a_img = umma::smem_addr(s_img);
  const uint32_t id128 = umma::idesc_bf16(128, 128), id16 = umma::idesc_bf16(128, 16);
  const int64_t n_tiles = (a.B + TILE - 1) / TILE;
  float ssq = 0.f;
  for (int64_t tile = int64_t(blockIdx.x) * NSLOT + slot; tile < n_tiles; tile += int64_t(gridDim.x) * NSLOT) {
    const int64_t b = tile * TILE + t;
    const bool valid = b < a.B;
    {  // inputs: 7 features, a constant 1 (bias of layer 0), zeros
      float x[KIN];
#pragma unroll
      for (int k = 0; k < KIN; k++) x[k] = 0.f;
      if (valid) {
        const int64_t s = a.idx ? a.idx[b] : b;
#pragma unroll
        for (int k = 0; k < NIN; k++) x[k] = a.feat[s * NIN + k];
        x[NIN] = 1.f;
      }
      const uint4 c0 = pack8(x), c1 = pack8(x + 8);
      *reinterpret_cast<uint4*>(s_x0 + umma::kmaj_off(t, 0, KIN)) = c0;
      *reinterpret_cast<uint4*>(s_x0 + umma::kmaj_off(t, 8, KIN)) = c1;
      if (a.save && valid) {
        uint4* g = reinterpret_cast<uint4*>(a.save + save_x0(a.B) + b * KIN);
        g[0] = c0;
        g[1] = c1;
      }
    }
    umma::fence_async_shared();
    slot_sync(slot);
    for (int l = 0; l < 5; l++) {
      if (t == 0) {
        umma::fence_after_sync();
        if (l == 0) {
          umma::mma_bf16(tacc, umma::kmaj_desc(a_x0, KIN, 0), umma::kmaj_desc(a_img + IMG_W0, KIN, 0), id128, 0);
        } else {
          const int img = l == 1 ? IMG_W1 : l == 2 ? IMG_W2 : l == 3 ? IMG_W3 : IMG_W4;
#pragma unroll 1
          for (int s = 0; s < H / 16; s++)
            umma::mma_bf16(tacc, umma::kmaj_desc(a_act, H, s), umma::kmaj_desc(a_img + img, H, s),
                           l == 4 ? id16 : id128, s > 0 ? 1u : 0u);
        }
        umma::commit(sync.mbar);
      }
      if (!sync.wait()) goto done;
      if (l < 4) {
        // z = acc (+ bias), h = silu(z): the next layer's operand
#pragma unroll 1
        for (int c0 = 0; c0 < H; c0 += 32) {
          float v[32];
          umma::tmem_ld32(lane_addr + uint32_t(c0), v);
          float z[32], h[32];
#pragma unroll
          for (int j = 0; j < 32; j++) {
            z[j] = l == 0 ? v[j] : v[j] + s_bias[(l - 1) * H + c0 + j];
            h[j] = silu(z[j]);
          }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const uint4 hv = pack8(h + 8 * q);
            *reinterpret_cast<uint4*>(s_act + umma::kmaj_off(t, c0 + 8 * q, H)) = hv;
            if (a.save && valid) {
              *reinterpret_cast<uint4*>(a.save + save_z(a.B, l) + b * H + c0 + 8 * q) = pack8(z + 8 * q);
              *reinterpret_cast<uint4*>(a.save + save_h(a.B, l) + b * H + c0 + 8 * q) = hv;
            }
          }
        }
      } else {
        float v[16];
        umma::tmem_ld16(lane_addr, v);
        float y[NO];
#pragma unroll
        for (int o = 0; o < NO; o++) y[o] = v[o] + s_bias[3 * H + o];
        if (valid) {
          if (a.out)
#pragma unroll
            for (int o = 0; o < NO; o++) a.out[b * NO + o] = y[o];
          if (a.target) {
            const int64_t s = a.idx ? a.idx[b] : b;
            float g[16];
#pragma unroll
            for (int o = 0; o < 16; o++) g[o] = 0.f;
#pragma unroll
            for (int o = 0; o < NO; o++) {
              const float e = y[o] - a.target[s * NO + o];
              ssq += e * e;
              g[o] = a.loss_scale * e;
            }
            if (a.dz4) {
              uint4* gd = reinterpret_cast<uint4*>(a.dz4 + b * NOUT);
              gd[0] = pack8(g);
              gd[1] = pack8(g + 8);
            }
          }
        }
      }
      // TMEM read and operand written before the next MMA
      umma::fence_before_sync();
      umma::fence_async_shared();
      slot_sync(slot);
    }
  }
done:
  if (a.loss) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ssq += __shfl_xor_sync(0xffffffffu, ssq, off);
    if ((t & 31) == 0 && ssq != 0.f) atomicAdd(a.loss, double(ssq));
  }
  teardown(tbase, 128 * NSLOT);
}

// ---------------------------------------------------------------------------
// Backward through the activations: dZ3, dZ2, dZ1, dZ0
// ---------------------------------------------------------------------------
struct BwdArgs {
  const uint8_t* img;          // backward BF16 image (transposed weights)
  const __nv_bfloat16* save;   // saved activations
  const __nv_bfloat16* dz4;    // [B][16]
  int64_t B;
  __nv_bfloat16* dz;           // [4][B][128]: dZ0..dZ3
  unsigned* status;
};

constexpr int BWD_SLOT = TILE * H * 2 + TILE * NOUT * 2;  // one tile's operand and output gradient
constexpr int BWD_SMEM = IMG_BWD + NSLOT * BWD_SLOT + 64;

__global__ void __launch_bounds__(128 * NSLOT, 1) mlp_backward_kernel(BwdArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  const int slot = threadIdx.x >> 7, t = threadIdx.x & 127, w = t >> 5;
  uint8_t* s_img = sm;
  uint8_t* s_act = sm + IMG_BWD + slot * BWD_SLOT;
  uint8_t* s_d4 = s_act + TILE * H * 2;
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(sm + IMG_BWD + NSLOT * BWD_SLOT);  // one per slot
  uint32_t* s_tslot = reinterpret_cast<uint32_t*>(s_mbar + NSLOT);
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.img);
    uint4* dst = reinterpret_cast<uint4*>(s_img);
    for (int i = threadIdx.x; i < IMG_BWD / 16; i += blockDim.x) dst[i] = src[i];
  }
  const uint32_t tbase = setup(s_mbar, NSLOT, s_tslot, 128 * NSLOT);
  TileSync sync{umma::smem_addr(s_mbar + slot), 0u, a.status, slot};
  const uint32_t tacc = tbase + uint32_t(slot * 128);  // this slot's 128 accumulator columns
  const uint32_t lane_addr = tacc + (uint32_t(w * 32) << 16);
  const uint32_t a_act = umma::smem_addr(s_act), a_d4 = umma::smem_addr(s_d4), a_img = umma::smem_addr(s_img);
  const uint32_t id128 = umma::idesc_bf16(128, 128);
  const int64_t n_tiles = (a.B + TILE - 1) / TILE;
  for (int64_t tile = int64_t(blockIdx.x) * NSLOT + slot; tile < n_tiles; tile += int64_t(gridDim.x) * NSLOT) {
    const int64_t b = tile * TILE + t;
    const bool valid = b < a.B;
    {
      uint4 c0 = make_uint4(0, 0, 0, 0), c1 = c0;
      if (valid) {
        const uint4* g = reinterpret_cast<const uint4*>(a.dz4 + b * NOUT);
        c0 = g[0];
        c1 = g[1];
      }
      *reinterpret_cast<uint4*>(s_d4 + umma::kmaj_off(t, 0, NOUT)) = c0;
      *reinterpret_cast<uint4*>(s_d4 + umma::kmaj_off(t, 8, NOUT)) = c1;
    }
    umma::fence_async_shared();
    slot_sync(slot);
    // layer l's input gradient: dH_{l-1} = dZ_l W_l, then dZ_{l-1} = dH_{l-1} silu'(Z_{l-1})
    for (int l = 4; l >= 1; l--) {
      if (t == 0) {
        umma::fence_after_sync();
        if (l == 4) {
          umma::mma_bf16(tacc, umma::kmaj_desc(a_d4, NOUT, 0), umma::kmaj_desc(a_img + IMG_T4, NOUT, 0), id128, 0);
        } else {
          const int img = l == 1 ? IMG_T1 : l == 2 ? IMG_T2 : IMG_T3;
#pragma unroll 1
          for (int s = 0; s < H / 16; s++)
            umma::mma_bf16(tacc, umma::kmaj_desc(a_act, H, s), umma::kmaj_desc(a_img + img, H, s), id128,
                           s > 0 ? 1u : 0u);
        }
        umma::commit(sync.mbar);
      }
      const int lo = l - 1;  // layer whose pre-activation gradient this is
      // the saved pre-activations of this row, 32 columns at a time, loaded one
      // chunk ahead (the first before the wait) to hide their latency
      const __nv_bfloat16* zrow = a.save + save_z(a.B, lo) + b * H;
      auto load_z = [&](uint4* z4, int c0) {
#pragma unroll
        for (int q = 0; q < 4; q++)
          z4[q] = valid ? *reinterpret_cast<const uint4*>(zrow + c0 + 8 * q) : make_uint4(0u, 0u, 0u, 0u);
      };
      uint4 zc[4];
      load_z(zc, 0);
      if (!sync.wait()) goto done;
#pragma unroll 1
      for (int c0 = 0; c0 < H; c0 += 32) {
        uint4 zn[4];
        if (c0 + 32 < H) load_z(zn, c0 + 32);
        float v[32];
        umma::tmem_ld32(lane_addr + uint32_t(c0), v);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          float z[8], d[8];
          unpack8(zc[q], z);
#pragma unroll
          for (int j = 0; j < 8; j++) d[j] = valid ? v[8 * q + j] * dsilu(z[j]) : 0.f;
          const uint4 dv = pack8(d);
          *reinterpret_cast<uint4*>(s_act + umma::kmaj_off(t, c0 + 8 * q, H)) = dv;
          if (valid) *reinterpret_cast<uint4*>(a.dz + int64_t(lo) * a.B * H + b * H + c0 + 8 * q) = dv;
        }
#pragma unroll
        for (int q = 0; q < 4; q++) zc[q] = zn[q];
      }
      umma::fence_before_sync();
      umma::fence_async_shared();
      slot_sync(slot);
    }
  }
done:
  teardown(tbase, 128 * NSLOT);
}

// ---------------------------------------------------------------------------
// Weight gradients: per CTA, chunks of KC batch rows; partial sums [cta][N_PARAM]
// ---------------------------------------------------------------------------
struct WgArgs {
  const __nv_bfloat16* save;
  const __nv_bfloat16* dz;   // [4][B][128]
  const __nv_bfloat16* dz4;  // [B][16]
  int64_t B;
  float* partial;            // [gridDim.x][N_PARAM]
  unsigned* status;
};

constexpr int WG_A = H * KC * 2;      // one [128 x KC] operand
constexpr int WG_BA = NAUG * KC * 2;  // one [144 x KC] operand
constexpr int WG_B16 = 16 * KC * 2;   // one [16 x KC] operand
constexpr int WG_BUF = 5 * WG_A + 3 * WG_BA + 2 * WG_B16;  // one chunk's operands
constexpr int WG_THREADS = 256;
constexpr int WG_SMEM = 2 * WG_BUF + 64;  // two chunks: one staged while the other's MMAs run
// TMEM columns of the five accumulators (32-column aligned; 512 allocated)
constexpr int ACC1 = 0, ACC2 = 160, ACC3 = 320, ACC0 = 480, ACC4 = 496;

// Column q (0..7) of an 8 x 8 BF16 block held as 8 rows of 16 bytes: the 8
// values of that column as 16 bytes (row 0 first).
__device__ __forceinline__ uint4 column8(const uint4 v[8], int q) {
  const uint32_t sel = (q & 1) ? 0x7632u : 0x5410u;  // high or low 16-bit half of each word
  uint32_t w[8];
#pragma unroll
  for (int r = 0; r < 8; r++) w[r] = (&v[r].x)[q >> 1];
  uint4 o;
  o.x = __byte_perm(w[0], w[1], sel);
  o.y = __byte_perm(w[2], w[3], sel);
  o.z = __byte_perm(w[4], w[5], sel);
  o.w = __byte_perm(w[6], w[7], sel);
  return o;
}

// rows [0, F) of a K-major [rows x KC] tile <- transpose of a [KC][F] row-major
// BF16 block (batch rows b0 .. b0+KC; rows past B are zero). Each task is one
// 8-feature chunk of 8 consecutive batch rows: eight 16-byte loads, an 8 x 8
// transpose in registers, eight 16-byte stores of core-matrix rows.
template <int F>
__device__ __forceinline__ void stage_t(uint8_t* dst, const __nv_bfloat16* src, int64_t b0, int64_t B) {
  constexpr int kChunks = F / 8, kTasks = kChunks * (KC / 8);
  for (int task = threadIdx.x; task < kTasks; task += blockDim.x) {
    const int ch = task % kChunks, rg = task / kChunks;
    uint4 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int64_t b = b0 + rg * 8 + r;
      v[r] = b < B ? *reinterpret_cast<const uint4*>(src + b * F + ch * 8) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int q = 0; q < 8; q++)
      *reinterpret_cast<uint4*>(dst + umma::kmaj_off(ch * 8 + q, rg * 8, KC)) = column8(v, q);
  }
}
__device__ __forceinline__ void stage_t16(uint8_t* dst, const __nv_bfloat16* src, int64_t b0, int64_t B) {
  stage_t<16>(dst, src, b0, B);
}

struct WgBuf {
  uint8_t* A[5];  // dZ0^T, dZ1^T, dZ2^T, dZ3^T, H3^T
  uint8_t* B[3];  // [H0|1]^T, [H1|1]^T, [H2|1]^T
  uint8_t* X;     // X0^T
  uint8_t* D4;    // dZ4^T
  uint8_t* base;
  __device__ explicit WgBuf(uint8_t* base_) : base(base_) {
    for (int i = 0; i < 5; i++) A[i] = base + i * WG_A;
    for (int i = 0; i < 3; i++) B[i] = base + 5 * WG_A + i * WG_BA;
    X = base + 5 * WG_A + 3 * WG_BA;
    D4 = X + WG_B16;
  }
  // the chunk of KC batch rows from b0, transposed into K-major operands. The
  // tasks of the eight 128-feature operands (one 8-feature chunk of 8 rows
  // each) are spread over all threads, two per thread with both tasks' loads
  // issued before either's stores, so no thread runs the operands one after
  // another while the others wait at the barrier.
  __device__ void stage(const WgArgs& a, int64_t b0) {
    constexpr int kPer = (H / 8) * (KC / 8), kWide = 8 * kPer;
    static_assert(kWide == 2 * WG_THREADS, "two wide tasks per thread");
    uint4 v[2][8];
    int ch[2], rg[2];
    uint8_t* dst[2];
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int task = threadIdx.x + u * WG_THREADS, op = task / kPer, lt = task % kPer;
      ch[u] = lt % (H / 8);
      rg[u] = lt / (H / 8);
      // operands 0-3: dZ0..dZ3; 4: H3; 5-7: H0..H2
      const __nv_bfloat16* src = op < 4 ? a.dz + int64_t(op) * a.B * H : a.save + save_h(a.B, op == 4 ? 3 : op - 5);
      dst[u] = op < 5 ? base + op * WG_A : base + 5 * WG_A + (op - 5) * WG_BA;  // A[op] or B[op - 5]
#pragma unroll
      for (int r = 0; r < 8; r++) {
        const int64_t b = b0 + rg[u] * 8 + r;
        v[u][r] = b < a.B ? *reinterpret_cast<const uint4*>(src + b * H + ch[u] * 8) : make_uint4(0u, 0u, 0u, 0u);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; u++)
#pragma unroll
      for (int q = 0; q < 8; q++)
        *reinterpret_cast<uint4*>(dst[u] + umma::kmaj_off(ch[u] * 8 + q, rg[u] * 8, KC)) = column8(v[u], q);
    stage_t16(X, a.save + save_x0(a.B), b0, a.B);
    stage_t16(D4, a.dz4, b0, a.B);
  }
  // every accumulator += this chunk's product (one thread)
  __device__ void issue(uint32_t tbase, bool first) const {
    const uint32_t idA = umma::idesc_bf16(128, NAUG), id16 = umma::idesc_bf16(128, 16);
#pragma unroll 1
    for (int s = 0; s < KC / 16; s++) {
      const uint32_t acc = (first && s == 0) ? 0u : 1u;
#pragma unroll
      for (int l = 1; l <= 3; l++)
        umma::mma_bf16(tbase + uint32_t(l == 1 ? ACC1 : l == 2 ? ACC2 : ACC3),
                       umma::kmaj_desc(umma::smem_addr(A[l]), KC, s), umma::kmaj_desc(umma::smem_addr(B[l - 1]), KC, s),
                       idA, acc);
      umma::mma_bf16(tbase + ACC0, umma::kmaj_desc(umma::smem_addr(A[0]), KC, s),
                     umma::kmaj_desc(umma::smem_addr(X), KC, s), id16, acc);
      umma::mma_bf16(tbase + ACC4, umma::kmaj_desc(umma::smem_addr(A[4]), KC, s),
                     umma::kmaj_desc(umma::smem_addr(D4), KC, s), id16, acc);
    }
  }
};

// The CTA's chunks in turn through two operand buffers: while the tensor core
// multiplies chunk i from one buffer, the threads stage chunk i + 1 into the
// other (after the MMAs of chunk i - 1, which read it, are done).
__global__ void __launch_bounds__(WG_THREADS, 1) mlp_wgrad_kernel(WgArgs a) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(sm + 2 * WG_BUF);  // one per buffer
  uint32_t* s_tslot = reinterpret_cast<uint32_t*>(s_mbar + 2);
  const int t = threadIdx.x;
  // constant rows of the augmented operands: a row of ones, then zeros
  for (int task = t; task < 2 * 3 * (NAUG - H) * (KC / 8); task += blockDim.x) {
    const int g = task % (KC / 8), r = H + (task / (KC / 8)) % (NAUG - H), i = task / (KC / 8) / (NAUG - H);
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = r == H ? 1.f : 0.f;
    uint8_t* op = sm + (i / 3) * WG_BUF + 5 * WG_A + (i % 3) * WG_BA;  // WgBuf::B[i % 3] of buffer i / 3
    *reinterpret_cast<uint4*>(op + umma::kmaj_off(r, g * 8, KC)) = pack8(v);
  }
  const uint32_t tbase = setup(s_mbar, 2, s_tslot, 512);
  TileSync sync0{umma::smem_addr(s_mbar), 0u, a.status}, sync1{umma::smem_addr(s_mbar + 1), 0u, a.status};
  auto wait_buf = [&](int k) { return k == 0 ? sync0.wait() : sync1.wait(); };
  const int64_t n_chunks = (a.B + KC - 1) / KC;
  float db4 = 0.f;
  int i = 0;  // chunks of this CTA issued
  if (int64_t(blockIdx.x) < n_chunks) WgBuf(sm).stage(a, int64_t(blockIdx.x) * KC);
  umma::fence_async_shared();
  __syncthreads();
  for (int64_t ch = blockIdx.x; ch < n_chunks; ch += gridDim.x, i++) {
    const int cur = i & 1;
    if (t == 0) {
      umma::fence_after_sync();
      WgBuf(sm + cur * WG_BUF).issue(tbase, i == 0);
      umma::commit(cur == 0 ? sync0.mbar : sync1.mbar);
    }
    // bias gradient of the output layer: this thread's output t & 15 over the chunk's rows
    // t >> 4 and (t >> 4) + 16 (two independent loads, no thread waits on a serial sum)
#pragma unroll
    for (int j = t >> 4; j < KC; j += WG_THREADS / 16) {
      const int64_t b = ch * KC + j;
      if (b < a.B) db4 += __bfloat162float(a.dz4[b * 16 + (t & 15)]);
    }
    const int64_t nx = ch + gridDim.x;
    if (nx < n_chunks) {
      if (i >= 1 && !wait_buf(cur ^ 1)) goto done;  // chunk i - 1 has read the other buffer
      WgBuf(sm + (cur ^ 1) * WG_BUF).stage(a, nx * KC);
      umma::fence_async_shared();
    }
    __syncthreads();  // the next chunk's operands staged before it is issued
  }
  if (i > 0 && !wait_buf((i - 1) & 1)) goto done;  // the last chunk, and with it every earlier one
  {
    float* P = a.partial + int64_t(blockIdx.x) * N_PARAM;
    const int row = t & 127, half = t >> 7;  // TMEM lane; which accumulators this warpgroup reads
    const uint32_t lane_addr = tbase + (uint32_t(((t >> 5) & 3) * 32) << 16);
    if (i == 0) {  // this CTA had no rows
      for (int k = t; k < N_PARAM; k += blockDim.x) P[k] = 0.f;
    } else {
      for (int l = 1 + half; l <= 3; l += 2) {  // layers 1, 3 | 2
        const uint32_t base = lane_addr + uint32_t(l == 1 ? ACC1 : l == 2 ? ACC2 : ACC3);
        const int offW = l == 1 ? OFF_W1 : l == 2 ? OFF_W2 : OFF_W3;
        const int offB = l == 1 ? OFF_B1 : l == 2 ? OFF_B2 : OFF_B3;
#pragma unroll 1
        for (int c0 = 0; c0 < H; c0 += 32) {
          float v[32];
          umma::tmem_ld32(base + uint32_t(c0), v);
#pragma unroll
          for (int j = 0; j < 32; j++) P[offW + row * H + c0 + j] = v[j];
        }
        float v[16];
        umma::tmem_ld16(base + uint32_t(H), v);
        P[offB + row] = v[0];
      }
      if (half == 1) {
        float v[16];
        umma::tmem_ld16(lane_addr + ACC0, v);
#pragma unroll
        for (int j = 0; j < 16; j++) P[OFF_W0 + row * KIN + j] = v[j];
        umma::tmem_ld16(lane_addr + ACC4, v);
#pragma unroll
        for (int j = 0; j < 16; j++) P[OFF_W4 + j * H + row] = v[j];
      }
      // db4: the two lanes of a warp with the same output, then the warps in order
      // (a fixed order: the same bits every run); the operand buffers are free now
      db4 += __shfl_xor_sync(0xffffffffu, db4, 16);
      float* s_db4 = reinterpret_cast<float*>(sm);  // [warps][16]
      if ((t & 31) < 16) s_db4[(t >> 5) * 16 + (t & 15)] = db4;
      __syncthreads();
      if (t < 16) {
        float sum = 0.f;
        for (int wq = 0; wq < WG_THREADS / 32; wq++) sum += s_db4[wq * 16 + t];
        P[OFF_B4 + t] = sum;
      }
    }
  }
done:
  teardown(tbase, 512);
}

// ---------------------------------------------------------------------------
// Gradient reduction, Adam and the BF16 images (one thread per parameter)
// ---------------------------------------------------------------------------
struct AdamArgs {
  const float* partial;
  int n_part;
  float* params;
  float* m;
  float* v;
  float* grad;         // summed gradient (written when non-null)
  uint8_t* img_fwd;
  uint8_t* img_bwd;
  const int* step;     // Adam step count including this update
  float lr;
  int apply;           // 0: only sum the gradient
};

__device__ __forceinline__ void write_images(const AdamArgs& a, int p, float w) {
  const __nv_bfloat16 h = __float2bfloat16_rn(w);
  auto put = [&](uint8_t* img, int off, int r, int k, int K) {
    *reinterpret_cast<__nv_bfloat16*>(img + off + umma::kmaj_off(r, k, K)) = h;
  };
  if (p < OFF_W1) {
    const int o = (p - OFF_W0) / KIN, i = (p - OFF_W0) % KIN;
    put(a.img_fwd, IMG_W0, o, i, KIN);
  } else if (p < OFF_B1) {
    const int l = (p - OFF_W1) / (H * H), e = (p - OFF_W1) % (H * H), o = e / H, i = e % H;
    put(a.img_fwd, IMG_W1 + l * H * H * 2, o, i, H);
    put(a.img_bwd, IMG_T1 + l * H * H * 2, i, o, H);
  } else if (p >= OFF_W4 && p < OFF_B4) {
    const int o = (p - OFF_W4) / H, i = (p - OFF_W4) % H;
    put(a.img_fwd, IMG_W4, o, i, H);
    put(a.img_bwd, IMG_T4, i, o, NOUT);
  }
}

__global__ void mlp_adam_kernel(AdamArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N_PARAM) return;
  float g = 0.f;
  for (int c = 0; c < a.n_part; c++) g += a.partial[int64_t(c) * N_PARAM + p];
  if (a.grad) a.grad[p] = g;
  if (!a.apply) return;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const int t = max(*a.step, 1);  // advanced by mlp_step_kernel before this update
  const float m = b1 * a.m[p] + (1.f - b1) * g;
  const float v = b2 * a.v[p] + (1.f - b2) * g * g;
  a.m[p] = m;
  a.v[p] = v;
  const float mh = m / (1.f - powf(b1, float(t)));
  const float vh = v / (1.f - powf(b2, float(t)));
  const float w = a.params[p] - a.lr * mh / (sqrtf(vh) + eps);
  a.params[p] = w;
  write_images(a, p, w);
}

__global__ void mlp_images_kernel(AdamArgs a) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N_PARAM) write_images(a, p, a.params[p]);
}

__global__ void mlp_step_kernel(int* step, double* loss) {
  *step += 1;
  *loss = 0.0;
}

// uniform sample indices in [0, n) from a counter-based hash (splitmix64)
__global__ void mlp_sample_kernel(int64_t* idx, int64_t B, int64_t n, uint64_t seed, const int* step) {
  const int64_t b = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= B) return;
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t(*step) * uint64_t(B) + uint64_t(b) + 1);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  idx[b] = int64_t(z % uint64_t(n));
}

// One GEMM D[128 x N] = A[128 x K] B[N x K]^T through the same tcgen05 path
// (operands row-major BF16 in global memory), for testing the descriptors.
__global__ void __launch_bounds__(128, 1) umma_gemm_test_kernel(const __nv_bfloat16* A, const __nv_bfloat16* B,
                                                               int N, int K, float* D, unsigned* status) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* sa = sm;
  uint8_t* sb = sm + 128 * K * 2;
  uint64_t* s_mbar = reinterpret_cast<uint64_t*>(sb + N * K * 2);
  uint32_t* s_tslot = reinterpret_cast<uint32_t*>(s_mbar + 1);
  const int t = threadIdx.x, w = t >> 5;
  for (int i = t; i < 128 * K; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16*>(sa + umma::kmaj_off(i / K, i % K, K)) = A[i];
  for (int i = t; i < N * K; i += blockDim.x)
    *reinterpret_cast<__nv_bfloat16*>(sb + umma::kmaj_off(i / K, i % K, K)) = B[i];
  const uint32_t tbase = setup(s_mbar, 1, s_tslot, 256);
  TileSync sync{umma::smem_addr(s_mbar), 0u, status};
  umma::fence_async_shared();
  __syncthreads();
  if (t == 0) {
    umma::fence_after_sync();
    for (int s = 0; s < K / 16; s++)
      umma::mma_bf16(tbase, umma::kmaj_desc(umma::smem_addr(sa), K, s), umma::kmaj_desc(umma::smem_addr(sb), K, s),
                     umma::idesc_bf16(128, N), s > 0 ? 1u : 0u);
    umma::commit(sync.mbar);
  }
  if (sync.wait()) {
    for (int c0 = 0; c0 < N; c0 += 16) {
      float v[16];
      umma::tmem_ld16(tbase + (uint32_t(w * 32) << 16) + uint32_t(c0), v);
      for (int j = 0; j < 16; j++) D[t * N + c0 + j] = v[j];
    }
  }
  teardown(tbase, 256);
}

// Distance from each point to the nearest of m wall points (the surrogate's
// wall-distance input): one thread per point, wall points staged through
// shared memory in tiles of 1024.
constexpr int WD_TILE = 1024;
__global__ void __launch_bounds__(256) wall_distance_kernel(const float* __restrict__ pts, int64_t n,
                                                             const float* __restrict__ wall, int64_t m,
                                                             float* __restrict__ out) {
  __shared__ float sw[3 * WD_TILE];
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const float px = i < n ? pts[3 * i] : 0.f, py = i < n ? pts[3 * i + 1] : 0.f, pz = i < n ? pts[3 * i + 2] : 0.f;
  float best = 3.0e38f;
  for (int64_t t0 = 0; t0 < m; t0 += WD_TILE) {
    const int cnt = int(m - t0 < WD_TILE ? m - t0 : WD_TILE);
    __syncthreads();
    for (int j = threadIdx.x; j < 3 * cnt; j += blockDim.x) sw[j] = wall[3 * t0 + j];
    __syncthreads();
#pragma unroll 4
    for (int j = 0; j < cnt; j++) {
      const float dx = px - sw[3 * j], dy = py - sw[3 * j + 1], dz = pz - sw[3 * j + 2];
      best = fminf(best, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
    }
  }
  if (i < n) out[i] = sqrtf(best);
}

}  // namespace mlp
}  // namespace nf

// ---------------------------------------------------------------------------
// Host object and C ABI
// ---------------------------------------------------------------------------
using namespace nf::mlp;

namespace {

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (count <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    n = count;
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

std::string g_mlp_error;

}  // namespace

struct nf_mlp {
  cudaStream_t stream = nullptr;
  int n_sm = 148;
  Buf<float> params, m, v, grad, partial, feat, target, out;
  Buf<uint8_t> img_fwd, img_bwd;
  Buf<int> step;
  Buf<double> loss;
  Buf<unsigned> status;
  Buf<int64_t> idx;
  Buf<__nv_bfloat16> save, dz, dz4;
  int64_t n_data = 0;
  int64_t batch = 0;
  int n_wg = 0;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_batch = 0;
  uint64_t graph_seed = 0;
  float graph_lr = 0.f;
  std::string err;

  int64_t ensured = 0;
  void ensure_batch(int64_t B) {
    if (B != ensured && graph) {  // the captured step holds this batch's buffers
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    ensured = B;
    save.alloc(size_t(save_size(B)));
    dz.alloc(size_t(4) * B * H);
    dz4.alloc(size_t(B) * NOUT);
    idx.alloc(size_t(B));
    n_wg = int(std::min<int64_t>(n_sm, (B + KC - 1) / KC));
    partial.alloc(size_t(n_wg) * N_PARAM);
  }
  AdamArgs adam_args(float lr, int apply) {
    AdamArgs a{};
    a.partial = partial.p;
    a.n_part = n_wg;
    a.params = params.p;
    a.m = m.p;
    a.v = v.p;
    a.grad = grad.p;
    a.img_fwd = img_fwd.p;
    a.img_bwd = img_bwd.p;
    a.step = step.p;
    a.lr = lr;
    a.apply = apply;
    return a;
  }
  // forward (+ loss gradient), backward, weight gradients, reduction (+ Adam)
  void enqueue_pass(const float* f, const float* tg, const int64_t* ix, int64_t B, float lr, int apply) {
    FwdArgs fa{};
    fa.img = img_fwd.p;
    fa.params = params.p;
    fa.feat = f;
    fa.target = tg;
    fa.idx = ix;
    fa.B = B;
    fa.save = save.p;
    fa.dz4 = dz4.p;
    fa.loss = loss.p;
    fa.loss_scale = 2.0f / float(B * NO);
    fa.status = status.p;
    const int n_cta = std::min(tile_ctas(B), n_sm);
    mlp_forward_kernel<<<n_cta, 128 * NSLOT, FWD_SMEM, stream>>>(fa);
    BwdArgs ba{img_bwd.p, save.p, dz4.p, B, dz.p, status.p};
    mlp_backward_kernel<<<n_cta, 128 * NSLOT, BWD_SMEM, stream>>>(ba);
    WgArgs wa{save.p, dz.p, dz4.p, B, partial.p, status.p};
    mlp_wgrad_kernel<<<n_wg, WG_THREADS, WG_SMEM, stream>>>(wa);
    mlp_adam_kernel<<<(N_PARAM + 255) / 256, 256, 0, stream>>>(adam_args(lr, apply));
  }
  void check_status() {
    unsigned st = 0;
    ck(cudaMemcpyAsync(&st, status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, stream), "status D2H");
    ck(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    if (st) throw std::runtime_error("tensor-core wait timed out in an MLP kernel");
  }
  ~nf_mlp() {
    if (graph) cudaGraphExecDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

template <typename F>
int mlp_guarded(nf_mlp* m, F&& fn) {
  if (!m) return NF_ERR_ARG;
  try {
    return fn();
  } catch (const std::exception& e) {
    m->err = e.what();
    return NF_ERR_CUDA;
  }
}

void set_kernel_smem() {
  ck(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM), "smem attr");
  ck(cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, BWD_SMEM), "smem attr");
  ck(cudaFuncSetAttribute(mlp_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, WG_SMEM), "smem attr");
  ck(cudaFuncSetAttribute(umma_gemm_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024),
     "smem attr");
}

}  // namespace

extern "C" {

int nf_mlp_param_count(void) { return N_PARAM; }

nf_mlp* nf_mlp_create(uint64_t seed) {
  auto m = std::make_unique<nf_mlp>();
  try {
    set_kernel_smem();
    ck(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    ck(cudaDeviceGetAttribute(&m->n_sm, cudaDevAttrMultiProcessorCount, dev), "attr");
    std::vector<float> p(N_PARAM, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int rows, int cols, int used_rows, int used_cols, int fan_in) {
      std::uniform_real_distribution<float> u(-1.f / std::sqrt(float(fan_in)), 1.f / std::sqrt(float(fan_in)));
      for (int r = 0; r < used_rows; r++)
        for (int c = 0; c < used_cols; c++) p[size_t(off + r * cols + c)] = u(rng);
      (void)rows;
    };
    fill(OFF_W0, H, KIN, H, NIN + 1, NIN);  // weights and the bias column
    fill(OFF_W1, H, H, H, H, H);
    fill(OFF_W2, H, H, H, H, H);
    fill(OFF_W3, H, H, H, H, H);
    fill(OFF_B1, 1, 3 * H, 1, 3 * H, H);
    fill(OFF_W4, NOUT, H, NO, H, H);
    fill(OFF_B4, 1, NOUT, 1, NO, H);
    m->params.alloc(N_PARAM);
    m->m.alloc(N_PARAM);
    m->v.alloc(N_PARAM);
    m->grad.alloc(N_PARAM);
    m->img_fwd.alloc(IMG_FWD);
    m->img_bwd.alloc(IMG_BWD);
    m->step.alloc(1);
    m->loss.alloc(1);
    m->status.alloc(1);
    ck(cudaMemcpyAsync(m->params.p, p.data(), N_PARAM * sizeof(float), cudaMemcpyHostToDevice, m->stream), "H2D");
    ck(cudaMemsetAsync(m->m.p, 0, N_PARAM * sizeof(float), m->stream), "memset");
    ck(cudaMemsetAsync(m->v.p, 0, N_PARAM * sizeof(float), m->stream), "memset");
    ck(cudaMemsetAsync(m->img_fwd.p, 0, IMG_FWD, m->stream), "memset");
    ck(cudaMemsetAsync(m->img_bwd.p, 0, IMG_BWD, m->stream), "memset");
    ck(cudaMemsetAsync(m->step.p, 0, sizeof(int), m->stream), "memset");
    ck(cudaMemsetAsync(m->loss.p, 0, sizeof(double), m->stream), "memset");
    ck(cudaMemsetAsync(m->status.p, 0, sizeof(unsigned), m->stream), "memset");
    mlp_images_kernel<<<(N_PARAM + 255) / 256, 256, 0, m->stream>>>(m->adam_args(0.f, 0));
    ck(cudaGetLastError(), "images");
    ck(cudaStreamSynchronize(m->stream), "sync");
  } catch (const std::exception& e) {
    g_mlp_error = std::string("nf_mlp_create: ") + e.what();
    return nullptr;
  }
  return m.release();
}

const char* nf_mlp_last_error(const nf_mlp* m) { return m ? m->err.c_str() : g_mlp_error.c_str(); }

void nf_mlp_destroy(nf_mlp* m) {
  if (m && m->stream) cudaStreamSynchronize(m->stream);
  delete m;
}

int nf_mlp_get_params(nf_mlp* m, float* out) {
  return mlp_guarded(m, [&]() -> int {
    if (!out) return NF_ERR_ARG;
    ck(cudaMemcpyAsync(out, m->params.p, N_PARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream), "D2H");
    ck(cudaStreamSynchronize(m->stream), "sync");
    return NF_OK;
  });
}

int nf_mlp_set_params(nf_mlp* m, const float* in) {
  return mlp_guarded(m, [&]() -> int {
    if (!in) return NF_ERR_ARG;
    ck(cudaMemcpyAsync(m->params.p, in, N_PARAM * sizeof(float), cudaMemcpyHostToDevice, m->stream), "H2D");
    mlp_images_kernel<<<(N_PARAM + 255) / 256, 256, 0, m->stream>>>(m->adam_args(0.f, 0));
    ck(cudaGetLastError(), "images");
    ck(cudaStreamSynchronize(m->stream), "sync");
    return NF_OK;
  });
}

int nf_mlp_set_data(nf_mlp* m, const float* features, const float* targets, int64_t n) {
  return mlp_guarded(m, [&]() -> int {
    if (!features || !targets || n <= 0) return NF_ERR_ARG;
    m->feat.alloc(size_t(n) * NIN);
    m->target.alloc(size_t(n) * NO);
    ck(cudaMemcpyAsync(m->feat.p, features, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, m->stream),
       "H2D");
    ck(cudaMemcpyAsync(m->target.p, targets, size_t(n) * NO * sizeof(float), cudaMemcpyHostToDevice, m->stream),
       "H2D");
    ck(cudaStreamSynchronize(m->stream), "sync");
    m->n_data = n;
    return NF_OK;
  });
}

int nf_mlp_train(nf_mlp* m, int64_t steps, int64_t batch, float lr, uint64_t seed, int n_report,
                 double* loss_report, double* ms_out) {
  return mlp_guarded(m, [&]() -> int {
    if (steps < 0 || batch <= 0 || m->n_data <= 0 || n_report < 0 || (n_report > 0 && !loss_report))
      return NF_ERR_ARG;
    m->ensure_batch(batch);
    if (!m->graph || m->graph_batch != batch || m->graph_seed != seed || m->graph_lr != lr) {
      if (m->graph) cudaGraphExecDestroy(m->graph);
      m->graph = nullptr;
      cudaGraph_t g = nullptr;
      ck(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal), "capture");
      mlp_step_kernel<<<1, 1, 0, m->stream>>>(m->step.p, m->loss.p);  // loss = 0 (step advanced below)
      mlp_sample_kernel<<<int((batch + 255) / 256), 256, 0, m->stream>>>(m->idx.p, batch, m->n_data, seed, m->step.p);
      m->enqueue_pass(m->feat.p, m->target.p, m->idx.p, batch, lr, 1);
      ck(cudaStreamEndCapture(m->stream, &g), "capture");
      ck(cudaGraphInstantiate(&m->graph, g, 0), "instantiate");
      cudaGraphDestroy(g);
      m->graph_batch = batch;
      m->graph_seed = seed;
      m->graph_lr = lr;
    }
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    ck(cudaEventRecord(e0, m->stream), "event");
    // n_report segments; after each, the mean squared error of its last step
    int64_t done = 0;
    for (int r = 0; r < std::max(n_report, 1); r++) {
      const int64_t upto = n_report > 0 ? steps * (r + 1) / n_report : steps;
      for (; done < upto; done++) ck(cudaGraphLaunch(m->graph, m->stream), "graph launch");
      if (n_report > 0) {
        double l = 0;
        ck(cudaMemcpyAsync(&l, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream), "D2H");
        ck(cudaStreamSynchronize(m->stream), "sync");
        loss_report[r] = l / double(batch * NO);
      }
    }
    ck(cudaEventRecord(e1, m->stream), "event");
    ck(cudaEventSynchronize(e1), "event");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "event");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_out) *ms_out = ms;
    m->check_status();
    return NF_OK;
  });
}

int nf_mlp_gradients(nf_mlp* m, const float* features, const float* targets, int64_t n, float* grad_out,
                     double* loss_out) {
  return mlp_guarded(m, [&]() -> int {
    if (!features || !targets || n <= 0 || !grad_out) return NF_ERR_ARG;
    m->ensure_batch(n);
    Buf<float> f, tg;
    f.alloc(size_t(n) * NIN);
    tg.alloc(size_t(n) * NO);
    ck(cudaMemcpyAsync(f.p, features, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, m->stream), "H2D");
    ck(cudaMemcpyAsync(tg.p, targets, size_t(n) * NO * sizeof(float), cudaMemcpyHostToDevice, m->stream), "H2D");
    ck(cudaMemsetAsync(m->loss.p, 0, sizeof(double), m->stream), "memset");
    m->enqueue_pass(f.p, tg.p, nullptr, n, 0.f, 0);
    ck(cudaGetLastError(), "launch");
    ck(cudaMemcpyAsync(grad_out, m->grad.p, N_PARAM * sizeof(float), cudaMemcpyDeviceToHost, m->stream), "D2H");
    double l = 0;
    ck(cudaMemcpyAsync(&l, m->loss.p, sizeof(double), cudaMemcpyDeviceToHost, m->stream), "D2H");
    ck(cudaStreamSynchronize(m->stream), "sync");
    if (loss_out) *loss_out = l / double(n * NO);
    m->check_status();
    return NF_OK;
  });
}

int nf_mlp_predict(nf_mlp* m, const float* features, int64_t n, float* out, double* ms_out) {
  return mlp_guarded(m, [&]() -> int {
    if (!features || !out || n <= 0) return NF_ERR_ARG;
    Buf<float> f, o;
    f.alloc(size_t(n) * NIN);
    o.alloc(size_t(n) * NO);
    ck(cudaMemcpyAsync(f.p, features, size_t(n) * NIN * sizeof(float), cudaMemcpyHostToDevice, m->stream), "H2D");
    FwdArgs fa{};
    fa.img = m->img_fwd.p;
    fa.params = m->params.p;
    fa.feat = f.p;
    fa.B = n;
    fa.out = o.p;
    fa.status = m->status.p;
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "event");
    ck(cudaEventCreate(&e1), "event");
    ck(cudaEventRecord(e0, m->stream), "event");
    mlp_forward_kernel<<<std::min(tile_ctas(n), m->n_sm), 128 * NSLOT, FWD_SMEM, m->stream>>>(fa);
    ck(cudaGetLastError(), "launch");
    ck(cudaEventRecord(e1, m->stream), "event");
    ck(cudaMemcpyAsync(out, o.p, size_t(n) * NO * sizeof(float), cudaMemcpyDeviceToHost, m->stream), "D2H");
    ck(cudaStreamSynchronize(m->stream), "sync");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, e0, e1), "event");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_out) *ms_out = ms;
    m->check_status();
    return NF_OK;
  });
}

int nf_wall_distance(const float* points, int64_t n, const float* wall, int64_t m, float* out) {
  if (!points || !wall || !out || n <= 0 || m <= 0) return NF_ERR_ARG;
  try {
    Buf<float> p, w, o;
    p.alloc(size_t(3) * n);
    w.alloc(size_t(3) * m);
    o.alloc(size_t(n));
    ck(cudaMemcpy(p.p, points, size_t(3) * n * sizeof(float), cudaMemcpyHostToDevice), "H2D");
    ck(cudaMemcpy(w.p, wall, size_t(3) * m * sizeof(float), cudaMemcpyHostToDevice), "H2D");
    wall_distance_kernel<<<unsigned((n + 255) / 256), 256>>>(p.p, n, w.p, m, o.p);
    ck(cudaGetLastError(), "wall distance launch");
    ck(cudaMemcpy(out, o.p, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
  } catch (const std::exception& e) {
    g_mlp_error = e.what();
    return NF_ERR_CUDA;
  }
  return NF_OK;
}

int nf_mlp_gemm_selftest(const uint16_t* A, const uint16_t* B, int N, int K, float* D) {
  if (!A || !B || !D || N < 16 || N > 256 || N % 16 || K < 16 || K > 256 || K % 16) return NF_ERR_ARG;
  try {
    set_kernel_smem();
    Buf<__nv_bfloat16> a, b;
    Buf<float> d;
    Buf<unsigned> st;
    a.alloc(size_t(128) * K);
    b.alloc(size_t(N) * K);
    d.alloc(size_t(128) * N);
    st.alloc(1);
    ck(cudaMemcpy(a.p, A, size_t(128) * K * 2, cudaMemcpyHostToDevice), "H2D");
    ck(cudaMemcpy(b.p, B, size_t(N) * K * 2, cudaMemcpyHostToDevice), "H2D");
    ck(cudaMemset(st.p, 0, sizeof(unsigned)), "memset");
    const int smem = (128 + N) * K * 2 + 64;
    umma_gemm_test_kernel<<<1, 128, smem>>>(a.p, b.p, N, K, d.p, st.p);
    ck(cudaGetLastError(), "launch");
    ck(cudaDeviceSynchronize(), "sync");
    unsigned s = 0;
    ck(cudaMemcpy(&s, st.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "D2H");
    if (s) throw std::runtime_error("tensor-core wait timed out");
    ck(cudaMemcpy(D, d.p, size_t(128) * N * 4, cudaMemcpyDeviceToHost), "D2H");
  } catch (const std::exception& e) {
    g_mlp_error = e.what();
    return NF_ERR_CUDA;
  }
  return NF_OK;
}

}  // extern "C"
