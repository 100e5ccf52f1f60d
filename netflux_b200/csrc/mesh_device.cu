// Device-side construction of the face-based grid: the same Mesh as the host
// builder (mesh.cpp), bit for bit, with the face matching, the orderings, the
// geometry, the projected areas and the Hilbert renumbering done on the GPU.
//
// What it follows is what mesh.cpp follows: FV_Grid::create_face_structure
// (FV_Grid.cpp:21-152) and calc_geometry_properties (154-205),
// Faces::sort (GeometryUtilities.cpp:484-513), the tetrahedron and triangle
// geometry (GeometryUtilities.cpp:289-325), calc_Delta_S (Solver.cpp:276-298):
//   1. every tetrahedron face keyed by its sorted node triple; two stable
//      radix sorts (third node, then the first two) give the records in
//      (triple, cell, local face) order, as the host's sort of packed keys;
//   2. runs of equal triples: two records are an interior face owned by the
//      lower cell (whose local face defines the face's nodes), one record a
//      boundary candidate, more an error; interior faces sorted by (i, j);
//   3. marker triangles matched to candidates by binary search, ghosts
//      numbered in marker order, each patch's faces ordered by (i, ghost);
//   4. cell volumes and centroids, face normals, areas, centroid-to-face
//      vectors and ghost centroids with the host's operations in the host's
//      order (this file is compiled with -fmad=false, so nothing is fused);
//      the projected areas summed per cell in face order through a per-cell
//      list of its faces; Hilbert keys of the centroids and a stable sort.
// Radix sorts and scans are CUB's (CUDA toolkit); everything else is below.
// Errors are detected on the device and reported with the host builder's
// messages for the same input (the first offending element in input order).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cub/cub.cuh>
#include <string>
#include <vector>

#include "../../include/netflux_b200.h"
#include "mesh.hpp"
#include "mesh_common.hpp"

namespace nf {
void set_last_error_text(const std::string& msg);  // solver.cu
}

namespace {

using nf::MeshError;

struct CudaFail : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaFail(std::string(what) + ": " + cudaGetErrorString(e));
}

// Device buffer owned for the duration of one build.
template <typename T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  explicit Buf(size_t count = 0) { alloc(count); }
  void alloc(size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    if (count) ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
};

inline int blocks(int64_t n, int b = 256) { return int((n + b - 1) / b); }

// First offending element per error kind (INT64_MAX: none).
enum : int { kBadNode = 0, kDegenerate = 1, kShared = 2, kMarkerNode = 3, kNoMatch = 4, kTwice = 5, kErrKinds = 6 };

__device__ __forceinline__ void note_error(unsigned long long* first, int kind, long long where) {
  atomicMin(first + kind, (unsigned long long)where);
}

// ---- 1. face records ----
// tet (after the reader's node 1 <-> 2 swap, GeometryUtilities.cpp:452-455)
__global__ void tets_kernel(const int64_t* __restrict__ in, int64_t N, int64_t n_nodes, uint32_t* __restrict__ tet,
                            unsigned long long* first) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int64_t v[4] = {in[4 * c], in[4 * c + 2], in[4 * c + 1], in[4 * c + 3]};
  bool ok = true;
  for (int q = 0; q < 4; q++) {
    ok = ok && v[q] >= 0 && v[q] < n_nodes;
    tet[4 * c + q] = uint32_t(ok ? v[q] : 0);
  }
  if (!ok) note_error(first, kBadNode, c);
}

__device__ __forceinline__ void face_triple(const uint32_t* __restrict__ tet, uint32_t pay, uint32_t t[3]) {
  const uint32_t c = pay >> 2, k = pay & 3u;
  t[0] = tet[4 * size_t(c) + nf::tet_face(k, 0)];
  t[1] = tet[4 * size_t(c) + nf::tet_face(k, 1)];
  t[2] = tet[4 * size_t(c) + nf::tet_face(k, 2)];
  nf::sort3(t[0], t[1], t[2]);
}

// record r = 4 c + k: payload c << 2 | k, first key its triple's third node
__global__ void records_kernel(const uint32_t* __restrict__ tet, int64_t M, uint32_t* __restrict__ key3,
                               uint32_t* __restrict__ pay, unsigned long long* first) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  uint32_t t[3];
  face_triple(tet, uint32_t(r), t);
  if (t[0] == t[1] || t[1] == t[2]) note_error(first, kDegenerate, r >> 2);
  key3[r] = t[2];
  pay[r] = uint32_t(r);
}

// second key: the triple's first two nodes, packed in 2 * nb bits
__global__ void key12_kernel(const uint32_t* __restrict__ tet, const uint32_t* __restrict__ pay, int64_t M, int nb,
                             uint64_t* __restrict__ key12) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  uint32_t t[3];
  face_triple(tet, pay[r], t);
  key12[r] = (uint64_t(t[0]) << nb) | t[1];
}

// ---- 2. runs of equal triples ----
__device__ __forceinline__ bool same3(const uint32_t a[3], const uint32_t b[3]) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

// flags: interior face starting at r (run of two), boundary candidate (run of one)
__global__ void runs_kernel(const uint32_t* __restrict__ tet, const uint32_t* __restrict__ pay, int64_t M,
                            int* __restrict__ is_int, int* __restrict__ is_bnd, unsigned long long* first) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  uint32_t t[3], u[3];
  face_triple(tet, pay[r], t);
  bool start = true;
  if (r > 0) {
    face_triple(tet, pay[r - 1], u);
    start = !same3(t, u);
  }
  int len = 1;
  if (start) {
    if (r + 1 < M) {
      face_triple(tet, pay[r + 1], u);
      if (same3(t, u)) {
        len = 2;
        if (r + 2 < M) {
          face_triple(tet, pay[r + 2], u);
          if (same3(t, u)) len = 3;
        }
      }
    }
    if (len > 2) note_error(first, kShared, 0);
  }
  is_int[r] = start && len == 2;
  is_bnd[r] = start && len == 1;
}

// interior face (i, j, local face of i) and boundary candidate (triple, cell, local face)
__global__ void compact_kernel(const uint32_t* __restrict__ tet, const uint32_t* __restrict__ pay, int64_t M,
                               const int* __restrict__ is_int, const int* __restrict__ pos_int,
                               const int* __restrict__ is_bnd, const int* __restrict__ pos_bnd,
                               uint64_t* __restrict__ ij, uint32_t* __restrict__ ik, uint32_t* __restrict__ btri,
                               uint32_t* __restrict__ bpay) {
  const int64_t r = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (r >= M) return;
  if (is_int[r]) {
    // the two records are in payload order: the first is the lower cell,
    // which found the face first in the reference's cell loop
    const uint32_t a = pay[r], b = pay[r + 1];
    const int q = pos_int[r];
    ij[q] = (uint64_t(a >> 2) << 32) | (b >> 2);
    ik[q] = a & 3u;
  } else if (is_bnd[r]) {
    uint32_t t[3];
    face_triple(tet, pay[r], t);
    const int q = pos_bnd[r];
    btri[3 * size_t(q)] = t[0];
    btri[3 * size_t(q) + 1] = t[1];
    btri[3 * size_t(q) + 2] = t[2];
    bpay[q] = pay[r];
  }
}

// ---- 3. marker triangles ----
__device__ __forceinline__ int cmp3(const uint32_t a[3], const uint32_t* b) {
  for (int q = 0; q < 3; q++)
    if (a[q] != b[q]) return a[q] < b[q] ? -1 : 1;
  return 0;
}

// candidate of each marker triangle (in key order, binary search), and the
// first triangle that claims each candidate
__global__ void match_kernel(const int64_t* __restrict__ tris, int64_t T, int64_t n_nodes,
                             const uint32_t* __restrict__ btri, int64_t NB, int* __restrict__ cand,
                             unsigned long long* __restrict__ first_t, unsigned long long* first) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= T) return;
  uint32_t v[3];
  for (int q = 0; q < 3; q++) {
    const int64_t n = tris[3 * t + q];
    if (n < 0 || n >= n_nodes) {
      note_error(first, kMarkerNode, t);
      cand[t] = -1;
      return;
    }
    v[q] = uint32_t(n);
  }
  nf::sort3(v[0], v[1], v[2]);
  int64_t lo = 0, hi = NB;  // first candidate not below v
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (cmp3(v, btri + 3 * mid) > 0) lo = mid + 1;
    else hi = mid;
  }
  if (lo >= NB || cmp3(v, btri + 3 * lo) != 0) {
    note_error(first, kNoMatch, t);
    cand[t] = -1;
    return;
  }
  cand[t] = int(lo);
  atomicMin(first_t + lo, (unsigned long long)t);
}

// a triangle whose candidate an earlier triangle claimed lists its face twice
__global__ void twice_kernel(const int* __restrict__ cand, int64_t T, const unsigned long long* __restrict__ first_t,
                             unsigned long long* first) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= T || cand[t] < 0) return;
  if (first_t[cand[t]] != (unsigned long long)t) note_error(first, kTwice, t);
}

// boundary face of triangle t: sort key (patch, owner cell), value t
__global__ void gface_kernel(const int* __restrict__ cand, const uint32_t* __restrict__ bpay,
                             const int* __restrict__ patch_of, int64_t T, uint64_t* __restrict__ key,
                             uint32_t* __restrict__ tval) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= T) return;
  key[t] = (uint64_t(uint32_t(patch_of[t])) << 32) | (bpay[cand[t]] >> 2);
  tval[t] = uint32_t(t);
}

// ---- 4. geometry (GeometryUtilities.cpp:289-325, FV_Grid.cpp:154-205, 237-267) ----
struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 ld3(const double* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 scale(double s, D3 a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {  // Eigen's operand order
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ double dot(D3 a, D3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

__global__ void cell_geometry_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tet, int64_t N,
                                     double* __restrict__ vol, double* __restrict__ cen) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const D3 n0 = ld3(nodes + 3 * size_t(tet[4 * c])), n1 = ld3(nodes + 3 * size_t(tet[4 * c + 1])),
           n2 = ld3(nodes + 3 * size_t(tet[4 * c + 2])), n3 = ld3(nodes + 3 * size_t(tet[4 * c + 3]));
  vol[c] = dot(cross(sub(n1, n0), sub(n2, n0)), sub(n3, n0)) / 6;
  const D3 m = scale(1.0 / 4, add(add(add(n0, n1), n2), n3));
  cen[3 * c] = m.x;
  cen[3 * c + 1] = m.y;
  cen[3 * c + 2] = m.z;
}

struct FaceOut {
  uint32_t *face_i, *face_j, *face_nodes;
  int32_t* face_patch;
  double *S, *ri, *rj, *nhat, *area, *cen;
};

// face f between cells i and j (j >= N: a ghost, whose centroid this face sets)
__device__ void face_geometry(const double* __restrict__ nodes, int64_t N, int64_t f, uint32_t i, uint32_t j,
                              const uint32_t fn[3], FaceOut o) {
  for (int q = 0; q < 3; q++) o.face_nodes[3 * f + q] = fn[q];
  const D3 n0 = ld3(nodes + 3 * size_t(fn[0])), n1 = ld3(nodes + 3 * size_t(fn[1])), n2 = ld3(nodes + 3 * size_t(fn[2]));
  D3 S = scale(0.5, cross(sub(n1, n0), sub(n2, n0)));  // triangle_calc_face_normal
  const D3 fc = {((n0.x + n1.x) + n2.x) / 3, ((n0.y + n1.y) + n2.y) / 3, ((n0.z + n1.z) + n2.z) / 3};
  const D3 ci = ld3(o.cen + 3 * size_t(i));
  if (j >= uint32_t(N)) {  // calc_ghost_centroid: 2 * face centroid - centroid_i
    const D3 cg = sub(scale(2, fc), ci);
    o.cen[3 * size_t(j)] = cg.x;
    o.cen[3 * size_t(j) + 1] = cg.y;
    o.cen[3 * size_t(j) + 2] = cg.z;
  }
  const D3 cj = ld3(o.cen + 3 * size_t(j));
  if (dot(S, sub(cj, ci)) < 0) S = scale(-1, S);  // point from i to j
  const D3 r_i = sub(fc, ci), r_j = sub(fc, cj);
  const double z = dot(S, S);
  const double a = sqrt(z);
  const double Sv[3] = {S.x, S.y, S.z}, Ri[3] = {r_i.x, r_i.y, r_i.z}, Rj[3] = {r_j.x, r_j.y, r_j.z};
  for (int d = 0; d < 3; d++) {
    o.S[3 * f + d] = Sv[d];
    o.ri[3 * f + d] = Ri[d];
    o.rj[3 * f + d] = Rj[d];
    o.nhat[3 * f + d] = z > 0 ? Sv[d] / a : Sv[d];  // Eigen normalized()
  }
  o.area[f] = a;
  o.face_i[f] = i;
  o.face_j[f] = j;
  o.face_patch[f] = -1;
}

__global__ void interior_geometry_kernel(const double* __restrict__ nodes, const uint32_t* __restrict__ tet,
                                         int64_t N, const uint64_t* __restrict__ ij, const uint32_t* __restrict__ ik,
                                         int64_t NIF, FaceOut o) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= NIF) return;
  const uint32_t i = uint32_t(ij[f] >> 32), j = uint32_t(ij[f] & 0xffffffffu), k = ik[f];
  const uint32_t fn[3] = {tet[4 * size_t(i) + nf::tet_face(k, 0)], tet[4 * size_t(i) + nf::tet_face(k, 1)],
                          tet[4 * size_t(i) + nf::tet_face(k, 2)]};
  face_geometry(nodes, N, f, i, j, fn, o);
}

// boundary face NIF + s: the s-th in (patch, i, ghost) order, triangle t
__global__ void boundary_geometry_kernel(const double* __restrict__ nodes, int64_t N, int64_t NIF,
                                         const uint64_t* __restrict__ key, const uint32_t* __restrict__ tval,
                                         const int64_t* __restrict__ tris, int64_t T, FaceOut o) {
  const int64_t s = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= T) return;
  const uint32_t t = tval[s];
  const uint32_t fn[3] = {uint32_t(tris[3 * size_t(t)]), uint32_t(tris[3 * size_t(t) + 1]),
                          uint32_t(tris[3 * size_t(t) + 2])};
  const int64_t f = NIF + s;
  face_geometry(nodes, N, f, uint32_t(key[s] & 0xffffffffu), uint32_t(N + t), fn, o);
  o.face_patch[f] = int32_t(key[s] >> 32);
}

// calc_Delta_S: both cells of every interior face, in face order; entry 2 f
// is (i, f), 2 f + 1 is (j, f)
__global__ void ds_pairs_kernel(const uint32_t* __restrict__ face_i, const uint32_t* __restrict__ face_j, int64_t NIF,
                                uint32_t* __restrict__ cell, uint32_t* __restrict__ face, int* __restrict__ count) {
  const int64_t f = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (f >= NIF) return;
  cell[2 * f] = face_i[f];
  cell[2 * f + 1] = face_j[f];
  face[2 * f] = face[2 * f + 1] = uint32_t(f);
  atomicAdd(count + face_i[f], 1);
  atomicAdd(count + face_j[f], 1);
}

// each cell sums 0.5 |S| of its faces in face order, as the reference's face
// loop reaches it
__global__ void ds_sum_kernel(const uint32_t* __restrict__ face_sorted, const int* __restrict__ off, int64_t N,
                              const double* __restrict__ S, double* __restrict__ dS) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N) return;
  double s[3] = {0.0, 0.0, 0.0};
  for (int e = off[c]; e < off[c + 1]; e++) {
    const size_t f = face_sorted[e];
    for (int d = 0; d < 3; d++) {
      const double tmp = 0.5 * fabs(S[3 * f + d]);
      s[d] += tmp;
    }
  }
  for (int d = 0; d < 3; d++) dS[3 * c + d] = s[d];
}

__global__ void hilbert_kernel(const double* __restrict__ cen, int64_t N, double lo0, double lo1, double lo2,
                               double q, uint64_t* __restrict__ key, uint32_t* __restrict__ cell) {
  const int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const double lo[3] = {lo0, lo1, lo2};
  uint32_t u[3];
  for (int d = 0; d < 3; d++) {
    const double v = (cen[3 * c + d] - lo[d]) * q;
    u[d] = uint32_t(fmin(fmax(v, 0.0), double((1u << nf::kHilbertBits) - 1)));
  }
  key[c] = nf::hilbert3(u[0], u[1], u[2], nf::kHilbertBits);
  cell[c] = uint32_t(c);
}

// CUB radix sort of (key, value) pairs on bits [0, end_bit), stable
template <typename K, typename V>
void sort_pairs(K* keys, K* keys_alt, V* vals, V* vals_alt, int64_t n, int end_bit, cudaStream_t st, K** out_keys,
                V** out_vals) {
  cub::DoubleBuffer<K> kb(keys, keys_alt);
  cub::DoubleBuffer<V> vb(vals, vals_alt);
  size_t bytes = 0;
  ck(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kb, vb, n, 0, end_bit, st), "radix sort size");
  Buf<unsigned char> tmp(std::max<size_t>(bytes, 1));
  ck(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, kb, vb, n, 0, end_bit, st), "radix sort");
  *out_keys = kb.Current();
  *out_vals = vb.Current();
}

void exclusive_sum(const int* in, int* out, int64_t n, cudaStream_t st) {
  size_t bytes = 0;
  ck(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, st), "scan size");
  Buf<unsigned char> tmp(std::max<size_t>(bytes, 1));
  ck(cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n, st), "scan");
}

template <typename T>
void to_host(std::vector<T>& h, const T* d, size_t n, cudaStream_t st) {
  h.resize(n);
  if (n) ck(cudaMemcpyAsync(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H");
}

int bits_for(int64_t n) {
  int b = 1;
  while (b < 32 && (int64_t(1) << b) < n) b++;
  return b;
}

}  // namespace

namespace nf {

Mesh build_mesh_device(const std::vector<double>& nodes, const std::vector<int64_t>& tets_in,
                       const std::vector<MarkerInput>& markers) {
  Mesh m;
  if (nodes.size() % 3 || tets_in.size() % 4) throw MeshError("node or tet array has a wrong length");
  m.n_nodes = int64_t(nodes.size() / 3);
  const int64_t N = int64_t(tets_in.size() / 4);
  m.n_cells = N;
  if (N == 0) throw MeshError("mesh has no volume elements");
  if (m.n_nodes >= (int64_t(1) << 32) || N >= (int64_t(1) << 30))
    throw MeshError("mesh too large for 32-bit node / 30-bit cell indices");
  const int64_t M = 4 * N;
  const int nb = bits_for(m.n_nodes);
  cudaStream_t st = nullptr;
  ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};

  Buf<unsigned long long> first{kErrKinds};
  {
    std::vector<unsigned long long> h(kErrKinds, ~0ull);
    ck(cudaMemcpyAsync(first.p, h.data(), kErrKinds * sizeof(unsigned long long), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaStreamSynchronize(st), "sync");
  }
  auto errors = [&]() {
    std::vector<unsigned long long> h(kErrKinds);
    ck(cudaMemcpyAsync(h.data(), first.p, kErrKinds * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "sync");
    return h;
  };

  // ---- 1. tets and face records, sorted by (triple, cell, local face) ----
  Buf<double> d_nodes{nodes.size()};
  Buf<int64_t> d_tin{tets_in.size()};
  Buf<uint32_t> d_tet{size_t(M)};
  ck(cudaMemcpyAsync(d_nodes.p, nodes.data(), nodes.size() * sizeof(double), cudaMemcpyHostToDevice, st), "H2D");
  ck(cudaMemcpyAsync(d_tin.p, tets_in.data(), tets_in.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st), "H2D");
  tets_kernel<<<blocks(N), 256, 0, st>>>(d_tin.p, N, m.n_nodes, d_tet.p, first.p);
  ck(cudaGetLastError(), "tets");
  {
    const auto e = errors();
    if (e[kBadNode] != ~0ull) throw MeshError("tet " + std::to_string(e[kBadNode]) + " references a missing node");
  }
  d_tin.alloc(0);
  Buf<uint32_t> k3{size_t(M)}, k3b{size_t(M)}, pay{size_t(M)}, payb{size_t(M)};
  records_kernel<<<blocks(M), 256, 0, st>>>(d_tet.p, M, k3.p, pay.p, first.p);
  ck(cudaGetLastError(), "records");
  {
    const auto e = errors();
    if (e[kDegenerate] != ~0ull) throw MeshError("degenerate tet " + std::to_string(e[kDegenerate]));
  }
  uint32_t *k3s = nullptr, *pays = nullptr;
  sort_pairs(k3.p, k3b.p, pay.p, payb.p, M, nb, st, &k3s, &pays);
  uint32_t* pay_alt = pays == pay.p ? payb.p : pay.p;
  Buf<uint64_t> k12{size_t(M)}, k12b{size_t(M)};
  key12_kernel<<<blocks(M), 256, 0, st>>>(d_tet.p, pays, M, nb, k12.p);
  ck(cudaGetLastError(), "keys");
  uint64_t* k12s = nullptr;
  uint32_t* recs = nullptr;  // payloads in (triple, cell, local face) order
  sort_pairs(k12.p, k12b.p, pays, pay_alt, M, 2 * nb, st, &k12s, &recs);
  k12.alloc(0);
  k12b.alloc(0);
  k3.alloc(0);
  k3b.alloc(0);

  // ---- 2. interior faces and boundary candidates ----
  Buf<int> is_int{size_t(M)}, is_bnd{size_t(M)}, pos_int{size_t(M)}, pos_bnd{size_t(M)};
  runs_kernel<<<blocks(M), 256, 0, st>>>(d_tet.p, recs, M, is_int.p, is_bnd.p, first.p);
  ck(cudaGetLastError(), "runs");
  exclusive_sum(is_int.p, pos_int.p, M, st);
  exclusive_sum(is_bnd.p, pos_bnd.p, M, st);
  int last[4];
  ck(cudaMemcpyAsync(&last[0], pos_int.p + (M - 1), sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  ck(cudaMemcpyAsync(&last[1], is_int.p + (M - 1), sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  ck(cudaMemcpyAsync(&last[2], pos_bnd.p + (M - 1), sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  ck(cudaMemcpyAsync(&last[3], is_bnd.p + (M - 1), sizeof(int), cudaMemcpyDeviceToHost, st), "D2H");
  {
    const auto e = errors();
    if (e[kShared] != ~0ull) throw MeshError("a face is shared by more than two cells");
  }
  const int64_t NIF = int64_t(last[0]) + last[1], NBC = int64_t(last[2]) + last[3];
  Buf<uint64_t> ij{size_t(std::max<int64_t>(NIF, 1))}, ijb{size_t(std::max<int64_t>(NIF, 1))};
  Buf<uint32_t> ik{size_t(std::max<int64_t>(NIF, 1))}, ikb{size_t(std::max<int64_t>(NIF, 1))};
  Buf<uint32_t> btri{size_t(3 * std::max<int64_t>(NBC, 1))}, bpay{size_t(std::max<int64_t>(NBC, 1))};
  compact_kernel<<<blocks(M), 256, 0, st>>>(d_tet.p, recs, M, is_int.p, pos_int.p, is_bnd.p, pos_bnd.p, ij.p, ik.p,
                                            btri.p, bpay.p);
  ck(cudaGetLastError(), "compact");
  is_int.alloc(0);
  is_bnd.alloc(0);
  pos_int.alloc(0);
  pos_bnd.alloc(0);
  pay.alloc(0);
  payb.alloc(0);
  uint64_t* ijs = nullptr;
  uint32_t* iks = nullptr;
  if (NIF > 0) sort_pairs(ij.p, ijb.p, ik.p, ikb.p, NIF, 32 + bits_for(N), st, &ijs, &iks);  // Faces::sort: (i, j)

  // ---- 3. boundary faces from the markers (ghosts in marker order) ----
  std::vector<int64_t> tris;
  std::vector<int> patch_of;
  std::vector<int64_t> moff{0};
  // the host builder reads the markers in order: a marker with a wrong
  // triangle array is reported after any error in the markers before it
  size_t bad_marker = markers.size();
  for (size_t p = 0; p < markers.size(); p++) {
    if (markers[p].tris.size() % 3) {
      bad_marker = p;
      break;
    }
    tris.insert(tris.end(), markers[p].tris.begin(), markers[p].tris.end());
    const int64_t K = int64_t(markers[p].tris.size() / 3);
    patch_of.insert(patch_of.end(), size_t(K), int(p));
    moff.push_back(moff.back() + K);
  }
  const int64_t T = int64_t(patch_of.size());
  if (N + T >= (int64_t(1) << 32)) throw MeshError("too many cells for 32-bit indices");
  Buf<int64_t> d_tris{size_t(3 * std::max<int64_t>(T, 1))};
  Buf<int> d_patch{size_t(std::max<int64_t>(T, 1))}, cand{size_t(std::max<int64_t>(T, 1))};
  Buf<unsigned long long> first_t{size_t(std::max<int64_t>(NBC, 1))};
  Buf<uint64_t> gkey{size_t(std::max<int64_t>(T, 1))}, gkeyb{size_t(std::max<int64_t>(T, 1))};
  Buf<uint32_t> gval{size_t(std::max<int64_t>(T, 1))}, gvalb{size_t(std::max<int64_t>(T, 1))};
  uint64_t* gkeys = gkey.p;
  uint32_t* gvals = gval.p;
  if (T > 0) {
    ck(cudaMemcpyAsync(d_tris.p, tris.data(), tris.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemcpyAsync(d_patch.p, patch_of.data(), patch_of.size() * sizeof(int), cudaMemcpyHostToDevice, st), "H2D");
    ck(cudaMemsetAsync(first_t.p, 0xff, first_t.n * sizeof(unsigned long long), st), "memset");
    match_kernel<<<blocks(T), 256, 0, st>>>(d_tris.p, T, m.n_nodes, btri.p, NBC, cand.p, first_t.p, first.p);
    ck(cudaGetLastError(), "match");
    twice_kernel<<<blocks(T), 256, 0, st>>>(cand.p, T, first_t.p, first.p);
    ck(cudaGetLastError(), "twice");
    // the host builder stops at the first offending triangle in marker order
    const auto e = errors();
    const unsigned long long bad = std::min({e[kMarkerNode], e[kNoMatch], e[kTwice]});
    if (bad != ~0ull) {
      const size_t p = size_t(patch_of[size_t(bad)]);
      const std::string& name = markers[p].name;
      if (bad == e[kMarkerNode]) throw MeshError("marker '" + name + "' references a missing node");
      if (bad == e[kNoMatch])
        throw MeshError("marker '" + name + "' element " + std::to_string(int64_t(bad) - moff[p]) +
                        " matches no boundary face of a tetrahedron");
      throw MeshError("boundary face listed twice in the markers");
    }
  }
  if (bad_marker < markers.size())
    throw MeshError("marker '" + markers[bad_marker].name + "' has a wrong triangle array");
  if (T > 0) {
    gface_kernel<<<blocks(T), 256, 0, st>>>(cand.p, bpay.p, d_patch.p, T, gkey.p, gval.p);
    ck(cudaGetLastError(), "gface");
    // stable: within (patch, i) the triangles keep marker order, i.e. ghost order
    sort_pairs(gkey.p, gkeyb.p, gval.p, gvalb.p, T, 32 + bits_for(int64_t(markers.size()) + 1), st, &gkeys, &gvals);
  }
  m.n_uncovered = NBC - T;
  const int64_t NG = T, F = NIF + NG, NT = N + NG;
  m.n_faces = F;
  m.n_interior_faces = NIF;

  // ---- 4. geometry ----
  Buf<double> vol{size_t(NT)}, cen{size_t(3 * NT)};
  ck(cudaMemsetAsync(vol.p, 0, vol.n * sizeof(double), st), "memset");
  ck(cudaMemsetAsync(cen.p, 0, cen.n * sizeof(double), st), "memset");
  cell_geometry_kernel<<<blocks(N), 256, 0, st>>>(d_nodes.p, d_tet.p, N, vol.p, cen.p);
  ck(cudaGetLastError(), "cell geometry");
  Buf<uint32_t> face_i{size_t(F)}, face_j{size_t(F)}, face_nodes{size_t(3 * F)};
  Buf<int32_t> face_patch{size_t(F)};
  Buf<double> S{size_t(3 * F)}, ri{size_t(3 * F)}, rj{size_t(3 * F)}, nhat{size_t(3 * F)}, area{size_t(F)};
  const FaceOut o{face_i.p, face_j.p, face_nodes.p, face_patch.p, S.p, ri.p, rj.p, nhat.p, area.p, cen.p};
  if (NIF > 0) interior_geometry_kernel<<<blocks(NIF), 256, 0, st>>>(d_nodes.p, d_tet.p, N, ijs, iks, NIF, o);
  if (T > 0) boundary_geometry_kernel<<<blocks(T), 256, 0, st>>>(d_nodes.p, N, NIF, gkeys, gvals, d_tris.p, T, o);
  ck(cudaGetLastError(), "face geometry");
  // projected areas, per cell in face order
  Buf<double> dS{size_t(3 * N)};
  {
    const int64_t E = 2 * NIF;
    Buf<uint32_t> cell{size_t(std::max<int64_t>(E, 1))}, cellb{size_t(std::max<int64_t>(E, 1))};
    Buf<uint32_t> face{size_t(std::max<int64_t>(E, 1))}, faceb{size_t(std::max<int64_t>(E, 1))};
    Buf<int> count{size_t(N + 1)}, off{size_t(N + 1)};
    ck(cudaMemsetAsync(count.p, 0, count.n * sizeof(int), st), "memset");
    if (NIF > 0) ds_pairs_kernel<<<blocks(NIF), 256, 0, st>>>(face_i.p, face_j.p, NIF, cell.p, face.p, count.p);
    ck(cudaGetLastError(), "dS pairs");
    uint32_t *cs = cell.p, *fs = face.p;
    if (E > 0) sort_pairs(cell.p, cellb.p, face.p, faceb.p, E, bits_for(N), st, &cs, &fs);
    exclusive_sum(count.p, off.p, N + 1, st);
    ds_sum_kernel<<<blocks(N), 256, 0, st>>>(fs, off.p, N, S.p, dS.p);
    ck(cudaGetLastError(), "dS");
  }

  // ---- results to the host ----
  to_host(m.face_i, face_i.p, size_t(F), st);
  to_host(m.face_j, face_j.p, size_t(F), st);
  to_host(m.face_patch, face_patch.p, size_t(F), st);
  to_host(m.face_nodes, face_nodes.p, size_t(3 * F), st);
  to_host(m.S, S.p, size_t(3 * F), st);
  to_host(m.ri, ri.p, size_t(3 * F), st);
  to_host(m.rj, rj.p, size_t(3 * F), st);
  to_host(m.nhat, nhat.p, size_t(3 * F), st);
  to_host(m.area, area.p, size_t(F), st);
  to_host(m.vol, vol.p, size_t(NT), st);
  to_host(m.centroid, cen.p, size_t(3 * NT), st);
  to_host(m.dS, dS.p, size_t(3 * N), st);
  to_host(m.tet, d_tet.p, size_t(M), st);
  ck(cudaStreamSynchronize(st), "sync");
  for (size_t p = 0; p < markers.size(); p++) {
    Patch P;
    P.type = markers[p].type;
    P.first_face = NIF + moff[p];
    P.n_faces = moff[p + 1] - moff[p];
    P.name = markers[p].name;
    m.patches.push_back(P);
  }

  // ---- Hilbert renumbering of the centroids (mesh.cpp hilbert_renumber) ----
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t c = 0; c < N; c++)
    for (int d = 0; d < 3; d++) {
      lo[d] = std::min(lo[d], m.centroid[size_t(3 * c + d)]);
      hi[d] = std::max(hi[d], m.centroid[size_t(3 * c + d)]);
    }
  double ext = 0;
  for (int d = 0; d < 3; d++) ext = std::max(ext, hi[d] - lo[d]);
  if (!(ext > 0)) ext = 1;
  const double q = double((1u << kHilbertBits) - 1) / ext;
  {
    Buf<uint64_t> key{size_t(N)}, keyb{size_t(N)};
    Buf<uint32_t> cell{size_t(N)}, cellb{size_t(N)};
    hilbert_kernel<<<blocks(N), 256, 0, st>>>(cen.p, N, lo[0], lo[1], lo[2], q, key.p, cell.p);
    ck(cudaGetLastError(), "hilbert");
    uint64_t* ks = nullptr;
    uint32_t* order = nullptr;
    sort_pairs(key.p, keyb.p, cell.p, cellb.p, N, 3 * kHilbertBits, st, &ks, &order);  // (key, cell): stable
    std::vector<uint32_t> h;
    to_host(h, order, size_t(N), st);
    ck(cudaStreamSynchronize(st), "sync");
    m.ref_of_dev.resize(size_t(N));
    m.dev_of_ref.resize(size_t(N));
    for (int64_t k = 0; k < N; k++) {
      m.ref_of_dev[size_t(k)] = h[size_t(k)];
      m.dev_of_ref[size_t(h[size_t(k)])] = k;
    }
  }
  m.nodes = nodes;
  m.case_offsets = {0, N};
  return m;
}

}  // namespace nf

extern "C" nf_mesh* nf_mesh_from_arrays_device(int64_t n_nodes, const double* nodes, int64_t n_cells,
                                               const int64_t* tets, int n_markers, const char* const* marker_names,
                                               const int* marker_types, const int64_t* marker_offsets,
                                               const int64_t* marker_tris, int device) {
  try {
    if (n_nodes <= 0 || n_cells <= 0 || !nodes || !tets || n_markers < 0 ||
        (n_markers && (!marker_names || !marker_types || !marker_offsets || !marker_tris)))
      throw MeshError("invalid arguments");
    int prev = 0;
    ck(cudaGetDevice(&prev), "cudaGetDevice");
    if (device >= 0) ck(cudaSetDevice(device), "cudaSetDevice");
    struct Restore {
      int dev;
      ~Restore() { cudaSetDevice(dev); }
    } restore{prev};
    std::vector<double> nd(nodes, nodes + 3 * n_nodes);
    std::vector<int64_t> tt(tets, tets + 4 * n_cells);
    std::vector<nf::MarkerInput> mk(static_cast<size_t>(n_markers));
    for (int i = 0; i < n_markers; i++) {
      mk[size_t(i)].name = marker_names[i];
      mk[size_t(i)].type = marker_types[i];
      const int64_t b = marker_offsets[i], e = marker_offsets[i + 1];
      if (e < b) throw MeshError("marker offsets must be non-decreasing");
      mk[size_t(i)].tris.assign(marker_tris + 3 * b, marker_tris + 3 * e);
    }
    auto* h = new nf_mesh;
    h->m = nf::build_mesh_device(nd, tt, mk);
    return h;
  } catch (const CudaFail& e) {
    nf::set_last_error_text(std::string("Error creating grid on the device: ") + e.what());
    return nullptr;
  } catch (const std::exception& e) {
    nf::set_last_error_text(std::string("Error creating grid:\n") + e.what());
    return nullptr;
  }
}
