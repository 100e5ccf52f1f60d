// Pieces of the face-grid construction shared by the host builder
// (mesh.cpp) and the device builder (mesh_device.cu): the local faces of a
// tetrahedron, the sorted node triple that keys a face, and the 3-D Hilbert
// index of the cell renumbering.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define NF_HD __host__ __device__
#else
#define NF_HD
#endif

namespace nf {

// Local faces of a tetrahedron, get_face_element_k_of_tetrahedron
// (GeometryUtilities.cpp:71-101).
constexpr int kTetFace[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
// kTetFace[k][q] as a function (face k leaves out vertex 3 - k), usable in
// device code with run-time indices
NF_HD inline int tet_face(int k, int q) { return q < 3 - k ? q : q + 1; }

NF_HD inline void sort3(uint32_t& a, uint32_t& b, uint32_t& c) {
  uint32_t t;
  if (a > b) { t = a; a = b; b = t; }
  if (b > c) { t = b; b = c; c = t; }
  if (a > b) { t = a; a = b; b = t; }
}

// ---- 3-D Hilbert index (Skilling, "Programming the Hilbert curve", AIP
// Conf. Proc. 707, 2004: axes -> transposed index, then bit interleave) ----
NF_HD inline uint64_t hilbert3(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t M = 1u << (bits - 1);
  for (uint32_t Q = M; Q > 1; Q >>= 1) {  // inverse undo
    const uint32_t P = Q - 1;
    for (int i = 0; i < 3; i++) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        uint32_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  for (int i = 1; i < 3; i++) X[i] ^= X[i - 1];  // Gray encode
  uint32_t t = 0;
  for (uint32_t Q = M; Q > 1; Q >>= 1)
    if (X[2] & Q) t ^= Q - 1;
  for (int i = 0; i < 3; i++) X[i] ^= t;
  uint64_t h = 0;
  for (int b = bits - 1; b >= 0; b--)
    for (int i = 0; i < 3; i++) h = (h << 1) | ((X[i] >> b) & 1u);
  return h;
}

// Bits per axis of the Hilbert keys.
constexpr int kHilbertBits = 21;

}  // namespace nf
