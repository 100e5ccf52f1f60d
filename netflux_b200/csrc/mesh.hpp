// Host-side face-based grid: the structure-of-arrays mesh the device kernels
// consume, built once from an SU2 file or from node/tet/marker arrays.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace nf {

struct MeshError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct Patch {
  int type = 0;             // NF_BC_*
  int64_t first_face = 0;   // reference face index of the first face
  int64_t n_faces = 0;
  int case_index = 0;
  std::string name;
};

// Face-based grid in the reference's numbering and order (FV_Grid), plus the
// space-filling-curve renumbering used on the device.
struct Mesh {
  int64_t n_nodes = 0;
  int64_t n_cells = 0;           // interior cells
  int64_t n_faces = 0;           // all faces
  int64_t n_interior_faces = 0;
  int64_t n_uncovered = 0;       // boundary tet faces listed by no marker (dropped)

  // Per face, reference order: interior faces sorted by (i, j), then every
  // patch's faces sorted by (i, ghost). face_j >= n_cells marks a ghost.
  std::vector<uint32_t> face_i, face_j;
  std::vector<int32_t> face_patch;  // -1 for interior faces
  std::vector<double> S, ri, rj;    // [F][3]
  std::vector<double> nhat, area;   // S.normalized(), S.norm(): [F][3], [F]
  // Per cell incl. ghosts: volume (0 for ghosts) and centroid.
  std::vector<double> vol, centroid;
  std::vector<double> dS;           // [n_cells][3], Blazek's projected areas

  // Primal data kept for the node-based geometry of the fast kernels.
  std::vector<double> nodes;        // [n_nodes][3]
  std::vector<uint32_t> tet;        // [n_cells][4] node ids after the reader's 1<->2 swap
  std::vector<uint32_t> face_nodes; // [F][3] node ids of each face element
  std::vector<Patch> patches;

  // Device numbering (Hilbert order of centroids, per case).
  std::vector<int64_t> dev_of_ref, ref_of_dev;
  std::vector<int64_t> case_offsets{0, 0};  // [n_cases + 1], contiguous cell ranges

  int n_cases() const { return int(case_offsets.size()) - 1; }
  int64_t n_ghost() const { return n_faces - n_interior_faces; }
};

struct MarkerInput {
  std::string name;
  int type = 0;
  std::vector<int64_t> tris;  // [K][3]
};

// tets: node ids as listed in an SU2 file (the reader swaps nodes 1 and 2).
Mesh build_mesh(const std::vector<double>& nodes, const std::vector<int64_t>& tets,
                const std::vector<MarkerInput>& markers);

// Parse an SU2 file; names/types give every marker's boundary type.
Mesh read_su2(const std::string& path, const std::vector<std::string>& names, const std::vector<int>& types);

Mesh concat_meshes(const std::vector<const Mesh*>& parts);

// The same Mesh, bit for bit, built on the current CUDA device
// (mesh_device.cu): face matching, orderings, geometry and the Hilbert
// renumbering run as kernels; the result is copied back to the host.
Mesh build_mesh_device(const std::vector<double>& nodes, const std::vector<int64_t>& tets,
                       const std::vector<MarkerInput>& markers);

}  // namespace nf

// The C ABI's opaque mesh handle (include/netflux_b200.h).
struct nf_mesh {
  nf::Mesh m;
};
