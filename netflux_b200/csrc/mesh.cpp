// Host-side construction of the face-based grid.
//
// Follows geometry::PrimalGrid::read_su2_mesh (PrimalGrid.cpp:140-244) and
// geometry::FV_Grid (FV_Grid.cpp:21-205) in what they produce — face order,
// orientation and every floating-point operation of the geometry — but finds
// faces by sorting packed node keys instead of a std::map, and adds the
// Hilbert-curve renumbering the device layout uses.
//
// Compiled with -ffp-contract=off: the geometry must round exactly as the
// reference's (no fused multiply-add on the x86-64 baseline it targets).
#include "mesh.hpp"
#include "mesh_common.hpp"

#include "../../include/netflux_b200.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <atomic>
#include <thread>
#include <unordered_map>

namespace nf {
namespace {

// ---- host threads for the large loops and sorts. Every parallel loop writes
// disjoint elements and every sorted sequence has distinct keys, so the mesh
// is the same, bit for bit, whatever the thread count. ----
// NETFLUX_B200_HOST_THREADS (1..64) overrides the thread count (tests use 1
// to check that the parallel build gives the serial one's mesh); a cap set by
// nf_set_host_threads (callers that build several meshes at once on their own
// threads) bounds the default.
std::atomic<int> g_thread_cap{0};

int host_threads(size_t n) {
  if (n < (size_t(1) << 16)) return 1;
  if (const char* e = std::getenv("NETFLUX_B200_HOST_THREADS")) {
    const int t = std::atoi(e);
    if (t >= 1 && t <= 64) return t;
  }
  const unsigned hw = std::thread::hardware_concurrency();
  int t = int(std::min(16u, std::max(1u, hw)));
  const int cap = g_thread_cap.load(std::memory_order_relaxed);
  if (cap > 0) t = std::min(t, cap);
  return t;
}

// fn(begin, end) over [0, n) in contiguous chunks; fn must not throw
template <class F>
void parallel_for(int64_t n, F&& fn) {
  const int T = host_threads(size_t(n));
  if (T == 1) {
    fn(int64_t(0), n);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < T; t++) {
    const int64_t b = n * t / T, e = n * (t + 1) / T;
    th.emplace_back([&fn, b, e] { fn(b, e); });
  }
  for (auto& x : th) x.join();
}

// std::sort of chunks in parallel, then pairwise merges; cmp must be a strict
// order under which no two elements are equal (so the result is unique)
template <class T, class Cmp>
void parallel_sort(std::vector<T>& v, Cmp cmp) {
  const int P = host_threads(v.size());
  if (P == 1) {
    std::sort(v.begin(), v.end(), cmp);
    return;
  }
  std::vector<size_t> cut(size_t(P) + 1);
  for (int t = 0; t <= P; t++) cut[size_t(t)] = v.size() * size_t(t) / size_t(P);
  parallel_for(P, [&](int64_t b, int64_t e) {
    for (int64_t t = b; t < e; t++) std::sort(v.begin() + cut[size_t(t)], v.begin() + cut[size_t(t) + 1], cmp);
  });
  for (int w = 1; w < P; w *= 2) {
    std::vector<std::thread> th;
    for (int t = 0; t + w < P; t += 2 * w) {
      const size_t b = cut[size_t(t)], mid = cut[size_t(t + w)], e = cut[size_t(std::min(t + 2 * w, P))];
      th.emplace_back([&v, &cmp, b, mid, e] { std::inplace_merge(v.begin() + b, v.begin() + mid, v.begin() + e, cmp); });
    }
    for (auto& x : th) x.join();
  }
}

using V3 = std::array<double, 3>;

inline V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 add(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 scale(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
// Eigen's cross (a1 b2 - a2 b1, a2 b0 - a0 b2, a0 b1 - a1 b0).
inline V3 cross(const V3& a, const V3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
// Reductions summed left to right: (a0 b0 + a1 b1) + a2 b2.
inline double dot(const V3& a, const V3& b) { return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]; }

inline V3 node(const std::vector<double>& nodes, int64_t n) {
  return {nodes[3 * n], nodes[3 * n + 1], nodes[3 * n + 2]};
}

struct FaceKey {
  uint64_t hi, lo;  // sorted node ids (a<<32|b, c<<32|payload)
};

// Hilbert order of the cells [begin, end) (reference numbering) by centroid.
void hilbert_renumber(Mesh& m, int64_t begin, int64_t end) {
  const int bits = kHilbertBits;
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t c = begin; c < end; c++)
    for (int d = 0; d < 3; d++) {
      lo[d] = std::min(lo[d], m.centroid[3 * c + d]);
      hi[d] = std::max(hi[d], m.centroid[3 * c + d]);
    }
  double ext = 0;
  for (int d = 0; d < 3; d++) ext = std::max(ext, hi[d] - lo[d]);
  if (!(ext > 0)) ext = 1;
  const double q = double((1u << bits) - 1) / ext;
  std::vector<std::pair<uint64_t, int64_t>> keys(size_t(end - begin));
  parallel_for(end - begin, [&](int64_t k0, int64_t k1) {
    for (int64_t c = begin + k0; c < begin + k1; c++) {
      uint32_t u[3];
      for (int d = 0; d < 3; d++) {
        double v = (m.centroid[3 * c + d] - lo[d]) * q;
        u[d] = uint32_t(std::min(std::max(v, 0.0), double((1u << bits) - 1)));
      }
      keys[size_t(c - begin)] = {hilbert3(u[0], u[1], u[2], bits), c};
    }
  });
  parallel_sort(keys, [](const std::pair<uint64_t, int64_t>& x, const std::pair<uint64_t, int64_t>& y) {
    return x < y;  // (key, cell): distinct
  });
  for (int64_t k = 0; k < end - begin; k++) {
    m.ref_of_dev[size_t(begin + k)] = keys[size_t(k)].second;
    m.dev_of_ref[size_t(keys[size_t(k)].second)] = begin + k;
  }
}

}  // namespace

Mesh build_mesh(const std::vector<double>& nodes, const std::vector<int64_t>& tets_in,
                const std::vector<MarkerInput>& markers) {
  Mesh m;
  if (nodes.size() % 3 || tets_in.size() % 4) throw MeshError("node or tet array has a wrong length");
  m.n_nodes = int64_t(nodes.size() / 3);
  const int64_t N = int64_t(tets_in.size() / 4);
  m.n_cells = N;
  if (N == 0) throw MeshError("mesh has no volume elements");
  if (m.n_nodes >= (int64_t(1) << 32) || N >= (int64_t(1) << 31))
    throw MeshError("mesh too large for 32-bit node / 31-bit cell indices");

  // salome_to_vtk_connectivity (GeometryUtilities.cpp:452-455): swap 1 <-> 2.
  std::vector<uint32_t> tet(size_t(4 * N));
  for (int64_t c = 0; c < N; c++) {
    const int64_t* t = &tets_in[size_t(4 * c)];
    const int64_t v[4] = {t[0], t[2], t[1], t[3]};
    for (int q = 0; q < 4; q++) {
      if (v[q] < 0 || v[q] >= m.n_nodes) throw MeshError("tet " + std::to_string(c) + " references a missing node");
      tet[size_t(4 * c + q)] = uint32_t(v[q]);
    }
  }

  // ---- face matching by sort (replaces the std::map of FV_Grid.cpp:38-64) ----
  // the low 32 bits of a key carry (cell << 2 | local face)
  if (N >= (int64_t(1) << 30)) throw MeshError("mesh too large (>= 2^30 cells)");
  std::vector<FaceKey> rec(size_t(4 * N));
  for (int64_t c = 0; c < N; c++)
    for (int k = 0; k < 4; k++) {
      uint32_t a = tet[size_t(4 * c + kTetFace[k][0])], b = tet[size_t(4 * c + kTetFace[k][1])],
               d = tet[size_t(4 * c + kTetFace[k][2])];
      sort3(a, b, d);
      if (a == b || b == d) throw MeshError("degenerate tet " + std::to_string(c));
      // payload: cell (31 bits) and local face (2 bits) in the low 32 bits
      rec[size_t(4 * c + k)] = {(uint64_t(a) << 32) | b, (uint64_t(d) << 32) | (uint64_t(c) << 2 | uint64_t(k))};
    }
  parallel_sort(rec, [](const FaceKey& x, const FaceKey& y) {  // lo carries (cell, face): distinct
    return x.hi != y.hi ? x.hi < y.hi : x.lo < y.lo;
  });

  struct IFace {
    uint32_t i, j;
    uint8_t k;  // local face of cell i (its node order defines the face element)
  };
  std::vector<IFace> interior;
  interior.reserve(size_t(2 * N + 16));
  struct BFace {
    uint64_t hi, lo_nodes;  // key
    uint32_t cell;
    uint8_t k;
  };
  std::vector<BFace> bcand;
  const uint64_t kNodeMask = ~uint64_t(0xffffffffu);
  for (size_t r = 0; r < rec.size();) {
    size_t e = r + 1;
    while (e < rec.size() && rec[e].hi == rec[r].hi && (rec[e].lo & kNodeMask) == (rec[r].lo & kNodeMask)) e++;
    if (e - r > 2) throw MeshError("a face is shared by more than two cells");
    auto cell_of = [&](size_t q) { return uint32_t((rec[q].lo & 0xffffffffu) >> 2); };
    auto k_of = [&](size_t q) { return uint8_t(rec[q].lo & 3u); };
    if (e - r == 2) {
      // sorted by payload: the first record has the lower cell, which is the
      // cell that discovered the face first in the reference's cell loop
      interior.push_back({cell_of(r), cell_of(r + 1), k_of(r)});
    } else {
      bcand.push_back({rec[r].hi, rec[r].lo & kNodeMask, cell_of(r), k_of(r)});
    }
    r = e;
  }
  rec.clear();
  rec.shrink_to_fit();
  parallel_sort(interior, [](const IFace& x, const IFace& y) {
    return x.i != y.i ? x.i < y.i : x.j < y.j;  // Faces::sort (GeometryUtilities.cpp:484-513); two tets share one face at most
  });

  // ---- boundary faces: markers in file order, ghosts numbered in that order ----
  std::unordered_map<uint64_t, std::vector<size_t>> bindex;  // hash of key -> candidates
  bindex.reserve(bcand.size() * 2 + 1);
  auto hkey = [](uint64_t hi, uint64_t lo) { return hi * 0x9E3779B97F4A7C15ull ^ (lo >> 32); };
  for (size_t q = 0; q < bcand.size(); q++) bindex[hkey(bcand[q].hi, bcand[q].lo_nodes)].push_back(q);
  std::vector<uint8_t> bused(bcand.size(), 0);

  struct GFace {
    uint32_t i, ghost;
    int64_t marker_elem;  // index into the marker's triangle list
  };
  std::vector<std::vector<GFace>> pfaces(markers.size());
  int64_t j_ghost = N;
  for (size_t p = 0; p < markers.size(); p++) {
    const auto& mk = markers[p];
    if (mk.tris.size() % 3) throw MeshError("marker '" + mk.name + "' has a wrong triangle array");
    const int64_t K = int64_t(mk.tris.size() / 3);
    for (int64_t t = 0; t < K; t++) {
      uint32_t v[3];
      for (int q = 0; q < 3; q++) {
        int64_t n = mk.tris[size_t(3 * t + q)];
        if (n < 0 || n >= m.n_nodes) throw MeshError("marker '" + mk.name + "' references a missing node");
        v[q] = uint32_t(n);
      }
      uint32_t a = v[0], b = v[1], d = v[2];
      sort3(a, b, d);
      const uint64_t hi = (uint64_t(a) << 32) | b, lo = uint64_t(d) << 32;
      auto it = bindex.find(hkey(hi, lo));
      size_t hit = size_t(-1);
      if (it != bindex.end())
        for (size_t q : it->second)
          if (bcand[q].hi == hi && bcand[q].lo_nodes == lo) hit = q;
      if (hit == size_t(-1))
        throw MeshError("marker '" + mk.name + "' element " + std::to_string(t) +
                        " matches no boundary face of a tetrahedron");
      if (bused[hit]) throw MeshError("boundary face listed twice in the markers");
      bused[hit] = 1;
      pfaces[p].push_back({bcand[hit].cell, uint32_t(j_ghost), t});
      j_ghost++;
    }
    std::sort(pfaces[p].begin(), pfaces[p].end(), [](const GFace& x, const GFace& y) {
      return x.i != y.i ? x.i < y.i : x.ghost < y.ghost;
    });
  }
  for (uint8_t u : bused) m.n_uncovered += u ? 0 : 1;
  const int64_t NG = j_ghost - N;
  const int64_t NIF = int64_t(interior.size());
  const int64_t F = NIF + NG;
  if (N + NG >= (int64_t(1) << 32)) throw MeshError("too many cells for 32-bit indices");
  m.n_faces = F;
  m.n_interior_faces = NIF;

  // ---- cell geometry (GeometryUtilities.cpp:289-316) ----
  const int64_t NT = N + NG;
  m.vol.assign(size_t(NT), 0.0);
  m.centroid.assign(size_t(3 * NT), 0.0);
  for (int64_t c = 0; c < N; c++) {
    const V3 n0 = node(nodes, tet[size_t(4 * c)]), n1 = node(nodes, tet[size_t(4 * c + 1)]),
             n2 = node(nodes, tet[size_t(4 * c + 2)]), n3 = node(nodes, tet[size_t(4 * c + 3)]);
    const V3 ab = sub(n1, n0), ac = sub(n2, n0), ad = sub(n3, n0);
    m.vol[size_t(c)] = dot(cross(ab, ac), ad) / 6;
    const V3 cen = scale(1.0 / 4, add(add(add(n0, n1), n2), n3));
    for (int d = 0; d < 3; d++) m.centroid[size_t(3 * c + d)] = cen[d];
  }

  // ---- face list and face geometry (FV_Grid.cpp:154-205, 237-267) ----
  m.face_i.resize(static_cast<size_t>(F));
  m.face_j.resize(static_cast<size_t>(F));
  m.face_patch.assign(size_t(F), -1);
  m.S.resize(size_t(3 * F));
  m.ri.resize(size_t(3 * F));
  m.rj.resize(size_t(3 * F));
  m.nhat.resize(size_t(3 * F));
  m.area.resize(static_cast<size_t>(F));
  m.face_nodes.resize(size_t(3 * F));
  auto face_geometry = [&](int64_t f, uint32_t i, uint32_t j, const uint32_t fn[3]) {
    for (int q = 0; q < 3; q++) m.face_nodes[size_t(3 * f + q)] = fn[q];
    const V3 n0 = node(nodes, fn[0]), n1 = node(nodes, fn[1]), n2 = node(nodes, fn[2]);
    V3 S = scale(0.5, cross(sub(n1, n0), sub(n2, n0)));  // triangle_calc_face_normal
    const V3 fc = {((n0[0] + n1[0]) + n2[0]) / 3, ((n0[1] + n1[1]) + n2[1]) / 3, ((n0[2] + n1[2]) + n2[2]) / 3};
    const V3 ci = {m.centroid[3 * size_t(i)], m.centroid[3 * size_t(i) + 1], m.centroid[3 * size_t(i) + 2]};
    if (j >= uint32_t(N)) {  // calc_ghost_centroid: 2 * face centroid - centroid_i
      const V3 cg = sub(scale(2, fc), ci);
      for (int d = 0; d < 3; d++) m.centroid[3 * size_t(j) + d] = cg[d];
    }
    const V3 cj = {m.centroid[3 * size_t(j)], m.centroid[3 * size_t(j) + 1], m.centroid[3 * size_t(j) + 2]};
    if (dot(S, sub(cj, ci)) < 0) S = scale(-1, S);  // point from i to j
    const V3 r_i = sub(fc, ci), r_j = sub(fc, cj);
    const double z = dot(S, S);
    const double a = std::sqrt(z);
    for (int d = 0; d < 3; d++) {
      m.S[size_t(3 * f + d)] = S[d];
      m.ri[size_t(3 * f + d)] = r_i[d];
      m.rj[size_t(3 * f + d)] = r_j[d];
      m.nhat[size_t(3 * f + d)] = z > 0 ? S[d] / a : S[d];  // Eigen normalized()
    }
    m.area[size_t(f)] = a;
    m.face_i[size_t(f)] = i;
    m.face_j[size_t(f)] = j;
  };
  // interior faces write only their own face's entries (j < N: no ghost centroid)
  parallel_for(NIF, [&](int64_t f0, int64_t f1) {
    for (int64_t f = f0; f < f1; f++) {
      const IFace& x = interior[size_t(f)];
      uint32_t fn[3];
      for (int q = 0; q < 3; q++) fn[q] = tet[size_t(4 * x.i + kTetFace[x.k][q])];
      face_geometry(f, x.i, x.j, fn);
    }
  });
  int64_t f = NIF;
  for (size_t p = 0; p < markers.size(); p++) {
    Patch P;
    P.type = markers[p].type;
    P.first_face = f;
    P.n_faces = int64_t(pfaces[p].size());
    P.name = markers[p].name;
    m.patches.push_back(P);
    for (const GFace& g : pfaces[p]) {
      uint32_t fn[3];
      for (int q = 0; q < 3; q++) fn[q] = uint32_t(markers[p].tris[size_t(3 * g.marker_elem + q)]);
      face_geometry(f, g.i, g.ghost, fn);
      m.face_patch[size_t(f)] = int32_t(p);
      f++;
    }
  }

  // ---- Delta S (calc_Delta_S, Solver.cpp:276-298): interior faces only ----
  m.dS.assign(size_t(3 * N), 0.0);
  for (int64_t g = 0; g < NIF; g++) {
    for (int d = 0; d < 3; d++) {
      const double tmp = 0.5 * std::abs(m.S[size_t(3 * g + d)]);
      m.dS[3 * size_t(m.face_i[size_t(g)]) + d] += tmp;
      m.dS[3 * size_t(m.face_j[size_t(g)]) + d] += tmp;
    }
  }

  m.nodes = nodes;
  m.tet = std::move(tet);
  m.dev_of_ref.resize(static_cast<size_t>(N));
  m.ref_of_dev.resize(static_cast<size_t>(N));
  m.case_offsets = {0, N};
  hilbert_renumber(m, 0, N);
  return m;
}

// ---------------------------------------------------------------------------
// SU2 reader (PrimalGrid.cpp:140-244)
// ---------------------------------------------------------------------------
namespace {

struct Cursor {
  const char* p;
  const char* end;
  void skip_ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
  }
  std::string token() {
    skip_ws();
    const char* s = p;
    while (p < end && !(*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    return std::string(s, p);
  }
  long long integer(const char* what) {
    skip_ws();
    char* e = nullptr;
    long long v = std::strtoll(p, &e, 10);
    if (e == p) throw MeshError(std::string("expected an integer for ") + what);
    p = e;
    return v;
  }
  double real() {
    skip_ws();
    char* e = nullptr;
    double v = std::strtod(p, &e);  // correctly rounded, as istream >> double
    if (e == p) throw MeshError("expected a number in the point list");
    p = e;
    return v;
  }
  void skip_line() {
    while (p < end && *p != '\n') p++;
  }
};

void expect(const std::string& got, const char* want) {
  if (got != want)
    throw MeshError("symbol '" + got + "' parsed instead of correct symbol '" + want + "'");
}

}  // namespace

Mesh read_su2(const std::string& path, const std::vector<std::string>& names, const std::vector<int>& types) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) throw MeshError("Couldn't open the mesh file: " + path);
  std::string buf(size_t(in.tellg()), '\0');
  in.seekg(0);
  in.read(&buf[0], std::streamsize(buf.size()));
  Cursor cur{buf.data(), buf.data() + buf.size()};

  expect(cur.token(), "NDIME=");
  if (cur.integer("NDIME") != 3) throw MeshError("Only three dimensions (NDIME=3) is accepted");
  expect(cur.token(), "NELEM=");
  const long long NE = cur.integer("NELEM");
  if (NE < 0) throw MeshError("negative NELEM");
  std::vector<int64_t> tets;
  tets.reserve(size_t(4 * NE));
  for (long long e = 0; e < NE; e++) {
    long long id = cur.integer("element type");
    if (id != 10) {
      if (id == 12 || id == 13 || id == 14)
        throw MeshError("only tetrahedral meshes are supported (element type " + std::to_string(id) + ")");
      throw MeshError("Illegal su2 volume element identifier (" + std::to_string(id) + ")");
    }
    for (int q = 0; q < 4; q++) tets.push_back(cur.integer("tet node"));
    cur.skip_line();
  }
  expect(cur.token(), "NPOIN=");
  const long long NP = cur.integer("NPOIN");
  std::vector<double> nodes(size_t(3 * NP));
  for (long long n = 0; n < 3 * NP; n++) nodes[size_t(n)] = cur.real();  // exactly x y z per point
  expect(cur.token(), "NMARK=");
  const long long NM = cur.integer("NMARK");
  std::vector<MarkerInput> markers(static_cast<size_t>(NM));
  for (long long k = 0; k < NM; k++) {
    expect(cur.token(), "MARKER_TAG=");
    markers[size_t(k)].name = cur.token();
    auto it = std::find(names.begin(), names.end(), markers[size_t(k)].name);
    if (it == names.end())
      throw MeshError("Patch with name '" + markers[size_t(k)].name + "' is not named in input file");
    markers[size_t(k)].type = types[size_t(it - names.begin())];
    expect(cur.token(), "MARKER_ELEMS=");
    const long long ME = cur.integer("MARKER_ELEMS");
    for (long long e = 0; e < ME; e++) {
      long long id = cur.integer("marker element type");
      if (id != 5) {
        if (id == 9) throw MeshError("only triangular boundary elements are supported");
        throw MeshError("Illegal su2 element identifier (" + std::to_string(id) + ")");
      }
      for (int q = 0; q < 3; q++) markers[size_t(k)].tris.push_back(cur.integer("triangle node"));
      cur.skip_line();
    }
  }
  return build_mesh(nodes, tets, markers);
}

// ---------------------------------------------------------------------------
// Batched meshes: concatenation with per-case offsets
// ---------------------------------------------------------------------------
Mesh concat_meshes(const std::vector<const Mesh*>& parts) {
  if (parts.empty()) throw MeshError("no meshes to concatenate");
  Mesh m;
  int64_t NC = 0, NG = 0, NF = 0;
  for (const Mesh* p : parts) {
    NC += p->n_cells;
    NG += p->n_ghost();
    NF += p->n_faces;
    m.n_nodes += p->n_nodes;
    m.n_uncovered += p->n_uncovered;
  }
  if (NC + NG >= (int64_t(1) << 31)) throw MeshError("batched mesh too large");
  m.n_cells = NC;
  m.n_faces = NF;
  m.vol.assign(size_t(NC + NG), 0.0);
  m.centroid.assign(size_t(3 * (NC + NG)), 0.0);
  m.dS.reserve(size_t(3 * NC));
  m.case_offsets.assign(1, 0);
  int64_t cell0 = 0, ghost0 = NC, face0 = 0, node0 = 0;
  int case_index = 0;
  for (const Mesh* p : parts) {
    m.nodes.insert(m.nodes.end(), p->nodes.begin(), p->nodes.end());
    for (uint32_t v : p->tet) m.tet.push_back(uint32_t(node0 + v));
    for (uint32_t v : p->face_nodes) m.face_nodes.push_back(uint32_t(node0 + v));
    for (int c = 0; c < p->n_cases(); c++) m.case_offsets.push_back(cell0 + p->case_offsets[size_t(c + 1)]);
    for (int64_t f = 0; f < p->n_faces; f++) {
      const uint32_t i = p->face_i[size_t(f)], j = p->face_j[size_t(f)];
      m.face_i.push_back(uint32_t(cell0 + i));
      m.face_j.push_back(j < uint32_t(p->n_cells) ? uint32_t(cell0 + j) : uint32_t(ghost0 + (j - p->n_cells)));
      const int32_t fp = p->face_patch[size_t(f)];
      m.face_patch.push_back(fp < 0 ? -1 : int32_t(fp + m.patches.size()));
      m.area.push_back(p->area[size_t(f)]);
      for (int d = 0; d < 3; d++) {
        m.S.push_back(p->S[size_t(3 * f + d)]);
        m.ri.push_back(p->ri[size_t(3 * f + d)]);
        m.rj.push_back(p->rj[size_t(3 * f + d)]);
        m.nhat.push_back(p->nhat[size_t(3 * f + d)]);
      }
    }
    for (int64_t c = 0; c < p->n_cells; c++) {
      m.vol[size_t(cell0 + c)] = p->vol[size_t(c)];
      for (int d = 0; d < 3; d++) m.centroid[size_t(3 * (cell0 + c) + d)] = p->centroid[size_t(3 * c + d)];
    }
    for (int64_t g = 0; g < p->n_ghost(); g++)
      for (int d = 0; d < 3; d++)
        m.centroid[size_t(3 * (ghost0 + g) + d)] = p->centroid[size_t(3 * (p->n_cells + g) + d)];
    m.dS.insert(m.dS.end(), p->dS.begin(), p->dS.end());
    for (const Patch& P : p->patches) {
      Patch Q = P;
      Q.first_face += face0;
      Q.case_index += case_index;
      m.patches.push_back(Q);
    }
    for (int64_t c = 0; c < p->n_cells; c++) {
      m.dev_of_ref.push_back(cell0 + p->dev_of_ref[size_t(c)]);
      m.ref_of_dev.push_back(cell0 + p->ref_of_dev[size_t(c)]);
    }
    cell0 += p->n_cells;
    ghost0 += p->n_ghost();
    face0 += p->n_faces;
    node0 += p->n_nodes;
    case_index += p->n_cases();
  }
  // interior-face count is per case; the batched face list interleaves them,
  // so n_interior_faces counts all interior faces
  for (const Mesh* p : parts) m.n_interior_faces += p->n_interior_faces;
  return m;
}

}  // namespace nf

extern "C" int nf_set_host_threads(int n) {
  if (n < 0 || n > 64) return NF_ERR_ARG;
  nf::g_thread_cap.store(n, std::memory_order_relaxed);
  return NF_OK;
}
