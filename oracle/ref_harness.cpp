// Driver for the NetFlux reference solver, compiled from the unmodified
// reference sources (see oracle/Makefile).
//
// ORACLE-ONLY TEST INFRASTRUCTURE: used by tests/ and bench.py's CPU baseline
// leg as the checker. Never part of the product path.
//
// It does what NetFlux's Driver::solve does (Driver.cpp:24-61: calc_timestep,
// then step, per time step) on a case directory holding mesh.su2 + input.yml,
// with three additions a test needs:
//   * an initial state read from <case>/U0.bin (AoS double[N][5], reference
//     cell order) instead of the freestream. The primitives are set to
//     cons_to_prim(U0) as well, because calc_timestep reads the primitives of
//     the last evaluated stage (Solver.cpp:250) and at step 0 those must match
//     the initial state.
//   * raw binary dumps of the state and of the last stage's intermediates
//     (primitives incl. ghosts, gradient, limiter, flux balance) and of the
//     face-based grid, for parity checks;
//   * a wall-clock timing of the step loop alone (mesh build excluded).
//
// Usage: nf_ref <case_dir> <out_dir> [--steps N] [--geometry] [--time] [--quiet]
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "Solver.hpp"
#include "geometry/FV_Grid.hpp"
#include "geometry/PrimalGrid.hpp"

namespace {

class HarnessSolver : public EulerSolver {
 public:
  using EulerSolver::EulerSolver;

  // Replace the freestream initial state (SolverData.cpp:50-58) by U0.
  void set_initial_state(const std::vector<double>& U0, Index n_cells) {
    VecField& U = solver_data->get_solution();
    VecField& U_old = solver_data->get_solution_old();
    VecField& V = solver_data->get_primvars();
    for (Index i = 0; i < n_cells; i++) {
      for (int k = 0; k < 5; k++) {
        U(i, k) = U0[5 * size_t(i) + k];
        U_old(i, k) = U0[5 * size_t(i) + k];
      }
      const EulerVecMap u = U.get_variable<EulerVec>(i);
      EulerVecMap v = V.get_variable<EulerVec>(i);
      EulerEqs::cons_to_prim(u, v);
    }
  }
};

template <typename T>
void write_raw(const std::string& path, const T* data, size_t n) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot write " + path);
  if (n && std::fwrite(data, sizeof(T), n, f) != n) throw std::runtime_error("short write " + path);
  std::fclose(f);
}

std::vector<double> read_doubles(const std::string& path) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) return {};
  std::streamsize bytes = in.tellg();
  in.seekg(0);
  std::vector<double> v(size_t(bytes) / sizeof(double));
  in.read(reinterpret_cast<char*>(v.data()), bytes);
  return v;
}

void dump_field(const std::string& path, const VecField& f) {
  std::vector<double> out(size_t(f.size()) * f.rows());
  for (Index i = 0; i < f.size(); i++)
    for (Index k = 0; k < f.rows(); k++) out[size_t(i) * f.rows() + k] = f(i, k);
  write_raw(path, out.data(), out.size());
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s <case_dir> <out_dir> [--steps N] [--geometry] [--time] [--quiet]\n", argv[0]);
    return 2;
  }
  std::string case_dir = argv[1], out_dir = argv[2];
  long steps = -1;
  bool geometry = false, timing = false, quiet = false;
  for (int a = 3; a < argc; a++) {
    if (!std::strcmp(argv[a], "--steps") && a + 1 < argc) steps = std::atol(argv[++a]);
    else if (!std::strcmp(argv[a], "--geometry")) geometry = true;
    else if (!std::strcmp(argv[a], "--time")) timing = true;
    else if (!std::strcmp(argv[a], "--quiet")) quiet = true;
  }
  if (quiet) std::cout.setstate(std::ios::failbit);
  if (out_dir.back() != '/') out_dir += '/';
  try {
    Config config{case_dir};
    geometry::PrimalGrid primal{config};
    geometry::FV_Grid fv{config, primal};
    HarnessSolver solver{config, primal, fv};
    const Index NC = config.get_N_INTERIOR_CELLS();
    const Index NT = config.get_N_TOTAL_CELLS();
    const Index NF = config.get_N_TOTAL_FACES();

    std::string cd = case_dir.back() == '/' ? case_dir : case_dir + "/";
    std::vector<double> U0 = read_doubles(cd + "U0.bin");
    if (!U0.empty()) {
      if (U0.size() != size_t(NC) * 5) throw std::runtime_error("U0.bin has the wrong size");
      solver.set_initial_state(U0, NC);
    }

    if (geometry) {
      const auto& faces = fv.get_faces();
      const auto& cells = fv.get_cells();
      std::vector<uint32_t> ij(2 * size_t(NF));
      std::vector<double> S(3 * size_t(NF)), ri(3 * size_t(NF)), rj(3 * size_t(NF));
      for (Index f = 0; f < NF; f++) {
        ij[2 * f] = faces.get_cell_i(f);
        ij[2 * f + 1] = faces.get_cell_j(f);
        for (int d = 0; d < 3; d++) {
          S[3 * f + d] = faces.get_face_normal(f)[d];
          ri[3 * f + d] = faces.get_centroid_to_face_i(f)[d];
          rj[3 * f + d] = faces.get_centroid_to_face_j(f)[d];
        }
      }
      std::vector<double> vol(NT), cen(3 * size_t(NT));
      for (Index c = 0; c < NT; c++) {
        vol[c] = cells.get_cell_volume(c);
        for (int d = 0; d < 3; d++) cen[3 * size_t(c) + d] = cells.get_centroid(c)[d];
      }
      const auto& ed = dynamic_cast<const EulerSolverData&>(solver.get_solver_data());
      std::vector<double> dS(3 * size_t(NT));
      for (Index c = 0; c < NT; c++)
        for (int d = 0; d < 3; d++) dS[3 * size_t(c) + d] = ed.get_Delta_S()[c][d];
      std::vector<uint32_t> patches;
      for (const auto& p : fv.get_patches()) {
        patches.push_back(uint32_t(p.boundary_type));
        patches.push_back(p.FIRST_FACE);
        patches.push_back(p.N_FACES);
      }
      write_raw(out_dir + "face_ij.u32", ij.data(), ij.size());
      write_raw(out_dir + "face_S.f64", S.data(), S.size());
      write_raw(out_dir + "face_ri.f64", ri.data(), ri.size());
      write_raw(out_dir + "face_rj.f64", rj.data(), rj.size());
      write_raw(out_dir + "cell_vol.f64", vol.data(), vol.size());
      write_raw(out_dir + "cell_centroid.f64", cen.data(), cen.size());
      write_raw(out_dir + "cell_dS.f64", dS.data(), dS.size());
      write_raw(out_dir + "patches.u32", patches.data(), patches.size());
    }

    if (steps < 0) steps = long(config.get_n_timesteps());
    std::vector<double> dts;
    config.set_timestep(0);
    config.set_time(0.0);
    auto t0 = std::chrono::steady_clock::now();
    for (long s = 0; s < steps; s++) {  // Driver.cpp:31-57 without output
      solver.calc_timestep(config);
      solver.step(config);
      config.set_timestep(config.get_timestep() + 1);
      config.set_time(config.get_time() + config.get_delta_time());
      dts.push_back(config.get_delta_time());
    }
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();

    const SolverData& sd = solver.get_solver_data();
    dump_field(out_dir + "U.f64", sd.get_solution());
    write_raw(out_dir + "dt.f64", dts.data(), dts.size());
    if (steps > 0) {
      dump_field(out_dir + "V.f64", sd.get_primvars());
      dump_field(out_dir + "R.f64", sd.get_flux_balance());
      if (config.get_spatial_order() == SpatialOrder::Second) {
        const GradField& g = sd.get_primvars_gradient();
        // Eigen column-major 5x3 per cell: entry (k, d) at 5*d + k.
        write_raw(out_dir + "grad.f64", g[0], size_t(g.size()) * 15);
        dump_field(out_dir + "limiter.f64", sd.get_primvars_limiter());
      }
    }
    std::FILE* meta = std::fopen((out_dir + "meta.txt").c_str(), "w");
    std::fprintf(meta, "n_interior_cells %u\nn_total_cells %u\nn_interior_faces %u\nn_total_faces %u\n"
                       "steps %ld\nseconds %.9f\n",
                 NC, NT, config.get_N_INTERIOR_FACES(), NF, steps, secs);
    std::fclose(meta);
    if (timing)
      std::fprintf(stderr, "nf_ref: %ld steps on %u cells in %.6f s\n", steps, NC, secs);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "nf_ref error: %s\n", e.what());
    return 1;
  }
  return 0;
}
