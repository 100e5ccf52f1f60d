// Drop-in replacement for NetFlux's src/Solver.cpp: the same class
// declarations (include/Solver.hpp), with the explicit step on the B200
// library (include/netflux_b200.h). Driver.cpp, Output.cpp, NetFlux.cpp,
// Config*, geometry/*, SolverData.cpp and Numerics.cpp are linked unchanged.
//
// Build: compile this file against NetFlux's include/ and link it, instead of
// src/Solver.cpp, with the other NetFlux objects and -lnetflux_b200.
//
// Solver::step and TVD_RK3 are non-virtual (Solver.hpp:22, 53) and the class
// layout is fixed by the header, so each Solver's device solver lives in a
// side table keyed by the object's address.
//
// Mapping (reference -> here):
//   EulerSolver ctor (Solver.cpp:135-142)   device mesh from the PrimalGrid /
//                                           FV_Grid arrays, nf_create,
//                                           nf_set_state with the solution and
//                                           nf_set_state_old with solution_old
//                                           (SolverData.cpp:50-58)
//   EulerSolver::calc_timestep (232-274)    nf_calc_timestep; the reference's
//                                           "Invalid dt calculated" throw
//   Solver::step (34-52)                    nf_step; U is downloaded into
//                                           solver_data when Output will write
//                                           after this step (Driver.cpp:45-50,
//                                           Output.cpp:19-21) or at the last one
//   evaluate_* / set_constant_ghost_values  done by the device step
//
// Environment: NETFLUX_B200_PRECISION = fp64 (default) | fp64_ref | mixed | mixed32.
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "Solver.hpp"
#include "netflux_b200.h"

using namespace geometry;

namespace {

// Device solver of each live Solver object. The reference's Solver has no
// destructor this file could define (Solver.hpp declares none, and Driver
// destroys it through its implicit one), so an entry outlives its Solver: its
// device memory is released when a new Solver takes the same address (the old
// object is then gone) or at exit. NetFlux's Driver creates one Solver per run.
// Never destroyed, so the exit handler below can still walk it.
std::map<const Solver*, nf_solver*>& table() {
  static auto* t = new std::map<const Solver*, nf_solver*>;
  return *t;
}

// Device solvers are released at exit by a handler registered after the
// first one is created: handlers run in reverse order of registration, so
// this one runs before the CUDA runtime's own teardown (a static object's
// destructor could run after it).
void release_all() {
  for (auto& kv : table()) nf_destroy(kv.second);
  table().clear();
}

nf_solver* device_of(const Solver* s) {
  auto it = table().find(s);
  if (it == table().end()) throw std::runtime_error("B200 solver missing for this Solver object");
  return it->second;
}

void check(int rc, nf_solver* s) {
  if (rc != NF_OK) throw std::runtime_error(std::string("netflux_b200: ") + nf_last_error(s));
}

int bc_code(BoundaryType t) {
  switch (t) {
    case BoundaryType::NoSlipWall: return NF_BC_NO_SLIP_WALL;
    case BoundaryType::SlipWall: return NF_BC_SLIP_WALL;
    case BoundaryType::FarField: return NF_BC_FAR_FIELD;
  }
  throw std::runtime_error("unknown boundary type");
}

int precision_from_env() {
  const char* v = std::getenv("NETFLUX_B200_PRECISION");
  if (!v || !*v || std::strcmp(v, "fp64") == 0) return NF_PREC_FP64;
  if (std::strcmp(v, "fp64_ref") == 0) return NF_PREC_FP64_REF;
  if (std::strcmp(v, "mixed") == 0) return NF_PREC_MIXED;
  if (std::strcmp(v, "mixed32") == 0) return NF_PREC_MIXED32;
  throw std::runtime_error(std::string("NETFLUX_B200_PRECISION: unknown value ") + v);
}

// The device mesh from the grids Driver built: nodes and tetrahedra from
// PrimalGrid (PrimalGrid.cpp:140-244), the boundary from FV_Grid, which has
// consumed PrimalGrid's element patches by then (FV_Grid.cpp:142) and keeps
// every face's nodes in face order (face_elements, reordered with the faces,
// FV_Grid.cpp:207-226): patch q is faces [FIRST_FACE, FIRST_FACE + N_FACES).
// nf_mesh_from_arrays takes tets in the order an SU2 file lists them and
// applies the reader's node 1 <-> 2 swap itself (GeometryUtilities.cpp:
// 452-455), so the swap is undone here.
nf_mesh* mesh_from_grids(const PrimalGrid& pg, const FV_Grid& fv) {
  const auto& nodes = pg.get_nodes();
  std::vector<double> xyz(nodes.size() * 3);
  for (size_t i = 0; i < nodes.size(); i++) {
    xyz[3 * i] = nodes[i].x();
    xyz[3 * i + 1] = nodes[i].y();
    xyz[3 * i + 2] = nodes[i].z();
  }
  const Elements& vol = pg.get_volume_elements();
  std::vector<int64_t> tets(size_t(vol.size()) * 4);
  for (Index e = 0; e < vol.size(); e++) {
    if (vol.get_element_type(e) != ElementType::Tetrahedron)
      throw std::runtime_error("netflux_b200 supports tetrahedral meshes only");
    const Index* n = vol.get_element_nodes(e);
    tets[4 * size_t(e) + 0] = n[0];
    tets[4 * size_t(e) + 1] = n[2];
    tets[4 * size_t(e) + 2] = n[1];
    tets[4 * size_t(e) + 3] = n[3];
  }
  const Elements& faces = pg.get_face_elements();
  std::vector<std::string> names;
  std::vector<int> types;
  std::vector<int64_t> offsets{0}, tris;
  for (const auto& p : fv.get_patches()) {
    names.push_back("patch" + std::to_string(names.size()));
    types.push_back(bc_code(p.boundary_type));
    for (Index f = p.FIRST_FACE; f < p.FIRST_FACE + p.N_FACES; f++) {
      if (faces.get_element_type(f) != ElementType::Triangle)
        throw std::runtime_error("netflux_b200 supports triangular boundary faces only");
      const Index* n = faces.get_element_nodes(f);
      tris.push_back(n[0]);
      tris.push_back(n[1]);
      tris.push_back(n[2]);
    }
    offsets.push_back(int64_t(tris.size() / 3));
  }
  std::vector<const char*> cnames;
  for (const auto& n : names) cnames.push_back(n.c_str());
  nf_mesh* m = nf_mesh_from_arrays(int64_t(nodes.size()), xyz.data(), int64_t(vol.size()), tets.data(),
                                   int(cnames.size()), cnames.data(), types.data(), offsets.data(), tris.data());
  if (!m) throw std::runtime_error(std::string("netflux_b200: ") + nf_last_error(nullptr));
  return m;
}

}  // namespace

Solver::Solver(const Config& config, const PrimalGrid& primal_grid, const FV_Grid& FV_grid)
    : primal_grid{primal_grid}, FV_grid{FV_grid} {
  (void)config;
}

void Solver::step(const Config& config) {
  nf_solver* s = device_of(this);
  check(nf_step(s), s);
  const size_t next = config.get_timestep() + 1;
  if (next % config.get_write_stride() == 0 || next >= config.get_n_timesteps()) {
    VecField& U = solver_data->get_solution();
    check(nf_get_state(s, U[0], int64_t(U.size())), s);
  }
}

EulerSolver::EulerSolver(const Config& config, const PrimalGrid& primal_grid, const FV_Grid& FV_grid)
    : Solver(config, primal_grid, FV_grid) {
  solver_data = make_unique<EulerSolverData>(config);
  validity_checker = make_unique<EulerValidityChecker>(config);
  nf_mesh* m = mesh_from_grids(primal_grid, FV_grid);
  nf_params p;
  nf_params_default(&p);
  p.time_scheme = config.get_time_scheme() == TimeScheme::TVD_RK3 ? NF_TVD_RK3 : NF_EXPLICIT_EULER;
  p.spatial_order = config.get_spatial_order() == SpatialOrder::Second ? NF_SECOND_ORDER : NF_FIRST_ORDER;
  p.limiter = config.get_limiter() == Limiter::Barth ? NF_LIMITER_BARTH : NF_LIMITER_NONE;
  p.precision = precision_from_env();
  p.cfl = config.get_CFL();
  for (int k = 0; k < 5; k++) p.freestream[k] = config.get_primvars_inf(k);
  nf_solver* s = nf_create(m, &p);
  nf_mesh_destroy(m);
  if (!s) throw std::runtime_error(std::string("netflux_b200: ") + nf_last_error(nullptr));
  static const bool registered = (std::atexit(release_all) == 0);
  (void)registered;
  auto stale = table().find(this);
  if (stale != table().end()) nf_destroy(stale->second);  // a destroyed Solver's, at this address
  table()[this] = s;
  const VecField& U = solver_data->get_solution();  // free stream (SolverData.cpp:50-58)
  check(nf_set_state(s, U[0], int64_t(U.size())), s);
  // solution_old as the reference leaves it (zero after the free-stream
  // start): the first TVD_RK3 step combines with it (Solver.cpp:127-132)
  const VecField& U_old = solver_data->get_solution_old();
  check(nf_set_state_old(s, U_old[0], int64_t(U_old.size())), s);
}

void EulerSolver::calc_timestep(Config& config) {
  nf_solver* s = device_of(this);
  double dt = 0.0;
  const int rc = nf_calc_timestep(s, &dt);
  if (rc == NF_ERR_DT) throw std::runtime_error("Invalid dt calculated (dt = " + std::to_string(dt) + ")");
  check(rc, s);
  config.set_delta_time(dt);
}

// The device step evaluates ghosts, gradient, limiter and fluxes itself.
void EulerSolver::evaluate_inviscid_fluxes(const Config&) {}
void EulerSolver::set_constant_ghost_values(const Config&) {}
void EulerSolver::evaluate_gradient(const Config&) {}
void EulerSolver::evaluate_limiter(const Config&) {}
