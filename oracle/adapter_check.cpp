// Test infrastructure only (oracle).  Links the reference's own compiled
// translation units (oracle/_ref/obj_exact) with the drop-in adapter
// (optimisation2forme_b200/adapters/navier_stokes_o2f.cpp, built with
// O2F_ADAPTER_NS=o2f_adapter so both definitions coexist) and libo2f.so, and
// compares, on one mesh and state, what the reference's functions and the
// adapter's leave in the Mesh, bit for bit:
//   computeAdvectionTerm + computeDiffusionTerm (R, gradients, L/R states, tau)
//   computeResidual (R vectors and Mesh fields)
//   computeLiftDragCoefficients
//   compute_hllc_flux on every edge's interface states
//   apply_boundary_conditions / apply_diffusion_bc /
//   apply_InterfaceStates_boundary_conditions for every code
// Prints one JSON line with the mismatch counts; exit status 0 when all are 0.
//
// Usage: o2f_adapter_check <config>  (mesh_name, state_load_path, physics)
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "advection.hpp"
#include "boundary.hpp"
#include "compute.hpp"
#include "diffusion.hpp"
#include "init.hpp"
#include "mesh.hpp"
#include "params.hpp"
#include "shape_optimization.hpp"
#include "utils.hpp"

namespace o2f_adapter {
using namespace navier_stokes;
void computeAdvectionTerm(Mesh&, const SimulationParams&);
void computeDiffusionTerm(Mesh&, const SimulationParams&);
void computeResidual(Mesh&, const SimulationParams&, std::vector<double>&, std::vector<double>&,
                     std::vector<double>&, std::vector<double>&);
void computeLiftDragCoefficients(const Mesh&, const SimulationParams&, double&, double&);
void compute_hllc_flux(Edge&, const SimulationParams&, double&, double&, double&, double&);
void apply_boundary_conditions(const SimulationParams&, const char, double&, double&, double&, double&);
void apply_diffusion_bc(const SimulationParams&, const char, double&, double&, double&, double&, double&);
void apply_InterfaceStates_boundary_conditions(const SimulationParams&, const char, double, double, double, double,
                                               double&, double&, double&, double&, double&, double&);
}  // namespace o2f_adapter

using namespace navier_stokes;

namespace {

// Progress on stderr, so that a failing run shows how far it got.
void phase(const char* what) {
  std::fprintf(stderr, "o2f_adapter_check: %s\n", what);
  std::fflush(stderr);
}

// Same bits, except that +0.0 and -0.0 count as equal (see the adapter's
// computeAdvectionTerm).
bool same(double a, double b) {
  if (a == 0.0 && b == 0.0) return true;
  uint64_t x, y;
  std::memcpy(&x, &a, 8);
  std::memcpy(&y, &b, 8);
  return x == y;
}

long count_cells(const Mesh& a, const Mesh& b, bool grads) {
  long bad = 0;
  for (size_t i = 0; i < a.cells.size(); ++i) {
    const Cell &p = a.cells[i], &q = b.cells[i];
    bad += !same(p.R_rho, q.R_rho) + !same(p.R_rho_u, q.R_rho_u) + !same(p.R_rho_v, q.R_rho_v) + !same(p.R_E, q.R_E);
    if (grads)
      bad += !same(p.rho_x, q.rho_x) + !same(p.rho_u_x, q.rho_u_x) + !same(p.rho_v_x, q.rho_v_x) +
             !same(p.E_x, q.E_x) + !same(p.rho_y, q.rho_y) + !same(p.rho_u_y, q.rho_u_y) +
             !same(p.rho_v_y, q.rho_v_y) + !same(p.E_y, q.E_y);
  }
  return bad;
}

long count_edges(const Mesh& a, const Mesh& b, bool tau) {
  long bad = 0;
  for (size_t e = 0; e < a.edges.size(); ++e) {
    const Edge &p = a.edges[e], &q = b.edges[e];
    bad += !same(p.rho_L, q.rho_L) + !same(p.rho_u_L, q.rho_u_L) + !same(p.rho_v_L, q.rho_v_L) +
           !same(p.E_L, q.E_L) + !same(p.rho_R, q.rho_R) + !same(p.rho_u_R, q.rho_u_R) +
           !same(p.rho_v_R, q.rho_v_R) + !same(p.E_R, q.E_R);
    if (tau && p.boundaryCondition == 'w')
      bad += !same(p.tau_xx, q.tau_xx) + !same(p.tau_yy, q.tau_yy) + !same(p.tau_xy_yx, q.tau_xy_yx);
  }
  return bad;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <config>\n", argv[0]);
    return 2;
  }
  try {
    SimulationParams params;
    if (!load_config(argv[1], params)) throw std::runtime_error("cannot read config");
    params.finalize();
    Mesh ref(params);
    initialize_flow_field(ref, params);
    loadCellStates(ref, params);
    Mesh ada = ref;
    phase("reference mesh and state loaded");

    // advection + diffusion, as Simulator::rk3_substep calls them
    computeAdvectionTerm(ref, params);
    phase("reference advection done");
    o2f_adapter::computeAdvectionTerm(ada, params);
    phase("adapter advection done");
    const long adv_cells = count_cells(ref, ada, true), adv_edges = count_edges(ref, ada, false);
    computeDiffusionTerm(ref, params);
    o2f_adapter::computeDiffusionTerm(ada, params);
    phase("diffusion done");
    const long res_cells = count_cells(ref, ada, true), res_edges = count_edges(ref, ada, true);

    // computeResidual and the forces on fresh copies
    Mesh ref2 = ref, ada2 = ref;
    // the reference writes into vectors of the cell count (it does not resize them)
    const size_t nc = ref.cells.size();
    std::vector<double> a0(nc), a1(nc), a2(nc), a3(nc), b0, b1, b2, b3;
    computeResidual(ref2, params, a0, a1, a2, a3);
    o2f_adapter::computeResidual(ada2, params, b0, b1, b2, b3);
    phase("computeResidual done");
    long cr = 0;
    for (size_t i = 0; i < a0.size(); ++i)
      cr += !same(a0[i], b0[i]) + !same(a1[i], b1[i]) + !same(a2[i], b2[i]) + !same(a3[i], b3[i]);
    cr += count_cells(ref2, ada2, true) + count_edges(ref2, ada2, true);
    double CLr = 0, CDr = 0, CLa = 0, CDa = 0;
    computeLiftDragCoefficients(ref2, params, CLr, CDr);
    o2f_adapter::computeLiftDragCoefficients(ada2, params, CLa, CDa);
    const double force_err = std::max(std::fabs(CLr - CLa) / std::max(std::fabs(CLr), 1e-300),
                                      std::fabs(CDr - CDa) / std::max(std::fabs(CDr), 1e-300));

    phase("forces done");
    // compute_hllc_flux on every edge's interface states
    long hllc = 0;
    for (auto& e : ref2.edges) {
      double f[4], g[4];
      compute_hllc_flux(e, params, f[0], f[1], f[2], f[3]);
      o2f_adapter::compute_hllc_flux(e, params, g[0], g[1], g[2], g[3]);
      for (int k = 0; k < 4; ++k) hllc += !same(f[k], g[k]);
    }

    phase("hllc done");
    // the boundary functions for every code on a cell's state
    long bc = 0;
    const char codes[] = {'i', 'o', 'f', 'w', '\0', 'x'};
    const Cell& c0 = ref2.cells[ref2.cells.size() / 2];
    for (char code : codes) {
      double r[4] = {c0.rho, c0.rho_u, c0.rho_v, c0.E}, s[4] = {c0.rho, c0.rho_u, c0.rho_v, c0.E};
      apply_boundary_conditions(params, code, r[0], r[1], r[2], r[3]);
      o2f_adapter::apply_boundary_conditions(params, code, s[0], s[1], s[2], s[3]);
      for (int k = 0; k < 4; ++k) bc += !same(r[k], s[k]);
      double R1[4], R2[4], nx = 1.0, ny = 0.0;
      apply_InterfaceStates_boundary_conditions(params, code, c0.rho, c0.rho_u, c0.rho_v, c0.E, R1[0], R1[1], R1[2],
                                                R1[3], nx, ny);
      o2f_adapter::apply_InterfaceStates_boundary_conditions(params, code, c0.rho, c0.rho_u, c0.rho_v, c0.E, R2[0],
                                                             R2[1], R2[2], R2[3], nx, ny);
      for (int k = 0; k < 4; ++k) bc += !same(R1[k], R2[k]);
      double t1[5] = {1.5, -2.5, 3.5, -4.5, 5.5}, t2[5] = {1.5, -2.5, 3.5, -4.5, 5.5};
      apply_diffusion_bc(params, code, t1[0], t1[1], t1[2], t1[3], t1[4]);
      o2f_adapter::apply_diffusion_bc(params, code, t2[0], t2[1], t2[2], t2[3], t2[4]);
      for (int k = 0; k < 5; ++k) bc += !same(t1[k], t2[k]);
    }
    std::printf("{\"cells\": %zu, \"edges\": %zu, \"advection_cells\": %ld, \"advection_edges\": %ld, "
                "\"residual_cells\": %ld, \"residual_edges\": %ld, \"compute_residual\": %ld, "
                "\"force_rel_err\": %.3e, \"hllc\": %ld, \"bc\": %ld}\n",
                ref.cells.size(), ref.edges.size(), adv_cells, adv_edges, res_cells, res_edges, cr, force_err, hllc,
                bc);
    const bool ok = adv_cells == 0 && adv_edges == 0 && res_cells == 0 && res_edges == 0 && cr == 0 && hllc == 0 &&
                    bc == 0 && force_err <= 1e-11;
    return ok ? 0 : 1;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "o2f_adapter_check: %s\n", e.what());
    return 1;
  }
}
