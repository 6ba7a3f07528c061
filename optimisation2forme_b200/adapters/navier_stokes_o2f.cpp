// Drop-in replacements, with the reference's own signatures, of the hot-path
// entry points of ThibaultMaurelOujia/Optimisation2Forme, implemented on the
// o2f C ABI (include/o2f.h).  A maintainer links this file and libo2f.so
// into the reference build in place of the definitions it replaces:
//
//   computeAdvectionTerm                       include/advection.hpp:19
//   compute_hllc_flux                          include/advection.hpp:16
//   computeDiffusionTerm                       include/diffusion.hpp:16
//   apply_boundary_conditions                  include/boundary.hpp:13
//   apply_diffusion_bc                         include/boundary.hpp:15
//   apply_InterfaceStates_boundary_conditions  include/boundary.hpp:17-20
//   computeResidual                            include/shape_optimization.hpp:26-27
//   optimizeShape                              include/shape_optimization.hpp:29
//   computeLiftDragCoefficients                include/compute.hpp:18
//
// One o2f context per process, created from params.mesh_name on first use
// (the reference is one mesh per process too: its scratch buffers are
// function-static).  Cell states cross in the reference's cell order; the
// gradients, interface states and wall stresses that the reference leaves
// in Mesh::cells / Mesh::edges are written back after every residual.
// Errors become std::runtime_error with the library's message, as the
// reference throws.
//
// The functions are defined in namespace O2F_ADAPTER_NS (default
// navier_stokes, the drop-in); building with another name lets one binary
// hold both the reference's definitions and these, side by side.
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "o2f.h"
#include "shape_optimization.hpp"
#include "advection.hpp"
#include "boundary.hpp"
#include "compute.hpp"
#include "diffusion.hpp"

#ifndef O2F_ADAPTER_NS
#define O2F_ADAPTER_NS navier_stokes
#endif

namespace O2F_ADAPTER_NS {
namespace NS = ::navier_stokes;
namespace {

o2f_ctx* g_ctx = nullptr;

void check(int status) {
  if (status != O2F_OK) throw std::runtime_error(o2f_last_error());
}

o2f_params to_o2f(const NS::SimulationParams& p) {
  o2f_params q;
  o2f_params_default(&q);
  q.gamma = p.gamma;
  q.viscosity = p.viscosity;
  q.Pr = p.Pr;
  q.cp = p.cp;
  q.cfl_number = p.cfl_number;
  q.final_time = p.final_time;
  q.inflow_velocity = p.inflow_velocity;
  q.rho_ref = p.rho_ref;
  q.p_ref = p.p_ref;
  q.verbosity = p.verbosity;
  return q;
}

o2f_ctx* context(const NS::SimulationParams& p) {
  const o2f_params q = to_o2f(p);
  if (!g_ctx) check(o2f_create_from_msh(p.mesh_name.c_str(), &q, nullptr, &g_ctx));
  check(o2f_set_params(g_ctx, &q));
  return g_ctx;
}

void upload(o2f_ctx* c, const NS::Mesh& mesh) {
  std::vector<double> U(4 * mesh.cells.size());
  for (size_t i = 0; i < mesh.cells.size(); ++i) {
    const NS::Cell& k = mesh.cells[i];
    U[4 * i] = k.rho;
    U[4 * i + 1] = k.rho_u;
    U[4 * i + 2] = k.rho_v;
    U[4 * i + 3] = k.E;
  }
  check(o2f_state_set(c, U.data()));
}

// Edge L/R states and wall stresses of the last residual into Mesh::edges.
void download_edges(o2f_ctx* c, NS::Mesh& mesh) {
  const size_t ne = mesh.edges.size();
  std::vector<double> lr(8 * ne), tau(3 * ne);
  check(o2f_debug_get(c, "edge_LR", lr.data()));
  check(o2f_debug_get(c, "edge_tau", tau.data()));
  for (size_t e = 0; e < ne; ++e) {
    NS::Edge& g = mesh.edges[e];
    g.rho_L = lr[8 * e];
    g.rho_u_L = lr[8 * e + 1];
    g.rho_v_L = lr[8 * e + 2];
    g.E_L = lr[8 * e + 3];
    g.rho_R = lr[8 * e + 4];
    g.rho_u_R = lr[8 * e + 5];
    g.rho_v_R = lr[8 * e + 6];
    g.E_R = lr[8 * e + 7];
    g.tau_xx = tau[3 * e];
    g.tau_yy = tau[3 * e + 1];
    g.tau_xy_yx = tau[3 * e + 2];
  }
}

// Green-Gauss gradients of the last residual into Mesh::cells (the
// reference's computeScalarGradientAdvection leaves them there).
void download_gradients(o2f_ctx* c, NS::Mesh& mesh) {
  const size_t nc = mesh.cells.size();
  std::vector<double> g(8 * nc);
  check(o2f_debug_get(c, "grad", g.data()));
  for (size_t i = 0; i < nc; ++i) {
    NS::Cell& k = mesh.cells[i];
    const double* q = g.data() + 8 * i;
    k.rho_x = q[0];
    k.rho_u_x = q[1];
    k.rho_v_x = q[2];
    k.E_x = q[3];
    k.rho_y = q[4];
    k.rho_u_y = q[5];
    k.rho_v_y = q[6];
    k.E_y = q[7];
  }
}

// Residual of the mesh's state into Cell::R_*, with the given viscosity
// (0: the advection terms alone).
void residual_into(o2f_ctx* c, NS::Mesh& mesh, const NS::SimulationParams& params, double viscosity) {
  o2f_params q = to_o2f(params);
  q.viscosity = viscosity;
  check(o2f_set_params(c, &q));
  upload(c, mesh);
  const size_t n = mesh.cells.size();
  std::vector<double> R(4 * n);
  check(o2f_residual(c, R.data()));
  for (size_t i = 0; i < n; ++i) {
    mesh.cells[i].R_rho = R[4 * i];
    mesh.cells[i].R_rho_u = R[4 * i + 1];
    mesh.cells[i].R_rho_v = R[4 * i + 2];
    mesh.cells[i].R_E = R[4 * i + 3];
  }
}

// Shape parameter file: "name = value" (fixed) or "name *= value"
// (optimised), later lines win, as the reference's loadParamsGeneric.
void read_shape_params(const std::string& path, o2f_shape_params& s, std::vector<int>& ids, double& beta) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open shape parameter file " + path);
  std::string line;
  while (std::getline(in, line)) {
    const size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    const bool opt = eq > 0 && line[eq - 1] == '*';
    std::string name = line.substr(0, opt ? eq - 1 : eq);
    name.erase(0, name.find_first_not_of(" \t"));
    name.erase(name.find_last_not_of(" \t") + 1);
    const double v = std::stod(line.substr(eq + 1));
    int id = -1;
    if (name == "pos_x") s.pos_x = v;
    else if (name == "c") s.c = v;
    else if (name == "m") { s.m = v; id = O2F_PARAM_M; }
    else if (name == "p") { s.p = v; id = O2F_PARAM_P; }
    else if (name == "t") { s.t = v; id = O2F_PARAM_T; }
    else if (name == "beta") beta = v;
    if (opt && id >= 0) {
      bool seen = false;
      for (int k : ids) seen = seen || k == id;
      if (!seen) ids.push_back(id);
    }
  }
}

}  // namespace

// computeAdvectionTerm (src/advection.cpp:415-466): R = the advection terms
// of the mesh's state, with the gradients and interface states it leaves.
// Computed as the residual with zero viscosity (the diffusion terms are then
// exact zeros; a residual entry that is itself zero may come out as -0.0
// where the reference has +0.0 or the reverse).
void computeAdvectionTerm(NS::Mesh& mesh, const NS::SimulationParams& params) {
  o2f_ctx* c = context(params);
  residual_into(c, mesh, params, 0.0);
  download_gradients(c, mesh);
  download_edges(c, mesh);
}

// computeDiffusionTerm (src/diffusion.cpp:206-243): the reference adds the
// viscous terms to R as left by computeAdvectionTerm of the same state, which
// is how every reference caller uses it (Simulator::rk3_substep,
// computeResidual).  Here R becomes the whole residual of the mesh's state,
// summed in the reference's order, so after the pair of calls R holds the
// reference's bits; the wall stresses go to Mesh::edges.
void computeDiffusionTerm(NS::Mesh& mesh, const NS::SimulationParams& params) {
  o2f_ctx* c = context(params);
  residual_into(c, mesh, params, params.viscosity);
  download_edges(c, mesh);
}

// compute_hllc_flux (src/advection.cpp:335-412) of one edge from its
// interface states, on the GPU (o2f_hllc_flux; callers with many edges use
// that array form directly).
void compute_hllc_flux(NS::Edge& edge, const NS::SimulationParams& params, double& edge_flux_rho,
                       double& edge_flux_rho_u, double& edge_flux_rho_v, double& edge_flux_E) {
  const double lr[8] = {edge.rho_L, edge.rho_u_L, edge.rho_v_L, edge.E_L,
                        edge.rho_R, edge.rho_u_R, edge.rho_v_R, edge.E_R};
  const double n[2] = {edge.edgeNormal.x, edge.edgeNormal.y};
  double f[4];
  check(o2f_hllc_flux(1, lr, n, params.gamma, f));
  edge_flux_rho = f[0];
  edge_flux_rho_u = f[1];
  edge_flux_rho_v = f[2];
  edge_flux_E = f[3];
}

// apply_boundary_conditions (src/boundary.cpp:84-94): the "inflow_outflow_x"
// boundary state of code boundaryCondition (o2f_bc_states).
void apply_boundary_conditions(const NS::SimulationParams& params, const char boundaryCondition, double& rho,
                               double& rho_u, double& rho_v, double& E) {
  if (params.boundary_conditions != "inflow_outflow_x")
    throw std::invalid_argument("Unknown boundary condition: " + params.boundary_conditions);
  const o2f_params q = to_o2f(params);
  const uint8_t code = static_cast<uint8_t>(boundaryCondition);
  double u[4] = {rho, rho_u, rho_v, E};
  check(o2f_bc_states(&q, 1, &code, u));
  rho = u[0];
  rho_u = u[1];
  rho_v = u[2];
  E = u[3];
}

// apply_diffusion_bc (src/boundary.cpp:101-127) (o2f_bc_diffusion).
void apply_diffusion_bc(const NS::SimulationParams& params, const char boundaryCondition, double& tau_xx,
                        double& tau_yy, double& tau_xy_yx, double& q_x, double& q_y) {
  (void)params;
  const uint8_t code = static_cast<uint8_t>(boundaryCondition);
  double t[5] = {tau_xx, tau_yy, tau_xy_yx, q_x, q_y};
  check(o2f_bc_diffusion(1, &code, t));
  tau_xx = t[0];
  tau_yy = t[1];
  tau_xy_yx = t[2];
  q_x = t[3];
  q_y = t[4];
}

// apply_InterfaceStates_boundary_conditions (src/boundary.cpp:48-80): the
// ghost right state of a boundary edge (o2f_bc_ghosts); nx, ny are unused,
// as in the reference.
void apply_InterfaceStates_boundary_conditions(const NS::SimulationParams& params, const char boundaryCondition,
                                               double rho_L, double rho_u_L, double rho_v_L, double E_L,
                                               double& rho_R, double& rho_u_R, double& rho_v_R, double& E_R,
                                               double& nx, double& ny) {
  (void)nx;
  (void)ny;
  const o2f_params q = to_o2f(params);
  const uint8_t code = static_cast<uint8_t>(boundaryCondition);
  const double L[4] = {rho_L, rho_u_L, rho_v_L, E_L};
  double Rg[4];
  check(o2f_bc_ghosts(&q, 1, &code, L, Rg));
  rho_R = Rg[0];
  rho_u_R = Rg[1];
  rho_v_R = Rg[2];
  E_R = Rg[3];
}

void computeResidual(NS::Mesh& mesh, const NS::SimulationParams& params, std::vector<double>& R_rho,
                     std::vector<double>& R_rho_u, std::vector<double>& R_rho_v, std::vector<double>& R_E) {
  o2f_ctx* c = context(params);
  upload(c, mesh);
  const size_t n = mesh.cells.size();
  std::vector<double> R(4 * n);
  check(o2f_residual(c, R.data()));
  R_rho.resize(n);
  R_rho_u.resize(n);
  R_rho_v.resize(n);
  R_E.resize(n);
  for (size_t i = 0; i < n; ++i) {
    R_rho[i] = mesh.cells[i].R_rho = R[4 * i];
    R_rho_u[i] = mesh.cells[i].R_rho_u = R[4 * i + 1];
    R_rho_v[i] = mesh.cells[i].R_rho_v = R[4 * i + 2];
    R_E[i] = mesh.cells[i].R_E = R[4 * i + 3];
  }
  download_gradients(c, mesh);
  download_edges(c, mesh);
}

void computeLiftDragCoefficients(const NS::Mesh& mesh, const NS::SimulationParams& params, double& C_L, double& C_D) {
  (void)mesh;  // the context holds the interface states of the last residual
  double f[3];
  check(o2f_forces(context(params), 0.0, f));
  C_L = f[0];
  C_D = f[1];
}

void optimizeShape(NS::Mesh& mesh, const NS::SimulationParams& params, double eps) {
  o2f_ctx* c = context(params);
  upload(c, mesh);
  check(o2f_residual(c, nullptr));
  o2f_shape_params s{0.355, 1.0, 0.02, 0.4, 0.12};
  std::vector<int> ids;
  double beta = 1.0;
  read_shape_params(params.shape_param_file, s, ids, beta);
  std::vector<double> grad(ids.size() ? ids.size() : 1);
  double out[3];
  check(o2f_optimize_shape(c, &s, ids.data(), (int)ids.size(), beta, eps, 1e-6, grad.data(), out));
  static const char* kNames[] = {"m", "p", "t"};
  std::cout << "[preview] J = " << out[0] << "  (BiCGSTAB " << (long long)out[1] << " iterations, relres " << out[2]
            << ")\n";
  for (size_t k = 0; k < ids.size(); ++k) std::cout << "  - dJ/d" << kNames[ids[k]] << " = " << grad[k] << "\n";
}

}  // namespace O2F_ADAPTER_NS
