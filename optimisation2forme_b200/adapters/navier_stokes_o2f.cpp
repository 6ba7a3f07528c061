// Drop-in replacements, with the reference's own signatures, of the hot-path
// entry points of ThibaultMaurelOujia/Optimisation2Forme, implemented on the
// o2f C ABI (include/o2f.h).  A maintainer links this file and libo2f.so
// into the reference build in place of the definitions it replaces:
//
//   computeResidual              include/shape_optimization.hpp:26-27
//   optimizeShape                include/shape_optimization.hpp:29
//   computeLiftDragCoefficients  include/compute.hpp:18
//
// One o2f context per process, created from params.mesh_name on first use
// (the reference is one mesh per process too: its scratch buffers are
// function-static).  Cell states cross in the reference's cell order; the
// interface states and wall stresses that the reference leaves in
// Mesh::edges are written back after every residual.  Errors become
// std::runtime_error with the library's message, as the reference throws.
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "o2f.h"
#include "shape_optimization.hpp"
#include "compute.hpp"

namespace navier_stokes {
namespace {

o2f_ctx* g_ctx = nullptr;

void check(int status) {
  if (status != O2F_OK) throw std::runtime_error(o2f_last_error());
}

o2f_params to_o2f(const SimulationParams& p) {
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

o2f_ctx* context(const SimulationParams& p) {
  const o2f_params q = to_o2f(p);
  if (!g_ctx) check(o2f_create_from_msh(p.mesh_name.c_str(), &q, nullptr, &g_ctx));
  check(o2f_set_params(g_ctx, &q));
  return g_ctx;
}

void upload(o2f_ctx* c, const Mesh& mesh) {
  std::vector<double> U(4 * mesh.cells.size());
  for (size_t i = 0; i < mesh.cells.size(); ++i) {
    const Cell& k = mesh.cells[i];
    U[4 * i] = k.rho;
    U[4 * i + 1] = k.rho_u;
    U[4 * i + 2] = k.rho_v;
    U[4 * i + 3] = k.E;
  }
  check(o2f_state_set(c, U.data()));
}

// Edge L/R states and wall stresses of the last residual into Mesh::edges.
void download_edges(o2f_ctx* c, Mesh& mesh) {
  const size_t ne = mesh.edges.size();
  std::vector<double> lr(8 * ne), tau(3 * ne);
  check(o2f_debug_get(c, "edge_LR", lr.data()));
  check(o2f_debug_get(c, "edge_tau", tau.data()));
  for (size_t e = 0; e < ne; ++e) {
    Edge& g = mesh.edges[e];
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

void computeResidual(Mesh& mesh, const SimulationParams& params, std::vector<double>& R_rho,
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
  download_edges(c, mesh);
}

void computeLiftDragCoefficients(const Mesh& mesh, const SimulationParams& params, double& C_L, double& C_D) {
  (void)mesh;  // the context holds the interface states of the last residual
  double f[3];
  check(o2f_forces(context(params), 0.0, f));
  C_L = f[0];
  C_D = f[1];
}

void optimizeShape(Mesh& mesh, const SimulationParams& params, double eps) {
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

}  // namespace navier_stokes
