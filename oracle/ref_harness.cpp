// Test infrastructure only (oracle).  A command-line driver around the
// reference solver's OWN translation units, compiled from the reference
// sources by oracle/build_ref.sh into oracle/_ref/.  It exists to pin the
// CPU restatement (oracle/o2f_oracle.c) and the CUDA path against the
// reference's arithmetic, and to time the reference's OpenMP CPU path.
//
// Every mode builds the reference Mesh (src/mesh.cpp:7-283, through the gmsh
// shim), sets the initial state exactly as Simulator::initialize_fields does
// (src/simulation.cpp:51-56) and then calls the reference functions.  The
// only restated pieces are the time loop (src/simulation.cpp:68-171, which
// cannot be compiled without SFML) and a BiCGSTAB driver (Eigen is absent).
//
// One process handles one mesh: the reference sizes function-static scratch
// buffers on the first call (src/advection.cpp:9-23, src/diffusion.cpp:9-25).
//
// Usage:  o2f_ref <mode> <config> <outdir> [args...]
//   topo                      topology and geometry arrays
//   residual                  computeResidual + gradients, interface states,
//                             wall tau, C_L/C_D and J
//   jt <x.f64>                applyJacobianTranspose(x) after one residual
//   rhs                       assembleAdjointRHS after one residual
//   grad <lambda.f64>         computeShapeGradient(lambda)
//   perturb <name> <eps>      applyShapePerturbationNACA12 geometry
//   march <nsteps>            the SSP-RK3 time loop for nsteps steps
//   bench <reps>              timings of computeResidual / applyJacobianTranspose
//   eval <steps> <iters> <thermal>
//                             one reduced shape-gradient evaluation, timed by
//                             phase: <steps> SSP-RK3 steps (diffusive dt bound
//                             with the thermal diffusivity when <thermal> is 1),
//                             J and the adjoint right-hand side, <iters>
//                             identity-preconditioned BiCGSTAB iterations on
//                             applyJacobianTranspose, computeShapeGradient
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
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

namespace navier_stokes {
// Functions defined in src/shape_optimization.cpp without a header declaration.
void loadParamsGeneric(const std::string&, std::vector<std::string>&, std::vector<double>&,
                       std::vector<std::string>&);
double getParamOrDefault(const std::vector<std::string>&, const std::vector<double>&,
                         const std::string&, double);
void applyJacobianTranspose(Mesh&, const SimulationParams&, const std::vector<double>&,
                            const std::vector<double>&, const std::vector<double>&,
                            const std::vector<double>&, std::vector<double>&, std::vector<double>&,
                            std::vector<double>&, std::vector<double>&, double);
void assembleAdjointRHS(Mesh&, const SimulationParams&, std::vector<double>&, std::vector<double>&,
                        std::vector<double>&, std::vector<double>&, double);
void updateDerivedGeometry(Mesh&);
double computeDirectObjectiveTerm(Mesh&, const SimulationParams&, double);
void computeShapeGradient(Mesh&, const SimulationParams&, const std::vector<double>&,
                          const std::vector<std::string>&, const std::vector<double>&,
                          const std::vector<std::string>&, std::vector<double>&, double, double);
}  // namespace navier_stokes

using namespace navier_stokes;

namespace {

std::string g_out;

void dump_f64(const std::string& name, const std::vector<double>& v) {
  std::ofstream f(g_out + "/" + name + ".f64", std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(double)));
}

void dump_i64(const std::string& name, const std::vector<long long>& v) {
  std::ofstream f(g_out + "/" + name + ".i64", std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(long long)));
}

std::vector<double> read_f64(const std::string& path, std::size_t n) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + path);
  std::vector<double> v(n);
  f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(double)));
  if (!f) throw std::runtime_error("short read " + path);
  return v;
}

long long idx(std::size_t i) { return i == std::size_t(-1) ? -1LL : (long long)i; }

void dump_topology(const Mesh& m) {
  std::vector<double> vxy, elen, en, ec, cvol, cc;
  std::vector<long long> vbc, voff{0}, vcells, vord, ev, ecell, ebc, coff{0}, cedges, cvoff{0}, cverts,
      cnoff{0}, cnbrs;
  for (const auto& v : m.vertices) {
    vxy.push_back(v.p.x);
    vxy.push_back(v.p.y);
    vbc.push_back((unsigned char)v.boundaryCondition);
    for (auto c : v.cellIDs) vcells.push_back((long long)c);
    voff.push_back((long long)vcells.size());
    for (auto c : v.cellIDsOrdered) vord.push_back((long long)c);
  }
  for (const auto& e : m.edges) {
    ev.push_back((long long)e.leftVertexID);
    ev.push_back((long long)e.rightVertexID);
    ecell.push_back(idx(e.leftCellID));
    ecell.push_back(idx(e.rightCellID));
    ebc.push_back((unsigned char)e.boundaryCondition);
    elen.push_back(e.edgeLength);
    en.push_back(e.edgeNormal.x);
    en.push_back(e.edgeNormal.y);
    ec.push_back(e.centre.x);
    ec.push_back(e.centre.y);
  }
  for (const auto& c : m.cells) {
    for (auto e : c.edgeIDs) cedges.push_back((long long)e);
    coff.push_back((long long)cedges.size());
    for (auto v : c.verticeIDs) cverts.push_back((long long)v);
    cvoff.push_back((long long)cverts.size());
    for (auto n : c.neighbourIDs) cnbrs.push_back((long long)n);
    cnoff.push_back((long long)cnbrs.size());
    cvol.push_back(c.cellVolume);
    cc.push_back(c.centre.x);
    cc.push_back(c.centre.y);
  }
  dump_f64("vert_xy", vxy);
  dump_i64("vert_bc", vbc);
  dump_i64("vert_cells_off", voff);
  dump_i64("vert_cells", vcells);
  dump_i64("vert_cells_ord", vord);
  dump_i64("edge_v", ev);
  dump_i64("edge_c", ecell);
  dump_i64("edge_bc", ebc);
  dump_f64("edge_len", elen);
  dump_f64("edge_n", en);
  dump_f64("edge_ctr", ec);
  dump_i64("cell_edges_off", coff);
  dump_i64("cell_edges", cedges);
  dump_i64("cell_verts_off", cvoff);
  dump_i64("cell_verts", cverts);
  dump_i64("cell_nbrs_off", cnoff);
  dump_i64("cell_nbrs", cnbrs);
  dump_f64("cell_vol", cvol);
  dump_f64("cell_ctr", cc);
}

void dump_state(const Mesh& m, const std::string& name) {
  std::vector<double> u;
  for (const auto& c : m.cells) {
    u.push_back(c.rho);
    u.push_back(c.rho_u);
    u.push_back(c.rho_v);
    u.push_back(c.E);
  }
  dump_f64(name, u);
}

void dump_residual_outputs(const Mesh& m, const SimulationParams& p, double beta) {
  std::vector<double> R, G, LR, tau;
  for (const auto& c : m.cells) {
    R.insert(R.end(), {c.R_rho, c.R_rho_u, c.R_rho_v, c.R_E});
    G.insert(G.end(), {c.rho_x, c.rho_u_x, c.rho_v_x, c.E_x, c.rho_y, c.rho_u_y, c.rho_v_y, c.E_y});
  }
  for (const auto& e : m.edges) {
    LR.insert(LR.end(), {e.rho_L, e.rho_u_L, e.rho_v_L, e.E_L, e.rho_R, e.rho_u_R, e.rho_v_R, e.E_R});
    tau.insert(tau.end(), {e.tau_xx, e.tau_xy_yx, e.tau_yy});
  }
  dump_f64("R", R);
  dump_f64("grad", G);
  dump_f64("edge_LR", LR);
  dump_f64("edge_tau", tau);
  double CL = 0, CD = 0;
  computeLiftDragCoefficients(m, p, CL, CD);
  double J = computeDirectObjectiveTerm(const_cast<Mesh&>(m), p, beta);
  dump_f64("forces", {CL, CD, J, beta});
}

void residual(Mesh& m, const SimulationParams& p) {
  const std::size_t n = m.cells.size();
  std::vector<double> r(n), ru(n), rv(n), rE(n);
  computeResidual(m, p, r, ru, rv, rE);
}

// Restatement of Simulator::time_loop / step_SSP_RK3 / rk3_substep
// (src/simulation.cpp:68-171) without the SFML output step and without the
// config reload.  Records per step: dt, t, and the L2 norm of R_rho of the
// first stage (the residual of the state at the start of the step).
void march_core(Mesh& mesh, const SimulationParams& p, int nsteps, bool thermal, std::vector<double>& dts,
                std::vector<double>& ts, std::vector<double>& rnorm) {
  double t = 0.0;
  int it = 0;
  // Thermal bound (no reference counterpart): the diffusive limit with the
  // heat flux's effective diffusivity kappa*(gamma-1) when it exceeds mu.
  const double mu_dt =
      thermal ? std::max(p.viscosity, p.viscosity * p.cp / p.Pr * (p.gamma - 1.0)) : p.viscosity;
  while (t < p.final_time && it < nsteps) {
    double max_wave = 1e-8;
    double min_h = std::numeric_limits<double>::infinity();
    for (std::size_t cid = 0; cid < mesh.cells.size(); ++cid) {
      const Cell& cell = mesh.cells[cid];
      double rho = cell.rho, ru = cell.rho_u, rv = cell.rho_v, E = cell.E;
      double u = ru / rho, v = rv / rho;
      double kinetic = 0.5 * (ru * ru + rv * rv) / rho;
      double pr = (p.gamma - 1.0) * (E - kinetic);
      double c = std::sqrt(p.gamma * pr / rho);
      double speed = std::hypot(u, v) + c;
      max_wave = std::max(max_wave, speed);
      double perimeter = 0.0;
      for (auto eid : cell.edgeIDs) perimeter += mesh.edges[eid].edgeLength;
      double h = 2.0 * cell.cellVolume / perimeter;
      min_h = std::min(min_h, h);
    }
    double dt_adv = p.cfl_number * min_h / max_wave;
    double dt_diff = 0.5 * (min_h * min_h) / mu_dt;
    double dt = std::min(dt_adv, dt_diff);
    for (auto& c : mesh.cells) {
      c.rho_old = c.rho;
      c.rho_u_old = c.rho_u;
      c.rho_v_old = c.rho_v;
      c.E_old = c.E;
    }
    const double cs[3][2] = {{0.0, 1.0}, {3.0 / 4.0, 1.0 / 4.0}, {1.0 / 3.0, 2.0 / 3.0}};
    for (int s = 0; s < 3; ++s) {
      computeAdvectionTerm(mesh, p);
      computeDiffusionTerm(mesh, p);
      if (s == 0) {
        double acc = 0.0;
        for (const auto& c : mesh.cells) acc += c.R_rho * c.R_rho;
        rnorm.push_back(std::sqrt(acc));
      }
      const double c0 = cs[s][0], c1 = cs[s][1];
      for (auto& cell : mesh.cells) {
        cell.rho = c0 * cell.rho_old + c1 * (cell.rho + dt * (cell.R_rho));
        cell.rho_u = c0 * cell.rho_u_old + c1 * (cell.rho_u + dt * (cell.R_rho_u));
        cell.rho_v = c0 * cell.rho_v_old + c1 * (cell.rho_v + dt * (cell.R_rho_v));
        cell.E = c0 * cell.E_old + c1 * (cell.E + dt * (cell.R_E));
      }
    }
    dts.push_back(dt);
    t += dt;
    ts.push_back(t);
    ++it;
  }
}

void march(Mesh& mesh, const SimulationParams& p, int nsteps) {
  std::vector<double> dts, ts, rnorm;
  march_core(mesh, p, nsteps, false, dts, ts, rnorm);
  dump_f64("march_dt", dts);
  dump_f64("march_t", ts);
  dump_f64("march_rnorm", rnorm);
  dump_state(mesh, "U");
}

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// y = J^T x through the reference's applyJacobianTranspose, vectors
// interleaved 4*i+k as the reference's JacobianOpT packs them
// (src/shape_optimization.cpp:616-629).
struct JtOp {
  Mesh& mesh;
  const SimulationParams& p;
  std::vector<double> xr, xru, xrv, xE, yr, yru, yrv, yE;
  JtOp(Mesh& m, const SimulationParams& pp, std::size_t n)
      : mesh(m), p(pp), xr(n), xru(n), xrv(n), xE(n), yr(n), yru(n), yrv(n), yE(n) {}
  void operator()(const std::vector<double>& x, std::vector<double>& y) {
    const std::size_t n = xr.size();
#pragma omp parallel for
    for (std::size_t i = 0; i < n; ++i) {
      xr[i] = x[4 * i];
      xru[i] = x[4 * i + 1];
      xrv[i] = x[4 * i + 2];
      xE[i] = x[4 * i + 3];
    }
    applyJacobianTranspose(mesh, p, xr, xru, xrv, xE, yr, yru, yrv, yE, 1e-6);
#pragma omp parallel for
    for (std::size_t i = 0; i < n; ++i) {
      y[4 * i] = yr[i];
      y[4 * i + 1] = yru[i];
      y[4 * i + 2] = yrv[i];
      y[4 * i + 3] = yE[i];
    }
  }
};

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
#pragma omp parallel for reduction(+ : s)
  for (std::size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

// `iters` iterations of identity-preconditioned BiCGSTAB (van der Vorst,
// 1992) on J^T lambda = b from lambda = 0, the algorithm the reference calls
// from Eigen (src/shape_optimization.cpp:699-716); returns ||r|| / ||b|| of
// the recurrence residual.
double bicgstab_iters(JtOp& A, const std::vector<double>& b, int iters, std::vector<double>& x) {
  const std::size_t n = b.size();
  std::vector<double> r = b, r0 = b, p(n, 0.0), v(n, 0.0), s(n), t(n);
  x.assign(n, 0.0);
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  const double bn = std::sqrt(dot(b, b));
  for (int it = 0; it < iters; ++it) {
    const double rho_new = dot(r0, r);
    const double beta = (rho_new / rho) * (alpha / omega);
#pragma omp parallel for
    for (std::size_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    A(p, v);
    alpha = rho_new / dot(r0, v);
#pragma omp parallel for
    for (std::size_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    A(s, t);
    omega = dot(t, s) / dot(t, t);
#pragma omp parallel for
    for (std::size_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i] + omega * s[i];
      r[i] = s[i] - omega * t[i];
    }
    rho = rho_new;
  }
  return std::sqrt(dot(r, r)) / (bn > 0 ? bn : 1.0);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <mode> <config> <outdir> [args]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  g_out = argv[3];
  try {
    SimulationParams params;
    if (!load_config(argv[2], params)) throw std::runtime_error("cannot read config");
    params.finalize();
    std::vector<std::string> names_all, names;
    std::vector<double> values_all;
    loadParamsGeneric(params.shape_param_file, names_all, values_all, names);
    const double beta = getParamOrDefault(names_all, values_all, "beta", 1);

    Mesh mesh(params);
    initialize_flow_field(mesh, params);
    loadCellStates(mesh, params);
    const std::size_t nc = mesh.cells.size();

    if (mode == "topo") {
      dump_topology(mesh);
    } else if (mode == "residual") {
      residual(mesh, params);
      dump_residual_outputs(mesh, params, beta);
    } else if (mode == "jt") {
      residual(mesh, params);
      auto x = read_f64(argv[4], 4 * nc);
      std::vector<double> xr(nc), xru(nc), xrv(nc), xE(nc), yr(nc), yru(nc), yrv(nc), yE(nc);
      for (std::size_t i = 0; i < nc; ++i) {
        xr[i] = x[4 * i];
        xru[i] = x[4 * i + 1];
        xrv[i] = x[4 * i + 2];
        xE[i] = x[4 * i + 3];
      }
      applyJacobianTranspose(mesh, params, xr, xru, xrv, xE, yr, yru, yrv, yE, 1e-6);
      std::vector<double> y(4 * nc);
      for (std::size_t i = 0; i < nc; ++i) {
        y[4 * i] = yr[i];
        y[4 * i + 1] = yru[i];
        y[4 * i + 2] = yrv[i];
        y[4 * i + 3] = yE[i];
      }
      dump_f64("jt_y", y);
    } else if (mode == "rhs") {
      residual(mesh, params);
      std::vector<double> br, bru, brv, bE;
      assembleAdjointRHS(mesh, params, br, bru, brv, bE, beta);
      std::vector<double> b(4 * nc);
      for (std::size_t i = 0; i < nc; ++i) {
        b[4 * i] = br[i];
        b[4 * i + 1] = bru[i];
        b[4 * i + 2] = brv[i];
        b[4 * i + 3] = bE[i];
      }
      dump_f64("rhs_b", b);
    } else if (mode == "grad") {
      auto lambda = read_f64(argv[4], 4 * nc);
      std::vector<double> g;
      computeShapeGradient(mesh, params, lambda, names_all, values_all, names, g, beta, 1e-6);
      dump_f64("shape_grad", g);
      dump_residual_outputs(mesh, params, beta);
    } else if (mode == "perturb") {
      const std::string name = argv[4];
      const double eps = std::atof(argv[5]);
      applyShapePerturbationNACA12(mesh, params, name, names_all, values_all, eps);
      dump_topology(mesh);
      residual(mesh, params);
      dump_residual_outputs(mesh, params, beta);
    } else if (mode == "march") {
      march(mesh, params, std::atoi(argv[4]));
    } else if (mode == "eval") {
      const int nsteps = std::max(0, std::atoi(argv[4]));
      const int iters = std::max(0, std::atoi(argv[5]));
      const bool thermal = argc > 6 && std::atoi(argv[6]) != 0;
      residual(mesh, params);  // sizes the static scratch buffers (not timed)
      std::vector<double> dts, ts, rnorm;
      const double t0 = now_s();
      march_core(mesh, params, nsteps, thermal, dts, ts, rnorm);
      const double t1 = now_s();
      residual(mesh, params);
      double CL = 0, CD = 0;
      computeLiftDragCoefficients(mesh, params, CL, CD);
      const double J = computeDirectObjectiveTerm(mesh, params, beta);
      std::vector<double> br, bru, brv, bE;
      assembleAdjointRHS(mesh, params, br, bru, brv, bE, beta);
      std::vector<double> b(4 * nc), lambda;
      for (std::size_t i = 0; i < nc; ++i) {
        b[4 * i] = br[i];
        b[4 * i + 1] = bru[i];
        b[4 * i + 2] = brv[i];
        b[4 * i + 3] = bE[i];
      }
      const double t2 = now_s();
      JtOp op(mesh, params, nc);
      const double relres = bicgstab_iters(op, b, iters, lambda);
      const double t3 = now_s();
      std::vector<double> g;
      computeShapeGradient(mesh, params, lambda, names_all, values_all, names, g, beta, 1e-6);
      const double t4 = now_s();
      std::printf("{\"cells\": %zu, \"threads\": %d, \"steps\": %d, \"iters\": %d, \"steps_s\": %.9g, "
                  "\"objective_s\": %.9g, \"bicgstab_s\": %.9g, \"gradient_s\": %.9g, \"total_s\": %.9g, "
                  "\"J\": %.17g, \"relres\": %.9g, \"n_params\": %zu}\n",
                  nc, omp_get_max_threads(), nsteps, iters, t1 - t0, t2 - t1, t3 - t2, t4 - t3, t4 - t0, J, relres,
                  g.size());
    } else if (mode == "bench") {
      // Per-call wall times of the reference's computeResidual and
      // applyJacobianTranspose, `reps` samples each (the first residual call
      // sizes the static scratch buffers and is not timed).
      const int reps = std::max(1, std::atoi(argv[4]));
      residual(mesh, params);
      std::vector<double> t_res, t_jt;
      for (int r = 0; r < reps; ++r) {
        double t0 = now_s();
        residual(mesh, params);
        t_res.push_back(now_s() - t0);
      }
      std::vector<double> x(nc, 1e-3), y0(nc), y1(nc), y2(nc), y3(nc);
      for (int r = 0; r < reps; ++r) {
        double t0 = now_s();
        applyJacobianTranspose(mesh, params, x, x, x, x, y0, y1, y2, y3, 1e-6);
        t_jt.push_back(now_s() - t0);
      }
      std::printf("{\"cells\": %zu, \"edges\": %zu, \"threads\": %d, \"residual_s\": [", nc, mesh.edges.size(),
                  omp_get_max_threads());
      for (int r = 0; r < reps; ++r) std::printf("%s%.9g", r ? ", " : "", t_res[r]);
      std::printf("], \"jt_s\": [");
      for (int r = 0; r < reps; ++r) std::printf("%s%.9g", r ? ", " : "", t_jt[r]);
      std::printf("]}\n");
    } else {
      throw std::runtime_error("unknown mode " + mode);
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "o2f_ref: %s\n", e.what());
    return 1;
  }
  return 0;
}
