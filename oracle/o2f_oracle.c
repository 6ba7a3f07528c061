/* Test infrastructure only (oracle): sequential FP64 restatement of the
 * reference hot path.  Each function names the reference lines it follows;
 * expressions keep the reference's association order and the file is
 * compiled with -ffp-contract=off, so on reference-valid meshes (vertex
 * valence <= 4, zero angle of attack) the results equal the reference's own
 * output bit for bit.  Extensions without a reference counterpart (valence >=
 * 5, angle of attack, the t parameter, the residual-drop stop) follow the
 * same formulas as the CUDA path. */
#include "o2f_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define PI_D 3.14159265358979323846

static double smin(double a, double b) { return (b < a) ? b : a; }
static double smax(double a, double b) { return (a < b) ? b : a; }
static double sclamp(double v, double lo, double hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

typedef struct fs_t {
  double rho, ru, rv, E;
  double cos_a, sin_a, q_inf;
} fs_t;

/* Freestream of apply_inflow_outflow_bc (src/boundary.cpp:10-17) rotated by
 * the angle of attack; q_inf of src/compute.cpp:93-100. */
static fs_t freestream(const o2fo_params* p) {
  fs_t f;
  double rho0 = p->rho_ref, p0 = p->p_ref, M = p->inflow_velocity;
  double a0 = sqrt(p->gamma * p0 / rho0);
  double u0 = M * a0;
  double alpha = p->aoa_deg * (PI_D / 180.0);
  f.cos_a = p->aoa_deg == 0.0 ? 1.0 : cos(alpha);
  f.sin_a = p->aoa_deg == 0.0 ? 0.0 : sin(alpha);
  double ux = u0 * f.cos_a, uy = u0 * f.sin_a;
  double kinetic = 0.5 * rho0 * (ux * ux + uy * uy);
  f.rho = rho0;
  f.ru = rho0 * ux;
  f.rv = rho0 * uy;
  f.E = p->p_ref / (p->gamma - 1.0) + kinetic;
  double U_inf = M * sqrt(p->gamma * p0 / rho0);
  f.q_inf = 0.5 * (rho0 * U_inf * U_inf);
  return f;
}

/* apply_inflow_outflow_bc (src/boundary.cpp:7-45). */
static void bc_state(int code, const fs_t* f, double* q) {
  if (code == 'i' || code == 'f') {
    q[0] = f->rho;
    q[1] = f->ru;
    q[2] = f->rv;
    q[3] = f->E;
  } else if (code == 'w') {
    const double kinetic_old = 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0];
    const double e_internal = q[3] - kinetic_old;
    q[1] = 0.0;
    q[2] = 0.0;
    q[3] = e_internal;
  }
}

/* apply_InterfaceStates_boundary_conditions (src/boundary.cpp:48-80). */
static void bc_ghost(int code, const fs_t* f, const double* L, double* R) {
  R[0] = L[0];
  R[1] = L[1];
  R[2] = L[2];
  R[3] = L[3];
  if (code == 'i' || code == 'o' || code == 'f') {
    bc_state(code, f, R);
  } else if (code == 'w') {
    R[1] = -L[1];
    R[2] = -L[2];
  }
}

static double pressure(double rho, double u, double v, double E, double gamma) {
  double kinetic = 0.5 * rho * (u * u + v * v);
  return (gamma - 1.0) * (E - kinetic);
}

/* compute_hllc_flux (src/advection.cpp:335-412). */
static void hllc(const double* Ls, const double* Rs, double enx, double eny, double gamma, double* F) {
  double nx = -enx, ny = -eny;
  double rho_L = Ls[0];
  double u_L = (Ls[1] * (nx) + Ls[2] * ny) / rho_L;
  double v_L = (Ls[1] * (-ny) + Ls[2] * nx) / rho_L;
  double E_L = Ls[3];
  double p_L = pressure(rho_L, u_L, v_L, E_L, gamma);
  double c_L = sqrt(gamma * p_L / rho_L);
  double rho_R = Rs[0];
  double u_R = (Rs[1] * (nx) + Rs[2] * ny) / rho_R;
  double v_R = (Rs[1] * (-ny) + Rs[2] * nx) / rho_R;
  double E_R = Rs[3];
  double p_R = pressure(rho_R, u_R, v_R, E_R, gamma);
  double c_R = sqrt(gamma * p_R / rho_R);
  double S_L = smin(u_L - c_L, u_R - c_R);
  double S_R = smax(u_L + c_L, u_R + c_R);
  double numer = p_R - p_L + rho_L * u_L * (S_L - u_L) - rho_R * u_R * (S_R - u_R);
  double denom = rho_L * (S_L - u_L) - rho_R * (S_R - u_R);
  double S_star = numer / denom;
  double rho_L_star = rho_L * (S_L - u_L) / (S_L - S_star);
  double rho_R_star = rho_R * (S_R - u_R) / (S_R - S_star);
  double rho_v_L_star = rho_L_star * v_L;
  double rho_v_R_star = rho_R_star * v_R;
  double p_star = p_L + rho_L * (S_L - u_L) * (S_star - u_L);
  double E_L_star = ((S_L - u_L) * E_L - p_L * u_L + p_star * S_star) / (S_L - S_star);
  double E_R_star = ((S_R - u_R) * E_R - p_R * u_R + p_star * S_star) / (S_R - S_star);
  double rho_u_L_star = rho_L_star * S_star;
  double rho_u_R_star = rho_R_star * S_star;
  double fu, fv;
  if (S_L >= 0.0) {
    F[0] = rho_L * u_L;
    fu = rho_L * u_L * u_L + p_L;
    fv = rho_L * u_L * v_L;
    F[3] = (E_L + p_L) * u_L;
  } else if (S_L <= 0.0 && S_star >= 0.0) {
    F[0] = rho_u_L_star;
    fu = rho_u_L_star * rho_u_L_star / rho_L_star + p_star;
    fv = rho_v_L_star * rho_u_L_star / rho_L_star;
    F[3] = (E_L_star + p_star) * rho_u_L_star / rho_L_star;
  } else if (S_star <= 0.0 && S_R >= 0.0) {
    F[0] = rho_u_R_star;
    fu = rho_u_R_star * rho_u_R_star / rho_R_star + p_star;
    fv = rho_v_R_star * rho_u_R_star / rho_R_star;
    F[3] = (E_R_star + p_star) * rho_u_R_star / rho_R_star;
  } else {
    F[0] = rho_R * u_R;
    fu = rho_R * u_R * u_R + p_R;
    fv = rho_R * u_R * v_R;
    F[3] = (E_R + p_R) * u_R;
  }
  F[1] = (fu * nx + fv * (-ny));
  F[2] = (fu * ny + fv * (nx));
}

/* Cell -> vertex interpolation of nf fields stored [ncells][nf]
 * (src/advection.cpp:26-128, src/diffusion.cpp:29-136); valence >= 5
 * extension as documented in the header. */
static void vertex_interp(const o2fo_mesh* m, const double* X, int nf, double* out) {
  for (int64_t v = 0; v < m->nv; ++v) {
    const int64_t o = m->vert_coff[v], n = m->vert_coff[v + 1] - o;
    const double px = m->vxy[2 * v], py = m->vxy[2 * v + 1];
    double* r = out + nf * v;
    for (int k = 0; k < nf; ++k) r[k] = 0.0;
    if (n == 3) {
      const int64_t id0 = m->vert_cells[o], id1 = m->vert_cells[o + 1], id2 = m->vert_cells[o + 2];
      const double *c0 = m->cctr + 2 * id0, *c1 = m->cctr + 2 * id1, *c2 = m->cctr + 2 * id2;
      double w0_num = (c1[0] - px) * (c2[1] - py) - (c2[0] - px) * (c1[1] - py);
      double w0_den = (c1[0] - c0[0]) * (c2[1] - c0[1]) - (c2[0] - c0[0]) * (c1[1] - c0[1]);
      double w0 = (w0_num / w0_den);
      double w1_num = (c2[0] - px) * (c0[1] - py) - (c0[0] - px) * (c2[1] - py);
      double w1_den = (c1[0] - c0[0]) * (c2[1] - c0[1]) - (c2[0] - c0[0]) * (c1[1] - c0[1]);
      double w1 = (w1_num / w1_den);
      double w2 = 1 - w0 - w1;
      for (int k = 0; k < nf; ++k) r[k] = w0 * X[nf * id0 + k] + w1 * X[nf * id1 + k] + w2 * X[nf * id2 + k];
    } else if (n >= 4) {
      const int64_t* ord = m->vert_cells_ord + o;
      double d[64], ux[64], uy[64], w[64];
      if (n > 64) continue;
      for (int64_t k = 0; k < n; ++k) {
        double dx = m->cctr[2 * ord[k]] - px, dy = m->cctr[2 * ord[k] + 1] - py;
        d[k] = hypot(dx, dy);
        ux[k] = dx / d[k];
        uy[k] = dy / d[k];
      }
      if (n > 4 && m->vbc[v] != 0) {
        for (int64_t k = 0; k < n; ++k) w[k] = 1.0 / d[k];
      } else {
        for (int64_t k = 0; k < n; ++k) {
          int64_t km1 = (k + n - 1) % n, kp1 = (k + 1) % n;
          double cos_prev = sclamp(ux[km1] * ux[k] + uy[km1] * uy[k], -1.0, 1.0);
          double cos_next = sclamp(ux[k] * ux[kp1] + uy[k] * uy[kp1], -1.0, 1.0);
          double theta_prev = acos(cos_prev);
          double theta_next = acos(cos_next);
          w[k] = (tan(0.5 * theta_prev) + tan(0.5 * theta_next)) / d[k];
        }
      }
      double wsum = 0.0;
      for (int64_t k = 0; k < n; ++k) wsum += w[k];
      for (int64_t k = 0; k < n; ++k) w[k] /= wsum;
      for (int f = 0; f < nf; ++f) {
        double acc = w[0] * X[nf * ord[0] + f];
        for (int64_t k = 1; k < n; ++k) acc = acc + w[k] * X[nf * ord[k] + f];
        r[f] = acc;
      }
    } else if (n == 2) {
      const int64_t id0 = m->vert_cells[o], id1 = m->vert_cells[o + 1];
      for (int k = 0; k < nf; ++k) r[k] = 0.5 * (X[nf * id0 + k] + X[nf * id1 + k]);
    } else if (n == 1) {
      const int64_t id0 = m->vert_cells[o];
      for (int k = 0; k < nf; ++k) r[k] = X[nf * id0 + k];
    }
  }
}

static double limiter_alpha(int kind, double phi_i, double phi_pred, double phi_min, double phi_max,
                            double cellArea, double k_eps) {
  if (kind == 0) { /* computeVenkatAlpha (src/advection.cpp:209-230) */
    const double delta = phi_pred - phi_i;
    if (fabs(delta) < DBL_EPSILON) return 1.0;
    const double h = sqrt(cellArea / PI_D);
    const double eps = k_eps * k_eps * k_eps * h * h * h;
    double a = (delta > 0.0) ? (phi_max - phi_i) : (phi_min - phi_i);
    double d = delta;
    double alpha = (a * a + eps + 2.0 * a * d) / (a * a + eps + 2.0 * d * d);
    return sclamp(alpha, 0.0, 1.0);
  }
  /* computeBarthJespersenAlpha (src/advection.cpp:195-207) */
  double alpha = 1.0;
  if (fabs(phi_pred - phi_i) < DBL_EPSILON) return alpha;
  if (phi_pred > phi_i)
    alpha = smin(1.0, (phi_max - phi_i) / (phi_pred - phi_i));
  else if (phi_pred < phi_i)
    alpha = smin(1.0, (phi_min - phi_i) / (phi_pred - phi_i));
  return alpha;
}

void o2fo_residual(const o2fo_mesh* m, const o2fo_params* p, const double* U, double* R, double* grad_out,
                   double* LR_out, double* tau_out, double* vU_out) {
  const int64_t nc = m->nc, ne = m->ne, nv = m->nv;
  const fs_t fs = freestream(p);
  double* vq = (double*)malloc(sizeof(double) * 4 * nv);
  double* eq = (double*)malloc(sizeof(double) * 4 * ne);
  double* G = (double*)malloc(sizeof(double) * 8 * nc);
  double* LR = LR_out ? LR_out : (double*)malloc(sizeof(double) * 8 * ne);
  double* F = (double*)malloc(sizeof(double) * 4 * ne);
  double* tq = (double*)malloc(sizeof(double) * 5 * nc);
  double* vtq = (double*)malloc(sizeof(double) * 5 * nv);
  double* etq = (double*)malloc(sizeof(double) * 5 * ne);
  /* computeScalarGradientAdvection (src/advection.cpp:6-191) */
  vertex_interp(m, U, 4, vq);
  for (int64_t v = 0; v < nv; ++v) {
    const int c = (int)m->vbc[v];
    if (c == 'i' || c == 'o' || c == 'f' || c == 'w') bc_state(c, &fs, vq + 4 * v);
  }
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t a = m->edge_v[2 * e], b = m->edge_v[2 * e + 1];
    for (int k = 0; k < 4; ++k) eq[4 * e + k] = 0.5 * (vq[4 * a + k] + vq[4 * b + k]);
    const int c = (int)m->edge_bc[e];
    if (c == 'i' || c == 'o' || c == 'f' || c == 'w') bc_state(c, &fs, eq + 4 * e);
  }
  for (int64_t i = 0; i < nc; ++i) {
    double* g = G + 8 * i;
    for (int k = 0; k < 8; ++k) g[k] = 0.0;
    const double cv = m->cvol[i];
    for (int64_t j = m->cell_eoff[i]; j < m->cell_eoff[i + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      double el = m->elen[e], enx = m->en[2 * e], eny = m->en[2 * e + 1];
      if (m->edge_c[2 * e] == i) {
        enx = -enx;
        eny = -eny;
      }
      for (int k = 0; k < 4; ++k) g[k] += eq[4 * e + k] * el * enx / cv;
      for (int k = 0; k < 4; ++k) g[4 + k] += eq[4 * e + k] * el * eny / cv;
    }
  }
  /* computeInterfaceStates (src/advection.cpp:232-321) */
  for (int64_t cid = 0; cid < nc; ++cid) {
    const double* u = U + 4 * cid;
    const double* g = G + 8 * cid;
    double mn[4], mx[4], al[4];
    for (int k = 0; k < 4; ++k) mn[k] = mx[k] = u[k];
    for (int64_t j = m->cell_eoff[cid]; j < m->cell_eoff[cid + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      const int64_t other = (m->edge_c[2 * e] == cid) ? m->edge_c[2 * e + 1] : m->edge_c[2 * e];
      if (other < 0) continue;
      const double* nb = U + 4 * other;
      for (int k = 0; k < 4; ++k) {
        if (nb[k] < mn[k]) mn[k] = nb[k];
        if (nb[k] > mx[k]) mx[k] = nb[k];
      }
    }
    const double cx = m->cctr[2 * cid], cy = m->cctr[2 * cid + 1], vol = m->cvol[cid];
    for (int k = 0; k < 4; ++k) al[k] = 1.0;
    for (int64_t j = m->cell_eoff[cid]; j < m->cell_eoff[cid + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      const double dx = m->ectr[2 * e] - cx, dy = m->ectr[2 * e + 1] - cy;
      for (int k = 0; k < 4; ++k) {
        const double phi_i = u[k];
        const double phi_pred = phi_i + g[k] * dx + g[4 + k] * dy;
        al[k] = smin(al[k], limiter_alpha(p->limiter, phi_i, phi_pred, mn[k], mx[k], vol, p->limiter_k));
      }
    }
    for (int64_t j = m->cell_eoff[cid]; j < m->cell_eoff[cid + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      const double dx = m->ectr[2 * e] - cx, dy = m->ectr[2 * e + 1] - cy;
      double st[4];
      for (int k = 0; k < 4; ++k) st[k] = u[k] + al[k] * (g[k] * dx + g[4 + k] * dy);
      if (m->edge_c[2 * e] == cid) {
        for (int k = 0; k < 4; ++k) LR[8 * e + k] = st[k];
        const int c = (int)m->edge_bc[e];
        if (c == 'i' || c == 'o' || c == 'f' || c == 'w') bc_ghost(c, &fs, st, LR + 8 * e + 4);
      } else if (m->edge_c[2 * e + 1] == cid) {
        for (int k = 0; k < 4; ++k) LR[8 * e + 4 + k] = st[k];
      }
    }
  }
  /* HLLC and the residual gather (src/advection.cpp:433-464) */
  for (int64_t e = 0; e < ne; ++e) hllc(LR + 8 * e, LR + 8 * e + 4, m->en[2 * e], m->en[2 * e + 1], p->gamma, F + 4 * e);
  for (int64_t cid = 0; cid < nc; ++cid) {
    double* r = R + 4 * cid;
    for (int k = 0; k < 4; ++k) r[k] = 0.0;
    for (int64_t j = m->cell_eoff[cid]; j < m->cell_eoff[cid + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      const double sign = (m->edge_c[2 * e] == cid ? +1.0 : -1.0);
      const double L = m->elen[e];
      for (int k = 0; k < 4; ++k) r[k] += sign * F[4 * e + k] * L;
    }
    const double invV = 1.0 / m->cvol[cid];
    for (int k = 0; k < 4; ++k) r[k] *= -invV;
  }
  /* computeDiffusionTerm (src/diffusion.cpp:206-243) */
  const double mu = p->viscosity, gamma = p->gamma, kappa = p->viscosity * p->cp / p->Pr;
  for (int64_t cid = 0; cid < nc; ++cid) {
    const double* u = U + 4 * cid;
    const double* g = G + 8 * cid;
    double uu = u[1] / u[0];
    double vv = u[2] / u[0];
    double u_x = (g[1] - uu * g[0]) / u[0];
    double v_y = (g[4 + 2] - vv * g[4 + 0]) / u[0];
    double u_y = (g[4 + 1] - uu * g[4 + 0]) / u[0];
    double v_x = (g[2] - vv * g[0]) / u[0];
    double* t = tq + 5 * cid;
    t[0] = 2 * mu * u_x - 2.0 / 3.0 * mu * (u_x + v_y);
    t[1] = 2 * mu * v_y - 2.0 / 3.0 * mu * (u_x + v_y);
    t[2] = mu * (u_y + v_x);
    double T_x = (gamma - 1.0) * ((g[3] * u[0] - u[3] * g[0]) / (u[0] * u[0]) - (uu * u_x + vv * v_x));
    double T_y = (gamma - 1.0) * ((g[4 + 3] * u[0] - u[3] * g[4 + 0]) / (u[0] * u[0]) - (uu * u_y + vv * v_y));
    t[3] = -kappa * T_x;
    t[4] = -kappa * T_y;
  }
  vertex_interp(m, tq, 5, vtq);
  for (int64_t v = 0; v < nv; ++v) {
    const int c = (int)m->vbc[v];
    if (c == 'f' || c == 'w')
      for (int k = 0; k < 5; ++k) vtq[5 * v + k] = 0.0;
  }
  if (tau_out)
    for (int64_t i = 0; i < 3 * ne; ++i) tau_out[i] = 0.0;
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t a = m->edge_v[2 * e], b = m->edge_v[2 * e + 1];
    double* t = etq + 5 * e;
    for (int k = 0; k < 5; ++k) t[k] = 0.5 * (vtq[5 * a + k] + vtq[5 * b + k]);
    const int c = (int)m->edge_bc[e];
    if (c == 'f' || c == 'w')
      for (int k = 0; k < 5; ++k) t[k] = 0.0;
    if (c == 'w' && tau_out) {
      tau_out[3 * e] = t[0];
      tau_out[3 * e + 1] = t[2];
      tau_out[3 * e + 2] = t[1];
    }
  }
  for (int64_t i = 0; i < nc; ++i) {
    const double cv = m->cvol[i];
    const double uu = U[4 * i + 1] / U[4 * i];
    const double vv = U[4 * i + 2] / U[4 * i];
    double* r = R + 4 * i;
    for (int64_t j = m->cell_eoff[i]; j < m->cell_eoff[i + 1]; ++j) {
      const int64_t e = m->cell_edges[j];
      double el = m->elen[e], enx = m->en[2 * e], eny = m->en[2 * e + 1];
      if (m->edge_c[2 * e] == i) {
        enx = -enx;
        eny = -eny;
      }
      const double* t = etq + 5 * e;
      r[1] += t[0] * el * enx / cv + t[2] * el * eny / cv;
      r[2] += t[2] * el * enx / cv + t[1] * el * eny / cv;
      r[3] += (uu * t[0] + vv * t[2] - t[3]) * el * enx / cv + (uu * t[2] + vv * t[1] - t[4]) * el * eny / cv;
    }
  }
  if (grad_out) memcpy(grad_out, G, sizeof(double) * 8 * nc);
  if (vU_out) memcpy(vU_out, vq, sizeof(double) * 4 * nv);
  free(vq);
  free(eq);
  free(G);
  if (!LR_out) free(LR);
  free(F);
  free(tq);
  free(vtq);
  free(etq);
}

/* computeLiftDragCoefficients (src/compute.cpp:92-132) and
 * computeDirectObjectiveTerm (src/shape_optimization.cpp:893-939), summed in
 * edge order (one thread). */
void o2fo_forces(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* tau, double beta,
                 double* out) {
  const fs_t fs = freestream(p);
  double Fy = 0.0, Fx = 0.0, FyJ = 0.0, FxJ = 0.0;
  for (int64_t e = 0; e < m->ne; ++e) {
    if (m->edge_bc[e] != 'w') continue;
    const double nx = m->en[2 * e], ny = m->en[2 * e + 1], A = m->elen[e];
    const double* s = LR + 8 * e;
    double pr = (p->gamma - 1.0) * (s[3] - 0.5 * (s[1] * s[1] + s[2] * s[2]) / s[0]);
    double txx = tau[3 * e], txy = tau[3 * e + 1], tyy = tau[3 * e + 2];
    double l = (-pr * ny + txy * nx + tyy * ny) * A;
    double d = (-pr * nx + txx * nx + txy * ny) * A;
    Fy += l;
    Fx += d;
    if (m->ectr[2 * e] > 1.3) continue;
    FyJ += l;
    FxJ += d;
  }
  const double corde = 1;
  const double L = Fy * fs.cos_a - Fx * fs.sin_a, D = Fx * fs.cos_a + Fy * fs.sin_a;
  const double LJ = FyJ * fs.cos_a - FxJ * fs.sin_a, DJ = FxJ * fs.cos_a + FyJ * fs.sin_a;
  out[0] = L / (fs.q_inf * corde);
  out[1] = D / (fs.q_inf * corde);
  const double CL = LJ / (fs.q_inf * corde), CD = DJ / (fs.q_inf * corde);
  out[2] = -CL + beta * CD;
}

/* EdgeFluxJac blocks and applyJacobianTranspose
 * (src/shape_optimization.cpp:232-484), accumulation in edge order. */
void o2fo_jt(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* x, double* y) {
  const fs_t fs = freestream(p);
  const double eps = 1e-6;
  memset(y, 0, sizeof(double) * 4 * m->nc);
  for (int64_t e = 0; e < m->ne; ++e) {
    const double* Ls = LR + 8 * e;
    const double* Rs = LR + 8 * e + 4;
    const int code = (int)m->edge_bc[e];
    const double enx = m->en[2 * e], eny = m->en[2 * e + 1], L = m->elen[e];
    double FUL[4][4], FUR[4][4];
    for (int j = 0; j < 4; ++j) {
      double Lp[4], Lm[4], Rp[4], Rm[4], fp[4], fm[4];
      for (int k = 0; k < 4; ++k) {
        Lp[k] = Lm[k] = Ls[k];
        Rp[k] = Rm[k] = Rs[k];
      }
      Lp[j] = Ls[j] + eps;
      Lm[j] = Ls[j] - eps;
      if (code != 0) {
        bc_ghost(code, &fs, Lp, Rp);
        bc_ghost(code, &fs, Lm, Rm);
      }
      hllc(Lp, Rp, enx, eny, p->gamma, fp);
      hllc(Lm, Rm, enx, eny, p->gamma, fm);
      for (int r = 0; r < 4; ++r) FUL[r][j] = (fp[r] - fm[r]) / (2 * eps);
      for (int k = 0; k < 4; ++k) {
        Rp[k] = Rm[k] = Rs[k];
      }
      Rp[j] = Rs[j] + eps;
      Rm[j] = Rs[j] - eps;
      hllc(Ls, Rp, enx, eny, p->gamma, fp);
      hllc(Ls, Rm, enx, eny, p->gamma, fm);
      for (int r = 0; r < 4; ++r) FUR[r][j] = (fp[r] - fm[r]) / (2 * eps);
    }
    const int64_t iL = m->edge_c[2 * e];
    const double invV_L = 1.0 / m->cvol[iL];
    double D[4];
    if (code != 0) {
      for (int k = 0; k < 4; ++k) D[k] = (-x[4 * iL + k] * invV_L) * L;
      for (int k = 0; k < 4; ++k)
        y[4 * iL + k] += (FUL[0][k] * D[0] + FUL[1][k] * D[1] + FUL[2][k] * D[2] + FUL[3][k] * D[3]);
      continue;
    }
    const int64_t iR = m->edge_c[2 * e + 1];
    const double invV_R = 1.0 / m->cvol[iR];
    for (int k = 0; k < 4; ++k) D[k] = (-x[4 * iL + k] * invV_L + x[4 * iR + k] * invV_R) * L;
    for (int k = 0; k < 4; ++k)
      y[4 * iL + k] += (FUL[0][k] * D[0] + FUL[1][k] * D[1] + FUL[2][k] * D[2] + FUL[3][k] * D[3]);
    for (int k = 0; k < 4; ++k)
      y[4 * iR + k] += (FUR[0][k] * D[0] + FUR[1][k] * D[1] + FUR[2][k] * D[2] + FUR[3][k] * D[3]);
  }
}

/* assembleAdjointRHS (src/shape_optimization.cpp:491-554). */
void o2fo_rhs(const o2fo_mesh* m, const o2fo_params* p, const double* LR, double beta, double* b) {
  const fs_t fs = freestream(p);
  const double corde = 1;
  memset(b, 0, sizeof(double) * 4 * m->nc);
  for (int64_t e = 0; e < m->ne; ++e) {
    if (m->edge_bc[e] != 'w') continue;
    const int64_t iL = m->edge_c[2 * e];
    const double A_f = m->elen[e], nx = m->en[2 * e], ny = m->en[2 * e + 1];
    const double* s = LR + 8 * e;
    const double g = p->gamma;
    double dp[4];
    dp[0] = 0.5 * (g - 1.0) * ((s[1] * s[1] + s[2] * s[2]) / (s[0] * s[0]));
    dp[1] = -(g - 1.0) * (s[1] / s[0]);
    dp[2] = -(g - 1.0) * (s[2] / s[0]);
    dp[3] = (g - 1.0);
    const double coeff_CL = +(ny * fs.cos_a - nx * fs.sin_a) * A_f / (fs.q_inf * corde);
    for (int k = 0; k < 4; ++k) b[4 * iL + k] += coeff_CL * dp[k];
    const double coeff_CD = (-(nx * fs.cos_a) - ny * fs.sin_a) * A_f / (fs.q_inf * corde) * beta;
    for (int k = 0; k < 4; ++k) b[4 * iL + k] += coeff_CD * dp[k];
  }
}

/* Simulator::time_loop / step_SSP_RK3 / rk3_substep
 * (src/simulation.cpp:68-171). */
int64_t o2fo_march(const o2fo_mesh* m, const o2fo_params* p, double* U, int64_t max_steps, double drop_tol,
                   double* dts, double* hist, double* t_out) {
  const int64_t nc = m->nc;
  double* Uo = (double*)malloc(sizeof(double) * 4 * nc);
  double* R = (double*)malloc(sizeof(double) * 4 * nc);
  double t = 0.0, h0 = 0.0;
  int64_t it = 0;
  int drop_hit = 0;
  double min_h = INFINITY;
  for (int64_t c = 0; c < nc; ++c) {
    double perimeter = 0.0;
    for (int64_t j = m->cell_eoff[c]; j < m->cell_eoff[c + 1]; ++j) perimeter += m->elen[m->cell_edges[j]];
    double h = 2.0 * m->cvol[c] / perimeter;
    min_h = smin(min_h, h);
  }
  while (t < p->final_time && it < max_steps && !drop_hit) {
    double max_wave = 1e-8;
    for (int64_t c = 0; c < nc; ++c) {
      const double *q = U + 4 * c;
      double u = q[1] / q[0], v = q[2] / q[0];
      double kinetic = 0.5 * (q[1] * q[1] + q[2] * q[2]) / q[0];
      double pr = (p->gamma - 1.0) * (q[3] - kinetic);
      double cs = sqrt(p->gamma * pr / q[0]);
      double speed = hypot(u, v) + cs;
      max_wave = smax(max_wave, speed);
    }
    double dt_adv = p->cfl_number * min_h / max_wave;
    double mu_dt = p->viscosity;
    if (p->dt_mode == 1) mu_dt = smax(p->viscosity, p->viscosity * p->cp / p->Pr * (p->gamma - 1.0));
    double dt_diff = 0.5 * (min_h * min_h) / mu_dt;
    double dt = smin(dt_adv, dt_diff);
    memcpy(Uo, U, sizeof(double) * 4 * nc);
    static const double cs[3][2] = {{0.0, 1.0}, {3.0 / 4.0, 1.0 / 4.0}, {1.0 / 3.0, 2.0 / 3.0}};
    for (int s = 0; s < 3; ++s) {
      o2fo_residual(m, p, U, R, NULL, NULL, NULL, NULL);
      if (s == 0) {
        double acc = 0.0;
        for (int64_t c = 0; c < nc; ++c) acc += R[4 * c] * R[4 * c];
        const double nrm = sqrt(acc);
        if (hist) hist[it] = nrm;
        if (it == 0) h0 = nrm;
        if (drop_tol > 0.0 && h0 > 0.0 && nrm <= drop_tol * h0) drop_hit = 1;
      }
      for (int64_t i = 0; i < 4 * nc; ++i) U[i] = cs[s][0] * Uo[i] + cs[s][1] * (U[i] + dt * (R[i]));
    }
    if (dts) dts[it] = dt;
    t += dt;
    ++it;
  }
  if (t_out) *t_out = t;
  free(Uo);
  free(R);
  return it;
}

/* yc_naca4 / yt_naca4 (src/shape_optimization.cpp:807-826). */
static double yc_naca4(double mm, double pp, double xr) {
  xr = sclamp(xr, 0.0, 1.0);
  if (mm == 0.0) return 0.0;
  if (xr <= pp) return mm / (pp * pp) * (2.0 * pp * xr - xr * xr);
  return mm / ((1.0 - pp) * (1.0 - pp)) * ((1.0 - 2.0 * pp) + 2.0 * pp * xr - xr * xr);
}

static double yt_naca4(double t, double c, double xr) {
  xr = sclamp(xr, 0.0, 1.0);
  return 5.0 * t * c * (0.2969 * sqrt(xr) - 0.1260 * xr - 0.3516 * xr * xr + 0.2843 * xr * xr * xr -
                        0.1015 * xr * xr * xr * xr);
}

/* applyShapePerturbationNACA12 + updateDerivedGeometry
 * (src/shape_optimization.cpp:748-890).  `out` must own copies of the
 * mutable arrays; topology pointers are shared.  param: 0 m, 1 p, 2 t. */
void o2fo_perturb(const o2fo_mesh* m, const o2fo_params* p, const o2fo_shape* s, int param, double eps,
                  o2fo_mesh* out) {
  (void)p;
  memcpy(out->vxy, m->vxy, sizeof(double) * 2 * m->nv);
  memcpy(out->cvol, m->cvol, sizeof(double) * m->nc);
  memcpy(out->cctr, m->cctr, sizeof(double) * 2 * m->nc);
  memcpy(out->elen, m->elen, sizeof(double) * m->ne);
  memcpy(out->en, m->en, sizeof(double) * 2 * m->ne);
  memcpy(out->ectr, m->ectr, sizeof(double) * 2 * m->ne);
  const double pos_x = s->pos_x, c = s->c, m0 = s->m, p0 = s->p, t0 = s->t;
  double m1 = m0, p1 = p0, t1 = t0;
  if (param == 0)
    m1 = m0 + eps;
  else if (param == 1)
    p1 = p0 + eps;
  else if (param == 2)
    t1 = t0 + eps;
  else
    return;
  for (int64_t v = 0; v < m->nv; ++v) {
    if (m->vbc[v] != 'w') continue;
    const double x_local = out->vxy[2 * v] - pos_x;
    const double xr = x_local / c;
    if (xr >= 0.9) continue;
    const double yc0 = yc_naca4(m0, p0, xr);
    const double yt0 = yt_naca4(t1, c, xr);
    const double sgn = (out->vxy[2 * v + 1] >= yc0) ? +1.0 : -1.0;
    const double yc1 = yc_naca4(m1, p1, xr);
    out->vxy[2 * v] = pos_x + xr * c;
    out->vxy[2 * v + 1] = yc1 + sgn * yt0;
  }
  for (int64_t e = 0; e < m->ne; ++e) {
    const int64_t a = m->edge_v[2 * e], b = m->edge_v[2 * e + 1];
    if (m->edge_bc[e] != 'w' && m->vbc[a] != 'w' && m->vbc[b] != 'w') continue;
    const double* A = out->vxy + 2 * a;
    const double* B = out->vxy + 2 * b;
    double tx = A[0] - B[0], ty = A[1] - B[1], tz = 0.0;
    double len = sqrt(tx * tx + ty * ty + tz * tz);
    double nx = ty / len, ny = -tx / len;
    const int64_t cl = m->edge_c[2 * e];
    const int64_t o = m->cell_voff[cl], nn = m->cell_voff[cl + 1] - o;
    const double* n0 = out->vxy + 2 * m->cell_verts[o];
    const double* n1 = out->vxy + 2 * m->cell_verts[o + 1];
    const double* n2 = out->vxy + 2 * m->cell_verts[o + 2];
    if (nn == 3) {
      double ax = n1[0] - n0[0], ay = n1[1] - n0[1], bx = n2[0] - n0[0], by = n2[1] - n0[1];
      out->cvol[cl] = fabs(0.5 * (ax * by - bx * ay));
      out->cctr[2 * cl] = 1.0 / 3.0 * (n0[0] + n1[0] + n2[0]);
      out->cctr[2 * cl + 1] = 1.0 / 3.0 * (n0[1] + n1[1] + n2[1]);
    } else if (nn == 4) {
      const double* n3 = out->vxy + 2 * m->cell_verts[o + 3];
      double ax = n1[0] - n0[0], ay = n1[1] - n0[1], bx = n2[0] - n0[0], by = n2[1] - n0[1];
      double qx = n1[0] - n2[0], qy = n1[1] - n2[1], rx = n3[0] - n2[0], ry = n3[1] - n2[1];
      out->cvol[cl] = 0.5 * (fabs(ax * by - bx * ay) + fabs(qx * ry - rx * qy));
      out->cctr[2 * cl] = 0.25 * (n0[0] + n1[0] + n2[0] + n3[0]);
      out->cctr[2 * cl + 1] = 0.25 * (n0[1] + n1[1] + n2[1] + n3[1]);
    }
    double ex = 0.5 * (A[0] + B[0]), ey = 0.5 * (A[1] + B[1]);
    double dx = out->cctr[2 * cl] - ex, dy = out->cctr[2 * cl + 1] - ey;
    if (dx * nx + dy * ny < 0) {
      nx = -nx;
      ny = -ny;
    }
    out->elen[e] = len;
    out->en[2 * e] = nx;
    out->en[2 * e + 1] = ny;
    out->ectr[2 * e] = ex;
    out->ectr[2 * e + 1] = ey;
  }
}

static void mesh_copy(const o2fo_mesh* m, o2fo_mesh* c) {
  *c = *m;
  c->vxy = (double*)malloc(sizeof(double) * 2 * m->nv);
  c->cvol = (double*)malloc(sizeof(double) * m->nc);
  c->cctr = (double*)malloc(sizeof(double) * 2 * m->nc);
  c->elen = (double*)malloc(sizeof(double) * m->ne);
  c->en = (double*)malloc(sizeof(double) * 2 * m->ne);
  c->ectr = (double*)malloc(sizeof(double) * 2 * m->ne);
}

static void mesh_free(o2fo_mesh* c) {
  free(c->vxy);
  free(c->cvol);
  free(c->cctr);
  free(c->elen);
  free(c->en);
  free(c->ectr);
}

/* computeShapeGradient (src/shape_optimization.cpp:942-1016). */
void o2fo_shape_gradient(const o2fo_mesh* m, const o2fo_params* p, const double* U, const double* lambda,
                         const o2fo_shape* s, const int* params, int n, double beta, double eps, double* grad) {
  const int64_t nc = m->nc, ne = m->ne;
  double* Rp = (double*)malloc(sizeof(double) * 4 * nc);
  double* Rm = (double*)malloc(sizeof(double) * 4 * nc);
  double* LR = (double*)malloc(sizeof(double) * 8 * ne);
  double* tau = (double*)malloc(sizeof(double) * 3 * ne);
  o2fo_mesh mp;
  mesh_copy(m, &mp);
  for (int k = 0; k < n; ++k) {
    double Jpm[2], f[3];
    for (int sg = 0; sg < 2; ++sg) {
      o2fo_perturb(m, p, s, params[k], sg == 0 ? eps : -eps, &mp);
      o2fo_residual(&mp, p, U, sg == 0 ? Rp : Rm, NULL, LR, tau, NULL);
      o2fo_forces(&mp, p, LR, tau, beta, f);
      Jpm[sg] = f[2];
    }
    double dot = 0.0;
    for (int64_t i = 0; i < 4 * nc; ++i) dot += lambda[i] * ((Rp[i] - Rm[i]) / (2.0 * eps));
    grad[k] = (Jpm[0] - Jpm[1]) / (2.0 * eps) - dot;
  }
  mesh_free(&mp);
  free(Rp);
  free(Rm);
  free(LR);
  free(tau);
}

static double dot(const double* a, const double* b, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* BiCGSTAB (van der Vorst 1992), identity preconditioner, restarted every
 * `restart` iterations with a true-residual check, as solveAdjointSystem
 * drives Eigen's solver (src/shape_optimization.cpp:693-731). */
int o2fo_bicgstab(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* b, double tol,
                  int64_t max_iter, int64_t restart, double* x, int64_t* iters, double* relres_out) {
  const int64_t n = 4 * m->nc;
  double *r = malloc(sizeof(double) * n), *r0 = malloc(sizeof(double) * n), *pp = malloc(sizeof(double) * n),
         *v = malloc(sizeof(double) * n), *s = malloc(sizeof(double) * n), *t = malloc(sizeof(double) * n);
  memset(x, 0, sizeof(double) * n);
  const double bb = dot(b, b, n), bnorm = sqrt(bb);
  const double tol2 = tol * tol * bb;
  int64_t total = 0;
  double relres = INFINITY;
  if (bb == 0.0) relres = 0.0;
  while (bb > 0.0 && total < max_iter) {
    o2fo_jt(m, p, LR, x, t);
    for (int64_t i = 0; i < n; ++i) {
      r[i] = b[i] - t[i];
      r0[i] = r[i];
      pp[i] = v[i] = 0.0;
    }
    double rr = dot(r, r, n), r0r0 = rr, rho = 1.0, alpha = 1.0, omega = 1.0;
    int64_t it = 0, cap = restart < max_iter - total ? restart : max_iter - total;
    while (rr > tol2 && it < cap) {
      double rho_new = dot(r0, r, n);
      if (fabs(rho_new) < DBL_EPSILON * DBL_EPSILON * r0r0) {
        memcpy(r0, r, sizeof(double) * n);
        rho_new = r0r0 = rr;
      }
      const double beta = (rho_new / rho) * (alpha / omega);
      rho = rho_new;
      for (int64_t i = 0; i < n; ++i) pp[i] = r[i] + beta * (pp[i] - omega * v[i]);
      o2fo_jt(m, p, LR, pp, v);
      alpha = rho / dot(r0, v, n);
      for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
      o2fo_jt(m, p, LR, s, t);
      const double tt = dot(t, t, n);
      omega = tt > 0.0 ? dot(t, s, n) / tt : 0.0;
      for (int64_t i = 0; i < n; ++i) {
        x[i] = x[i] + alpha * pp[i] + omega * s[i];
        r[i] = s[i] - omega * t[i];
      }
      rr = dot(r, r, n);
      ++it;
      if (omega == 0.0) break;
    }
    total += it;
    o2fo_jt(m, p, LR, x, t);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
    relres = sqrt(dot(r, r, n)) / (bnorm > 0 ? bnorm : 1.0);
    if (relres <= tol || !isfinite(relres) || it == 0) break;
  }
  if (iters) *iters = total;
  if (relres_out) *relres_out = relres;
  free(r);
  free(r0);
  free(pp);
  free(v);
  free(s);
  free(t);
  return relres <= tol ? 0 : 1;
}
