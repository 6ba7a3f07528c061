// CUDA kernels of the residual, time step, forces, adjoint operator and shape
// perturbation, templated on the arithmetic type T (double / float).
//
// Every floating-point expression keeps the association order of the
// reference expression it restates (cited per kernel).  The FP64
// instantiation is compiled with -fmad=false, so no multiply-add is fused and
// each operation rounds exactly as the reference's does on x86-64; sqrt and
// division are IEEE round-to-nearest on both sides (quotients that share a
// divisor come from one reciprocal through qdiv, which returns the same bits
// as the division; qdiv.h).  Summations follow the
// reference's Cell::edgeIDs / Vertex::cellIDs order, which the host build
// reproduces (mesh_host.cpp).  The FP64 residual is therefore bit-identical to
// the reference for the same mesh and state.
#pragma once

#include <cfloat>
#include <cstdint>

#include "device_types.hpp"
#include "qdiv.h"

namespace o2f {

constexpr int kBlock = 256;
constexpr double kDblEps = 2.220446049250313080847263336181640625e-16;  // DBL_EPSILON

// Gate: when `gate` is non-null and *gate != 0 the kernel does nothing.  Used
// by the device-driven loops (time stepping, BiCGSTAB) to turn the launches
// that follow a stop condition into no-ops.
__device__ __forceinline__ bool gated(const int* gate) { return gate != nullptr && *(volatile const int*)gate != 0; }

// std::min / std::max / std::clamp semantics (NaN propagation included).
template <typename T>
__device__ __forceinline__ T smin(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__device__ __forceinline__ T smax(T a, T b) { return (a < b) ? b : a; }
template <typename T>
__device__ __forceinline__ T sclamp(T v, T lo, T hi) { return (v < lo) ? lo : (hi < v) ? hi : v; }

template <typename T>
__device__ __forceinline__ Vec4<T> v4(T a, T b, T c, T d) {
  Vec4<T> r;
  r.a = a;
  r.b = b;
  r.c = c;
  r.d = d;
  return r;
}

// apply_inflow_outflow_bc (src/boundary.cpp:7-45): inlet / far field take the
// freestream, outlet keeps the state, a wall keeps rho and the internal energy
// with zero momentum.
template <typename T>
__device__ __forceinline__ void bc_state(uint8_t code, const Phys& ph, T& r, T& ru, T& rv, T& E) {
  if (code == 'i' || code == 'f') {
    r = (T)ph.fs_rho;
    ru = (T)ph.fs_rhou;
    rv = (T)ph.fs_rhov;
    E = (T)ph.fs_E;
  } else if (code == 'w') {
    const T kinetic_old = (T)0.5 * (ru * ru + rv * rv) / r;
    const T e_internal = E - kinetic_old;
    ru = (T)0.0;
    rv = (T)0.0;
    E = e_internal;
  }
}

// apply_InterfaceStates_boundary_conditions (src/boundary.cpp:48-80): the
// ghost right state of a boundary edge built from its left state.
template <typename T>
__device__ __forceinline__ Vec4<T> bc_ghost(uint8_t code, const Phys& ph, const Vec4<T>& L) {
  Vec4<T> R = L;
  if (code == 'i' || code == 'o' || code == 'f') {
    bc_state(code, ph, R.a, R.b, R.c, R.d);
  } else if (code == 'w') {
    R.b = -L.b;
    R.c = -L.c;
  }
  return R;
}

// pressure / sound_speed (src/advection.cpp:325-332).
template <typename T>
__device__ __forceinline__ T pressure(T rho, T u, T v, T E, T gamma) {
  const T kinetic = (T)0.5 * rho * (u * u + v * v);
  return (gamma - (T)1.0) * (E - kinetic);
}

// compute_hllc_flux (src/advection.cpp:335-412): rotated HLLC with the normal
// -edgeNormal, Davis wave speeds, flux rotated back.
template <typename T>
__device__ __forceinline__ Vec4<T> hllc(const Vec4<T>& Ls, const Vec4<T>& Rs, T enx, T eny, T gamma) {
  const T nx = -enx, ny = -eny;
  const T rho_L = Ls.a;
  const T u_L = (Ls.b * (nx) + Ls.c * ny) / rho_L;
  const T v_L = (Ls.b * (-ny) + Ls.c * nx) / rho_L;
  const T E_L = Ls.d;
  const T p_L = pressure(rho_L, u_L, v_L, E_L, gamma);
  const T c_L = sqrt(gamma * p_L / rho_L);
  const T rho_R = Rs.a;
  const T u_R = (Rs.b * (nx) + Rs.c * ny) / rho_R;
  const T v_R = (Rs.b * (-ny) + Rs.c * nx) / rho_R;
  const T E_R = Rs.d;
  const T p_R = pressure(rho_R, u_R, v_R, E_R, gamma);
  const T c_R = sqrt(gamma * p_R / rho_R);

  const T S_L = smin(u_L - c_L, u_R - c_R);
  const T S_R = smax(u_L + c_L, u_R + c_R);
  const T numer = p_R - p_L + rho_L * u_L * (S_L - u_L) - rho_R * u_R * (S_R - u_R);
  const T denom = rho_L * (S_L - u_L) - rho_R * (S_R - u_R);
  const T S_star = numer / denom;
  const T rho_L_star = rho_L * (S_L - u_L) / (S_L - S_star);
  const T rho_R_star = rho_R * (S_R - u_R) / (S_R - S_star);
  const T rho_v_L_star = rho_L_star * v_L;
  const T rho_v_R_star = rho_R_star * v_R;
  const T p_star = p_L + rho_L * (S_L - u_L) * (S_star - u_L);
  const T E_L_star = ((S_L - u_L) * E_L - p_L * u_L + p_star * S_star) / (S_L - S_star);
  const T E_R_star = ((S_R - u_R) * E_R - p_R * u_R + p_star * S_star) / (S_R - S_star);
  const T rho_u_L_star = rho_L_star * S_star;
  const T rho_u_R_star = rho_R_star * S_star;

  T f_rho, f_u, f_v, f_E;
  if (S_L >= (T)0.0) {
    f_rho = rho_L * u_L;
    f_u = rho_L * u_L * u_L + p_L;
    f_v = rho_L * u_L * v_L;
    f_E = (E_L + p_L) * u_L;
  } else if (S_L <= (T)0.0 && S_star >= (T)0.0) {
    f_rho = rho_u_L_star;
    f_u = rho_u_L_star * rho_u_L_star / rho_L_star + p_star;
    f_v = rho_v_L_star * rho_u_L_star / rho_L_star;
    f_E = (E_L_star + p_star) * rho_u_L_star / rho_L_star;
  } else if (S_star <= (T)0.0 && S_R >= (T)0.0) {
    f_rho = rho_u_R_star;
    f_u = rho_u_R_star * rho_u_R_star / rho_R_star + p_star;
    f_v = rho_v_R_star * rho_u_R_star / rho_R_star;
    f_E = (E_R_star + p_star) * rho_u_R_star / rho_R_star;
  } else {
    f_rho = rho_R * u_R;
    f_u = rho_R * u_R * u_R + p_R;
    f_v = rho_R * u_R * v_R;
    f_E = (E_R + p_R) * u_R;
  }
  return v4<T>(f_rho, (f_u * nx + f_v * (-ny)), (f_u * ny + f_v * (nx)), f_E);
}

// computeVenkatAlpha (src/advection.cpp:209-230) with eps = (k h)^3
// precomputed per cell; computeBarthJespersenAlpha (:195-207).
template <typename T>
__device__ __forceinline__ T limiter_alpha(int kind, T phi_i, T phi_pred, T phi_min, T phi_max, T eps) {
  if (kind == 0) {
    const T delta = phi_pred - phi_i;
    if (fabs(delta) < (T)kDblEps) return (T)1.0;
    T a = (delta > (T)0.0) ? (phi_max - phi_i) : (phi_min - phi_i);
    const T d = delta;
    T alpha = (a * a + eps + (T)2.0 * a * d) / (a * a + eps + (T)2.0 * d * d);
    return sclamp(alpha, (T)0.0, (T)1.0);
  }
  T alpha = (T)1.0;
  if (fabs(phi_pred - phi_i) < (T)kDblEps) return alpha;
  if (phi_pred > phi_i) {
    alpha = smin((T)1.0, (phi_max - phi_i) / (phi_pred - phi_i));
  } else if (phi_pred < phi_i) {
    alpha = smin((T)1.0, (phi_min - phi_i) / (phi_pred - phi_i));
  }
  return alpha;
}

// ---------------------------------------------------------------------------
// K1: cell -> vertex interpolation of the state (src/advection.cpp:26-131),
// weights precomputed in the reference's order, then the vertex boundary
// override (:129-130).  The generic weighted sum reproduces every valence case
// of the reference exactly: w=1 copies, w=0.5 halves, and the 3- and 4-cell
// sums keep the reference's left-to-right association.
template <typename T>
__device__ __forceinline__ void vertex_state_at(int64_t v, int64_t nv, const int32_t* __restrict__ voff,
                                                         const int32_t* __restrict__ vcid,
                                                         const T* __restrict__ vw,
                                                         const uint8_t* __restrict__ vbc,
                                                         const Vec4<T>* __restrict__ U, Phys ph,
                                                         Vec4<T>* __restrict__ vq) {
  const int o0 = voff[v], o1 = voff[v + 1];
  T a = (T)0.0, b = (T)0.0, c = (T)0.0, d = (T)0.0;
  if (o1 > o0) {
    T w = vw[o0];
    Vec4<T> u = U[vcid[o0]];
    a = w * u.a;
    b = w * u.b;
    c = w * u.c;
    d = w * u.d;
    for (int k = o0 + 1; k < o1; ++k) {
      w = vw[k];
      u = U[vcid[k]];
      a = a + w * u.a;
      b = b + w * u.b;
      c = c + w * u.c;
      d = d + w * u.d;
    }
  }
  const uint8_t code = vbc[v];
  if (code) bc_state(code, ph, a, b, c, d);
  vq[v] = v4<T>(a, b, c, d);
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_vertex_state(int64_t nv, const int32_t* __restrict__ voff,
                                                         const int32_t* __restrict__ vcid,
                                                         const T* __restrict__ vw,
                                                         const uint8_t* __restrict__ vbc,
                                                         const Vec4<T>* __restrict__ U, Phys ph,
                                                         Vec4<T>* __restrict__ vq, const int* gate) {
  if (gated(gate)) return;
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  vertex_state_at<T>(v, nv, voff, vcid, vw, vbc, U, ph, vq);
}

// K3: the same interpolation for the five viscous quantities
// (src/diffusion.cpp:29-140) with apply_diffusion_bc (src/boundary.cpp:101-127):
// far field and wall vertices are zeroed.
template <typename T>
__device__ __forceinline__ void vertex_visc_at(int64_t v, int64_t nv, const int32_t* __restrict__ voff,
                                                        const int32_t* __restrict__ vcid,
                                                        const T* __restrict__ vw,
                                                        const uint8_t* __restrict__ vbc,
                                                        const Vec4<T>* __restrict__ ctq,
                                                        const T* __restrict__ ctqy,
                                                        Vec4<T>* __restrict__ vtq, T* __restrict__ vtqy) {
  const int o0 = voff[v], o1 = voff[v + 1];
  T a = (T)0.0, b = (T)0.0, c = (T)0.0, d = (T)0.0, e = (T)0.0;
  if (o1 > o0) {
    T w = vw[o0];
    int cid = vcid[o0];
    Vec4<T> t = ctq[cid];
    T q = ctqy[cid];
    a = w * t.a;
    b = w * t.b;
    c = w * t.c;
    d = w * t.d;
    e = w * q;
    for (int k = o0 + 1; k < o1; ++k) {
      w = vw[k];
      cid = vcid[k];
      t = ctq[cid];
      q = ctqy[cid];
      a = a + w * t.a;
      b = b + w * t.b;
      c = c + w * t.c;
      d = d + w * t.d;
      e = e + w * q;
    }
  }
  const uint8_t code = vbc[v];
  if (code == 'f' || code == 'w') a = b = c = d = e = (T)0.0;
  vtq[v] = v4<T>(a, b, c, d);
  vtqy[v] = e;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_vertex_visc(int64_t nv, const int32_t* __restrict__ voff,
                                                        const int32_t* __restrict__ vcid,
                                                        const T* __restrict__ vw,
                                                        const uint8_t* __restrict__ vbc,
                                                        const Vec4<T>* __restrict__ ctq,
                                                        const T* __restrict__ ctqy,
                                                        Vec4<T>* __restrict__ vtq, T* __restrict__ vtqy,
                                                        const int* gate) {
  if (gated(gate)) return;
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  vertex_visc_at<T>(v, nv, voff, vcid, vw, vbc, ctq, ctqy, vtq, vtqy);
}

// K2: per cell -- edge values from the vertex states and the Green-Gauss
// gradient (src/advection.cpp:136-188), neighbour min/max, limiter and
// interface states (:236-321), and the cell viscous stress and heat flux from
// the unlimited gradients (src/diffusion.cpp:223-241).
//
// kPlain = false divides the Green-Gauss terms by the volume through one
// reciprocal (qdiv_flag) and returns false, having written nothing, if any
// quotient left qdiv's range; cell_gradient_at then redoes the cell with
// kPlain = true (IEEE divisions), out of line.
//
// kAlpha (linearisations only; 0 everywhere else): 1 stores the limiter
// values of the cell in alpha[c], 2 uses alpha[c] instead of computing them
// (the limiter held at a base state).
template <typename T, bool kWriteGrad, bool kPlain, int kAlpha = 0>
__device__ __forceinline__ bool cell_gradient_body(int64_t c,
    int64_t nc, const int32_t* __restrict__ slot, Geom<T> g, const int2* __restrict__ ev,
    const int2* __restrict__ ec, const uint8_t* __restrict__ ebc, const Vec4<T>* __restrict__ U,
    const Vec4<T>* __restrict__ vq, Phys ph, Vec4<T>* __restrict__ eL, Vec4<T>* __restrict__ eR,
    Vec4<T>* __restrict__ ctq, T* __restrict__ ctqy, Vec4<T>* __restrict__ grad, Vec4<T>* __restrict__ alpha = nullptr) {
  const Vec4<T> cg = g.cgeom[c];
  const T cx = cg.a, cy = cg.b, cv = cg.c, veps = cg.d;
  const Vec4<T> u = U[c];
  // The cell's edges are the slots before the first empty one.  All index
  // and geometry loads of every edge are issued before the arithmetic, so
  // the gathers of one cell overlap instead of forming one chain per edge.
  int sl[4], nk = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) sl[k] = slot[(int64_t)k * nc + c];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (sl[k] >= 0 && nk == k) nk = k + 1;
  int2 evv[4], cc[4];
  uint8_t code[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k < nk) {
      const int e = sl[k] >> 1;
      evv[k] = ev[e];
      cc[k] = ec[e];
      code[k] = ebc[e];
    }
  }

  // the eight Green-Gauss terms of every edge divide by the cell volume
  const T ycv = recip_for_div(cv);
  bool ok = true;
  auto over_v = [&](T a) -> T {
    if constexpr (kPlain) return a / cv;
    else return qdiv_flag(a, cv, ycv, ok);
  };
  T gx0 = (T)0.0, gx1 = (T)0.0, gx2 = (T)0.0, gx3 = (T)0.0;
  T gy0 = (T)0.0, gy1 = (T)0.0, gy2 = (T)0.0, gy3 = (T)0.0;
  T mn0 = u.a, mn1 = u.b, mn2 = u.c, mn3 = u.d;
  T mx0 = u.a, mx1 = u.b, mx2 = u.c, mx3 = u.d;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= nk) continue;
    const int s = sl[k];
    const int e = s >> 1;
    const bool left = (s & 1) == 0;
    const Vec4<T> va = vq[evv[k].x], vb = vq[evv[k].y];
    const Vec4<T> eg = g.egeom[e];
    const int o = left ? cc[k].y : cc[k].x;
    Vec4<T> un = u;
    if (o >= 0) un = U[o];
    T er = (T)0.5 * (va.a + vb.a);
    T eru = (T)0.5 * (va.b + vb.b);
    T erv = (T)0.5 * (va.c + vb.c);
    T eE = (T)0.5 * (va.d + vb.d);
    if (code[k]) bc_state(code[k], ph, er, eru, erv, eE);
    const T el = eg.c;
    T enx = eg.a, eny = eg.b;
    if (left) {
      enx = -enx;
      eny = -eny;
    }
    gx0 += over_v(er * el * enx);
    gx1 += over_v(eru * el * enx);
    gx2 += over_v(erv * el * enx);
    gx3 += over_v(eE * el * enx);
    gy0 += over_v(er * el * eny);
    gy1 += over_v(eru * el * eny);
    gy2 += over_v(erv * el * eny);
    gy3 += over_v(eE * el * eny);
    if (o >= 0) {
      if (un.a < mn0) mn0 = un.a;
      if (un.a > mx0) mx0 = un.a;
      if (un.b < mn1) mn1 = un.b;
      if (un.b > mx1) mx1 = un.b;
      if (un.c < mn2) mn2 = un.c;
      if (un.c > mx2) mx2 = un.c;
      if (un.d < mn3) mn3 = un.d;
      if (un.d > mx3) mx3 = un.d;
    }
  }

  if (!kPlain && !ok) return false;

  const int kind = ph.limiter;
  T al0 = (T)1.0, al1 = (T)1.0, al2 = (T)1.0, al3 = (T)1.0;
  T dxk[4], dyk[4];
  if constexpr (kAlpha == 2) {
    const Vec4<T> a = alpha[c];
    al0 = a.a;
    al1 = a.b;
    al2 = a.c;
    al3 = a.d;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= nk) continue;
      const Vec2<T> ce = g.ectr[sl[k] >> 1];
      dxk[k] = ce.a - cx;
      dyk[k] = ce.b - cy;
    }
    (void)kind;
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= nk) continue;
      const Vec2<T> ce = g.ectr[sl[k] >> 1];
      const T dx = ce.a - cx, dy = ce.b - cy;
      dxk[k] = dx;
      dyk[k] = dy;
      al0 = smin(al0, limiter_alpha(kind, u.a, u.a + gx0 * dx + gy0 * dy, mn0, mx0, veps));
      al1 = smin(al1, limiter_alpha(kind, u.b, u.b + gx1 * dx + gy1 * dy, mn1, mx1, veps));
      al2 = smin(al2, limiter_alpha(kind, u.c, u.c + gx2 * dx + gy2 * dy, mn2, mx2, veps));
      al3 = smin(al3, limiter_alpha(kind, u.d, u.d + gx3 * dx + gy3 * dy, mn3, mx3, veps));
    }
    if constexpr (kAlpha == 1) alpha[c] = v4<T>(al0, al1, al2, al3);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (k >= nk) continue;
    const int s = sl[k];
    const int e = s >> 1;
    const T dx = dxk[k], dy = dyk[k];
    const Vec4<T> st = v4<T>(u.a + al0 * (gx0 * dx + gy0 * dy), u.b + al1 * (gx1 * dx + gy1 * dy),
                             u.c + al2 * (gx2 * dx + gy2 * dy), u.d + al3 * (gx3 * dx + gy3 * dy));
    if ((s & 1) == 0) {
      eL[e] = st;
      if (code[k]) eR[e] = bc_ghost(code[k], ph, st);
    } else {
      eR[e] = st;
    }
  }

  // Viscous stress and heat flux at the cell (src/diffusion.cpp:227-240).
  const T mu = (T)ph.mu, gamma = (T)ph.gamma, kappa = (T)ph.kappa;
  const T yrho = recip_for_div(u.a);
  const T uu = qdiv(u.b, u.a, yrho);
  const T vv = qdiv(u.c, u.a, yrho);
  const T u_x = qdiv(gx1 - uu * gx0, u.a, yrho);
  const T v_y = qdiv(gy2 - vv * gy0, u.a, yrho);
  const T u_y = qdiv(gy1 - uu * gy0, u.a, yrho);
  const T v_x = qdiv(gx2 - vv * gx0, u.a, yrho);
  const T two_thirds = (T)(2.0 / 3.0);
  const T tau_xx = (T)2 * mu * u_x - two_thirds * mu * (u_x + v_y);
  const T tau_yy = (T)2 * mu * v_y - two_thirds * mu * (u_x + v_y);
  const T tau_xy = mu * (u_y + v_x);
  const T T_x = (gamma - (T)1.0) * ((gx3 * u.a - u.d * gx0) / (u.a * u.a) - (uu * u_x + vv * v_x));
  const T T_y = (gamma - (T)1.0) * ((gy3 * u.a - u.d * gy0) / (u.a * u.a) - (uu * u_y + vv * v_y));
  ctq[c] = v4<T>(tau_xx, tau_yy, tau_xy, -kappa * T_x);
  ctqy[c] = -kappa * T_y;
  if (kWriteGrad) {
    grad[2 * c] = v4<T>(gx0, gx1, gx2, gx3);
    grad[2 * c + 1] = v4<T>(gy0, gy1, gy2, gy3);
  }
  return true;
}

template <typename T, bool kWriteGrad, int kAlpha = 0>
__device__ __noinline__ void cell_gradient_plain(int64_t c,
    int64_t nc, const int32_t* __restrict__ slot, Geom<T> g, const int2* __restrict__ ev,
    const int2* __restrict__ ec, const uint8_t* __restrict__ ebc, const Vec4<T>* __restrict__ U,
    const Vec4<T>* __restrict__ vq, Phys ph, Vec4<T>* __restrict__ eL, Vec4<T>* __restrict__ eR,
    Vec4<T>* __restrict__ ctq, T* __restrict__ ctqy, Vec4<T>* __restrict__ grad, Vec4<T>* __restrict__ alpha) {
  cell_gradient_body<T, kWriteGrad, true, kAlpha>(c, nc, slot, g, ev, ec, ebc, U, vq, ph, eL, eR, ctq, ctqy, grad,
                                                  alpha);
}

template <typename T, bool kWriteGrad, int kAlpha = 0>
__device__ __forceinline__ void cell_gradient_at(int64_t c,
    int64_t nc, const int32_t* __restrict__ slot, Geom<T> g, const int2* __restrict__ ev,
    const int2* __restrict__ ec, const uint8_t* __restrict__ ebc, const Vec4<T>* __restrict__ U,
    const Vec4<T>* __restrict__ vq, Phys ph, Vec4<T>* __restrict__ eL, Vec4<T>* __restrict__ eR,
    Vec4<T>* __restrict__ ctq, T* __restrict__ ctqy, Vec4<T>* __restrict__ grad,
    Vec4<T>* __restrict__ alpha = nullptr) {
  if (!cell_gradient_body<T, kWriteGrad, false, kAlpha>(c, nc, slot, g, ev, ec, ebc, U, vq, ph, eL, eR, ctq, ctqy, grad,
                                                        alpha))
    cell_gradient_plain<T, kWriteGrad, kAlpha>(c, nc, slot, g, ev, ec, ebc, U, vq, ph, eL, eR, ctq, ctqy, grad, alpha);
}

template <typename T, bool kWriteGrad>
__global__ void __launch_bounds__(kBlock, 3) k_cell_gradient(
    int64_t nc, const int32_t* __restrict__ slot, Geom<T> g, const int2* __restrict__ ev,
    const int2* __restrict__ ec, const uint8_t* __restrict__ ebc, const Vec4<T>* __restrict__ U,
    const Vec4<T>* __restrict__ vq, Phys ph, Vec4<T>* __restrict__ eL, Vec4<T>* __restrict__ eR,
    Vec4<T>* __restrict__ ctq, T* __restrict__ ctqy, Vec4<T>* __restrict__ grad, const int* gate) {
  if (gated(gate)) return;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  cell_gradient_at<T, kWriteGrad>(c, nc, slot, g, ev, ec, ebc, U, vq, ph, eL, eR, ctq, ctqy, grad);
}

// K4: per edge -- HLLC flux (src/advection.cpp:433-437) and the edge viscous
// quantities with their boundary conditions (src/diffusion.cpp:145-170).
template <typename T>
__device__ __forceinline__ void edge_flux_at(int64_t e, int64_t ne, Geom<T> g, const int2* __restrict__ ev,
                                                      const uint8_t* __restrict__ ebc,
                                                      const Vec4<T>* __restrict__ eL,
                                                      const Vec4<T>* __restrict__ eR,
                                                      const Vec4<T>* __restrict__ vtq,
                                                      const T* __restrict__ vtqy, Phys ph,
                                                      Vec4<T>* __restrict__ F, Vec4<T>* __restrict__ etq,
                                                      T* __restrict__ etqy) {
  const Vec4<T> eg = g.egeom[e];
  F[e] = hllc(eL[e], eR[e], eg.a, eg.b, (T)ph.gamma);
  const int2 vv = ev[e];
  const Vec4<T> a = vtq[vv.x], b = vtq[vv.y];
  T txx = (T)0.5 * (a.a + b.a);
  T tyy = (T)0.5 * (a.b + b.b);
  T txy = (T)0.5 * (a.c + b.c);
  T qx = (T)0.5 * (a.d + b.d);
  T qy = (T)0.5 * (vtqy[vv.x] + vtqy[vv.y]);
  const uint8_t code = ebc[e];
  if (code == 'f' || code == 'w') txx = tyy = txy = qx = qy = (T)0.0;
  etq[e] = v4<T>(txx, tyy, txy, qx);
  etqy[e] = qy;
}

template <typename T>
__global__ void __launch_bounds__(kBlock, 4) k_edge_flux(int64_t ne, Geom<T> g, const int2* __restrict__ ev,
                                                      const uint8_t* __restrict__ ebc,
                                                      const Vec4<T>* __restrict__ eL,
                                                      const Vec4<T>* __restrict__ eR,
                                                      const Vec4<T>* __restrict__ vtq,
                                                      const T* __restrict__ vtqy, Phys ph,
                                                      Vec4<T>* __restrict__ F, Vec4<T>* __restrict__ etq,
                                                      T* __restrict__ etqy, const int* gate) {
  if (gated(gate)) return;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  edge_flux_at<T>(e, ne, g, ev, ebc, eL, eR, vtq, vtqy, ph, F, etq, etqy);
}

// Partial sum of squares of a block, written to part[blockIdx.x].
__device__ __forceinline__ double block_sum(double v, double* smem) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += smem[w];
  }
  return s;  // valid in thread 0
}

// RK3 stage parameters for the fused residual + update.
struct RkStage {
  double c0, c1;        // U = c0*U_old + c1*(U + dt*R)
  const double* dt;     // device scalar
  int snapshot;         // 1: copy U to U_old first (stage 1)
  double* norm_part;    // per-block partial sums of R_rho^2 (stage 1), or null
};

// K5: per cell -- residual gather R = -(1/V) sum sign*F*L
// (src/advection.cpp:439-464), then the viscous Green-Gauss divergence added
// to R (src/diffusion.cpp:176-201).  kRk fuses the SSP-RK3 stage update of
// Simulator::rk3_substep (src/simulation.cpp:159-167).
// Returns R_rho^2 of cell c for the residual-norm partial sums (0 unless
// kRk with norm partials requested).
template <typename T, bool kRk>
__device__ __forceinline__ double cell_residual_at(int64_t c, int64_t nc, const int32_t* __restrict__ slot, Geom<T> g,
                                                   const Vec4<T>* __restrict__ F, const Vec4<T>* __restrict__ etq,
                                                   const T* __restrict__ etqy, Vec4<T>* __restrict__ U,
                                                   Vec4<T>* __restrict__ Uold, Vec4<T>* __restrict__ R,
                                                   const RkStage& rk) {
  double r2 = 0.0;
  const T cv = g.cgeom[c].c;
  int sl[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) sl[k] = slot[(int64_t)k * nc + c];
  T a0 = (T)0.0, a1 = (T)0.0, a2 = (T)0.0, a3 = (T)0.0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int s = sl[k];
    if (s < 0) break;
    const int e = s >> 1;
    const T sign = ((s & 1) == 0) ? (T)1.0 : (T)-1.0;
    const T L = g.egeom[e].c;
    const Vec4<T> f = F[e];
    a0 += sign * f.a * L;
    a1 += sign * f.b * L;
    a2 += sign * f.c * L;
    a3 += sign * f.d * L;
  }
  const T invV = (T)1.0 / cv;
  const T ycv = recip_for_div(cv, invV);
  a0 *= -invV;
  a1 *= -invV;
  a2 *= -invV;
  a3 *= -invV;
  Vec4<T> u = U[c];
  const T uu = u.b / u.a;
  const T vv = u.c / u.a;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int s = sl[k];
    if (s < 0) break;
    const int e = s >> 1;
    const Vec4<T> eg = g.egeom[e];
    const T el = eg.c;
    T enx = eg.a, eny = eg.b;
    if ((s & 1) == 0) {
      enx = -enx;
      eny = -eny;
    }
    const Vec4<T> t = etq[e];
    const T qy = etqy[e];
    a1 += qdiv(t.a * el * enx, cv, ycv) + qdiv(t.c * el * eny, cv, ycv);
    a2 += qdiv(t.c * el * enx, cv, ycv) + qdiv(t.b * el * eny, cv, ycv);
    a3 += qdiv((uu * t.a + vv * t.c - t.d) * el * enx, cv, ycv) +
          qdiv((uu * t.c + vv * t.b - qy) * el * eny, cv, ycv);
  }
  R[c] = v4<T>(a0, a1, a2, a3);
  if (kRk) {
    if (rk.norm_part) r2 = (double)a0 * (double)a0;
    const T dt = (T)(*rk.dt);
    const T c0 = (T)rk.c0, c1 = (T)rk.c1;
    Vec4<T> uo;
    if (rk.snapshot) {
      uo = u;
      Uold[c] = u;
    } else {
      uo = Uold[c];
    }
    u.a = c0 * uo.a + c1 * (u.a + dt * (a0));
    u.b = c0 * uo.b + c1 * (u.b + dt * (a1));
    u.c = c0 * uo.c + c1 * (u.c + dt * (a2));
    u.d = c0 * uo.d + c1 * (u.d + dt * (a3));
    U[c] = u;
  }
  return r2;
}

template <typename T, bool kRk>
__global__ void __launch_bounds__(kBlock) k_cell_residual(int64_t nc, const int32_t* __restrict__ slot, Geom<T> g,
                                                          const Vec4<T>* __restrict__ F,
                                                          const Vec4<T>* __restrict__ etq,
                                                          const T* __restrict__ etqy, Vec4<T>* __restrict__ U,
                                                          Vec4<T>* __restrict__ Uold, Vec4<T>* __restrict__ R,
                                                          RkStage rk, const int* gate) {
  __shared__ double smem[kBlock / 32];
  if (gated(gate)) return;
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double r2 = 0.0;
  if (c < nc) r2 = cell_residual_at<T, kRk>(c, nc, slot, g, F, etq, etqy, U, Uold, R, rk);
  if (kRk && rk.norm_part) {
    const double s = block_sum(r2, smem);
    if (threadIdx.x == 0) rk.norm_part[blockIdx.x] = s;
  }
}

}  // namespace o2f
