// Headless field image: the reference's live SFML view (Simulator::output_step,
// src/simulation.cpp:176-199) as an RGB buffer, with no window.
//   * cell scalar: computeCellScalar (src/compute.cpp:6-60);
//   * pixel -> cell: the cell containing the pixel centre
//     x = x_min + (i + 0.5) Lx / Nx, y = y_min + (j + 0.5) Ly / Ny
//     (Mesh::pixelToPhysical, src/mesh.cpp:349-353), with the reference's
//     point-in-triangle test (pointInTriangle, :401-411; a quadrilateral is the
//     triangles (A,B,C) and (A,C,D), :446-452).  Here every cell scans the
//     pixels of its bounding box on the GPU; a pixel inside several cells
//     (on a shared edge) takes the lowest cell number, one inside none is
//     black (the reference's search returns -1 there through its border
//     cells);
//   * colour: render_scalar_field_unstructured (src/renderer_colormap.cpp:
//     10-47) with colormap_B_W_R and colormap_schlieren_bluewhite
//     (include/renderer_colormap.hpp:16-95), whose interpolation runs in
//     float as the reference's lerp(float, float, float) does; image row
//     ny-1-j holds pixel row j.
// Included by solver.cu only (non-template kernels).
#pragma once

#include <climits>

#include "kernels.cuh"

namespace o2f {

enum RenderField : int {
  kFieldRho = 0, kFieldRhoU, kFieldRhoV, kFieldE, kFieldU, kFieldV, kFieldUx, kFieldUy, kFieldVx, kFieldVy,
  kFieldDiv, kFieldP
};

// computeCellScalar for one cell; grad = (x-gradients, y-gradients) of the
// conserved variables from the last residual (gradient fields only).
__global__ void k_cell_scalar(int64_t nc, const Vec4<double>* __restrict__ U, const Vec4<double>* __restrict__ grad,
                              int field, double gamma, double* __restrict__ out) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const Vec4<double> q = U[c];
  double u = 0.0, v = 0.0;
  if (q.a != 0.0) {
    u = q.b / q.a;
    v = q.c / q.a;
  }
  const double rho_div = q.a != 0.0 ? q.a : 1.0;
  double s = 0.0;
  switch (field) {
    case kFieldRho: s = q.a; break;
    case kFieldRhoU: s = q.b; break;
    case kFieldRhoV: s = q.c; break;
    case kFieldE: s = q.d; break;
    case kFieldU: s = u; break;
    case kFieldV: s = v; break;
    case kFieldP: {
      const double kinetic = 0.5 * (q.b * q.b + q.c * q.c) / q.a;
      s = (gamma - 1.0) * (q.d - kinetic);
      break;
    }
    default: {
      const Vec4<double> gx = grad[2 * c], gy = grad[2 * c + 1];  // .a rho, .b rho_u, .c rho_v
      const double u_x = (gx.b - u * gx.a) / rho_div;
      const double u_y = (gy.b - u * gy.a) / rho_div;
      const double v_x = (gx.c - v * gx.a) / rho_div;
      const double v_y = (gy.c - v * gy.a) / rho_div;
      if (field == kFieldUx) s = u_x;
      else if (field == kFieldUy) s = u_y;
      else if (field == kFieldVx) s = v_x;
      else if (field == kFieldVy) s = v_y;
      else s = u_x + v_y;
    }
  }
  out[c] = s;
}

// Per-block min and max of the cell scalar (the reference's
// "if (min > s) min = s; if (max < s) max = s").
__global__ void __launch_bounds__(kBlock) k_scalar_minmax(int64_t n, const double* __restrict__ s,
                                                          double* __restrict__ part) {
  __shared__ double smn[kBlock], smx[kBlock];
  double mn = INFINITY, mx = -INFINITY;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double x = s[i];
    if (mn > x) mn = x;
    if (mx < x) mx = x;
  }
  smn[threadIdx.x] = mn;
  smx[threadIdx.x] = mx;
  __syncthreads();
  for (int o = kBlock / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      if (smn[threadIdx.x] > smn[threadIdx.x + o]) smn[threadIdx.x] = smn[threadIdx.x + o];
      if (smx[threadIdx.x] < smx[threadIdx.x + o]) smx[threadIdx.x] = smx[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = smn[0];
    part[2 * blockIdx.x + 1] = smx[0];
  }
}

struct RenderView {
  double x_min, y_min, Lx, Ly;
  int nx, ny;
};

// pointInTriangle (src/mesh.cpp:401-411).
__device__ __forceinline__ bool point_in_triangle(double x, double y, Vec2<double> v0, Vec2<double> v1,
                                                  Vec2<double> v2) {
  const double dX = x - v2.a, dY = y - v2.b;
  const double dX21 = v2.a - v1.a, dY12 = v1.b - v2.b;
  double D = dY12 * (v0.a - v2.a) + dX21 * (v0.b - v2.b);
  double s = dY12 * dX + dX21 * dY;
  double t = (v2.b - v0.b) * dX + (v0.a - v2.a) * dY;
  if (D < 0) {
    s = -s;
    t = -t;
    D = -D;
  }
  return (s >= 0 && t >= 0 && (s + t) <= D);
}

// Every cell marks the pixels whose centre it contains; the key keeps the
// lowest mesh-file cell number and carries the device cell index.
__global__ void k_raster_cells(int64_t nc, const int32_t* __restrict__ cverts, const uint8_t* __restrict__ ctype,
                               const Vec2<double>* __restrict__ vxy, const int32_t* __restrict__ ref_id, RenderView w,
                               unsigned long long* __restrict__ pix) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int n = ctype[c];
  Vec2<double> p[4];
  double xlo = INFINITY, xhi = -INFINITY, ylo = INFINITY, yhi = -INFINITY;
  for (int k = 0; k < n; ++k) {
    p[k] = vxy[cverts[4 * c + k]];
    xlo = fmin(xlo, p[k].a);
    xhi = fmax(xhi, p[k].a);
    ylo = fmin(ylo, p[k].b);
    yhi = fmax(yhi, p[k].b);
  }
  // pixel centres inside the bounding box (one pixel of margin each way;
  // the exact test below decides)
  const int i0 = max(0, (int)floor((xlo - w.x_min) / w.Lx * w.nx - 0.5) - 1);
  const int i1 = min(w.nx - 1, (int)floor((xhi - w.x_min) / w.Lx * w.nx - 0.5) + 1);
  const int j0 = max(0, (int)floor((ylo - w.y_min) / w.Ly * w.ny - 0.5) - 1);
  const int j1 = min(w.ny - 1, (int)floor((yhi - w.y_min) / w.Ly * w.ny - 0.5) + 1);
  const unsigned long long key = ((unsigned long long)(uint32_t)ref_id[c] << 32) | (uint32_t)c;
  for (int j = j0; j <= j1; ++j) {
    const double y = w.y_min + (j + 0.5) * w.Ly / w.ny;
    for (int i = i0; i <= i1; ++i) {
      const double x = w.x_min + (i + 0.5) * w.Lx / w.nx;
      const bool in = (n == 3) ? point_in_triangle(x, y, p[0], p[1], p[2])
                               : (point_in_triangle(x, y, p[0], p[1], p[2]) || point_in_triangle(x, y, p[0], p[2], p[3]));
      if (in) atomicMin(&pix[(int64_t)j * w.nx + i], key);
    }
  }
}

// lerp(float, float, float) of the reference's colour maps.
__device__ __forceinline__ float cmap_lerp(float a, float b, float t) { return a + (b - a) * t; }

__device__ __forceinline__ unsigned char cmap_to8(double x) {
  return (unsigned char)(fmax(0.0, fmin(1.0, x)) * 255.0 + 0.5);
}

// colormap_B_W_R: blue - white - red.
__device__ void cmap_bwr(double t_, unsigned char* rgb) {
  const double t = fmax(0.0, fmin(1.0, t_));
  double b, g, r;
  if (t < 0.25) b = cmap_lerp(0.3f, 1.0f, (float)(t / 0.25));
  else if (t < 0.5) b = 1.0;
  else if (t < 0.75) b = cmap_lerp(1.0f, 0.0f, (float)((t - 0.5) / 0.25));
  else b = 0.0;
  if (t < 0.25) g = 0.0;
  else if (t < 0.5) g = cmap_lerp(0.0f, 1.0f, (float)((t - 0.25) / 0.25));
  else if (t < 0.75) g = cmap_lerp(1.0f, 0.0f, (float)((t - 0.5) / 0.25));
  else g = 0.0;
  if (t < 0.25) r = 0.0;
  else if (t < 0.5) r = cmap_lerp(0.0f, 1.0f, (float)((t - 0.25) / 0.25));
  else if (t < 0.75) r = 1.0;
  else r = cmap_lerp(1.0f, 0.5f, (float)((t - 0.75) / 0.25));
  rgb[0] = cmap_to8(r);
  rgb[1] = cmap_to8(g);
  rgb[2] = cmap_to8(b);
}

// colormap_schlieren_bluewhite: black - blue - white.
__device__ void cmap_schlieren(double t_, unsigned char* rgb) {
  const double t = fmax(0.0, fmin(1.0, t_));
  if (t < 0.7) {
    const double s = t / 0.7;
    rgb[0] = 0;
    rgb[1] = 0;
    rgb[2] = (unsigned char)(cmap_lerp(0.0f, 255.0f, (float)s) + 0.5);
  } else {
    const double s = (t - 0.7) / 0.3;
    const unsigned char v = (unsigned char)(cmap_lerp(0.0f, 255.0f, (float)s) + 0.5);
    rgb[0] = v;
    rgb[1] = v;
    rgb[2] = 255;
  }
}

__global__ void k_colour_pixels(int nx, int ny, const unsigned long long* __restrict__ pix,
                                const double* __restrict__ scalar, double fmin_, double span, int schlieren,
                                unsigned char* __restrict__ rgb) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (int64_t)nx * ny) return;
  const int i = (int)(p % nx), j = (int)(p / nx);
  unsigned char col[3] = {0, 0, 0};
  const unsigned long long key = pix[p];
  if (key != ULLONG_MAX) {
    const double w = scalar[(uint32_t)(key & 0xffffffffull)];
    double t = (w - fmin_) / span;
    if (schlieren) {
      t = sqrt(fmax(0.0, t));
      cmap_schlieren(t, col);
    } else {
      cmap_bwr(t, col);
    }
  }
  unsigned char* o = rgb + 3 * ((int64_t)(ny - 1 - j) * nx + i);
  o[0] = col[0];
  o[1] = col[1];
  o[2] = col[2];
}

}  // namespace o2f
