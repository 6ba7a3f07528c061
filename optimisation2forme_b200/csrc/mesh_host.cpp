// Host-side mesh build.  Integer topology must equal the reference's exactly,
// so the construction follows src/mesh.cpp:7-297 step for step:
//   * edges are keyed by (vmin, vmax) in an ordered map, so edge ids are the
//     lexicographic order of that key; the first cell that records an edge is
//     its left cell, the second its right cell (recordEdge, :288-297);
//   * the normal is made unit and flipped to point toward the left cell (:199-209);
//   * Cell::edgeIDs, Cell::neighbourIDs and Vertex::cellIDs are
//     std::unordered_set<std::size_t> in the reference, and their iteration
//     order fixes the floating-point summation order of every gather.  The
//     same containers are filled here with the same insertion sequence, which
//     yields the same iteration order with the same standard library;
//   * Vertex::cellIDsOrdered sorts (atan2, cell) pairs with std::sort (:231-248).
#include "mesh_host.hpp"

#include <algorithm>
#include <tuple>
#include <iterator>
#include <charconv>
#include <cstring>
#include <cmath>
#include <fstream>
#include <map>
#include <numeric>
#include <set>
#include <sstream>
#include <stdexcept>
#include <unordered_set>

namespace o2f {

namespace {

struct MeshError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline double clamp1(double v) { return (v < -1.0) ? -1.0 : (1.0 < v) ? 1.0 : v; }

// Volume and centre of cell c from its vertices (src/mesh.cpp:140-171).
void cell_geometry(HostMesh& m, int64_t c) {
  const int64_t o0 = m.cell_voff[c], nn = m.cell_voff[c + 1] - o0;
  const int64_t* n = &m.cell_verts[o0];
  const double x0 = m.vx[n[0]], y0 = m.vy[n[0]], x1 = m.vx[n[1]], y1 = m.vy[n[1]], x2 = m.vx[n[2]],
               y2 = m.vy[n[2]];
  if (nn == 3) {
    double ax = x1 - x0, ay = y1 - y0, bx = x2 - x0, by = y2 - y0;
    m.cvol[c] = std::abs(0.5 * (ax * by - bx * ay));
    m.ccx[c] = 1.0 / 3.0 * (x0 + x1 + x2);
    m.ccy[c] = 1.0 / 3.0 * (y0 + y1 + y2);
  } else {
    const double x3 = m.vx[n[3]], y3 = m.vy[n[3]];
    double ax = x1 - x0, ay = y1 - y0, bx = x2 - x0, by = y2 - y0;
    double cx = x1 - x2, cy = y1 - y2, ex = x3 - x2, ey = y3 - y2;
    m.cvol[c] = 0.5 * (std::abs(ax * by - bx * ay) + std::abs(cx * ey - ex * cy));
    m.ccx[c] = 0.25 * (x0 + x1 + x2 + x3);
    m.ccy[c] = 0.25 * (y0 + y1 + y2 + y3);
  }
}

// Length, unit normal toward the left cell and centre of edge e
// (src/mesh.cpp:196-222); needs the left cell's centre.
void edge_geometry(HostMesh& m, int64_t e) {
  const int64_t a = m.e_v0[e], b = m.e_v1[e], cl = m.e_cl[e];
  double tx = m.vx[a] - m.vx[b], ty = m.vy[a] - m.vy[b], tz = 0.0;
  double len = std::sqrt(tx * tx + ty * ty + tz * tz);
  double nx = ty / len, ny = -tx / len;
  double ex = 0.5 * (m.vx[a] + m.vx[b]), ey = 0.5 * (m.vy[a] + m.vy[b]);
  double dx = m.ccx[cl] - ex, dy = m.ccy[cl] - ey;
  if (dx * nx + dy * ny < 0) {
    nx = -nx;
    ny = -ny;
  }
  m.elen[e] = len;
  m.enx[e] = nx;
  m.eny[e] = ny;
  m.ecx[e] = ex;
  m.ecy[e] = ey;
}

// Vertex::cellIDsOrdered: the cells of every vertex sorted by the angle of
// their centre about the vertex (src/mesh.cpp:238-247).
// Vertices are independent: threads split them, with the same result.
void vertex_cell_order(HostMesh& m) {
  m.vert_cells_ord.assign(m.vert_cells.size(), 0);
#pragma omp parallel
  {
    std::vector<std::pair<double, int64_t>> tmp;
#pragma omp for schedule(static)
    for (int64_t v = 0; v < m.nv; ++v) {
      tmp.clear();
      for (int64_t k = m.vert_coff[v]; k < m.vert_coff[v + 1]; ++k) {
        const int64_t c = m.vert_cells[k];
        tmp.emplace_back(std::atan2(m.ccy[c] - m.vy[v], m.ccx[c] - m.vx[v]), c);
      }
      std::sort(tmp.begin(), tmp.end(), [](auto& a, auto& b) { return a.first < b.first; });
      int64_t o = m.vert_coff[v];
      for (auto& pr : tmp) m.vert_cells_ord[o++] = pr.second;
    }
  }
}

}  // namespace

std::map<std::pair<int64_t, int64_t>, uint8_t> boundary_segments(const o2f_mesh_desc& d, HostMesh& m) {
  // Boundary segments (src/mesh.cpp:76-109): the edge code is keyed by
  // (vmin, vmax); both vertices take the code; later segments win.
  std::map<std::pair<int64_t, int64_t>, uint8_t> bc;
  for (int64_t s = 0; s < d.n_segments; ++s) {
    int64_t a = d.segments[2 * s], b = d.segments[2 * s + 1];
    if (a < 0 || b < 0 || a >= m.nv || b >= m.nv) throw MeshError("boundary segment vertex out of range");
    uint8_t code = d.segment_bc[s];
    if (code != 'i' && code != 'o' && code != 'f' && code != 'w') throw MeshError("unknown boundary code");
    bc[{std::min(a, b), std::max(a, b)}] = code;
    m.vbc[a] = code;
    m.vbc[b] = code;
  }
  return bc;
}

void finish_geometry(HostMesh& m) {
  m.cvol.resize(m.nc);
  m.ccx.resize(m.nc);
  m.ccy.resize(m.nc);
  m.elen.resize(m.ne);
  m.enx.resize(m.ne);
  m.eny.resize(m.ne);
  m.ecx.resize(m.ne);
  m.ecy.resize(m.ne);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < m.nc; ++c) cell_geometry(m, c);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m.ne; ++e) edge_geometry(m, e);
  vertex_cell_order(m);
  compute_vertex_weights(m);
}

HostMesh build_mesh(const o2f_mesh_desc& d) {
  if (d.n_nodes <= 0 || d.n_cells <= 0 || !d.node_xy || !d.cell_offsets || !d.cell_nodes)
    throw std::invalid_argument("mesh description: empty or null arrays");
  if (d.n_segments > 0 && (!d.segments || !d.segment_bc))
    throw std::invalid_argument("mesh description: null boundary arrays");
  HostMesh m;
  m.nv = d.n_nodes;
  m.nc = d.n_cells;
  m.vx.resize(m.nv);
  m.vy.resize(m.nv);
  m.vbc.assign(m.nv, 0);
  for (int64_t i = 0; i < m.nv; ++i) {
    m.vx[i] = d.node_xy[2 * i];
    m.vy[i] = d.node_xy[2 * i + 1];
  }
  const std::map<std::pair<int64_t, int64_t>, uint8_t> bc = boundary_segments(d, m);
  // Cells (src/mesh.cpp:112-177).
  std::map<std::pair<int64_t, int64_t>, std::pair<int64_t, int64_t>> edge_map;
  std::vector<std::unordered_set<std::size_t>> vcells(m.nv);
  m.cell_voff.resize(m.nc + 1);
  m.cvol.resize(m.nc);
  m.ccx.resize(m.nc);
  m.ccy.resize(m.nc);
  m.cell_voff[0] = 0;
  auto record_edge = [&](int64_t va, int64_t vb, int64_t cell) {
    std::pair<int64_t, int64_t> k{std::min(va, vb), std::max(va, vb)};
    auto it = edge_map.find(k);
    if (it == edge_map.end()) {
      edge_map.emplace(k, std::pair<int64_t, int64_t>{cell, -1});
    } else {
      if (it->second.second != -1) throw MeshError("edge shared by more than two cells");
      it->second.second = cell;
    }
  };
  for (int64_t c = 0; c < m.nc; ++c) {
    int64_t o0 = d.cell_offsets[c], o1 = d.cell_offsets[c + 1];
    int64_t nn = o1 - o0;
    if (nn != 3 && nn != 4) throw MeshError("only triangles and quadrilaterals are supported");
    int64_t n[4];
    for (int64_t k = 0; k < nn; ++k) {
      n[k] = d.cell_nodes[o0 + k];
      if (n[k] < 0 || n[k] >= m.nv) throw MeshError("cell vertex out of range");
      m.cell_verts.push_back(n[k]);
    }
    m.cell_voff[c + 1] = (int64_t)m.cell_verts.size();
    cell_geometry(m, c);
    for (int64_t k = 0; k < nn; ++k) vcells[n[k]].insert((std::size_t)c);
    for (int64_t k = 0; k < nn; ++k) record_edge(n[k], n[(k + 1) % nn], c);
  }
  // Edges (src/mesh.cpp:182-229).
  m.ne = (int64_t)edge_map.size();
  m.e_v0.resize(m.ne);
  m.e_v1.resize(m.ne);
  m.e_cl.resize(m.ne);
  m.e_cr.resize(m.ne);
  m.ebc.assign(m.ne, 0);
  m.elen.resize(m.ne);
  m.enx.resize(m.ne);
  m.eny.resize(m.ne);
  m.ecx.resize(m.ne);
  m.ecy.resize(m.ne);
  std::vector<std::unordered_set<std::size_t>> cedges(m.nc), cnbrs(m.nc);
  int64_t e = 0;
  for (const auto& [key, cells] : edge_map) {
    const int64_t a = key.first, b = key.second, cl = cells.first, cr = cells.second;
    m.e_v0[e] = a;
    m.e_v1[e] = b;
    m.e_cl[e] = cl;
    m.e_cr[e] = cr;
    auto itbc = bc.find(key);
    if (itbc != bc.end()) m.ebc[e] = itbc->second;
    if (cr == -1 && m.ebc[e] == 0) throw MeshError("boundary edge without a boundary condition");
    if (cr != -1 && m.ebc[e] != 0) throw MeshError("interior edge carries a boundary condition");
    edge_geometry(m, e);
    cedges[cl].insert((std::size_t)e);
    if (cr != -1) {
      cedges[cr].insert((std::size_t)e);
      cnbrs[cl].insert((std::size_t)cr);
      cnbrs[cr].insert((std::size_t)cl);
    }
    ++e;
  }
  edge_map.clear();
  m.cell_eoff.assign(m.nc + 1, 0);
  m.cell_noff.assign(m.nc + 1, 0);
  for (int64_t c = 0; c < m.nc; ++c) {
    for (auto x : cedges[c]) m.cell_edges.push_back((int64_t)x);
    m.cell_eoff[c + 1] = (int64_t)m.cell_edges.size();
    for (auto x : cnbrs[c]) m.cell_nbrs.push_back((int64_t)x);
    m.cell_noff[c + 1] = (int64_t)m.cell_nbrs.size();
    std::unordered_set<std::size_t>().swap(cedges[c]);
    std::unordered_set<std::size_t>().swap(cnbrs[c]);
  }
  // Vertex cell lists and the atan2 order (src/mesh.cpp:231-248).
  m.vert_coff.assign(m.nv + 1, 0);
  for (int64_t v = 0; v < m.nv; ++v) {
    for (auto c : vcells[v]) m.vert_cells.push_back((int64_t)c);
    m.vert_coff[v + 1] = (int64_t)m.vert_cells.size();
    m.max_valence = std::max<int64_t>(m.max_valence, (int64_t)vcells[v].size());
    std::unordered_set<std::size_t>().swap(vcells[v]);
  }
  vertex_cell_order(m);
  for (int64_t c = 0; c < m.nc; ++c) {
    int64_t n = m.cell_eoff[c + 1] - m.cell_eoff[c];
    if (n != m.cell_voff[c + 1] - m.cell_voff[c]) throw MeshError("cell with a repeated vertex");
  }
  compute_vertex_weights(m);
  return m;
}

namespace {

// Twice the signed area of cell c (shoelace over its vertices in file order).
double signed_area2(const HostMesh& m, int64_t c) {
  const int64_t o0 = m.cell_voff[c], nn = m.cell_voff[c + 1] - o0;
  double a = 0.0;
  for (int64_t k = 0; k < nn; ++k) {
    const int64_t i = m.cell_verts[o0 + k], j = m.cell_verts[o0 + (k + 1) % nn];
    a += m.vx[i] * m.vy[j] - m.vx[j] * m.vy[i];
  }
  return a;
}

}  // namespace

void set_coordinates(HostMesh& m, const double* xy) {
  if (!xy) throw std::invalid_argument("null coordinates");
  for (int64_t i = 0; i < 2 * m.nv; ++i)
    if (!std::isfinite(xy[i])) throw std::invalid_argument("non-finite vertex coordinate");
  std::vector<double> ox = m.vx, oy = m.vy;
  std::vector<int8_t> side(m.nc);
  for (int64_t c = 0; c < m.nc; ++c) side[c] = signed_area2(m, c) > 0.0 ? 1 : -1;
  for (int64_t v = 0; v < m.nv; ++v) {
    m.vx[v] = xy[2 * v];
    m.vy[v] = xy[2 * v + 1];
  }
  for (int64_t c = 0; c < m.nc; ++c) {
    const double a = signed_area2(m, c);
    if (a == 0.0 || (a > 0.0 ? 1 : -1) != side[c]) {
      m.vx.swap(ox);
      m.vy.swap(oy);
      throw MeshError("the new coordinates fold or collapse cell " + std::to_string(c));
    }
  }
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < m.nc; ++c) cell_geometry(m, c);
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < m.ne; ++e) edge_geometry(m, e);
  vertex_cell_order(m);
  compute_vertex_weights(m);
}

void compute_vertex_weights(HostMesh& m) {
  m.vert_wcells.assign(m.vert_cells.size(), 0);
  m.vert_w.assign(m.vert_cells.size(), 0.0);
  // vertices are independent: threads split them, with the same result
#pragma omp parallel
  {
  std::vector<double> w, d, ux, uy;
#pragma omp for schedule(static)
  for (int64_t v = 0; v < m.nv; ++v) {
    const int64_t o = m.vert_coff[v], n = m.vert_coff[v + 1] - o;
    const double px = m.vx[v], py = m.vy[v];
    if (n == 3) {
      // Barycentric weights of the vertex in the triangle of the three cell
      // centres, in Vertex::cellIDs order (src/advection.cpp:29-50).
      const int64_t i0 = m.vert_cells[o], i1 = m.vert_cells[o + 1], i2 = m.vert_cells[o + 2];
      const double c0x = m.ccx[i0], c0y = m.ccy[i0], c1x = m.ccx[i1], c1y = m.ccy[i1], c2x = m.ccx[i2],
                   c2y = m.ccy[i2];
      double w0_num = (c1x - px) * (c2y - py) - (c2x - px) * (c1y - py);
      double w0_den = (c1x - c0x) * (c2y - c0y) - (c2x - c0x) * (c1y - c0y);
      double w0 = (w0_num / w0_den);
      double w1_num = (c2x - px) * (c0y - py) - (c0x - px) * (c2y - py);
      double w1_den = (c1x - c0x) * (c2y - c0y) - (c2x - c0x) * (c1y - c0y);
      double w1 = (w1_num / w1_den);
      double w2 = 1 - w0 - w1;
      m.vert_wcells[o] = i0;
      m.vert_wcells[o + 1] = i1;
      m.vert_wcells[o + 2] = i2;
      m.vert_w[o] = w0;
      m.vert_w[o + 1] = w1;
      m.vert_w[o + 2] = w2;
    } else if (n == 2) {
      // 0.5*(a+b) == 0.5*a + 0.5*b exactly (halving is exact).
      m.vert_wcells[o] = m.vert_cells[o];
      m.vert_wcells[o + 1] = m.vert_cells[o + 1];
      m.vert_w[o] = 0.5;
      m.vert_w[o + 1] = 0.5;
    } else if (n == 1) {
      m.vert_wcells[o] = m.vert_cells[o];
      m.vert_w[o] = 1.0;
    } else if (n >= 4) {
      const int64_t* ord = &m.vert_cells_ord[o];
      w.assign(n, 0.0);
      d.assign(n, 0.0);
      ux.assign(n, 0.0);
      uy.assign(n, 0.0);
      for (int64_t k = 0; k < n; ++k) {
        double dx = m.ccx[ord[k]] - px, dy = m.ccy[ord[k]] - py;
        d[k] = std::hypot(dx, dy);
        ux[k] = dx / d[k];
        uy[k] = dy / d[k];
      }
      const bool boundary_fan = (n > 4) && m.vbc[v] != 0;
      if (!boundary_fan) {
        // Mean-value weights (src/advection.cpp:75-99); for n == 4 this is the
        // reference formula term for term.
        for (int64_t k = 0; k < n; ++k) {
          int64_t km1 = (k + n - 1) % n, kp1 = (k + 1) % n;
          double cos_prev = clamp1(ux[km1] * ux[k] + uy[km1] * uy[k]);
          double cos_next = clamp1(ux[k] * ux[kp1] + uy[k] * uy[kp1]);
          double theta_prev = std::acos(cos_prev);
          double theta_next = std::acos(cos_next);
          w[k] = (std::tan(0.5 * theta_prev) + std::tan(0.5 * theta_next)) / d[k];
        }
      } else {
        // Open fan at a boundary vertex with >= 5 cells: inverse distance.
        for (int64_t k = 0; k < n; ++k) w[k] = 1.0 / d[k];
      }
      double wsum = 0.0;
      for (int64_t k = 0; k < n; ++k) wsum += w[k];
      for (int64_t k = 0; k < n; ++k) {
        m.vert_wcells[o + k] = ord[k];
        m.vert_w[o + k] = w[k] / wsum;
      }
    }
  }
  }  // omp parallel
}

Stencil jacobian_stencil(const HostMesh& m, const std::vector<int64_t>& perm, const std::vector<int64_t>& cinv) {
  const int64_t nc = m.nc;
  // ring(c): cells sharing a vertex with c, ascending (new numbering)
  std::vector<int64_t> roff(nc + 1, 0);
  std::vector<std::vector<int32_t>> ring(nc);
#pragma omp parallel
  {
    std::vector<int32_t> tmp;
#pragma omp for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t co = perm[c];
      tmp.clear();
      for (int64_t k = m.cell_voff[co]; k < m.cell_voff[co + 1]; ++k) {
        const int64_t v = m.cell_verts[k];
        for (int64_t q = m.vert_coff[v]; q < m.vert_coff[v + 1]; ++q) tmp.push_back((int32_t)cinv[m.vert_cells[q]]);
      }
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      ring[c] = tmp;
    }
  }
  // S(c) = ring(ring(c))
  Stencil st;
  std::vector<std::vector<int32_t>> sten(nc);
#pragma omp parallel
  {
    std::vector<int32_t> tmp;
#pragma omp for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
      tmp.clear();
      for (int32_t a : ring[c]) tmp.insert(tmp.end(), ring[a].begin(), ring[a].end());
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      sten[c] = tmp;
    }
  }
  std::vector<std::vector<int32_t>>().swap(ring);
  st.off.assign(nc + 1, 0);
  for (int64_t c = 0; c < nc; ++c) st.off[c + 1] = st.off[c] + (int64_t)sten[c].size();
  st.idx.resize(st.off[nc]);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < nc; ++c) std::copy(sten[c].begin(), sten[c].end(), st.idx.begin() + st.off[c]);
  std::vector<std::vector<int32_t>>().swap(sten);
  // greedy colouring in new order: the colours of every cell sharing some
  // S(i) with j are taken
  st.color.assign(nc, -1);
  std::vector<int64_t> mark;
  for (int64_t j = 0; j < nc; ++j) {
    for (int64_t a = st.off[j]; a < st.off[j + 1]; ++a) {
      const int32_t i = st.idx[a];
      for (int64_t b = st.off[i]; b < st.off[i + 1]; ++b) {
        const int32_t col = st.color[st.idx[b]];
        if (col >= 0) mark[col] = j;
      }
    }
    int32_t col = 0;
    while (col < st.ncolor && mark[col] == j) ++col;
    if (col == st.ncolor) {
      ++st.ncolor;
      mark.push_back(-1);
    }
    st.color[j] = col;
  }
  return st;
}

double min_cell_h(const HostMesh& m) {
  double min_h = INFINITY;
  for (int64_t c = 0; c < m.nc; ++c) {
    double perimeter = 0.0;
    for (int64_t k = m.cell_eoff[c]; k < m.cell_eoff[c + 1]; ++k) perimeter += m.elen[m.cell_edges[k]];
    double h = 2.0 * m.cvol[c] / perimeter;
    min_h = std::min(min_h, h);
  }
  return min_h;
}

namespace {

// Hilbert index of (x, y) on a 2^order grid (classic rotate-and-flip walk).
uint64_t hilbert_d(uint32_t x, uint32_t y, int order) {
  uint64_t d = 0;
  for (uint64_t s = uint64_t(1) << (order - 1); s > 0; s >>= 1) {
    uint32_t rx = (x & s) ? 1u : 0u;
    uint32_t ry = (y & s) ? 1u : 0u;
    d += s * s * ((3u * rx) ^ ry);
    if (ry == 0) {
      if (rx == 1) {
        x = (uint32_t)(s - 1) - (x & (uint32_t)(s - 1)) + (x & ~(uint32_t)(s - 1));
        y = (uint32_t)(s - 1) - (y & (uint32_t)(s - 1)) + (y & ~(uint32_t)(s - 1));
        x &= (uint32_t)((uint64_t(1) << order) - 1);
        y &= (uint32_t)((uint64_t(1) << order) - 1);
      }
      std::swap(x, y);
    }
  }
  return d;
}

}  // namespace

std::vector<int64_t> hilbert_order(const std::vector<double>& x, const std::vector<double>& y) {
  const size_t n = x.size();
  std::vector<int64_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  if (n == 0) return perm;
  double x0 = *std::min_element(x.begin(), x.end()), x1 = *std::max_element(x.begin(), x.end());
  double y0 = *std::min_element(y.begin(), y.end()), y1 = *std::max_element(y.begin(), y.end());
  double span = std::max(x1 - x0, y1 - y0);
  if (!(span > 0)) return perm;
  const int order = 31;
  const double scale = (double)((uint64_t(1) << order) - 1) / span;
  std::vector<uint64_t> key(n);
  for (size_t i = 0; i < n; ++i) {
    uint32_t ix = (uint32_t)std::llround((x[i] - x0) * scale);
    uint32_t iy = (uint32_t)std::llround((y[i] - y0) * scale);
    key[i] = hilbert_d(ix, iy, order);
  }
  std::stable_sort(perm.begin(), perm.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
  return perm;
}

int64_t export_mesh_array(const HostMesh& m, const std::string& w, void* out) {
  auto put_i = [&](const std::vector<int64_t>& v) {
    if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(int64_t));
    return (int64_t)v.size();
  };
  auto put_d = [&](const std::vector<double>& v) {
    if (out && !v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(double));
    return (int64_t)v.size();
  };
  auto inter_i = [&](const std::vector<int64_t>& a, const std::vector<int64_t>& b) {
    std::vector<int64_t> r(2 * a.size());
    for (size_t i = 0; i < a.size(); ++i) {
      r[2 * i] = a[i];
      r[2 * i + 1] = b[i];
    }
    return put_i(r);
  };
  auto inter_d = [&](const std::vector<double>& a, const std::vector<double>& b) {
    std::vector<double> r(2 * a.size());
    for (size_t i = 0; i < a.size(); ++i) {
      r[2 * i] = a[i];
      r[2 * i + 1] = b[i];
    }
    return put_d(r);
  };
  auto bytes_i = [&](const std::vector<uint8_t>& a) { return put_i(std::vector<int64_t>(a.begin(), a.end())); };
  if (w == "edge_v") return inter_i(m.e_v0, m.e_v1);
  if (w == "edge_c") return inter_i(m.e_cl, m.e_cr);
  if (w == "edge_bc") return bytes_i(m.ebc);
  if (w == "vert_bc") return bytes_i(m.vbc);
  if (w == "cell_edges_off") return put_i(m.cell_eoff);
  if (w == "cell_edges") return put_i(m.cell_edges);
  if (w == "vert_cells_off") return put_i(m.vert_coff);
  if (w == "vert_cells") return put_i(m.vert_cells);
  if (w == "vert_cells_ord") return put_i(m.vert_cells_ord);
  if (w == "vert_wcells") return put_i(m.vert_wcells);
  if (w == "cell_verts_off") return put_i(m.cell_voff);
  if (w == "cell_verts") return put_i(m.cell_verts);
  if (w == "cell_nbrs_off") return put_i(m.cell_noff);
  if (w == "cell_nbrs") return put_i(m.cell_nbrs);
  if (w == "vert_xy") return inter_d(m.vx, m.vy);
  if (w == "edge_len") return put_d(m.elen);
  if (w == "edge_n") return inter_d(m.enx, m.eny);
  if (w == "edge_ctr") return inter_d(m.ecx, m.ecy);
  if (w == "cell_vol") return put_d(m.cvol);
  if (w == "cell_ctr") return inter_d(m.ccx, m.ccy);
  if (w == "vert_w") return put_d(m.vert_w);
  if (w == "min_h") return put_d(std::vector<double>{min_cell_h(m)});
  throw std::invalid_argument("unknown mesh array '" + w + "'");
}

o2f_mesh_desc MshData::desc() const {
  o2f_mesh_desc d{};
  d.n_nodes = (int64_t)xy.size() / 2;
  d.node_xy = xy.data();
  d.n_segments = (int64_t)seg_bc.size();
  d.segments = seg.data();
  d.segment_bc = seg_bc.data();
  d.n_cells = (int64_t)coff.size() - 1;
  d.cell_offsets = coff.data();
  d.cell_nodes = cnodes.data();
  return d;
}

namespace {

// One msh file's content as read, before the element walk.
struct MshElem {
  int type, phys, entity;
  int64_t n[4];
};
struct MshRaw {
  std::vector<std::tuple<int64_t, double, double>> nodes;  // (tag, x, y), file order
  std::map<std::pair<int, int>, std::string> names;
  std::vector<MshElem> elems;
  bool have_format = false;
};

int msh_nodes_of(int type) { return type == 1 ? 2 : type == 2 ? 3 : type == 3 ? 4 : type == 15 ? 1 : -1; }

void msh_names(std::istream& in, MshRaw& raw) {
  int n = 0;
  in >> n;
  for (int i = 0; i < n; ++i) {
    int dim, tag;
    std::string name;
    in >> dim >> tag;
    std::getline(in, name);
    auto a = name.find('"'), b = name.rfind('"');
    if (a != std::string::npos && b > a) name = name.substr(a + 1, b - a - 1);
    raw.names[{dim, tag}] = name;
  }
}

// The stream reader: any layout istream accepts.
MshRaw parse_msh2_stream(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw std::ios_base::failure("cannot open " + path);
  MshRaw raw;
  std::string line;
  while (std::getline(in, line)) {
    if (line.rfind("$MeshFormat", 0) == 0) {
      double ver;
      int ft, ds;
      in >> ver >> ft >> ds;
      if (ver < 2.0 || ver >= 3.0 || ft != 0) throw std::ios_base::failure("only ASCII MSH 2.x is supported");
      raw.have_format = true;
    } else if (line.rfind("$PhysicalNames", 0) == 0) {
      msh_names(in, raw);
    } else if (line.rfind("$Nodes", 0) == 0) {
      int64_t n = 0;
      in >> n;
      for (int64_t i = 0; i < n; ++i) {
        int64_t tag;
        double x, y, z;
        in >> tag >> x >> y >> z;
        raw.nodes.emplace_back(tag, x, y);
      }
    } else if (line.rfind("$Elements", 0) == 0) {
      int64_t n = 0;
      in >> n;
      raw.elems.reserve(n);
      for (int64_t i = 0; i < n; ++i) {
        int64_t id;
        int type, ntags;
        in >> id >> type >> ntags;
        MshElem e{type, 0, 0, {0, 0, 0, 0}};
        for (int k = 0; k < ntags; ++k) {
          int t;
          in >> t;
          if (k == 0) e.phys = t;
          if (k == 1) e.entity = t;
        }
        const int nn = msh_nodes_of(type);
        if (nn < 0) throw std::ios_base::failure("unsupported element type " + std::to_string(type));
        for (int k = 0; k < nn; ++k) in >> e.n[k];
        raw.elems.push_back(e);
      }
    }
    if (!in && !in.eof()) throw std::ios_base::failure("parse error in " + path);
  }
  return raw;
}

// Field scanner for the parallel reader: numbers separated by spaces, tabs
// or a carriage return; std::from_chars rounds decimal input exactly as the
// stream does (correct rounding).
struct Scan {
  const char* p;
  const char* e;
  void skip() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  }
  template <typename X>
  bool num(X& v) {
    skip();
    if (p < e && *p == '+') ++p;
    const auto r = std::from_chars(p, e, v);
    if (r.ec != std::errc() || r.ptr == p) return false;
    p = r.ptr;
    return true;
  }
  bool at_end() {
    skip();
    return p == e;
  }
};

// Line starts of [b, e): every line ends with '\n'.
bool split_lines(const char* b, const char* e, int64_t n, std::vector<const char*>& starts) {
  if (n < 0) return false;
  starts.clear();
  starts.reserve(n + 1);
  const char* p = b;
  for (int64_t i = 0; i < n; ++i) {
    if (p >= e) return false;
    starts.push_back(p);
    const char* q = static_cast<const char*>(std::memchr(p, '\n', e - p));
    if (!q) return false;
    p = q + 1;
  }
  starts.push_back(p);
  return true;
}

// The whole file in memory, node and element lines parsed by all threads.
// Returns false for anything outside the plain layout (one section of each
// kind, one entry per line), which the stream reader then handles.
bool parse_msh2_parallel(const std::string& path, MshRaw& raw) {
  std::ifstream in(path, std::ios::binary | std::ios::ate);
  if (!in) return false;
  std::string buf((size_t)in.tellg(), '\0');
  in.seekg(0);
  if (!in.read(&buf[0], (std::streamsize)buf.size())) return false;
  auto section = [&](const char* tag) -> int64_t {  // position after the header line, -1 if absent or repeated
    const std::string key = std::string("\n") + tag;
    size_t pos = buf.rfind(tag, 0) == 0 ? 0 : buf.find(key);
    if (pos == std::string::npos) return -1;
    if (pos != 0) ++pos;
    if (buf.find(key, pos + 1) != std::string::npos) return -2;
    const size_t nl = buf.find('\n', pos);
    return nl == std::string::npos ? -1 : (int64_t)nl + 1;
  };
  const int64_t fmt = section("$MeshFormat"), nam = section("$PhysicalNames"), nod = section("$Nodes"),
                ele = section("$Elements");
  if (fmt < 0 || nod < 0 || ele < 0 || nam == -2) return false;
  {
    std::istringstream f(buf.substr(fmt, 64));
    double ver;
    int ft, ds;
    if (!(f >> ver >> ft >> ds) || ver < 2.0 || ver >= 3.0 || ft != 0) return false;
    raw.have_format = true;
  }
  if (nam >= 0) {
    std::istringstream f(buf.substr(nam, buf.find("$EndPhysicalNames", nam) - nam));
    msh_names(f, raw);
    if (!f && !f.eof()) return false;
  }
  const char* base = buf.data();
  const char* end = base + buf.size();
  std::vector<const char*> starts;
  // $Nodes
  {
    Scan h{base + nod, end};
    int64_t n = 0;
    if (!h.num(n)) return false;
    const char* first = static_cast<const char*>(std::memchr(h.p, '\n', end - h.p));
    if (!first || !split_lines(first + 1, end, n, starts)) return false;
    raw.nodes.resize(n);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < n; ++i) {
      Scan sc{starts[i], starts[i + 1] - 1};
      int64_t tag;
      double x, y, z;
      if (!sc.num(tag) || !sc.num(x) || !sc.num(y) || !sc.num(z) || !sc.at_end()) bad = 1;
      else raw.nodes[i] = {tag, x, y};
    }
    if (bad) return false;
  }
  // $Elements
  {
    Scan h{base + ele, end};
    int64_t n = 0;
    if (!h.num(n)) return false;
    const char* first = static_cast<const char*>(std::memchr(h.p, '\n', end - h.p));
    if (!first || !split_lines(first + 1, end, n, starts)) return false;
    raw.elems.resize(n);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t i = 0; i < n; ++i) {
      Scan sc{starts[i], starts[i + 1] - 1};
      int64_t id;
      int type, ntags;
      MshElem el{0, 0, 0, {0, 0, 0, 0}};
      bool ok = sc.num(id) && sc.num(type) && sc.num(ntags) && ntags >= 0;
      for (int k = 0; ok && k < ntags; ++k) {
        int t;
        ok = sc.num(t);
        if (k == 0) el.phys = t;
        if (k == 1) el.entity = t;
      }
      const int nn = msh_nodes_of(type);
      ok = ok && nn > 0;
      for (int k = 0; ok && k < nn; ++k) ok = sc.num(el.n[k]);
      el.type = type;
      if (!ok || !sc.at_end()) bad = 1;
      else raw.elems[i] = el;
    }
    if (bad) return false;
  }
  return true;
}

// Gmsh exposes, for an MSH 2.2 file: nodes in tag order (a repeated tag
// keeps its last line), physical groups in (dim, tag) order, their
// elementary entities in ascending order, and per entity the element types
// in ascending order with the elements of a type in file order.  Mesh::Mesh
// walks exactly that (src/mesh.cpp:20-179): lines of groups named
// Inlet/Outlet/FreeStream/Wall/Airfoil give boundary codes, triangles and
// quads give cells.
MshData assemble_msh(const std::string& path, MshRaw& raw) {
  if (!raw.have_format) throw std::ios_base::failure("missing $MeshFormat in " + path);
  MshData out;
  auto& nodes = raw.nodes;
  std::stable_sort(nodes.begin(), nodes.end(),
                   [](const auto& a, const auto& b) { return std::get<0>(a) < std::get<0>(b); });
  std::vector<int64_t> tags;
  tags.reserve(nodes.size());
  for (size_t i = 0; i < nodes.size(); ++i) {
    if (i + 1 < nodes.size() && std::get<0>(nodes[i + 1]) == std::get<0>(nodes[i])) continue;  // last one wins
    tags.push_back(std::get<0>(nodes[i]));
    out.xy.push_back(std::get<1>(nodes[i]));
    out.xy.push_back(std::get<2>(nodes[i]));
  }
  // tag -> vertex: a table when the tags are about dense (Gmsh numbers them
  // 1..N), else a binary search
  std::vector<int64_t> lut;
  if (!tags.empty() && tags.front() >= 0 && tags.back() <= 4 * (int64_t)tags.size() + 16) {
    lut.assign(tags.back() + 1, -1);
    for (size_t i = 0; i < tags.size(); ++i) lut[tags[i]] = (int64_t)i;
  }
  auto vid = [&](int64_t tag) {
    if (!lut.empty()) {
      if (tag >= 0 && tag < (int64_t)lut.size() && lut[tag] >= 0) return lut[tag];
      throw std::ios_base::failure("element references unknown node " + std::to_string(tag));
    }
    auto it = std::lower_bound(tags.begin(), tags.end(), tag);
    if (it == tags.end() || *it != tag)
      throw std::ios_base::failure("element references unknown node " + std::to_string(tag));
    return (int64_t)(it - tags.begin());
  };
  const auto& elems = raw.elems;
  auto dim_of = [](int type) { return type == 15 ? 0 : type == 1 ? 1 : 2; };
  std::set<std::pair<int, int>> groups;
  for (const auto& e : elems)
    if (e.phys != 0) groups.insert({dim_of(e.type), e.phys});
  out.coff.push_back(0);
  for (const auto& [dim, tag] : groups) {
    std::string name;
    auto itn = raw.names.find({dim, tag});
    if (itn != raw.names.end()) name = itn->second;
    uint8_t code = name == "Inlet" ? 'i'
                 : name == "Outlet" ? 'o'
                 : name == "FreeStream" ? 'f'
                 : (name == "Wall" || name == "Airfoil") ? 'w'
                 : 0;
    std::set<int> ents;
    for (const auto& e : elems)
      if (dim_of(e.type) == dim && e.phys == tag) ents.insert(e.entity);
    for (int ent : ents) {
      for (int type : {1, 2, 3}) {
        for (const auto& e : elems) {
          if (e.type != type || e.entity != ent || dim_of(e.type) != dim) continue;
          if (type == 1) {
            if (code != 0) {
              out.seg.push_back(vid(e.n[0]));
              out.seg.push_back(vid(e.n[1]));
              out.seg_bc.push_back(code);
            }
          } else {
            int nn = type == 2 ? 3 : 4;
            for (int k = 0; k < nn; ++k) out.cnodes.push_back(vid(e.n[k]));
            out.coff.push_back((int64_t)out.cnodes.size());
          }
        }
      }
    }
  }
  return out;
}

}  // namespace

MshData read_msh2(const std::string& path) {
  constexpr std::streamoff kParallelFrom = 1 << 20;  // bytes; smaller files take the stream reader
  MshRaw raw;
  {
    std::ifstream probe(path, std::ios::binary | std::ios::ate);
    if (!probe) throw std::ios_base::failure("cannot open " + path);
    if (probe.tellg() >= kParallelFrom && parse_msh2_parallel(path, raw)) return assemble_msh(path, raw);
  }
  raw = parse_msh2_stream(path);
  return assemble_msh(path, raw);
}

}  // namespace o2f
