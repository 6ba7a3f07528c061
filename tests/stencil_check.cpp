// CPU check of o2f::jacobian_stencil (optimisation2forme_b200/csrc/mesh_host.cpp),
// the host part of the consistent adjoint: on triangulated and quad grids,
// numbered directly and by a random permutation,
//   * S(i) is exactly the cells within two vertex rings of i (brute force);
//   * the relation is symmetric;
//   * no S(i) holds two cells of one colour.
// Exits 1 on the first violation.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <random>
#include <set>
#include <vector>

#include "mesh_host.hpp"

namespace {

int check(bool triangles, int nx, int ny, unsigned seed) {
  // (nx+1) x (ny+1) nodes; boundary segments around the rectangle
  std::vector<double> xy;
  for (int j = 0; j <= ny; ++j)
    for (int i = 0; i <= nx; ++i) {
      xy.push_back(i + 0.1 * ((i * 7 + j * 3) % 5));
      xy.push_back(j + 0.1 * ((i * 5 + j * 11) % 7));
    }
  auto id = [&](int i, int j) { return (int64_t)j * (nx + 1) + i; };
  std::vector<int64_t> off{0}, nodes, seg;
  std::vector<uint8_t> bc;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const int64_t a = id(i, j), b = id(i + 1, j), c = id(i + 1, j + 1), d = id(i, j + 1);
      if (triangles) {
        nodes.insert(nodes.end(), {a, b, c});
        off.push_back((int64_t)nodes.size());
        nodes.insert(nodes.end(), {a, c, d});
      } else {
        nodes.insert(nodes.end(), {a, b, c, d});
      }
      off.push_back((int64_t)nodes.size());
    }
  for (int i = 0; i < nx; ++i) {
    seg.insert(seg.end(), {id(i, 0), id(i + 1, 0), id(i, ny), id(i + 1, ny)});
    bc.insert(bc.end(), {'f', 'f'});
  }
  for (int j = 0; j < ny; ++j) {
    seg.insert(seg.end(), {id(0, j), id(0, j + 1), id(nx, j), id(nx, j + 1)});
    bc.insert(bc.end(), {'w', 'f'});
  }
  o2f_mesh_desc d{};
  d.n_nodes = (int64_t)xy.size() / 2;
  d.node_xy = xy.data();
  d.n_segments = (int64_t)bc.size();
  d.segments = seg.data();
  d.segment_bc = bc.data();
  d.n_cells = (int64_t)off.size() - 1;
  d.cell_offsets = off.data();
  d.cell_nodes = nodes.data();
  const o2f::HostMesh m = o2f::build_mesh(d);
  const int64_t nc = m.nc;
  std::vector<int64_t> perm(nc), cinv(nc);
  std::iota(perm.begin(), perm.end(), 0);
  if (seed) std::shuffle(perm.begin(), perm.end(), std::mt19937(seed));
  for (int64_t c = 0; c < nc; ++c) cinv[perm[c]] = c;
  const o2f::Stencil st = o2f::jacobian_stencil(m, perm, cinv);
  // brute force in the original numbering
  std::vector<std::set<int64_t>> ring(nc);
  for (int64_t c = 0; c < nc; ++c)
    for (int64_t k = m.cell_voff[c]; k < m.cell_voff[c + 1]; ++k) {
      const int64_t v = m.cell_verts[k];
      for (int64_t q = m.vert_coff[v]; q < m.vert_coff[v + 1]; ++q) ring[c].insert(m.vert_cells[q]);
    }
  int64_t max_s = 0;
  for (int64_t c = 0; c < nc; ++c) {
    std::set<int64_t> want;
    for (int64_t a : ring[perm[c]])
      for (int64_t b : ring[a]) want.insert(cinv[b]);
    std::vector<int64_t> got(st.idx.begin() + st.off[c], st.idx.begin() + st.off[c + 1]);
    if (!std::is_sorted(got.begin(), got.end()) || std::set<int64_t>(got.begin(), got.end()) != want ||
        got.size() != want.size()) {
      std::printf("stencil of cell %lld differs from the two-ring\n", (long long)c);
      return 1;
    }
    max_s = std::max<int64_t>(max_s, (int64_t)got.size());
    std::set<int32_t> cols;
    for (int64_t j : got) {
      if (!std::binary_search(st.idx.begin() + st.off[j], st.idx.begin() + st.off[j + 1], (int32_t)c)) {
        std::printf("stencil not symmetric at (%lld, %lld)\n", (long long)c, (long long)j);
        return 1;
      }
      if (!cols.insert(st.color[j]).second) {
        std::printf("two cells of colour %d in the stencil of cell %lld\n", st.color[j], (long long)c);
        return 1;
      }
    }
  }
  std::printf("%s %dx%d perm %u: %lld cells, max stencil %lld, %d colours\n", triangles ? "triangles" : "quads", nx,
              ny, seed, (long long)nc, (long long)max_s, st.ncolor);
  return 0;
}

}  // namespace

int main() {
  int bad = 0;
  bad |= check(true, 14, 9, 0);
  bad |= check(true, 14, 9, 5);
  bad |= check(false, 11, 12, 0);
  bad |= check(false, 11, 12, 9);
  std::printf("stencil_check: %s\n", bad ? "FAILED" : "ok");
  return bad;
}
