// Host-side mesh build: topology and geometry in the reference's order, the
// cell->vertex interpolation weights, and the Hilbert renumbering used on the
// device.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "o2f.h"

namespace o2f {

// Topology and geometry in reference order (src/mesh.cpp:7-283).
struct HostMesh {
  int64_t nv = 0, nc = 0, ne = 0;
  // vertices
  std::vector<double> vx, vy;
  std::vector<uint8_t> vbc;
  std::vector<int64_t> vert_coff, vert_cells;  // Vertex::cellIDs iteration order
  std::vector<int64_t> vert_cells_ord;         // Vertex::cellIDsOrdered (atan2 sort)
  // interpolation weights, aligned with vert_wcells (same offsets as vert_coff)
  std::vector<int64_t> vert_wcells;
  std::vector<double> vert_w;
  // cells
  std::vector<int64_t> cell_voff, cell_verts;  // Cell::verticeIDs
  std::vector<double> cvol, ccx, ccy;
  std::vector<int64_t> cell_eoff, cell_edges;  // Cell::edgeIDs iteration order
  std::vector<int64_t> cell_noff, cell_nbrs;   // Cell::neighbourIDs iteration order
  // edges, (vmin,vmax) lexicographic order
  std::vector<int64_t> e_v0, e_v1, e_cl, e_cr;  // e_cr = -1 on boundary edges
  std::vector<uint8_t> ebc;
  std::vector<double> elen, enx, eny, ecx, ecy;
  int64_t max_valence = 0;
};

HostMesh build_mesh(const o2f_mesh_desc& desc);

// The same mesh with the integer topology built on the GPU (topo_gpu.cu):
// the edge order of the reference's std::map by a stable radix sort of the
// (vmin, vmax) keys, and the iteration orders of its std::unordered_set
// members by emulation (uset_order.h); geometry and weights on the host as
// in build_mesh.  Equal to build_mesh's result array for array.
HostMesh build_mesh_gpu(const o2f_mesh_desc& desc, void* stream);

// Pieces shared by the two builds.  boundary_segments validates the
// segments, sets the vertex codes and returns the edge codes by (vmin, vmax)
// (later segments win); finish_geometry fills every geometric array of a
// mesh whose topology and coordinates are set.
std::map<std::pair<int64_t, int64_t>, uint8_t> boundary_segments(const o2f_mesh_desc& d, HostMesh& m);
void finish_geometry(HostMesh& m);

// New vertex coordinates (xy[2*v], xy[2*v+1] in file order) for a built mesh
// of the same topology: every geometric quantity (cell volumes and centres,
// edge lengths, normals and centres, the atan2 cell order of the vertices,
// interpolation weights) is recomputed with the arithmetic of build_mesh, so
// the result equals build_mesh of a description with these coordinates.
// Throws std::invalid_argument for non-finite coordinates and a
// std::runtime_error, leaving the mesh unchanged, when a cell would collapse
// or change orientation.
void set_coordinates(HostMesh& m, const double* xy);
// Reads an ASCII MSH 2.2 file the way the reference's Gmsh import sees it and
// returns the equivalent description (the vectors own the storage).
struct MshData {
  std::vector<double> xy;
  std::vector<int64_t> seg;
  std::vector<uint8_t> seg_bc;
  std::vector<int64_t> coff, cnodes;
  o2f_mesh_desc desc() const;
};
MshData read_msh2(const std::string& path);

// Weights of the cell->vertex interpolation (src/advection.cpp:26-131):
// valence 1 copy, 2 average, 3 barycentric from the cell centres, 4
// mean-value weights over the atan2-ordered cells.  Valence >= 5 (left
// untouched by the reference) uses the same mean-value formula generalised to
// n cells at interior vertices and inverse-distance weights at boundary
// vertices.  Fills vert_wcells / vert_w.  `only` limits the recomputation to
// the listed vertices (empty: all).
void compute_vertex_weights(HostMesh& m);

// 2V / perimeter per cell with the perimeter summed in Cell::edgeIDs order
// (src/simulation.cpp:98-104); returns the minimum.
double min_cell_h(const HostMesh& m);

// Copies one named array (reference order) into out (if non-null); returns
// its length.  Throws std::invalid_argument for an unknown name.
int64_t export_mesh_array(const HostMesh& m, const std::string& which, void* out);

// Stencil of the full residual Jacobian: for every cell c (numbered by
// cinv: new = cinv[old], perm the inverse), the cells within two vertex
// rings, S(c), as an ascending CSR in the new numbering (the relation is
// symmetric); and a greedy colouring of the cells in new order such that no
// S(i) holds two cells of one colour.
struct Stencil {
  std::vector<int64_t> off;
  std::vector<int32_t> idx;
  std::vector<int32_t> color;
  int32_t ncolor = 0;
};
Stencil jacobian_stencil(const HostMesh& m, const std::vector<int64_t>& perm, const std::vector<int64_t>& cinv);

// Hilbert-curve order of points (x, y): returns perm with perm[new] = old.
std::vector<int64_t> hilbert_order(const std::vector<double>& x, const std::vector<double>& y);

}  // namespace o2f
