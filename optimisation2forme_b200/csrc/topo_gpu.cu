// Mesh topology on the GPU, equal to the host build (mesh_host.cpp), which
// follows Mesh::Mesh (src/mesh.cpp:7-297) with its std::map and
// std::unordered_set containers:
//   * edges: the std::map<(vmin, vmax), (cL, cR)> of recordEdge gives edge
//     ids in lexicographic key order, cL the first cell that records the
//     edge, cR the second.  Here every (cell, local edge) slot emits its key,
//     a stable radix sort orders the slots by key (equal keys keep the slot
//     order, which is the recording order), and a scan of the key changes
//     numbers the edges;
//   * Cell::edgeIDs, Cell::neighbourIDs, Vertex::cellIDs: one thread per
//     cell or vertex replays the insertion sequence of the host build into
//     the emulated set order (uset_order.h);
//   * edge boundary codes: binary search of the (vmin, vmax) keys of the
//     boundary segments.
// Geometry, the atan2 vertex order and the interpolation weights stay on the
// host (finish_geometry), where they use the same libm as the reference.
// Errors are those of the host build; when a mesh has several faults the
// one reported is the one the host loop meets first for the same kind.
#include <cub/cub.cuh>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh_host.hpp"
#include "solver.hpp"
#include "uset_order.h"

namespace o2f {
namespace {

constexpr int kTB = 256;

enum TopoError : int {
  kErrCellSize = 0,     // only triangles and quadrilaterals
  kErrVertexRange = 1,  // cell vertex out of range
  kErrShared = 2,       // edge shared by more than two cells
  kErrNoBc = 3,         // boundary edge without a boundary condition
  kErrBcInside = 4,     // interior edge carries a boundary condition
  kErrRepeated = 5,     // cell with a repeated vertex
  kErrValence = 6,      // a set larger than the emulation handles
};

// First fault: the lowest (kind, index) wins, the order in which the host
// loops meet them for one kind.
__device__ __forceinline__ void topo_fail(unsigned long long* err, int kind, int64_t index) {
  atomicMin(err, ((unsigned long long)kind << 48) | (unsigned long long)index);
}

__global__ void k_cell_slots(int64_t nc, int64_t nv, const int64_t* __restrict__ off, const int64_t* __restrict__ nodes,
                             uint64_t* __restrict__ key, uint32_t* __restrict__ slot, uint32_t* __restrict__ slot_cell,
                             uint32_t* __restrict__ vkey, uint32_t* __restrict__ vval, unsigned long long* err) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int64_t o0 = off[c], nn = off[c + 1] - o0;
  if (nn != 3 && nn != 4) {
    topo_fail(err, kErrCellSize, c);
    return;
  }
  for (int64_t k = 0; k < nn; ++k) {
    const int64_t a = nodes[o0 + k];
    if (a < 0 || a >= nv) {
      topo_fail(err, kErrVertexRange, c);
      return;
    }
  }
  for (int64_t k = 0; k < nn; ++k) {
    const int64_t a = nodes[o0 + k], b = nodes[o0 + (k + 1) % nn];
    const uint64_t lo = (uint64_t)(a < b ? a : b), hi = (uint64_t)(a < b ? b : a);
    key[o0 + k] = (lo << 32) | hi;
    slot[o0 + k] = (uint32_t)(o0 + k);
    slot_cell[o0 + k] = (uint32_t)c;
    vkey[o0 + k] = (uint32_t)a;  // vertex -> cell pairs in cell order
    vval[o0 + k] = (uint32_t)c;
  }
}

__global__ void k_edge_heads(int64_t n, const uint64_t* __restrict__ key, uint32_t* __restrict__ head,
                             unsigned long long* err) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  head[p] = (p == 0 || key[p] != key[p - 1]) ? 1u : 0u;
  if (p >= 2 && key[p] == key[p - 2]) topo_fail(err, kErrShared, p);
}

// eid = inclusive scan of the heads, minus one.
__global__ void k_edges(int64_t n, const uint64_t* __restrict__ key, const uint32_t* __restrict__ slot,
                        const uint32_t* __restrict__ slot_cell, const uint32_t* __restrict__ scan,
                        int32_t* __restrict__ e_v, int32_t* __restrict__ e_c, int32_t* __restrict__ edge_of_slot) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int64_t e = (int64_t)scan[p] - 1;
  edge_of_slot[slot[p]] = (int32_t)e;
  if (p == 0 || key[p] != key[p - 1]) {
    e_v[2 * e] = (int32_t)(key[p] >> 32);
    e_v[2 * e + 1] = (int32_t)(key[p] & 0xffffffffu);
    e_c[2 * e] = (int32_t)slot_cell[slot[p]];
    e_c[2 * e + 1] = (p + 1 < n && key[p + 1] == key[p]) ? (int32_t)slot_cell[slot[p + 1]] : -1;
  }
}

__global__ void k_edge_codes(int64_t ne, const int32_t* __restrict__ e_v, const int32_t* __restrict__ e_c,
                             int64_t nb, const uint64_t* __restrict__ bkey, const uint8_t* __restrict__ bcode,
                             uint8_t* __restrict__ ebc, unsigned long long* err) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const uint64_t k = ((uint64_t)(uint32_t)e_v[2 * e] << 32) | (uint32_t)e_v[2 * e + 1];
  int64_t lo = 0, hi = nb;
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (bkey[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  const uint8_t code = (lo < nb && bkey[lo] == k) ? bcode[lo] : 0;
  ebc[e] = code;
  const bool boundary = e_c[2 * e + 1] < 0;
  if (boundary && code == 0) topo_fail(err, kErrNoBc, e);
  if (!boundary && code != 0) topo_fail(err, kErrBcInside, e);
}

// Cell::edgeIDs and Cell::neighbourIDs: the host build inserts, edge by edge
// in ascending id, the edge into both of its cells and each cell into the
// other's neighbours.
__global__ void k_cell_sets(int64_t nc, const int64_t* __restrict__ off, const int32_t* __restrict__ edge_of_slot,
                            const int32_t* __restrict__ e_c, int32_t* __restrict__ cedges,
                            int32_t* __restrict__ cnbrs, int32_t* __restrict__ n_nbrs, unsigned long long* err) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const int64_t o0 = off[c];
  const int nn = (int)(off[c + 1] - o0);
  int32_t es[4];
  for (int k = 0; k < nn; ++k) es[k] = edge_of_slot[o0 + k];
  for (int i = 1; i < nn; ++i)  // ascending edge id
    for (int j = i; j > 0 && es[j - 1] > es[j]; --j) {
      const int32_t t = es[j];
      es[j] = es[j - 1];
      es[j - 1] = t;
    }
  uint64_t le[4], ln[4];  // a cell inserts at most 4 edges and 4 neighbours
  int ne_ = 0, nnb = 0;
  for (int k = 0; k < nn; ++k) {
    const int32_t e = es[k];
    uset_insert(le, ne_, (uint64_t)e);
    const int32_t cl = e_c[2 * e], cr = e_c[2 * e + 1];
    if (cr >= 0) uset_insert(ln, nnb, (uint64_t)(cl == c ? cr : cl));
  }
  if (ne_ != nn) topo_fail(err, kErrRepeated, c);
  for (int k = 0; k < ne_; ++k) cedges[o0 + k] = (int32_t)le[k];
  for (int k = 0; k < nnb; ++k) cnbrs[4 * c + k] = (int32_t)ln[k];
  n_nbrs[c] = nnb;
}

// Vertex::cellIDs: cells inserted in ascending order; [voff[v], voff[v+1])
// of the vertex-sorted pairs holds them in that order.
__global__ void k_vertex_sets(int64_t nv, const uint32_t* __restrict__ voff, const uint32_t* __restrict__ vcell,
                              int32_t* __restrict__ vcells, int32_t* __restrict__ vcount, unsigned long long* err) {
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const uint32_t a = voff[v], b = voff[v + 1];
  if (b - a > (uint32_t)kUsetMax) {
    topo_fail(err, kErrValence, v);
    vcount[v] = 0;
    return;
  }
  uint64_t l[kUsetMax];
  int n = 0;
  for (uint32_t i = a; i < b; ++i) uset_insert(l, n, (uint64_t)vcell[i]);
  for (int k = 0; k < n; ++k) vcells[a + k] = (int32_t)l[k];
  vcount[v] = n;
}

__global__ void k_vertex_counts(int64_t n, const uint32_t* __restrict__ vkey, uint32_t* __restrict__ count) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicAdd(&count[vkey[i]], 1u);
}

void check_cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(O2F_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename X>
struct DevBuf {
  X* p = nullptr;
  cudaStream_t s = nullptr;
  DevBuf(size_t n, cudaStream_t st) : s(st) {
    check_cuda(cudaMallocAsync(&p, (n ? n : 1) * sizeof(X), s), "cudaMallocAsync");
  }
  ~DevBuf() {
    if (p) cudaFreeAsync(p, s);
  }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

int grid_of(int64_t n) { return (int)((n + kTB - 1) / kTB); }

}  // namespace

HostMesh build_mesh_gpu(const o2f_mesh_desc& d, void* stream_ptr) {
  if (d.n_nodes <= 0 || d.n_cells <= 0 || !d.node_xy || !d.cell_offsets || !d.cell_nodes)
    throw std::invalid_argument("mesh description: empty or null arrays");
  if (d.n_segments > 0 && (!d.segments || !d.segment_bc))
    throw std::invalid_argument("mesh description: null boundary arrays");
  const int64_t nc = d.n_cells, nv = d.n_nodes, nnz = d.cell_offsets[nc] - d.cell_offsets[0];
  if (d.cell_offsets[0] != 0 || nnz <= 0 || nnz >= (int64_t)1 << 31 || nv >= (int64_t)1 << 31)
    throw std::invalid_argument("mesh description: offsets must start at 0 and sizes fit 31 bits");
  cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
  HostMesh m;
  m.nv = nv;
  m.nc = nc;
  m.vx.resize(nv);
  m.vy.resize(nv);
  m.vbc.assign(nv, 0);
  for (int64_t i = 0; i < nv; ++i) {
    m.vx[i] = d.node_xy[2 * i];
    m.vy[i] = d.node_xy[2 * i + 1];
  }
  const auto bc = boundary_segments(d, m);
  std::vector<uint64_t> bkey;
  std::vector<uint8_t> bcode;
  for (const auto& [k, code] : bc) {  // ascending (vmin, vmax)
    bkey.push_back(((uint64_t)k.first << 32) | (uint64_t)k.second);
    bcode.push_back(code);
  }

  DevBuf<int64_t> off(nc + 1, s), nodes(nnz, s);
  DevBuf<uint64_t> key(nnz, s), key_sorted(nnz, s), dbkey(bkey.size(), s);
  DevBuf<uint32_t> slot(nnz, s), slot_sorted(nnz, s), slot_cell(nnz, s), head(nnz, s), scan(nnz, s);
  DevBuf<uint32_t> vkey(nnz, s), vkey_sorted(nnz, s), vval(nnz, s), vval_sorted(nnz, s), vcnt(nv + 1, s), voff(nv + 1, s);
  DevBuf<int32_t> edge_of_slot(nnz, s), cedges(nnz, s), cnbrs(4 * nc, s), n_nbrs(nc, s), vcells(nnz, s), vcount(nv, s);
  DevBuf<uint8_t> dbcode(bcode.size(), s);
  DevBuf<unsigned long long> err(1, s);
  check_cuda(cudaMemcpyAsync(off.p, d.cell_offsets, (nc + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, s), "copy");
  check_cuda(cudaMemcpyAsync(nodes.p, d.cell_nodes, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, s), "copy");
  if (!bkey.empty()) {
    check_cuda(cudaMemcpyAsync(dbkey.p, bkey.data(), bkey.size() * 8, cudaMemcpyHostToDevice, s), "copy");
    check_cuda(cudaMemcpyAsync(dbcode.p, bcode.data(), bcode.size(), cudaMemcpyHostToDevice, s), "copy");
  }
  check_cuda(cudaMemsetAsync(err.p, 0xff, sizeof(unsigned long long), s), "memset");
  check_cuda(cudaMemsetAsync(vcnt.p, 0, (nv + 1) * sizeof(uint32_t), s), "memset");

  auto fail_if = [&]() {
    unsigned long long e = 0;
    check_cuda(cudaMemcpyAsync(&e, err.p, sizeof(e), cudaMemcpyDeviceToHost, s), "copy");
    check_cuda(cudaStreamSynchronize(s), "topology build");
    if (e == ~0ull) return;
    // the host build's messages (the index of the first fault is in the low
    // 48 bits, which those messages do not carry)
    const int kind = (int)(e >> 48);
    static const char* msg[] = {"only triangles and quadrilaterals are supported", "cell vertex out of range",
                                "edge shared by more than two cells", "boundary edge without a boundary condition",
                                "interior edge carries a boundary condition", "cell with a repeated vertex",
                                "vertex valence above the GPU build's limit"};
    if (kind == kErrValence) throw TopologyLimit(O2F_ERR_MESH, msg[kind]);
    throw Error(O2F_ERR_MESH, msg[kind]);
  };

  k_cell_slots<<<grid_of(nc), kTB, 0, s>>>(nc, nv, off.p, nodes.p, key.p, slot.p, slot_cell.p, vkey.p, vval.p, err.p);
  check_cuda(cudaGetLastError(), "k_cell_slots");
  fail_if();

  // edges: stable sort of the slots by (vmin, vmax)
  size_t tmp_bytes = 0;
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, key_sorted.p, slot.p, slot_sorted.p,
                                             (int)nnz, 0, 64, s), "sort");
  size_t tmp2 = 0;
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, tmp2, vkey.p, vkey_sorted.p, vval.p, vval_sorted.p, (int)nnz, 0,
                                             32, s), "sort");
  size_t tmp3 = 0;
  check_cuda(cub::DeviceScan::InclusiveSum(nullptr, tmp3, head.p, scan.p, (int)nnz, s), "scan");
  size_t tmp4 = 0;
  check_cuda(cub::DeviceScan::ExclusiveSum(nullptr, tmp4, vcnt.p, voff.p, (int)(nv + 1), s), "scan");
  DevBuf<unsigned char> tmp(std::max(std::max(tmp_bytes, tmp2), std::max(tmp3, tmp4)), s);
  const size_t tb = std::max(std::max(tmp_bytes, tmp2), std::max(tmp3, tmp4));
  size_t t = tb;
  check_cuda(cub::DeviceRadixSort::SortPairs(tmp.p, t, key.p, key_sorted.p, slot.p, slot_sorted.p, (int)nnz, 0, 64, s),
             "sort");
  k_edge_heads<<<grid_of(nnz), kTB, 0, s>>>(nnz, key_sorted.p, head.p, err.p);
  t = tb;
  check_cuda(cub::DeviceScan::InclusiveSum(tmp.p, t, head.p, scan.p, (int)nnz, s), "scan");
  uint32_t ne32 = 0;
  check_cuda(cudaMemcpyAsync(&ne32, scan.p + (nnz - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, s), "copy");
  fail_if();
  const int64_t ne = ne32;
  m.ne = ne;
  DevBuf<int32_t> e_v(2 * ne, s), e_c(2 * ne, s);
  DevBuf<uint8_t> ebc(ne, s);
  k_edges<<<grid_of(nnz), kTB, 0, s>>>(nnz, key_sorted.p, slot_sorted.p, slot_cell.p, scan.p, e_v.p, e_c.p,
                                       edge_of_slot.p);
  k_edge_codes<<<grid_of(ne), kTB, 0, s>>>(ne, e_v.p, e_c.p, (int64_t)bkey.size(), dbkey.p, dbcode.p, ebc.p, err.p);
  k_cell_sets<<<grid_of(nc), kTB, 0, s>>>(nc, off.p, edge_of_slot.p, e_c.p, cedges.p, cnbrs.p, n_nbrs.p, err.p);
  // vertices: stable sort of the (vertex, cell) pairs by vertex
  t = tb;
  check_cuda(cub::DeviceRadixSort::SortPairs(tmp.p, t, vkey.p, vkey_sorted.p, vval.p, vval_sorted.p, (int)nnz, 0, 32, s),
             "sort");
  k_vertex_counts<<<grid_of(nnz), kTB, 0, s>>>(nnz, vkey.p, vcnt.p);
  t = tb;
  check_cuda(cub::DeviceScan::ExclusiveSum(tmp.p, t, vcnt.p, voff.p, (int)(nv + 1), s), "scan");
  k_vertex_sets<<<grid_of(nv), kTB, 0, s>>>(nv, voff.p, vval_sorted.p, vcells.p, vcount.p, err.p);
  check_cuda(cudaGetLastError(), "topology kernels");
  fail_if();

  // back to the host arrays
  std::vector<int32_t> hv(2 * ne), hc(2 * ne), hce(nnz), hcn(4 * nc), hnn(nc), hvc(nnz), hvn(nv);
  std::vector<uint32_t> hvo(nv + 1);
  m.ebc.resize(ne);
  check_cuda(cudaMemcpyAsync(hv.data(), e_v.p, hv.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hc.data(), e_c.p, hc.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(m.ebc.data(), ebc.p, ne, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hce.data(), cedges.p, hce.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hcn.data(), cnbrs.p, hcn.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hnn.data(), n_nbrs.p, hnn.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hvc.data(), vcells.p, hvc.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hvn.data(), vcount.p, hvn.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaMemcpyAsync(hvo.data(), voff.p, hvo.size() * 4, cudaMemcpyDeviceToHost, s), "copy");
  check_cuda(cudaStreamSynchronize(s), "topology build");

  m.e_v0.resize(ne);
  m.e_v1.resize(ne);
  m.e_cl.resize(ne);
  m.e_cr.resize(ne);
  for (int64_t e = 0; e < ne; ++e) {
    m.e_v0[e] = hv[2 * e];
    m.e_v1[e] = hv[2 * e + 1];
    m.e_cl[e] = hc[2 * e];
    m.e_cr[e] = hc[2 * e + 1];
  }
  m.cell_voff.assign(d.cell_offsets, d.cell_offsets + nc + 1);
  m.cell_verts.assign(d.cell_nodes, d.cell_nodes + nnz);
  m.cell_eoff = m.cell_voff;
  m.cell_edges.assign(hce.begin(), hce.end());
  m.cell_noff.assign(nc + 1, 0);
  m.cell_nbrs.clear();
  m.cell_nbrs.reserve(4 * nc);
  for (int64_t c = 0; c < nc; ++c) {
    for (int k = 0; k < hnn[c]; ++k) m.cell_nbrs.push_back(hcn[4 * c + k]);
    m.cell_noff[c + 1] = (int64_t)m.cell_nbrs.size();
  }
  m.vert_coff.assign(nv + 1, 0);
  m.vert_cells.clear();
  m.vert_cells.reserve(nnz);
  for (int64_t v = 0; v < nv; ++v) {
    for (int k = 0; k < hvn[v]; ++k) m.vert_cells.push_back(hvc[hvo[v] + k]);
    m.vert_coff[v + 1] = (int64_t)m.vert_cells.size();
    m.max_valence = std::max<int64_t>(m.max_valence, hvn[v]);
  }
  finish_geometry(m);
  return m;
}

}  // namespace o2f
