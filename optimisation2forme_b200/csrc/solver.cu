// Host drivers of the solver context: device upload of the renumbered mesh and
// the launch sequences of the residual, time loop, adjoint and shape gradient.
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

#include "deform.cuh"
#include "ilu.cuh"
#include "jacobian.cuh"
#include "render.cuh"
#include "kernels_adjoint.cuh"

namespace o2f {

void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(O2F_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceArena::~DeviceArena() {
  for (void* p : ptrs_) cudaFree(p);
}

void* DeviceArena::raw(size_t bytes) {
  void* p = nullptr;
  if (bytes == 0) bytes = 32;
  O2F_CUDA(cudaMalloc(&p, bytes));
  ptrs_.push_back(p);
  bytes_ += bytes;
  return p;
}

namespace {

template <typename X>
void h2d(X* dst, const std::vector<X>& src, cudaStream_t s) {
  if (!src.empty()) O2F_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(X), cudaMemcpyHostToDevice, s));
}

void validate_params(const o2f_params& p) {
  if (!(p.gamma > 1.0) || !(p.viscosity >= 0.0) || !(p.Pr > 0.0) || !(p.cp > 0.0) || !(p.rho_ref > 0.0) ||
      !(p.p_ref > 0.0) || !(p.cfl_number > 0.0) || !(p.inflow_velocity >= 0.0) || !(p.limiter_k > 0.0))
    throw Error(O2F_ERR_ARG, "invalid physical parameters");
  if (p.limiter != O2F_LIMITER_VENKAT && p.limiter != O2F_LIMITER_BARTH_JESPERSEN)
    throw Error(O2F_ERR_ARG, "unknown limiter");
  if (p.precision != O2F_PREC_F64 && p.precision != O2F_PREC_F32) throw Error(O2F_ERR_ARG, "unknown precision");
  if (p.adjoint_precision != O2F_PREC_F64 && p.adjoint_precision != O2F_PREC_F32)
    throw Error(O2F_ERR_ARG, "unknown adjoint_precision");
  if (p.adjoint_sweeps != O2F_SWEEPS_AUTO && p.adjoint_sweeps != O2F_SWEEPS_BLOCK &&
      p.adjoint_sweeps != O2F_SWEEPS_WAITING)
    throw Error(O2F_ERR_ARG, "unknown adjoint_sweeps");
  if (p.adjoint_precond != O2F_PRECOND_NONE && p.adjoint_precond != O2F_PRECOND_ILU0)
    throw Error(O2F_ERR_ARG, "unknown adjoint preconditioner");
  if (p.dt_mode != O2F_DT_REFERENCE && p.dt_mode != O2F_DT_THERMAL) throw Error(O2F_ERR_ARG, "unknown dt_mode");
  if (p.adjoint_jacobian != O2F_JAC_REFERENCE && p.adjoint_jacobian != O2F_JAC_FULL &&
      p.adjoint_jacobian != O2F_JAC_FROZEN)
    throw Error(O2F_ERR_ARG, "unknown adjoint_jacobian");
  if (!(p.adjoint_fd_step > 0.0) || !(p.adjoint_fd_step < 1.0)) throw Error(O2F_ERR_ARG, "adjoint_fd_step out of range");
  if (!(p.adjoint_shift >= 0.0) || !(p.adjoint_shift < 1e6)) throw Error(O2F_ERR_ARG, "adjoint_shift out of range");
}

}  // namespace

Solver::Solver(const o2f_mesh_desc& desc, const o2f_params& p, cudaStream_t stream) {
  validate_params(p);
  int dev_count = 0;
  O2F_CUDA(cudaGetDeviceCount(&dev_count));
  if (stream) {
    stream_ = stream;
  } else {
    O2F_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    own_stream_ = true;
  }
  // Large meshes: integer topology on the GPU (the same mesh, array for
  // array; topo_gpu.cu), unless a vertex has more cells than its set
  // emulation handles.
  try {
    bool built = false;
    if (desc.n_cells >= kGpuTopologyCells) {
      try {
        hm_ = build_mesh_gpu(desc, stream_);
        built = true;
      } catch (const TopologyLimit&) {
      }
    }
    if (!built) hm_ = build_mesh(desc);
  } catch (...) {
    // the destructor does not run for a failed constructor
    if (own_stream_) cudaStreamDestroy(stream_);
    try {
      throw;
    } catch (const Error&) {
      throw;
    } catch (const std::invalid_argument& e) {
      throw Error(O2F_ERR_ARG, e.what());
    } catch (const std::runtime_error& e) {
      throw Error(O2F_ERR_MESH, e.what());
    }
  }
  if (hm_.nc >= (int64_t(1) << 30) || hm_.ne >= (int64_t(1) << 30)) throw Error(O2F_ERR_MESH, "mesh too large");
  O2F_CUDA(cudaEventCreate(&ev0_));
  O2F_CUDA(cudaEventCreate(&ev1_));
  // Pinned mailbox of the device-driven loops (step / Krylov state), kept
  // for the context's life: no pinned allocation or free during a solve,
  // whose implicit synchronisation could disturb another thread's stream
  // capture.
  O2F_CUDA(cudaMallocHost(&mailbox_, std::max(sizeof(StepState), sizeof(KrylovState))));
  params_ = p;
  min_h_ = min_cell_h(hm_);
  upload_mesh();
  set_params(p);
  state_freestream();
  sync();
}

Solver::~Solver() {
  if (stream_) cudaStreamSynchronize(stream_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (mailbox_) cudaFreeHost(mailbox_);
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
}

void Solver::sync() { O2F_CUDA(cudaStreamSynchronize(stream_)); }

void Solver::compute_phys() { phys_ = phys_of(params_); }

Phys phys_of(const o2f_params& p) {
  Phys ph{};
  ph.gamma = p.gamma;
  ph.mu = p.viscosity;
  ph.cp = p.cp;
  ph.Pr = p.Pr;
  ph.kappa = p.viscosity * p.cp / p.Pr;  // src/diffusion.cpp:210
  // Freestream (src/boundary.cpp:10-17), rotated by the angle of attack;
  // cos(0) = 1 and sin(0) = 0 keep the reference's values bit for bit.
  const double rho0 = p.rho_ref, p0 = p.p_ref, M = p.inflow_velocity;
  const double a0 = std::sqrt(p.gamma * p0 / rho0);
  const double u0 = M * a0;
  const double alpha = p.aoa_deg * (3.14159265358979323846 / 180.0);
  ph.cos_a = std::cos(alpha);
  ph.sin_a = std::sin(alpha);
  if (p.aoa_deg == 0.0) {
    ph.cos_a = 1.0;
    ph.sin_a = 0.0;
  }
  const double ux = u0 * ph.cos_a, uy = u0 * ph.sin_a;
  const double kinetic = 0.5 * rho0 * (ux * ux + uy * uy);
  ph.fs_rho = rho0;
  ph.fs_rhou = rho0 * ux;
  ph.fs_rhov = rho0 * uy;
  ph.fs_E = p.p_ref / (p.gamma - 1.0) + kinetic;
  // q_inf of computeLiftDragCoefficients (src/compute.cpp:93-100).
  const double a_inf = std::sqrt(p.gamma * p0 / rho0);
  const double U_inf = M * a_inf;
  ph.q_inf = 0.5 * (rho0 * U_inf * U_inf);
  ph.limiter_k = p.limiter_k;
  ph.limiter = p.limiter;
  return ph;
}

void Solver::set_params(const o2f_params& p) {
  validate_params(p);
  params_ = p;
  compute_phys();
  k_venkat_eps<double><<<grid(topo_.nc), kBlock, 0, stream_>>>(topo_.nc, p.limiter_k, geom_.cgeom);
  O2F_CUDA(cudaGetLastError());
  invalidate_linearisation();
  f32_geom_valid_ = false;  // the FP32 geometry copy holds the old limiter eps
}

void Solver::upload_mesh() {
  const HostMesh& m = hm_;
  const int64_t nc = m.nc, ne = m.ne, nv = m.nv;
  // Hilbert order of cells and vertices; edges follow their lower-numbered cell.
  cperm_ = hilbert_order(m.ccx, m.ccy);
  vperm_ = hilbert_order(m.vx, m.vy);
  cinv_.assign(nc, 0);
  vinv_.assign(nv, 0);
  for (int64_t i = 0; i < nc; ++i) cinv_[cperm_[i]] = i;
  for (int64_t i = 0; i < nv; ++i) vinv_[vperm_[i]] = i;
  std::vector<int64_t> ekey(ne);
  for (int64_t e = 0; e < ne; ++e) {
    int64_t a = cinv_[m.e_cl[e]];
    int64_t b = m.e_cr[e] >= 0 ? cinv_[m.e_cr[e]] : a;
    ekey[e] = std::min(a, b);
  }
  eperm_.resize(ne);
  std::iota(eperm_.begin(), eperm_.end(), 0);
  std::stable_sort(eperm_.begin(), eperm_.end(), [&](int64_t x, int64_t y) { return ekey[x] < ekey[y]; });
  einv_.assign(ne, 0);
  for (int64_t i = 0; i < ne; ++i) einv_[eperm_[i]] = i;

  topo_.nc = nc;
  topo_.ne = ne;
  topo_.nv = nv;
  topo_.nnz = (int64_t)m.vert_wcells.size();

  // Cells.
  std::vector<int32_t> slot(4 * nc, -1), jslot(4 * nc, -1), cverts(4 * nc, -1);
  std::vector<uint8_t> ctype(nc);
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t co = cperm_[c];
    const int64_t o0 = m.cell_eoff[co], o1 = m.cell_eoff[co + 1];
    std::vector<int64_t> ids(m.cell_edges.begin() + o0, m.cell_edges.begin() + o1);
    for (int64_t k = 0; k < o1 - o0; ++k) {
      const int64_t eo = ids[k];
      const int side = (m.e_cl[eo] == co) ? 0 : 1;
      slot[k * nc + c] = (int32_t)(2 * einv_[eo] + side);
    }
    std::sort(ids.begin(), ids.end());
    for (int64_t k = 0; k < o1 - o0; ++k) {
      const int64_t eo = ids[k];
      const int side = (m.e_cl[eo] == co) ? 0 : 1;
      jslot[k * nc + c] = (int32_t)(2 * einv_[eo] + side);
    }
    const int64_t v0 = m.cell_voff[co], v1 = m.cell_voff[co + 1];
    ctype[c] = (uint8_t)(v1 - v0);
    for (int64_t k = 0; k < v1 - v0; ++k) cverts[4 * c + k] = (int32_t)vinv_[m.cell_verts[v0 + k]];
  }
  // Edges.
  std::vector<int2> ev(ne), ec(ne);
  std::vector<uint8_t> ebc(ne);
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t eo = eperm_[e];
    ev[e] = make_int2((int)vinv_[m.e_v0[eo]], (int)vinv_[m.e_v1[eo]]);
    ec[e] = make_int2((int)cinv_[m.e_cl[eo]], m.e_cr[eo] >= 0 ? (int)cinv_[m.e_cr[eo]] : -1);
    ebc[e] = m.ebc[eo];
  }
  // Vertices.
  std::vector<int32_t> voff(nv + 1);
  std::vector<uint8_t> vbc(nv);
  voff[0] = 0;
  for (int64_t v = 0; v < nv; ++v) {
    const int64_t vo = vperm_[v];
    voff[v + 1] = voff[v] + (int32_t)(m.vert_coff[vo + 1] - m.vert_coff[vo]);
    vbc[v] = m.vbc[vo];
  }
  // Wall edges in ascending reference id; cells owning them.
  wall_edges_host_.clear();
  std::vector<std::vector<int32_t>> wc_edges(nc);
  std::vector<int32_t> wall_cells;
  for (int64_t eo = 0; eo < ne; ++eo) {
    if (m.ebc[eo] != 'w') continue;
    wall_edges_host_.push_back((int32_t)einv_[eo]);
    const int64_t c = cinv_[m.e_cl[eo]];
    if (wc_edges[c].empty()) wall_cells.push_back((int32_t)c);
    wc_edges[c].push_back((int32_t)einv_[eo]);
  }
  std::vector<int32_t> wc_off{0}, wc_list;
  for (int32_t c : wall_cells) {
    for (int32_t e : wc_edges[c]) wc_list.push_back(e);
    wc_off.push_back((int32_t)wc_list.size());
  }
  // Shape-perturbation sets (src/shape_optimization.cpp:750-755,857-859).
  std::vector<int32_t> pverts, pedges, pcells, pwverts;
  std::vector<uint8_t> cmark(nc, 0), vmark(nv, 0);
  for (int64_t v = 0; v < nv; ++v)
    if (vbc[v] == 'w') pverts.push_back((int32_t)v);
  for (int64_t e = 0; e < ne; ++e) {
    if (ebc[e] == 'w' || vbc[ev[e].x] == 'w' || vbc[ev[e].y] == 'w') {
      pedges.push_back((int32_t)e);
      const int c = ec[e].x;
      if (!cmark[c]) {
        cmark[c] = 1;
        pcells.push_back(c);
      }
    }
  }
  for (int32_t c : pcells)
    for (int k = 0; k < ctype[c]; ++k) vmark[cverts[4 * c + k]] = 1;
  for (int32_t v : pverts) vmark[v] = 1;
  for (int64_t v = 0; v < nv; ++v)
    if (vmark[v]) pwverts.push_back((int32_t)v);

  // Device upload.
  cudaStream_t s = stream_;
  topo_.slot = arena_.alloc<int32_t>(slot.size());
  topo_.jslot = arena_.alloc<int32_t>(jslot.size());
  topo_.cverts = arena_.alloc<int32_t>(cverts.size());
  topo_.ctype = arena_.alloc<uint8_t>(ctype.size());
  topo_.ev = arena_.alloc<int2>(ne);
  topo_.ec = arena_.alloc<int2>(ne);
  topo_.ebc = arena_.alloc<uint8_t>(ne);
  topo_.voff = arena_.alloc<int32_t>(nv + 1);
  topo_.vbc = arena_.alloc<uint8_t>(nv);
  topo_.n_wall = (int64_t)wall_edges_host_.size();
  topo_.wall_edges = arena_.alloc<int32_t>(wall_edges_host_.size());
  topo_.n_wall_cells = (int64_t)wall_cells.size();
  topo_.wall_cells = arena_.alloc<int32_t>(wall_cells.size());
  topo_.wall_cell_off = arena_.alloc<int32_t>(wc_off.size());
  topo_.wall_cell_edges = arena_.alloc<int32_t>(wc_list.size());
  topo_.n_pert_verts = (int64_t)pverts.size();
  topo_.pert_verts = arena_.alloc<int32_t>(pverts.size());
  topo_.n_pert_edges = (int64_t)pedges.size();
  topo_.pert_edges = arena_.alloc<int32_t>(pedges.size());
  topo_.n_pert_cells = (int64_t)pcells.size();
  topo_.pert_cells = arena_.alloc<int32_t>(pcells.size());
  topo_.n_pert_wverts = (int64_t)pwverts.size();
  topo_.pert_wverts = arena_.alloc<int32_t>(pwverts.size());
  h2d(topo_.slot, slot, s);
  h2d(topo_.jslot, jslot, s);
  h2d(topo_.cverts, cverts, s);
  h2d(topo_.ctype, ctype, s);
  h2d(topo_.ev, ev, s);
  h2d(topo_.ec, ec, s);
  h2d(topo_.ebc, ebc, s);
  h2d(topo_.voff, voff, s);
  h2d(topo_.vbc, vbc, s);
  h2d(topo_.wall_edges, wall_edges_host_, s);
  h2d(topo_.wall_cells, wall_cells, s);
  h2d(topo_.wall_cell_off, wc_off, s);
  h2d(topo_.wall_cell_edges, wc_list, s);
  h2d(topo_.pert_verts, pverts, s);
  h2d(topo_.pert_edges, pedges, s);
  h2d(topo_.pert_cells, pcells, s);
  h2d(topo_.pert_wverts, pwverts, s);

  upload_geometry();

  work_ = alloc_work();
  U_ = arena_.alloc<Vec4<double>>(nc);
  Uold_ = arena_.alloc<Vec4<double>>(nc);
  norm_part_ = arena_.alloc<double>(grid(nc));
  step_ = arena_.alloc<StepState>(1);
  part_ = arena_.alloc<double>(kRedGrid * 4);
  ticket_ = arena_.alloc<unsigned int>(4);
  scal_ = arena_.alloc<double>(16);
  ks_ = arena_.alloc<KrylovState>(1);
  O2F_CUDA(cudaMemsetAsync(ticket_, 0, 4 * sizeof(unsigned int), s));
  O2F_CUDA(cudaMemsetAsync(ks_, 0, sizeof(KrylovState), s));
  sync();  // host staging vectors go out of scope
  setup_ilu_host(jslot, ec, ebc);
}

// Geometry of the host mesh in device order: cell centres and volumes, edge
// normals, lengths and centres, vertex coordinates, and the interpolation
// weights with their cells (the weights' cell order follows the geometry:
// Vertex::cellIDsOrdered).  The buffers are allocated on the first call and
// overwritten by later ones (set_vertex_coords), so captured graphs stay valid.
void Solver::upload_geometry() {
  const HostMesh& m = hm_;
  const int64_t nc = m.nc, ne = m.ne, nv = m.nv;
  std::vector<Vec4<double>> cgeom(nc);
  for (int64_t c = 0; c < nc; ++c) {
    const int64_t co = cperm_[c];
    cgeom[c] = Vec4<double>{m.ccx[co], m.ccy[co], m.cvol[co], 0.0};
  }
  std::vector<Vec4<double>> egeom(ne);
  std::vector<Vec2<double>> ectr(ne);
  for (int64_t e = 0; e < ne; ++e) {
    const int64_t eo = eperm_[e];
    egeom[e] = Vec4<double>{m.enx[eo], m.eny[eo], m.elen[eo], 0.0};
    ectr[e] = Vec2<double>{m.ecx[eo], m.ecy[eo]};
  }
  std::vector<int32_t> vcid(topo_.nnz);
  std::vector<double> vw(topo_.nnz);
  std::vector<Vec2<double>> vxy(nv);
  int64_t j = 0;
  for (int64_t v = 0; v < nv; ++v) {
    const int64_t vo = vperm_[v];
    for (int64_t k = m.vert_coff[vo]; k < m.vert_coff[vo + 1]; ++k, ++j) {
      vcid[j] = (int32_t)cinv_[m.vert_wcells[k]];
      vw[j] = m.vert_w[k];
    }
    vxy[v] = Vec2<double>{m.vx[vo], m.vy[vo]};
  }
  if (!geom_.cgeom) {
    topo_.vcid = arena_.alloc<int32_t>(vcid.size());
    topo_.vcid_ord = topo_.vcid;
    geom_.cgeom = arena_.alloc<Vec4<double>>(nc);
    geom_.egeom = arena_.alloc<Vec4<double>>(ne);
    geom_.ectr = arena_.alloc<Vec2<double>>(ne);
    geom_.vxy = arena_.alloc<Vec2<double>>(nv);
    geom_.vw = arena_.alloc<double>(vw.size());
  }
  cudaStream_t s = stream_;
  h2d(topo_.vcid, vcid, s);
  h2d(geom_.cgeom, cgeom, s);
  h2d(geom_.egeom, egeom, s);
  h2d(geom_.ectr, ectr, s);
  h2d(geom_.vxy, vxy, s);
  h2d(geom_.vw, vw, s);
  sync();  // the staging vectors go out of scope
}

void Solver::set_vertex_coords(const double* xy) {
  NvtxRange nvtx_("o2f set_vertex_coords");
  try {
    set_coordinates(hm_, xy);
  } catch (const std::invalid_argument& e) {
    throw Error(O2F_ERR_ARG, e.what());
  } catch (const std::runtime_error& e) {
    throw Error(O2F_ERR_MESH, e.what());
  }
  min_h_ = min_cell_h(hm_);
  upload_geometry();
  set_params(params_);  // limiter eps from the new volumes; J^T blocks and FP32 geometry invalid
  have_residual_ = false;
  have_lambda_ = false;
}

void Solver::deform_shape(const o2f_shape_params& from, const o2f_shape_params& to, int power) {
  NvtxRange nvtx_("o2f deform_shape");
  if (power < 1 || power > 8) throw Error(O2F_ERR_ARG, "IDW power must be in [1, 8]");
  if (from.pos_x != to.pos_x || from.c != to.c)
    throw Error(O2F_ERR_ARG, "deform_shape moves m, p, t; pos_x and c must not change");
  const int64_t nv = topo_.nv;
  cudaStream_t s = stream_;
  if (!deform_alloc_) {
    std::vector<uint8_t> vbc(nv);
    for (int64_t v = 0; v < nv; ++v) vbc[v] = hm_.vbc[vperm_[v]];
    std::vector<int32_t> src;
    for (int64_t v = 0; v < nv; ++v)
      if (vbc[v] != 0) src.push_back((int32_t)v);
    if (src.empty()) throw Error(O2F_ERR_MESH, "the mesh has no boundary vertices");
    n_idw_src_ = (int64_t)src.size();
    idw_src_ = arena_.alloc<int32_t>(src.size());
    idw_sxy_ = arena_.alloc<Vec2<double>>(src.size());
    idw_sd_ = arena_.alloc<Vec2<double>>(src.size());
    dvxy_ = arena_.alloc<Vec2<double>>(nv);
    h2d(idw_src_, src, s);
    sync();
    deform_alloc_ = true;
  }
  // wall vertices to the new shape (the perturbation of the shape gradient)
  O2F_CUDA(cudaMemcpyAsync(dvxy_, geom_.vxy, nv * sizeof(Vec2<double>), cudaMemcpyDeviceToDevice, s));
  ShapeArgs a{};
  a.pos_x = from.pos_x;
  a.c = from.c;
  a.m0 = from.m;
  a.p0 = from.p;
  a.t0 = from.t;
  a.m1 = to.m;
  a.p1 = to.p;
  a.t1 = to.t;
  if (topo_.n_pert_verts)
    k_perturb_vertices<<<grid(topo_.n_pert_verts), kBlock, 0, s>>>(topo_.n_pert_verts, topo_.pert_verts, a, dvxy_);
  k_idw_sources<<<grid(n_idw_src_), kBlock, 0, s>>>(n_idw_src_, idw_src_, geom_.vxy, dvxy_, idw_sxy_, idw_sd_);
  k_idw_deform<<<(int)((nv + kIdwTile - 1) / kIdwTile), kIdwTile, 0, s>>>(nv, topo_.vbc, geom_.vxy, n_idw_src_,
                                                                       idw_sxy_, idw_sd_, power, dvxy_);
  O2F_CUDA(cudaGetLastError());
  launches_ += 3;
  std::vector<Vec2<double>> moved(nv);
  O2F_CUDA(cudaMemcpyAsync(moved.data(), dvxy_, nv * sizeof(Vec2<double>), cudaMemcpyDeviceToHost, s));
  sync();
  std::vector<double> xy(2 * nv);
  for (int64_t v = 0; v < nv; ++v) {
    xy[2 * vperm_[v]] = moved[v].a;
    xy[2 * vperm_[v] + 1] = moved[v].b;
  }
  set_vertex_coords(xy.data());
}

void Solver::render_field(const std::string& field, int nx, int ny, const std::string& cmap, const double* range_in,
                          unsigned char* rgb, double* range_out) {
  NvtxRange nvtx_("o2f render_field");
  static const char* names[] = {"rho", "rho_u", "rho_v", "E", "u", "v", "u_x", "u_y", "v_x", "v_y", "div", "p"};
  int f = -1;
  for (int k = 0; k < 12; ++k)
    if (field == names[k]) f = k;
  if (field == "pressure") f = kFieldP;
  if (f < 0) throw Error(O2F_ERR_ARG, "unknown field '" + field + "' (computeCellScalar)");
  if (nx <= 0 || ny <= 0 || (int64_t)nx * ny > (int64_t)1 << 28) throw Error(O2F_ERR_ARG, "image size out of range");
  if (!rgb) throw Error(O2F_ERR_ARG, "null image");
  const int64_t nc = topo_.nc, npix = (int64_t)nx * ny;
  cudaStream_t s = stream_;
  // the gradient fields read the Green-Gauss gradients of a residual of the current state
  const bool needs_grad = f >= kFieldUx && f <= kFieldDiv;
  if (needs_grad) {
    launch_residual(geom_, work_, U_, nullptr, true, nullptr);
    have_residual_ = true;
  }
  if (!render_ref_id_) {
    std::vector<int32_t> ids(nc);
    for (int64_t c = 0; c < nc; ++c) ids[c] = (int32_t)cperm_[c];
    render_ref_id_ = arena_.alloc<int32_t>(nc);
    render_scalar_ = arena_.alloc<double>(nc);
    render_part_ = arena_.alloc<double>(2 * 1184);
    h2d(render_ref_id_, ids, s);
  }
  k_cell_scalar<<<grid(nc), kBlock, 0, s>>>(nc, U_, work_.grad, f, params_.gamma, render_scalar_);
  const int parts = std::min(grid(nc), 1184);
  k_scalar_minmax<<<parts, kBlock, 0, s>>>(nc, render_scalar_, render_part_);
  std::vector<double> part(2 * parts);
  O2F_CUDA(cudaMemcpyAsync(part.data(), render_part_, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
  // view: the bounding box of the vertices (Mesh::Mesh, src/mesh.cpp:27-44)
  double x_min = INFINITY, x_max = -INFINITY, y_min = INFINITY, y_max = -INFINITY;
  for (int64_t v = 0; v < hm_.nv; ++v) {
    x_min = std::min(x_min, hm_.vx[v]);
    x_max = std::max(x_max, hm_.vx[v]);
    y_min = std::min(y_min, hm_.vy[v]);
    y_max = std::max(y_max, hm_.vy[v]);
  }
  sync();
  double smin = INFINITY, smax = -INFINITY;
  for (int k = 0; k < parts; ++k) {
    if (smin > part[2 * k]) smin = part[2 * k];
    if (smax < part[2 * k + 1]) smax = part[2 * k + 1];
  }
  double fmin_ = smin, fmax_ = smax;
  if (range_in) {
    fmin_ = range_in[0];
    fmax_ = range_in[1];
  } else if (f == kFieldP) {
    // Simulator::output_step (src/simulation.cpp:188-193): pressure range in steps of 5000
    const double step = 5000.0;
    fmin_ = std::floor(smin / step) * step;
    fmax_ = std::ceil(smax / step) * step;
  }
  if (range_out) {
    range_out[0] = fmin_;
    range_out[1] = fmax_;
  }
  const double span = fmax_ - fmin_;
  std::memset(rgb, 0, 3 * (size_t)npix);
  if (!(span > 0.0)) return;  // render_scalar_field_unstructured draws nothing
  // per-call scratch (the image size varies), freed on every exit
  struct Scratch {
    void* p = nullptr;
    cudaStream_t s;
    ~Scratch() {
      if (p) cudaFreeAsync(p, s);
    }
  } pix_buf{nullptr, s}, img_buf{nullptr, s};
  O2F_CUDA(cudaMallocAsync(&pix_buf.p, npix * sizeof(unsigned long long), s));
  O2F_CUDA(cudaMallocAsync(&img_buf.p, 3 * npix, s));
  auto* pix = static_cast<unsigned long long*>(pix_buf.p);
  auto* img = static_cast<unsigned char*>(img_buf.p);
  RenderView w{x_min, y_min, std::abs(x_max - x_min), std::abs(y_max - y_min), nx, ny};
  O2F_CUDA(cudaMemsetAsync(pix, 0xff, npix * sizeof(unsigned long long), s));
  k_raster_cells<<<grid(nc), kBlock, 0, s>>>(nc, topo_.cverts, topo_.ctype, geom_.vxy, render_ref_id_, w, pix);
  k_colour_pixels<<<(int)((npix + kBlock - 1) / kBlock), kBlock, 0, s>>>(nx, ny, pix, render_scalar_, fmin_, span,
                                                                         cmap == "schlieren" ? 1 : 0, img);
  O2F_CUDA(cudaGetLastError());
  O2F_CUDA(cudaMemcpyAsync(rgb, img, 3 * npix, cudaMemcpyDeviceToHost, s));
  sync();
  launches_ += 4;
}

// Reverse Cuthill-McKee order of the cell adjacency graph (BFS from a
// pseudo-peripheral cell, neighbours by increasing degree, reversed), and the
// level sets of the factorization in that order.
void Solver::setup_ilu_host(const std::vector<int32_t>& jslot, const std::vector<int2>& ec,
                            const std::vector<uint8_t>& ebc) {
  const int64_t nc = topo_.nc;
  ilu_nbr_h_.assign(4 * nc, -1);
  for (int64_t c = 0; c < nc; ++c)
    for (int k = 0; k < 4; ++k) {
      const int sl = jslot[k * nc + c];
      if (sl < 0) continue;
      const int e = sl >> 1;
      if (ebc[e] != 0) continue;
      ilu_nbr_h_[k * nc + c] = (sl & 1) == 0 ? ec[e].y : ec[e].x;
    }
  auto nbr = [&](int64_t c, int k) { return ilu_nbr_h_[k * nc + c]; };
  std::vector<int> deg(nc, 0);
  for (int64_t c = 0; c < nc; ++c)
    for (int k = 0; k < 4; ++k) deg[c] += nbr(c, k) >= 0;
  std::vector<int> seen(nc, 0);
  std::vector<int32_t> lvl(nc);
  int stamp = 0;
  auto bfs = [&](int32_t root, std::vector<int32_t>& out) {  // BFS order into out, depth into lvl
    out.clear();
    out.push_back(root);
    lvl[root] = 0;
    ++stamp;
    seen[root] = stamp;
    for (size_t h = 0; h < out.size(); ++h) {
      const int32_t u = out[h];
      int32_t nb[4];
      int n = 0;
      for (int k = 0; k < 4; ++k) {
        const int32_t v = nbr(u, k);
        if (v >= 0 && seen[v] != stamp) nb[n++] = v;
      }
      std::sort(nb, nb + n, [&](int32_t a, int32_t b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
      for (int i = 0; i < n; ++i) {
        if (seen[nb[i]] == stamp) continue;
        seen[nb[i]] = stamp;
        lvl[nb[i]] = lvl[u] + 1;
        out.push_back(nb[i]);
      }
    }
  };
  std::vector<int32_t> order;
  order.reserve(nc);
  std::vector<char> placed(nc, 0);
  std::vector<int32_t> comp;
  for (int64_t start = 0; start < nc; ++start) {
    if (placed[start]) continue;
    // pseudo-peripheral root: repeat the BFS from the farthest low-degree cell
    int32_t root = (int32_t)start;
    int depth = -1;
    for (int it = 0; it < 4; ++it) {
      bfs(root, comp);
      const int d = lvl[comp.back()];
      if (d <= depth) break;
      depth = d;
      int32_t best = comp.back();
      for (auto r = comp.rbegin(); r != comp.rend() && lvl[*r] == d; ++r)
        if (deg[*r] < deg[best]) best = *r;
      root = best;
    }
    bfs(root, comp);
    for (int32_t c : comp) placed[c] = 1;
    order.insert(order.end(), comp.begin(), comp.end());
  }
  std::reverse(order.begin(), order.end());
  ilu_pos_h_.assign(nc, 0);
  for (int64_t i = 0; i < nc; ++i) ilu_pos_h_[order[i]] = (int32_t)i;
  std::vector<int32_t> lev(nc, 0);
  auto bucket = [&](int nl, std::vector<int32_t>& off, std::vector<int32_t>& cells) {
    off.assign(nl + 1, 0);
    for (int64_t c = 0; c < nc; ++c) off[lev[c] + 1]++;
    for (int l = 0; l < nl; ++l) off[l + 1] += off[l];
    cells.assign(nc, 0);
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int64_t i = 0; i < nc; ++i) cells[fill[lev[order[i]]]++] = order[i];
  };
  int nlo = 0;
  for (int64_t i = 0; i < nc; ++i) {
    const int32_t c = order[i];
    int l = 0;
    for (int k = 0; k < 4; ++k) {
      const int32_t o = nbr(c, k);
      if (o >= 0 && ilu_pos_h_[o] < i) l = std::max(l, lev[o] + 1);
    }
    lev[c] = l;
    nlo = std::max(nlo, l + 1);
  }
  bucket(nlo, lo_off_h_, lo_cells_h_);
  // Sweep orders: the forward solve's rows by forward level (the
  // factorization's level sets above, each in RCM order), the backward
  // solve's by the levels of the upper-triangle dependencies.  Both are
  // topological orders of their triangle, so each row computes exactly what
  // it computes in the RCM order, but the rows a warp claims together no
  // longer wait on one another.
  std::vector<int32_t> levu(nc, 0);
  int nup = 0;
  for (int64_t i = nc - 1; i >= 0; --i) {
    const int32_t c = order[i];
    int l = 0;
    for (int k = 0; k < 4; ++k) {
      const int32_t o = nbr(c, k);
      if (o >= 0 && ilu_pos_h_[o] > i) l = std::max(l, levu[o] + 1);
    }
    levu[c] = l;
    nup = std::max(nup, l + 1);
  }
  std::vector<int32_t> up_off(nup + 1, 0);
  for (int64_t c = 0; c < nc; ++c) up_off[levu[c] + 1]++;
  for (int l = 0; l < nup; ++l) up_off[l + 1] += up_off[l];
  ilu_sweep_h_.assign(2 * nc, 0);
  std::copy(lo_cells_h_.begin(), lo_cells_h_.end(), ilu_sweep_h_.begin());
  {
    std::vector<int32_t> fill(up_off.begin(), up_off.end() - 1);
    for (int64_t i = nc - 1; i >= 0; --i) ilu_sweep_h_[nc + fill[levu[order[i]]]++] = order[i];
  }
  ilu_n_up_ = nup;
  // level offsets of both sweep orders, forward then backward
  ilu_lev_off_h_.assign(lo_off_h_.begin(), lo_off_h_.end());
  ilu_lev_off_h_.insert(ilu_lev_off_h_.end(), up_off.begin(), up_off.end());
  // Records of the block sweeps, per sweep position p (8 int32): the row,
  // the sweep positions of its dependencies in slot order (-1: none), their
  // slots (8 bits each), and for the backward sweep the row's forward
  // position (where its forward value is).
  {
    std::vector<int32_t> posf(nc), posb(nc);
    for (int64_t p = 0; p < nc; ++p) {
      posf[ilu_sweep_h_[p]] = (int32_t)p;
      posb[ilu_sweep_h_[nc + p]] = (int32_t)p;
    }
    ilu_rec_h_.assign(16 * nc, -1);
    for (int dir = 0; dir < 2; ++dir)
      for (int64_t p = 0; p < nc; ++p) {
        const int32_t c = ilu_sweep_h_[dir * nc + p];
        int32_t* rec = ilu_rec_h_.data() + 8 * (dir * nc + p);
        rec[0] = c;
        int nd = 0;
        uint32_t slots = 0xffffffffu;
        for (int k = 0; k < 4; ++k) {
          const int32_t o = nbr(c, k);
          if (o < 0) continue;
          const bool dep = dir == 0 ? ilu_pos_h_[o] < ilu_pos_h_[c] : ilu_pos_h_[o] > ilu_pos_h_[c];
          if (!dep) continue;
          rec[1 + nd] = dir == 0 ? posf[o] : posb[o];
          slots = (slots & ~(0xffu << (8 * nd))) | ((uint32_t)k << (8 * nd));
          ++nd;
        }
        rec[5] = (int32_t)slots;
        rec[6] = posf[c];
        rec[7] = 0;
      }
  }
  ilu_order_h_ = std::move(order);
  ilu_.nc = nc;
  ilu_.n_lo = nlo;
  ilu_.n_up = nup;
  ilu_.spin_limit = kSweepSpinLimit;
  ilu_.stall_row = -1;
}

void Solver::ilu_factor() {
  NvtxRange nvtx_("o2f ilu_factor");
  const int64_t nc = topo_.nc;
  cudaStream_t s = stream_;
  if (!ilu_alloc_) {
    ilu_.nbr = arena_.alloc<int32_t>(4 * nc);
    ilu_.pos = arena_.alloc<int32_t>(nc);
    ilu_.A = arena_.alloc<double>(80 * nc);
    ilu_.Dinv = arena_.alloc<double>(16 * nc);
    ilu_.order = arena_.alloc<int32_t>(nc);
    ilu_.sweep = arena_.alloc<int32_t>(2 * nc);
    ilu_.lev_off = arena_.alloc<int32_t>(ilu_lev_off_h_.size());
    ilu_.rec = arena_.alloc<int32_t>(16 * nc);
    ilu_.out_f = arena_.alloc<Vec4<double>>(nc);
    ilu_.out_b = arena_.alloc<Vec4<double>>(nc);
    ilu_.pack = arena_.alloc<double>((nc + 31) / 32 * 32 * 144);
    ilu_.lo_cells = arena_.alloc<int32_t>(nc);
    ilu_.tmp = arena_.alloc<Vec4<double>>(nc);
    ilu_.sync = arena_.alloc<SweepSync>(2);
    ilu_status_ = arena_.alloc<int>(1);
    phat_ = arena_.alloc<Vec4<double>>(nc);
    shat_ = arena_.alloc<Vec4<double>>(nc);
    h2d(ilu_.nbr, ilu_nbr_h_, s);
    h2d(ilu_.pos, ilu_pos_h_, s);
    h2d(ilu_.order, ilu_order_h_, s);
    h2d(ilu_.sweep, ilu_sweep_h_, s);
    h2d(ilu_.lev_off, ilu_lev_off_h_, s);
    h2d(ilu_.rec, ilu_rec_h_, s);
    O2F_CUDA(cudaFuncSetAttribute(k_ilu_sweep_cta<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSweepSmem));
    O2F_CUDA(cudaFuncSetAttribute(k_ilu_sweep_cta<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kSweepSmem));
    h2d(ilu_.lo_cells, lo_cells_h_, s);
    k_ilu_empty<<<grid(nc), kBlock, 0, s>>>(nc, ilu_.tmp);
    O2F_CUDA(cudaMemsetAsync(ilu_.sync, 0, 2 * sizeof(SweepSync), s));
    sync();
    ilu_alloc_ = true;
  }
  O2F_CUDA(cudaMemsetAsync(ilu_status_, 0, sizeof(int), s));
  if (full_jac())  // ILU(0) of the full operator on the first-order pattern
    k_ilu_assemble_full<<<grid(nc), kBlock, 0, s>>>(nc, fjac_off_, fjac_idx_, fjac_blk_, params_.adjoint_shift, ilu_);
  else
    k_ilu_assemble<<<grid(nc), kBlock, 0, s>>>(nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk_,
                                               params_.adjoint_shift, ilu_);
  for (int l = 0; l < ilu_.n_lo; ++l) {
    const int n = lo_off_h_[l + 1] - lo_off_h_[l];
    k_ilu_factor<<<(n + 127) / 128, 128, 0, s>>>(ilu_.lo_cells + lo_off_h_[l], n, ilu_, ilu_status_);
  }
  // the factor blocks in the block sweeps' order
  k_ilu_pack<<<(int)((2 * nc * 5 + 255) / 256), 256, 0, s>>>((int)nc, ilu_);
  O2F_CUDA(cudaGetLastError());
  launches_ += 2 + ilu_.n_lo;
  int st = 0;
  O2F_CUDA(cudaMemcpyAsync(&st, ilu_status_, sizeof(int), cudaMemcpyDeviceToHost, s));
  sync();
  if (st) throw Error(O2F_ERR_BREAKDOWN, "singular block in the ILU(0) factorization");
}

// O2F_SWEEPS_AUTO: triangles up to this many rows are swept by one thread
// block (measured on B200 per adjoint iteration alone, block / waiting:
// 3.9 / 5.2 ms at 75k rows, 6.9 / 8.1 at 151k, 13.1 / 11.8 at 301k; side by
// side with other contexts' solves the block sweep is ahead at every size).
constexpr int64_t kIluCtaMaxRows = 200000;

// z = M^{-1} r = U^{-1} L^{-1} r: the forward sweep into ilu_.tmp, the
// backward sweep into z; one launch per triangle, either one block walking
// the levels or persistent warps that wait on their rows' dependencies.
void Solver::ilu_apply(const Vec4<double>* r, Vec4<double>* z, const int* gate) {
  cudaStream_t s = stream_;
  const int n = (int)ilu_.nc;
  const int mode = params_.adjoint_sweeps;
  const bool block = mode == O2F_SWEEPS_BLOCK || (mode == O2F_SWEEPS_AUTO && n <= kIluCtaMaxRows);
  if (!ilu_waiting_ && block) {  // one block per triangle, level by level
    k_ilu_sweep_cta<true><<<1, kSweepCtaThreads, kSweepSmem, s>>>(n, ilu_, r, z, gate);
    k_ilu_sweep_cta<false><<<1, kSweepCtaThreads, kSweepSmem, s>>>(n, ilu_, nullptr, z, gate);
    return;
  }
  const int blocks = ilu_sweep_blocks(n);
  k_ilu_sweep<true><<<blocks, kSweepBlock, 0, s>>>(n, ilu_, r, z, gate);  // r -> ilu_.tmp
  k_ilu_sweep<false><<<blocks, kSweepBlock, 0, s>>>(n, ilu_, nullptr, z, gate);  // ilu_.tmp -> z
}

// Test hook: the next solves run the waiting sweeps (k_ilu_sweep) with
// `spin_limit` polls per wait, and with `stall` the first row of the forward order never writes its
// value, so the rows that depend on it wait out their limit (no fault:
// every wait is bounded).  spin_limit <= 0 and stall = 0 restore the
// defaults.  Takes effect for the solves that start after the call.
void Solver::debug_ilu_stall(int stall, long long spin_limit) {
  ilu_.spin_limit = spin_limit > 0 ? spin_limit : kSweepSpinLimit;
  ilu_.stall_row = stall && !ilu_sweep_h_.empty() ? ilu_sweep_h_[0] : -1;
  ilu_waiting_ = stall != 0 || spin_limit > 0;  // the hook needs the sweeps that wait
}

// A sweep whose dependency wait ran out leaves an invalid result: report it
// (and clear the flag so the context stays usable).
void Solver::ilu_check_sweeps() {
  SweepSync h[2];
  O2F_CUDA(cudaMemcpyAsync(h, ilu_.sync, sizeof(h), cudaMemcpyDeviceToHost, stream_));
  sync();
  if (h[0].err || h[1].err) {
    const int zero[2] = {0, 0};
    O2F_CUDA(cudaMemcpyAsync(&ilu_.sync[0].err, &zero[0], sizeof(int), cudaMemcpyHostToDevice, stream_));
    O2F_CUDA(cudaMemcpyAsync(&ilu_.sync[1].err, &zero[1], sizeof(int), cudaMemcpyHostToDevice, stream_));
    sync();
    throw Error(O2F_ERR_CUDA, "ILU triangular sweep: dependency wait exceeded its limit");
  }
}

Work<double> Solver::alloc_work() {
  Work<double> w{};
  w.vq = arena_.alloc<Vec4<double>>(topo_.nv);
  w.eL = arena_.alloc<Vec4<double>>(topo_.ne);
  w.eR = arena_.alloc<Vec4<double>>(topo_.ne);
  w.ctq = arena_.alloc<Vec4<double>>(topo_.nc);
  w.ctqy = arena_.alloc<double>(topo_.nc);
  w.vtq = arena_.alloc<Vec4<double>>(topo_.nv);
  w.vtqy = arena_.alloc<double>(topo_.nv);
  w.F = arena_.alloc<Vec4<double>>(topo_.ne);
  w.etq = arena_.alloc<Vec4<double>>(topo_.ne);
  w.etqy = arena_.alloc<double>(topo_.ne);
  w.grad = arena_.alloc<Vec4<double>>(2 * topo_.nc);
  w.R = arena_.alloc<Vec4<double>>(topo_.nc);
  return w;
}

o2f_mesh_info Solver::info() const {
  o2f_mesh_info i{};
  i.n_cells = hm_.nc;
  i.n_edges = hm_.ne;
  i.n_vertices = hm_.nv;
  i.n_wall_edges = topo_.n_wall;
  int64_t nb = 0;
  for (int64_t e = 0; e < hm_.ne; ++e) nb += hm_.e_cr[e] < 0;
  i.n_boundary_edges = nb;
  i.max_vertex_valence = hm_.max_valence;
  i.min_h = min_h_;
  i.device_bytes = arena_.bytes();
  return i;
}

int64_t Solver::export_array(const std::string& w, void* out) const { return export_mesh_array(hm_, w, out); }

void Solver::to_internal(const double* ref, Vec4<double>* dev) {
  const int64_t nc = hm_.nc;
  std::vector<Vec4<double>> tmp(nc);
  for (int64_t c = 0; c < nc; ++c) {
    const double* q = ref + 4 * cperm_[c];
    tmp[c] = Vec4<double>{q[0], q[1], q[2], q[3]};
  }
  O2F_CUDA(cudaMemcpyAsync(dev, tmp.data(), nc * sizeof(Vec4<double>), cudaMemcpyHostToDevice, stream_));
  sync();
}

void Solver::to_reference(const Vec4<double>* dev, double* ref) {
  const int64_t nc = hm_.nc;
  std::vector<Vec4<double>> tmp(nc);
  O2F_CUDA(cudaMemcpyAsync(tmp.data(), dev, nc * sizeof(Vec4<double>), cudaMemcpyDeviceToHost, stream_));
  sync();
  for (int64_t c = 0; c < nc; ++c) {
    double* q = ref + 4 * cperm_[c];
    q[0] = tmp[c].a;
    q[1] = tmp[c].b;
    q[2] = tmp[c].c;
    q[3] = tmp[c].d;
  }
}

void Solver::state_set(const double* U_ref) {
  to_internal(U_ref, U_);
  have_residual_ = false;
  invalidate_linearisation();
}

void Solver::state_get(double* U_ref) { to_reference(U_, U_ref); }

void Solver::state_freestream() {
  // init_one_x (src/init.cpp:57-81) == the freestream boundary state.
  k_fill_state<double><<<grid(topo_.nc), kBlock, 0, stream_>>>(
      topo_.nc, Vec4<double>{phys_.fs_rho, phys_.fs_rhou, phys_.fs_rhov, phys_.fs_E}, U_);
  O2F_CUDA(cudaGetLastError());
  have_residual_ = false;
  invalidate_linearisation();
}

void Solver::cell_permutation(int64_t* new_of_old) const {
  std::memcpy(new_of_old, cinv_.data(), cinv_.size() * sizeof(int64_t));
}

void Solver::launch_residual(const Geom<double>& g, const Work<double>& w, Vec4<double>* U, const int* gate,
                             bool write_grad, const void* rkp, int alpha_mode) {
  const Topo& t = topo_;
  cudaStream_t s = stream_;
  k_vertex_state<double><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, U, phys_, w.vq, gate);
  if (alpha_mode == 1)
    k_cell_gradient_alpha<1><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U, w.vq, phys_, w.eL,
                                                            w.eR, w.ctq, w.ctqy, fjac_alpha_);
  else if (alpha_mode == 2)
    k_cell_gradient_alpha<2><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U, w.vq, phys_, w.eL,
                                                            w.eR, w.ctq, w.ctqy, fjac_alpha_);
  else if (write_grad)
    k_cell_gradient<double, true><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U, w.vq, phys_,
                                                                w.eL, w.eR, w.ctq, w.ctqy, w.grad, gate);
  else
    k_cell_gradient<double, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U, w.vq, phys_,
                                                                 w.eL, w.eR, w.ctq, w.ctqy, w.grad, gate);
  k_vertex_visc<double><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, w.ctq, w.ctqy, w.vtq,
                                                      w.vtqy, gate);
  k_edge_flux<double><<<grid(t.ne), kBlock, 0, s>>>(t.ne, g, t.ev, t.ebc, w.eL, w.eR, w.vtq, w.vtqy, phys_, w.F,
                                                    w.etq, w.etqy, gate);
  if (rkp) {
    const RkStage rk = *static_cast<const RkStage*>(rkp);
    k_cell_residual<double, true><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U, Uold_, w.R,
                                                                rk, gate);
  } else {
    k_cell_residual<double, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U, Uold_,
                                                                 w.R, RkStage{}, gate);
  }
  launches_ += 5;
  O2F_CUDA(cudaGetLastError());
}

void Solver::residual(double* R_ref) {
  NvtxRange nvtx_("o2f residual");
  if (f32()) {
    ensure_f32();
    f32_state_sync();
  }
  O2F_CUDA(cudaEventRecord(ev0_, stream_));
  if (f32())
    launch_residual_f32(nullptr, nullptr);
  else
    launch_residual(geom_, work_, U_, nullptr, true, nullptr);
  O2F_CUDA(cudaEventRecord(ev1_, stream_));
  if (f32()) f32_publish_interfaces();
  sync();
  float ms = 0.f;
  O2F_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
  last_residual_ms_ = ms;
  have_residual_ = true;
  invalidate_linearisation();
  if (R_ref) to_reference(work_.R, R_ref);
}

void Solver::profile_kernels(int reps, double* ms_out) {
  NvtxRange nvtx_("o2f profile_kernels");
  if (reps <= 0) throw Error(O2F_ERR_ARG, "reps must be positive");
  const Topo& t = topo_;
  const Geom<double>& g = geom_;
  const Work<double>& w = work_;
  cudaStream_t s = stream_;
  launch_residual(geom_, work_, U_, nullptr, false, nullptr);  // fresh interface states
  have_residual_ = true;
  invalidate_linearisation();
  build_jt_blocks();
  if (!tmp_) tmp_ = arena_.alloc<Vec4<double>>(topo_.nc);
  if (!s_) s_ = arena_.alloc<Vec4<double>>(topo_.nc);
  O2F_CUDA(cudaMemsetAsync(s_, 0, topo_.nc * sizeof(Vec4<double>), s));
  if (f32()) {  // the residual kernels of this context's precision
    ensure_f32();
    f32_state_sync();
    launch_residual_f32(nullptr, nullptr);
  }
  for (int k = 0; k < O2F_K_COUNT; ++k) {
    O2F_CUDA(cudaEventRecord(ev0_, s));
    for (int r = 0; r < reps; ++r) {
      if (f32() && k <= O2F_K_CELL_RESIDUAL) {
        profile_kernel_f32(k);
        continue;
      }
      switch (k) {
        case O2F_K_VERTEX_STATE:
          k_vertex_state<double><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, U_, phys_, w.vq,
                                                               nullptr);
          break;
        case O2F_K_CELL_GRADIENT:
          k_cell_gradient<double, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, t.ev, t.ec, t.ebc, U_, w.vq,
                                                                       phys_, w.eL, w.eR, w.ctq, w.ctqy, w.grad,
                                                                       nullptr);
          break;
        case O2F_K_VERTEX_VISC:
          k_vertex_visc<double><<<grid(t.nv), kBlock, 0, s>>>(t.nv, t.voff, t.vcid, g.vw, t.vbc, w.ctq, w.ctqy, w.vtq,
                                                              w.vtqy, nullptr);
          break;
        case O2F_K_EDGE_FLUX:
          k_edge_flux<double><<<grid(t.ne), kBlock, 0, s>>>(t.ne, g, t.ev, t.ebc, w.eL, w.eR, w.vtq, w.vtqy, phys_,
                                                            w.F, w.etq, w.etqy, nullptr);
          break;
        case O2F_K_CELL_RESIDUAL:
          k_cell_residual<double, false><<<grid(t.nc), kBlock, 0, s>>>(t.nc, t.slot, g, w.F, w.etq, w.etqy, U_,
                                                                       Uold_, w.R, RkStage{}, nullptr);
          break;
        case O2F_K_JT_APPLY:
          jt_apply_dev(s_, tmp_);
          break;
        case O2F_K_JT_BLOCKS:
          k_jt_blocks<<<(int)((t.ne + 127) / 128), 128, 0, s>>>(t.ne, g, t.ebc, w.eL, w.eR, phys_, 1e-6, blk_);
          break;
      }
    }
    O2F_CUDA(cudaEventRecord(ev1_, s));
    O2F_CUDA(cudaGetLastError());
    sync();
    float ms = 0.f;
    O2F_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    ms_out[k] = (double)ms / reps;
  }
  launches_ += (int64_t)reps * O2F_K_COUNT;
}

void Solver::debug_get(const std::string& which, double* out) {
  if (!have_residual_) throw Error(O2F_ERR_STATE, "no residual has been evaluated");
  const int64_t nc = hm_.nc, ne = hm_.ne, nv = hm_.nv;
  if (which == "R") {
    to_reference(work_.R, out);
  } else if (which == "grad") {
    std::vector<Vec4<double>> g(2 * nc);
    O2F_CUDA(cudaMemcpy(g.data(), work_.grad, g.size() * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    for (int64_t c = 0; c < nc; ++c) {
      double* q = out + 8 * cperm_[c];
      const Vec4<double>&x = g[2 * c], &y = g[2 * c + 1];
      const double vals[8] = {x.a, x.b, x.c, x.d, y.a, y.b, y.c, y.d};
      std::memcpy(q, vals, sizeof(vals));
    }
  } else if (which == "edge_LR" || which == "edge_tau" || which == "edge_F") {
    std::vector<Vec4<double>> L(ne), R(ne);
    if (which == "edge_LR") {
      O2F_CUDA(cudaMemcpy(L.data(), work_.eL, ne * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
      O2F_CUDA(cudaMemcpy(R.data(), work_.eR, ne * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    } else if (which == "edge_F") {
      O2F_CUDA(cudaMemcpy(L.data(), work_.F, ne * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    } else {
      O2F_CUDA(cudaMemcpy(L.data(), work_.etq, ne * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    }
    for (int64_t e = 0; e < ne; ++e) {
      const int64_t eo = eperm_[e];
      if (which == "edge_LR") {
        const double vals[8] = {L[e].a, L[e].b, L[e].c, L[e].d, R[e].a, R[e].b, R[e].c, R[e].d};
        std::memcpy(out + 8 * eo, vals, sizeof(vals));
      } else if (which == "edge_F") {
        const double vals[4] = {L[e].a, L[e].b, L[e].c, L[e].d};
        std::memcpy(out + 4 * eo, vals, sizeof(vals));
      } else {
        // The reference stores tau only on wall edges (src/diffusion.cpp:158-162).
        const bool wall = hm_.ebc[eo] == 'w';
        const double vals[3] = {wall ? L[e].a : 0.0, wall ? L[e].c : 0.0, wall ? L[e].b : 0.0};
        std::memcpy(out + 3 * eo, vals, sizeof(vals));
      }
    }
  } else if (which == "vertex_U") {
    std::vector<Vec4<double>> q(nv);
    O2F_CUDA(cudaMemcpy(q.data(), work_.vq, nv * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    for (int64_t v = 0; v < nv; ++v) {
      double* o = out + 4 * vperm_[v];
      o[0] = q[v].a;
      o[1] = q[v].b;
      o[2] = q[v].c;
      o[3] = q[v].d;
    }
  } else {
    throw Error(O2F_ERR_ARG, "unknown debug array '" + which + "'");
  }
}

void Solver::rk3_run(int64_t max_steps, double drop_tol, double* history, int64_t* steps_done, double* t_out) {
  NvtxRange nvtx_("o2f rk3_run");
  if (max_steps < 0) throw Error(O2F_ERR_ARG, "max_steps < 0");
  if (hist_cap_ < std::max<int64_t>(max_steps, 1)) {
    hist_cap_ = std::max<int64_t>(max_steps, 1);
    hist_dev_ = arena_.alloc<double>(hist_cap_);
  }
  StepState st{};
  st.t = 0.0;
  st.final_time = params_.final_time;
  st.cfl = params_.cfl_number;
  st.min_h = min_h_;
  st.mu = params_.viscosity;
  if (params_.dt_mode == O2F_DT_THERMAL)
    st.mu = std::max(params_.viscosity, params_.viscosity * params_.cp / params_.Pr * (params_.gamma - 1.0));
  st.drop_tol = drop_tol;
  st.max_steps = max_steps;
  O2F_CUDA(cudaMemcpyAsync(step_, &st, sizeof(st), cudaMemcpyHostToDevice, stream_));
  const int* gate = &step_->stop;
  const double* dt = &step_->dt;
  const RkStage s1{0.0, 1.0, dt, 1, norm_part_};
  const RkStage s2{3.0 / 4.0, 1.0 / 4.0, dt, 0, nullptr};
  const RkStage s3{1.0 / 3.0, 2.0 / 3.0, dt, 0, nullptr};
  const int nparts = grid(topo_.nc);
  const int wave_grid = std::min(grid(topo_.nc), 148 * 8);
  // One CUDA graph holds kStepsPerGraph steps; steps past a stop condition
  // are no-ops (every kernel checks the gate).
  const int kStepsPerGraph = topo_.nc < 200000 ? 16 : 4;
  // FP64 path: the reference arithmetic.  Mixed path: FP32 residual, FP64
  // state update (solver_f32.cu).
  const bool mixed = f32();
  if (mixed) {
    ensure_f32();
    f32_state_sync();
  }
  auto stage = [&](const RkStage* rk) {
    if (mixed)
      launch_residual_f32(gate, rk, rk == &s3 ? Ukeep_ : nullptr);
    else
      launch_residual(geom_, work_, U_, gate, false, rk);
  };
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  O2F_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < kStepsPerGraph; ++i) {
    k_step_begin<<<1, 1, 0, stream_>>>(step_);
    k_wave_speed<double><<<wave_grid, kBlock, 0, stream_>>>(topo_.nc, U_, params_.gamma, step_);
    k_step_dt<<<1, 1, 0, stream_>>>(step_);
    stage(&s1);
    k_step_norm<<<1, 1024, 0, stream_>>>(norm_part_, nparts, hist_dev_, step_);
    stage(&s2);
    stage(&s3);
    k_step_end<<<1, 1, 0, stream_>>>(step_);
  }
  O2F_CUDA(cudaStreamEndCapture(stream_, &graph));
  O2F_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  StepState* host_st = static_cast<StepState*>(mailbox_);
  int64_t launched = 0;
  try {
    while (true) {
      O2F_CUDA(cudaGraphLaunch(exec, stream_));
      launched += kStepsPerGraph;
      launches_ += kStepsPerGraph * 20;
      if (launched % (kStepsPerGraph * 4) == 0 || launched >= max_steps) {
        O2F_CUDA(cudaMemcpyAsync(host_st, step_, sizeof(StepState), cudaMemcpyDeviceToHost, stream_));
        sync();
        if (host_st->stop) break;
      }
    }
  } catch (...) {
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    throw;
  }
  const StepState fin = *host_st;
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (history && fin.step > 0)
    O2F_CUDA(cudaMemcpy(history, hist_dev_, std::min<int64_t>(fin.step, max_steps) * sizeof(double),
                        cudaMemcpyDeviceToHost));
  if (steps_done) *steps_done = fin.step;
  if (t_out) *t_out = fin.t;
  // Mixed path: the forces, J, the Jacobian blocks and the adjoint
  // right-hand side linearise about the last stage's input state, as in the
  // FP64 path; one FP64 residual of that state gives its interface states.
  if (mixed && fin.step > 0) {
    launch_residual(geom_, work_, Ukeep_, nullptr, false, nullptr);
    sync();
  }
  have_residual_ = fin.step > 0;
  invalidate_linearisation();
  if (fin.stop == 2) throw Error(O2F_ERR_NONFINITE, "non-finite state or residual in the time loop");
}

void Solver::forces(double beta, double* out3) {
  if (!have_residual_) throw Error(O2F_ERR_STATE, "no residual has been evaluated");
  k_forces<double><<<1, kBlock, 0, stream_>>>(topo_.n_wall, topo_.wall_edges, geom_, work_.eL, work_.etq, phys_,
                                              beta, scal_);
  O2F_CUDA(cudaGetLastError());
  O2F_CUDA(cudaMemcpyAsync(out3, scal_, 3 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
}

void Solver::build_jt_blocks() {
  NvtxRange nvtx_("o2f jt_blocks");
  if (blk_valid_) return;
  if (!have_residual_) throw Error(O2F_ERR_STATE, "no residual has been evaluated");
  if (!blk_) blk_ = arena_.alloc<double>(32 * topo_.ne);
  k_jt_blocks<<<(int)((topo_.ne + 127) / 128), 128, 0, stream_>>>(topo_.ne, geom_, topo_.ebc, work_.eL, work_.eR,
                                                                   phys_, 1e-6, blk_);
  O2F_CUDA(cudaGetLastError());
  if (mixed_adjoint()) f32_blocks();
  blk_valid_ = true;
}

void Solver::jt_apply_dev(const Vec4<double>* x, Vec4<double>* y) {
  if (full_jac())
    k_fjt_apply<<<grid(topo_.nc), kBlock, 0, stream_>>>(topo_.nc, fjac_off_, fjac_idx_, fjac_blk_, x, y);
  else
    k_jt_apply<<<grid(topo_.nc), kBlock, 0, stream_>>>(topo_.nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk_, x, y);
  O2F_CUDA(cudaGetLastError());
}

// Stencils (two vertex rings), their colouring, and the wall edges each cell
// reaches; host work, once per mesh topology.
void Solver::setup_full_jacobian() {
  NvtxRange nvtx_("o2f full_jacobian_setup");
  if (fjac_setup_) return;
  const HostMesh& m = hm_;
  const int64_t nc = m.nc;
  Stencil stc = jacobian_stencil(m, cperm_, cinv_);
  const std::vector<int64_t>& soff = stc.off;
  const std::vector<int32_t>& sidx = stc.idx;
  const std::vector<int32_t>& color = stc.color;
  const int32_t ncol = stc.ncolor;
  fjac_coff_h_.assign(ncol + 1, 0);
  for (int64_t j = 0; j < nc; ++j) ++fjac_coff_h_[color[j] + 1];
  for (int32_t c = 0; c < ncol; ++c) fjac_coff_h_[c + 1] += fjac_coff_h_[c];
  std::vector<int32_t> ccells(nc);
  std::vector<int64_t> fill(fjac_coff_h_.begin(), fjac_coff_h_.end() - 1);
  for (int64_t j = 0; j < nc; ++j) ccells[fill[color[j]]++] = (int32_t)j;
  // wall edges (objective terms) reaching each cell: those of its stencil's owners
  std::vector<int64_t> wcount(nc + 1, 0);
  const int64_t nw = (int64_t)wall_edges_host_.size();
  std::vector<int32_t> wcell(nw);
  for (int64_t w = 0; w < nw; ++w) {
    const int64_t eo = eperm_[wall_edges_host_[w]];
    wcell[w] = (int32_t)cinv_[m.e_cl[eo]];
    for (int64_t a = soff[wcell[w]]; a < soff[wcell[w] + 1]; ++a) ++wcount[sidx[a] + 1];
  }
  for (int64_t j = 0; j < nc; ++j) wcount[j + 1] += wcount[j];
  std::vector<int32_t> widx(wcount[nc]);
  std::vector<int64_t> wfill(wcount.begin(), wcount.end() - 1);
  for (int64_t w = 0; w < nw; ++w)
    for (int64_t a = soff[wcell[w]]; a < soff[wcell[w] + 1]; ++a) widx[wfill[sidx[a]]++] = (int32_t)w;
  fjac_nnzb_ = soff[nc];
  cudaStream_t st = stream_;
  fjac_off_ = arena_.alloc<int64_t>(nc + 1);
  fjac_idx_ = arena_.alloc<int32_t>(sidx.size());
  fjac_ccells_ = arena_.alloc<int32_t>(nc);
  fjac_woff_ = arena_.alloc<int64_t>(nc + 1);
  fjac_widx_ = arena_.alloc<int32_t>(std::max<size_t>(widx.size(), 1));
  h2d(fjac_off_, soff, st);
  h2d(fjac_idx_, sidx, st);
  h2d(fjac_ccells_, ccells, st);
  h2d(fjac_woff_, wcount, st);
  if (!widx.empty()) h2d(fjac_widx_, widx, st);
  fjac_blk_ = arena_.alloc<double>(16 * fjac_nnzb_);
  fjac_gL_ = arena_.alloc<double>(4 * nc);
  fjac_gD_ = arena_.alloc<double>(4 * nc);
  fjac_tlp_ = arena_.alloc<double>(std::max<int64_t>(nw, 1));
  fjac_tdp_ = arena_.alloc<double>(std::max<int64_t>(nw, 1));
  fjac_tlm_ = arena_.alloc<double>(std::max<int64_t>(nw, 1));
  fjac_tdm_ = arena_.alloc<double>(std::max<int64_t>(nw, 1));
  fjac_Up_ = arena_.alloc<Vec4<double>>(nc);
  fjac_Rp_ = arena_.alloc<Vec4<double>>(nc);
  fjac_alpha_ = arena_.alloc<Vec4<double>>(nc);
  sync();
  fjac_setup_ = true;
}

// The full Jacobian and dC_L/dU, dC_D/dU about the current state: for every
// colour and component, two residuals (state +- eps on the colour's cells),
// then the columns of the blocks and the objective gradient.  Leaves the
// residual and interface states of the current state in the context.
void Solver::build_full_jacobian() {
  NvtxRange nvtx_("o2f full_jacobian");
  if (fjac_valid_) return;
  setup_full_jacobian();
  const int64_t nc = topo_.nc, nw = topo_.n_wall;
  cudaStream_t st = stream_;
  const Phys& ph = phys_;
  const double a_inf = std::sqrt(ph.gamma * params_.p_ref / params_.rho_ref);
  // Steps of 1e-9 relative: the reference's Venkatakrishnan eps = (K h)^3 is
  // absolute, so for E and rho*u (1e5 and 1e2 in SI units) the limiter turns
  // over within ~1e-4 absolute on fine cells; larger steps difference across
  // that turn (1e-6: 2e-2 off the directional derivative, 1e-8: 7e-4,
  // 1e-10: 2e-5 with roundoff reaching 1e-5 in dJ/dU).
  FjacEps e{};
  e.h = params_.adjoint_fd_step;
  e.floor[0] = 1e-2 * ph.fs_rho;
  e.floor[1] = 1e-2 * ph.fs_rho * a_inf;
  e.floor[2] = 1e-2 * ph.fs_rho * a_inf;
  e.floor[3] = 1e-2 * ph.fs_E;
  O2F_CUDA(cudaMemsetAsync(fjac_gL_, 0, 4 * nc * sizeof(double), st));
  O2F_CUDA(cudaMemsetAsync(fjac_gD_, 0, 4 * nc * sizeof(double), st));
  O2F_CUDA(cudaMemcpyAsync(fjac_Up_, U_, nc * sizeof(Vec4<double>), cudaMemcpyDeviceToDevice, st));
  // frozen limiter: the limiter values of the current state, held in every
  // perturbed residual
  const int amode = params_.adjoint_jacobian == O2F_JAC_FROZEN ? 2 : 0;
  if (amode) launch_residual(geom_, work_, U_, nullptr, false, nullptr, 1);
  const int64_t ncol = (int64_t)fjac_coff_h_.size() - 1;
  for (int64_t col = 0; col < ncol; ++col) {
    const int32_t* cells = fjac_ccells_ + fjac_coff_h_[col];
    const int64_t n = fjac_coff_h_[col + 1] - fjac_coff_h_[col];
    for (int k = 0; k < 4; ++k) {
      k_fjac_perturb<<<grid(n), kBlock, 0, st>>>(n, cells, U_, fjac_Up_, k, 1.0, e);
      launch_residual(geom_, work_, fjac_Up_, nullptr, false, nullptr, amode);
      O2F_CUDA(cudaMemcpyAsync(fjac_Rp_, work_.R, nc * sizeof(Vec4<double>), cudaMemcpyDeviceToDevice, st));
      if (nw) k_fjac_wall_terms<<<grid(nw), kBlock, 0, st>>>(nw, topo_.wall_edges, geom_, work_.eL, work_.etq, ph,
                                                              fjac_tlp_, fjac_tdp_);
      k_fjac_perturb<<<grid(n), kBlock, 0, st>>>(n, cells, U_, fjac_Up_, k, -1.0, e);
      launch_residual(geom_, work_, fjac_Up_, nullptr, false, nullptr, amode);
      if (nw) k_fjac_wall_terms<<<grid(nw), kBlock, 0, st>>>(nw, topo_.wall_edges, geom_, work_.eL, work_.etq, ph,
                                                              fjac_tlm_, fjac_tdm_);
      k_fjac_extract<<<grid(n), kBlock, 0, st>>>(n, cells, fjac_off_, fjac_idx_, U_, fjac_Rp_, work_.R, k, e,
                                                  fjac_blk_);
      if (nw)
        k_fjac_grad_extract<<<grid(n), kBlock, 0, st>>>(n, cells, fjac_woff_, fjac_widx_, U_, fjac_tlp_, fjac_tdp_,
                                                         fjac_tlm_, fjac_tdm_, k, e, fjac_gL_, fjac_gD_);
      k_fjac_restore<<<grid(n), kBlock, 0, st>>>(n, cells, U_, fjac_Up_);
      O2F_CUDA(cudaGetLastError());
      launches_ += 7;
    }
  }
  // the residual and interface states of the state itself
  launch_residual(geom_, work_, U_, nullptr, false, nullptr);
  O2F_CUDA(cudaGetLastError());
  sync();
  have_residual_ = true;
  blk_valid_ = false;  // the first-order blocks follow the interface states just computed
  fjac_valid_ = true;
}

void Solver::jt_apply(const double* x_ref, double* y_ref) {
  if (full_jac()) build_full_jacobian();
  build_jt_blocks();
  if (!tmp_) tmp_ = arena_.alloc<Vec4<double>>(topo_.nc);
  if (!s_) s_ = arena_.alloc<Vec4<double>>(topo_.nc);
  to_internal(x_ref, s_);
  if (f32() && !full_jac()) {
    k_jt_apply<<<grid(topo_.nc), kBlock, 0, stream_>>>(topo_.nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk32_, s_,
                                                       tmp_);
    O2F_CUDA(cudaGetLastError());
  } else {
    jt_apply_dev(s_, tmp_);
  }
  to_reference(tmp_, y_ref);
}

void Solver::adjoint_rhs(double beta, double* b_ref) {
  if (!have_residual_) throw Error(O2F_ERR_STATE, "no residual has been evaluated");
  if (!b_) b_ = arena_.alloc<Vec4<double>>(topo_.nc);
  if (full_jac()) {  // dJ/dU of the whole objective
    build_full_jacobian();
    k_fjac_rhs<<<grid(4 * topo_.nc), kBlock, 0, stream_>>>(4 * topo_.nc, fjac_gL_, fjac_gD_, beta,
                                                           reinterpret_cast<double*>(b_));
    O2F_CUDA(cudaGetLastError());
    if (b_ref) to_reference(b_, b_ref);
    return;
  }
  O2F_CUDA(cudaMemsetAsync(b_, 0, topo_.nc * sizeof(Vec4<double>), stream_));
  if (topo_.n_wall_cells > 0)
    k_adjoint_rhs<<<grid(topo_.n_wall_cells), kBlock, 0, stream_>>>(topo_.n_wall_cells, topo_.wall_cells,
                                                                     topo_.wall_cell_off, topo_.wall_cell_edges,
                                                                     geom_, work_.eL, phys_, beta, b_);
  O2F_CUDA(cudaGetLastError());
  if (b_ref) to_reference(b_, b_ref);
}

void Solver::adjoint_solve(double beta, double tol, int64_t max_iter, int64_t restart, double* lambda_ref,
                           int64_t* iters, double* relres_out, const double* guess_ref, const double* rhs_ref) {
  NvtxRange nvtx_("o2f adjoint_solve");
  if (!(tol > 0.0) || max_iter <= 0 || restart <= 0) throw Error(O2F_ERR_ARG, "invalid solver settings");
  const bool full = full_jac();
  if (full) build_full_jacobian();  // first: it recomputes the interface states
  build_jt_blocks();                // (the preconditioner's blocks in the full mode)
  if (rhs_ref) {  // a given right-hand side instead of dJ/dU
    if (!b_) b_ = arena_.alloc<Vec4<double>>(topo_.nc);
    to_internal(rhs_ref, b_);
  } else {
    adjoint_rhs(beta, nullptr);
  }
  const int64_t nc = topo_.nc, n4 = 4 * nc;
  // Grid of the Krylov vector kernels: one cell per thread up to the fixed
  // reduction grid, so a small solve leaves the rest of the GPU to others.
  const int kgrid = (int)std::min<int64_t>(kRedGrid, std::max<int64_t>(1, (nc + kBlock - 1) / kBlock));
  auto need = [&](Vec4<double>*& p) {
    if (!p) p = arena_.alloc<Vec4<double>>(nc);
  };
  need(lam_);
  need(r_);
  need(r0_);
  need(p_);
  need(v_);
  need(s_);
  need(t_);
  need(tmp_);
  double* x = reinterpret_cast<double*>(lam_);
  if (guess_ref)  // warm start: the first chunk's residual is b - J^T lambda0
    to_internal(guess_ref, lam_);
  else
    O2F_CUDA(cudaMemsetAsync(lam_, 0, nc * sizeof(Vec4<double>), stream_));
  // ||b||^2
  k_dot2<<<kgrid, kBlock, 0, stream_>>>(n4, reinterpret_cast<double*>(b_), reinterpret_cast<double*>(b_), nullptr,
                                           nullptr, part_, ticket_, scal_);
  double bb[2];
  O2F_CUDA(cudaMemcpyAsync(bb, scal_, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  sync();
  const double bnorm = std::sqrt(bb[0]);
  KrylovState ks{};
  ks.tol2 = tol * tol * bb[0];
  int64_t total = 0;
  double relres = INFINITY;
  // Right-preconditioned BiCGSTAB: phat = M^{-1} p, shat = M^{-1} s; the
  // recurrence residual r stays the true residual of J^T lambda = b.
  bool precond = params_.adjoint_precond == O2F_PRECOND_ILU0;
  Vec4<double>* ph = p_;
  Vec4<double>* sh = s_;
  if (precond) {
    try {
      ilu_factor();
      ph = phat_;
      sh = shat_;
    } catch (const Error& e) {
      // A singular diagonal block (e.g. a cell whose pressure went negative):
      // this solve runs the reference's identity-preconditioned iteration.
      if (e.code != O2F_ERR_BREAKDOWN) throw;
      precond = false;
      if (params_.verbosity >= 1) std::fprintf(stderr, "[adjoint] ILU(0) breakdown: identity preconditioner\n");
    }
  }
  const int kItersPerGraph = precond ? 1 : 8;
  const int kernels_per_iter = 5 + (precond ? 4 : 0);
  const int* kgate = &ks_->stop;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  O2F_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
  for (int i = 0; i < kItersPerGraph; ++i) {
    k_bicg_p<<<kgrid, kBlock, 0, stream_>>>(n4, reinterpret_cast<double*>(r_), reinterpret_cast<double*>(r0_),
                                               reinterpret_cast<double*>(p_), reinterpret_cast<double*>(v_), ks_);
    if (precond) ilu_apply(p_, ph, kgate);
    if (full)
      k_bicg_fjt_v<<<kgrid, kBlock, 0, stream_>>>(nc, fjac_off_, fjac_idx_, fjac_blk_, ph, v_, r0_, part_, ks_);
    else if (mixed_adjoint())  // FP32 blocks; restarts take the true residual with the FP64 operator
      k_bicg_jt_v<<<kgrid, kBlock, 0, stream_>>>(nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk32_, ph, v_, r0_,
                                                    part_, ks_);
    else
      k_bicg_jt_v<<<kgrid, kBlock, 0, stream_>>>(nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk_, ph, v_, r0_,
                                                    part_, ks_);
    k_bicg_s<<<kgrid, kBlock, 0, stream_>>>(n4, reinterpret_cast<double*>(r_), reinterpret_cast<double*>(v_),
                                               reinterpret_cast<double*>(s_), ks_);
    if (precond) ilu_apply(s_, sh, kgate);
    if (full)
      k_bicg_fjt_t<<<kgrid, kBlock, 0, stream_>>>(nc, fjac_off_, fjac_idx_, fjac_blk_, sh, s_, t_, part_, ks_);
    else if (mixed_adjoint())
      k_bicg_jt_t<<<kgrid, kBlock, 0, stream_>>>(nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk32_, sh, s_, t_,
                                                    part_, ks_);
    else
      k_bicg_jt_t<<<kgrid, kBlock, 0, stream_>>>(nc, topo_.jslot, geom_, topo_.ec, topo_.ebc, blk_, sh, s_, t_,
                                                    part_, ks_);
    k_bicg_xr<<<kgrid, kBlock, 0, stream_>>>(n4, x, reinterpret_cast<double*>(ph), reinterpret_cast<double*>(sh),
                                                reinterpret_cast<double*>(s_), reinterpret_cast<double*>(t_),
                                                reinterpret_cast<double*>(r_), reinterpret_cast<double*>(r0_), part_,
                                                ks_);
  }
  O2F_CUDA(cudaStreamEndCapture(stream_, &graph));
  O2F_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  KrylovState* hks = static_cast<KrylovState*>(mailbox_);
  int err = O2F_OK;
  std::string msg;
  try {
    if (bb[0] == 0.0) {
      relres = 0.0;
    } else {
      while (total < max_iter) {
        // One restart chunk: solveWithGuess (src/shape_optimization.cpp:712).
        ks.chunk_max = std::min<int64_t>(restart, max_iter - total);
        ks.it = total;
        O2F_CUDA(cudaMemcpyAsync(ks_, &ks, sizeof(KrylovState), cudaMemcpyHostToDevice, stream_));
        jt_apply_dev(lam_, tmp_);
        k_bicg_start<<<kgrid, kBlock, 0, stream_>>>(n4, reinterpret_cast<double*>(b_),
                                                       reinterpret_cast<double*>(tmp_), reinterpret_cast<double*>(r_),
                                                       reinterpret_cast<double*>(r0_), reinterpret_cast<double*>(p_),
                                                       reinterpret_cast<double*>(v_), part_, ks_);
        O2F_CUDA(cudaGetLastError());
        int64_t launched = 0;
        while (true) {
          O2F_CUDA(cudaMemcpyAsync(hks, ks_, sizeof(KrylovState), cudaMemcpyDeviceToHost, stream_));
          sync();
          if (hks->stop) break;
          const int reps = launched < 64 ? 1 : 4;
          for (int r = 0; r < reps; ++r) O2F_CUDA(cudaGraphLaunch(exec, stream_));
          launched += reps * kItersPerGraph;
          launches_ += (int64_t)reps * kItersPerGraph * kernels_per_iter;
        }
        const int64_t chunk_its = hks->it_chunk;
        total += chunk_its;
        // True residual (src/shape_optimization.cpp:716-717).
        jt_apply_dev(lam_, tmp_);
        k_bicg_start<<<kgrid, kBlock, 0, stream_>>>(n4, reinterpret_cast<double*>(b_),
                                                       reinterpret_cast<double*>(tmp_), reinterpret_cast<double*>(s_),
                                                       reinterpret_cast<double*>(t_), reinterpret_cast<double*>(p_),
                                                       reinterpret_cast<double*>(v_), part_, ks_);
        O2F_CUDA(cudaMemcpyAsync(hks, ks_, sizeof(KrylovState), cudaMemcpyDeviceToHost, stream_));
        sync();
        if (precond) ilu_check_sweeps();
        relres = std::sqrt(hks->rr) / (bnorm > 0 ? bnorm : 1.0);
        if (params_.verbosity >= 1) std::fprintf(stderr, "[adjoint] iters=%lld  relres=%g\n", (long long)total, relres);
        if (relres <= tol) break;
        if (!std::isfinite(relres)) {
          err = O2F_ERR_NONFINITE;
          msg = "BiCGSTAB diverged";
          break;
        }
        if (chunk_its == 0) {
          err = O2F_ERR_BREAKDOWN;
          msg = "BiCGSTAB breakdown";
          break;
        }
      }
      if (err == O2F_OK && relres > tol) {
        err = O2F_ERR_NOT_CONVERGED;
        msg = "BiCGSTAB did not converge";
      }
    }
  } catch (...) {
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    throw;
  }
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  have_lambda_ = true;
  if (iters) *iters = total;
  if (relres_out) *relres_out = relres;
  if (lambda_ref) to_reference(lam_, lambda_ref);
  if (err != O2F_OK) throw Error(err, msg);
}

void Solver::ensure_pert_buffers() {
  if (pert_alloc_) return;
  pgeom_.cgeom = arena_.alloc<Vec4<double>>(topo_.nc);
  pgeom_.egeom = arena_.alloc<Vec4<double>>(topo_.ne);
  pgeom_.ectr = arena_.alloc<Vec2<double>>(topo_.ne);
  pgeom_.vxy = arena_.alloc<Vec2<double>>(topo_.nv);
  pgeom_.vw = arena_.alloc<double>(topo_.nnz);
  pwork_ = alloc_work();
  Rp_ = arena_.alloc<Vec4<double>>(topo_.nc);
  pert_alloc_ = true;
}

void Solver::perturbed_geometry(const o2f_shape_params& sp, int id, double eps) {
  ensure_pert_buffers();
  cudaStream_t s = stream_;
  O2F_CUDA(cudaMemcpyAsync(pgeom_.cgeom, geom_.cgeom, topo_.nc * sizeof(Vec4<double>), cudaMemcpyDeviceToDevice, s));
  O2F_CUDA(cudaMemcpyAsync(pgeom_.egeom, geom_.egeom, topo_.ne * sizeof(Vec4<double>), cudaMemcpyDeviceToDevice, s));
  O2F_CUDA(cudaMemcpyAsync(pgeom_.ectr, geom_.ectr, topo_.ne * sizeof(Vec2<double>), cudaMemcpyDeviceToDevice, s));
  O2F_CUDA(cudaMemcpyAsync(pgeom_.vxy, geom_.vxy, topo_.nv * sizeof(Vec2<double>), cudaMemcpyDeviceToDevice, s));
  O2F_CUDA(cudaMemcpyAsync(pgeom_.vw, geom_.vw, topo_.nnz * sizeof(double), cudaMemcpyDeviceToDevice, s));
  ShapeArgs a{};
  a.pos_x = sp.pos_x;
  a.c = sp.c;
  a.m0 = sp.m;
  a.p0 = sp.p;
  a.t0 = sp.t;
  a.m1 = sp.m;
  a.p1 = sp.p;
  a.t1 = sp.t;
  if (id == O2F_PARAM_M)
    a.m1 = sp.m + eps;
  else if (id == O2F_PARAM_P)
    a.p1 = sp.p + eps;
  else if (id == O2F_PARAM_T)
    a.t1 = sp.t + eps;
  else
    throw Error(O2F_ERR_ARG, "unknown shape parameter id");
  const Topo& t = topo_;
  if (t.n_pert_verts)
    k_perturb_vertices<<<grid(t.n_pert_verts), kBlock, 0, s>>>(t.n_pert_verts, t.pert_verts, a, pgeom_.vxy);
  if (t.n_pert_cells)
    k_perturb_cells<double><<<grid(t.n_pert_cells), kBlock, 0, s>>>(t.n_pert_cells, t.pert_cells, t.cverts, t.ctype,
                                                                     t.nc, pgeom_.vxy, params_.limiter_k, pgeom_.cgeom);
  if (t.n_pert_edges)
    k_perturb_edges<double><<<grid(t.n_pert_edges), kBlock, 0, s>>>(t.n_pert_edges, t.pert_edges, t.ev, t.ec,
                                                                     pgeom_.vxy, pgeom_.cgeom, pgeom_.egeom,
                                                                     pgeom_.ectr);
  if (t.n_pert_wverts)
    k_vertex_weights<double><<<grid(t.n_pert_wverts), kBlock, 0, s>>>(t.n_pert_wverts, t.pert_wverts, t.voff, t.vcid,
                                                                       t.vcid, t.vbc, pgeom_.vxy, pgeom_.cgeom,
                                                                       pgeom_.vw);
  O2F_CUDA(cudaGetLastError());
}

void Solver::shape_gradient(const o2f_shape_params& sp, const int* ids, int n, double beta, double eps,
                            const double* lambda_ref, double* grad) {
  NvtxRange nvtx_("o2f shape_gradient");
  if (n < 0 || (n > 0 && (!ids || !grad))) throw Error(O2F_ERR_ARG, "invalid parameter list");
  if (!(eps > 0.0)) throw Error(O2F_ERR_ARG, "eps must be positive");
  if (!lam_) lam_ = arena_.alloc<Vec4<double>>(topo_.nc);
  if (lambda_ref) {
    to_internal(lambda_ref, lam_);
  } else if (!have_lambda_) {
    throw Error(O2F_ERR_STATE, "no adjoint solution: solve first or pass lambda");
  }
  // computeShapeGradient starts with a residual of the unperturbed mesh (:955-956).
  launch_residual(geom_, work_, U_, nullptr, false, nullptr);
  have_residual_ = true;
  invalidate_linearisation();
  for (int k = 0; k < n; ++k) {
    double J[2];
    for (int sgn = 0; sgn < 2; ++sgn) {
      perturbed_geometry(sp, ids[k], sgn == 0 ? eps : -eps);
      launch_residual(pgeom_, pwork_, U_, nullptr, false, nullptr);
      k_forces<double><<<1, kBlock, 0, stream_>>>(topo_.n_wall, topo_.wall_edges, pgeom_, pwork_.eL, pwork_.etq,
                                                  phys_, beta, scal_ + 4 + 4 * sgn);
      if (sgn == 0)
        O2F_CUDA(cudaMemcpyAsync(Rp_, pwork_.R, topo_.nc * sizeof(Vec4<double>), cudaMemcpyDeviceToDevice, stream_));
    }
    k_lambda_dR<double><<<kRedGrid, kBlock, 0, stream_>>>(topo_.nc, lam_, Rp_, pwork_.R, 2.0 * eps, part_, ticket_,
                                                          scal_ + 12);
    O2F_CUDA(cudaGetLastError());
    double h[16];
    O2F_CUDA(cudaMemcpyAsync(h, scal_, 16 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    sync();
    J[0] = h[4 + 2];
    J[1] = h[8 + 2];
    const double dJ_direct = (J[0] - J[1]) / (2.0 * eps);
    grad[k] = dJ_direct - h[12];
  }
}

void Solver::debug_perturbed(const o2f_shape_params& sp, int id, double eps, const std::string& which,
                             double* out) {
  perturbed_geometry(sp, id, eps);
  sync();
  const int64_t nc = hm_.nc, ne = hm_.ne, nv = hm_.nv;
  if (which == "cell_vol" || which == "cell_ctr") {
    std::vector<Vec4<double>> g(nc);
    O2F_CUDA(cudaMemcpy(g.data(), pgeom_.cgeom, nc * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t co = cperm_[c];
      if (which == "cell_vol") {
        out[co] = g[c].c;
      } else {
        out[2 * co] = g[c].a;
        out[2 * co + 1] = g[c].b;
      }
    }
  } else if (which == "edge_len" || which == "edge_n" || which == "edge_ctr") {
    std::vector<Vec4<double>> g(ne);
    std::vector<Vec2<double>> ce(ne);
    O2F_CUDA(cudaMemcpy(g.data(), pgeom_.egeom, ne * sizeof(Vec4<double>), cudaMemcpyDeviceToHost));
    O2F_CUDA(cudaMemcpy(ce.data(), pgeom_.ectr, ne * sizeof(Vec2<double>), cudaMemcpyDeviceToHost));
    for (int64_t e = 0; e < ne; ++e) {
      const int64_t eo = eperm_[e];
      if (which == "edge_len") {
        out[eo] = g[e].c;
      } else if (which == "edge_n") {
        out[2 * eo] = g[e].a;
        out[2 * eo + 1] = g[e].b;
      } else {
        out[2 * eo] = ce[e].a;
        out[2 * eo + 1] = ce[e].b;
      }
    }
  } else if (which == "vert_xy") {
    std::vector<Vec2<double>> g(nv);
    O2F_CUDA(cudaMemcpy(g.data(), pgeom_.vxy, nv * sizeof(Vec2<double>), cudaMemcpyDeviceToHost));
    for (int64_t v = 0; v < nv; ++v) {
      out[2 * vperm_[v]] = g[v].a;
      out[2 * vperm_[v] + 1] = g[v].b;
    }
  } else if (which == "vert_w") {
    std::vector<double> w(topo_.nnz);
    O2F_CUDA(cudaMemcpy(w.data(), pgeom_.vw, w.size() * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int32_t> voff(nv + 1);
    // Rebuild the internal CSR offsets to map back to reference order.
    int64_t acc = 0;
    for (int64_t v = 0; v < nv; ++v) {
      voff[v] = (int32_t)acc;
      acc += hm_.vert_coff[vperm_[v] + 1] - hm_.vert_coff[vperm_[v]];
    }
    for (int64_t v = 0; v < nv; ++v) {
      const int64_t vo = vperm_[v];
      for (int64_t k = hm_.vert_coff[vo]; k < hm_.vert_coff[vo + 1]; ++k)
        out[k] = w[voff[v] + (k - hm_.vert_coff[vo])];
    }
  } else {
    throw Error(O2F_ERR_ARG, "unknown perturbed array '" + which + "'");
  }
}

}  // namespace o2f
