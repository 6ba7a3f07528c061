/*
 * o2f.h -- C ABI of the B200 implementation of the shape-gradient hot path of
 * the 2-D compressible Navier-Stokes adjoint shape optimiser
 * (ThibaultMaurelOujia/Optimisation2Forme).
 *
 * The reference has no FFI layer: its path is a set of C++ free functions in
 * namespace navier_stokes that mutate an array-of-structs Mesh&.  Each entry
 * point below replaces one of them (reference file:line in its comment).  The
 * device-resident solver context plays the role of the reference Mesh: it owns
 * the renumbered mesh, the cell state, the interface states and wall stresses
 * left by the last residual, and all scratch memory.
 *
 * Conventions
 *  - Every function returns O2F_OK (0) or a negative o2f_status; no exception
 *    crosses the ABI.  o2f_last_error() returns a message for the calling
 *    thread's last failure.
 *  - Arrays at the boundary are in the REFERENCE orders (cells in Gmsh element
 *    order, edges in (vmin,vmax) lexicographic order), interleaved 4*i+k for
 *    per-cell 4-vectors (rho, rho_u, rho_v, E) exactly like the reference's
 *    adjoint vectors (src/shape_optimization.cpp:616-629).  Internally the
 *    mesh is renumbered along a Hilbert curve; that permutation never leaks.
 *  - Pointers passed with a *_host suffix are host memory; *_dev pointers are
 *    device memory on the context's device.  All work is issued on the
 *    context's stream; functions that return host values synchronise it.
 *  - One context per host thread at a time (like the reference, which is not
 *    reentrant); several contexts may coexist in one process, unlike the
 *    reference whose function-static scratch buffers tie a process to one
 *    mesh size (src/advection.cpp:9-23).
 */
#ifndef O2F_H
#define O2F_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum o2f_status {
  O2F_OK = 0,
  O2F_ERR_ARG = -1,        /* invalid argument (null pointer, bad size)       */
  O2F_ERR_IO = -2,         /* file cannot be opened / parsed                  */
  O2F_ERR_MESH = -3,       /* mesh topology unsupported or inconsistent       */
  O2F_ERR_CUDA = -4,       /* CUDA runtime error                              */
  O2F_ERR_NONFINITE = -5,  /* NaN/Inf in a state, residual or Krylov scalar   */
  O2F_ERR_NOT_CONVERGED = -6, /* iteration cap reached before tolerance      */
  O2F_ERR_BREAKDOWN = -7,  /* BiCGSTAB breakdown (rho or omega ~ 0)          */
  O2F_ERR_STATE = -8,      /* call order violated (e.g. adjoint before a residual) */
  O2F_ERR_INTERNAL = -9    /* host out of memory or an unexpected internal error */
} o2f_status;

/* Boundary codes, identical to the reference's char codes
 * (src/mesh.cpp:84-108, src/boundary.cpp:19-42). */
#define O2F_BC_NONE 0
#define O2F_BC_INLET 'i'
#define O2F_BC_OUTLET 'o'
#define O2F_BC_FARFIELD 'f'
#define O2F_BC_WALL 'w'

/* Limiter choice.  VENKAT is the reference's live limiter
 * (src/advection.cpp:209-230, eps=(k*h)^3); BARTH_JESPERSEN is the
 * reference's commented-out alternative (src/advection.cpp:195-207). */
#define O2F_LIMITER_VENKAT 0
#define O2F_LIMITER_BARTH_JESPERSEN 1

/* Preconditioner of the adjoint BiCGSTAB.  NONE is the reference's
 * Eigen::IdentityPreconditioner (src/shape_optimization.cpp:699); ILU0 is a
 * block (4x4) ILU(0) of J^T in reverse Cuthill-McKee order.  Both solve the
 * same system to the same true-residual tolerance. */
#define O2F_PRECOND_NONE 0
#define O2F_PRECOND_ILU0 1

/* Diffusive time-step bound.  REFERENCE is 0.5*min_h^2/mu
 * (src/simulation.cpp:109).  THERMAL uses 0.5*min_h^2/max(mu, kappa*(gamma-1)):
 * the reference's heat flux q = -kappa*grad((gamma-1)*e) has no 1/R factor
 * (src/diffusion.cpp:237-240), so its effective diffusivity is kappa*(gamma-1),
 * which the reference's bound ignores; on cells below ~1e-5 chord that term
 * is the explicit stability limit.  The residual is the same in both modes. */
#define O2F_DT_REFERENCE 0
#define O2F_DT_THERMAL 1

/* Operator of the adjoint.  REFERENCE is the reference's: J^T of the
 * first-order HLLC flux by finite differences and the inviscid wall-pressure
 * right-hand side (applyJacobianTranspose / assembleAdjointRHS,
 * src/shape_optimization.cpp:237-554).  FULL is the consistent adjoint: the
 * Jacobian of the whole residual (reconstruction, limiter, diffusion,
 * boundary conditions) by coloured central differences about the current
 * state, stored as 4x4 blocks, and dJ/dU of the whole objective (pressure and
 * wall stresses) by the same perturbations.  It changes the results. */
#define O2F_JAC_REFERENCE 0
#define O2F_JAC_FULL 1
/* FROZEN: as FULL with the limiter values held at the current state (the
 * usual linearisation of limited schemes: reconstruction, fluxes, diffusion
 * and objective differentiated, the limiter's own derivative left out). */
#define O2F_JAC_FROZEN 2

/* Triangular sweeps of the block ILU(0) preconditioner.  BLOCK: one thread
 * block walks the dependency levels (one SM per sweep: best when several
 * contexts solve at once, and alone on small meshes); WAITING: persistent
 * warps on up to 64 SMs, each row waiting on its dependencies (best alone on
 * large meshes); AUTO: BLOCK up to 200,000 cells, else WAITING. */
#define O2F_SWEEPS_AUTO 0
#define O2F_SWEEPS_BLOCK 1
#define O2F_SWEEPS_WAITING 2

/* Arithmetic of the residual / Jacobian-transpose kernels. */
#define O2F_PREC_F64 0 /* FP64 throughout (parity mode)                           */
#define O2F_PREC_F32 1 /* FP32 residual and JT, FP64 reductions, dt and Krylov     */

/* Physics and numerics.  Field names and defaults mirror the reference's
 * SimulationParams (include/params.hpp:15-81) plus the keys the reference
 * hard-codes (marked NEW).  o2f_params_default() fills the reference
 * defaults after SimulationParams::finalize() (src/params.cpp:5-8). */
typedef struct o2f_params {
  double gamma;           /* 1.4                                              */
  double viscosity;       /* dynamic viscosity mu [Pa s]                      */
  double Pr;              /* Prandtl number                                    */
  double cp;              /* 1005                                              */
  double cfl_number;      /* CFL of the global time step                       */
  double final_time;      /* time-loop end (src/simulation.cpp:75)             */
  double inflow_velocity; /* freestream Mach number (src/boundary.cpp:12)      */
  double rho_ref;         /* 1.225                                             */
  double p_ref;           /* 101325                                            */
  double aoa_deg;         /* NEW: angle of attack, rotates the freestream and
                             the lift/drag axes; 0 reproduces the reference    */
  double limiter_k;       /* NEW: Venkatakrishnan K, eps=(K h)^3; reference 1e-2 */
  double adjoint_shift;   /* NEW: ILU(0) preconditioner built from J^T + s*|D_c| I
                             (D_c: diagonal block, |.|: max row sum); 0 = plain
                             ILU(0).  Changes the preconditioner only.          */
  int limiter;            /* NEW: O2F_LIMITER_*                                */
  int precision;          /* NEW: O2F_PREC_*                                   */
  int adjoint_precond;    /* NEW: O2F_PRECOND_* (default ILU0)                 */
  int dt_mode;            /* NEW: O2F_DT_* diffusive time-step bound             */
  int verbosity;        /* >= 1: "[adjoint] iters=.. relres=.." per restart chunk
                             on stderr, as src/shape_optimization.cpp:719 prints */
  int adjoint_jacobian;   /* NEW: O2F_JAC_* operator and right-hand side of the
                             adjoint (default REFERENCE)                        */
  double adjoint_fd_step; /* NEW: relative step of the FULL Jacobian's central
                             differences (default 1e-9)                         */
  int adjoint_precision;  /* NEW: O2F_PREC_F32 streams the Jacobian blocks of the
                             BiCGSTAB products in FP32, every restart taking the
                             true residual with the FP64 operator (iterative
                             refinement: same solution and tolerance); F64
                             default.  FP32 contexts always do this.             */
  int adjoint_sweeps;     /* NEW: O2F_SWEEPS_* triangular sweeps of the block
                             ILU(0) preconditioner (same results, bit for bit) */
} o2f_params;

void o2f_params_default(o2f_params* p);

/* Mesh description in the reference's construction order (src/mesh.cpp:7-283):
 *  - nodes in vertex order (Gmsh node-tag order);
 *  - boundary segments in physical-group order: a vertex touched by several
 *    groups keeps the LAST code, as in the reference (src/mesh.cpp:84-108);
 *  - cells (triangles: 3 vertices, quads: 4) in element order, counter- or
 *    clockwise.  cell_offsets[n_cells] = total vertex count. */
typedef struct o2f_mesh_desc {
  int64_t n_nodes;
  const double* node_xy;     /* [n_nodes*2]                                    */
  int64_t n_segments;
  const int64_t* segments;   /* [n_segments*2] vertex indices                  */
  const uint8_t* segment_bc; /* [n_segments] O2F_BC_* codes                    */
  int64_t n_cells;
  const int64_t* cell_offsets; /* [n_cells+1]                                  */
  const int64_t* cell_nodes;   /* vertex indices                               */
} o2f_mesh_desc;

typedef struct o2f_mesh_info {
  int64_t n_cells, n_edges, n_vertices;
  int64_t n_wall_edges, n_boundary_edges;
  int64_t max_vertex_valence;
  double min_h; /* min over cells of 2V/perimeter (src/simulation.cpp:98-104) */
  size_t device_bytes;
} o2f_mesh_info;

typedef struct o2f_ctx o2f_ctx;
typedef struct o2f_host_mesh o2f_host_mesh;

const char* o2f_last_error(void);
const char* o2f_version(void);

/* Host-only mesh build (no GPU needed): the topology, geometry and
 * interpolation weights the context is built from, in reference order.  The
 * construction replaces navier_stokes::Mesh::Mesh (src/mesh.cpp:7-283) and
 * recordEdge (:288-297).  Export names: see o2f_mesh_export.  .msh files
 * (ASCII MSH 2.x) from 1 MB have their node and element lines parsed by all
 * host threads, with the result of the stream parser used below that size
 * and for irregular layouts. */
int o2f_host_mesh_create(const o2f_mesh_desc* mesh, o2f_host_mesh** out);
int o2f_host_mesh_from_msh(const char* path, o2f_host_mesh** out);

/* No counterpart in the reference.  As o2f_host_mesh_create, with the
 * integer topology built on the GPU on `stream` (NULL: the default stream):
 * the std::map edge order by a stable radix sort of the (vmin, vmax) keys,
 * the std::unordered_set iteration orders of Vertex::cellIDs, Cell::edgeIDs
 * and Cell::neighbourIDs by emulation (valence up to 257); geometry and
 * weights on the host.  Every exported array equals o2f_host_mesh_create's. */
int o2f_host_mesh_create_gpu(const o2f_mesh_desc* mesh, void* stream, o2f_host_mesh** out);
int o2f_host_mesh_export(const o2f_host_mesh* mesh, const char* which, void* out, int64_t* count);
int o2f_host_mesh_destroy(o2f_host_mesh* mesh);

/* No counterpart in the reference.  New vertex coordinates for a host mesh
 * of unchanged topology, node_xy[2*n_nodes] in the description's node order:
 * volumes, centres, edge normals and centres, the atan2 cell order of the
 * vertices (Mesh::Mesh, src/mesh.cpp:140-248) and the interpolation weights
 * are recomputed with the arithmetic of o2f_host_mesh_create, so every
 * exported array equals that of a mesh created from these coordinates.
 * O2F_ERR_ARG for non-finite coordinates; O2F_ERR_MESH, mesh unchanged, when
 * a cell would collapse or change orientation. */
int o2f_host_mesh_set_coords(o2f_host_mesh* mesh, const double* node_xy);

/* Binary state checkpoint, alongside the reference's text state file
 * (saveCellStates / loadCellStates, src/utils.cpp:29-107), which it does not
 * replace.  The same values in the same cell order, exactly: a 64-byte header
 * (magic "O2FSOA1", version, field count, cell count, time, steps, FNV-1a
 * hash of the payload) and the four conserved fields as contiguous float64
 * arrays.  U_host: 4 values per cell, interleaved (4i+k), mesh-file cell
 * order, as o2f_state_set / o2f_state_get.  Host only (no GPU).
 * o2f_checkpoint_read: O2F_ERR_IO for a missing, foreign, truncated or
 * corrupted file and for a cell count other than n_cells; time and steps
 * may be NULL. */
int o2f_checkpoint_write(const char* path, int64_t n_cells, const double* U_host, double time, int64_t steps);
int o2f_checkpoint_read(const char* path, int64_t n_cells, double* U_host, double* time, int64_t* steps);

/* Build a context: replaces navier_stokes::Mesh::Mesh(params)
 * (src/mesh.cpp:7-283; include/mesh.hpp:116) followed by the solver set-up.
 * `stream` is a cudaStream_t (NULL: the context creates its own). */
int o2f_create(const o2f_mesh_desc* mesh, const o2f_params* params, void* stream, o2f_ctx** out);
/* Same, reading an ASCII MSH 2.2 file with physical groups named Inlet,
 * Outlet, FreeStream, Wall or Airfoil, as the reference's Gmsh import does. */
int o2f_create_from_msh(const char* path, const o2f_params* params, void* stream, o2f_ctx** out);
int o2f_destroy(o2f_ctx* ctx);
int o2f_set_params(o2f_ctx* ctx, const o2f_params* params);
int o2f_get_info(const o2f_ctx* ctx, o2f_mesh_info* info);

/* Topology and geometry in reference order, for checking the mesh build
 * (integer arrays must equal the reference's exactly).  `which` selects one
 * array; *count receives its length; pass out=NULL to query the length.
 * Names: "edge_v","edge_c","edge_bc","cell_edges_off","cell_edges",
 * "vert_cells_off","vert_cells","vert_cells_ord","cell_verts_off",
 * "cell_verts","vert_bc" (int64) and "vert_xy","edge_len","edge_n",
 * "edge_ctr","cell_vol","cell_ctr","vert_w" (double). */
int o2f_mesh_export(const o2f_ctx* ctx, const char* which, void* out, int64_t* count);

/* Cell state, [n_cells*4] interleaved, reference cell order.  Replaces
 * loadCellStates / saveCellStates (src/utils.cpp:29-107) at the device
 * boundary; the text format itself is handled by the host helpers. */
int o2f_state_set(o2f_ctx* ctx, const double* U_host);
int o2f_state_get(o2f_ctx* ctx, double* U_host);
/* Uniform freestream, init_one_x (src/init.cpp:57-81), rotated by aoa. */
int o2f_state_freestream(o2f_ctx* ctx);

/* One residual evaluation: computeAdvectionTerm + computeDiffusionTerm
 * (src/advection.cpp:415-466, src/diffusion.cpp:206-243), i.e.
 * computeResidual (src/shape_optimization.cpp:171-189).  Leaves the interface
 * states and wall stresses in the context (as the reference leaves them in
 * Mesh::edges).  R_host may be NULL. */
int o2f_residual(o2f_ctx* ctx, double* R_host);

/* Per-stage arrays of the last residual, reference order:
 * "grad" [n_cells*8] (rho_x,rho_u_x,rho_v_x,E_x,rho_y,...), "edge_LR"
 * [n_edges*8], "edge_tau" [n_edges*3], "vertex_U" [n_vertices*4], "R". */
int o2f_debug_get(o2f_ctx* ctx, const char* which, double* out_host);

/* SSP-RK3 time loop, Simulator::time_loop (src/simulation.cpp:68-142):
 * steps while t < final_time, at most max_steps steps, and (NEW) stops when
 * ||R_rho||_2 has dropped by drop_tol relative to the first step (0: off).
 * history_host (may be NULL) receives ||R_rho||_2 of each step's first stage,
 * [max_steps]. */
int o2f_rk3_run(o2f_ctx* ctx, int64_t max_steps, double drop_tol, double* history_host,
                int64_t* steps_done, double* t_out);

/* computeLiftDragCoefficients (src/compute.cpp:92-132) and
 * computeDirectObjectiveTerm J = -C_L + beta*C_D
 * (src/shape_optimization.cpp:893-939, wall edges with centre.x > 1.3
 * skipped), from the interface states of the last residual.
 * forces_out = {C_L, C_D, J}. */
int o2f_forces(o2f_ctx* ctx, double beta, double* forces_out);

/* y = J^T x, applyJacobianTranspose (src/shape_optimization.cpp:237-484),
 * about the interface states of the last residual.  x, y [n_cells*4]. */
int o2f_jt_apply(o2f_ctx* ctx, const double* x_host, double* y_host);

/* b = dJ/dU, assembleAdjointRHS (src/shape_optimization.cpp:491-554). */
int o2f_adjoint_rhs(o2f_ctx* ctx, double beta, double* b_host);

/* Solve J^T lambda = b with restarted BiCGSTAB, solveAdjointSystem
 * (src/shape_optimization.cpp:658-740): inner chunks of `restart`
 * iterations, a true-residual check after each, stop at relres <= tol.
 * lambda_host may be NULL (lambda stays in the context). */
int o2f_adjoint_solve(o2f_ctx* ctx, double beta, double tol, int64_t max_iter, int64_t restart,
                      double* lambda_host, int64_t* iters, double* relres);

/* NEW: o2f_adjoint_solve started from lambda0_host (reference order)
 * instead of zero -- the warm start of the learned predictor.  The solution
 * criterion is unchanged: true relres <= tol. */
/* No counterpart in the reference.  J^T lambda = rhs (rhs: 4 values per
 * cell, interleaved, mesh-file cell order) with the context's operator,
 * preconditioner and stopping rule of o2f_adjoint_solve; lambda0_host may be
 * NULL (start from zero).  For outer iterations built on the adjoint
 * operator, e.g. defect correction. */
int o2f_adjoint_solve_rhs(o2f_ctx* ctx, const double* rhs_host, double tol, int64_t max_iter, int64_t restart,
                          const double* lambda0_host, double* lambda_host, int64_t* iters, double* relres);

int o2f_adjoint_solve_guess(o2f_ctx* ctx, double beta, double tol, int64_t max_iter, int64_t restart,
                            const double* lambda0_host, double* lambda_host, int64_t* iters, double* relres);

/* NACA-4 shape parameters (src/shape_optimization.cpp:830-834 defaults). */
typedef struct o2f_shape_params {
  double pos_x; /* 0.355 */
  double c;     /* 1.0   */
  double m;     /* 0.02  */
  double p;     /* 0.4   */
  double t;     /* 0.12  */
} o2f_shape_params;

/* Gradient parameter selectors. */
#define O2F_PARAM_M 0
#define O2F_PARAM_P 1
#define O2F_PARAM_T 2 /* NEW: the reference returns without perturbing for t */

/* Shape gradient g_k = dJ_direct/dtheta_k - lambda . dR/dtheta_k by central
 * differences, computeShapeGradient (src/shape_optimization.cpp:942-1016),
 * with applyShapePerturbationNACA12 + updateDerivedGeometry (:748-890).
 * lambda_host == NULL uses the context's last adjoint solution. */
int o2f_shape_gradient(o2f_ctx* ctx, const o2f_shape_params* shape, const int* param_ids, int n_params,
                       double beta, double eps, const double* lambda_host, double* grad_out);

/* The whole of optimizeShape (src/shape_optimization.cpp:1022-1067):
 * J from the current interface states, adjoint solve, shape gradient.
 * out = {J, iters, relres}. */
int o2f_optimize_shape(o2f_ctx* ctx, const o2f_shape_params* shape, const int* param_ids, int n_params,
                       double beta, double eps, double tol, double* grad_out, double* out);

/* Geometry after applyShapePerturbationNACA12(param, eps) for checking:
 * "vert_xy","edge_len","edge_n","edge_ctr","cell_vol","cell_ctr","vert_w". */
int o2f_debug_perturbed(o2f_ctx* ctx, const o2f_shape_params* shape, int param_id, double eps,
                        const char* which, double* out_host);

/* Device pointers (n_cells*4, interleaved, INTERNAL Hilbert order) and
 * the permutation old->new, for device-resident callers. */
int o2f_state_device(o2f_ctx* ctx, double** U_dev);
int o2f_cell_permutation(const o2f_ctx* ctx, int64_t* new_of_old_host);

/* Timing of the last o2f_residual and the number of kernels launched so far. */
typedef struct o2f_timing {
  double residual_ms;  /* last o2f_residual */
  int64_t kernel_launches;
} o2f_timing;
int o2f_get_timing(const o2f_ctx* ctx, o2f_timing* t);

/* Kernel classes timed by o2f_profile_kernels (no reference counterpart:
 * per-kernel CUDA-event timing replaces the reference's wall-clock
 * time_tic/time_toc printouts, src/utils.cpp:13-23). */
#define O2F_K_VERTEX_STATE 0  /* cell -> vertex state interpolation          */
#define O2F_K_CELL_GRADIENT 1 /* Green-Gauss, limiter, interface states, tau  */
#define O2F_K_VERTEX_VISC 2   /* cell -> vertex tau/q interpolation           */
#define O2F_K_EDGE_FLUX 3     /* HLLC + edge viscous values                   */
#define O2F_K_CELL_RESIDUAL 4 /* residual gather + viscous divergence         */
#define O2F_K_JT_APPLY 5      /* matrix-free J^T x                            */
#define O2F_K_JT_BLOCKS 6     /* finite-difference flux Jacobian blocks       */
#define O2F_K_COUNT 7
/* Launches each kernel class `reps` times back to back on the context stream
 * (about the current state) and writes the mean duration of one launch in
 * milliseconds, measured with CUDA events on that stream, to
 * ms_out[O2F_K_COUNT]. */
int o2f_profile_kernels(o2f_ctx* ctx, int reps, double* ms_out);

/* Batched time loop (no reference counterpart: the reference solves one
 * candidate per process, run_opti.sh).  A batch references n existing
 * contexts of one precision, all O2F_PREC_F64 or all O2F_PREC_F32 (each with
 * its own mesh, flow parameters and state; all on one device, the batch runs
 * on the first context's stream); the contexts must outlive the batch, must
 * not be used while a batch call runs and must keep their precision.
 * o2f_batch_rk3_run advances every candidate by SSP-RK3 exactly as
 * o2f_rk3_run would (bit-identical states, each candidate with its own
 * dt and stop condition; FP32 contexts run the mixed-precision residual and
 * leave the FP64 linearisation of their last stage, as o2f_rk3_run does)
 * with one grouped launch per phase for the whole batch, captured in a CUDA
 * graph.  Per candidate: steps_done, t_out,
 * status_out (O2F_OK or O2F_ERR_NONFINITE); any may be NULL.  After the run
 * each context holds the interface states of its last stage, so
 * o2f_forces / o2f_adjoint_solve / o2f_shape_gradient apply per context. */
typedef struct o2f_batch o2f_batch;
int o2f_batch_create(o2f_ctx* const* ctxs, int n, o2f_batch** out);
int o2f_batch_destroy(o2f_batch* batch);
/* Autotuner: times every phase of the grouped step with block sizes
 * 128/256/512 and 1/2/4 entities per thread (reps launches each, CUDA
 * events), keeps the fastest, and caches it for batches of the same size
 * bucket (log2 of the total cells).  config_out (may be NULL) receives
 * {block, tile} for the O2F_BATCH_PHASES phases: vertex state, cell
 * gradient, vertex viscous, edge flux, cell residual, wave speed. */
#define O2F_BATCH_PHASES 6
int o2f_batch_tune(o2f_batch* batch, int reps, int* config_out);
int o2f_batch_rk3_run(o2f_batch* batch, int64_t max_steps, double drop_tol, int64_t* steps_done, double* t_out,
                      int* status_out);
/* Kernels launched by the batch so far (grouped phases and step kernels). */
int o2f_batch_launches(o2f_batch* batch, int64_t* launches);
/* ||R_rho||_2 history of candidate `index` from the last o2f_batch_rk3_run. */
int o2f_batch_history(o2f_batch* batch, int index, double* history_host, int64_t count);

/* Warm-start network (no reference counterpart).  Inputs per point:
 * {x, y, m, p, t, Mach, AoA} (float32, 7 per point); outputs: 8 float32
 * (normalised state and adjoint, as the caller defines them).  Fourier
 * features of (x, y) (32 seeded frequencies, scale freq_scale) and the raw
 * inputs feed 4 hidden layers of 256 SiLU units.  Training (MSE, Adam) and
 * inference run on the GPU in this library's tcgen05 kernels: BF16 weights
 * and activations, FP32 accumulation, FP32 master weights.  max_batch bounds
 * the points per GEMM pass (128 .. 2^20). */
typedef struct o2f_mlp o2f_mlp;
int o2f_mlp_create(int max_batch, float freq_scale, uint64_t seed, void* stream, o2f_mlp** out);
int o2f_mlp_destroy(o2f_mlp* net);
int o2f_mlp_n_params(o2f_mlp* net, int64_t* n);
/* Copies a training set to the device: inputs [n*7], targets [n*8]. */
int o2f_mlp_set_data(o2f_mlp* net, const float* inputs, const float* targets, int64_t n);
/* `steps` Adam steps on seeded minibatches of `batch` points; loss_history
 * (may be NULL) receives the minibatch MSE of each step. */
int o2f_mlp_train(o2f_mlp* net, int steps, int batch, float lr, uint64_t seed, float* loss_history);
int o2f_mlp_predict(o2f_mlp* net, const float* inputs, int64_t n, float* outputs);
/* Gradient of the MSE on one batch (n <= max_batch) without an update:
 * grads [o2f_mlp_n_params] in the parameter layout W0,b0,...,W4,b4 (W_l
 * row-major [out][in]; layer sizes 128->256->256->256->256->16, outputs 8..15
 * are padding and stay zero). */
int o2f_mlp_gradients(o2f_mlp* net, const float* inputs, const float* targets, int n, float* grads, float* loss);
/* Parameters (same layout) and the Fourier frequencies [64] (may be NULL). */
int o2f_mlp_get_params(o2f_mlp* net, float* params, float* freq);
int o2f_mlp_set_params(o2f_mlp* net, const float* params);

/* Array forms of the reference's per-edge and per-state functions, which the
 * reference calls one edge or one state at a time inside its loops; n of
 * them per call, evaluated on the GPU by the residual's own device functions
 * (same bits as the reference).  Host arrays in, host arrays out; no context.
 *
 * o2f_hllc_flux: compute_hllc_flux (src/advection.cpp:335-412;
 * include/advection.hpp:16).  LR_host[8*i..8*i+7] = rho_L, rho_u_L, rho_v_L,
 * E_L, rho_R, rho_u_R, rho_v_R, E_R of edge i, normal_host[2*i..] its
 * Edge::edgeNormal (nx, ny); flux_host[4*i..] receives the four fluxes. */
int o2f_hllc_flux(int64_t n, const double* LR_host, const double* normal_host, double gamma, double* flux_host);
/* apply_boundary_conditions for "inflow_outflow_x" (src/boundary.cpp:7-45,
 * 84-94; include/boundary.hpp:13): U_host[4*i..] (rho, rho_u, rho_v, E) is
 * replaced by the boundary state of code codes[i] (O2F_BC_*; other codes
 * leave it).  The freestream comes from params (inflow_velocity, rho_ref,
 * p_ref, gamma; aoa_deg 0 is the reference). */
int o2f_bc_states(const o2f_params* params, int64_t n, const uint8_t* codes, double* U_host);
/* apply_InterfaceStates_boundary_conditions (src/boundary.cpp:48-80;
 * include/boundary.hpp:17-20): the ghost right state R_host[4*i..] of a
 * boundary edge from its left state L_host[4*i..]. */
int o2f_bc_ghosts(const o2f_params* params, int64_t n, const uint8_t* codes, const double* L_host, double* R_host);
/* apply_diffusion_bc (src/boundary.cpp:101-127; include/boundary.hpp:15):
 * tq_host[5*i..] = tau_xx, tau_yy, tau_xy, q_x, q_y, zeroed for far-field
 * and wall codes. */
int o2f_bc_diffusion(int64_t n, const uint8_t* codes, double* tq_host);

/* Test hook of the failure path (no counterpart in the reference).  The
 * block-ILU(0) sweeps wait, bounded, on the ready flags of the rows they
 * depend on; a wait that runs out makes the solve return O2F_ERR_CUDA and
 * leaves the context usable.  Small triangles are swept without waits (one
 * thread block, level by level); while the hook is set (stall != 0 or
 * spin_limit > 0) the solves started after the call use the waiting sweeps,
 * with spin_limit polls per wait (<= 0: the default of 2^22) and, with stall
 * != 0, one row that never writes its value, so the failure path can be
 * exercised without any GPU fault; stall = 0, spin_limit = 0 restores the
 * defaults. */
int o2f_debug_ilu_stall(o2f_ctx* ctx, int stall, int64_t spin_limit);

/* No counterpart in the reference.  For callers that may not allocate
 * device memory during a call -- a host time loop calling it every step,
 * where cudaMalloc would synchronise the device, or a host that owns all
 * device memory through its own pool or budget.  Residual of the current
 * state (as o2f_residual, interface states left in the context) and its
 * ||R_rho||_2 written to *norm_out, with NO device allocation on the call:
 * the norm reduction's scratch is a static device array of 33,280 bytes.
 * Limit: meshes of at most 16,777,216 cells (O2F_ERR_ARG beyond).  Calls
 * that overlap on one device share that scratch and race: serialise them.
 * The first call on a device looks up the scratch address
 * (cudaGetSymbolAddress); make it before any stream capture.  That address
 * is cached for the life of the process: after a cudaDeviceReset of the
 * device, do not call this entry point on it again.  In an FP32 context the
 * residual is o2f_residual's FP32 one (FP64 R, FP64 norm); such a context
 * needs one o2f_residual or o2f_rk3_run before the first call, which
 * allocate its FP32 buffers (O2F_ERR_STATE otherwise). */
int o2f_residual_norm_noalloc(o2f_ctx* ctx, double* norm_out);

/* No counterpart in the reference, whose outer loop (mesh_opti/run_opti.sh)
 * re-meshes each new shape with Gmsh and restarts the solver.  New vertex
 * coordinates for the context's mesh, same topology (node_xy as for
 * o2f_host_mesh_set_coords): the device geometry is rebuilt exactly as
 * o2f_create would build it from these coordinates, the flow state is kept,
 * and a residual must be evaluated again before o2f_forces or the adjoint
 * (O2F_ERR_STATE otherwise).  Errors as o2f_host_mesh_set_coords. */
int o2f_set_vertex_coords(o2f_ctx* ctx, const double* node_xy);

/* No counterpart in the reference.  Moves the context's mesh from the NACA
 * shape `from` to the shape `to` (m, p, t change; pos_x and c must be equal):
 * wall vertices by the formula of applyShapePerturbationNACA12
 * (src/shape_optimization.cpp:828-890; wall vertices at xr >= 0.9 stay),
 * interior vertices by inverse distance weighting of the boundary
 * displacements, weights |r|^-power with power in [1, 8], far-field, inlet
 * and outlet vertices fixed; then as o2f_set_vertex_coords. */
int o2f_deform_shape(o2f_ctx* ctx, const o2f_shape_params* from, const o2f_shape_params* to, int power);

/* Headless counterpart of the reference's live SFML view (Simulator::
 * output_step, src/simulation.cpp:176-199): the cell scalar of
 * computeCellScalar (src/compute.cpp:6-60; field "rho", "rho_u", "rho_v",
 * "E", "u", "v", "p" / "pressure", or from the Green-Gauss gradients of a
 * residual of the current state "u_x", "u_y", "v_x", "v_y", "div"), drawn
 * on an nx-by-ny image of the mesh's bounding box, each pixel coloured by
 * the cell containing its centre (Mesh::computePixelsToCellIDs,
 * src/mesh.cpp:349-511; black outside the mesh) with colormap_B_W_R, or
 * colormap_schlieren_bluewhite of sqrt(t) for cmap "schlieren"
 * (src/renderer_colormap.cpp:10-47).  Colour range: range_in {fmin, fmax},
 * or with range_in NULL the cells' min and max (for the pressure rounded
 * outward to multiples of 5000, as output_step does); written to range_out
 * if not NULL.  rgb_out: nx*ny*3 bytes, top image row first; all black when
 * fmax <= fmin, as the reference draws nothing then. */
int o2f_render_field(o2f_ctx* ctx, const char* field, int nx, int ny, const char* cmap, const double* range_in,
                     uint8_t* rgb_out, double* range_out);

#ifdef __cplusplus
}
#endif

#endif /* O2F_H */
