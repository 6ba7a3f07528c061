/* Test infrastructure only (oracle): a sequential FP64 CPU restatement of the
 * reference's hot path, used by tests/, __graft_entry__.smoke() and the CPU
 * baseline of bench.py to check the CUDA path.  Never linked into the product.
 *
 * The mesh is passed as plain arrays in the reference's own orders (edge ids =
 * (vmin,vmax) lexicographic order; per-cell edge lists and per-vertex cell
 * lists in the iteration order of the reference's std::unordered_set), as
 * exported by o2f_host_mesh_export and checked against the reference's Mesh. */
#ifndef O2F_ORACLE_H
#define O2F_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct o2fo_mesh {
  int64_t nv, nc, ne;
  /* vertices */
  double* vxy;                 /* [2nv]  (mutable: shape perturbation) */
  const int64_t* vbc;          /* [nv]   boundary code                 */
  const int64_t* vert_coff;    /* [nv+1]                               */
  const int64_t* vert_cells;   /* Vertex::cellIDs iteration order       */
  const int64_t* vert_cells_ord; /* Vertex::cellIDsOrdered              */
  /* cells */
  const int64_t* cell_eoff;    /* [nc+1]                               */
  const int64_t* cell_edges;   /* Cell::edgeIDs iteration order         */
  const int64_t* cell_voff;    /* [nc+1]                               */
  const int64_t* cell_verts;   /* Cell::verticeIDs                      */
  double* cvol;                /* [nc]                                 */
  double* cctr;                /* [2nc]                                */
  /* edges */
  const int64_t* edge_v;       /* [2ne] (vmin, vmax)                   */
  const int64_t* edge_c;       /* [2ne] (left, right or -1)            */
  const int64_t* edge_bc;      /* [ne]                                 */
  double* elen;                /* [ne]                                 */
  double* en;                  /* [2ne]                                */
  double* ectr;                /* [2ne]                                */
} o2fo_mesh;

typedef struct o2fo_params {
  double gamma, viscosity, Pr, cp, cfl_number, final_time, inflow_velocity, rho_ref, p_ref;
  double aoa_deg, limiter_k;
  int limiter; /* 0 Venkatakrishnan, 1 Barth-Jespersen */
  int dt_mode; /* 0 reference diffusive dt, 1 also bounded by kappa*(gamma-1) */
} o2fo_params;

typedef struct o2fo_shape {
  double pos_x, c, m, p, t;
} o2fo_shape;

/* computeResidual: R [4nc]; optional outputs (may be NULL): grad [8nc],
 * LR [8ne] interface states, tau [3ne] stored wall stress, vU [4nv]. */
void o2fo_residual(const o2fo_mesh* m, const o2fo_params* p, const double* U, double* R, double* grad, double* LR,
                   double* tau, double* vU);
/* out = {C_L, C_D, J(beta)} from LR and tau. */
void o2fo_forces(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* tau, double beta,
                 double* out);
/* y = J^T x about LR (edge-order accumulation). */
void o2fo_jt(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* x, double* y);
void o2fo_rhs(const o2fo_mesh* m, const o2fo_params* p, const double* LR, double beta, double* b);
/* SSP-RK3 steps (Simulator::time_loop); U in/out; dts, hist [max_steps]. */
int64_t o2fo_march(const o2fo_mesh* m, const o2fo_params* p, double* U, int64_t max_steps, double drop_tol,
                   double* dts, double* hist, double* t_out);
/* Perturbed geometry of applyShapePerturbationNACA12 written into `out`
 * (a mesh whose mutable arrays are caller-owned copies of `m`'s). */
void o2fo_perturb(const o2fo_mesh* m, const o2fo_params* p, const o2fo_shape* s, int param, double eps,
                  o2fo_mesh* out);
void o2fo_shape_gradient(const o2fo_mesh* m, const o2fo_params* p, const double* U, const double* lambda,
                         const o2fo_shape* s, const int* params, int n, double beta, double eps, double* grad);
/* Restarted BiCGSTAB on J^T lambda = b; returns 0 converged, 1 not converged. */
int o2fo_bicgstab(const o2fo_mesh* m, const o2fo_params* p, const double* LR, const double* b, double tol,
                  int64_t max_iter, int64_t restart, double* x, int64_t* iters, double* relres);

#ifdef __cplusplus
}
#endif

#endif
