/*
 * refcpu.h — CPU oracle for the NexDynIPC contact step (test infrastructure).
 *
 * This library is the parity checker, not the product: only tests/, the
 * smoke check in __graft_entry__.py and bench.py's CPU-baseline leg load it.
 * It restates, in plain C++ (no Eigen/Boost, which are absent here), the
 * reference's CPU implementation of IPCSolver::step and everything below it
 * (nexdynipc/src/Dynamics/IPCSolver.cpp:808-1231 and the files it calls).
 * Each function in refcpu.cpp cites the reference lines it follows.
 *
 * It shares the scene / state / contact structs of the product's public
 * header include/nxd.h so that both sides read identical inputs.
 */
#ifndef NXD_REFCPU_H
#define NXD_REFCPU_H

#include "../include/nxd.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nxo_world nxo_world;

nxo_world* nxo_create(const nxd_scene_desc* desc);
void nxo_destroy(nxo_world* w);

/* literal_min_distance: 1 = the reference's O(N^2 V (V+F)) loop as written,
 *   0 = the pruned loop (same result whenever the minimum is below 1e-6).
 * min_distance_stride: literal loop visits only bodies i % stride == 0 (used
 *   to time a bounded sample; results are then not the reference's).
 * num_threads: OpenMP threads for the independent loops (1 = serial, as the
 *   reference runs). */
void nxo_set_options(nxo_world* w, int literal_min_distance, int min_distance_stride,
                     int num_threads);

int nxo_step(nxo_world* w, double dt);
int nxo_get_state(nxo_world* w, const nxd_state* out);
int nxo_set_state(nxo_world* w, const nxd_state* in);
int nxo_get_diagnostics(nxo_world* w, nxd_diagnostics* out);
int nxo_get_joint_state(nxo_world* w, double* lambda6, double* stiffness);
/* Per-phase wall time of the last step in seconds:
 * [0] assembly+candidates, [1] adaptive barrier (min distance), [2] CCD,
 * [3] detectContacts, [4] ALM/Newton loop, [5] total. */
void nxo_last_step_times(nxo_world* w, double* out6);

int64_t nxo_body_pairs(nxo_world* w, double r, int32_t* pairs, int64_t cap);
int nxo_build_candidates(nxo_world* w, double activation_distance, nxd_candidates* out);
int nxo_detect_contacts(nxo_world* w, const double* x, nxd_contact* out, int32_t cap,
                        int32_t* count, int32_t* raw_count);
double nxo_scene_min_distance(nxo_world* w, int literal);
double nxo_max_step(nxo_world* w, double dt);

int nxo_set_form_state(nxo_world* w, const nxd_contact* contacts, int32_t n,
                       const double* normal_forces, const double* x_hat, double dt);
int nxo_form_value(nxo_world* w, int32_t form, const double* x, double* out);
int nxo_form_gradient(nxo_world* w, int32_t form, const double* x, double* grad);
/* Dense (6n x 6n, row-major) Hessian of a form, duplicates summed. */
int nxo_form_hessian_dense(nxo_world* w, int32_t form, const double* x, double* H);
int nxo_normal_forces(nxo_world* w, const double* x, double* out, int32_t n);
/* LinearSolver on a caller's 6x6-block BSR matrix: blocks become triplets
 * in storage order, then the same per-component dense LDL^T as the Newton
 * solve.  Returns NXD_OK or NXD_FACTOR_FAILED. */
/* Full-IPC time step (restates nxd_ipc_step). */
int nxo_ipc_step(nxo_world* w, double dt, const nxd_ipc_params* p, nxd_ipc_stats* stats);
int nxo_linear_solve(int32_t n_rows, int64_t nnzb, const int32_t* row_ptr, const int32_t* col_idx,
                     const double* vals, const double* b, double* x);
/* LDL^T solve of H dx = b with the oracle's solver (dense H input). */
int nxo_ldlt_solve(const double* H, int32_t n, const double* b, double* x);

/* select_top_k_indices (ContactAssembler.cpp:67-88) on a score array:
 * std::nth_element + std::sort from this toolchain's libstdc++. */
void nxo_select_top_k(const double* scores, int32_t n, int32_t k, int32_t* out_idx);
/* std::sort of an index array by score (IPCSolver.cpp:571-577 uses it). */
void nxo_std_sort(const double* keys, int32_t n, int32_t* idx_inout);

/* The shared elementary functions (nexdynipc_b200/csrc/nx_libm.h):
 * fn 0 sin, 1 cos, 2 atan2(x, y), 3 log, 4 exp, 5 tanh, 6 cosh. */
void nxo_libm(int32_t fn, const double* x, const double* y, double* out, int32_t n);

/* Stand-alone pieces used by the ported known-answer tests. */
double nxo_barrier_value(double d, double dhat, double kappa);
double nxo_barrier_gradient(double d, double dhat, double kappa);
double nxo_barrier_hessian(double d, double dhat, double kappa);
double nxo_friction_value(const double* u, double N, double mu, double eps);
void nxo_friction_gradient(const double* u, double N, double mu, double eps, double* g);
void nxo_friction_hessian(const double* u, double N, double mu, double eps, double* H9);
double nxo_friction_value_smooth(const double* u, double N, double mu, double eps);
void nxo_friction_gradient_smooth(const double* u, double N, double mu, double eps, double* g);
void nxo_friction_hessian_smooth(const double* u, double N, double mu, double eps, double* H9);
/* Interval root finder on a 1-D polynomial sum c_k t^k (IntervalRootFinder.h:163-190):
 * returns 1 and the root interval if found. */
int nxo_interval_root_poly(const double* coeffs, int32_t degree, double lo, double hi,
                           double tol, double* root_lo, double* root_hi);

/* Geometry accessors (primitives numbered over bodies in world order). */
int32_t nxo_body_count(nxo_world* w);
void nxo_prim_counts(nxo_world* w, int64_t* nv, int64_t* nf, int64_t* ne);
void nxo_prim_topology(nxo_world* w, int32_t* vbody, int32_t* fbody, int32_t* fvert, int32_t* ebody, int32_t* evert);
void nxo_world_vertices_at(nxo_world* w, const double* x, double* wv, double* pos);
void nxo_local_vertices(nxo_world* w, double* vloc, double* quat);

/* Primitive-level contact model (full IPC), ipc_cpu.cpp. */
int nxo_ipc_candidates(nxo_world* w, const double* x, const double* dx, double inflation, int32_t* pt, int64_t pt_cap,
                       int32_t* ee, int64_t ee_cap, int64_t* n_pt, int64_t* n_ee);
int nxo_ipc_barrier(nxo_world* w, const double* x, double dhat, double kappa, double* energy, double* grad, double* H,
                    int64_t* n_pairs, int64_t* n_active);
double nxo_ipc_max_step(nxo_world* w, const double* x, const double* dx, double eta, int64_t* n_pairs);
int nxo_ipc_friction(nxo_world* w, const double* x_lag, const double* x, double dhat, double kappa, double mu, double eps,
                     double* energy, double* grad, double* H, int64_t* n_friction);
int nxo_ipc_pair(int32_t kind, const double* X12, double dhat, double kappa, double* d2, int32_t* type, double* e,
                 double* g12, double* H_sub, double* H_raw, double* H_full);
double nxo_ipc_accd(int32_t kind, const double* X12, const double* D12, double t_max, double eta, int32_t max_iter,
                    int32_t* iters);
double nxo_ipc_dist2(int32_t kind, const double* X12);
void nxo_ipc_friction_derivs(int32_t kind, const double* X12, const double* Xs12, double dhat, double kappa, double mu,
                             double eps, double* g12, double* H, double* Hs, int32_t* type);

#ifdef __cplusplus
}
#endif

#endif
