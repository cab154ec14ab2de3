/*
 * g2o_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU restatement of g2o's Gauss-Newton / Levenberg-Marquardt iteration
 * over a BlockSolver (the path the CUDA backend replaces). It is the checker
 * for the parity tests, the CPU baseline of bench.py and the reference of
 * __graft_entry__.smoke(). Nothing in the product library links or calls it.
 *
 * Parity status: the reference itself cannot be compiled in this environment
 * (it needs Eigen3, which is absent), so this restatement is pinned against
 * the reference's own unit-test fixtures instead: the 36x36 block system of
 * unit_test/solver/sparse_system_helper.cpp (solve within isApprox 1e-6), the
 * analytic-vs-numeric Jacobian tests (unit_test/slam2d/jacobians_slam2d.cpp,
 * unit_test/slam3d/jacobians_slam3d.cpp), the Huber derivative tests
 * (unit_test/general/robust_kernel_tests.cpp) and the two-pose SE3
 * convergence tests (unit_test/slam3d/optimization_slam3d.cpp).
 *
 * The functions mirror the C-ABI of include/g2o_cuda.h one for one, with the
 * prefix orc_ instead of g2oc_, so a test calls both with the same arguments.
 */
#ifndef G2O_ORACLE_H
#define G2O_ORACLE_H

#include "../include/g2o_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

int orc_create(const g2oc_graph* graph, orc_problem** out);
void orc_destroy(orc_problem* p);
int orc_set_params(orc_problem* p, const g2oc_params* params);
void orc_default_params(g2oc_params* params);
int orc_set_threads(int n); /* OpenMP threads for the all-cores baseline */
int orc_get_hessian_info(orc_problem* p, g2oc_hessian_info* info);
int orc_set_estimates(orc_problem* p, const double* pose, const double* point);
int orc_download(orc_problem* p, double* pose, double* point);
int orc_optimize(orc_problem* p, int iterations, g2oc_iteration_stats* stats, int* done);
int orc_chi2(orc_problem* p, double* chi2, double* robust_chi2);
int orc_errors(orc_problem* p, double* errors);
int orc_jacobians(orc_problem* p, double* jac0, double* jac1);
/* central differences with delta 1e-9 through oplus, the reference's
   BaseFixedSizedEdge::linearizeOplusN (g2o/core/base_fixed_sized_edge.hpp:152-194) */
int orc_numeric_jacobians(orc_problem* p, double* jac0, double* jac1);
int orc_build_system(orc_problem* p);
int orc_get_pattern(orc_problem* p, int32_t* hpp_rc, int32_t* hpl_rc, int32_t* schur_rc);
int orc_get_hessian(orc_problem* p, double* hpp, double* hll, double* hpl, double* b);
int orc_schur(orc_problem* p, double lambda, double* schur_blocks, double* bschur);
int orc_solve(orc_problem* p, double lambda, double* x, int32_t* pcg_iterations);
/* SparseOptimizer::update(x): oplus of every free vertex by its part of x (Hessian order) */
int orc_update(orc_problem* p, const double* x);
int orc_solve_block_system(int32_t linear_solver, const g2oc_params* params, int32_t num_block_rows,
                           const int32_t* block_offsets, int32_t nnzb, const int32_t* block_rc,
                           const double* values, const double* b, double* x, int32_t* iterations);

/* building blocks exposed for the unit tests */
void orc_huber(double e2, double delta, double* rho3);
void orc_compute_dq_dR(const double* R_rowmajor, double* dq_dR_3x9_colmajor_index);
void orc_rot_to_quat(const double* R_rowmajor, double* q_xyzw);
void orc_se3quat_exp(const double* update6, double* se3quat7);
double orc_normalize_theta(double theta);

#ifdef __cplusplus
}
#endif
#endif
