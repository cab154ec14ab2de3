/*
 * g2o_cuda.h -- C-ABI of the B200 (sm_100a) solver backend.
 *
 * This is the drop-in boundary between g2o's host C++ (SparseOptimizer,
 * OptimizationAlgorithmFactory) and the device solver. Only plain pointers,
 * sizes and status codes cross it; no C++, Eigen or torch types.
 *
 * Each entry point names the g2o interface it replaces (paths are relative to
 * the g2o source tree):
 *
 *   g2oc_create / g2oc_destroy      OptimizationAlgorithmFactory::construct
 *                                   (g2o/core/optimization_algorithm_factory.cpp:74-84)
 *                                   and ~OptimizationAlgorithm
 *   g2oc_construct                  the creator's name parsing
 *                                   (g2o/solvers/pcg/solver_pcg.cpp:49-72)
 *   g2oc_upload                     SparseOptimizer::initializeOptimization +
 *                                   buildIndexMapping + BlockSolver::buildStructure
 *                                   (g2o/core/sparse_optimizer.cpp:175-287,
 *                                    g2o/core/block_solver.hpp:110-269)
 *   g2oc_optimize                   SparseOptimizer::optimize with
 *                                   OptimizationAlgorithm{Levenberg,GaussNewton}::solve
 *                                   (g2o/core/sparse_optimizer.cpp:393-455,
 *                                    g2o/core/optimization_algorithm_levenberg.cpp:60-153,
 *                                    g2o/core/optimization_algorithm_gauss_newton.cpp:48-93)
 *   g2oc_iterate                    OptimizationAlgorithm::solve(iteration, online)
 *   g2oc_chi2 / g2oc_errors         computeActiveErrors + activeChi2 / activeRobustChi2
 *                                   (g2o/core/sparse_optimizer.cpp:78-130)
 *   g2oc_jacobians                  Edge::linearizeOplus (per-edge Jacobians)
 *   g2oc_build_system               BlockSolver::buildSystem (g2o/core/block_solver.hpp:492-565)
 *   g2oc_get_pattern / g2oc_get_hessian   the Hpp/Hpl/Hll/Hschur block patterns and
 *                                   values (SparseBlockMatrix::blockCols order)
 *   g2oc_schur                      BlockSolver::setLambda + the Schur part of
 *                                   BlockSolver::solve (g2o/core/block_solver.hpp:331-448, 567-606)
 *   g2oc_solve                      setLambda + BlockSolver::solve + restoreDiagonal
 *   g2oc_solver_init                BlockSolver::init -> LinearSolver::init
 *                                   (g2o/core/block_solver.hpp:609-616)
 *   g2oc_multiply_hessian           BlockSolverBase::multiplyHessian (g2o/core/block_solver.h:96)
 *   g2oc_solve_block_system         LinearSolver<MatrixType>::solve(A, x, b)
 *                                   (g2o/core/linear_solver.h:64-65) on a caller block matrix
 *   g2oc_compute_marginals          SparseOptimizer::computeMarginals -> BlockSolver::computeMarginals
 *                                   -> LinearSolver::solvePattern on Hpp (g2o/core/sparse_optimizer.cpp:585-610,
 *                                    g2o/core/block_solver.hpp:478-490, g2o/core/linear_solver.h:78-90, 165-173)
 *   g2oc_solve_pattern_block_system LinearSolver::solvePattern(spinv, blockIndices, A) on a caller
 *                                   block matrix
 *   g2oc_download / g2oc_set_estimates   vertex estimate read-back / write
 *
 * Conventions
 *   - Every function returns G2OC_OK (0) or a positive G2OC_ERR_* code and
 *     never aborts the process. g2oc_last_error() gives a message.
 *   - All host buffers are owned by the caller. A context owns its device
 *     memory and one CUDA stream. A context is not thread-safe; use one per
 *     host thread.
 *   - Vertices are given in g2o id order: poses first (index 0..num_poses-1),
 *     then points. The Hessian order follows SparseOptimizer::buildIndexMapping:
 *     free non-marginalized vertices in that order, then marginalized ones;
 *     fixed vertices get no Hessian index.
 *   - Edges are given in insertion (internalId) order.
 *   - Block patterns are listed column-major over the upper triangle
 *     (column, then row), the order of SparseBlockMatrix::blockCols(); block
 *     values are dense row-major.
 */
#ifndef G2O_CUDA_H
#define G2O_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define G2OC_ABI_VERSION 5 /* 5: g2oc_graph's pose edges (EdgeSE3Expmap beside projection edges),
                             g2oc_hessian_info.num_active_pose_edges; 4: the BAL camera and
                             observation types; 3: g2oc_graph.stereo_bf (EdgeStereoSE3ProjectXYZ);
                             2: focal_length_y */

/* status codes */
#define G2OC_OK 0
#define G2OC_ERR_INVALID_ARGUMENT 1 /* null pointer, bad size, bad enum */
#define G2OC_ERR_BAD_GRAPH 2        /* unsupported types, index out of range, empty graph */
#define G2OC_ERR_CUDA 3             /* a CUDA runtime call failed */
#define G2OC_ERR_NOT_PD 4           /* Cholesky met a non-positive pivot */
#define G2OC_ERR_NAN 5              /* non-finite value in error, Hessian or update */
#define G2OC_ERR_STATE 6            /* call order violated (e.g. optimize before upload) */
#define G2OC_ERR_NO_DEVICE 7        /* no CUDA device or wrong architecture */
#define G2OC_ERR_UNKNOWN_SOLVER 8   /* g2oc_construct: name not registered */
#define G2OC_ERR_TIMEOUT 9          /* a bounded device-side wait gave up */
#define G2OC_ERR_NOT_SUPPORTED 10   /* combination not implemented */
#define G2OC_ERR_NOT_CONVERGED 11   /* an iterative refinement stopped above its tolerance */

/* vertex / edge types (g2o class names) */
#define G2OC_POSE_SE2 1        /* VertexSE2: estimate (x, y, theta) */
#define G2OC_POSE_SE3 2        /* VertexSE3: Isometry3, 12 doubles: R row-major (9) then t (3) */
#define G2OC_POSE_SE3EXPMAP 3  /* VertexSE3Expmap: SE3Quat::toVector (tx,ty,tz,qx,qy,qz,qw) */
#define G2OC_POSE_BAL_CAMERA 4 /* VertexCameraBAL (g2o/examples/bal/bal_example.cpp:67-93): 9 doubles
                                  (rx, ry, rz angle-axis, tx, ty, tz, f, k1, k2), additive update */

#define G2OC_EDGE_SE2 1            /* EdgeSE2(VertexSE2, VertexSE2), D=3, measurement (x,y,theta) */
#define G2OC_EDGE_SE3 2            /* EdgeSE3(VertexSE3, VertexSE3), D=6, measurement Isometry3 (12) */
#define G2OC_EDGE_PROJECT_XYZ2UV 3 /* EdgeProjectXYZ2UV(VertexPointXYZ, VertexSE3Expmap), D=2 */
#define G2OC_EDGE_SE3_EXPMAP 5 /* EdgeSE3Expmap(VertexSE3Expmap, VertexSE3Expmap), D=6, measurement
                                 SE3Quat (7, toVector: the edge's _measurement, not the file's inverse) */
#define G2OC_EDGE_SE3_PROJECT_XYZ 4 /* EdgeSE3ProjectXYZ(VertexPointXYZ, VertexSE3Expmap), D=2, with
                                     fx = focal_length, fy = focal_length_y, (cx, cy) = principal_point */
#define G2OC_EDGE_STEREO_SE3_PROJECT_XYZ 6 /* EdgeStereoSE3ProjectXYZ(VertexPointXYZ, VertexSE3Expmap), D=3,
                                            measurement (u_left, v_left, u_right); fx, fy, (cx, cy) as
                                            SE3_PROJECT_XYZ and bf = stereo_bf
                                            (g2o/types/sba/edge_project_stereo_xyz.h:38-77) */
#define G2OC_EDGE_BAL_OBSERVATION 7 /* EdgeObservationBAL(VertexCameraBAL, VertexPointBAL), D=2
                                       (g2o/examples/bal/bal_example.cpp:143-203): error = prediction -
                                       measurement with the radial-distortion pinhole model. As for every
                                       projection edge of this ABI, vertex0 is the point and vertex1 the
                                       camera (the reverse of the class's vertex order), and the Jacobians
                                       are j0 = d e / d point (2x3), j1 = d e / d camera (2x9). Points are
                                       the num_points array (VertexPointBAL: 3 doubles, additive). */

/* algorithm / linear solver / precision */
#define G2OC_ALGO_GAUSS_NEWTON 0
#define G2OC_ALGO_LEVENBERG 1
#define G2OC_ALGO_DOGLEG 2 /* OptimizationAlgorithmDogleg (g2o/core/optimization_algorithm_dogleg.cpp:62-180) */
#define G2OC_ALGO_STRUCTURE_ONLY 3 /* StructureOnlySolver<3> (g2o/solvers/structure_only/structure_only_solver.h:57-215):
                                     every iteration is calc(points, 1, max_trials_after_failure) */

#define G2OC_LINEAR_PCG 0      /* block-Jacobi PCG (LinearSolverPCG semantics) */
#define G2OC_LINEAR_CHOLESKY 1 /* dense Cholesky of the (reduced) system */

#define G2OC_PREC_FP64 0  /* every kernel in FP64 */
#define G2OC_PREC_MIXED 1 /* FP32 J/H/Schur/SpMV + FP64 refinement, FP64 chi2 and LM control */

/* SolverResult of OptimizationAlgorithm::solve (g2o/core/optimization_algorithm.h:48) */
#define G2OC_RESULT_OK 1
#define G2OC_RESULT_FAIL -1
#define G2OC_RESULT_TERMINATE 2

typedef struct g2oc_graph {
  int32_t pose_type;           /* G2OC_POSE_* */
  int32_t num_poses;
  const double* pose_estimate; /* num_poses * {3, 12, 7, 9} */
  const uint8_t* pose_fixed;   /* num_poses, may be NULL (none fixed) */
  int32_t num_points;          /* VertexPointXYZ count (0 for pose graphs) */
  const double* point_estimate;/* num_points * 3 */
  const uint8_t* point_fixed;  /* num_points, may be NULL */
  int32_t edge_type;           /* G2OC_EDGE_* */
  int32_t num_edges;
  const int32_t* edge_vertex;  /* num_edges * 2: (vertex0, vertex1). For
                                  the projection edges (PROJECT_XYZ2UV,
                                  SE3_PROJECT_XYZ, STEREO_SE3_PROJECT_XYZ,
                                  BAL_OBSERVATION) vertex0 is a point index and
                                  vertex1 a pose index; otherwise both are pose
                                  indices. */
  const double* measurement;   /* num_edges * {3, 12, 2} */
  const double* information;   /* num_edges * D*D, row-major, symmetric */
  const double* robust_delta;  /* num_edges Huber deltas; <= 0 or NULL: no kernel */
  double focal_length;         /* CameraParameters (PROJECT_XYZ2UV); fx of SE3_PROJECT_XYZ */
  double principal_point[2];
  double focal_length_y;       /* fy of SE3_PROJECT_XYZ and STEREO_SE3_PROJECT_XYZ; ignored otherwise */
  double stereo_bf;            /* EdgeStereoSE3ProjectXYZ::bf (baseline times fx); ignored otherwise */
  /* A second edge set, EdgeSE3Expmap between the VertexSE3Expmap cameras of
     a projection-edge graph (PROJECT_XYZ2UV, SE3_PROJECT_XYZ,
     STEREO_SE3_PROJECT_XYZ): BlockSolver assembles both kinds into one
     system (g2o/core/block_solver.hpp:492-565), e.g. odometry or loop
     constraints beside the observations of a visual SLAM back end. 0: none. */
  int32_t num_pose_edges;
  const int32_t* pose_edge_vertex;      /* num_pose_edges * 2 pose indices (vertex0, vertex1) */
  const double* pose_edge_measurement;  /* num_pose_edges * 7: the edge's _measurement as SE3Quat::toVector */
  const double* pose_edge_information;  /* num_pose_edges * 36, row-major, (omega, upsilon) order */
  const double* pose_edge_robust_delta; /* num_pose_edges Huber deltas; <= 0 or NULL: no kernel */
} g2oc_graph;

typedef struct g2oc_params {
  int32_t algorithm;                 /* G2OC_ALGO_* */
  int32_t linear_solver;             /* G2OC_LINEAR_* */
  int32_t precision;                 /* G2OC_PREC_* */
  int32_t pcg_max_iterations;        /* -1: system dimension (LinearSolverPCG::_maxIter) */
  double pcg_tolerance;              /* 1e-6 (LinearSolverPCG::_tolerance) */
  int32_t pcg_absolute_tolerance;    /* 1 (LinearSolverPCG::_absoluteTolerance) */
  int32_t max_trials_after_failure;  /* 10 ("maxTrialsAfterFailure" property) */
  double initial_lambda;             /* 0: tau * max diag(H) ("initialLambda" property) */
  double tau;                        /* 1e-5 */
  int32_t refine_max_iterations;     /* mixed precision: max FP64 refinement corrections per solve (default 2);
                                        -1: no FP64 residual check, the FP32-stored system's solution is the step */
  double refine_tolerance;           /* reserved (default 1e-10) */
  double initial_delta;              /* Dogleg "initialDelta": initial trust radius (1e4) */
  double lambda_factor;              /* Dogleg "lambdaFactor" (10); Dogleg's "initialLambda" is
                                        initial_lambda (the dl_* names set 1e-7, <= 0 means 1e-7) and
                                        its "maxTrialsAfterFailure" max_trials_after_failure (100) */
} g2oc_params;

/* one per outer iteration, the fields of G2OBatchStatistics (g2o/core/batch_stats.h:40-82) */
typedef struct g2oc_iteration_stats {
  int32_t iteration;
  int32_t result;                 /* G2OC_RESULT_* */
  int32_t levenberg_iterations;   /* trials in this iteration */
  int32_t iterations_linear_solver; /* PCG iterations, summed over trials */
  double chi2;                    /* activeRobustChi2 after the iteration */
  double lambda;                  /* current LM lambda after the iteration */
  double time_residuals;          /* seconds, device-timed */
  double time_quadratic_form;
  double time_schur_complement;
  double time_linear_solver;
  double time_update;
  double time_iteration;
  double trust_radius;            /* Dogleg: Delta after the iteration */
  int32_t dogleg_step;            /* Dogleg: last step, 0 undefined, 1 steepest descent, 2 Gauss-Newton, 3 dogleg */
} g2oc_iteration_stats;

typedef struct g2oc_hessian_info {
  int32_t num_free_poses;   /* Hpp block rows */
  int32_t num_free_points;  /* Hll block rows (marginalized) */
  int32_t pose_dim;         /* 3 or 6 */
  int32_t point_dim;        /* 3 or 0 */
  int32_t hpp_nnzb;         /* upper blocks incl. diagonal */
  int32_t hpl_nnzb;
  int32_t schur_nnzb;       /* upper blocks incl. diagonal, 0 without Schur */
  int32_t num_active_edges;
  int64_t vector_size;      /* Solver::vectorSize() */
  int64_t schur_pairs;      /* co-observing Hpl block pairs (a < b) summed into off-diagonal Schur blocks */
  int32_t num_active_pose_edges; /* active edges of the pose edge set (g2oc_graph.num_pose_edges) */
} g2oc_hessian_info;

/* per-kernel launch count and (when timing is on) summed CUDA-event time */
typedef struct g2oc_kernel_stat {
  char name[32];
  int64_t launches;
  double total_ms;
} g2oc_kernel_stat;

/* outcome of g2oc_backward */
typedef struct g2oc_backward_stats {
  int32_t refinement_steps;   /* Gauss-Newton solves applied to the exact-Hessian residual */
  int32_t pcg_iterations;     /* summed over those solves (0 with Cholesky) */
  double relative_residual;   /* |dL/dx - H v| / |dL/dx| at the end */
} g2oc_backward_stats;

typedef struct g2oc_ctx g2oc_ctx;

/* library */
int g2oc_abi_version(void);
const char* g2oc_last_error(void);
void g2oc_default_params(g2oc_params* params);
/* Registered names, ';'-separated, into buf (OptimizationAlgorithmFactory::listSolvers). */
int g2oc_list_solvers(char* buf, size_t buf_size);
/* Fill params from a registered name such as "lm_cuda" or "gn_cuda_pcg6_3".
   Unknown names return G2OC_ERR_UNKNOWN_SOLVER and leave params untouched
   (the factory returns nullptr for them). */
int g2oc_construct(const char* name, g2oc_params* params);

/* context */
int g2oc_create(int device, g2oc_ctx** out);
void g2oc_destroy(g2oc_ctx* ctx);
int g2oc_set_params(g2oc_ctx* ctx, const g2oc_params* params);
/* the context's CUDA stream (cudaStream_t), for callers that order their own
   work or CUDA events after the solver's */
int g2oc_get_stream(g2oc_ctx* ctx, void** stream);

/* graph */
int g2oc_upload(g2oc_ctx* ctx, const g2oc_graph* graph);
int g2oc_get_hessian_info(g2oc_ctx* ctx, g2oc_hessian_info* info);
int g2oc_set_estimates(g2oc_ctx* ctx, const double* pose_estimate, const double* point_estimate);
int g2oc_download(g2oc_ctx* ctx, double* pose_estimate, double* point_estimate);
/* restore the estimates given to g2oc_upload (device copy); the whole-graph
   counterpart of OptimizableGraph::push/pop (g2o/core/optimizable_graph.cpp) */
int g2oc_restore_initial_estimates(g2oc_ctx* ctx);

/* optimization: stats may be NULL, else iterations entries */
int g2oc_optimize(g2oc_ctx* ctx, int iterations, g2oc_iteration_stats* stats, int* iterations_done);
/* one outer iteration, OptimizationAlgorithm::solve(iteration, false): the
   per-call form an adapter uses when SparseOptimizer::optimize drives the
   loop. iteration == 0 starts a run (linear solver init, lambda init) as
   g2oc_optimize does; stats may be NULL; *result gets G2OC_RESULT_*. */
int g2oc_iterate(g2oc_ctx* ctx, int iteration, g2oc_iteration_stats* stats, int* result);

/* parity hooks at the current estimate */
int g2oc_chi2(g2oc_ctx* ctx, double* chi2, double* robust_chi2);
int g2oc_errors(g2oc_ctx* ctx, double* errors);                 /* num_active_edges * D */
int g2oc_jacobians(g2oc_ctx* ctx, double* jac0, double* jac1);  /* row-major D x dim(v0), D x dim(v1) */
int g2oc_build_system(g2oc_ctx* ctx);
int g2oc_get_pattern(g2oc_ctx* ctx, int32_t* hpp_rc, int32_t* hpl_rc, int32_t* schur_rc); /* pairs (row, col) */
int g2oc_get_hessian(g2oc_ctx* ctx, double* hpp, double* hll, double* hpl, double* b);
int g2oc_schur(g2oc_ctx* ctx, double lambda, double* schur_blocks, double* bschur);
int g2oc_solve(g2oc_ctx* ctx, double lambda, double* x, int32_t* pcg_iterations);
/* The Solver calls of a BlockSolverCuda adapter (g2o/core/solver.h:44-153,
   g2o/core/block_solver.h:96-149) map onto this ABI as: buildStructure ->
   g2oc_upload; buildSystem -> g2oc_set_estimates + g2oc_build_system;
   setLambda + solve + restoreDiagonal -> g2oc_solve(lambda) (lambda is added
   to a copy of the diagonal; the stored Hessian never changes, so nothing is
   left to restore); Solver::b() and saveHessian -> g2oc_get_hessian.
   BlockSolver::init -> LinearSolver::init (g2o/core/block_solver.hpp:609-616,
   g2o/solvers/pcg/linear_solver_pcg.h:54-59): forget the PCG residual that
   the next solve's stopping rule would carry over from the previous one. */
int g2oc_solver_init(g2oc_ctx* ctx);
/* BlockSolverBase::multiplyHessian(dest, src) (g2o/core/block_solver.h:96,
   _Hpp->multiplySymmetricUpperTriangle): dest = Hpp src, Hpp the pose part of
   the last g2oc_build_system; src and dest hold num_free_poses * pose_dim
   doubles in Hessian order. */
int g2oc_multiply_hessian(g2oc_ctx* ctx, const double* src, double* dest);
/* StructureOnlySolver<3>::calc(points, num_iters, num_max_trials) on every
   free landmark of a bundle adjustment, the cameras held fixed: each landmark
   runs its own Levenberg-Marquardt on its 3x3 system (one thread per
   landmark). G2OC_ERR_NOT_SUPPORTED for pose graphs. */
int g2oc_structure_only(g2oc_ctx* ctx, int32_t num_iters, int32_t num_max_trials);
/* Marginal covariances: blocks of Hpp^-1, Hpp the pose part of H built at the
   current estimates (no lambda; for bundle adjustment the camera blocks only,
   as BlockSolver::computeMarginals passes _Hpp). block_indices holds
   num_blocks pairs (row, col) of Hessian block indices (free poses in
   Hessian order, as vertex hessianIndex()); out gets num_blocks row-major
   pose_dim x pose_dim blocks. FP64 selected inversion of the tiled Cholesky
   factor; G2OC_ERR_NOT_PD when Hpp is not positive definite (a free gauge). */
int g2oc_compute_marginals(g2oc_ctx* ctx, int32_t num_blocks, const int32_t* block_indices, double* out);

/* instrumentation, the device-side counterpart of G2OBatchStatistics /
   ScopedTictoc (g2o/core/batch_stats.h:40-82, g2o/stuff/tictoc.h:59):
   enable (and reset) per-kernel launch counting with CUDA-event timing on the
   context's stream; read the per-kernel counts and times and the total count */
int g2oc_set_kernel_timing(g2oc_ctx* ctx, int enable);
int g2oc_get_kernel_stats(g2oc_ctx* ctx, g2oc_kernel_stat* out, int capacity, int* count, int64_t* total_launches);

/* Adjoint of the optimum (no counterpart in the reference, which has no
   differentiation): implicit-function-theorem gradients of a loss L(x*) on the
   current (converged) estimates x* with respect to each edge's measurement and
   the log of a scale on its information matrix (Omega_e -> exp(s_e) Omega_e,
   at s_e = 0). dL_dx is dL/dx in the vertices' update coordinates
   (VertexSE3Expmap: the 6-vector [omega, upsilon] of T <- exp(.) T; points: 3),
   in vertex order: num_poses * 6 values, then num_points * 3; entries of fixed
   or inactive vertices are ignored. With F = 1/2 sum_e rho(e^T Omega e) and
   G = grad F, one extra solve v = H^-1 dL/dx gives dL/dtheta = -(dG/dtheta)^T v.
   H is the exact Hessian of F: the context's Gauss-Newton Schur solve (its
   precision and linear solver) is refined in FP64 against Hessian-vector
   products taken as central differences of the FP64 gradient. Outputs, in
   edge order: dL_dmeas (num_edges * 2) and dL_dlogw (num_edges); inactive
   edges get 0. Bundle adjustment (EDGE_PROJECT_XYZ2UV) only;
   G2OC_ERR_NOT_SUPPORTED otherwise, G2OC_ERR_NOT_CONVERGED when the
   refinement stalls (the gradients are still written). The estimates are left
   unchanged. */
int g2oc_backward(g2oc_ctx* ctx, const double* dL_dx, double* dL_dmeas, double* dL_dlogw,
                  g2oc_backward_stats* stats);

/* ---- sharded bundle adjustment (one process per GPU)
 * Each rank uploads every camera and its own share of the points with their
 * edges; per LM trial the ranks sum their parts of the reduced camera system
 * (the Schur complement and its right-hand side, in the dense-tile layout),
 * of chi2 and of the gain-ratio scale through the caller's all-reduce, and
 * then take identical steps: the reduced solve is replicated, the landmark
 * back-substitution and updates stay local. The scheme of
 * BlockSolver::solve (g2o/core/block_solver.hpp:331-477) with the sum over
 * landmarks split across ranks; g2o has no distributed counterpart.
 * allreduce(user, device_ptr, count, dtype, op, stream) must combine count
 * elements at device_ptr across all ranks in place (G2OC_RED_SUM or
 * G2OC_RED_MAX; G2OC_DT_F32 or G2OC_DT_F64), ordered after the work already
 * on `stream` (the context's CUDA stream) and before the work enqueued on it
 * after the call returns; it returns 0 on success. Every rank calls it at
 * the same points in the same order. Call before g2oc_upload; supported for
 * the projection-edge graphs (EdgeProjectXYZ2UV, EdgeSE3ProjectXYZ,
 * EdgeStereoSE3ProjectXYZ) with at least 32 free cameras, the PCG linear
 * solver, FP64 or mixed precision without FP64 refinement
 * (refine_max_iterations = -1). A pose edge set (g2oc_graph.num_pose_edges)
 * belongs to rank 0's graph alone: its terms are added once, before the
 * ranks sum; another rank's upload with pose edges returns
 * G2OC_ERR_NOT_SUPPORTED. world = 1 switches it off. */
#define G2OC_RED_SUM 0
#define G2OC_RED_MAX 1
#define G2OC_DT_F32 0
#define G2OC_DT_F64 1
typedef int (*g2oc_allreduce_fn)(void* user, void* device_ptr, int64_t count, int32_t dtype, int32_t op, void* stream);
int g2oc_set_sharding(g2oc_ctx* ctx, int32_t rank, int32_t world, g2oc_allreduce_fn allreduce, void* user);

/* Batched windows (no counterpart in the reference, where each window would be
   its own SparseOptimizer): many independent bundle adjustments
   (VertexSE3Expmap + VertexPointXYZ + EdgeProjectXYZ2UV, same camera
   parameters, no fixed points) packed into one context and optimized together.
   Every window runs OptimizationAlgorithmLevenberg::solve on its own (own
   lambda, trials, Terminate rules; g2o/core/optimization_algorithm_levenberg.cpp:60-153)
   with its reduced camera system solved by a dense Cholesky
   (LinearSolverDense, g2o/solvers/dense/linear_solver_dense.h:57-105), while
   each kernel runs over all windows; one LM round is captured in a CUDA graph
   and replayed until every window has finished. The Hessian and Schur
   complement are formed in the context's precision; the Cholesky is FP64.
   g2oc_upload_windows replaces the context's graph; g2oc_optimize_windows
   writes one g2oc_window_stats per window; g2oc_download_window reads one
   window's estimates (its own vertex numbering). */
typedef struct g2oc_window_stats {
  int32_t iterations;        /* LM iterations completed */
  int32_t trials;            /* LM trials in all */
  int32_t result;            /* G2OC_RESULT_* of the last iteration */
  int32_t solve_ok;          /* the last dense factorization succeeded */
  int32_t cholesky_threads;  /* threads per window of the dense solve (autotuned) */
  int32_t rounds;            /* rounds the batch ran */
  double chi2_initial;       /* robust chi2 before the first iteration */
  double chi2;               /* robust chi2 at the end */
  double lambda;
} g2oc_window_stats;

int g2oc_upload_windows(g2oc_ctx* ctx, int32_t num_windows, const g2oc_graph* windows);
int g2oc_optimize_windows(g2oc_ctx* ctx, int32_t iterations, g2oc_window_stats* stats);
int g2oc_download_window(g2oc_ctx* ctx, int32_t window, double* pose, double* point);

/* LinearSolver::solve on a caller block matrix: symmetric, upper blocks given
   column-major as (row, col) block pairs with row-major dense values; block
   sizes from block_offsets (num_blocks + 1 entries, scalar offsets). x gets
   the solution; PCG uses the LinearSolverPCG defaults from params. */
int g2oc_solve_block_system(g2oc_ctx* ctx, int32_t linear_solver, int32_t num_block_rows,
                            const int32_t* block_offsets, int32_t nnzb, const int32_t* block_rc,
                            const double* values, const double* b, double* x,
                            int32_t* iterations);
/* LinearSolver::solvePattern on a caller block matrix given as for
   g2oc_solve_block_system: num_blocks pairs (row, col) of block indices in
   block_indices, the blocks of A^-1 into out (row-major, num_blocks * bs * bs). */
int g2oc_solve_pattern_block_system(g2oc_ctx* ctx, int32_t nb, const int32_t* block_offsets, int32_t nnzb,
                                    const int32_t* block_rc, const double* values, int32_t num_blocks,
                                    const int32_t* block_indices, double* out);

/* g2oc_solve_block_system_static: no counterpart in the reference. The
   block-Jacobi PCG solve of g2oc_solve_block_system (same kernels, same
   results) for callers that cannot allocate device memory, e.g. code running
   in a process whose GPU memory is capped or pre-partitioned, under a
   caller-owned allocator, or in a plugin that must not grow the device
   footprint. It allocates nothing: its device scratch is one file-scope
   array of G2OC_STATIC_SCRATCH_BYTES that every GPU loading this library
   holds until process exit, and its host scratch is file-scope too. Inputs
   and outputs are the caller's host arrays, as for g2oc_solve_block_system
   (uniform block size 3 or 6, upper blocks column-major). A system whose
   scratch exceeds the limit is rejected with G2OC_ERR_INVALID_ARGUMENT. The
   first call on a device looks up the array's device address (with that
   device current); make that first call before any CUDA stream capture.
   Calls share the scratch (later calls overwrite it; host callers are
   serialized by a mutex) and run on cudaStreamPerThread, returning after the
   result is copied back, or, on an error, after the work already queued has
   finished. The stopping rule always uses the absolute tolerance (g2o's
   default, LinearSolverPCG absoluteTolerance = true): the result equals
   g2oc_solve_block_system's under a context whose pcg_absolute_tolerance is
   1. The device is made current for the call and the caller's current
   device is restored before returning. */
#define G2OC_STATIC_SCRATCH_BYTES (16u << 20)
int g2oc_solve_block_system_static(int device, int32_t num_block_rows, int32_t block_size, int32_t nnzb,
                                   const int32_t* block_rc, const double* values, const double* b, double* x,
                                   double pcg_tolerance, int32_t pcg_max_iterations, int32_t* iterations);

#ifdef __cplusplus
}
#endif

#endif /* G2O_CUDA_H */
