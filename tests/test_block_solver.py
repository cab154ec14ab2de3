"""BlockSolverCuda: the device behind g2o's Solver interface
(g2o/core/solver.h:44-153, g2o/core/block_solver.h:96-149), for an
OptimizationAlgorithm that drives the iteration itself.

The algorithms here are OptimizationAlgorithmLevenberg::solve
(g2o/core/optimization_algorithm_levenberg.cpp:60-176) and
OptimizationAlgorithmGaussNewton::solve
(g2o/core/optimization_algorithm_gauss_newton.cpp:48-93), restated in the test
harness. They call only the Solver methods (init, buildStructure,
buildSystem, setLambda, solve, restoreDiagonal, b, x); the host graph (vertex
update, errors, push / pop) is the oracle's, in the role of g2o's own
SparseOptimizer. Checked per call against the oracle's BlockSolver and, for
the whole run, against the oracle's optimize() of the same graph:
* buildSystem: H and b per block within 1e-10 relative;
* setLambda + solve + restoreDiagonal: x within 1e-6 (PCG) / 1e-9
  (Cholesky); a solve after restoreDiagonal is the undamped solve;
* multiplyHessian: Hpp src;
* LM over BlockSolverCuda: the same LM trials per iteration and chi2 within
  1e-6 per iteration; Gauss-Newton within 1e-8.
"""
import math

import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import ALGO_GAUSS_NEWTON, LINEAR_CHOLESKY



@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


def relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_block_err(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def lambda_init(solver, tau):
    """computeLambdaInit (optimization_algorithm_levenberg.cpp:155-167): tau
    times the largest diagonal entry of the free vertices' Hessian blocks."""
    hpp_rc = solver.pattern()[0]
    hpp, hll, _, _ = solver.hessian()
    m = 0.0
    for k, (r, c) in enumerate(hpp_rc):
        if r == c:
            m = max(m, float(np.abs(np.diag(hpp[k])).max()))
    if len(hll):
        m = max(m, float(np.abs(np.diagonal(hll, axis1=1, axis2=2)).max()))
    return tau * m


def levenberg_over_solver(solver, host, iterations, tau=1e-5, max_trials=10):
    """OptimizationAlgorithmLevenberg::solve (optimization_algorithm_levenberg.cpp:60-153)
    over a Solver, one entry per outer iteration: (trials, robust chi2)."""
    solver.init(host.graph)
    solver.build_structure()
    out = []
    lam = ni = None
    for it in range(iterations):
        current = host.chi2()[1]
        solver.build_system(*host.estimates())
        if it == 0:
            lam, ni = lambda_init(solver, tau), 2.0
        b = solver.b()
        trials = 0
        rho = 0.0
        while True:
            backup = host.estimates()                    # push
            solver.set_lambda(lam, backup=True)
            ok = solver.solve()
            x = solver.x()
            host.update(x)
            solver.restore_diagonal()
            temp = host.chi2()[1] if ok else float("inf")
            rho = current - temp
            scale = float(x @ (lam * x + b)) + 1e-3 if ok else 1.0   # computeScale + 1e-3
            rho /= scale
            trials += 1
            if rho > 0 and math.isfinite(temp) and ok:
                alpha = min(1.0 - (2 * rho - 1) ** 3, 2.0 / 3.0)
                lam *= max(1.0 / 3.0, alpha)
                ni = 2.0
                current = temp
            else:
                lam *= ni
                ni *= 2
                host.set_estimates(*backup)                # pop
                if not math.isfinite(lam):
                    break
            if not (rho < 0 and trials < max_trials):
                break
        out.append((trials, host.chi2()[1]))
        if trials == max_trials or rho == 0 or not math.isfinite(lam):
            break
    return out


def gauss_newton_over_solver(solver, host, iterations):
    """OptimizationAlgorithmGaussNewton::solve (optimization_algorithm_gauss_newton.cpp:48-93)."""
    solver.init(host.graph)
    solver.build_structure()
    out = []
    for _ in range(iterations):
        solver.build_system(*host.estimates())
        assert solver.solve()
        host.update(solver.x())
        out.append(host.chi2()[1])
    return out


class OracleSolver:
    """The Solver calls on the oracle's own BlockSolver: pins the restated
    algorithms above on the CPU (they must reproduce the oracle's optimize()
    exactly when the solver is the oracle's)."""

    def __init__(self, g, **prm):
        self.o = type(self).oracle.OracleProblem(g, type(self).oracle.default_params(**prm))
        self.lam = 0.0

    def init(self, g, online=False):
        return True

    def build_structure(self, zero_blocks=False):
        return True

    def build_system(self, pose, point):
        self.o.set_estimates(pose, point)
        self.o.build_system()
        self._b = self.o.hessian()[3]
        return True

    def set_lambda(self, lam, backup=False):
        self.lam = lam
        return True

    def solve(self):
        st, self._x, _ = self.o.solve(self.lam)
        return st == 0

    def restore_diagonal(self):
        self.lam = 0.0

    def x(self):
        return self._x

    def b(self):
        return self._b

    def hessian(self):
        return self.o.hessian()

    def pattern(self):
        return self.o.pattern()


def test_restated_algorithms_reproduce_oracle_on_cpu(oracle_lib):
    OracleSolver.oracle = oracle_lib
    g = synth.bundle_adjustment(num_cameras=12, num_points=500, seed=7)
    ref = oracle_lib.OracleProblem(g)
    _, so = ref.optimize(8)
    run = levenberg_over_solver(OracleSolver(g), oracle_lib.OracleProblem(g), 8)
    assert [(s["levenberg_iterations"], s["chi2"]) for s in so] == run
    prm = dict(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY)
    p = synth.pose_graph_2d(num_poses=200, num_closures=60, seed=5)
    ref = oracle_lib.OracleProblem(p, oracle_lib.default_params(**prm))
    _, so = ref.optimize(4)
    run = gauss_newton_over_solver(OracleSolver(p, **prm), oracle_lib.OracleProblem(p, oracle_lib.default_params(**prm)),
                                   4)
    assert [s["chi2"] for s in so] == run


@pytest.mark.gpu
def test_block_solver_calls_match_oracle(backend, oracle_lib):
    g = synth.bundle_adjustment(num_cameras=30, num_points=2000, seed=17)
    o = oracle_lib.OracleProblem(g)
    solver = backend.BlockSolverCuda(backend.LinearSolverCudaPCG())
    assert solver.init(g) and solver.build_structure()
    assert solver.supports_schur() and solver.schur()
    assert not solver.update_structure([], [])
    o.build_system()
    assert solver.build_system(*o.estimates())
    for a, b in zip(solver.hessian(), o.hessian()):
        if a.ndim > 1:
            assert rel_block_err(a, b) < 1e-10
        else:
            assert relnorm(a, b) < 1e-10
    assert relnorm(solver.b(), o.hessian()[3]) < 1e-10
    # damped solve, then restoreDiagonal: the next solve is the undamped one
    for lam in (1e-2, 0.0):   # both carry the PCG residual from the first solve to the second
        assert solver.set_lambda(lam, backup=True)
        assert solver.solve()
        solver.restore_diagonal()
        st, xo, _ = o.solve(lam)
        assert st == 0
        assert relnorm(solver.x(), xo) < 1e-6, (lam, relnorm(solver.x(), xo))
    # multiplyHessian: the pose part, Hpp src
    hpp_rc = solver.pattern()[0]
    hpp = o.hessian()[0]
    pd = 6
    ncam = o.info.num_free_poses
    src = np.random.default_rng(1).normal(size=ncam * pd)
    want = np.zeros_like(src)
    for k, (r, c) in enumerate(hpp_rc):
        want[r * pd:(r + 1) * pd] += hpp[k] @ src[c * pd:(c + 1) * pd]
        if r != c:
            want[c * pd:(c + 1) * pd] += hpp[k].T @ src[r * pd:(r + 1) * pd]
    assert relnorm(solver.multiply_hessian(src), want) < 1e-12
    solver.close()


@pytest.mark.gpu
def test_levenberg_over_block_solver_cuda_matches_oracle(backend, oracle_lib):
    g = synth.bundle_adjustment(num_cameras=40, num_points=3000, seed=7)
    ref = oracle_lib.OracleProblem(g)
    _, so = ref.optimize(15)
    host = oracle_lib.OracleProblem(g)
    solver = backend.BlockSolverCuda(backend.LinearSolverCudaPCG())
    run = levenberg_over_solver(solver, host, 15)
    solver.close()
    assert len(run) == len(so)
    for (trials, chi2), s in zip(run, so):
        assert trials == s["levenberg_iterations"], (s["iteration"], trials, s["levenberg_iterations"])
        assert abs(chi2 - s["chi2"]) <= 1e-6 * s["chi2"], (s["iteration"], chi2, s["chi2"])


@pytest.mark.gpu
def test_gauss_newton_over_block_solver_cuda_cholesky(backend, oracle_lib):
    g = synth.pose_graph_2d(num_poses=800, num_closures=300, seed=5)
    prm = dict(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY)
    ref = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    _, so = ref.optimize(6)
    host = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    solver = backend.BlockSolverCuda(backend.LinearSolverCudaCholesky(), algorithm=ALGO_GAUSS_NEWTON)
    run = gauss_newton_over_solver(solver, host, 6)
    solver.close()
    for chi2, s in zip(run, so):
        assert abs(chi2 - s["chi2"]) <= 1e-8 * s["chi2"], (s["iteration"], chi2, s["chi2"])


@pytest.mark.gpu
def test_linear_solver_cuda_solves_reference_fixture(backend):
    # LinearSolver<MatrixType>::solve(A, x, b) on the reference's 36x36 block
    # system (unit_test/solver/linear_solver_test.cpp:84-101), both solvers
    from tests.test_oracle_pinning import is_approx, load_sparse_system
    offs, rc, vals, b, x_ref, _ = load_sparse_system()
    for ls in (backend.LinearSolverCudaCholesky(), backend.LinearSolverCudaPCG(tolerance=1e-20, max_iterations=200)):
        for _ in range(2):
            ok, x = ls.solve(offs, rc, vals, b)
            assert ok and is_approx(x, x_ref, 1e-6), type(ls).__name__
