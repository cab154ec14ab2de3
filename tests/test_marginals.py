"""Marginal covariances (g2oc_compute_marginals, g2oc_solve_pattern_block_system):
the selected inverse of the tiled FP64 Cholesky against g2o's golden 36x36
inverse (unit_test/solver/linear_solver_test.cpp:103-134, isApprox 1e-6 per
block) and against a dense FP64 inverse of the oracle's Hpp."""
import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, LINEAR_CHOLESKY, PREC_MIXED

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


def dense_hpp(rc, blocks, nb, bs):
    H = np.zeros((nb * bs, nb * bs))
    for (r, c), B in zip(rc, blocks):
        H[r * bs:(r + 1) * bs, c * bs:(c + 1) * bs] = B
        H[c * bs:(c + 1) * bs, r * bs:(r + 1) * bs] = B.T
    return H


def blocks_of(M, pairs, bs):
    return np.array([M[r * bs:(r + 1) * bs, c * bs:(c + 1) * bs] for r, c in pairs])


def test_golden_inverse_pattern(backend):
    from tests.test_oracle_pinning import is_approx, load_sparse_system
    offs, rc, vals, _, _, inv = load_sparse_system()
    nb = len(offs) - 1
    # the reference test's pattern: every diagonal block
    diag = [(i, i) for i in range(nb)]
    st, out = backend.solve_pattern_block_system(offs, rc, vals, diag)
    assert st == 0
    for (r, c), B in zip(diag, out):
        assert is_approx(B, inv[3 * r:3 * r + 3, 3 * c:3 * c + 3], 1e-6), (r, c)
    # every block, both triangles: the whole inverse
    allp = [(r, c) for r in range(nb) for c in range(nb)]
    st, out = backend.solve_pattern_block_system(offs, rc, vals, allp)
    assert st == 0
    full = np.zeros((3 * nb, 3 * nb))
    for (r, c), B in zip(allp, out):
        full[3 * r:3 * r + 3, 3 * c:3 * c + 3] = B
    assert np.abs(full - inv).max() <= 1e-9 * np.abs(inv).max()
    assert np.abs(full - full.T).max() <= 1e-12 * np.abs(inv).max()


def test_not_positive_definite_pattern(backend):
    offs = np.array([0, 3, 6], np.int32)
    rc = np.array([[0, 0], [0, 1], [1, 1]], np.int32)
    vals = np.concatenate([np.eye(3).ravel(), 2 * np.eye(3).ravel(), np.eye(3).ravel()])
    st, _ = backend.solve_pattern_block_system(offs, rc, vals, [(0, 0)])
    assert st == 4  # G2OC_ERR_NOT_PD


@pytest.mark.parametrize("kind", ["pg2d", "pg3d"])
def test_pose_graph_marginals_match_dense_inverse(backend, oracle_lib, kind):
    if kind == "pg2d":
        g = synth.pose_graph_2d(num_poses=500, num_closures=200, seed=41)
    else:
        g = synth.pose_graph_3d(num_rings=4, per_ring=60, radius=10.0, seed=42)
    prm = dict(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY)
    c = backend.CudaProblem(g, backend.default_params(**prm))
    c.optimize(5)
    pose, _ = c.estimates()
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    o.set_estimates(pose)
    o.build_system()
    hpp = o.hessian()[0]
    rc = o.pattern()[0]
    nb, bs = c.info.num_free_poses, c.info.pose_dim
    Hinv = np.linalg.inv(dense_hpp(rc, hpp, nb, bs))
    # g2o_cli's -computeMarginals pattern: (i, i) and (i-1, i), plus far pairs
    pairs = [(i, i) for i in range(nb)] + [(i - 1, i) for i in range(1, nb)] + [(0, nb - 1), (nb - 1, 3)]
    got = c.compute_marginals(pairs)
    want = blocks_of(Hinv, pairs, bs)
    scale = np.abs(Hinv).max()
    assert np.abs(got - want).max() <= 1e-8 * scale
    c.close()


def test_bundle_adjustment_marginals_are_the_camera_blocks(backend, oracle_lib):
    """BlockSolver::computeMarginals passes Hpp: for bundle adjustment the
    (block-diagonal) camera part, not the Schur complement."""
    g = synth.bundle_adjustment(num_cameras=30, num_points=2000, seed=43)
    c = backend.CudaProblem(g, backend.default_params(algorithm=ALGO_LEVENBERG))
    c.optimize(3)
    pose, point = c.estimates()
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params())
    o.set_estimates(pose, point)
    o.build_system()
    hpp = o.hessian()[0]
    nb = c.info.num_free_poses
    pairs = [(i, i) for i in range(nb)] + [(i - 1, i) for i in range(1, nb)]
    got = c.compute_marginals(pairs)
    for k, (r, cc) in enumerate(pairs):
        want = np.linalg.inv(hpp[r]) if r == cc else np.zeros((6, 6))
        assert np.abs(got[k] - want).max() <= 1e-9 * np.abs(np.linalg.inv(hpp[cc])).max(), (r, cc)
    c.close()
    # mixed precision: H in FP32, inverse in FP64
    m = backend.CudaProblem(g, backend.default_params(precision=PREC_MIXED))
    m.set_estimates(pose, point)
    gm = m.compute_marginals([(0, 0)])
    assert np.abs(gm[0] - np.linalg.inv(hpp[0])).max() <= 1e-4 * np.abs(np.linalg.inv(hpp[0])).max()
    m.close()


def test_gauge_free_pose_graph_is_not_positive_definite(backend):
    g = synth.pose_graph_2d(num_poses=50, num_closures=10, seed=44)
    g.pose_fixed[:] = 0
    c = backend.CudaProblem(g, backend.default_params(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY))
    with pytest.raises(backend.G2ocError) as e:
        c.compute_marginals([(0, 0)])
    assert e.value.status == 4
    with pytest.raises(backend.G2ocError):
        c.compute_marginals([(0, 10**6)])
    c.close()
