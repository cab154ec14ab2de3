"""Pin the oracle (FP64 CPU restatement) against the reference's own tests.

Each test restates one of g2o's unit tests on the oracle:
* the 36x36 block system of unit_test/solver/sparse_system_helper.cpp solved
  twice within isApprox(1e-6) (unit_test/solver/linear_solver_test.cpp:84-101),
  fixture extracted by tests/golden/make_fixtures.py;
* analytic vs central-difference Jacobians, 1e-6
  (unit_test/slam2d/jacobians_slam2d.cpp:42-66,
   unit_test/slam3d/jacobians_slam3d.cpp:43-67, evaluate_jacobian.h:64-95);
* dq/dR vs an independent derivative, 1e-7 (jacobians_slam3d.cpp:201-233);
* Huber rho' and rho'' vs numeric derivatives, 1e-5 / 1e-3
  (unit_test/general/robust_kernel_tests.cpp:72-161);
* two-pose EdgeSE3 problems converge under GN and LM: chi2 < 1e-6, pose
  within 1e-3 (unit_test/slam3d/optimization_slam3d.cpp:62-148).
"""
import json
import math
import os

import numpy as np
import pytest

from g2o_b200.abi import (ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, EDGE_SE2, EDGE_SE3, LINEAR_CHOLESKY, LINEAR_PCG,
                          POSE_SE2, POSE_SE3, Graph)

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sparse_system_36.json")


def load_sparse_system():
    d = json.load(open(GOLDEN))
    offs = [0] + d["row_block_indices"]
    blocks = sorted(d["blocks"], key=lambda b: (b["col"], b["row"]))
    rc = np.array([[b["row"], b["col"]] for b in blocks], np.int32)
    vals = np.concatenate([b["values"] for b in blocks])
    return np.array(offs, np.int32), rc, vals, np.array(d["b"]), np.array(d["x"]), np.array(d["inverse"]).reshape(36, 36)


def is_approx(a, b, prec):
    return np.linalg.norm(a - b) <= prec * min(np.linalg.norm(a), np.linalg.norm(b))


def test_sparse_system_fixture_is_consistent():
    offs, rc, vals, b, x, inv = load_sparse_system()
    A = np.zeros((36, 36))
    k = 0
    for r, c in rc:
        M = vals[k:k + 9].reshape(3, 3)
        k += 9
        A[3 * r:3 * r + 3, 3 * c:3 * c + 3] = M
        A[3 * c:3 * c + 3, 3 * r:3 * r + 3] = M.T
    assert is_approx(np.linalg.solve(A, b), x, 1e-6)
    assert np.abs(np.linalg.inv(A) - inv).max() < 1e-9


def test_oracle_cholesky_solves_reference_system_twice(oracle_lib):
    offs, rc, vals, b, x, _ = load_sparse_system()
    for _ in range(2):
        st, sol, _ = oracle_lib.solve_block_system(LINEAR_CHOLESKY, offs, rc, vals, b)
        assert st == 0
        assert is_approx(sol, x, 1e-6)


def test_oracle_pcg_solves_reference_system(oracle_lib):
    offs, rc, vals, b, x, _ = load_sparse_system()
    prm = oracle_lib.default_params(pcg_tolerance=1e-20, pcg_max_iterations=200)
    st, sol, it = oracle_lib.solve_block_system(LINEAR_PCG, offs, rc, vals, b, prm)
    assert st == 0 and it > 0
    assert is_approx(sol, x, 1e-6)


def _random_se2(rng):
    return rng.uniform(-1, 1, 3)


def _random_iso(rng):
    # randomIsometry3 of unit_test/test_helper/random_state.h:33-40
    aa = rng.uniform(-1, 1, 3) + rng.uniform(-1, 1, 3)
    th = np.linalg.norm(aa)
    k = aa / th
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    R = np.eye(3) + math.sin(th) * K + (1 - math.cos(th)) * K @ K
    return np.concatenate([R.reshape(9), rng.uniform(-1, 1, 3)])


def _pair_graph(pose_type, edge_type, poses, meas, n_edges):
    ev = np.stack([np.arange(0, 2 * n_edges, 2), np.arange(1, 2 * n_edges, 2)], 1)
    D = 3 if edge_type == EDGE_SE2 else 6
    info = np.tile(np.eye(D).reshape(1, -1), (n_edges, 1))
    return Graph(pose_type, edge_type, np.array(poses), ev, np.array(meas), info)


def test_edge_se2_jacobian_matches_numeric(oracle_lib):
    rng = np.random.default_rng(1)
    n = 2000
    poses = [_random_se2(rng) for _ in range(2 * n)]
    meas = [_random_se2(rng) for _ in range(n)]
    p = oracle_lib.OracleProblem(_pair_graph(POSE_SE2, EDGE_SE2, poses, meas, n))
    a0, a1 = p.jacobians()
    n0, n1 = p.jacobians(numeric=True)
    assert np.abs(a0 - n0).max() < 1e-6
    assert np.abs(a1 - n1).max() < 1e-6


def test_edge_se3_jacobian_matches_numeric(oracle_lib):
    rng = np.random.default_rng(2)
    n = 2000
    poses = [_random_iso(rng) for _ in range(2 * n)]
    meas = [_random_iso(rng) for _ in range(n)]
    p = oracle_lib.OracleProblem(_pair_graph(POSE_SE3, EDGE_SE3, poses, meas, n))
    a0, a1 = p.jacobians()
    n0, n1 = p.jacobians(numeric=True)
    assert np.abs(a0 - n0).max() < 1e-6
    assert np.abs(a1 - n1).max() < 1e-6


def _compact_quat_branch(R, branch):
    """The reference's rotation-matrix -> (qx,qy,qz) functor of
    jacobians_slam3d.cpp:161-195 with the branch held fixed."""
    if branch < 0:
        t = math.sqrt(R[0, 0] + R[1, 1] + R[2, 2] + 1.0)
        t = 0.5 / t
        return np.array([(R[2, 1] - R[1, 2]) * t, (R[0, 2] - R[2, 0]) * t, (R[1, 0] - R[0, 1]) * t])
    i = branch
    j, k = (i + 1) % 3, (i + 2) % 3
    q = np.zeros(3)
    t = math.sqrt(R[i, i] - R[j, j] - R[k, k] + 1.0)
    q[i] = 0.5 * t
    t = 0.5 / t
    q[j] = (R[j, i] + R[i, j]) * t
    q[k] = (R[k, i] + R[i, k]) * t
    w = (R[k, j] - R[j, k]) * t
    return -q if w < 0 else q


def test_dq_dR_matches_derivative_of_reference_functor(oracle_lib):
    rng = np.random.default_rng(3)
    for _ in range(500):
        iso = _random_iso(rng)
        R = iso[:9].reshape(3, 3)
        tr = np.trace(R)
        if tr > 0:
            branch = -1
        else:
            branch = 0
            if R[1, 1] > R[0, 0]:
                branch = 1
            if R[2, 2] > R[branch, branch]:
                branch = 2
        if branch >= 0 and not (R[0, 0] > R[1, 1] and R[0, 0] > R[2, 2]) and branch == 0:
            continue  # tie region where the two reference branch rules differ
        D = oracle_lib.dq_dR(R)
        h = 1e-7
        num = np.zeros((3, 9))
        for c in range(3):
            for r in range(3):
                Rp, Rm = R.copy(), R.copy()
                Rp[r, c] += h
                Rm[r, c] -= h
                num[:, c * 3 + r] = (_compact_quat_branch(Rp, branch) - _compact_quat_branch(Rm, branch)) / (2 * h)
        assert np.abs(D - num).max() < 1e-7


@pytest.mark.parametrize("e_factor", ["sq", "lin", "out"])
def test_huber_derivatives(oracle_lib, e_factor):
    delta = 0.07
    e = {"sq": 0.99 * delta * delta, "lin": 0.99 * delta, "out": 1.5 * delta}[e_factor]

    def ev(v):
        return oracle_lib.huber(v, delta)[0]

    rho = oracle_lib.huber(e, delta)
    assert rho[0] != 0.0
    d = 1e-9
    assert abs(rho[1] - (ev(e + d) - ev(e - d)) / (2 * d)) < 1e-5
    k = 1e-5
    r1 = (2 * ev(e) - 5 * ev(e - k) + 4 * ev(e - 2 * k) - ev(e - 3 * k)) / (k * k)
    r2 = (2 * ev(e) - 5 * ev(e + k) + 4 * ev(e + 2 * k) - ev(e + 3 * k)) / (k * k)
    assert abs(rho[2] - 0.5 * (r1 + r2)) < 1e-3


def _two_pose_graph(second):
    ident = np.concatenate([np.eye(3).reshape(9), np.zeros(3)])
    return Graph(POSE_SE3, EDGE_SE3, np.stack([ident, second]), np.array([[0, 1]]), ident[None, :],
                 np.eye(6).reshape(1, 36), pose_fixed=np.array([1, 0], np.uint8))


def _axis_angle_iso(deg, axis):
    k = np.asarray(axis, float) / np.linalg.norm(axis)
    th = math.radians(deg)
    K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
    R = np.eye(3) + math.sin(th) * K + (1 - math.cos(th)) * K @ K
    return np.concatenate([R.reshape(9), np.zeros(3)])


@pytest.mark.parametrize("algo", [ALGO_GAUSS_NEWTON, ALGO_LEVENBERG])
@pytest.mark.parametrize("case", ["translation", "rotation"])
def test_two_pose_se3_converges(oracle_lib, algo, case):
    if case == "translation":
        second = np.concatenate([np.eye(3).reshape(9), [10.0, 10.0, 10.0]])
    else:
        second = _axis_angle_iso(2.0, [1, 1, 1])
    g = _two_pose_graph(second)
    p = oracle_lib.OracleProblem(g, oracle_lib.default_params(algorithm=algo, linear_solver=LINEAR_CHOLESKY))
    assert p.chi2()[0] > 0
    done, _ = p.optimize(100)
    assert done > 0
    assert p.chi2()[0] < 1e-6
    pose, _ = p.estimates()
    assert np.abs(pose[1, 9:]).max() < 1e-3
    assert np.abs(np.diag(pose[1, :9].reshape(3, 3)) - 1).max() < 1e-3


@pytest.mark.parametrize("focal_y", [None, 455.0])
def test_projection_jacobians_match_numeric(oracle_lib, focal_y):
    """EdgeProjectXYZ2UV (fx = fy) and EdgeSE3ProjectXYZ (fx != fy): the
    analytic Jacobians against central differences with g2o's step 1e-9
    (BaseFixedSizedEdge::linearizeOplus numeric form,
    g2o/core/base_fixed_sized_edge.hpp:161-193)."""
    from g2o_b200 import synth
    g = synth.bundle_adjustment(num_cameras=12, num_points=400, seed=17, focal_y=focal_y)
    p = oracle_lib.OracleProblem(g)
    a0, a1 = p.jacobians()
    n0, n1 = p.jacobians(numeric=True)
    for a, n in ((a0, n0), (a1, n1)):
        assert np.abs(a - n).max() <= 1e-5 * max(1.0, np.abs(a).max())
    # fx and fy act on their own rows: the v row scales with fy alone
    if focal_y is not None:
        g2 = g.copy()
        g2.focal_length_y = 500.0
        b0, b1 = oracle_lib.OracleProblem(g2).jacobians()
        np.testing.assert_allclose(a1[:, 0], b1[:, 0], rtol=1e-12)
        np.testing.assert_allclose(a1[:, 1], b1[:, 1] * (455.0 / 500.0), rtol=1e-12)


def test_stereo_projection_jacobians_match_numeric(oracle_lib):
    """EdgeStereoSE3ProjectXYZ (g2o/types/sba/edge_project_stereo_xyz.cpp:58-106):
    the analytic 3 x 3 and 3 x 6 Jacobians against central differences
    (step 1e-9, BaseFixedSizedEdge's numeric form); the right row differs
    from the left u row by the bf terms only."""
    from g2o_b200 import synth
    g = synth.stereo_bundle_adjustment(num_cameras=12, num_points=400, seed=17)
    p = oracle_lib.OracleProblem(g)
    a0, a1 = p.jacobians()
    n0, n1 = p.jacobians(numeric=True)
    assert a0.shape[1:] == (3, 3) and a1.shape[1:] == (3, 6)
    for a, n in ((a0, n0), (a1, n1)):
        assert np.abs(a - n).max() <= 1e-5 * max(1.0, np.abs(a).max())
    g2 = g.copy()
    g2.stereo_bf = 0.0
    b0, b1 = oracle_lib.OracleProblem(g2).jacobians()
    np.testing.assert_array_equal(b0[:, 2], b0[:, 0])
    np.testing.assert_array_equal(b1[:, 2, [2, 3]], b1[:, 0, [2, 3]])
    np.testing.assert_array_equal(a0[:, :2], b0[:, :2])
    np.testing.assert_array_equal(a1[:, :2], b1[:, :2])


def test_edge_se3_expmap_error_and_jacobians(oracle_lib):
    """EdgeSE3Expmap (g2o/types/sba/edge_se3_expmap.cpp:45-72): with T_i = I
    and C = I the error log(T_j^-1 C T_i) of T_j = exp(u)^-1 is u itself
    (SE3Quat::log inverts SE3Quat::exp, se3quat.h:165-230); g2o's analytic
    Jacobians (adjoints, without the left Jacobian of the log) match central
    differences to first order in the error."""
    from g2o_b200.abi import EDGE_SE3_EXPMAP, POSE_SE3EXPMAP
    rng = np.random.default_rng(7)
    n = 200
    us = rng.normal(0, 0.6, (n, 6))
    poses, meas = [], []
    for u in us:
        R = _rodrigues(u[:3])
        theta = np.linalg.norm(u[:3])
        K = _skew(u[:3])
        V = np.eye(3) + (1 - np.cos(theta)) / theta ** 2 * K + (theta - np.sin(theta)) / theta ** 3 * K @ K
        t = V @ u[3:]
        Rt = R.T  # T_j = exp(u)^-1 = (R^T, -R^T t)
        poses += [[0, 0, 0, 0, 0, 0, 1], list(-Rt @ t) + list(_quat_xyzw(Rt))]
        meas.append([0, 0, 0, 0, 0, 0, 1])
    g = Graph(POSE_SE3EXPMAP, EDGE_SE3_EXPMAP, np.array(poses), np.arange(2 * n).reshape(n, 2),
              np.array(meas, float), np.tile(np.eye(6).reshape(1, 36), (n, 1)))
    p = oracle_lib.OracleProblem(g)
    np.testing.assert_allclose(p.errors().reshape(n, 6), us, rtol=0, atol=1e-9)
    # near zero error the adjoints are the derivatives
    small = us * 1e-4
    poses2 = []
    for u in small:
        R = _rodrigues(u[:3])
        poses2 += [[0, 0, 0, 0, 0, 0, 1], list(-R.T @ u[3:]) + list(_quat_xyzw(R.T))]
    g2 = Graph(POSE_SE3EXPMAP, EDGE_SE3_EXPMAP, np.array(poses2), g.edge_vertex, g.measurement, g.information)
    p2 = oracle_lib.OracleProblem(g2)
    a0, a1 = p2.jacobians()
    n0, n1 = p2.jacobians(numeric=True)
    assert np.abs(a0 - n0).max() < 1e-3 and np.abs(a1 - n1).max() < 1e-3


def _skew(w):
    return np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])


def _rodrigues(w):
    th = np.linalg.norm(w)
    K = _skew(w)
    if th < 1e-12:
        return np.eye(3) + K
    return np.eye(3) + np.sin(th) / th * K + (1 - np.cos(th)) / th ** 2 * K @ K


def _quat_xyzw(R):
    w = 0.5 * np.sqrt(max(1.0 + R[0, 0] + R[1, 1] + R[2, 2], 0.0))
    x = 0.5 * np.sqrt(max(1.0 + R[0, 0] - R[1, 1] - R[2, 2], 0.0)) * np.sign(R[2, 1] - R[1, 2] or 1.0)
    y = 0.5 * np.sqrt(max(1.0 - R[0, 0] + R[1, 1] - R[2, 2], 0.0)) * np.sign(R[0, 2] - R[2, 0] or 1.0)
    z = 0.5 * np.sqrt(max(1.0 - R[0, 0] - R[1, 1] + R[2, 2], 0.0)) * np.sign(R[1, 0] - R[0, 1] or 1.0)
    q = np.array([x, y, z, w])
    return q / np.linalg.norm(q)
