"""The BAL path: VertexCameraBAL (angle-axis, translation, focal length, k1,
k2; additive update), VertexPointBAL and EdgeObservationBAL under
BlockSolver<9,3> with block-Jacobi PCG or a Cholesky
(g2o/examples/bal/bal_example.cpp:67-250).

CPU (the oracle's restatement):
* the prediction against the reference's formula written out here in plain
  Python (bal_example.cpp:160-200) on hand-picked cameras, the first-order
  branch at |w| == 0 included, and the error's sign (prediction - measurement);
* the oracle's forward-mode Jacobians against central differences;
* the oracle's LM with PCG and with its Cholesky reaching the same chi2.

GPU, through the C-ABI, against the oracle on a seeded 40-camera / 3,000-point
BAL problem: errors and Jacobians 1e-12 / 1e-10 relative, Hessian blocks,
gradient and Schur complement 1e-10 per block, 10-iteration LM trajectories
with PCG and with Cholesky and Gauss-Newton and Dogleg trajectories (same
trials, chi2 within 1e-6); at the full size (356 cameras, 226,730 points,
~1.27M observations) the 10-iteration LM + PCG trajectory against the
oracle's, committed in tests/golden/oracle_targets.json (same trials, chi2
within 1e-6 per iteration). Mixed precision, the structure-only solver, the
adjoint and the batched windows are built for SE3 cameras and refuse BAL.
"""
import math

import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import (ALGO_DOGLEG, ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, EDGE_BAL_OBSERVATION, LINEAR_CHOLESKY,
                          LINEAR_PCG, POSE_BAL_CAMERA, PREC_MIXED, Graph)


def reference_prediction(cam, X):
    """EdgeObservationBAL::operator() as written in bal_example.cpp:160-200."""
    w = cam[:3]
    theta = math.sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2])
    if theta > 0:
        v = [w[i] / theta for i in range(3)]
        cth, sth = math.cos(theta), math.sin(theta)
        vxp = [v[1] * X[2] - v[2] * X[1], v[2] * X[0] - v[0] * X[2], v[0] * X[1] - v[1] * X[0]]
        vdp = v[0] * X[0] + v[1] * X[1] + v[2] * X[2]
        p = [X[i] * cth + vxp[i] * sth + v[i] * vdp * (1 - cth) for i in range(3)]
    else:
        p = [X[0] + (w[1] * X[2] - w[2] * X[1]), X[1] + (w[2] * X[0] - w[0] * X[2]),
             X[2] + (w[0] * X[1] - w[1] * X[0])]
    p = [p[i] + cam[3 + i] for i in range(3)]
    q = [-p[0] / p[2], -p[1] / p[2]]
    r2 = q[0] * q[0] + q[1] * q[1]
    rp = 1 + cam[7] * r2 + cam[8] * r2 * r2
    return np.array([cam[6] * rp * q[0], cam[6] * rp * q[1]])


CASES = [
    # camera (w, t, f, k1, k2), point
    ([0.0, 0.0, 0.0, 0.1, -0.2, -5.0, 500.0, 0.0, 0.0], [0.3, 0.4, 1.0]),
    ([0.0, 0.0, 0.0, 0.0, 0.0, -4.0, 800.0, -0.05, 0.01], [1.0, -0.5, 0.5]),
    ([0.0, 0.0, math.pi / 2, 0.2, 0.1, -6.0, 450.0, 0.02, -0.003], [0.5, 1.5, -0.7]),
    ([0.3, -1.2, 0.8, -0.4, 0.7, -8.0, 620.0, -0.08, 0.02], [2.0, -1.0, 1.5]),
    ([1e-9, 2e-9, -1e-9, 0.0, 0.0, -3.0, 500.0, 0.0, 0.0], [0.1, 0.2, 0.3]),
]


def one_edge_graph(cam, X, z=(0.0, 0.0)):
    return Graph(POSE_BAL_CAMERA, EDGE_BAL_OBSERVATION, np.array([cam]), np.array([[0, 0]]), np.array([z]),
                 np.eye(2).reshape(1, 4), point_estimate=np.array([X]))


def test_oracle_prediction_known_answers(oracle_lib):
    for cam, X in CASES:
        z = (12.5, -3.25)
        o = oracle_lib.OracleProblem(one_edge_graph(cam, X, z))
        e = o.errors()[0]
        want = reference_prediction(cam, X) - np.array(z)  # error = prediction - measurement
        np.testing.assert_allclose(e, want, rtol=1e-13, atol=1e-12)


def test_oracle_jacobians_match_central_differences(oracle_lib):
    for cam, X in CASES:
        o = oracle_lib.OracleProblem(one_edge_graph(cam, X))
        jp, jc = o.jacobians()
        h = 1e-6
        num_c = np.zeros((2, 9))
        for k in range(9):
            a, b = list(cam), list(cam)
            a[k] += h * max(1.0, abs(cam[k]))
            b[k] -= h * max(1.0, abs(cam[k]))
            num_c[:, k] = (reference_prediction(a, X) - reference_prediction(b, X)) / (a[k] - b[k])
        num_p = np.zeros((2, 3))
        for k in range(3):
            a, b = list(X), list(X)
            a[k] += h
            b[k] -= h
            num_p[:, k] = (reference_prediction(cam, a) - reference_prediction(cam, b)) / (2 * h)
        np.testing.assert_allclose(jc[0], num_c, rtol=2e-6, atol=1e-5 * np.abs(num_c).max())
        np.testing.assert_allclose(jp[0], num_p, rtol=2e-6, atol=1e-5 * np.abs(num_p).max())


@pytest.fixture(scope="module")
def graph():
    g = synth.bal_problem(num_cameras=40, num_points=3000)
    assert g.edge_type == EDGE_BAL_OBSERVATION and g.pose_type == POSE_BAL_CAMERA
    return g


def test_generator_noise_model(oracle_lib, graph):
    """At the generating estimates the residuals are the 1 px pixel noise."""
    t = graph.copy()
    t.pose_estimate = graph.extra["truth_pose"]
    t.point_estimate = graph.extra["truth_point"]
    chi2, _ = oracle_lib.OracleProblem(t).chi2()
    assert abs(chi2 / (2 * graph.num_edges) - 1.0) < 0.05


def test_oracle_pcg_and_cholesky_agree(oracle_lib, graph):
    out = []
    for ls in (LINEAR_PCG, LINEAR_CHOLESKY):
        o = oracle_lib.OracleProblem(graph, oracle_lib.default_params(algorithm=ALGO_LEVENBERG, linear_solver=ls),
                                     threads=4)
        _, st = o.optimize(10)
        out.append([s["chi2"] for s in st])
    assert all(b < a for a, b in zip(out[0], out[0][1:]))
    assert abs(out[0][-1] - out[1][-1]) <= 1e-6 * out[1][-1]


# ---------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


def rel_block_err(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.gpu
def test_bal_errors_jacobians_hessian_schur(backend, oracle_lib, graph):
    o = oracle_lib.OracleProblem(graph, oracle_lib.default_params())
    c = backend.CudaProblem(graph, backend.OptimizationAlgorithmFactory.instance().construct("lm_cuda_pcg9_3"))
    assert c.errors().shape == (graph.num_edges, 2)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    (j0c, j1c), (j0o, j1o) = c.jacobians(), o.jacobians()
    assert j0c.shape[1:] == (2, 3) and j1c.shape[1:] == (2, 9)
    assert rel_block_err(j0c, j0o) < 1e-10 and rel_block_err(j1c, j1o) < 1e-10
    (a, b), (x, y) = c.chi2(), o.chi2()
    assert abs(a - x) <= 1e-12 * x and abs(b - y) <= 1e-12 * y
    o.build_system()
    c.build_system()
    hc, ho = c.hessian(), o.hessian()
    assert hc[0].shape[1:] == (9, 9) and hc[2].shape[1:] == (9, 3)
    for u, v in zip(hc[:3], ho[:3]):
        assert rel_block_err(u, v) < 1e-10
    n = o.info.num_free_poses * 9
    assert rel_block_err(hc[3][:n].reshape(-1, 9), ho[3][:n].reshape(-1, 9)) < 1e-10
    assert relnorm(hc[3][n:], ho[3][n:]) < 1e-10
    for lam in (1e-3, 10.0):
        Sc, bsc = c.schur(lam)
        So, bso = o.schur(lam)
        assert rel_block_err(Sc, So) < 1e-10 and relnorm(bsc, bso) < 1e-10
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("algo,linear", [(ALGO_LEVENBERG, LINEAR_PCG), (ALGO_LEVENBERG, LINEAR_CHOLESKY),
                                         (ALGO_GAUSS_NEWTON, LINEAR_PCG), (ALGO_DOGLEG, LINEAR_PCG)])
def test_bal_trajectory(backend, oracle_lib, graph, algo, linear):
    prm = {"algorithm": algo, "linear_solver": linear}
    if algo == ALGO_DOGLEG:
        prm.update(max_trials_after_failure=100, initial_lambda=1e-7)
    o = oracle_lib.OracleProblem(graph, oracle_lib.default_params(**prm), threads=4)
    c = backend.CudaProblem(graph, backend.default_params(**prm))
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    assert do == dc
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], (a["iteration"], a, b)
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["iteration"], a["chi2"], b["chi2"])
    po, qo = o.estimates()
    pc, qc = c.estimates()
    c.close()
    # the cameras' rotation and translation (the focal length and distortion
    # are weakly determined along the gauge directions of the problem)
    assert np.abs(pc[:, :6] - po[:, :6]).max() < 1e-4


@pytest.mark.gpu
def test_bal_full_size_matches_oracle_trajectory(backend):
    from tests.golden.make_oracle_targets import load
    t = load()["bal"]
    g = synth.bal_problem()
    assert g.digest() == t["digest"]
    c = backend.CudaProblem(g, backend.OptimizationAlgorithmFactory.instance().construct("lm_cuda_pcg9_3"))
    done, st = c.optimize(t["iterations"])
    c.close()
    assert done == t["done"]
    for s, chi2, trials in zip(st, t["chi2"], t["levenberg_iterations"]):
        assert s["levenberg_iterations"] == trials, (s["iteration"], s, trials)
        assert abs(s["chi2"] - chi2) <= 1e-6 * chi2, (s["iteration"], s["chi2"], chi2)


@pytest.mark.gpu
def test_bal_refused_where_unsupported(backend, graph):
    with pytest.raises(backend.G2ocError) as e:
        backend.CudaProblem(graph, backend.default_params(precision=PREC_MIXED))
    assert e.value.status == 10
    c = backend.CudaProblem(graph, backend.default_params())
    with pytest.raises(backend.G2ocError) as e:
        c.structure_only(1, 5)
    assert e.value.status == 10
    with pytest.raises(backend.G2ocError) as e:
        c.backward(np.zeros((graph.num_poses, 9)), np.zeros((graph.num_points, 3)))
    assert e.value.status == 10
    c.close()
    with pytest.raises(backend.G2ocError):
        backend.CudaWindows([graph])


def test_bal_file_round_trip(tmp_path):
    """The BAL text format of bal_example.cpp:264-330: header, observations
    (camera, point, x, y), 9 parameters per camera, 3 per point."""
    from g2o_b200.bal import parse_bal, read_bal, write_bal
    text = """2 3 4
0 0 -10.5 3.25
1 0 2.0 -1.0
0 2 0.5 0.75
1 1 7.0 8.0
0.1 0.2 0.3 1 2 3 500 -0.1 0.01
-0.1 0.0 0.05 0 0 -1 480 0 0
1 2 3
4 5 6
7 8 9
"""
    g = parse_bal(text)
    assert (g.pose_type, g.edge_type, g.num_poses, g.num_points, g.num_edges) == (
        POSE_BAL_CAMERA, EDGE_BAL_OBSERVATION, 2, 3, 4)
    np.testing.assert_array_equal(g.edge_vertex, [[0, 0], [0, 1], [2, 0], [1, 1]])  # (point, camera)
    np.testing.assert_array_equal(g.measurement[0], [-10.5, 3.25])
    np.testing.assert_array_equal(g.pose_estimate[0], [0.1, 0.2, 0.3, 1, 2, 3, 500, -0.1, 0.01])
    np.testing.assert_array_equal(g.point_estimate[2], [7, 8, 9])
    np.testing.assert_array_equal(g.information, np.tile(np.eye(2).reshape(1, 4), (4, 1)))
    big = synth.bal_problem(num_cameras=12, num_points=500)
    p = tmp_path / "bal.txt"
    write_bal(big, str(p))
    back = read_bal(str(p))
    for a in ("pose_estimate", "edge_vertex", "measurement", "information", "point_estimate"):
        np.testing.assert_array_equal(getattr(back, a), getattr(big, a))
    with pytest.raises(ValueError):
        parse_bal("2 3 4\n0 5 1 1\n")
