"""EdgeStereoSE3ProjectXYZ (g2o/types/sba/edge_project_stereo_xyz.h:38-77,
edge_project_stereo_xyz.cpp:34-106; D = 3: left (u, v) and right u) against
the FP64 oracle on a seeded stereo ring (100 cameras, 20k points): errors and
Jacobians 1e-12 relative, Hessian blocks, gradient and Schur blocks 1e-10
per block, 20-iteration LM trajectories (same trials, chi2 within 1e-6) with
PCG and with Cholesky, and the mixed-precision forms reaching the oracle's
final chi2 within 1e-6. The structure-only solver, the adjoint and the
batched windows are built for the two-row edges and refuse the stereo edge.
"""
import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import ALGO_LEVENBERG, EDGE_STEREO_SE3_PROJECT_XYZ, LINEAR_CHOLESKY, PREC_MIXED

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


@pytest.fixture(scope="module")
def graph():
    g = synth.stereo_bundle_adjustment(num_cameras=60, num_points=8000, seed=91)
    assert g.edge_type == EDGE_STEREO_SE3_PROJECT_XYZ
    return g


def rel_block_err(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_stereo_errors_jacobians_hessian_schur(backend, oracle_lib, graph):
    o = oracle_lib.OracleProblem(graph, oracle_lib.default_params())
    c = backend.CudaProblem(graph, backend.default_params())
    assert c.errors().shape == (graph.num_edges, 3)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    (j0c, j1c), (j0o, j1o) = c.jacobians(), o.jacobians()
    assert j0c.shape[1:] == (3, 3) and j1c.shape[1:] == (3, 6)
    assert rel_block_err(j0c, j0o) < 1e-12 and rel_block_err(j1c, j1o) < 1e-12
    (a, b), (x, y) = c.chi2(), o.chi2()
    assert abs(a - x) <= 1e-12 * x and abs(b - y) <= 1e-12 * y
    o.build_system()
    c.build_system()
    hc, ho = c.hessian(), o.hessian()
    for u, v in zip(hc[:3], ho[:3]):
        assert rel_block_err(u, v) < 1e-10
    n = o.info.num_free_poses * 6
    assert rel_block_err(hc[3][:n].reshape(-1, 6), ho[3][:n].reshape(-1, 6)) < 1e-10
    assert relnorm(hc[3][n:], ho[3][n:]) < 1e-10
    Sc, bsc = c.schur(1e-3)
    So, bso = o.schur(1e-3)
    assert rel_block_err(Sc, So) < 1e-10 and relnorm(bsc, bso) < 1e-10
    c.close()


@pytest.mark.parametrize("linear", ["pcg", "cholesky"])
def test_stereo_lm_trajectory(backend, oracle_lib, graph, linear):
    prm = {} if linear == "pcg" else {"linear_solver": LINEAR_CHOLESKY}
    o = oracle_lib.OracleProblem(graph, oracle_lib.default_params(**prm))
    c = backend.CudaProblem(graph, backend.default_params(**prm))
    do, so = o.optimize(20)
    dc, sc = c.optimize(20)
    assert do == dc == 20
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], (a["iteration"], a, b)
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["iteration"], a["chi2"], b["chi2"])
    c.close()


@pytest.mark.parametrize("solver", ["lm_cuda_mixed", "lm_cuda_mixed_fast"])
def test_stereo_mixed_reaches_oracle_chi2(backend, oracle_lib, graph, solver):
    o = oracle_lib.OracleProblem(graph, oracle_lib.default_params())
    _, so = o.optimize(20)
    target = so[-1]["chi2"]
    m = backend.CudaProblem(graph, backend.OptimizationAlgorithmFactory.instance().construct(solver))
    _, sm = m.optimize(30)
    m.close()
    assert min(s["chi2"] for s in sm) <= target * (1 + 1e-6), (solver, min(s["chi2"] for s in sm), target)


def test_stereo_baseline_enters_the_right_row(backend, graph):
    """bf moves the right-image residual only: with bf changed the left rows
    of the errors stay and the right row moves by (bf' - bf) / z."""
    c = backend.CudaProblem(graph, backend.default_params())
    e0 = c.errors()
    g2 = graph.copy()
    g2.stereo_bf = graph.stereo_bf * 0.5
    c2 = backend.CudaProblem(g2, backend.default_params())
    e1 = c2.errors()
    np.testing.assert_array_equal(e0[:, :2], e1[:, :2])
    assert np.all(e1[:, 2] < e0[:, 2])  # u_r = u - bf / z grows when bf shrinks: the residual drops
    c.close()
    c2.close()


def test_stereo_refused_where_unsupported(backend, graph):
    c = backend.CudaProblem(graph, backend.default_params())
    with pytest.raises(backend.G2ocError) as e:
        c.structure_only(1, 5)
    assert e.value.status == 10
    with pytest.raises(backend.G2ocError) as e:
        c.backward(np.zeros((graph.num_poses, 6)), np.zeros((graph.num_points, 3)))
    assert e.value.status == 10
    c.close()
    with pytest.raises(backend.G2ocError):
        backend.CudaWindows([graph])
