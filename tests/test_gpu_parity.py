"""Parity of the CUDA path (through the C-ABI) with the FP64 oracle on the same
seeded graphs.

Tolerances (FP64 path): errors and Jacobians 1e-12 relative; Hessian blocks,
gradient and Schur blocks 1e-10 relative per block (the bar for the plain
FP64 form); block patterns bit-exact; linear solves and LM trajectories
within the stated tolerances of each test.
"""
import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import (ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, LINEAR_CHOLESKY, LINEAR_PCG, PREC_MIXED)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


def small_ba(seed=7, cams=40, points=3000, **kw):
    return synth.bundle_adjustment(num_cameras=cams, num_points=points, seed=seed, **kw)


def rel_block_err(a, b):
    """max over blocks of |a-b|_max / max(|b|_max, tiny)"""
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def both(backend, oracle_lib, g, **prm):
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    c = backend.CudaProblem(g, backend.default_params(**prm))
    return o, c


# ----------------------------------------------------------------- BA
def test_ba_structure_is_bit_exact(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    for f in ("num_free_poses", "num_free_points", "hpp_nnzb", "hpl_nnzb", "schur_nnzb", "num_active_edges",
              "vector_size", "schur_pairs"):
        assert getattr(o.info, f) == getattr(c.info, f), f
    for a, b in zip(o.pattern(), c.pattern()):
        assert np.array_equal(a, b)


def test_ba_errors_jacobians_chi2(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    j0c, j1c = c.jacobians()
    j0o, j1o = o.jacobians()
    assert rel_block_err(j0c, j0o) < 1e-12
    assert rel_block_err(j1c, j1o) < 1e-12
    (a, b), (x, y) = c.chi2(), o.chi2()
    assert abs(a - x) <= 1e-12 * x and abs(b - y) <= 1e-12 * y


def test_ba_hessian_and_gradient(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    o.build_system()
    c.build_system()
    hpp_o, hll_o, hpl_o, b_o = o.hessian()
    hpp_c, hll_c, hpl_c, b_c = c.hessian()
    assert rel_block_err(hpp_c, hpp_o) < 1e-10
    assert rel_block_err(hll_c, hll_o) < 1e-10
    assert rel_block_err(hpl_c, hpl_o) < 1e-10
    n = o.info.num_free_poses * 6
    assert rel_block_err(b_c[:n].reshape(-1, 6), b_o[:n].reshape(-1, 6)) < 1e-10
    assert relnorm(b_c[n:], b_o[n:]) < 1e-10


@pytest.mark.parametrize("lam", [0.0, 1e-3, 10.0])
def test_ba_schur_complement(backend, oracle_lib, lam):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    o.build_system()
    c.build_system()
    So, bso = o.schur(lam)
    Sc, bsc = c.schur(lam)
    assert rel_block_err(Sc, So) < 1e-10
    assert relnorm(bsc, bso) < 1e-10


def test_ba_pcg_solve_matches_oracle(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    o.build_system()
    c.build_system()
    so, xo, ito = o.solve(1e-2)
    sc, xc, itc = c.solve(1e-2)
    assert so == 0 and sc == 0
    assert abs(itc - ito) <= 1
    assert relnorm(xc, xo) < 1e-6


@pytest.mark.parametrize("form,kernel", [("", "pcg_solve_tiles"), ("sparse", "pcg_solve"), ("kernels", "pcg_spmv")])
def test_pcg_forms_match_oracle(backend, oracle_lib, monkeypatch, form, kernel):
    """The three forms of the PCG solve (dense tiles for a nearly full reduced
    camera system, the sparse cooperative launch, three kernels per iteration)
    against the oracle. 90 cameras: a full Schur pattern, 6 tile rows with a
    ragged last one."""
    if form:
        monkeypatch.setenv("G2OC_PCG", form)
    else:
        monkeypatch.delenv("G2OC_PCG", raising=False)
    g = small_ba(seed=21, cams=90, points=7000)
    o, c = both(backend, oracle_lib, g)
    o.build_system()
    c.build_system()
    for lam in (1e2, 1e-2):
        so, xo, ito = o.solve(lam)
        sc, xc, itc = c.solve(lam)
        assert so == 0 and sc == 0
        assert abs(itc - ito) <= 1, (itc, ito)
        assert relnorm(xc, xo) < 1e-6
    _, ks = c.kernel_stats()
    assert ks.get(kernel, (0, 0.0))[0] > 0, ks
    do, so_ = o.optimize(5)
    dc, sc_ = c.optimize(5)
    for a, b in zip(sc_, so_):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"]
    cm = backend.CudaProblem(g, backend.default_params(precision=PREC_MIXED))
    _, sm = cm.optimize(5)
    assert abs(sm[-1]["chi2"] - so_[-1]["chi2"]) <= 1e-3 * so_[-1]["chi2"]


def test_ba_cholesky_solve_is_exact(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g, linear_solver=LINEAR_CHOLESKY)
    o.build_system()
    c.build_system()
    so, xo, _ = o.solve(1e-2)
    sc, xc, _ = c.solve(1e-2)
    assert so == 0 and sc == 0
    assert relnorm(xc, xo) < 1e-9


@pytest.mark.parametrize("cams,points", [(64, 4000), (140, 6000)])
def test_ba_tensor_core_cholesky_solve(backend, oracle_lib, cams, points):
    """lm_cuda_chol_mixed on a bundle adjustment whose reduced camera system
    is nearly full: the tensor-core Cholesky (tcgen05 3xTF32 tile products,
    FP64 diagonal tiles) of the FP32-stored Schur complement, refined on the
    FP64 residual, solves the damped system to 1e-9 of the oracle's FP64
    Cholesky solve (LinearSolverDense's role)."""
    g = small_ba(seed=23, cams=cams, points=points)
    prm = backend.OptimizationAlgorithmFactory.instance().construct("lm_cuda_chol_mixed")
    prm.refine_max_iterations = 10
    prm.refine_tolerance = 1e-14
    c = backend.CudaProblem(g, prm)
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(linear_solver=LINEAR_CHOLESKY))
    c.build_system()
    o.build_system()
    for lam in (1e-2, 1.0):
        st, xc, _ = c.solve(lam)
        so, xo, _ = o.solve(lam)
        assert st == 0 and so == 0
        assert relnorm(xc, xo) < 1e-9, (lam, relnorm(xc, xo))
    _, ks = c.kernel_stats()
    assert ks["tc_tiles"][0] > 0 and ks["tc_potrf"][0] > 0
    c.close()


def test_ba_tensor_core_cholesky_lm_trajectory(backend, oracle_lib):
    """LM over the tensor-core Cholesky with FP64 refinement of every step
    follows the oracle's FP64 Cholesky trajectory: the same trials and chi2
    within 1e-6 per iteration."""
    g = small_ba(seed=29, cams=64, points=4000)
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(linear_solver=LINEAR_CHOLESKY))
    c = backend.CudaProblem(g, backend.OptimizationAlgorithmFactory.instance().construct("lm_cuda_chol_mixed"))
    _, so = o.optimize(10)
    _, sc = c.optimize(10)
    c.close()
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], a["iteration"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["iteration"], a["chi2"], b["chi2"])


def test_ba_lm_trajectory(backend, oracle_lib):
    g = small_ba()
    o, c = both(backend, oracle_lib, g)
    do, so = o.optimize(20)
    dc, sc = c.optimize(20)
    assert do == dc == 20
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["chi2"], b["chi2"])
    po, qo = o.estimates()
    pc, qc = c.estimates()
    assert np.abs(pc - po).max() < 1e-5
    assert np.abs(qc - qo).max() < 1e-4


@pytest.mark.parametrize("refine", [2, -1])
def test_ba_mixed_precision_reaches_fp64_chi2(backend, oracle_lib, refine):
    """Mixed precision, with FP64 refinement of every step (refine 2) and
    with FP32 steps under FP64 LM control only (refine -1), reaches the FP64
    oracle's 20-iteration chi2 within 1e-6 inside 30 iterations."""
    g = small_ba()
    o = oracle_lib.OracleProblem(g)
    _, so = o.optimize(20)
    target = so[-1]["chi2"]
    c = backend.CudaProblem(g, backend.default_params(precision=PREC_MIXED, refine_max_iterations=refine))
    _, sc = c.optimize(30)
    best = min(s["chi2"] for s in sc)
    assert best <= target * (1 + 1e-6), (best, target)


def test_ba_fixed_points_and_duplicate_observations(backend, oracle_lib):
    g = small_ba(seed=11, cams=12, points=400)
    g.point_fixed[::7] = 1
    # duplicate a few observations (same camera observes the same point twice)
    dup = np.arange(0, g.num_edges, 97)
    for name in ("edge_vertex", "measurement", "information", "robust_delta"):
        a = getattr(g, name)
        setattr(g, name, np.ascontiguousarray(np.concatenate([a, a[dup]])))
    g.measurement[-len(dup):] += 0.5
    o, c = both(backend, oracle_lib, g)
    for a, b in zip(o.pattern(), c.pattern()):
        assert np.array_equal(a, b)
    o.build_system()
    c.build_system()
    for a, b in zip(c.hessian()[:3], o.hessian()[:3]):
        assert rel_block_err(a, b) < 1e-10
    do, so = o.optimize(5)
    dc, sc = c.optimize(5)
    assert abs(sc[-1]["chi2"] - so[-1]["chi2"]) <= 1e-6 * so[-1]["chi2"]


def test_ba_without_robust_kernel(backend, oracle_lib):
    g = small_ba(seed=5, cams=10, points=300)
    g.robust_delta = None
    o, c = both(backend, oracle_lib, g)
    (a, b), (x, y) = c.chi2(), o.chi2()
    assert a == pytest.approx(x, rel=1e-12) and b == pytest.approx(a, rel=0)
    o.build_system()
    c.build_system()
    assert rel_block_err(c.hessian()[0], o.hessian()[0]) < 1e-10


# ------------------------------------------------------------ pose graphs
def test_pose_graph_2d_gn_cholesky(backend, oracle_lib):
    g = synth.pose_graph_2d(num_poses=600, num_closures=200, seed=3)
    o, c = both(backend, oracle_lib, g, algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY)
    for a, b in zip(o.pattern(), c.pattern()):
        assert np.array_equal(a, b)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    j = c.jacobians(), o.jacobians()
    assert rel_block_err(j[0][0], j[1][0]) < 1e-12 and rel_block_err(j[0][1], j[1][1]) < 1e-12
    o.build_system()
    c.build_system()
    assert rel_block_err(c.hessian()[0], o.hessian()[0]) < 1e-10
    assert relnorm(c.hessian()[3], o.hessian()[3]) < 1e-10
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    assert do == dc == 10
    for a, b in zip(sc, so):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-8 * b["chi2"], (a["chi2"], b["chi2"])


def test_pose_graph_3d_lm(backend, oracle_lib):
    g = synth.pose_graph_3d(num_rings=4, per_ring=40, radius=10.0, seed=4)
    o, c = both(backend, oracle_lib, g, algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_CHOLESKY)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    j = c.jacobians(), o.jacobians()
    assert rel_block_err(j[0][0], j[1][0]) < 1e-10 and rel_block_err(j[0][1], j[1][1]) < 1e-10
    o.build_system()
    c.build_system()
    assert rel_block_err(c.hessian()[0], o.hessian()[0]) < 1e-10
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    assert do == dc
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-7 * b["chi2"], (a["chi2"], b["chi2"])


def test_pose_graph_pcg(backend, oracle_lib):
    g = synth.pose_graph_3d(num_rings=4, per_ring=40, radius=10.0, seed=4)
    o, c = both(backend, oracle_lib, g, algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_PCG)
    do, so = o.optimize(5)
    dc, sc = c.optimize(5)
    for a, b in zip(sc, so):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["chi2"], b["chi2"])


# -------------------------------------------------------- linear solvers
def test_reference_block_system_on_gpu(backend):
    from tests.test_oracle_pinning import is_approx, load_sparse_system
    offs, rc, vals, b, x, _ = load_sparse_system()
    for _ in range(2):
        st, sol, _ = backend.solve_block_system(LINEAR_CHOLESKY, offs, rc, vals, b)
        assert st == 0 and is_approx(sol, x, 1e-6)
    prm = backend.default_params(pcg_tolerance=1e-20, pcg_max_iterations=200)
    st, sol, it = backend.solve_block_system(LINEAR_PCG, offs, rc, vals, b, prm)
    assert st == 0 and it > 0 and is_approx(sol, x, 1e-6)


def test_pcg_block_system_above_16384_block_rows(backend):
    """The multi-kernel PCG's column pass writes one partial sum per block row;
    a block-tridiagonal SPD system of 20,000 3x3 block rows (past the 16,384
    slots a context starts with) solves to the direct solution."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    rng = np.random.default_rng(11)
    nb, bs = 20000, 3
    rc, vals = [], []
    for c in range(nb):
        if c > 0:
            rc.append((c - 1, c))
            vals.append(rng.uniform(-1, 1, (bs, bs)))
        M = rng.uniform(-1, 1, (bs, bs))
        rc.append((c, c))
        vals.append(M @ M.T + 8 * np.eye(bs))
    rc = np.array(rc, np.int32)
    vals = np.stack(vals)
    offs = np.arange(nb + 1, dtype=np.int32) * bs
    rows, cols, data = [], [], []
    for (r, c), M in zip(rc, vals):
        ii, jj = np.meshgrid(np.arange(bs) + r * bs, np.arange(bs) + c * bs, indexing="ij")
        rows += [ii.ravel()]
        cols += [jj.ravel()]
        data += [M.ravel()]
        if r != c:
            rows += [jj.ravel()]
            cols += [ii.ravel()]
            data += [M.ravel()]
    A = sp.csr_matrix((np.concatenate(data), (np.concatenate(rows), np.concatenate(cols))), shape=(nb * bs,) * 2)
    b = rng.normal(size=nb * bs)
    x_ref = spl.spsolve(A.tocsc(), b)
    prm = backend.default_params(pcg_tolerance=1e-24, pcg_max_iterations=300)
    st, x, it = backend.solve_block_system(LINEAR_PCG, offs, rc, vals.ravel(), b, prm)
    assert st == 0 and it > 0
    assert relnorm(x, x_ref) < 1e-9, relnorm(x, x_ref)


@pytest.mark.parametrize("cams", [40, 64])
def test_grid_barrier_wait_runs_out_and_reports_timeout(backend, monkeypatch, cams):
    """The persistent PCG's grid barriers wait a bounded time. A context
    created with G2OC_TEST_BARRIER_EXTRA expects one arrival more than the
    grid launches, so no barrier completes: every wait runs out, the kernel
    returns, and the host reports G2OC_ERR_TIMEOUT (no trap, no hang). The
    device stays usable: the same context's state is reset, and another
    context optimizes the same graph normally. 40 cameras: the sparse
    persistent solve; 64: the dense-tile solve."""
    from g2o_b200.abi import G2OC_ERR_TIMEOUT
    g = small_ba(seed=31, cams=cams, points=3000)
    monkeypatch.setenv("G2OC_TEST_BARRIER_EXTRA", "1")
    bad = backend.CudaProblem(g)
    monkeypatch.delenv("G2OC_TEST_BARRIER_EXTRA")
    with pytest.raises(backend.G2ocError) as ei:
        bad.optimize(1)
    assert ei.value.status == G2OC_ERR_TIMEOUT
    bad.close()
    good = backend.CudaProblem(g)
    done, st = good.optimize(2)
    good.close()
    assert done == 2 and st[-1]["chi2"] < st[0]["chi2"] * 10


def test_tensor_core_substitution_barrier_runs_out_and_reports_timeout(backend, monkeypatch):
    """The tensor-core Cholesky's cooperative substitutions (one grid barrier
    per tile step) wait a bounded time too: with one arrival too many
    expected, every wait runs out, the kernel returns and the host reports
    G2OC_ERR_TIMEOUT; another context then optimizes the same graph."""
    from g2o_b200.abi import G2OC_ERR_TIMEOUT
    g = small_ba(seed=23, cams=64, points=4000)
    fac = backend.OptimizationAlgorithmFactory.instance()
    monkeypatch.setenv("G2OC_TEST_BARRIER_EXTRA", "1")
    bad = backend.CudaProblem(g, fac.construct("lm_cuda_chol_mixed"))
    monkeypatch.delenv("G2OC_TEST_BARRIER_EXTRA")
    with pytest.raises(backend.G2ocError) as ei:
        bad.optimize(1)
    assert ei.value.status == G2OC_ERR_TIMEOUT
    bad.close()
    good = backend.CudaProblem(g, fac.construct("lm_cuda_chol_mixed"))
    done, st = good.optimize(2)
    _, ks = good.kernel_stats()
    good.close()
    assert done == 2 and st[-1]["chi2"] < st[0]["chi2"] * 10
    assert ks["tc_solve"][0] > 0


def test_not_positive_definite_is_reported(backend):
    offs = np.array([0, 3, 6], np.int32)
    rc = np.array([[0, 0], [0, 1], [1, 1]], np.int32)
    vals = np.concatenate([np.eye(3).ravel(), 2 * np.eye(3).ravel(), np.eye(3).ravel()])
    st, _, _ = backend.solve_block_system(LINEAR_CHOLESKY, offs, rc, vals, np.ones(6))
    assert st == 4  # G2OC_ERR_NOT_PD


def test_iterate_matches_optimize(backend):
    g = small_ba(seed=9, cams=20, points=800)
    a = backend.CudaProblem(g)
    b = backend.CudaProblem(g)
    _, sa = a.optimize(6)
    for i in range(6):
        res, st = b.iterate(i)
        assert res == 1
        assert st["chi2"] == sa[i]["chi2"]
    pa, qa = a.estimates()
    pb, qb = b.estimates()
    assert np.array_equal(pa, pb) and np.array_equal(qa, qb)


def test_reupload_keeps_structure_and_matches_fresh_context(backend):
    """g2oc_upload of a graph with the same topology reuses the index structure
    and the device buffers; the values (estimates, measurements, information,
    robust kernels) are all replaced. A changed topology rebuilds."""
    g = small_ba(seed=13, cams=20, points=800)
    rng = np.random.default_rng(2)
    g2 = g.copy()
    g2.measurement += rng.normal(scale=0.3, size=g2.measurement.shape)
    g2.information *= rng.uniform(0.5, 2.0, size=(g2.num_edges, 1))
    g2.point_estimate += rng.normal(scale=0.05, size=g2.point_estimate.shape)
    g2.pose_estimate[:, :3] += rng.normal(scale=0.01, size=(g2.num_poses, 3))
    g2.robust_delta = None
    a = backend.CudaProblem(g)
    a.optimize(3)
    for gn in (g2, g):
        a.upload(gn)
        b = backend.CudaProblem(gn)
        assert a.chi2() == b.chi2()
        _, sa = a.optimize(5)
        _, sb = b.optimize(5)
        assert [s["chi2"] for s in sa] == [s["chi2"] for s in sb]
        for x, y in zip(a.estimates(), b.estimates()):
            assert np.array_equal(x, y)
        b.close()
    g3 = g.copy()
    g3.point_fixed[::5] = 1
    a.upload(g3)
    b = backend.CudaProblem(g3)
    assert a.info.num_free_points == b.info.num_free_points < g.num_points
    _, sa = a.optimize(4)
    _, sb = b.optimize(4)
    assert [s["chi2"] for s in sa] == [s["chi2"] for s in sb]


def test_factory_constructed_solver_runs(backend, oracle_lib):
    fac = backend.OptimizationAlgorithmFactory.instance()
    g = synth.pose_graph_2d(num_poses=300, num_closures=100, seed=8)
    opt = backend.SparseOptimizer()
    opt.set_algorithm(fac.construct("gn_cuda"))
    opt.set_graph(g.copy())
    assert opt.initialize_optimization()
    assert opt.optimize(5) == 5
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(algorithm=ALGO_GAUSS_NEWTON,
                                                              linear_solver=LINEAR_CHOLESKY))
    o.optimize(5)
    assert abs(opt.active_chi2() - o.chi2()[0]) <= 1e-8 * o.chi2()[0]


# ------------------------------------------------------------ invalid graphs
def test_invalid_graphs_are_refused_at_upload(backend):
    """Graphs the reference would not optimize are refused with BAD_GRAPH at
    upload (g2oc_upload), not run: a vertex index out of range, no edge at
    all, and no active edge (every vertex of every edge fixed,
    allVerticesFixed)."""
    g = small_ba(cams=10, points=200)
    bad = g.copy()
    bad.edge_vertex[5, 1] = g.num_poses  # camera index past the end
    with pytest.raises(backend.G2ocError) as e:
        backend.CudaProblem(bad)
    assert e.value.status == 2
    empty = g.copy()
    empty.edge_vertex = empty.edge_vertex[:0].copy()
    empty.measurement = empty.measurement[:0].copy()
    empty.information = empty.information[:0].copy()
    empty.robust_delta = None
    with pytest.raises(backend.G2ocError) as e:
        backend.CudaProblem(empty)
    assert e.value.status == 2
    fixed = g.copy()
    fixed.pose_fixed = np.ones(g.num_poses, dtype=np.uint8)
    fixed.point_fixed = np.ones(g.num_points, dtype=np.uint8)
    with pytest.raises(backend.G2ocError) as e:
        backend.CudaProblem(fixed)
    assert e.value.status == 2


# ------------------------------------------- EdgeSE3ProjectXYZ (fx != fy)
def test_se3_project_xyz_matches_oracle(backend, oracle_lib):
    """EdgeSE3ProjectXYZ (g2o/types/sba/edge_project_xyz.cpp:43-100) on the
    same kernels as EdgeProjectXYZ2UV with its own fx, fy: errors, Jacobians,
    Hessian and a 20-iteration LM trajectory against the FP64 oracle."""
    from g2o_b200.abi import EDGE_SE3_PROJECT_XYZ
    g = small_ba(seed=21, focal_y=455.0)
    assert g.edge_type == EDGE_SE3_PROJECT_XYZ
    o, c = both(backend, oracle_lib, g)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    j0c, j1c = c.jacobians()
    j0o, j1o = o.jacobians()
    assert rel_block_err(j0c, j0o) < 1e-12 and rel_block_err(j1c, j1o) < 1e-12
    o.build_system()
    c.build_system()
    hc, ho = c.hessian(), o.hessian()
    for a, b in zip(hc[:3], ho[:3]):
        assert rel_block_err(a, b) < 1e-10
    do, so = o.optimize(20)
    dc, sc = c.optimize(20)
    assert do == dc == 20
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (a["chi2"], b["chi2"])
    # the same graph read as EdgeProjectXYZ2UV (fy := fx) is a different problem
    g2 = g.copy()
    g2.focal_length_y = g.focal_length
    assert abs(backend.CudaProblem(g2).chi2()[0] - c.chi2()[0]) > 1e-3 * c.chi2()[0]


def test_se3_project_xyz_windows_and_mixed(backend, oracle_lib):
    from g2o_b200.abi import EDGE_SE3_PROJECT_XYZ, LINEAR_CHOLESKY
    ws = [synth.bundle_adjustment(num_cameras=12 + 2 * i, num_points=300 + 50 * i, seed=60 + i, focal_y=455.0,
                                  num_fixed=1) for i in range(4)]
    assert all(w.edge_type == EDGE_SE3_PROJECT_XYZ for w in ws)
    cw = backend.CudaWindows(ws)
    st = cw.optimize(10)
    for w, g in enumerate(ws):
        o = oracle_lib.OracleProblem(g, oracle_lib.default_params(linear_solver=LINEAR_CHOLESKY))
        _, so = o.optimize(10)
        assert st[w]["iterations"] == len(so)
        assert abs(st[w]["chi2"] - so[-1]["chi2"]) <= 1e-8 * so[-1]["chi2"], (w, st[w]["chi2"], so[-1]["chi2"])
    cw.close()
    g = small_ba(seed=22, focal_y=455.0)
    o = oracle_lib.OracleProblem(g)
    _, so = o.optimize(20)
    m = backend.CudaProblem(g, backend.default_params(precision=PREC_MIXED))
    _, sm = m.optimize(30)
    assert min(s["chi2"] for s in sm) <= so[-1]["chi2"] * (1 + 1e-6)


# ------------------------------------------- OptimizationAlgorithmDogleg
@pytest.mark.parametrize("kind", ["pg2d_chol", "pg3d_chol", "pg3d_pcg", "ba"])
def test_dogleg_matches_oracle(backend, oracle_lib, kind):
    """dl_cuda* against the oracle's restatement of
    OptimizationAlgorithmDogleg::solve (optimization_algorithm_dogleg.cpp:62-180):
    per iteration the same tries and step type, chi2 and trust radius within
    1e-8 (FP64), over the iterations before convergence (there the gain
    ratio is a difference of nearly equal chi2 values and its sign is
    rounding)."""
    from g2o_b200.abi import ALGO_DOGLEG
    fac = backend.OptimizationAlgorithmFactory.instance()
    if kind == "pg2d_chol":
        g, name, iters = synth.pose_graph_2d(num_poses=600, num_closures=200, seed=3), "dl_cuda_chol", 4
    elif kind == "pg3d_chol":
        g, name, iters = synth.pose_graph_3d(num_rings=4, per_ring=40, radius=10.0, seed=4), "dl_cuda_chol", 4
    elif kind == "pg3d_pcg":
        g, name, iters = synth.pose_graph_3d(num_rings=4, per_ring=40, radius=10.0, seed=4), "dl_cuda_pcg", 4
    else:
        g, name, iters = small_ba(seed=23), "dl_cuda", 6
    prm = fac.construct(name)
    assert prm.algorithm == ALGO_DOGLEG
    o = oracle_lib.OracleProblem(g, prm)
    c = backend.CudaProblem(g, prm)
    do, so = o.optimize(iters)
    dc, sc = c.optimize(iters)
    assert do == dc
    tol = 1e-8 if kind != "pg3d_pcg" else 1e-6
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], (a, b)
        assert a["dogleg_step"] == b["dogleg_step"], (a, b)
        assert abs(a["chi2"] - b["chi2"]) <= tol * b["chi2"], (a["chi2"], b["chi2"])
        assert abs(a["trust_radius"] - b["trust_radius"]) <= 1e-6 * b["trust_radius"], (a, b)
    assert sc[-1]["chi2"] < sc[0]["chi2"] or kind == "ba"
    c.close()


# ------------------------------------------- StructureOnlySolver<3>
def test_structure_only_matches_oracle(backend, oracle_lib):
    """structure_only_cuda_3 (one small LM per landmark, cameras fixed)
    against the oracle's restatement of StructureOnlySolver<3>::calc
    (g2o/solvers/structure_only/structure_only_solver.h:66-215)."""
    from g2o_b200.abi import ALGO_STRUCTURE_ONLY
    fac = backend.OptimizationAlgorithmFactory.instance()
    prm = fac.construct("structure_only_cuda_3")
    assert prm.algorithm == ALGO_STRUCTURE_ONLY
    g = small_ba(seed=24)
    o = oracle_lib.OracleProblem(g, prm)
    c = backend.CudaProblem(g, prm)
    do, so = o.optimize(3)
    dc, sc = c.optimize(3)
    assert do == dc == 3
    for a, b in zip(sc, so):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-9 * b["chi2"], (a["chi2"], b["chi2"])
    (pc, qc), (po, qo) = c.estimates(), o.estimates()
    assert np.array_equal(pc, g.pose_estimate)  # cameras untouched
    assert np.abs(qc - qo).max() < 1e-9
    # the entry point with more inner iterations keeps lowering the chi2
    before = c.chi2()[1]
    c.structure_only(num_iters=5, num_max_trials=10)
    assert c.chi2()[1] <= before
    c.close()
    with pytest.raises(backend.G2ocError):
        backend.CudaProblem(synth.pose_graph_2d(num_poses=50, num_closures=10, seed=2)).structure_only()


# ------------------------------------------- EdgeSE3Expmap pose graph
@pytest.mark.parametrize("linear", ["chol", "pcg"])
def test_se3_expmap_pose_graph_matches_oracle(backend, oracle_lib, linear):
    """EdgeSE3Expmap between VertexSE3Expmap (g2o/types/sba/edge_se3_expmap.cpp)
    on the pose-graph kernels: errors 1e-12, Jacobians and Hessian 1e-10, a
    10-iteration LM trajectory (trial counts equal, chi2 1e-7; PCG 1e-6)."""
    from g2o_b200.abi import EDGE_SE3_EXPMAP
    g = synth.pose_graph_3d_expmap(num_rings=4, per_ring=40, radius=10.0, seed=4)
    assert g.edge_type == EDGE_SE3_EXPMAP
    lin = LINEAR_CHOLESKY if linear == "chol" else LINEAR_PCG
    o, c = both(backend, oracle_lib, g, algorithm=ALGO_LEVENBERG, linear_solver=lin)
    for a, b in zip(o.pattern(), c.pattern()):
        assert np.array_equal(a, b)
    assert relnorm(c.errors(), o.errors()) < 1e-12
    j = c.jacobians(), o.jacobians()
    assert rel_block_err(j[0][0], j[1][0]) < 1e-10 and rel_block_err(j[0][1], j[1][1]) < 1e-10
    o.build_system()
    c.build_system()
    assert rel_block_err(c.hessian()[0], o.hessian()[0]) < 1e-10
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    assert do == dc
    tol = 1e-7 if linear == "chol" else 1e-6
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"]
        assert abs(a["chi2"] - b["chi2"]) <= tol * b["chi2"], (a["chi2"], b["chi2"])
    assert sc[-1]["chi2"] < sc[0]["chi2"]
    c.close()


def test_pose_only_projection_edges(backend, oracle_lib):
    """EdgeSE3ProjectXYZOnlyPose (g2o/types/sba/edge_project_xyz_onlypose.cpp)
    is EdgeSE3ProjectXYZ with the point a constant: with every point fixed the
    BA path solves the cameras alone (no Schur complement), as ORB-SLAM's
    pose-only optimization does; LM trajectory against the oracle."""
    g = small_ba(seed=25, cams=12, points=1500, focal_y=455.0)
    g.point_fixed[:] = 1
    g.pose_fixed[:] = 0
    o, c = both(backend, oracle_lib, g, algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_CHOLESKY)
    assert c.info.num_free_points == 0 and c.info.schur_nnzb == 0
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    assert do == dc
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-8 * b["chi2"], (a["chi2"], b["chi2"])
    (pc, qc), (po, qo) = c.estimates(), o.estimates()
    assert np.abs(pc - po).max() < 1e-8
    assert np.array_equal(qc, g.point_estimate)
    c.close()
