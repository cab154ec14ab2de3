"""Parity at the full sizes of the synthetic configurations, through the C-ABI,
against the FP64 oracle run live on the same seeded graphs (all host cores)
and against the oracle trajectories committed in tests/golden/oracle_targets.json
(made by tests/golden/make_oracle_targets.py).

* BA, 1000 cameras / 200,000 points / ~1.03M edges, LM + Schur + PCG, 20
  iterations, FP64: the same number of LM trials in every iteration, robust
  chi2 within 1e-6 relative per iteration, camera translations within 5e-5 m
  and quaternions within 5e-5 (cameras on a 30 m ring: 2e-6 relative; both
  sides solve with PCG to the 1e-6 stopping rule, so each step differs at
  that level). Landmarks seen by three or more cameras through inlier
  measurements only (60% of them): 99.9% within 1e-3 m, and their edges'
  residuals within 1e-2 px (the cameras' difference moves a projection by
  ~3e-4 px at 25 m; triangulation from nearby cameras amplifies it in
  depth, not in the image). A landmark with an outlier observation (1% of the measurements
  are replaced by uniform pixels) sits where the Huber cost is nearly flat,
  and one seen twice with a short baseline is weakly determined along its
  rays: such landmarks follow the per-step PCG differences far more than the
  cameras do (up to 0.15 m, 0.4 px), so they are only counted. The mixed forms (FP64 refinement of every step,
  and FP32 steps under FP64 LM control) reach the oracle's 20-iteration chi2
  within 1e-6 relative.
* 2D pose graph, 3500 poses, Gauss-Newton + Cholesky, 10 iterations: chi2
  within 1e-8 per iteration, poses within 1e-6.
* 3D pose graph, 2500 poses, LM + Cholesky, 20 iterations, FP64: same trials,
  chi2 within 1e-7 per iteration; mixed precision reaches the oracle's final
  chi2 within 1e-6.
* Batched windows at the configuration's real sizes (10-60 cameras,
  500-8000 points): the 16 costliest of the 512 windows and 16 more spread
  over the list, each against the oracle run alone.
"""
import os

import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, LINEAR_CHOLESKY, LINEAR_PCG, PREC_MIXED

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


@pytest.fixture(scope="module")
def targets():
    from tests.golden.make_oracle_targets import load
    return load()


@pytest.fixture(scope="module")
def ba_graph():
    return synth.bundle_adjustment()


@pytest.fixture(scope="module")
def ba_oracle(oracle_lib, ba_graph):
    o = oracle_lib.OracleProblem(ba_graph, oracle_lib.default_params(), threads=THREADS)
    done, st = o.optimize(20)
    pose, point = o.estimates()
    err = o.errors()
    return done, st, pose, point, err


def check_against_golden(name, g, st, targets, rel):
    t = targets[name]
    assert g.digest() == t["digest"], f"{name}: the generator no longer gives the committed graph"
    assert len(st) == len(t["chi2"])
    for s, chi2, trials in zip(st, t["chi2"], t["levenberg_iterations"]):
        assert s["levenberg_iterations"] == trials
        assert abs(s["chi2"] - chi2) <= rel * chi2, (name, s["iteration"], s["chi2"], chi2)


def test_ba_full_size_fp64_matches_oracle(backend, ba_graph, ba_oracle, targets):
    done_o, so, po, qo, eo = ba_oracle
    check_against_golden("ba", ba_graph, so, targets, 1e-12)
    c = backend.CudaProblem(ba_graph, backend.default_params())
    done_c, sc = c.optimize(20)
    assert done_c == done_o == 20
    worst = 0.0
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], (a["iteration"], a, b)
        rel = abs(a["chi2"] - b["chi2"]) / b["chi2"]
        worst = max(worst, rel)
        assert rel <= 1e-6, (a["iteration"], a["chi2"], b["chi2"])
    pc, qc = c.estimates()
    ec = c.errors()
    c.close()
    # cameras: translation (m) and quaternion
    assert np.abs(pc - po).max() < 5e-5, np.abs(pc - po).max()
    # landmarks (m) and their edges' residuals (px): the well-determined ones
    pt = ba_graph.edge_vertex[:, 0]
    nobs = np.bincount(pt, minlength=ba_graph.num_points)
    nout = np.bincount(pt, weights=ba_graph.extra["outliers"].astype(float), minlength=ba_graph.num_points)
    good = (nobs >= 3) & (nout == 0)
    dq = np.abs(qc - qo).max(axis=1)
    de = np.abs(ec - eo).max(axis=1)
    de_good = de[good[pt]]
    print(f"BA full size: worst per-iteration chi2 difference {worst:.2e}, pose {np.abs(pc - po).max():.2e}; "
          f"{good.sum()} well-determined landmarks: 99.9% {np.quantile(dq[good], 0.999):.2e} max {dq[good].max():.2e} m, "
          f"residual {de_good.max():.2e} px; "
          f"all landmarks: 99.9% {np.quantile(dq, 0.999):.2e} max {dq.max():.2e} m, residual max {de.max():.2e} px")
    assert good.sum() > 0.5 * ba_graph.num_points
    assert np.quantile(dq[good], 0.999) < 1e-3, np.quantile(dq[good], 0.999)
    assert de_good.max() < 1e-2, de_good.max()


@pytest.mark.parametrize("solver", ["lm_cuda_mixed", "lm_cuda_mixed_fast"])
def test_ba_full_size_mixed_reaches_oracle_chi2(backend, ba_graph, ba_oracle, solver):
    target = ba_oracle[1][-1]["chi2"]
    prm = backend.OptimizationAlgorithmFactory.instance().construct(solver)
    c = backend.CudaProblem(ba_graph, prm)
    _, sc = c.optimize(30)
    c.close()
    hit = [s["iteration"] + 1 for s in sc if s["chi2"] <= target * (1 + 1e-6)]
    assert hit, (solver, min(s["chi2"] for s in sc), target)
    print(f"{solver}: oracle's 20-iteration chi2 reached after {hit[0]} iterations; "
          f"after 20: {(sc[19]['chi2'] - target) / target:+.2e} relative")


def test_pg2d_full_size_gauss_newton(backend, oracle_lib, targets):
    g = synth.pose_graph_2d()
    prm = dict(algorithm=ALGO_GAUSS_NEWTON, linear_solver=LINEAR_CHOLESKY)
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    c = backend.CudaProblem(g, backend.default_params(**prm))
    for a, b in zip(o.pattern(), c.pattern()):
        assert np.array_equal(a, b)
    do, so = o.optimize(10)
    dc, sc = c.optimize(10)
    check_against_golden("pg2d", g, so, targets, 1e-12)
    assert do == dc == 10
    for a, b in zip(sc, so):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-8 * b["chi2"], (a["iteration"], a["chi2"], b["chi2"])
    pc, _ = c.estimates()
    po, _ = o.estimates()
    c.close()
    assert np.abs(pc - po).max() < 1e-6, np.abs(pc - po).max()


def test_pg3d_full_size_levenberg(backend, oracle_lib, targets):
    g = synth.pose_graph_3d()
    prm = dict(algorithm=ALGO_LEVENBERG, linear_solver=LINEAR_CHOLESKY)
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(**prm))
    c = backend.CudaProblem(g, backend.default_params(**prm))
    do, so = o.optimize(20)
    dc, sc = c.optimize(20)
    check_against_golden("pg3d", g, so, targets, 1e-12)
    assert do == dc == 20
    for a, b in zip(sc, so):
        assert a["levenberg_iterations"] == b["levenberg_iterations"], a["iteration"]
        assert abs(a["chi2"] - b["chi2"]) <= 1e-7 * b["chi2"], (a["iteration"], a["chi2"], b["chi2"])
    pc, _ = c.estimates()
    po, _ = o.estimates()
    c.close()
    assert np.abs(pc - po).max() < 1e-5, np.abs(pc - po).max()


@pytest.mark.parametrize("solver", ["lm_cuda_chol_mixed", "lm_cuda_chol_mixed_fast"])
def test_pg3d_full_size_mixed_reaches_oracle_chi2(backend, targets, solver):
    g = synth.pose_graph_3d()
    target = targets["pg3d"]["final_chi2"]
    prm = backend.OptimizationAlgorithmFactory.instance().construct(solver)
    assert prm is not None and prm.precision == PREC_MIXED
    c = backend.CudaProblem(g, prm)
    _, sc = c.optimize(30)
    c.close()
    hit = [s["iteration"] + 1 for s in sc if s["chi2"] <= target * (1 + 1e-6)]
    assert hit, (solver, min(s["chi2"] for s in sc), target)


def window_sample():
    from g2o_b200 import shard
    sizes = synth.window_sizes()
    cost = [shard.window_cost(c, p) for c, p in sizes]
    costliest = sorted(range(len(sizes)), key=lambda w: -cost[w])[:16]
    spread = [w for w in range(0, len(sizes), 32) if w not in costliest][:16]
    return sorted(costliest + spread)


def test_windows_real_sizes_match_oracle(backend, oracle_lib):
    which = window_sample()
    ws = synth.windows(which=which)
    assert max(g.num_poses for g in ws) >= 50 and max(g.num_points for g in ws) >= 6000
    cw = backend.CudaWindows(ws)
    st = cw.optimize(10)
    for k, g in enumerate(ws):
        o = oracle_lib.OracleProblem(g, oracle_lib.default_params(linear_solver=LINEAR_CHOLESKY))
        _, so = o.optimize(10)
        po, qo = o.estimates()
        s = st[k]
        assert s["iterations"] == len(so), (which[k], s, len(so))
        assert s["trials"] == sum(x["levenberg_iterations"] for x in so), which[k]
        assert abs(s["chi2"] - so[-1]["chi2"]) <= 1e-8 * so[-1]["chi2"], (which[k], s["chi2"], so[-1]["chi2"])
        pc, qc = cw.estimates(k)
        assert np.abs(pc[:, :3] - po[:, :3]).max() < 1e-6, which[k]
        assert np.abs(qc - qo).max() < 1e-5, which[k]
    cw.close()
