"""Batched windows (g2oc_upload_windows / g2oc_optimize_windows): many
independent local bundle adjustments packed in one context, each running its
own Levenberg-Marquardt with a dense Cholesky of its reduced camera system.

Parity: every window against the FP64 oracle run alone with the same
algorithm (LM, Cholesky, 10 iterations): same iteration and trial counts and
final robust chi2 within 1e-8 relative for the FP64 context; final chi2
within 1e-3 relative for the mixed-precision context. A window gives the same
bits whether it is solved inside a batch or alone.
"""
import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import LINEAR_CHOLESKY, PREC_MIXED

pytestmark = pytest.mark.gpu

ITER = 10


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


@pytest.fixture(scope="module")
def small_windows():
    return synth.windows(24, cameras=(10, 24), points=(200, 900), seed=31)


def oracle_run(oracle_lib, g):
    o = oracle_lib.OracleProblem(g, oracle_lib.default_params(linear_solver=LINEAR_CHOLESKY))
    _, st = o.optimize(ITER)
    return st, o.estimates()


def test_windows_match_fp64_oracle(backend, oracle_lib, small_windows):
    cw = backend.CudaWindows(small_windows)
    st = cw.optimize(ITER)
    for w, g in enumerate(small_windows):
        so, (po, qo) = oracle_run(oracle_lib, g)
        s = st[w]
        assert s["iterations"] == len(so), (w, s, len(so))
        assert s["trials"] == sum(x["levenberg_iterations"] for x in so), w
        assert abs(s["chi2"] - so[-1]["chi2"]) <= 1e-8 * so[-1]["chi2"], (w, s["chi2"], so[-1]["chi2"])
        pc, qc = cw.estimates(w)
        assert np.abs(pc[:, :3] - po[:, :3]).max() < 1e-6
        assert np.abs(qc - qo).max() < 1e-5
    assert all(s["cholesky_threads"] in (128, 256, 512) for s in st)


def test_windows_mixed_precision_close_to_fp64_oracle(backend, oracle_lib, small_windows):
    cw = backend.CudaWindows(small_windows, backend.default_params(precision=PREC_MIXED))
    st = cw.optimize(ITER)
    for w, g in enumerate(small_windows):
        so, _ = oracle_run(oracle_lib, g)
        assert abs(st[w]["chi2"] - so[-1]["chi2"]) <= 1e-3 * so[-1]["chi2"], (w, st[w]["chi2"], so[-1]["chi2"])


def test_window_alone_equals_window_in_batch(backend, small_windows):
    cw = backend.CudaWindows(small_windows)
    st = cw.optimize(ITER)
    for w in (0, 7):
        one = backend.CudaWindows([small_windows[w]])
        s1 = one.optimize(ITER)[0]
        assert s1["chi2"] == st[w]["chi2"] and s1["trials"] == st[w]["trials"]
        for a, b in zip(one.estimates(0), cw.estimates(w)):
            assert np.array_equal(a, b)


def test_windows_rerun_and_iteration_limits(backend, small_windows):
    """A second optimize of the same context (the captured round replayed)
    from restored initial estimates gives the same result; 0 iterations leave
    every window untouched."""
    cw = backend.CudaWindows(small_windows[:6])
    a = cw.optimize(ITER)
    cw.restore_initial_estimates()
    b = cw.optimize(ITER)
    assert [s["chi2"] for s in a] == [s["chi2"] for s in b]
    cw.restore_initial_estimates()
    z = cw.optimize(0)
    assert all(s["iterations"] == 0 for s in z)
    p, q = cw.estimates(2)
    assert np.array_equal(p, small_windows[2].pose_estimate)


def test_windows_reupload_keeps_round_and_matches_fresh_context(backend, small_windows):
    """Re-uploading the same windows with new values keeps the captured round
    and the tuned dense solve; the result equals a fresh context's, bit for
    bit. New windows (other topology) rebuild everything."""
    ws = small_windows[:8]
    cw = backend.CudaWindows(ws)
    cw.optimize(ITER)
    moved = []
    for g in ws:
        g2 = g.copy()
        g2.measurement = g2.measurement + 0.25
        moved.append(g2)
    cw.upload(moved)
    a = cw.optimize(ITER)
    fresh = backend.CudaWindows(moved)
    b = fresh.optimize(ITER)
    assert [s["chi2"] for s in a] == [s["chi2"] for s in b]
    assert [s["trials"] for s in a] == [s["trials"] for s in b]
    for w in (0, 5):
        for x, y in zip(cw.estimates(w), fresh.estimates(w)):
            assert np.array_equal(x, y)
    other = small_windows[8:12]
    cw.upload(other)
    c = cw.optimize(ITER)
    d = backend.CudaWindows(other).optimize(ITER)
    assert [s["chi2"] for s in c] == [s["chi2"] for s in d]


def _merge(g0, g1):
    """One window made of two independent ones: its reduced camera system has
    zero blocks between the two camera groups."""
    from g2o_b200.abi import Graph

    def cat(a, b):
        return None if a is None else np.concatenate([a, b])

    ev1 = g1.edge_vertex + np.array([g0.num_points, g0.num_poses], dtype=g1.edge_vertex.dtype)
    return Graph(g0.pose_type, g0.edge_type, cat(g0.pose_estimate, g1.pose_estimate),
                 np.concatenate([g0.edge_vertex, ev1]), cat(g0.measurement, g1.measurement),
                 cat(g0.information, g1.information), cat(g0.pose_fixed, g1.pose_fixed),
                 cat(g0.point_estimate, g1.point_estimate), cat(g0.point_fixed, g1.point_fixed),
                 cat(g0.robust_delta, g1.robust_delta), g0.focal_length, tuple(g0.principal_point), "merged", {})


def test_windows_with_sparse_reduced_system(backend, oracle_lib, small_windows):
    """Windows whose cameras do not all co-observe (zero blocks in the dense
    matrix) against the FP64 oracle, batched with full ones."""
    ws = [_merge(small_windows[0], small_windows[1]), small_windows[2], _merge(small_windows[3], small_windows[4])]
    cw = backend.CudaWindows(ws)
    st = cw.optimize(ITER)
    for w, g in enumerate(ws):
        so, _ = oracle_run(oracle_lib, g)
        assert st[w]["iterations"] == len(so)
        assert st[w]["trials"] == sum(x["levenberg_iterations"] for x in so), w
        assert abs(st[w]["chi2"] - so[-1]["chi2"]) <= 1e-8 * so[-1]["chi2"], (w, st[w]["chi2"], so[-1]["chi2"])


def test_window_too_large_for_the_dense_solve_is_rejected(backend):
    """A window whose reduced camera system does not fit the dense solve's
    shared memory is refused at upload with NOT_SUPPORTED, not run."""
    big = synth.bundle_adjustment(num_cameras=150, num_points=400, min_obs=2, max_obs=4, seed=9)
    with pytest.raises(Exception, match="dense window solve"):
        backend.CudaWindows([big])
