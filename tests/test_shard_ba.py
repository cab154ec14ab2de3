"""Sharded bundle adjustment (g2oc_set_sharding): every rank holds every
camera and a share of the points; per LM trial the ranks sum their parts of
the reduced camera system, chi2 and the gain-ratio scale, then take the same
step. Run here as two and three ranks in one process on one GPU: contexts driven by
host threads whose all-reduce meets on the host (each rank's CUDA stream
is drained before the meeting, no kernel waits for another). The sharded run
must follow the single-context run of the whole graph: same trial counts,
chi2 per iteration within 1e-6 relative, camera translations within 1e-6 m and
points within 1e-5 m (FP64; 2e-5 / 2e-4 m with FP32 storage)."""
import threading

import numpy as np
import pytest

from g2o_b200 import synth
from g2o_b200.abi import PREC_MIXED

pytestmark = pytest.mark.gpu

ITER = 8


@pytest.fixture(scope="module")
def backend():
    from g2o_b200 import backend as B
    B.library()
    return B


class HostBus:
    """The ranks' meeting point: each all-reduce waits for every rank, rank 0
    combines the buffers on the device and writes the result to all."""

    def __init__(self, world):
        self.world = world
        self.bar = threading.Barrier(world, timeout=120)
        self.slots = [None] * world
        self.calls = 0

    def reducer(self, backend, rank):
        import torch

        def fn(ptr, count, dtype, op, stream):
            torch.cuda.ExternalStream(stream).synchronize()
            self.slots[rank] = (ptr, count, dtype)
            self.bar.wait()
            if rank == 0:
                self.calls += 1
                ts = [backend.device_tensor(*self.slots[r]) for r in range(self.world)]
                acc = ts[0].clone()
                for t in ts[1:]:
                    acc = acc + t if op == backend.RED_SUM else torch.maximum(acc, t)
                for t in ts:
                    t.copy_(acc)
                torch.cuda.synchronize()
            self.bar.wait()

        return fn


def run_sharded(backend, g, make_params, iters, world=2):
    shards = backend.split_points(g, world)
    bus = HostBus(world)
    out = [None] * world

    def work(r):
        try:
            prob = backend.CudaProblem(shards[r][0], make_params(), shard=(r, world, bus.reducer(backend, r)))
            done, st = prob.optimize(iters)
            pose, point = prob.estimates()
            out[r] = (done, st, pose, point)
            prob.close()
        except Exception as e:  # let the other rank leave its barrier
            out[r] = e
            bus.bar.abort()

    th = [threading.Thread(target=work, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=600)
    errs = [out[r] for r in range(world) if isinstance(out[r], Exception)]
    if errs:
        # the rank that failed first, not the ones whose all-reduce it broke
        first = [e for e in errs if "all-reduce returned" not in str(e)]
        raise (first or errs)[0]
    return out, shards, bus.calls


@pytest.mark.parametrize("precision,world", [("fp64", 2), ("mixed_fast", 2), ("fp64", 3)])
def test_shards_follow_the_single_context(backend, precision, world):
    g = synth.bundle_adjustment(num_cameras=60, num_points=6000, seed=41)
    fac = backend.OptimizationAlgorithmFactory.instance()
    name = "lm_cuda" if precision == "fp64" else "lm_cuda_mixed_fast"
    ref = backend.CudaProblem(g, fac.construct(name))
    done_ref, st_ref = ref.optimize(ITER)
    pose_ref, point_ref = ref.estimates()
    ref.close()
    out, shards, calls = run_sharded(backend, g, lambda: fac.construct(name), ITER, world)
    # metres, in a 20 m scene: FP64 sums in another order; FP32 storage of H and S
    tol_pose, tol_point = (1e-6, 1e-5) if precision == "fp64" else (2e-5, 2e-4)
    assert calls > 0
    for r, (done, st, pose, point) in enumerate(out):
        assert done == done_ref
        for a, b in zip(st, st_ref):
            assert a["levenberg_iterations"] == b["levenberg_iterations"], (r, a, b)
            assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (r, a["chi2"], b["chi2"])
        assert np.abs(pose[:, :3] - pose_ref[:, :3]).max() < tol_pose
        idx = shards[r][1]
        assert np.abs(point - point_ref[idx]).max() < tol_point
    # every rank holds the same cameras
    for r in range(1, world):
        assert np.array_equal(out[0][2], out[r][2])


def test_sharding_rejects_unsupported_setups(backend):
    g = synth.bundle_adjustment(num_cameras=60, num_points=2000, seed=42)
    fac = backend.OptimizationAlgorithmFactory.instance()
    with pytest.raises(Exception):  # FP64 refinement needs reductions the sharded path does not make
        prob = backend.CudaProblem(g, backend.default_params(precision=PREC_MIXED),
                                   shard=(0, 2, lambda *a: None))
        prob.optimize(1)
    with pytest.raises(Exception):
        backend.CudaProblem(g, fac.construct("lm_cuda"), shard=(2, 2, lambda *a: None))


def test_shards_with_a_pose_edge_set(backend):
    # the pose edges ride on shard 0 (split_points) and their terms are added
    # once before the ranks sum; PCG solves converged (the stiff odometry
    # blocks make the default stopping iteration depend on the last bits)
    g = synth.ba_with_odometry(num_cameras=40, num_points=3000)
    make = lambda: backend.default_params(pcg_tolerance=1e-14)  # noqa: E731
    ref = backend.CudaProblem(g, make())
    done_ref, st_ref = ref.optimize(ITER)
    pose_ref, point_ref = ref.estimates()
    ref.close()
    out, shards, calls = run_sharded(backend, g, make, ITER, 2)
    assert calls > 0
    assert shards[0][0].num_pose_edges == g.num_pose_edges and shards[1][0].num_pose_edges == 0
    for r, (done, st, pose, point) in enumerate(out):
        assert done == done_ref
        for a, b in zip(st, st_ref):
            assert a["levenberg_iterations"] == b["levenberg_iterations"], (r, a, b)
            assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (r, a["chi2"], b["chi2"])
        assert np.abs(pose[:, :3] - pose_ref[:, :3]).max() < 1e-5
        assert np.abs(point - point_ref[shards[r][1]]).max() < 1e-4


def test_pose_edges_on_another_rank_are_refused(backend):
    g = synth.ba_with_odometry(num_cameras=40, num_points=600)
    with pytest.raises(Exception, match="rank 0"):
        backend.CudaProblem(g, backend.default_params(), shard=(1, 2, lambda *a: None))


def test_shards_of_a_stereo_graph(backend):
    # EdgeStereoSE3ProjectXYZ (three-row edges): the shards keep bf
    g = synth.stereo_bundle_adjustment(num_cameras=60, num_points=6000, seed=93)
    make = lambda: backend.default_params()  # noqa: E731
    ref = backend.CudaProblem(g, make())
    done_ref, st_ref = ref.optimize(ITER)
    pose_ref, point_ref = ref.estimates()
    ref.close()
    out, shards, calls = run_sharded(backend, g, make, ITER, 2)
    assert calls > 0 and all(s.stereo_bf == g.stereo_bf for s, _ in shards)
    for r, (done, st, pose, point) in enumerate(out):
        assert done == done_ref
        for a, b in zip(st, st_ref):
            assert a["levenberg_iterations"] == b["levenberg_iterations"], (r, a, b)
            assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (r, a["chi2"], b["chi2"])
        assert np.abs(pose[:, :3] - pose_ref[:, :3]).max() < 1e-6
        assert np.abs(point - point_ref[shards[r][1]]).max() < 1e-5
