"""Sharded bundle adjustment across processes: two ranks, each a separate
process with its own context (g2oc_set_sharding), their all-reduce a real
torch.distributed collective (gloo, over 127.0.0.1) on host copies of the
context's device buffers. The reduction runs on the host after the rank's
CUDA stream is drained, so no kernel waits for another process; on one GPU
the two contexts time-share the device.

The sharded run must follow the single-context run of the whole graph: the
same trial counts, chi2 per iteration within 1e-6 relative, camera
translations within 1e-6 m, points within 1e-5 m (FP64).
"""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ITER = 8
GRAPH = dict(num_cameras=60, num_points=6000, seed=43)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    try:
        import torch
        import torch.distributed as dist
        from g2o_b200 import backend, synth

        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
        torch.cuda.set_device(0)

        def allreduce(ptr, count, dtype, op, stream):
            torch.cuda.ExternalStream(stream, device=0).synchronize()
            t = backend.device_tensor(ptr, count, dtype, 0)
            h = t.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.SUM if op == backend.RED_SUM else dist.ReduceOp.MAX)
            t.copy_(h)
            torch.cuda.synchronize()

        g = synth.bundle_adjustment(**GRAPH)
        sub, idx = backend.split_points(g, world)[rank]
        fac = backend.OptimizationAlgorithmFactory.instance()
        prob = backend.CudaProblem(sub, fac.construct("lm_cuda"), device=0, shard=(rank, world, allreduce))
        done, st = prob.optimize(ITER)
        pose, point = prob.estimates()
        prob.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, done, st, pose, point, idx))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e)))


def test_two_process_shards_follow_the_single_context():
    from g2o_b200 import backend, synth
    g = synth.bundle_adjustment(**GRAPH)
    fac = backend.OptimizationAlgorithmFactory.instance()
    ref = backend.CudaProblem(g, fac.construct("lm_cuda"))
    done_ref, st_ref = ref.optimize(ITER)
    pose_ref, point_ref = ref.estimates()
    ref.close()

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = {}
    for _ in range(world):
        item = q.get(timeout=600)
        res[item[0]] = item
    for p in ps:
        p.join(timeout=120)
    for r in range(world):
        assert len(res[r]) == 6, res[r]
    for r in range(world):
        _, done, st, pose, point, idx = res[r]
        assert done == done_ref
        for a, b in zip(st, st_ref):
            assert a["levenberg_iterations"] == b["levenberg_iterations"], (r, a, b)
            assert abs(a["chi2"] - b["chi2"]) <= 1e-6 * b["chi2"], (r, a["chi2"], b["chi2"])
        assert np.abs(pose[:, :3] - pose_ref[:, :3]).max() < 1e-6
        assert np.abs(point - point_ref[idx]).max() < 1e-5
    assert np.array_equal(res[0][3], res[1][3])  # every rank holds the same cameras
    for p in ps:
        assert p.exitcode == 0
