"""Multi-GPU sharding of the batched windows, host side, on CPU: two gloo
ranks compute the same cost-balanced assignment; together they cover every
window exactly once; the per-rank results combine by the same collectives the
bench uses (max of the device times, sum of the iteration counts)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from g2o_b200 import shard, synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = synth.window_sizes()
    costs = [shard.window_cost(c, p) for c, p in sizes]
    mine = shard.assign_windows(costs, world)[rank]
    lists = [None] * world
    dist.all_gather_object(lists, mine)
    # stand-ins for the bench's per-rank device time and iteration count
    t = torch.tensor([1.0 + rank])
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    n = torch.tensor([float(10 * len(mine))])
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    load = [sum(costs[w] for w in lst) for lst in lists]
    q.put((rank, lists, float(t.item()), float(n.item()), load))
    dist.destroy_process_group()


def test_windows_shard_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    lists = res[0][1]
    assert all(r[1] == lists for r in res)            # every rank computed the same assignment
    allw = sorted(w for lst in lists for w in lst)
    assert allw == list(range(512))                    # each window exactly once
    assert all(r[2] == 2.0 for r in res)               # max over ranks
    assert all(r[3] == 10.0 * 512 for r in res)        # sum over ranks
    load = res[0][4]
    assert max(load) <= 1.02 * min(load)               # cost-balanced


def test_assignment_is_deterministic_and_balanced():
    from g2o_b200 import shard
    costs = [float((7 * w) % 13 + 1) for w in range(100)]
    for world in (1, 3, 8):
        a = shard.assign_windows(costs, world)
        assert a == shard.assign_windows(costs, world)
        assert sorted(w for x in a for w in x) == list(range(100))


def test_split_points_partitions_the_bundle_adjustment():
    """The shards of a sharded bundle adjustment: every camera on every rank,
    each point and each edge on exactly one, point indices renumbered within
    the shard, edge data carried along."""
    import numpy as np
    from g2o_b200 import backend, synth
    g = synth.bundle_adjustment(num_cameras=30, num_points=2000, seed=8)
    for parts in (1, 2, 3):
        shards = backend.split_points(g, parts)
        assert sum(s.num_points for s, _ in shards) == g.num_points
        assert sum(s.num_edges for s, _ in shards) == g.num_edges
        seen = np.concatenate([idx for _, idx in shards])
        assert np.array_equal(np.sort(seen), np.arange(g.num_points))
        for s, idx in shards:
            assert s.num_poses == g.num_poses and np.array_equal(s.pose_estimate, g.pose_estimate)
            assert np.array_equal(s.pose_fixed, g.pose_fixed)
            assert np.array_equal(s.point_estimate, g.point_estimate[idx])
            orig = s.edge_vertex[:, 0] + idx[0]
            sel = np.isin(g.edge_vertex[:, 0], idx)
            assert np.array_equal(orig, g.edge_vertex[sel, 0])
            assert np.array_equal(s.edge_vertex[:, 1], g.edge_vertex[sel, 1])
            assert np.array_equal(s.measurement, g.measurement[sel])
            assert np.array_equal(s.information, g.information[sel])


def test_split_points_keeps_the_edge_parameters():
    """A stereo graph's shards keep bf (EdgeStereoSE3ProjectXYZ) and the
    intrinsics; the measurement rows stay three wide."""
    from g2o_b200 import backend, synth
    g = synth.stereo_bundle_adjustment(num_cameras=12, num_points=600, seed=5)
    for s, _ in backend.split_points(g, 2):
        assert s.edge_type == g.edge_type and s.stereo_bf == g.stereo_bf and s.stereo_bf > 0
        assert s.focal_length == g.focal_length and s.focal_length_y == g.focal_length_y
        assert tuple(s.principal_point) == tuple(g.principal_point)
        assert s.measurement.shape[1] == g.measurement.shape[1] == 3
