"""The .g2o text format (include/g2o_io.h) against the plain-Python
restatement oracle/g2o_text.py: loaded arrays bit-exact, saved text
byte-exact, the load counters equal. The first tests restate g2o's own
save/load tests (unit_test/general/graph_operations.cpp:186-405). No GPU."""
import os
import subprocess

import numpy as np
import pytest

from g2o_b200 import abi, synth
from g2o_b200.backend import G2ocError
from g2o_b200.g2ofile import SAVE_EDGE_SUBSET, SAVE_VERTEX_SUBSET, G2oFile
from oracle import g2o_text as gt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "g2o_b200", "g2o_cuda_cli")
ARRAYS = ["pose_estimate", "edge_vertex", "measurement", "information", "pose_fixed", "point_estimate",
          "point_fixed", "robust_delta"]


def same_graph(a, b):
    assert (a.pose_type, a.edge_type) == (b.pose_type, b.edge_type)
    for k in ARRAYS:
        x, y = getattr(a, k), getattr(b, k)
        if x is None or y is None:
            assert x is None and y is None, k
            continue
        assert x.shape == y.shape and np.array_equal(x, y), k
    assert a.focal_length == b.focal_length and tuple(a.principal_point) == tuple(b.principal_point)


def saved(f, tmp_path, name="out.g2o", **kw):
    p = str(tmp_path / name)
    f.save(p, **kw)
    return open(p).read()


def ids_of(text, prefix):
    out = []
    for line in text.splitlines():
        t = line.split()
        if t and t[0].startswith(prefix):
            out.append(tuple(int(x) for x in t[1:3]) if prefix == "EDGE_" else int(t[1]))
    return out


def fixed_of(text):
    return [int(x) for line in text.splitlines() if line.startswith("FIX") for x in line.split()[1:]]


# ------------------------------------------- g2o's GeneralGraphOperations fixture
@pytest.fixture
def three_pose_loop():
    """3 VertexSE2 at the origin, vertex 0 fixed, EdgeSE2 (i, i+1 mod 3) with
    measurement (1, 0, 0) and identity information."""
    n = 3
    g = abi.Graph(abi.POSE_SE2, abi.EDGE_SE2, np.zeros((n, 3)), [[i, (i + 1) % n] for i in range(n)],
                  np.tile([1.0, 0.0, 0.0], (n, 1)), np.tile(np.eye(3).reshape(-1), (n, 1)),
                  pose_fixed=np.array([1, 0, 0], dtype=np.uint8))
    return G2oFile.from_graph(g)


def test_saving_graph(three_pose_loop, tmp_path):
    text = saved(three_pose_loop, tmp_path)
    assert ids_of(text, "VERTEX_") == [0, 1, 2]
    assert fixed_of(text) == [0]
    assert ids_of(text, "EDGE_") == [(0, 1), (1, 2), (2, 0)]


def test_loading_graph(three_pose_loop, tmp_path):
    text = saved(three_pose_loop, tmp_path)
    f = G2oFile.parse(text)
    inf = f.info()
    assert inf["num_vertices"] == 3 and inf["num_edges"] == 3 and inf["num_fixed"] == 1
    g = f.graph()
    assert g.pose_type == abi.POSE_SE2
    assert sorted(map(tuple, g.edge_vertex.tolist())) == [(0, 1), (1, 2), (2, 0)]
    assert list(f.vertex_ids()[0]) == [0, 1, 2]


def test_save_subset_vertices(three_pose_loop, tmp_path):
    text = saved(three_pose_loop, tmp_path, mode=SAVE_VERTEX_SUBSET, ids=[0, 1])
    f = G2oFile.parse(text)
    assert f.info()["num_vertices"] == 2 and f.info()["num_edges"] == 1
    assert list(f.vertex_ids()[0]) == [0, 1]


def test_save_subset_edges(three_pose_loop, tmp_path):
    text = saved(three_pose_loop, tmp_path, mode=SAVE_EDGE_SUBSET, ids=[1])  # the edge (1, 2)
    f = G2oFile.parse(text)
    assert f.info()["num_vertices"] == 2 and f.info()["num_edges"] == 1
    assert ids_of(text, "EDGE_") == [(1, 2)]
    assert list(f.vertex_ids()[0]) == [1, 2]


# ------------------------------------------- library vs oracle on synthetic graphs
def graphs():
    return [("pg2d", synth.pose_graph_2d(num_poses=80, num_closures=30, seed=11)),
            ("pg3d", synth.pose_graph_3d(num_rings=3, per_ring=25, radius=8.0, seed=12)),
            ("ba", synth.bundle_adjustment(num_cameras=10, num_points=250, seed=13)),
            ("pg3d_expmap", synth.pose_graph_3d_expmap(num_rings=3, per_ring=25, radius=8.0, seed=14))]


@pytest.mark.parametrize("name,g", graphs(), ids=[n for n, _ in graphs()])
def test_save_and_load_match_the_oracle(name, g, tmp_path):
    rng = np.random.default_rng(5)
    total = g.num_poses + g.num_points
    ids = rng.permutation(np.arange(total) * 3 + 7)  # gaps, poses and points interleaved in id order
    pid, qid = ids[:g.num_poses], ids[g.num_poses:]
    f = G2oFile.from_graph(g, pid, qid if g.num_points else None, camera_param_id=4)
    text = saved(f, tmp_path)
    og = gt.from_graph(g, pid, qid if g.num_points else None, param_id=4)
    assert text == gt.write(og)
    f2 = G2oFile.parse(text)
    o2 = gt.parse(text)
    c = f2.info()
    for k, v in o2.counts.items():
        assert c[k] == v, k
    og2, opid, oqid = gt.to_graph(o2)
    same_graph(f2.graph(), og2)
    cp, cq = f2.vertex_ids()
    assert list(cp) == opid and list(cq) == oqid
    # a second round trip: an SE2 graph's text is stable (the six-digit
    # rounding happens once); a quaternion written with six digits is not
    # unit length, so SE3 rotations move in the last digit, as in g2o
    again = saved(f2, tmp_path, "again.g2o")
    if name == "pg2d":
        assert again == text
    g3 = G2oFile.parse(again).graph()
    np.testing.assert_allclose(g3.pose_estimate, og2.pose_estimate, rtol=0, atol=2e-5)


def test_estimates_written_back_and_saved(tmp_path):
    g = synth.bundle_adjustment(num_cameras=8, num_points=120, seed=21)
    f = G2oFile.from_graph(g)
    o = gt.from_graph(g)
    rng = np.random.default_rng(2)
    pose = g.pose_estimate.copy()
    pose[:, :3] += rng.normal(0, 0.1, (g.num_poses, 3))
    point = g.point_estimate + rng.normal(0, 0.1, g.point_estimate.shape)
    f.set_estimates(pose, point)
    for i in range(g.num_poses):
        o.vertices[i][1] = [float(x) for x in pose[i]]
    for i in range(g.num_points):
        o.vertices[g.num_poses + i][1] = [float(x) for x in point[i]]
    assert saved(f, tmp_path) == gt.write(o)
    np.testing.assert_array_equal(f.graph().point_estimate, point)


TRICKY = """# comment line
   # indented comment

PARAMS_CAMERAPARAMETERS 0 500 320 240 0.5
PARAMS_CAMERAPARAMETERS 0 400 1 1 0.5
PARAMS_CAMERAPARAMETERS 3 500 320 240
FIX 5
VERTEX_SE3:EXPMAP 5 0.1 0.2 0.3 0 0 0 -1
VERTEX_SE3:EXPMAP\t6\t1 0 0 0.01 0.02 0.03 2.0\r
VERTEX_SE3:EXPMAP 6 0 0 0 0 0 0 1
VERTEX_SE3:EXPMAP -1 0 0 0 0 0 0 1
VERTEX_SE3:EXPMAP 8 0 0 nan 0 0 0 1
VERTEX_SE3:EXPMAP 9 0 0 1e400 0 0 0 1
VERTEX_SE3:EXPMAP 10 +1.5 -.5 2. 0 0 0 1 trailing tokens ignored
VERTEX_TRACKXYZ 20 1 2 10
VERTEX_TRACKXYZ 21 -1 2 12
VERTEX_TRACKXYZ 22 0 0
VERTEX_TRACKXYZ 23 0.5 0.5 9.5
FIX 20 999 21 x 23
VERTEX_XY 30 1 2
ROBOTLASER1 0 0 0
EDGE_PROJECT_XYZ2UV:EXPMAP 20 5 0 320.5 240.25 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 21 6 3 300 200 2 0.5 2
EDGE_PROJECT_XYZ2UV:EXPMAP 23 10 0 310 230 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 20 6 7 1 2 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 20 77 0 1 2 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 5 20 0 1 2 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 20 20 0 1 2 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 23 5 0 1 2 1 0
EDGE_SE2_XY 5 30 1 2 1 0 1
EDGE_PROJECT_XYZ2UV:EXPMAP 21 10 0 3e2 2.1e+2 1 -0.0 1
"""


def test_malformed_and_edge_case_lines_match_the_oracle(tmp_path):
    f = G2oFile.parse(TRICKY)
    o = gt.parse(TRICKY)
    inf = f.info()
    for k, v in o.counts.items():
        assert inf[k] == v, (k, inf[k], v)
    assert inf["first_problem_line"] == o.first_problem_line
    assert inf["num_vertices"] == len(o.vertices) == 6
    assert inf["num_edges"] == len(o.edges) == 4
    assert inf["num_parameters"] == len(o.params) == 2
    assert inf["lines_unsupported"] == 2 and inf["fix_not_found"] == 2 and inf["lines_skipped"] == 1
    og, opid, oqid = gt.to_graph(o)
    same_graph(f.graph(), og)
    assert list(f.vertex_ids()[0]) == opid == [5, 6, 10]
    assert saved(f, tmp_path) == gt.write(o)
    # "FIX 5" came before vertex 5; "FIX 20 999 21 x 23" stops at "x"
    assert list(f.graph().pose_fixed) == [0, 0, 0]
    assert list(f.vertex_ids()[1]) == [20, 21, 23]
    assert list(f.graph().point_fixed) == [1, 1, 0]


def test_se3_pose_graph_quaternions(tmp_path):
    text = ("VERTEX_SE3:QUAT 0 0 0 0 0 0 0 1\n"
            "VERTEX_SE3:QUAT 1 1 2 3 0.1 0.2 0.3 0.927\n"       # not normalized: kept as written
            "EDGE_SE3:QUAT 0 1 1 2 3 0.2 0.4 0.6 1.854 " + " ".join(["1"] + ["0"] * 5 + ["1"] + ["0"] * 4 + ["1"]
                                                                    + ["0"] * 3 + ["1", "0", "0", "1", "0", "1"])
            + "\n")
    f = G2oFile.parse(text)
    o = gt.parse(text)
    og, _, _ = gt.to_graph(o)
    g = f.graph()
    same_graph(g, og)
    # the edge's quaternion is normalized on read (EdgeSE3::read), so its
    # rotation is orthonormal; the vertex's is not
    R = g.measurement[0, :9].reshape(3, 3)
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-15)
    assert np.array_equal(g.information[0].reshape(6, 6), np.eye(6))
    assert saved(f, tmp_path) == gt.write(o)


def test_renamed_types():
    text = "VERTEX_CAM 0 0 0 0\nVERTEX_CAM 1 1 0 0\nODOM 0 1 1 0 0 1 0 0 1 0 1\n"
    spec = "VERTEX_CAM=VERTEX_SE2, ODOM = EDGE_SE2,BAD,X=UNKNOWN_TAG"
    f = G2oFile.parse(text, spec)
    o = gt.parse(text, spec)
    assert f.info()["num_edges"] == 1 and f.info()["num_vertices"] == 2
    same_graph(f.graph(), gt.to_graph(o)[0])
    assert G2oFile.parse(text).info()["lines_unsupported"] == 2


def test_gauge_and_robust_kernel():
    g = synth.bundle_adjustment(num_cameras=6, num_points=60, seed=3)
    g.pose_fixed[:] = 0
    f = G2oFile.from_graph(g, pose_ids=np.arange(6) + 100, point_ids=np.arange(60))
    o = gt.from_graph(g, pose_ids=np.arange(6) + 100, point_ids=np.arange(60))
    # the points (dimension 3) have lower ids; the gauge is a camera
    assert f.fix_gauge() == gt.fix_gauge(o) == 100
    assert f.fix_gauge() == -1
    assert list(f.graph().pose_fixed) == [1, 0, 0, 0, 0, 0]
    f.set_robust_huber(2.5)
    assert np.all(f.graph().robust_delta == 2.5)
    f.set_robust_huber(0.0)
    assert f.graph().robust_delta is None
    pg = G2oFile.parse("VERTEX_SE2 0 0 0 0\nVERTEX_SE2 1 1 0 0\nVERTEX_SE2 2 2 0 0\nVERTEX_SE2 3 2 0 0\n"
                       "EDGE_SE2 0 1 1 0 0 1 0 0 1 0 1\nEDGE_SE2 1 2 1 0 0 1 0 0 1 0 1\n"
                       "EDGE_SE2 3 0 1 0 0 1 0 0 1 0 1\n")
    pg.set_robust_huber(1.0, non_sequential=True)
    assert list(pg.graph().robust_delta) == [0.0, 0.0, 1.0]
    with pytest.raises(G2ocError):
        pg.set_fixed(42)


def test_graphs_the_device_path_cannot_take():
    both = G2oFile.parse("VERTEX_SE2 0 0 0 0\nVERTEX_SE2 1 1 0 0\nEDGE_SE2 0 1 1 0 0 1 0 0 1 0 1\n"
                         "VERTEX_SE3:QUAT 2 0 0 0 0 0 0 1\nVERTEX_SE3:QUAT 3 0 0 0 0 0 0 1\n"
                         "EDGE_SE3:QUAT 2 3 0 0 0 0 0 0 1 " + "1 " * 21 + "\n")
    with pytest.raises(G2ocError) as e:
        both.graph()
    assert e.value.status == abi.G2OC_ERR_NOT_SUPPORTED
    cams = G2oFile.parse("PARAMS_CAMERAPARAMETERS 0 500 320 240 0.5\nPARAMS_CAMERAPARAMETERS 1 400 320 240 0.5\n"
                         "VERTEX_SE3:EXPMAP 0 0 0 0 0 0 0 1\nVERTEX_TRACKXYZ 1 0 0 5\nVERTEX_TRACKXYZ 2 0 1 5\n"
                         "EDGE_PROJECT_XYZ2UV:EXPMAP 1 0 0 1 2 1 0 1\nEDGE_PROJECT_XYZ2UV:EXPMAP 2 0 1 1 2 1 0 1\n")
    with pytest.raises(G2ocError) as e:
        cams.graph()
    assert e.value.status == abi.G2OC_ERR_NOT_SUPPORTED
    empty = G2oFile.parse("VERTEX_SE2 0 0 0 0\n")
    with pytest.raises(G2ocError) as e:
        empty.graph()
    assert e.value.status == abi.G2OC_ERR_BAD_GRAPH
    with pytest.raises(G2ocError):
        G2oFile.load("/nonexistent/file.g2o")
    assert G2oFile.parse("").info()["lines"] == 0


# ------------------------------------------- the command-line optimizer
def run_cli(*args, stdin=None):
    return subprocess.run([CLI, *args], input=stdin, capture_output=True, text=True, timeout=120)


def test_cli_lists_and_refuses(tmp_path):
    r = run_cli("-listSolvers")
    assert r.returncode == 0 and "lm_cuda" in r.stdout.split() and "gn_cuda_chol" in r.stdout.split()
    assert run_cli("-guess", "x.g2o").returncode == 1
    r = run_cli("-solver", "no_such_solver", "x.g2o")
    assert "Error allocating solver" in r.stderr
    p = tmp_path / "mixed.g2o"
    p.write_text("VERTEX_SE2 0 0 0 0\nVERTEX_XY 1 0 0\nEDGE_SE2_XY 0 1 1 1 1 0 1\n")
    assert run_cli("-i", "0", str(p)).returncode == 3
    p.write_text("# nothing\n")
    assert run_cli("-i", "0", str(p)).returncode == 1


def test_cli_zero_iterations_saves_what_g2o_would(tmp_path):
    g = synth.pose_graph_3d(num_rings=2, per_ring=15, radius=5.0, seed=8)
    g.pose_fixed[:] = 0
    src = tmp_path / "in.g2o"
    G2oFile.from_graph(g).save(str(src))
    out = tmp_path / "out.g2o"
    r = run_cli("-i", "0", "-o", str(out), str(src))
    assert r.returncode == 0, r.stderr
    assert "# graph is fixed by node 0" in r.stderr
    o = gt.parse(src.read_text())
    gt.fix_gauge(o)
    assert out.read_text() == gt.write(o)
    r2 = run_cli("-i", "0", "-o", str(tmp_path / "stdin.g2o"), "-", stdin=src.read_text())
    assert r2.returncode == 0 and (tmp_path / "stdin.g2o").read_text() == out.read_text()


# ------------------------------------------- loaded graphs on the device
@pytest.mark.gpu
def test_loaded_pose_graph_optimizes_like_the_oracle(oracle_lib, tmp_path):
    from g2o_b200 import backend
    g = synth.pose_graph_2d(num_poses=400, num_closures=150, seed=31)
    src = str(tmp_path / "pg2d.g2o")
    G2oFile.from_graph(g).save(src)
    f = G2oFile.load(src)
    f.fix_gauge()
    lg = f.graph()
    o = gt.parse(open(src).read())
    gt.fix_gauge(o)
    same_graph(lg, gt.to_graph(o)[0])
    prm = dict(algorithm=abi.ALGO_GAUSS_NEWTON, linear_solver=abi.LINEAR_CHOLESKY)
    c = backend.CudaProblem(lg, backend.default_params(**prm))
    orc = oracle_lib.OracleProblem(lg, oracle_lib.default_params(**prm))
    dc, sc = c.optimize(10)
    do, so = orc.optimize(10)
    assert dc == do == 10
    for a, b in zip(sc, so):
        assert abs(a["chi2"] - b["chi2"]) <= 1e-8 * b["chi2"], (a["chi2"], b["chi2"])
    pose, _ = c.estimates()
    f.set_estimates(pose)
    np.testing.assert_allclose(pose, orc.estimates()[0], rtol=0, atol=1e-8)
    c.close()


@pytest.mark.gpu
def test_cli_optimizes_a_bundle_adjustment_file(oracle_lib, tmp_path):
    g = synth.bundle_adjustment(num_cameras=20, num_points=1500, seed=32)
    src = tmp_path / "ba.g2o"
    G2oFile.from_graph(g).save(str(src))
    out, st = tmp_path / "ba_opt.g2o", tmp_path / "stats.txt"
    r = run_cli("-i", "10", "-v", "-solver", "lm_cuda", "-robustKernel", "Huber", "-robustKernelWidth", "2.447",
                "-o", str(out), "-stats", str(st), str(src))
    assert r.returncode == 0, r.stderr
    lines = [x for x in r.stderr.splitlines() if x.startswith("iteration= ")]
    assert 1 <= len(lines) <= 10 and "levenbergIter=" in lines[0]
    assert len(st.read_text().splitlines()) == len(lines)
    # the oracle on the same loaded graph, gauge and kernel
    f = G2oFile.load(str(src))
    f.fix_gauge()
    f.set_robust_huber(2.447)
    lg = f.graph()
    orc = oracle_lib.OracleProblem(lg, oracle_lib.default_params(algorithm=abi.ALGO_LEVENBERG,
                                                                 linear_solver=abi.LINEAR_PCG))
    done, so = orc.optimize(10)
    assert done == len(lines)
    chi = [float(x.split("chi2= ")[1].split()[0]) for x in lines]
    for a, b in zip(chi, so):
        assert abs(a - b["chi2"]) <= 1e-5 * b["chi2"] + 1e-6, (a, b["chi2"])
    res = G2oFile.load(str(out)).graph()
    pose, point = orc.estimates()
    # the saved file holds six significant digits (camera translations of
    # about 30, written as the inverse pose) on top of the trajectory's own
    # GPU/oracle difference; the initial perturbations are 0.05 and 0.1
    np.testing.assert_allclose(res.point_estimate, point, rtol=1e-5, atol=3e-4)
    np.testing.assert_allclose(res.pose_estimate, pose, rtol=1e-5, atol=1e-3)


@pytest.mark.gpu
def test_cli_compute_marginals(tmp_path):
    g = synth.pose_graph_2d(num_poses=40, num_closures=10, seed=33)
    src = tmp_path / "pg.g2o"
    G2oFile.from_graph(g).save(str(src))
    r = run_cli("-i", "3", "-solver", "gn_cuda_chol", "-computeMarginals", str(src))
    assert r.returncode == 0, r.stderr
    nfree = int((g.pose_fixed == 0).sum())
    assert r.stderr.count("Vertex id:") == nfree
    assert r.stderr.count("inv block :") == 2 * nfree - 1


@pytest.mark.gpu
def test_cli_dogleg_verbose(tmp_path):
    g = synth.pose_graph_2d(num_poses=60, num_closures=20, seed=34)
    src = tmp_path / "pg.g2o"
    G2oFile.from_graph(g).save(str(src))
    r = run_cli("-i", "5", "-v", "-solver", "dl_cuda_chol", "-o", str(tmp_path / "out.g2o"), str(src))
    assert r.returncode == 0, r.stderr
    lines = [x for x in r.stderr.splitlines() if x.startswith("iteration= ")]
    assert lines and all("Delta= " in x and "step= " in x and "tries= " in x for x in lines)


def test_cli_lists_the_new_algorithms_and_round_trips_se3_expmap(tmp_path):
    names = run_cli("-listSolvers").stdout.split()
    for n in ("dl_cuda", "dl_cuda_chol", "structure_only_cuda_3"):
        assert n in names
    g = synth.pose_graph_3d_expmap(num_rings=2, per_ring=12, radius=5.0, seed=9)
    src, out = tmp_path / "in.g2o", tmp_path / "out.g2o"
    G2oFile.from_graph(g).save(str(src))
    assert "EDGE_SE3:EXPMAP" in src.read_text()
    r = run_cli("-i", "0", "-o", str(out), str(src))
    assert r.returncode == 0, r.stderr
    # what g2o writes after reading it back (pose 0 was fixed already); not
    # the input bytes: the six-digit quaternions are not unit length
    assert out.read_text() == gt.write(gt.parse(src.read_text()))


def test_file_entry_points_refuse_bad_arguments(tmp_path, three_pose_loop):
    from g2o_b200.backend import library
    L = library()
    with pytest.raises(G2ocError) as e:
        three_pose_loop.save(str(tmp_path / "x.g2o"), mode=7)
    assert e.value.status == abi.G2OC_ERR_INVALID_ARGUMENT
    with pytest.raises(G2ocError):
        three_pose_loop.save(str(tmp_path / "x.g2o"), mode=SAVE_VERTEX_SUBSET, ids=[0, 99])
    with pytest.raises(G2ocError):
        three_pose_loop.save(str(tmp_path / "x.g2o"), mode=SAVE_EDGE_SUBSET, ids=[3])
    with pytest.raises(G2ocError):
        three_pose_loop.save("/nonexistent/dir/x.g2o")
    bad = abi.Graph(abi.POSE_SE2, abi.EDGE_SE2, np.zeros((2, 3)), [[0, 5]], np.zeros((1, 3)),
                    np.eye(3).reshape(1, 9))
    with pytest.raises(G2ocError):
        G2oFile.from_graph(bad)
    mismatched = abi.Graph(abi.POSE_SE2, abi.EDGE_SE3, np.zeros((2, 3)), [[0, 1]], np.zeros((1, 12)),
                           np.eye(6).reshape(1, 36))
    with pytest.raises(G2ocError):
        G2oFile.from_graph(mismatched)
    with pytest.raises(G2ocError):
        G2oFile.from_graph(abi.Graph(abi.POSE_SE2, abi.EDGE_SE2, np.zeros((2, 3)), [[0, 1]], np.zeros((1, 3)),
                                     np.eye(3).reshape(1, 9)), pose_ids=[4, 4])
    assert L.g2oc_file_get_info(None, None) == abi.G2OC_ERR_INVALID_ARGUMENT
    assert L.g2oc_file_graph(None, None) == abi.G2OC_ERR_INVALID_ARGUMENT
