"""Seeded synthetic graphs for the benchmark configurations.

No dataset is shipped with g2o for this path; these generators follow the
form of the reference's own example generators (g2o/examples/ba/ba_demo.cpp:
cameras on a trajectory looking at a point cloud, Gaussian pixel noise,
outliers handled by a Huber kernel; g2o/examples/sphere/create_sphere.cpp:
rings of SE3 poses with odometry and ring-to-ring edges, noise on the
translation and on the quaternion vector part) with the sizes of the
benchmark configurations:

* ``pose_graph_2d``  3,500 VertexSE2, Manhattan random walk, EdgeSE2 odometry
  and ~2,000 loop closures, GN + Cholesky.
* ``pose_graph_3d``  2,500 VertexSE3 on 10 rings x 250 on a 50 m sphere, EdgeSE3.
* ``bundle_adjustment``  1,000 VertexSE3Expmap on a 30 m ring, 200,000
  VertexPointXYZ in a 20x20x5 m box, ~1.0M EdgeProjectXYZ2UV, Huber.
* ``bal_problem``  the same scene seen by 356 BAL cameras (angle-axis pose,
  focal length, two radial distortion terms), ~227k points, ~1.2M
  EdgeObservationBAL (the shape of the Dubrovnik-356 problem of the BAL
  collection, whose files are not shipped), no robust kernel, nothing fixed.

Every generator takes a seed; the benchmark configurations use
20261203 + configuration index.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import (EDGE_BAL_OBSERVATION, EDGE_PROJECT_XYZ2UV, EDGE_SE2, EDGE_SE3_EXPMAP, EDGE_SE3_PROJECT_XYZ,
                  EDGE_SE3, EDGE_STEREO_SE3_PROJECT_XYZ, POSE_BAL_CAMERA, POSE_SE2, POSE_SE3,
                  POSE_SE3EXPMAP, Graph)

SEED_BASE = 20261203


# ------------------------------------------------------------------ helpers
# sin / cos from +, -, *, / and rint only. Each of those is one IEEE-754
# operation with a correctly rounded result, so the generated graphs are the
# same bits on every CPU; numpy's own float64 sin / cos dispatch to SIMD
# kernels chosen by the CPU's features, whose last bits differ between
# machines (and a last-bit change can flip a visibility decision of the BA
# generator). Range reduction by a two-part pi/2, then the Taylor series to
# r^17 on |r| <= pi/4 (truncation error below 1e-16).
_HALF_PI_HI = 1.5707963267948966
_HALF_PI_LO = 6.123233995736766e-17
_SIN_C = [(-1.0) ** k / math.factorial(2 * k + 1) for k in range(9)]
_COS_C = [(-1.0) ** k / math.factorial(2 * k) for k in range(10)]


def _sincos(x):
    x = np.asarray(x, dtype=np.float64)
    k = np.rint(x / _HALF_PI_HI)
    r = (x - k * _HALF_PI_HI) - k * _HALF_PI_LO
    r2 = r * r
    s = np.full_like(r, _SIN_C[-1])
    for c in reversed(_SIN_C[:-1]):
        s = s * r2 + c
    s = s * r
    c_ = np.full_like(r, _COS_C[-1])
    for c in reversed(_COS_C[:-1]):
        c_ = c_ * r2 + c
    q = np.mod(k, 4.0)
    sin = np.where(q == 0, s, np.where(q == 1, c_, np.where(q == 2, -s, -c_)))
    cos = np.where(q == 0, c_, np.where(q == 1, -s, np.where(q == 2, -c_, s)))
    return sin, cos


def _sin(x):
    return _sincos(x)[0]


def _cos(x):
    return _sincos(x)[1]


def _geometric(rng, p, size, kmax):
    """Geometric draws P(K = k) = (1 - p)^(k - 1) p, truncated at kmax: one
    uniform draw compared with the tails P(K > j) = (1 - p)^j, formed by
    products only (the same bits on every CPU)."""
    u = rng.random(size)
    k = np.ones(size, dtype=np.int64)
    q = 1.0
    for _ in range(1, kmax):
        q = q * (1.0 - p)
        k += (u < q)
    return k

# small-matrix products and norms written out elementwise, in a fixed order
# (numpy's matmul / einsum / norm pick BLAS or SIMD kernels by CPU)
def _mm(A, B):
    """(..., 3, 3) x (..., 3, 3)"""
    return np.stack([np.stack([(A[..., i, 0] * B[..., 0, j] + A[..., i, 1] * B[..., 1, j]) + A[..., i, 2] * B[..., 2, j]
                               for j in range(3)], -1) for i in range(3)], -2)


def _mv(A, v):
    """(..., 3, 3) x (..., 3)"""
    return np.stack([(A[..., i, 0] * v[..., 0] + A[..., i, 1] * v[..., 1]) + A[..., i, 2] * v[..., 2]
                     for i in range(3)], -1)


def _mtv(A, v):
    """(..., 3, 3)^T x (..., 3)"""
    return np.stack([(A[..., 0, i] * v[..., 0] + A[..., 1, i] * v[..., 1]) + A[..., 2, i] * v[..., 2]
                     for i in range(3)], -1)


def _norm(v):
    """Euclidean norm over the last axis (3 or 4 entries)."""
    acc = v[..., 0] * v[..., 0]
    for i in range(1, v.shape[-1]):
        acc = acc + v[..., i] * v[..., i]
    return np.sqrt(acc)


def _wrap(a):
    return (a + np.pi) % (2 * np.pi) - np.pi


def _rot_to_quat(R):
    """Rotation matrices (..., 3, 3) -> quaternions (..., 4) xyzw with w >= 0."""
    R = np.asarray(R, dtype=np.float64)
    q = np.empty(R.shape[:-2] + (4,))
    tr = R[..., 0, 0] + R[..., 1, 1] + R[..., 2, 2]
    w = 0.5 * np.sqrt(np.maximum(1.0 + tr, 0.0))
    x = 0.5 * np.sqrt(np.maximum(1.0 + R[..., 0, 0] - R[..., 1, 1] - R[..., 2, 2], 0.0))
    y = 0.5 * np.sqrt(np.maximum(1.0 - R[..., 0, 0] + R[..., 1, 1] - R[..., 2, 2], 0.0))
    z = 0.5 * np.sqrt(np.maximum(1.0 - R[..., 0, 0] - R[..., 1, 1] + R[..., 2, 2], 0.0))
    x = np.copysign(x, R[..., 2, 1] - R[..., 1, 2])
    y = np.copysign(y, R[..., 0, 2] - R[..., 2, 0])
    z = np.copysign(z, R[..., 1, 0] - R[..., 0, 1])
    q[..., 0], q[..., 1], q[..., 2], q[..., 3] = x, y, z, w
    q /= _norm(q)[..., None]
    return q


def _quat_to_rot(q):
    x, y, z, w = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    R = np.empty(q.shape[:-1] + (3, 3))
    R[..., 0, 0] = 1 - 2 * (y * y + z * z)
    R[..., 0, 1] = 2 * (x * y - z * w)
    R[..., 0, 2] = 2 * (x * z + y * w)
    R[..., 1, 0] = 2 * (x * y + z * w)
    R[..., 1, 1] = 1 - 2 * (x * x + z * z)
    R[..., 1, 2] = 2 * (y * z - x * w)
    R[..., 2, 0] = 2 * (x * z - y * w)
    R[..., 2, 1] = 2 * (y * z + x * w)
    R[..., 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _axis_angle(v):
    """Rodrigues: rotation vectors (..., 3) -> matrices."""
    v = np.asarray(v, dtype=np.float64)
    th = _norm(v)[..., None, None]
    K = np.zeros(v.shape[:-1] + (3, 3))
    K[..., 0, 1], K[..., 0, 2] = -v[..., 2], v[..., 1]
    K[..., 1, 0], K[..., 1, 2] = v[..., 2], -v[..., 0]
    K[..., 2, 0], K[..., 2, 1] = -v[..., 1], v[..., 0]
    with np.errstate(invalid="ignore", divide="ignore"):
        a = np.where(th > 1e-12, _sin(th) / th, 1.0)
        b = np.where(th > 1e-12, (1 - _cos(th)) / (th * th), 0.5)
    return np.eye(3) + a * K + b * _mm(K, K)


_ATAN_C = [(-1.0) ** k / (2 * k + 1) for k in range(14)]


def _atan(x):
    """arctan of x >= 0 from +, -, *, / and sqrt only (each correctly
    rounded, so the same bits on every CPU): x > 1 reflected to 1 / x, three
    half-angle steps atan(y) = 2 atan(y / (1 + sqrt(1 + y^2))) bring the
    argument below tan(pi / 32), then the Taylor series to y^27."""
    x = np.asarray(x, dtype=np.float64)
    inv = x > 1.0
    with np.errstate(divide="ignore"):
        y = np.where(inv, 1.0 / np.where(inv, x, 1.0), x)
    for _ in range(3):
        y = y / (1.0 + np.sqrt(1.0 + y * y))
    y2 = y * y
    s = np.full_like(y, _ATAN_C[-1])
    for c in reversed(_ATAN_C[:-1]):
        s = s * y2 + c
    a = 8.0 * (s * y)
    return np.where(inv, (_HALF_PI_HI - a) + _HALF_PI_LO, a)


def _rot_to_angle_axis(R):
    """Rotation matrices (..., 3, 3) -> angle-axis vectors (..., 3), angle in [0, pi]."""
    q = _rot_to_quat(R)
    v, w = q[..., :3], q[..., 3]
    s = _norm(v)
    with np.errstate(divide="ignore", invalid="ignore"):
        th = np.where(w > 0.0, 2.0 * _atan(s / np.where(w > 0.0, w, 1.0)), np.pi)
        k = np.where(s > 0.0, th / np.where(s > 0.0, s, 1.0), 0.0)
    return v * k[..., None]


def bal_project(cam, X):
    """EdgeObservationBAL's prediction (g2o/examples/bal/bal_example.cpp:160-200)
    for cameras (..., 9) and points (..., 3): Rodrigues rotation, translation,
    p = -P(0:2) / P(2), f (1 + k1 |p|^2 + k2 |p|^4) p."""
    w = cam[..., 0:3]
    th2 = (w[..., 0] * w[..., 0] + w[..., 1] * w[..., 1]) + w[..., 2] * w[..., 2]
    th = np.sqrt(th2)
    safe = np.where(th > 0.0, th, 1.0)
    v = w / safe[..., None]
    sth, cth = _sincos(th)
    vxp = np.stack([v[..., 1] * X[..., 2] - v[..., 2] * X[..., 1], v[..., 2] * X[..., 0] - v[..., 0] * X[..., 2],
                    v[..., 0] * X[..., 1] - v[..., 1] * X[..., 0]], -1)
    vdp = (v[..., 0] * X[..., 0] + v[..., 1] * X[..., 1]) + v[..., 2] * X[..., 2]
    P = (X * cth[..., None] + vxp * sth[..., None]) + (v * vdp[..., None]) * (1.0 - cth)[..., None]
    wxp = np.stack([w[..., 1] * X[..., 2] - w[..., 2] * X[..., 1], w[..., 2] * X[..., 0] - w[..., 0] * X[..., 2],
                    w[..., 0] * X[..., 1] - w[..., 1] * X[..., 0]], -1)
    P = np.where((th2 > 0.0)[..., None], P, X + wxp) + cam[..., 3:6]
    p0, p1 = -P[..., 0] / P[..., 2], -P[..., 1] / P[..., 2]
    r2 = p0 * p0 + p1 * p1
    rp = (1.0 + cam[..., 7] * r2) + (cam[..., 8] * r2) * r2
    fr = cam[..., 6] * rp
    return np.stack([fr * p0, fr * p1], -1)


def _compact_quat_noise(rng, n, sigma):
    """Rotation matrices from a quaternion whose vector part is N(0, sigma)."""
    qv = rng.normal(0.0, sigma, size=(n, 3))
    w = np.sqrt(np.maximum(1.0 - _norm(qv) ** 2, 0.0))
    return _quat_to_rot(np.concatenate([qv, w[:, None]], axis=1))


def _iso12(R, t):
    return np.concatenate([R.reshape(-1, 9), t.reshape(-1, 3)], axis=1)


# ---------------------------------------------------------- 2D pose graph
def pose_graph_2d(num_poses=3500, num_closures=2000, seed=SEED_BASE + 0):
    rng = np.random.default_rng(seed)
    # Manhattan random walk: 1 m steps, turn +-90 deg with p = 0.3
    pos = np.zeros((num_poses, 2))
    th = np.zeros(num_poses)
    for i in range(1, num_poses):
        t = th[i - 1]
        if rng.random() < 0.3:
            t = _wrap(t + (np.pi / 2 if rng.random() < 0.5 else -np.pi / 2))
        th[i] = t
        pos[i] = pos[i - 1] + np.round([math.cos(t), math.sin(t)])
    # candidate loop closures: non-consecutive pairs closer than 1.5 m
    cells = {}
    for i, p in enumerate(np.round(pos).astype(np.int64)):
        cells.setdefault((int(p[0]), int(p[1])), []).append(i)
    cand = []
    for (cx, cy), idx in cells.items():
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                other = cells.get((cx + dx, cy + dy))
                if not other:
                    continue
                for i in idx:
                    for j in other:
                        if j > i + 1 and np.hypot(*(pos[j] - pos[i])) < 1.5:
                            cand.append((i, j))
    cand = np.array(sorted(cand), dtype=np.int64).reshape(-1, 2)
    if len(cand) > num_closures:
        cand = cand[np.sort(rng.choice(len(cand), num_closures, replace=False))]
    pairs = np.concatenate([np.stack([np.arange(num_poses - 1), np.arange(1, num_poses)], 1), cand])
    # true relative poses Xi^-1 Xj
    i, j = pairs[:, 0], pairs[:, 1]
    d = pos[j] - pos[i]
    c, s = _cos(th[i]), _sin(th[i])
    rel = np.stack([c * d[:, 0] + s * d[:, 1], -s * d[:, 0] + c * d[:, 1], _wrap(th[j] - th[i])], 1)
    sig = np.array([0.05, 0.05, 0.01])
    meas = rel + rng.normal(0.0, 1.0, size=rel.shape) * sig
    meas[:, 2] = _wrap(meas[:, 2])
    info = np.tile(np.diag(1.0 / sig ** 2).reshape(1, 9), (len(pairs), 1))
    # initial guess: compose noisy odometry
    est = np.zeros((num_poses, 3))
    est[0] = [pos[0, 0], pos[0, 1], th[0]]
    for k in range(num_poses - 1):
        x, y, t = est[k]
        m = meas[k]
        est[k + 1] = [x + math.cos(t) * m[0] - math.sin(t) * m[1],
                      y + math.sin(t) * m[0] + math.cos(t) * m[1], _wrap(t + m[2])]
    fixed = np.zeros(num_poses, np.uint8)
    fixed[0] = 1
    g = Graph(POSE_SE2, EDGE_SE2, est, pairs.astype(np.int32), meas, info, pose_fixed=fixed,
              name=f"pose_graph_2d_{num_poses}")
    g.extra["truth"] = np.stack([pos[:, 0], pos[:, 1], th], 1)
    return g


# ---------------------------------------------------------- 3D pose graph
def pose_graph_3d(num_rings=10, per_ring=250, radius=50.0, seed=SEED_BASE + 1):
    rng = np.random.default_rng(seed)
    n = num_rings * per_ring
    R = np.zeros((n, 3, 3))
    t = np.zeros((n, 3))
    for k in range(num_rings):
        pol = np.pi * (k + 1) / (num_rings + 1)
        for j in range(per_ring):
            az = 2 * np.pi * j / per_ring
            idx = k * per_ring + j
            t[idx] = radius * np.array([_sin(pol) * _cos(az), _sin(pol) * _sin(az), _cos(pol)])
            R[idx] = _mm(_axis_angle(np.array([0.0, 0.0, az + np.pi / 2])), _axis_angle(np.array([pol - np.pi / 2, 0, 0])))
    edges = []
    for k in range(num_rings):
        base = k * per_ring
        for j in range(per_ring - 1):
            edges.append((base + j, base + j + 1))
        if k + 1 < num_rings:
            edges.append((base + per_ring - 1, base + per_ring))  # chain to the next ring
    odo = len(edges)
    for k in range(num_rings):
        base = k * per_ring
        edges.append((base, base + per_ring - 1))  # ring closure
    for k in range(num_rings - 1):
        a, b = k * per_ring, (k + 1) * per_ring
        nxt = t[b:b + per_ring]
        for j in range(per_ring):
            jj = int(np.argmin(_norm(nxt - t[a + j])))
            edges.append((a + j, b + jj))
    edges = np.array(edges, dtype=np.int64)
    i, j = edges[:, 0], edges[:, 1]
    Rt = np.transpose(R[i], (0, 2, 1))
    relR = _mm(Rt, R[j])
    relt = _mv(Rt, t[j] - t[i])
    sig_t, sig_r = 0.01, 0.005
    nR = _compact_quat_noise(rng, len(edges), sig_r)
    nt = rng.normal(0.0, sig_t, size=(len(edges), 3))
    mR = _mm(relR, nR)
    mt = relt + _mv(relR, nt)
    meas = _iso12(mR, mt)
    info = np.tile(np.diag([1 / sig_t ** 2] * 3 + [1 / (sig_r ** 2)] * 3).reshape(1, 36), (len(edges), 1))
    # initial guess: compose the noisy chain
    eR = np.zeros((n, 3, 3))
    et = np.zeros((n, 3))
    eR[0], et[0] = R[0], t[0]
    for k in range(odo):
        a, b = edges[k]
        eR[b] = _mm(eR[a], mR[k])
        et[b] = et[a] + _mv(eR[a], mt[k])
    fixed = np.zeros(n, np.uint8)
    fixed[0] = 1
    g = Graph(POSE_SE3, EDGE_SE3, _iso12(eR, et), edges.astype(np.int32), meas, info, pose_fixed=fixed,
              name=f"pose_graph_3d_{n}")
    g.extra["truth"] = _iso12(R, t)
    return g


def pose_graph_3d_expmap(num_rings=10, per_ring=250, radius=50.0, seed=SEED_BASE + 1):
    """The 3D pose graph as VertexSE3Expmap / EdgeSE3Expmap: T_i = X_i^-1
    (world to body) and C_ij = Z_ij^-1, so that log(T_j^-1 C_ij T_i) is the
    edge error; the information blocks reordered to (rotation, translation),
    the order of SE3Quat::log."""
    g = pose_graph_3d(num_rings, per_ring, radius, seed)

    def se3quat_of_inverse(iso):
        R = iso[:, :9].reshape(-1, 3, 3)
        t = iso[:, 9:]
        Rt = np.transpose(R, (0, 2, 1))
        return np.concatenate([-_mv(Rt, t), _rot_to_quat(Rt)], axis=1)

    perm = [3, 4, 5, 0, 1, 2]
    info = g.information.reshape(-1, 6, 6)[:, perm][:, :, perm].reshape(-1, 36)
    out = Graph(POSE_SE3EXPMAP, EDGE_SE3_EXPMAP, se3quat_of_inverse(g.pose_estimate), g.edge_vertex.copy(),
                se3quat_of_inverse(g.measurement), info, pose_fixed=g.pose_fixed.copy(),
                name=g.name.replace("pose_graph_3d", "pose_graph_3d_expmap"))
    out.extra["truth"] = se3quat_of_inverse(g.extra["truth"])
    return out


# ------------------------------------------------------ bundle adjustment
def _look_at(centers, target):
    fwd = target[None, :] - centers
    fwd /= _norm(fwd)[:, None]
    up = np.array([0.0, 0.0, 1.0])
    x = np.cross(fwd, up)
    x /= _norm(x)[:, None]
    y = np.cross(fwd, x)
    Rcw = np.stack([x, y, fwd], axis=1)  # rows: camera axes in world
    tcw = -_mv(Rcw, centers)
    return Rcw, tcw


def bundle_adjustment(num_cameras=1000, num_points=200_000, ring_radius=30.0, height=1.5,
                      box=(10.0, 10.0, 5.0), mean_obs=5.0, min_obs=2, max_obs=20,
                      focal=500.0, width=640, height_px=480, pixel_noise=1.0, outlier_ratio=0.01,
                      pose_noise=(0.05, 0.01), point_noise=0.1, num_fixed=2,
                      seed=SEED_BASE + 2, chunk=2048, focal_y=None):
    """Ring of inward-looking cameras observing a box of points (ba_demo form).
    With focal_y the edges are EdgeSE3ProjectXYZ with fx = focal, fy = focal_y
    (ORB-SLAM's form); otherwise EdgeProjectXYZ2UV with one focal length."""
    fy = focal if focal_y is None else focal_y
    rng = np.random.default_rng(seed)
    az = 2 * np.pi * np.arange(num_cameras) / num_cameras
    centers = np.stack([ring_radius * _cos(az), ring_radius * _sin(az), np.full(num_cameras, height)], 1)
    Rcw, tcw = _look_at(centers, np.array([0.0, 0.0, box[2] / 2]))
    X = np.stack([rng.uniform(-box[0], box[0], num_points), rng.uniform(-box[1], box[1], num_points),
                  rng.uniform(0.0, box[2], num_points)], 1)
    cx, cy = width / 2.0, height_px / 2.0
    kdraw = np.clip(_geometric(rng, 1.0 / mean_obs, num_points, max_obs), min_obs, max_obs)
    pts, cams, uvs = [], [], []
    for s in range(0, num_points, chunk):
        Xs = X[s:s + chunk]
        # camera coordinates of every point of the chunk in every camera
        Xc = np.stack([((Xs[:, None, 0] * Rcw[None, :, i, 0] + Xs[:, None, 1] * Rcw[None, :, i, 1])
                        + Xs[:, None, 2] * Rcw[None, :, i, 2]) + tcw[None, :, i] for i in range(3)], -1)
        z = Xc[..., 2]
        with np.errstate(divide="ignore", invalid="ignore"):
            u = focal * Xc[..., 0] / z + cx
            v = fy * Xc[..., 1] / z + cy
        vis = (z > 0.5) & (u >= 0) & (u < width) & (v >= 0) & (v < height_px)
        keys = rng.random(vis.shape)
        keys[~vis] = 2.0
        m = min(max_obs, num_cameras)
        cand = np.argpartition(keys, m - 1, axis=1)[:, :m]
        ck = np.take_along_axis(keys, cand, axis=1)
        cand = np.take_along_axis(cand, np.argsort(ck, axis=1), axis=1)
        k = np.minimum(kdraw[s:s + chunk], vis.sum(axis=1))
        k[k < 2] = 0
        take = np.arange(m)[None, :] < k[:, None]
        cand = np.where(take, cand, num_cameras)
        cand.sort(axis=1)  # cameras ascending within a point
        rows, cols = np.nonzero(cand < num_cameras)
        sel = cand[rows, cols]
        pts.append(s + rows)
        cams.append(sel)
        uvs.append(np.stack([u[rows, sel], v[rows, sel]], 1))
    pts = np.concatenate(pts)
    cams = np.concatenate(cams)
    uv = np.concatenate(uvs) + rng.normal(0.0, pixel_noise, size=(len(pts), 2))
    out = rng.random(len(pts)) < outlier_ratio
    uv[out] = np.stack([rng.uniform(0, width, out.sum()), rng.uniform(0, height_px, out.sum())], 1)
    # keep only observed points, renumbered in order
    used = np.unique(pts)
    remap = -np.ones(num_points, np.int64)
    remap[used] = np.arange(len(used))
    pts = remap[pts]
    Xt = X[used]
    # initial guess
    dR = _axis_angle(rng.normal(0.0, pose_noise[1], size=(num_cameras, 3)))
    dt = rng.normal(0.0, pose_noise[0], size=(num_cameras, 3))
    R0 = _mm(dR, Rcw)
    t0 = _mv(dR, tcw) + dt
    fixed = np.zeros(num_cameras, np.uint8)
    fixed[:num_fixed] = 1
    R0[:num_fixed], t0[:num_fixed] = Rcw[:num_fixed], tcw[:num_fixed]
    pose_est = np.concatenate([t0, _rot_to_quat(R0)], axis=1)
    X0 = Xt + rng.normal(0.0, point_noise, size=Xt.shape)
    E = len(pts)
    info = np.tile(np.eye(2).reshape(1, 4), (E, 1))
    g = Graph(POSE_SE3EXPMAP, EDGE_PROJECT_XYZ2UV if focal_y is None else EDGE_SE3_PROJECT_XYZ, pose_est,
              np.stack([pts, cams], 1).astype(np.int32), uv, info, pose_fixed=fixed,
              point_estimate=X0, point_fixed=np.zeros(len(Xt), np.uint8),
              robust_delta=np.full(E, math.sqrt(5.991)), focal_length=focal,
              principal_point=(cx, cy), name=f"bundle_adjustment_{num_cameras}x{len(Xt)}", focal_length_y=focal_y)
    g.extra["truth_pose"] = np.concatenate([tcw, _rot_to_quat(Rcw)], axis=1)
    g.extra["truth_point"] = Xt
    g.extra["outliers"] = out
    return g


def stereo_bundle_adjustment(num_cameras=100, num_points=20_000, baseline=0.12, focal=500.0, right_noise=0.5,
                             seed=SEED_BASE + 5, **kw):
    """EdgeStereoSE3ProjectXYZ (ORB-SLAM's stereo form): the ring bundle
    adjustment with fx = fy = focal and a right-image coordinate per
    observation, u_r = u - bf / z with bf = baseline * focal (z the true
    depth), plus its own pixel noise; information I_3, Huber on every edge."""
    g = bundle_adjustment(num_cameras=num_cameras, num_points=num_points, focal=focal, focal_y=focal, seed=seed, **kw)
    rng = np.random.default_rng(seed + 7919)
    tp, X = g.extra["truth_pose"], g.extra["truth_point"]
    R = _quat_to_rot(tp[:, 3:7])
    pts, cams = g.edge_vertex[:, 0], g.edge_vertex[:, 1]
    z = ((R[cams, 2, 0] * X[pts, 0] + R[cams, 2, 1] * X[pts, 1]) + R[cams, 2, 2] * X[pts, 2]) + tp[cams, 2]
    bf = baseline * focal
    E = g.num_edges
    meas = np.empty((E, 3))
    meas[:, :2] = g.measurement
    meas[:, 2] = g.measurement[:, 0] - bf / z + rng.normal(0.0, right_noise, E)
    info = np.tile(np.eye(3).reshape(1, 9), (E, 1))
    s = Graph(POSE_SE3EXPMAP, EDGE_STEREO_SE3_PROJECT_XYZ, g.pose_estimate, g.edge_vertex, meas, info,
              pose_fixed=g.pose_fixed, point_estimate=g.point_estimate, point_fixed=g.point_fixed,
              robust_delta=np.full(E, math.sqrt(7.815)), focal_length=focal, principal_point=g.principal_point,
              name=f"stereo_bundle_adjustment_{num_cameras}x{g.num_points}", focal_length_y=focal, stereo_bf=bf)
    s.extra = dict(g.extra)
    return s


def bal_problem(num_cameras=356, num_points=226_730, mean_obs=5.5, focal=500.0, k1=(-0.05, 0.05),
                k2=(-0.01, 0.01), pixel_noise=1.0, pose_noise=(0.05, 0.01), focal_noise=0.01, point_noise=0.1,
                seed=SEED_BASE + 6, **kw):
    """A BAL problem (g2o/examples/bal/bal_example.cpp: VertexCameraBAL,
    VertexPointBAL, EdgeObservationBAL, identity information, no robust
    kernel, no fixed vertex) on the ring scene of bundle_adjustment: the same
    visibility, the cameras turned half a turn about their x axis (BAL
    cameras look down -z, image y up), measurements from the BAL projection
    with per-camera focal length and radial distortion plus pixel noise. The
    initial guess perturbs the angle-axis, translation and focal length and
    starts the distortion at zero."""
    g = bundle_adjustment(num_cameras=num_cameras, num_points=num_points, mean_obs=mean_obs, focal=focal,
                          pixel_noise=0.0, outlier_ratio=0.0, num_fixed=0, seed=seed, **kw)
    rng = np.random.default_rng(seed + 104729)
    tp, X = g.extra["truth_pose"], g.extra["truth_point"]
    flip = np.diag([1.0, -1.0, -1.0])
    Rb = _mm(np.broadcast_to(flip, (num_cameras, 3, 3)), _quat_to_rot(tp[:, 3:7]))
    tb = tp[:, :3] * np.array([1.0, -1.0, -1.0])
    cam = np.empty((num_cameras, 9))
    cam[:, 0:3] = _rot_to_angle_axis(Rb)
    cam[:, 3:6] = tb
    cam[:, 6] = focal * (1.0 + rng.uniform(-0.02, 0.02, num_cameras))
    cam[:, 7] = rng.uniform(k1[0], k1[1], num_cameras)
    cam[:, 8] = rng.uniform(k2[0], k2[1], num_cameras)
    pts, cams = g.edge_vertex[:, 0], g.edge_vertex[:, 1]
    E = g.num_edges
    meas = bal_project(cam[cams], X[pts]) + rng.normal(0.0, pixel_noise, size=(E, 2))
    cam0 = cam.copy()
    cam0[:, 0:3] += rng.normal(0.0, pose_noise[1], size=(num_cameras, 3))
    cam0[:, 3:6] += rng.normal(0.0, pose_noise[0], size=(num_cameras, 3))
    cam0[:, 6] *= 1.0 + rng.normal(0.0, focal_noise, num_cameras)
    cam0[:, 7:9] = 0.0
    X0 = X + rng.normal(0.0, point_noise, size=X.shape)
    info = np.tile(np.eye(2).reshape(1, 4), (E, 1))
    b = Graph(POSE_BAL_CAMERA, EDGE_BAL_OBSERVATION, cam0, g.edge_vertex, meas, info,
              pose_fixed=np.zeros(num_cameras, np.uint8), point_estimate=X0,
              point_fixed=np.zeros(len(X), np.uint8), name=f"bal_{num_cameras}x{len(X)}")
    b.extra["truth_pose"] = cam
    b.extra["truth_point"] = X
    return b


def ba_with_odometry(num_cameras=40, num_points=3000, rot_sigma=0.01, trans_sigma=0.05, seed=SEED_BASE + 7, **kw):
    """The ring bundle adjustment with a second edge set: EdgeSE3Expmap
    odometry between consecutive cameras of the ring (and the last to the
    first). The measurement is C_ij = T_j E T_i^-1 from the generating poses
    with E = (R(w), u), w ~ N(0, rot_sigma^2), u ~ N(0, trans_sigma^2), so that
    the edge error log(T_j^-1 C_ij T_i) = log(E) is that noise (to first
    order), with information diag(1 / rot_sigma^2 x3, 1 / trans_sigma^2 x3) in
    (omega, upsilon) order and no robust kernel: the graph of a visual SLAM
    back end with odometry."""
    g = bundle_adjustment(num_cameras=num_cameras, num_points=num_points, seed=seed, **kw)
    add_odometry(g, rot_sigma, trans_sigma, seed + 15485863)
    g.name = g.name.replace("bundle_adjustment", "ba_odometry")
    return g


def add_odometry(g, rot_sigma=0.01, trans_sigma=0.05, seed=SEED_BASE + 7 + 15485863):
    """Attach the ring odometry of ba_with_odometry to a projection-edge graph
    whose extra["truth_pose"] holds its generating SE3Quat cameras."""
    num_cameras = g.num_poses
    rng = np.random.default_rng(seed)
    tp = g.extra["truth_pose"]
    R = _quat_to_rot(tp[:, 3:7])
    t = tp[:, :3]
    i = np.arange(num_cameras)
    j = (i + 1) % num_cameras
    RE = _axis_angle(rng.normal(0.0, rot_sigma, size=(num_cameras, 3)))
    tE = rng.normal(0.0, trans_sigma, size=(num_cameras, 3))
    Rit = np.transpose(R[i], (0, 2, 1))
    A = _mm(RE, Rit)  # E T_i^-1: rotation RE Ri^T, translation -RE Ri^T t_i + tE
    a = -_mv(A, t[i]) + tE
    Rc = _mm(R[j], A)
    tc = _mv(R[j], a) + t[j]
    info = np.diag([1.0 / rot_sigma ** 2] * 3 + [1.0 / trans_sigma ** 2] * 3).reshape(1, 36)
    g.pose_edge_vertex = np.stack([i, j], 1).astype(np.int32)
    g.pose_edge_measurement = np.concatenate([tc, _rot_to_quat(Rc)], axis=1)
    g.pose_edge_information = np.tile(info, (num_cameras, 1))
    g.pose_edge_robust_delta = None
    return g


def window_sizes(num_windows=512, cameras=(10, 60), points=(500, 8000), seed=SEED_BASE + 1000):
    """(cameras, points) of each window: log-uniform in the given ranges."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(num_windows):
        nc = int(round(math.exp(rng.uniform(math.log(cameras[0]), math.log(cameras[1])))))
        npt = int(round(math.exp(rng.uniform(math.log(points[0]), math.log(points[1])))))
        out.append((nc, npt))
    return out


def windows(num_windows=512, cameras=(10, 60), points=(500, 8000), obs=(2, 8), seed=SEED_BASE + 1000, which=None):
    """Local bundle-adjustment windows of uneven size: cameras and points
    log-uniform in the given ranges, each point seen by obs[0]..obs[1] cameras
    of its window; the BA generator (ring cameras, box points, 1 px noise, 1%
    outliers, Huber) seeded per window. `which`: the indices to generate
    (default all); window w is the same whichever others are generated."""
    sizes = window_sizes(num_windows, cameras, points, seed)
    idx = range(num_windows) if which is None else which
    return [bundle_adjustment(num_cameras=sizes[w][0], num_points=sizes[w][1], min_obs=obs[0], max_obs=obs[1],
                              seed=seed + 1 + w) for w in idx]


def adjoint_problem(num_cameras=200, num_points=40_000, seed=SEED_BASE + 4, robust=False):
    """The adjoint instance: the BA generator without outliers (and, unless
    asked, without a robust kernel), 200 cameras / 40k points by default."""
    g = bundle_adjustment(num_cameras=num_cameras, num_points=num_points, outlier_ratio=0.0, seed=seed)
    if not robust:
        g.robust_delta = None
    return g


def camera_centres(pose_est):
    """World positions of VertexSE3Expmap cameras (t, q world->camera): -R^T t."""
    t = pose_est[:, :3]
    q = pose_est[:, 3:7]  # x y z w
    R = _quat_to_rot(q)
    return -_mtv(R, t), R


def centre_loss(pose_est, truth_pose):
    """L = sum_i |c_i - c_i^truth|^2 and dL/dx in the update coordinates of
    VertexSE3Expmap (T <- exp([omega, upsilon]) T): dL/domega = 0,
    dL/dupsilon = -2 R (c - c^truth)."""
    c, R = camera_centres(pose_est)
    ct, _ = camera_centres(truth_pose)
    d = c - ct
    grad = np.zeros((len(pose_est), 6))
    grad[:, 3:] = -2.0 * _mv(R, d)
    return float((d * d).sum()), grad


CONFIGS = {
    "pg2d": lambda: pose_graph_2d(),
    "pg3d": lambda: pose_graph_3d(),
    "ba": lambda: bundle_adjustment(),
    "bal": lambda: bal_problem(),
}
