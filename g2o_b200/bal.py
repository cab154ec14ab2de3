"""Bundle Adjustment in the Large (BAL) problem files, the input of
g2o/examples/bal/bal_example.cpp (its parser: bal_example.cpp:264-330).

The text format: a header line "num_cameras num_points num_observations";
one line per observation "camera_index point_index x y"; then the 9
parameters of every camera (angle-axis rx ry rz, translation tx ty tz, focal
length f, radial distortion k1 k2), then the 3 coordinates of every point,
all whitespace-separated. The example builds one VertexCameraBAL per
camera (ids 0..C-1), one marginalized VertexPointBAL per point (ids C..),
one EdgeObservationBAL per observation with identity information and no
robust kernel, and fixes no vertex; read_bal returns that problem as a
Graph of this package's BAL types (edge_vertex rows are (point, camera)).

    g = read_bal("problem-49-7776-pre.txt")
    write_bal(g, "out.txt")
"""
from __future__ import annotations

import numpy as np

from .abi import EDGE_BAL_OBSERVATION, POSE_BAL_CAMERA, Graph

__all__ = ["read_bal", "write_bal", "parse_bal"]


def parse_bal(text: str, name: str = "bal") -> Graph:
    tok = text.split()
    if len(tok) < 3:
        raise ValueError("BAL file: missing header")
    nc, npt, nobs = int(tok[0]), int(tok[1]), int(tok[2])
    if nc <= 0 or npt < 0 or nobs <= 0:
        raise ValueError(f"BAL file: bad sizes {nc} cameras, {npt} points, {nobs} observations")
    need = 3 + 4 * nobs + 9 * nc + 3 * npt
    if len(tok) < need:
        raise ValueError(f"BAL file: {len(tok)} values, {need} expected")
    obs = np.array(tok[3:3 + 4 * nobs], dtype=np.float64).reshape(nobs, 4)
    cam_idx = obs[:, 0].astype(np.int64)
    pt_idx = obs[:, 1].astype(np.int64)
    if (cam_idx < 0).any() or (cam_idx >= nc).any() or (pt_idx < 0).any() or (pt_idx >= npt).any():
        raise ValueError("BAL file: observation index out of bounds")
    o = 3 + 4 * nobs
    cams = np.array(tok[o:o + 9 * nc], dtype=np.float64).reshape(nc, 9)
    o += 9 * nc
    pts = np.array(tok[o:o + 3 * npt], dtype=np.float64).reshape(npt, 3)
    ev = np.stack([pt_idx, cam_idx], 1).astype(np.int32)
    return Graph(POSE_BAL_CAMERA, EDGE_BAL_OBSERVATION, cams, ev, obs[:, 2:4].copy(),
                 np.tile(np.eye(2).reshape(1, 4), (nobs, 1)), pose_fixed=np.zeros(nc, np.uint8),
                 point_estimate=pts, point_fixed=np.zeros(npt, np.uint8), name=name)


def read_bal(path: str) -> Graph:
    with open(path) as f:
        return parse_bal(f.read(), name=path)


def write_bal(g: Graph, path: str):
    """The graph's BAL problem (estimates as they stand) in the BAL format."""
    if g.pose_type != POSE_BAL_CAMERA or g.edge_type != EDGE_BAL_OBSERVATION:
        raise ValueError("write_bal takes a BAL graph")
    ev = g.edge_vertex
    with open(path, "w") as f:
        f.write(f"{g.num_poses} {g.num_points} {g.num_edges}\n")
        for k in range(g.num_edges):
            f.write(f"{int(ev[k, 1])} {int(ev[k, 0])} {float(g.measurement[k, 0])!r} {float(g.measurement[k, 1])!r}\n")
        for c in g.pose_estimate:
            f.write("\n".join(repr(float(v)) for v in c) + "\n")
        for p in g.point_estimate:
            f.write("\n".join(repr(float(v)) for v in p) + "\n")
