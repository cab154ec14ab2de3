"""The .g2o text format through the library's loader and saver
(include/g2o_io.h): OptimizableGraph::load / save for the device path's
types (g2o/core/optimizable_graph.cpp:344-610).

    f = G2oFile.load("sphere.g2o")
    f.fix_gauge()
    graph, pose_ids, point_ids = f.graph(), *f.vertex_ids()
    ... optimize graph ...
    f.set_estimates(pose, point)
    f.save("sphere_opt.g2o")
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from .abi import (EDGE_DIM, MEAS_DIM, POSE_EST_DIM, SAVE_ALL, SAVE_EDGE_SUBSET, SAVE_VERTEX_SUBSET, G2ocFileInfo,
                  G2ocGraph, Graph)
from .backend import _check, library

__all__ = ["G2oFile", "SAVE_ALL", "SAVE_VERTEX_SUBSET", "SAVE_EDGE_SUBSET"]


def _enc(s: Optional[str]):
    return None if s is None else s.encode()


class G2oFile:
    """A loaded .g2o graph (g2oc_file handle)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    @classmethod
    def load(cls, path: str, renamed_types: Optional[str] = None) -> "G2oFile":
        h = C.c_void_p()
        _check(library().g2oc_file_load(_enc(path), _enc(renamed_types), C.byref(h)))
        return cls(h)

    @classmethod
    def parse(cls, text: str, renamed_types: Optional[str] = None) -> "G2oFile":
        b = text.encode()
        h = C.c_void_p()
        _check(library().g2oc_file_parse(b, len(b), _enc(renamed_types), C.byref(h)))
        return cls(h)

    @classmethod
    def from_graph(cls, graph: Graph, pose_ids: Optional[Sequence[int]] = None,
                   point_ids: Optional[Sequence[int]] = None, camera_param_id: int = 0) -> "G2oFile":
        """A graph built in code, to save (g2oc_file_from_graph)."""
        ip = C.POINTER(C.c_int32)
        pi = None if pose_ids is None else np.ascontiguousarray(pose_ids, dtype=np.int32)
        qi = None if point_ids is None else np.ascontiguousarray(point_ids, dtype=np.int32)
        cg = graph.to_c()
        h = C.c_void_p()
        _check(library().g2oc_file_from_graph(C.byref(cg), None if pi is None else pi.ctypes.data_as(ip),
                                              None if qi is None else qi.ctypes.data_as(ip), int(camera_param_id),
                                              C.byref(h)))
        return cls(h)

    def close(self):
        if self._h is not None and self._h.value:
            library().g2oc_file_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self) -> dict:
        inf = G2ocFileInfo()
        _check(library().g2oc_file_get_info(self._h, C.byref(inf)))
        return inf.as_dict()

    def graph(self) -> Graph:
        """A copy of the loaded graph (g2oc_file_graph)."""
        g = G2ocGraph()
        _check(library().g2oc_file_graph(self._h, C.byref(g)))
        P, N, E = g.num_poses, g.num_points, g.num_edges
        D, M, pd = EDGE_DIM[g.edge_type], MEAS_DIM[g.edge_type], POSE_EST_DIM[g.pose_type]

        def arr(ptr, n, shape, dtype=np.float64):
            if n == 0 or not ptr:
                return np.zeros(shape, dtype=dtype)
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True).reshape(shape)

        kw = {}
        if N:
            kw = dict(point_estimate=arr(g.point_estimate, N * 3, (N, 3)),
                      point_fixed=arr(g.point_fixed, N, (N,), np.uint8))
        Q = g.num_pose_edges
        if Q:  # EDGE_SE3:EXPMAP edges beside projection edges: the pose edge set
            kw.update(pose_edge_vertex=arr(g.pose_edge_vertex, 2 * Q, (Q, 2), np.int32),
                      pose_edge_measurement=arr(g.pose_edge_measurement, Q * 7, (Q, 7)),
                      pose_edge_information=arr(g.pose_edge_information, Q * 36, (Q, 36)),
                      pose_edge_robust_delta=arr(g.pose_edge_robust_delta, Q, (Q,))
                      if g.pose_edge_robust_delta else None)
        return Graph(g.pose_type, g.edge_type, arr(g.pose_estimate, P * pd, (P, pd)),
                     arr(g.edge_vertex, 2 * E, (E, 2), np.int32), arr(g.measurement, E * M, (E, M)),
                     arr(g.information, E * D * D, (E, D * D)), pose_fixed=arr(g.pose_fixed, P, (P,), np.uint8),
                     robust_delta=arr(g.robust_delta, E, (E,)) if g.robust_delta else None,
                     focal_length=g.focal_length, principal_point=(g.principal_point[0], g.principal_point[1]),
                     **kw)

    def vertex_ids(self):
        g = G2ocGraph()
        _check(library().g2oc_file_graph(self._h, C.byref(g)))
        pose = np.zeros(g.num_poses, dtype=np.int32)
        point = np.zeros(g.num_points, dtype=np.int32)
        ip = C.POINTER(C.c_int32)
        _check(library().g2oc_file_vertex_ids(self._h, pose.ctypes.data_as(ip), point.ctypes.data_as(ip)))
        return pose, point

    def set_fixed(self, vertex_id: int, fixed: bool = True):
        _check(library().g2oc_file_set_fixed(self._h, int(vertex_id), 1 if fixed else 0))

    def fix_gauge(self) -> int:
        """Fix the gauge as g2o_cli does; the fixed vertex id, or -1."""
        gid = C.c_int32()
        _check(library().g2oc_file_fix_gauge(self._h, C.byref(gid)))
        return gid.value

    def set_robust_huber(self, delta: float, non_sequential: bool = False):
        _check(library().g2oc_file_set_robust_huber(self._h, float(delta), 1 if non_sequential else 0))

    def set_estimates(self, pose: np.ndarray, point: Optional[np.ndarray] = None):
        dp = C.POINTER(C.c_double)
        pose = np.ascontiguousarray(pose, dtype=np.float64)
        pt = None if point is None or np.size(point) == 0 else np.ascontiguousarray(point, dtype=np.float64)
        _check(library().g2oc_file_set_estimates(self._h, pose.ctypes.data_as(dp),
                                                 None if pt is None else pt.ctypes.data_as(dp)))

    def save(self, path: str, mode: int = SAVE_ALL, ids: Optional[Sequence[int]] = None):
        a = np.ascontiguousarray(np.asarray([] if ids is None else ids, dtype=np.int32))
        ip = C.POINTER(C.c_int32)
        _check(library().g2oc_file_save(self._h, _enc(path), int(mode), a.ctypes.data_as(ip) if a.size else None,
                                        int(a.size)))
