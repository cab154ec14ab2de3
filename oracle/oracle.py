"""TEST INFRASTRUCTURE ONLY: ctypes loader of the FP64 CPU restatement
(oracle/liboracle.so, built from oracle/g2o_oracle.cpp by oracle/Makefile).

Used by tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() as
the checker; never by the product library.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from g2o_b200.abi import (BA_EDGES, EDGE_PROJECT_XYZ2UV, EDGE_SE3_PROJECT_XYZ, G2ocHessianInfo, G2ocIterationStats, G2ocParams,
                          Graph, POSE_DIM, POSE_EST_DIM)

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp = C.c_void_p
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        L.orc_create.argtypes = [C.c_void_p, C.POINTER(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_destroy.restype = None
        L.orc_set_params.argtypes = [vp, C.c_void_p]
        L.orc_default_params.argtypes = [C.c_void_p]
        L.orc_default_params.restype = None
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_hessian_info.argtypes = [vp, C.c_void_p]
        L.orc_set_estimates.argtypes = [vp, dp, dp]
        L.orc_download.argtypes = [vp, dp, dp]
        L.orc_optimize.argtypes = [vp, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.orc_chi2.argtypes = [vp, dp, dp]
        L.orc_errors.argtypes = [vp, dp]
        L.orc_jacobians.argtypes = [vp, dp, dp]
        L.orc_numeric_jacobians.argtypes = [vp, dp, dp]
        L.orc_build_system.argtypes = [vp]
        L.orc_get_pattern.argtypes = [vp, ip, ip, ip]
        L.orc_get_hessian.argtypes = [vp, dp, dp, dp, dp]
        L.orc_schur.argtypes = [vp, C.c_double, dp, dp]
        L.orc_solve.argtypes = [vp, C.c_double, dp, ip]
        L.orc_update.argtypes = [vp, dp]
        L.orc_solve_block_system.argtypes = [C.c_int32, C.c_void_p, C.c_int32, ip, C.c_int32, ip, dp, dp, dp, ip]
        L.orc_huber.argtypes = [C.c_double, C.c_double, dp]
        L.orc_huber.restype = None
        L.orc_compute_dq_dR.argtypes = [dp, dp]
        L.orc_compute_dq_dR.restype = None
        L.orc_rot_to_quat.argtypes = [dp, dp]
        L.orc_rot_to_quat.restype = None
        L.orc_se3quat_exp.argtypes = [dp, dp]
        L.orc_se3quat_exp.restype = None
        L.orc_normalize_theta.argtypes = [C.c_double]
        L.orc_normalize_theta.restype = C.c_double
        _LIB = L
    return _LIB


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def _check(st, what):
    if st != 0:
        raise RuntimeError(f"oracle {what} failed with status {st}")


def default_params(**kw) -> G2ocParams:
    p = G2ocParams()
    lib().orc_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class OracleProblem:
    """The oracle's SparseOptimizer + algorithm for one graph."""

    def __init__(self, graph: Graph, params: G2ocParams | None = None, threads: int = 1):
        self.graph = graph
        self._h = C.c_void_p()
        self._cg = graph.to_c()
        lib().orc_set_threads(threads)
        _check(lib().orc_create(C.byref(self._cg), C.byref(self._h)), "create")
        self.params = params or default_params()
        _check(lib().orc_set_params(self._h, C.byref(self.params)), "set_params")
        self.info = G2ocHessianInfo()
        _check(lib().orc_get_hessian_info(self._h, C.byref(self.info)), "info")

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().orc_destroy(self._h)
            self._h = C.c_void_p()

    def set_params(self, params: G2ocParams):
        self.params = params
        _check(lib().orc_set_params(self._h, C.byref(params)), "set_params")

    @property
    def is_ba(self):
        return self.graph.edge_type in BA_EDGES

    def estimates(self):
        g = self.graph
        pose = np.empty((g.num_poses, POSE_EST_DIM[g.pose_type]))
        point = np.empty((max(g.num_points, 1), 3))
        _check(lib().orc_download(self._h, _p(pose), _p(point)), "download")
        return pose, point[: g.num_points]

    def set_estimates(self, pose, point=None):
        pose = np.ascontiguousarray(pose, np.float64)
        pt = None if point is None else np.ascontiguousarray(point, np.float64)
        _check(lib().orc_set_estimates(self._h, _p(pose), None if pt is None else _p(pt)), "set_estimates")

    def optimize(self, iterations):
        stats = (G2ocIterationStats * max(iterations, 1))()
        done = C.c_int()
        _check(lib().orc_optimize(self._h, iterations, stats, C.byref(done)), "optimize")
        return done.value, [stats[i].as_dict() for i in range(min(iterations, max(done.value, 0)) or 0)] \
            if done.value > 0 else [stats[i].as_dict() for i in range(iterations)]

    def chi2(self):
        a, b = C.c_double(), C.c_double()
        _check(lib().orc_chi2(self._h, C.byref(a), C.byref(b)), "chi2")
        return a.value, b.value

    def errors(self, with_pose_edges=False):
        """Per active edge errors; with_pose_edges: also those of the pose
        edge set (they follow the projection edges' in the output)."""
        n, D, npe = self.info.num_active_edges, self.graph.edge_dim, self.info.num_active_pose_edges
        buf = np.empty(n * D + npe * 6)
        _check(lib().orc_errors(self._h, _p(buf)), "errors")
        e = buf[: n * D].reshape(n, D)
        return (e, buf[n * D:].reshape(npe, 6)) if with_pose_edges else e

    def _jac_shapes(self):
        D = self.graph.edge_dim
        pd = POSE_DIM[self.graph.pose_type]
        d0 = 3 if self.is_ba else pd
        n = self.info.num_active_edges
        return (n, D, d0), (n, D, pd)

    def jacobians(self, numeric=False):
        s0, s1 = self._jac_shapes()
        j0, j1 = np.empty(s0), np.empty(s1)
        f = lib().orc_numeric_jacobians if numeric else lib().orc_jacobians
        _check(f(self._h, _p(j0), _p(j1)), "jacobians")
        return j0, j1

    def build_system(self):
        _check(lib().orc_build_system(self._h), "build_system")

    def pattern(self):
        i = self.info
        hpp = np.empty((i.hpp_nnzb, 2), np.int32)
        hpl = np.empty((max(i.hpl_nnzb, 1), 2), np.int32)
        sch = np.empty((max(i.schur_nnzb, 1), 2), np.int32)
        _check(lib().orc_get_pattern(self._h, _p(hpp, C.c_int32), _p(hpl, C.c_int32), _p(sch, C.c_int32)), "pattern")
        return hpp, hpl[: i.hpl_nnzb], sch[: i.schur_nnzb]

    def hessian(self):
        i = self.info
        pd = i.pose_dim
        hpp = np.empty((i.hpp_nnzb, pd, pd))
        hll = np.empty((max(i.num_free_points, 1), 3, 3))
        hpl = np.empty((max(i.hpl_nnzb, 1), pd, 3))
        b = np.empty(i.vector_size)
        _check(lib().orc_get_hessian(self._h, _p(hpp), _p(hll), _p(hpl), _p(b)), "hessian")
        return hpp, hll[: i.num_free_points], hpl[: i.hpl_nnzb], b

    def schur(self, lam):
        i = self.info
        pd = i.pose_dim
        S = np.empty((i.schur_nnzb, pd, pd))
        bs = np.empty(i.num_free_poses * pd)
        _check(lib().orc_schur(self._h, lam, _p(S), _p(bs)), "schur")
        return S, bs

    def solve(self, lam):
        x = np.empty(self.info.vector_size)
        it = C.c_int32()
        st = lib().orc_solve(self._h, lam, _p(x), C.byref(it))
        return st, x, it.value

    def update(self, x):
        """SparseOptimizer::update(x) on the oracle's vertices."""
        x = np.ascontiguousarray(x, np.float64)
        _check(lib().orc_update(self._h, _p(x)), "update")


def solve_block_system(linear_solver, block_offsets, block_rc, values, b, params=None):
    block_offsets = np.ascontiguousarray(block_offsets, np.int32)
    block_rc = np.ascontiguousarray(block_rc, np.int32)
    values = np.ascontiguousarray(values, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    it = C.c_int32()
    prm = params or default_params()
    st = lib().orc_solve_block_system(linear_solver, C.byref(prm), len(block_offsets) - 1, _p(block_offsets, C.c_int32),
                                      len(block_rc), _p(block_rc, C.c_int32), _p(values), _p(b), _p(x), C.byref(it))
    return st, x, it.value


def huber(e2, delta):
    r = np.empty(3)
    lib().orc_huber(e2, delta, _p(r))
    return r


def dq_dR(R):
    R = np.ascontiguousarray(R, np.float64)
    out = np.empty(27)
    lib().orc_compute_dq_dR(_p(R), _p(out))
    return out.reshape(3, 9)


def rot_to_quat(R):
    R = np.ascontiguousarray(R, np.float64)
    q = np.empty(4)
    lib().orc_rot_to_quat(_p(R), _p(q))
    return q


def se3quat_exp(u):
    u = np.ascontiguousarray(u, np.float64)
    o = np.empty(7)
    lib().orc_se3quat_exp(_p(u), _p(o))
    return o


def normalize_theta(t):
    return lib().orc_normalize_theta(float(t))
