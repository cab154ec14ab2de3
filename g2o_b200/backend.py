"""Python host side of the B200 solver backend, over the C-ABI of
include/g2o_cuda.h (libg2o_b200.so, built in-tree by g2o_b200/build.py).

It mirrors the reference's plugin interface for this path:

* ``OptimizationAlgorithmFactory.instance().construct(name)`` returns the
  parameters of a registered algorithm ("lm_cuda", "gn_cuda_pcg6_3", ...) or
  ``None`` for an unknown name, as g2o's factory returns nullptr
  (g2o/core/optimization_algorithm_factory.cpp:74-84);
* ``SparseOptimizer`` holds a graph, ``initialize_optimization()`` uploads it
  (initializeOptimization + buildStructure), ``optimize(n)`` runs n outer
  iterations and returns the iteration count (0 on Fail, -1 when not
  initialized), ``active_chi2()`` / ``active_robust_chi2()`` give the chi2.

There is no CPU fallback: if the library or a CUDA device is missing, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import List, Optional

import numpy as np

from .abi import (BA_EDGES, EDGE_PROJECT_XYZ2UV, EDGE_SE3_PROJECT_XYZ, ERROR_NAMES, G2ocBackwardStats, G2ocGraph, G2ocHessianInfo,
                  G2ocIterationStats, G2ocKernelStat, G2ocParams, G2ocWindowStats, Graph, LINEAR_CHOLESKY, LINEAR_PCG,
                  POSE_DIM, POSE_EST_DIM)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libg2o_b200.so")
HEADER_PATH = os.path.join(_HERE, "..", "include", "g2o_cuda.h")
_LIB = None


class G2ocError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{ERROR_NAMES.get(status, status)}: {message}")
        self.status = status


# g2oc_allreduce_fn: (user, device_ptr, count, dtype, op, stream) -> status
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_void_p)
RED_SUM, RED_MAX = 0, 1
DT_F32, DT_F64 = 0, 1


def library() -> C.CDLL:
    """Load libg2o_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with `python -m g2o_b200.build`")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32)
    sig = {
        "g2oc_abi_version": ([], C.c_int),
        "g2oc_last_error": ([], C.c_char_p),
        "g2oc_default_params": ([vp], None),
        "g2oc_list_solvers": ([C.c_char_p, C.c_size_t], C.c_int),
        "g2oc_construct": ([C.c_char_p, vp], C.c_int),
        "g2oc_create": ([C.c_int, C.POINTER(vp)], C.c_int),
        "g2oc_destroy": ([vp], None),
        "g2oc_set_params": ([vp, vp], C.c_int),
        "g2oc_upload": ([vp, vp], C.c_int),
        "g2oc_get_hessian_info": ([vp, vp], C.c_int),
        "g2oc_set_estimates": ([vp, dp, dp], C.c_int),
        "g2oc_download": ([vp, dp, dp], C.c_int),
        "g2oc_optimize": ([vp, C.c_int, vp, C.POINTER(C.c_int)], C.c_int),
        "g2oc_iterate": ([vp, C.c_int, vp, C.POINTER(C.c_int)], C.c_int),
        "g2oc_chi2": ([vp, dp, dp], C.c_int),
        "g2oc_errors": ([vp, dp], C.c_int),
        "g2oc_jacobians": ([vp, dp, dp], C.c_int),
        "g2oc_build_system": ([vp], C.c_int),
        "g2oc_get_pattern": ([vp, ip, ip, ip], C.c_int),
        "g2oc_get_hessian": ([vp, dp, dp, dp, dp], C.c_int),
        "g2oc_schur": ([vp, C.c_double, dp, dp], C.c_int),
        "g2oc_solve": ([vp, C.c_double, dp, ip], C.c_int),
        "g2oc_solver_init": ([vp], C.c_int),
        "g2oc_multiply_hessian": ([vp, dp, dp], C.c_int),
        "g2oc_backward": ([vp, dp, dp, dp, vp], C.c_int),
        "g2oc_upload_windows": ([vp, C.c_int32, vp], C.c_int),
        "g2oc_optimize_windows": ([vp, C.c_int32, vp], C.c_int),
        "g2oc_download_window": ([vp, C.c_int32, dp, dp], C.c_int),
        "g2oc_solve_block_system": ([vp, C.c_int32, C.c_int32, ip, C.c_int32, ip, dp, dp, dp, ip], C.c_int),
        "g2oc_get_stream": ([vp, C.POINTER(vp)], C.c_int),
        "g2oc_restore_initial_estimates": ([vp], C.c_int),
        "g2oc_set_kernel_timing": ([vp, C.c_int], C.c_int),
        "g2oc_get_kernel_stats": ([vp, vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64)], C.c_int),
        "g2oc_solve_block_system_static": ([C.c_int, C.c_int32, C.c_int32, C.c_int32, ip, dp, dp, dp, C.c_double,
                                            C.c_int32, ip], C.c_int),
        "g2oc_set_sharding": ([vp, C.c_int32, C.c_int32, ALLREDUCE_FN, vp], C.c_int),
        "g2oc_compute_marginals": ([vp, C.c_int32, ip, dp], C.c_int),
        "g2oc_structure_only": ([vp, C.c_int32, C.c_int32], C.c_int),
        "g2oc_solve_pattern_block_system": ([vp, C.c_int32, ip, C.c_int32, ip, dp, C.c_int32, ip, dp], C.c_int),
        "g2oc_file_load": ([C.c_char_p, C.c_char_p, C.POINTER(vp)], C.c_int),
        "g2oc_file_parse": ([C.c_char_p, C.c_size_t, C.c_char_p, C.POINTER(vp)], C.c_int),
        "g2oc_file_from_graph": ([vp, ip, ip, C.c_int32, C.POINTER(vp)], C.c_int),
        "g2oc_file_free": ([vp], None),
        "g2oc_file_get_info": ([vp, vp], C.c_int),
        "g2oc_file_graph": ([vp, vp], C.c_int),
        "g2oc_file_vertex_ids": ([vp, ip, ip], C.c_int),
        "g2oc_file_set_fixed": ([vp, C.c_int32, C.c_int32], C.c_int),
        "g2oc_file_fix_gauge": ([vp, ip], C.c_int),
        "g2oc_file_set_robust_huber": ([vp, C.c_double, C.c_int32], C.c_int),
        "g2oc_file_set_estimates": ([vp, dp, dp], C.c_int),
        "g2oc_file_save": ([vp, C.c_char_p, C.c_int32, ip, C.c_int32], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _LIB = L
    return L


def header_symbols(path: Optional[str] = None) -> List[str]:
    """Function names declared in include/*.h (or in the one header given)."""
    inc = os.path.dirname(HEADER_PATH)
    paths = [path] if path else [os.path.join(inc, f) for f in sorted(os.listdir(inc)) if f.endswith(".h")]
    text = "".join(open(p).read() for p in paths)
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(g2oc_\w+)\s*\(", text, re.M)))


def _check(status):
    if status != 0:
        msg = library().g2oc_last_error()
        raise G2ocError(status, msg.decode() if msg else "")


def _p(a, t=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def default_params(**kw) -> G2ocParams:
    p = G2ocParams()
    library().g2oc_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


class OptimizationAlgorithmFactory:
    """Name registry of the backend's algorithms (g2o's OptimizationAlgorithmFactory)."""

    _instance = None

    @classmethod
    def instance(cls):
        if cls._instance is None:
            cls._instance = cls()
        return cls._instance

    def list_solvers(self) -> List[str]:
        buf = C.create_string_buffer(4096)
        _check(library().g2oc_list_solvers(buf, len(buf)))
        return buf.value.decode().split(";")

    def construct(self, name: str) -> Optional[G2ocParams]:
        p = G2ocParams()
        st = library().g2oc_construct(name.encode(), C.byref(p))
        if st != 0:
            return None
        return p


class CudaProblem:
    """One device context holding one graph: the C-ABI handle."""

    def __init__(self, graph: Graph, params: Optional[G2ocParams] = None, device: int = 0, shard=None):
        """shard = (rank, world, allreduce): this rank's part of a sharded
        bundle adjustment (g2oc_set_sharding); allreduce(ptr, count, dtype, op,
        stream) combines count elements at the device address ptr across the
        ranks in place, ordered on the CUDA stream `stream`."""
        self.graph = graph
        self._h = C.c_void_p()
        _check(library().g2oc_create(device, C.byref(self._h)))
        self.params = params or default_params()
        _check(library().g2oc_set_params(self._h, C.byref(self.params)))
        self._reduce_cb = None
        if shard is not None:
            rank, world, fn = shard

            def cb(user, ptr, count, dtype, op, stream):
                try:
                    fn(ptr, int(count), int(dtype), int(op), stream or 0)
                    return 0
                except Exception:  # reported to the C side as a failed all-reduce
                    import traceback
                    traceback.print_exc()
                    return 1

            self._reduce_cb = ALLREDUCE_FN(cb)  # kept alive with the context
            _check(library().g2oc_set_sharding(self._h, rank, world, self._reduce_cb, None))
        self._cg = graph.to_c()
        _check(library().g2oc_upload(self._h, C.byref(self._cg)))
        self.info = G2ocHessianInfo()
        _check(library().g2oc_get_hessian_info(self._h, C.byref(self.info)))

    def upload(self, graph: Graph):
        """Replace the graph (g2oc_upload). A graph with the same topology as
        the current one keeps the index structure and device buffers; only its
        values are copied."""
        cg = graph.to_c()
        _check(library().g2oc_upload(self._h, C.byref(cg)))
        self.graph, self._cg = graph, cg
        _check(library().g2oc_get_hessian_info(self._h, C.byref(self.info)))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            library().g2oc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def is_ba(self):
        return self.graph.edge_type in BA_EDGES

    def set_params(self, params: G2ocParams):
        self.params = params
        _check(library().g2oc_set_params(self._h, C.byref(params)))

    def stream(self) -> int:
        s = C.c_void_p()
        _check(library().g2oc_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def restore_initial_estimates(self):
        _check(library().g2oc_restore_initial_estimates(self._h))

    def set_kernel_timing(self, enable: bool):
        _check(library().g2oc_set_kernel_timing(self._h, 1 if enable else 0))

    def kernel_stats(self):
        arr = (G2ocKernelStat * 64)()
        n = C.c_int()
        tot = C.c_int64()
        _check(library().g2oc_get_kernel_stats(self._h, arr, 64, C.byref(n), C.byref(tot)))
        return tot.value, {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms) for i in range(min(n.value, 64))}

    def estimates(self):
        g = self.graph
        pose = np.empty((g.num_poses, POSE_EST_DIM[g.pose_type]))
        point = np.empty((max(g.num_points, 1), 3))
        _check(library().g2oc_download(self._h, _p(pose), _p(point)))
        return pose, point[: g.num_points]

    def set_estimates(self, pose, point=None):
        pose = np.ascontiguousarray(pose, np.float64)
        pt = None if point is None else np.ascontiguousarray(point, np.float64)
        _check(library().g2oc_set_estimates(self._h, _p(pose), _p(pt)))

    def optimize(self, iterations):
        stats = (G2ocIterationStats * max(iterations, 1))()
        done = C.c_int()
        _check(library().g2oc_optimize(self._h, iterations, stats, C.byref(done)))
        n = done.value if done.value > 0 else iterations
        out = []
        for i in range(iterations):
            if stats[i].levenberg_iterations == 0 and stats[i].time_iteration == 0 and i >= n:
                break
            out.append(stats[i].as_dict())
        return done.value, out

    def iterate(self, iteration):
        st = G2ocIterationStats()
        res = C.c_int()
        _check(library().g2oc_iterate(self._h, iteration, C.byref(st), C.byref(res)))
        return res.value, st.as_dict()

    def chi2(self):
        a, b = C.c_double(), C.c_double()
        _check(library().g2oc_chi2(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def errors(self, with_pose_edges=False):
        """Per active edge errors; with_pose_edges: also those of the pose
        edge set (they follow the projection edges' in the output)."""
        n, D, npe = self.info.num_active_edges, self.graph.edge_dim, self.info.num_active_pose_edges
        buf = np.empty(n * D + npe * 6)
        _check(library().g2oc_errors(self._h, _p(buf)))
        e = buf[: n * D].reshape(n, D)
        return (e, buf[n * D:].reshape(npe, 6)) if with_pose_edges else e

    def jacobians(self):
        D = self.graph.edge_dim
        pd = POSE_DIM[self.graph.pose_type]
        d0 = 3 if self.is_ba else pd
        n = self.info.num_active_edges
        j0, j1 = np.empty((n, D, d0)), np.empty((n, D, pd))
        _check(library().g2oc_jacobians(self._h, _p(j0), _p(j1)))
        return j0, j1

    def build_system(self):
        _check(library().g2oc_build_system(self._h))

    def pattern(self):
        i = self.info
        hpp = np.empty((i.hpp_nnzb, 2), np.int32)
        hpl = np.empty((max(i.hpl_nnzb, 1), 2), np.int32)
        sch = np.empty((max(i.schur_nnzb, 1), 2), np.int32)
        _check(library().g2oc_get_pattern(self._h, _p(hpp, C.c_int32), _p(hpl, C.c_int32), _p(sch, C.c_int32)))
        return hpp, hpl[: i.hpl_nnzb], sch[: i.schur_nnzb]

    def hessian(self):
        i = self.info
        pd = i.pose_dim
        hpp = np.empty((i.hpp_nnzb, pd, pd))
        hll = np.empty((max(i.num_free_points, 1), 3, 3))
        hpl = np.empty((max(i.hpl_nnzb, 1), pd, 3))
        b = np.empty(i.vector_size)
        _check(library().g2oc_get_hessian(self._h, _p(hpp), _p(hll), _p(hpl), _p(b)))
        return hpp, hll[: i.num_free_points], hpl[: i.hpl_nnzb], b

    def schur(self, lam):
        i = self.info
        pd = i.pose_dim
        S = np.empty((i.schur_nnzb, pd, pd))
        bs = np.empty(i.num_free_poses * pd)
        _check(library().g2oc_schur(self._h, lam, _p(S), _p(bs)))
        return S, bs

    def backward(self, dl_dpose, dl_dpoint):
        """g2oc_backward: implicit-function-theorem gradients of a loss on the
        current (converged) estimates with respect to each edge's measurement
        (num_edges x 2) and the log-scale of its information matrix
        (num_edges,). dl_dpose (num_poses x 6, [omega, upsilon] of the
        left-multiplied update) and dl_dpoint (num_points x 3) are dL/dx."""
        g = self.graph
        dx = np.ascontiguousarray(np.concatenate([np.asarray(dl_dpose, np.float64).reshape(-1),
                                                  np.asarray(dl_dpoint, np.float64).reshape(-1)]))
        dmeas = np.zeros((g.num_edges, 2))
        dlogw = np.zeros(g.num_edges)
        st = G2ocBackwardStats()
        _check(library().g2oc_backward(self._h, _p(dx), _p(dmeas), _p(dlogw), C.byref(st)))
        return dmeas, dlogw, {"refinement_steps": st.refinement_steps, "pcg_iterations": st.pcg_iterations,
                              "relative_residual": st.relative_residual}

    def structure_only(self, num_iters=1, num_max_trials=10):
        """StructureOnlySolver<3>::calc on every free landmark, cameras fixed."""
        _check(library().g2oc_structure_only(self._h, int(num_iters), int(num_max_trials)))

    def compute_marginals(self, block_indices):
        """Blocks of Hpp^-1 at the current estimates for (row, col) pairs of
        Hessian block indices (SparseOptimizer::computeMarginals)."""
        idx = np.ascontiguousarray(np.asarray(block_indices, np.int32).reshape(-1, 2))
        pd = self.info.pose_dim
        out = np.zeros((max(len(idx), 1), pd, pd))
        _check(library().g2oc_compute_marginals(self._h, len(idx), _p(idx, C.c_int32), _p(out)))
        return out[:len(idx)]

    def solve(self, lam):
        x = np.empty(self.info.vector_size)
        it = C.c_int32()
        st = library().g2oc_solve(self._h, lam, _p(x), C.byref(it))
        return st, x, it.value

    def solver_init(self):
        """BlockSolver::init -> LinearSolver::init: the next PCG solve carries
        no residual from the previous one."""
        _check(library().g2oc_solver_init(self._h))

    def multiply_hessian(self, src):
        """BlockSolverBase::multiplyHessian: Hpp src (pose part, Hessian order)."""
        src = np.ascontiguousarray(src, np.float64)
        dest = np.empty_like(src)
        _check(library().g2oc_multiply_hessian(self._h, _p(src), _p(dest)))
        return dest


class LinearSolverCudaPCG:
    """LinearSolverPCG's role (g2o/solvers/pcg/linear_solver_pcg.h:44-110):
    block-Jacobi PCG. Inside a BlockSolverCuda it solves the reduced system on
    the device; solve() is LinearSolver<MatrixType>::solve(A, x, b)
    (g2o/core/linear_solver.h:64-65) on a caller block matrix."""

    kind = LINEAR_PCG

    def __init__(self, tolerance=1e-6, max_iterations=-1, absolute_tolerance=True):
        self.tolerance = tolerance
        self.max_iterations = max_iterations
        self.absolute_tolerance = absolute_tolerance

    def params(self, **kw):
        return default_params(linear_solver=self.kind, pcg_tolerance=self.tolerance,
                              pcg_max_iterations=self.max_iterations,
                              pcg_absolute_tolerance=1 if self.absolute_tolerance else 0, **kw)

    def solve(self, block_offsets, block_rc, values, b, device=0):
        st, x, it = solve_block_system(self.kind, block_offsets, block_rc, values, b, self.params(), device)
        return st == 0, x


class LinearSolverCudaCholesky(LinearSolverCudaPCG):
    """LinearSolverEigen / LinearSolverDense's role
    (g2o/solvers/eigen/linear_solver_eigen.h:94-191,
    g2o/solvers/dense/linear_solver_dense.h:57-105): FP64 tiled Cholesky."""

    kind = LINEAR_CHOLESKY

    def __init__(self):
        super().__init__()


class BlockSolverCuda:
    """The Solver interface of g2o's BlockSolver (g2o/core/solver.h:44-153,
    g2o/core/block_solver.h:96-149) over one device context, for an
    OptimizationAlgorithm that drives the solve itself (the algorithm updates
    the host vertices and computes the errors between solves). The graph is
    uploaded by build_structure and the estimates pushed before each
    build_system; the Hessian stays on the device and only b and x cross."""

    def __init__(self, linear_solver: LinearSolverCudaPCG, device: int = 0, **params):
        self.linear_solver = linear_solver
        self.device = device
        self._params = linear_solver.params(**params)
        self._prob: Optional[CudaProblem] = None
        self._lambda = 0.0
        self._schur = True
        self._b = None
        self._x = None

    # Solver::init / buildStructure / updateStructure
    def init(self, graph: Graph, online: bool = False) -> bool:
        self.graph = graph
        if self._prob is not None:
            self._prob.solver_init()
        return True

    def build_structure(self, zero_blocks: bool = False) -> bool:
        if self._prob is None:
            self._prob = CudaProblem(self.graph, self._params, device=self.device)
        else:
            self._prob.upload(self.graph)
        self._prob.solver_init()
        n = self._prob.info.vector_size
        self._x = np.zeros(n)
        self._b = np.zeros(n)
        return True

    def update_structure(self, vset, edges) -> bool:
        return False  # incremental structure updates are not supported (as in LinearSolverPCG-based solvers)

    # Solver::buildSystem at the host estimates
    def build_system(self, pose_estimate, point_estimate=None) -> bool:
        self._prob.set_estimates(pose_estimate, point_estimate)
        self._prob.build_system()
        self._b = self._prob.hessian()[3]
        return True

    # Solver::setLambda / solve / restoreDiagonal
    def set_lambda(self, lam: float, backup: bool = False) -> bool:
        self._lambda = float(lam)
        return True

    def solve(self) -> bool:
        st, x, self.pcg_iterations = self._prob.solve(self._lambda)
        self._x = x
        return st == 0

    def restore_diagonal(self):
        self._lambda = 0.0

    def x(self):
        return self._x

    def b(self):
        return self._b

    def hessian(self):
        return self._prob.hessian()

    def pattern(self):
        return self._prob.pattern()

    def multiply_hessian(self, src):
        return self._prob.multiply_hessian(src)

    def compute_marginals(self, block_indices):
        return self._prob.compute_marginals(block_indices)

    def supports_schur(self) -> bool:
        return True

    def schur(self) -> bool:
        return self._schur

    def set_schur(self, s: bool):
        self._schur = bool(s)

    def close(self):
        if self._prob is not None:
            self._prob.close()
            self._prob = None


def device_tensor(ptr: int, count: int, dtype: int, device: int = 0):
    """A torch tensor viewing count FP32/FP64 elements at a device address
    (the buffers g2oc_allreduce_fn is given); no copy."""
    import torch

    class _View:
        pass

    v = _View()
    v.__cuda_array_interface__ = {"shape": (int(count),), "typestr": "<f4" if dtype == DT_F32 else "<f8",
                                  "data": (int(ptr), False), "version": 3, "strides": None, "stream": None}
    return torch.as_tensor(v, device=f"cuda:{device}")


def split_points(g: Graph, parts: int):
    """The shards of a bundle adjustment: every camera, and the points with
    their edges cut into `parts` contiguous ranges of point index; a pose edge
    set goes to shard 0 alone. Returns the sub-graphs and, per part, the
    original indices of its points."""
    bounds = [round(i * g.num_points / parts) for i in range(parts + 1)]
    out = []
    for r in range(parts):
        p0, p1 = bounds[r], bounds[r + 1]
        sel = (g.edge_vertex[:, 0] >= p0) & (g.edge_vertex[:, 0] < p1)
        ev = g.edge_vertex[sel].copy()
        ev[:, 0] -= p0

        def pick(a, rows=None):
            if a is None:
                return None
            return a[sel].copy() if rows is None else a[rows].copy()

        sub = Graph(g.pose_type, g.edge_type, g.pose_estimate.copy(), ev, pick(g.measurement), pick(g.information),
                    None if g.pose_fixed is None else g.pose_fixed.copy(), g.point_estimate[p0:p1].copy(),
                    None if g.point_fixed is None else g.point_fixed[p0:p1].copy(), pick(g.robust_delta),
                    g.focal_length, tuple(g.principal_point), f"{g.name}-shard{r}", {}, g.focal_length_y,
                    stereo_bf=g.stereo_bf)
        if r == 0 and g.num_pose_edges > 0:
            # camera-side terms: added once, by rank 0, before the ranks sum
            sub.pose_edge_vertex = g.pose_edge_vertex.copy()
            sub.pose_edge_measurement = g.pose_edge_measurement.copy()
            sub.pose_edge_information = g.pose_edge_information.copy()
            if g.pose_edge_robust_delta is not None:
                sub.pose_edge_robust_delta = g.pose_edge_robust_delta.copy()
        out.append((sub, np.arange(p0, p1)))
    return out


class CudaWindows:
    """Many independent bundle-adjustment windows in one context
    (g2oc_upload_windows / g2oc_optimize_windows / g2oc_download_window)."""

    def __init__(self, windows, params: Optional[G2ocParams] = None, device: int = 0):
        self.windows = list(windows)
        self._h = C.c_void_p()
        _check(library().g2oc_create(device, C.byref(self._h)))
        self.params = params or default_params()
        _check(library().g2oc_set_params(self._h, C.byref(self.params)))
        self.upload(self.windows)

    def upload(self, windows):
        """(Re-)upload the windows. The same windows with new values (same
        topology) keep the structure, the tuned dense solve and the captured
        LM round."""
        self.windows = list(windows)
        self._cg = [w.to_c() for w in self.windows]
        arr = (G2ocGraph * len(self._cg))(*self._cg)
        self._arr = arr
        _check(library().g2oc_upload_windows(self._h, len(self._cg), arr))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            library().g2oc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def stream(self) -> int:
        s = C.c_void_p()
        _check(library().g2oc_get_stream(self._h, C.byref(s)))
        return s.value or 0

    def restore_initial_estimates(self):
        _check(library().g2oc_restore_initial_estimates(self._h))

    def optimize(self, iterations):
        st = (G2ocWindowStats * len(self.windows))()
        _check(library().g2oc_optimize_windows(self._h, iterations, st))
        return [s.as_dict() for s in st]

    def estimates(self, w):
        g = self.windows[w]
        pose = np.empty((g.num_poses, 7))
        point = np.empty((max(g.num_points, 1), 3))
        _check(library().g2oc_download_window(self._h, w, _p(pose), _p(point)))
        return pose, point[: g.num_points]

    def estimates_all(self):
        """Every window's (pose, point) estimates from one download."""
        C = sum(g.num_poses for g in self.windows)
        P = sum(g.num_points for g in self.windows)
        pose = np.empty((C, 7))
        point = np.empty((max(P, 1), 3))
        _check(library().g2oc_download(self._h, _p(pose), _p(point)))
        out, c0, p0 = [], 0, 0
        for g in self.windows:
            out.append((pose[c0:c0 + g.num_poses], point[p0:p0 + g.num_points]))
            c0 += g.num_poses
            p0 += g.num_points
        return out

    def set_kernel_timing(self, enable: bool):
        _check(library().g2oc_set_kernel_timing(self._h, 1 if enable else 0))

    def kernel_stats(self):
        arr = (G2ocKernelStat * 64)()
        n = C.c_int()
        tot = C.c_int64()
        _check(library().g2oc_get_kernel_stats(self._h, arr, 64, C.byref(n), C.byref(tot)))
        return tot.value, {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms) for i in range(min(n.value, 64))}


def solve_block_system(linear_solver, block_offsets, block_rc, values, b, params=None, device=0):
    """LinearSolver::solve on a caller block matrix through a fresh context."""
    L = library()
    h = C.c_void_p()
    _check(L.g2oc_create(device, C.byref(h)))
    try:
        if params is not None:
            _check(L.g2oc_set_params(h, C.byref(params)))
        offs = np.ascontiguousarray(block_offsets, np.int32)
        rc = np.ascontiguousarray(block_rc, np.int32)
        vals = np.ascontiguousarray(values, np.float64)
        bb = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(bb)
        it = C.c_int32()
        st = L.g2oc_solve_block_system(h, linear_solver, len(offs) - 1, _p(offs, C.c_int32), len(rc),
                                       _p(rc, C.c_int32), _p(vals), _p(bb), _p(x), C.byref(it))
        return st, x, it.value
    finally:
        L.g2oc_destroy(h)


def solve_pattern_block_system(block_offsets, block_rc, values, block_indices, device=0):
    """LinearSolver::solvePattern on a caller block matrix: the requested
    (row, col) blocks of A^-1, row-major."""
    L = library()
    h = C.c_void_p()
    _check(L.g2oc_create(device, C.byref(h)))
    try:
        offs = np.ascontiguousarray(block_offsets, np.int32)
        rc = np.ascontiguousarray(block_rc, np.int32)
        vals = np.ascontiguousarray(values, np.float64)
        idx = np.ascontiguousarray(np.asarray(block_indices, np.int32).reshape(-1, 2))
        bs = int(offs[1] - offs[0])
        out = np.zeros((max(len(idx), 1), bs, bs))
        st = L.g2oc_solve_pattern_block_system(h, len(offs) - 1, _p(offs, C.c_int32), len(rc), _p(rc, C.c_int32),
                                               _p(vals), len(idx), _p(idx, C.c_int32), _p(out))
        return st, out[:len(idx)]
    finally:
        L.g2oc_destroy(h)


class SparseOptimizer:
    """The reference's SparseOptimizer driving the device algorithm
    (g2o/core/sparse_optimizer.cpp:209-287, 393-455)."""

    def __init__(self, device: int = 0):
        self.device = device
        self.graph: Optional[Graph] = None
        self.params: Optional[G2ocParams] = None
        self._problem: Optional[CudaProblem] = None
        self.batch_statistics = []

    def set_algorithm(self, params: G2ocParams):
        self.params = params
        if self._problem is not None:
            self._problem.set_params(params)

    def set_graph(self, graph: Graph):
        self.graph = graph
        self._problem = None

    def initialize_optimization(self) -> bool:
        if self.graph is None or self.graph.num_edges == 0:
            return False
        self._problem = CudaProblem(self.graph, self.params, self.device)
        return True

    def optimize(self, iterations: int) -> int:
        if self._problem is None:
            return -1
        done, stats = self._problem.optimize(iterations)
        self.batch_statistics = stats
        pose, point = self._problem.estimates()
        self.graph.pose_estimate[...] = pose
        if self.graph.point_estimate is not None:
            self.graph.point_estimate[...] = point
        return done

    def compute_marginals(self, block_indices):
        """SparseOptimizer::computeMarginals (sparse_optimizer.cpp:585-610):
        blocks of Hpp^-1 for (row, col) pairs of Hessian block indices."""
        return self._problem.compute_marginals(block_indices)

    def active_chi2(self) -> float:
        return self._problem.chi2()[0]

    def active_robust_chi2(self) -> float:
        return self._problem.chi2()[1]
