"""ctypes mirror of include/g2o_cuda.h (structs, constants) and the graph
container used to fill a ``g2oc_graph`` from numpy arrays.

The layouts here must match the C header byte for byte; tests/test_abi.py
checks the field offsets against a C compile of the header.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

G2OC_OK = 0
G2OC_ERR_INVALID_ARGUMENT = 1
G2OC_ERR_BAD_GRAPH = 2
G2OC_ERR_CUDA = 3
G2OC_ERR_NOT_PD = 4
G2OC_ERR_NAN = 5
G2OC_ERR_STATE = 6
G2OC_ERR_NO_DEVICE = 7
G2OC_ERR_UNKNOWN_SOLVER = 8
G2OC_ERR_TIMEOUT = 9
G2OC_ERR_NOT_SUPPORTED = 10

ERROR_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "BAD_GRAPH", 3: "CUDA", 4: "NOT_PD", 5: "NAN",
    6: "STATE", 7: "NO_DEVICE", 8: "UNKNOWN_SOLVER", 9: "TIMEOUT", 10: "NOT_SUPPORTED", 11: "NOT_CONVERGED",
}

POSE_SE2, POSE_SE3, POSE_SE3EXPMAP, POSE_BAL_CAMERA = 1, 2, 3, 4
EDGE_SE2, EDGE_SE3, EDGE_PROJECT_XYZ2UV, EDGE_SE3_PROJECT_XYZ, EDGE_SE3_EXPMAP = 1, 2, 3, 4, 5
EDGE_STEREO_SE3_PROJECT_XYZ = 6
EDGE_BAL_OBSERVATION = 7
# projection edges: vertex0 a point, vertex1 a camera
BA_EDGES = (EDGE_PROJECT_XYZ2UV, EDGE_SE3_PROJECT_XYZ, EDGE_STEREO_SE3_PROJECT_XYZ, EDGE_BAL_OBSERVATION)
ALGO_GAUSS_NEWTON, ALGO_LEVENBERG, ALGO_DOGLEG, ALGO_STRUCTURE_ONLY = 0, 1, 2, 3
LINEAR_PCG, LINEAR_CHOLESKY = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
RESULT_OK, RESULT_FAIL, RESULT_TERMINATE = 1, -1, 2

POSE_EST_DIM = {POSE_SE2: 3, POSE_SE3: 12, POSE_SE3EXPMAP: 7, POSE_BAL_CAMERA: 9}
POSE_DIM = {POSE_SE2: 3, POSE_SE3: 6, POSE_SE3EXPMAP: 6, POSE_BAL_CAMERA: 9}
EDGE_DIM = {EDGE_SE2: 3, EDGE_SE3: 6, EDGE_PROJECT_XYZ2UV: 2, EDGE_SE3_PROJECT_XYZ: 2, EDGE_SE3_EXPMAP: 6,
            EDGE_STEREO_SE3_PROJECT_XYZ: 3, EDGE_BAL_OBSERVATION: 2}
MEAS_DIM = {EDGE_SE2: 3, EDGE_SE3: 12, EDGE_PROJECT_XYZ2UV: 2, EDGE_SE3_PROJECT_XYZ: 2, EDGE_SE3_EXPMAP: 7,
            EDGE_STEREO_SE3_PROJECT_XYZ: 3, EDGE_BAL_OBSERVATION: 2}

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_i32p = C.POINTER(C.c_int32)


class G2ocGraph(C.Structure):
    _fields_ = [
        ("pose_type", C.c_int32),
        ("num_poses", C.c_int32),
        ("pose_estimate", _dp),
        ("pose_fixed", _u8p),
        ("num_points", C.c_int32),
        ("point_estimate", _dp),
        ("point_fixed", _u8p),
        ("edge_type", C.c_int32),
        ("num_edges", C.c_int32),
        ("edge_vertex", _i32p),
        ("measurement", _dp),
        ("information", _dp),
        ("robust_delta", _dp),
        ("focal_length", C.c_double),
        ("principal_point", C.c_double * 2),
        ("focal_length_y", C.c_double),
        ("stereo_bf", C.c_double),
        ("num_pose_edges", C.c_int32),
        ("pose_edge_vertex", _i32p),
        ("pose_edge_measurement", _dp),
        ("pose_edge_information", _dp),
        ("pose_edge_robust_delta", _dp),
    ]


class G2ocParams(C.Structure):
    _fields_ = [
        ("algorithm", C.c_int32),
        ("linear_solver", C.c_int32),
        ("precision", C.c_int32),
        ("pcg_max_iterations", C.c_int32),
        ("pcg_tolerance", C.c_double),
        ("pcg_absolute_tolerance", C.c_int32),
        ("max_trials_after_failure", C.c_int32),
        ("initial_lambda", C.c_double),
        ("tau", C.c_double),
        ("refine_max_iterations", C.c_int32),
        ("refine_tolerance", C.c_double),
        ("initial_delta", C.c_double),
        ("lambda_factor", C.c_double),
    ]


class G2ocIterationStats(C.Structure):
    _fields_ = [
        ("iteration", C.c_int32),
        ("result", C.c_int32),
        ("levenberg_iterations", C.c_int32),
        ("iterations_linear_solver", C.c_int32),
        ("chi2", C.c_double),
        ("lambda_", C.c_double),
        ("time_residuals", C.c_double),
        ("time_quadratic_form", C.c_double),
        ("time_schur_complement", C.c_double),
        ("time_linear_solver", C.c_double),
        ("time_update", C.c_double),
        ("time_iteration", C.c_double),
        ("trust_radius", C.c_double),
        ("dogleg_step", C.c_int32),
    ]

    def as_dict(self):
        return {f[0].rstrip("_"): getattr(self, f[0]) for f in self._fields_}


class G2ocKernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("total_ms", C.c_double)]


class G2ocWindowStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("trials", C.c_int32), ("result", C.c_int32), ("solve_ok", C.c_int32),
                ("cholesky_threads", C.c_int32), ("rounds", C.c_int32), ("chi2_initial", C.c_double),
                ("chi2", C.c_double), ("lambda_", C.c_double)]

    def as_dict(self):
        return {"iterations": self.iterations, "trials": self.trials, "result": self.result,
                "solve_ok": self.solve_ok, "cholesky_threads": self.cholesky_threads, "rounds": self.rounds,
                "chi2_initial": self.chi2_initial, "chi2": self.chi2, "lambda": self.lambda_}


class G2ocFileInfo(C.Structure):
    """g2oc_file_info (include/g2o_io.h)."""
    _fields_ = [("num_vertices", C.c_int32), ("num_edges", C.c_int32), ("num_parameters", C.c_int32),
                ("num_fixed", C.c_int32), ("lines", C.c_int32), ("lines_rejected", C.c_int32),
                ("lines_unsupported", C.c_int32), ("lines_skipped", C.c_int32), ("fix_not_found", C.c_int32),
                ("first_problem_line", C.c_int32), ("first_problem", C.c_char * 200)]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        d["first_problem"] = self.first_problem.decode()
        return d


SAVE_ALL, SAVE_VERTEX_SUBSET, SAVE_EDGE_SUBSET = 0, 1, 2


class G2ocBackwardStats(C.Structure):
    _fields_ = [("refinement_steps", C.c_int32), ("pcg_iterations", C.c_int32), ("relative_residual", C.c_double)]


class G2ocHessianInfo(C.Structure):
    _fields_ = [
        ("num_free_poses", C.c_int32),
        ("num_free_points", C.c_int32),
        ("pose_dim", C.c_int32),
        ("point_dim", C.c_int32),
        ("hpp_nnzb", C.c_int32),
        ("hpl_nnzb", C.c_int32),
        ("schur_nnzb", C.c_int32),
        ("num_active_edges", C.c_int32),
        ("vector_size", C.c_int64),
        ("schur_pairs", C.c_int64),
        ("num_active_pose_edges", C.c_int32),
    ]


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


@dataclass
class Graph:
    """A g2o graph in the C-ABI's structure-of-arrays form.

    Vertices are in g2o id order (poses, then points); edges in insertion
    order. ``pose_estimate`` rows follow the vertex type's estimate layout
    (VertexSE2 (x, y, theta); VertexSE3 12 doubles R row-major then t;
    VertexSE3Expmap SE3Quat::toVector).
    """

    pose_type: int
    edge_type: int
    pose_estimate: np.ndarray
    edge_vertex: np.ndarray
    measurement: np.ndarray
    information: np.ndarray
    pose_fixed: Optional[np.ndarray] = None
    point_estimate: Optional[np.ndarray] = None
    point_fixed: Optional[np.ndarray] = None
    robust_delta: Optional[np.ndarray] = None
    focal_length: float = 1.0
    principal_point: tuple = (0.0, 0.0)
    name: str = ""
    extra: dict = field(default_factory=dict)
    focal_length_y: Optional[float] = None  # fy of EdgeSE3ProjectXYZ / EdgeStereoSE3ProjectXYZ (None: focal_length)
    stereo_bf: float = 0.0  # EdgeStereoSE3ProjectXYZ::bf (baseline times fx)
    # EdgeSE3Expmap edges between the cameras of a projection-edge graph
    # (pose indices, SE3Quat::toVector measurement, 6x6 information, Huber deltas)
    pose_edge_vertex: Optional[np.ndarray] = None
    pose_edge_measurement: Optional[np.ndarray] = None
    pose_edge_information: Optional[np.ndarray] = None
    pose_edge_robust_delta: Optional[np.ndarray] = None

    def __post_init__(self):
        self.pose_estimate = np.ascontiguousarray(self.pose_estimate, dtype=np.float64)
        self.edge_vertex = np.ascontiguousarray(self.edge_vertex, dtype=np.int32)
        self.measurement = np.ascontiguousarray(self.measurement, dtype=np.float64)
        self.information = np.ascontiguousarray(self.information, dtype=np.float64)
        if self.pose_fixed is not None:
            self.pose_fixed = np.ascontiguousarray(self.pose_fixed, dtype=np.uint8)
        if self.point_estimate is not None:
            self.point_estimate = np.ascontiguousarray(self.point_estimate, dtype=np.float64)
        if self.point_fixed is not None:
            self.point_fixed = np.ascontiguousarray(self.point_fixed, dtype=np.uint8)
        if self.robust_delta is not None:
            self.robust_delta = np.ascontiguousarray(self.robust_delta, dtype=np.float64)
        if self.pose_edge_vertex is not None:
            self.pose_edge_vertex = np.ascontiguousarray(self.pose_edge_vertex, dtype=np.int32).reshape(-1, 2)
            self.pose_edge_measurement = np.ascontiguousarray(self.pose_edge_measurement, dtype=np.float64)
            self.pose_edge_information = np.ascontiguousarray(self.pose_edge_information, dtype=np.float64)
        if self.pose_edge_robust_delta is not None:
            self.pose_edge_robust_delta = np.ascontiguousarray(self.pose_edge_robust_delta, dtype=np.float64)

    @property
    def num_pose_edges(self) -> int:
        return 0 if self.pose_edge_vertex is None else int(self.pose_edge_vertex.shape[0])

    @property
    def num_poses(self) -> int:
        return int(self.pose_estimate.shape[0])

    @property
    def num_points(self) -> int:
        return 0 if self.point_estimate is None else int(self.point_estimate.shape[0])

    @property
    def num_edges(self) -> int:
        return int(self.edge_vertex.shape[0])

    @property
    def edge_dim(self) -> int:
        return EDGE_DIM[self.edge_type]

    def copy(self) -> "Graph":
        def c(a):
            return None if a is None else a.copy()

        return Graph(self.pose_type, self.edge_type, c(self.pose_estimate), c(self.edge_vertex),
                     c(self.measurement), c(self.information), c(self.pose_fixed),
                     c(self.point_estimate), c(self.point_fixed), c(self.robust_delta),
                     self.focal_length, tuple(self.principal_point), self.name, dict(self.extra),
                     self.focal_length_y, self.stereo_bf, c(self.pose_edge_vertex), c(self.pose_edge_measurement),
                     c(self.pose_edge_information), c(self.pose_edge_robust_delta))

    def digest(self) -> str:
        """SHA-256 of the graph's types, arrays and intrinsics: equal digests
        mean the same optimization problem, bit for bit."""
        import hashlib
        h = hashlib.sha256()
        h.update(np.array([self.pose_type, self.edge_type], np.int64).tobytes())
        for a in (self.pose_estimate, self.edge_vertex, self.measurement, self.information, self.pose_fixed,
                  self.point_estimate, self.point_fixed, self.robust_delta):
            h.update(b"-" if a is None else np.ascontiguousarray(a).tobytes())
        fy = self.focal_length if self.focal_length_y is None else self.focal_length_y
        h.update(np.array([self.focal_length, fy, *self.principal_point], np.float64).tobytes())
        if self.edge_type == EDGE_STEREO_SE3_PROJECT_XYZ:
            h.update(np.array([self.stereo_bf], np.float64).tobytes())
        if self.num_pose_edges:
            for a in (self.pose_edge_vertex, self.pose_edge_measurement, self.pose_edge_information,
                      self.pose_edge_robust_delta):
                h.update(b"-" if a is None else np.ascontiguousarray(a).tobytes())
        return h.hexdigest()

    def to_c(self) -> G2ocGraph:
        g = G2ocGraph()
        g.pose_type = self.pose_type
        g.num_poses = self.num_poses
        g.pose_estimate = _ptr(self.pose_estimate, C.c_double)
        g.pose_fixed = _ptr(self.pose_fixed, C.c_uint8)
        g.num_points = self.num_points
        g.point_estimate = _ptr(self.point_estimate, C.c_double)
        g.point_fixed = _ptr(self.point_fixed, C.c_uint8)
        g.edge_type = self.edge_type
        g.num_edges = self.num_edges
        g.edge_vertex = _ptr(self.edge_vertex, C.c_int32)
        g.measurement = _ptr(self.measurement, C.c_double)
        g.information = _ptr(self.information, C.c_double)
        g.robust_delta = _ptr(self.robust_delta, C.c_double)
        g.focal_length = float(self.focal_length)
        g.principal_point[0] = float(self.principal_point[0])
        g.principal_point[1] = float(self.principal_point[1])
        g.focal_length_y = float(self.focal_length if self.focal_length_y is None else self.focal_length_y)
        g.stereo_bf = float(self.stereo_bf)
        g.num_pose_edges = self.num_pose_edges
        g.pose_edge_vertex = _ptr(self.pose_edge_vertex, C.c_int32)
        g.pose_edge_measurement = _ptr(self.pose_edge_measurement, C.c_double)
        g.pose_edge_information = _ptr(self.pose_edge_information, C.c_double)
        g.pose_edge_robust_delta = _ptr(self.pose_edge_robust_delta, C.c_double)
        # keep the numpy arrays alive as long as the struct
        g._owner = self
        return g
