"""TEST INFRASTRUCTURE ONLY: a plain-Python restatement of g2o's text format
for the device path's types, the checker of the library's .g2o loader and
saver (include/g2o_io.h). Pure-Python loops: meant for small files.

Follows (paths relative to the g2o source tree):
  OptimizableGraph::load(istream)       g2o/core/optimizable_graph.cpp:344-522
  OptimizableGraph::save / saveSubset   g2o/core/optimizable_graph.cpp:539-606, 736-780
  setRenamedTypesFromString             g2o/core/optimizable_graph.cpp:619-644
  ParameterContainer::write             g2o/core/parameter_container.cpp:82-91
  readInformationMatrix / write         g2o/core/base_edge.h:165-180
  VertexSE2 / EdgeSE2 read, write       g2o/types/slam2d/vertex_se2.cpp:40-49, edge_se2.cpp:38-50
  VertexSE3 / EdgeSE3 read, write       g2o/types/slam3d/vertex_se3.cpp:46-55, edge_se3.cpp:43-58
  toVectorQT / fromVectorQT             g2o/types/slam3d/isometry3d_mappings.cpp:111-142
  VertexPointXYZ read, write            g2o/types/slam3d/vertex_pointxyz.cpp:40-46
  VertexSE3Expmap read, write           g2o/types/sba/vertex_se3_expmap.cpp:35-44
  SE3Quat(Vector7), inverse, normalizeRotation   g2o/types/slam3d/se3quat.h:64-86, 114-119, 251-256
  EdgeProjectXYZ2UV read, write         g2o/types/sba/edge_project_xyz2uv.cpp:38-48
  EdgeSE3Expmap read, write             g2o/types/sba/edge_se3_expmap.cpp:33-43
  CameraParameters read, write          g2o/types/sba/parameter_cameraparameters.cpp:33-57
  gaugeFreedom / findGauge              g2o/core/sparse_optimizer.cpp:132-173

The malformed-input rules (refused lines, type checks) and the orders the
reference leaves to pointer or hash order are those include/g2o_io.h states.
"""
from __future__ import annotations

import math
import re

import numpy as np

from g2o_b200.abi import (EDGE_PROJECT_XYZ2UV, EDGE_SE2, EDGE_SE3, EDGE_SE3_EXPMAP, POSE_SE2, POSE_SE3,
                          POSE_SE3EXPMAP, Graph)

VERTEX_TAGS = {"VERTEX_SE2": "se2", "VERTEX_SE3:QUAT": "se3", "VERTEX_SE3:EXPMAP": "expmap", "VERTEX_TRACKXYZ": "xyz"}
EDGE_TAGS = {"EDGE_SE2": "se2", "EDGE_SE3:QUAT": "se3", "EDGE_PROJECT_XYZ2UV:EXPMAP": "proj",
             "EDGE_SE3:EXPMAP": "se3exp"}
CAMERA_TAG = "PARAMS_CAMERAPARAMETERS"
TAG_OF_VERTEX = {v: k for k, v in VERTEX_TAGS.items()}
TAG_OF_EDGE = {v: k for k, v in EDGE_TAGS.items()}
_FLOAT = re.compile(r"[+-]?(\d+\.?\d*|\.\d+)([eE][+-]?\d+)?$")
_INT = re.compile(r"[+-]?\d+$")
_SPACE = re.compile(r"[ \t\r\v\f]+")


# ------------------------------------------------------------------ rotations
def quat_to_rot(x, y, z, w):
    tx, ty, tz = 2 * x, 2 * y, 2 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return [1 - (tyy + tzz), txy - twz, txz + twy,
            txy + twz, 1 - (txx + tzz), tyz - twx,
            txz - twy, tyz + twx, 1 - (txx + tyy)]


def rot_to_quat(R):
    """Shepperd's method, largest-diagonal branch; returns [x, y, z, w]."""
    q = [0.0, 0.0, 0.0, 0.0]
    t = R[0] + R[4] + R[8]
    if t > 0:
        t = math.sqrt(t + 1.0)
        q[3] = 0.5 * t
        t = 0.5 / t
        q[0] = (R[7] - R[5]) * t
        q[1] = (R[2] - R[6]) * t
        q[2] = (R[3] - R[1]) * t
    else:
        i = 0
        if R[4] > R[0]:
            i = 1
        if R[8] > R[i * 4]:
            i = 2
        j = (i + 1) % 3
        k = (j + 1) % 3
        t = math.sqrt(R[i * 4] - R[j * 4] - R[k * 4] + 1.0)
        q[i] = 0.5 * t
        t = 0.5 / t
        q[3] = (R[k * 3 + j] - R[j * 3 + k]) * t
        q[j] = (R[j * 3 + i] + R[i * 3 + j]) * t
        q[k] = (R[k * 3 + i] + R[i * 3 + k]) * t
    return q


def quat_normalize(q):
    n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]
    if n2 > 0:
        n = math.sqrt(n2)
        return [c / n for c in q]
    return list(q)


def quat_rotate(q, v):
    uv = [q[1] * v[2] - q[2] * v[1], q[2] * v[0] - q[0] * v[2], q[0] * v[1] - q[1] * v[0]]
    uv = [c + c for c in uv]
    return [v[0] + q[3] * uv[0] + (q[1] * uv[2] - q[2] * uv[1]),
            v[1] + q[3] * uv[1] + (q[2] * uv[0] - q[0] * uv[2]),
            v[2] + q[3] * uv[2] + (q[0] * uv[1] - q[1] * uv[0])]


def se3quat_inverse(v):
    qc = [-v[3], -v[4], -v[5], v[6]]
    t = quat_rotate(qc, [v[0] * -1.0, v[1] * -1.0, v[2] * -1.0])
    return t + qc


def iso_to_qt(iso):
    q = quat_normalize(rot_to_quat(iso[:9]))
    return [iso[9], iso[10], iso[11]] + q


# ------------------------------------------------------------------ parsing
def _num(tok):
    if tok is None or not _FLOAT.match(tok):
        return None
    v = float(tok)
    return v if math.isfinite(v) else None


def _int(tok):
    if tok is None or not _INT.match(tok):
        return None
    v = int(tok)
    return v if -2**31 <= v < 2**31 else None


class TextGraph:
    """Parameters, vertices (id -> [kind, estimate list, fixed]) and edges
    ([kind, id0, id1, param, measurement list, D*D information list, delta])
    in load order, plus the load counters."""

    def __init__(self):
        self.params = {}
        self.vertices = {}
        self.vorder = []
        self.edges = []
        self.counts = dict(lines=0, lines_rejected=0, lines_unsupported=0, lines_skipped=0, fix_not_found=0)
        self.first_problem_line = 0

    def _problem(self, lineno, key):
        self.counts[key] += 1
        if self.first_problem_line == 0:
            self.first_problem_line = lineno


def _renames(spec):
    out = {}
    if not spec:
        return out
    for item in spec.split(","):
        if item.count("=") != 1:
            continue
        a, b = (s.strip(" \t\n") for s in item.split("="))
        if b in VERTEX_TAGS or b in EDGE_TAGS or b == CAMERA_TAG:
            out[a] = b
    return out


def parse(text: str, renamed_types: str = None) -> TextGraph:
    g = TextGraph()
    ren = _renames(renamed_types)
    lines = text.split("\n")
    if lines and lines[-1] == "":
        lines.pop()
    for lineno, line in enumerate(lines, 1):
        g.counts["lines"] = lineno
        toks = [t for t in _SPACE.split(line) if t]
        if not toks or toks[0].startswith("#"):
            continue
        tag, rest = toks[0], toks[1:]
        if tag == "FIX":
            for t in rest:
                vid = _int(t)
                if vid is None:
                    break
                if vid in g.vertices:
                    g.vertices[vid][2] = 1
                else:
                    g.counts["fix_not_found"] += 1
            continue
        tag = ren.get(tag, tag)
        it = iter(rest)
        nxt = lambda: next(it, None)  # noqa: E731
        if tag == CAMERA_TAG:
            pid = _int(nxt())
            vals = [_num(nxt()) for _ in range(3)]
            if pid is None or None in vals:
                g._problem(lineno, "lines_rejected")
                continue
            bl = _num(nxt())
            if pid in g.params:
                g._problem(lineno, "lines_rejected")
                continue
            g.params[pid] = vals + [0.5 if bl is None else bl]
            continue
        if tag in VERTEX_TAGS:
            kind = VERTEX_TAGS[tag]
            vid = _int(nxt())
            n = 7 if kind in ("se3", "expmap") else 3
            vals = [_num(nxt()) for _ in range(n)]
            if vid is None or None in vals or vid < 0 or vid in g.vertices:
                g._problem(lineno, "lines_rejected")
                continue
            if kind == "se3":
                est = quat_to_rot(vals[3], vals[4], vals[5], vals[6]) + vals[:3]
            elif kind == "expmap":
                q = vals[3:7]
                if q[3] < 0:
                    q = [c * -1 for c in q]
                q = quat_normalize(q)
                est = se3quat_inverse(vals[:3] + q)
            else:
                est = vals
            g.vertices[vid] = [kind, est, 0]
            g.vorder.append(vid)
            continue
        if tag in EDGE_TAGS:
            kind = EDGE_TAGS[tag]
            i0, i1 = _int(nxt()), _int(nxt())
            if i0 is None or i1 is None or i0 not in g.vertices or i1 not in g.vertices or i0 == i1:
                g._problem(lineno, "lines_rejected")
                continue
            k0, k1 = g.vertices[i0][0], g.vertices[i1][0]
            ok = (kind == "se2" and k0 == k1 == "se2") or (kind == "se3" and k0 == k1 == "se3") or \
                 (kind == "proj" and k0 == "xyz" and k1 == "expmap") or (kind == "se3exp" and k0 == k1 == "expmap")
            if not ok:
                g._problem(lineno, "lines_rejected")
                continue
            pid = -1
            if kind == "proj":
                pid = _int(nxt())
                if pid is None:
                    g._problem(lineno, "lines_rejected")
                    continue
            nm, D = {"se2": (3, 3), "se3": (7, 6), "proj": (2, 2), "se3exp": (7, 6)}[kind]
            m = [_num(nxt()) for _ in range(nm)]
            up = [_num(nxt()) for _ in range(D * (D + 1) // 2)]
            if None in m or None in up or (kind == "proj" and pid not in g.params):
                g._problem(lineno, "lines_rejected")
                continue
            info = [0.0] * (D * D)
            k = 0
            for i in range(D):
                for j in range(i, D):
                    info[i * D + j] = info[j * D + i] = up[k]
                    k += 1
            if kind == "se3":
                q = quat_normalize(m[3:7])
                m = quat_to_rot(*q) + m[:3]
            elif kind == "se3exp":
                q = m[3:7]
                if q[3] < 0:
                    q = [c * -1 for c in q]
                m = se3quat_inverse(m[:3] + quat_normalize(q))
            g.edges.append([kind, i0, i1, pid, m, info, 0.0])
            continue
        if tag.startswith("VERTEX_") or tag.startswith("EDGE_"):
            g._problem(lineno, "lines_unsupported")
            continue
        g.counts["lines_skipped"] += 1
    return g


# ------------------------------------------------------------------ graph view
def to_graph(g: TextGraph):
    """(Graph, pose_ids, point_ids) as g2oc_file_graph / g2oc_file_vertex_ids
    return them; None when there is no edge or more than one edge type."""
    kinds = {e[0] for e in g.edges}
    if len(kinds) != 1:
        return None
    ek = kinds.pop()
    pk = {"se2": "se2", "se3": "se3", "proj": "expmap", "se3exp": "expmap"}[ek]
    pose_ids = sorted(v for v, r in g.vertices.items() if r[0] == pk)
    point_ids = sorted(v for v, r in g.vertices.items() if r[0] == "xyz") if ek == "proj" else []
    pidx = {v: i for i, v in enumerate(pose_ids)}
    qidx = {v: i for i, v in enumerate(point_ids)}
    ev = []
    for e in g.edges:
        ev.append([qidx[e[1]], pidx[e[2]]] if ek == "proj" else [pidx[e[1]], pidx[e[2]]])
    deltas = [e[6] for e in g.edges]
    kw = {}
    if ek == "proj":
        cam = g.params[g.edges[0][3]]
        kw = dict(point_estimate=np.array([g.vertices[v][1] for v in point_ids], dtype=np.float64).reshape(-1, 3),
                  point_fixed=np.array([g.vertices[v][2] for v in point_ids], dtype=np.uint8),
                  focal_length=cam[0], principal_point=(cam[1], cam[2]))
    gr = Graph({"se2": POSE_SE2, "se3": POSE_SE3, "expmap": POSE_SE3EXPMAP}[pk],
               {"se2": EDGE_SE2, "se3": EDGE_SE3, "proj": EDGE_PROJECT_XYZ2UV, "se3exp": EDGE_SE3_EXPMAP}[ek],
               np.array([g.vertices[v][1] for v in pose_ids], dtype=np.float64),
               np.array(ev, dtype=np.int32).reshape(-1, 2),
               np.array([e[4] for e in g.edges], dtype=np.float64),
               np.array([e[5] for e in g.edges], dtype=np.float64),
               pose_fixed=np.array([g.vertices[v][2] for v in pose_ids], dtype=np.uint8),
               robust_delta=np.array(deltas, dtype=np.float64) if any(d > 0 for d in deltas) else None, **kw)
    return gr, pose_ids, point_ids


def fix_gauge(g: TextGraph):
    dim = {"se2": 3, "xyz": 3, "se3": 6, "expmap": 6}
    maxd = max(dim[r[0]] for r in g.vertices.values())
    cand = sorted(v for v, r in g.vertices.items() if dim[r[0]] == maxd)
    if any(g.vertices[v][2] for v in cand):
        return -1
    g.vertices[cand[0]][2] = 1
    return cand[0]


# ------------------------------------------------------------------ writing
def _f(v):
    return "%g " % v


def _vertex_line(vid, rec):
    kind, est, fixed = rec
    if kind == "se3":
        vals = iso_to_qt(est)
    elif kind == "expmap":
        vals = se3quat_inverse(est)
    else:
        vals = est
    s = TAG_OF_VERTEX[kind] + " " + "%d " % vid + "".join(_f(x) for x in vals) + "\n"
    if fixed:
        s += "FIX %d\n" % vid
    return s


def _edge_line(e):
    kind, i0, i1, pid, m, info, _ = e
    s = TAG_OF_EDGE[kind] + " " + "%d %d " % (i0, i1)
    if kind == "proj":
        s += "%d " % pid
    s += "".join(_f(x) for x in (iso_to_qt(m) if kind == "se3" else se3quat_inverse(m) if kind == "se3exp" else m))
    D = {"se2": 3, "se3": 6, "proj": 2, "se3exp": 6}[kind]
    s += "".join(_f(info[i * D + j]) for i in range(D) for j in range(i, D))
    return s + "\n"


def write(g: TextGraph, mode: int = 0, ids=()) -> str:
    """save (mode 0), saveSubset(VertexSet) (1, vertex ids), saveSubset(EdgeSet) (2, edge indices)."""
    out = []
    for pid in sorted(g.params):
        out.append(CAMERA_TAG + " " + "%d " % pid + "".join(_f(x) for x in g.params[pid]) + "\n")
    if mode == 0:
        vs = {v for e in g.edges for v in (e[1], e[2])}
        es = list(range(len(g.edges)))
    elif mode == 1:
        vs = set(ids)
        es = [k for k, e in enumerate(g.edges) if e[1] in vs and e[2] in vs]
    else:
        es = sorted(set(ids))
        vs = {v for k in es for v in (g.edges[k][1], g.edges[k][2])}
    for v in sorted(vs):
        out.append(_vertex_line(v, g.vertices[v]))
    for k in es:
        out.append(_edge_line(g.edges[k]))
    return "".join(out)


def from_graph(gr: Graph, pose_ids=None, point_ids=None, param_id: int = 0) -> TextGraph:
    """A TextGraph holding a graph built in code (g2oc_file_from_graph)."""
    g = TextGraph()
    pk = {POSE_SE2: "se2", POSE_SE3: "se3", POSE_SE3EXPMAP: "expmap"}[gr.pose_type]
    ek = {EDGE_SE2: "se2", EDGE_SE3: "se3", EDGE_PROJECT_XYZ2UV: "proj", EDGE_SE3_EXPMAP: "se3exp"}[gr.edge_type]
    P, N = gr.num_poses, gr.num_points
    pid = list(range(P)) if pose_ids is None else [int(v) for v in pose_ids]
    qid = list(range(P, P + N)) if point_ids is None else [int(v) for v in point_ids]
    for i in range(P):
        fx = 0 if gr.pose_fixed is None else int(gr.pose_fixed[i] != 0)
        g.vertices[pid[i]] = [pk, [float(x) for x in gr.pose_estimate[i]], fx]
        g.vorder.append(pid[i])
    for i in range(N):
        fx = 0 if gr.point_fixed is None else int(gr.point_fixed[i] != 0)
        g.vertices[qid[i]] = ["xyz", [float(x) for x in gr.point_estimate[i]], fx]
        g.vorder.append(qid[i])
    if ek == "proj":
        g.params[param_id] = [float(gr.focal_length), float(gr.principal_point[0]), float(gr.principal_point[1]), 0.5]
    for k in range(gr.num_edges):
        a, b = (int(x) for x in gr.edge_vertex[k])
        i0 = qid[a] if ek == "proj" else pid[a]
        d = 0.0 if gr.robust_delta is None else float(gr.robust_delta[k])
        g.edges.append([ek, i0, pid[b], param_id if ek == "proj" else -1, [float(x) for x in gr.measurement[k]],
                        [float(x) for x in np.asarray(gr.information[k]).reshape(-1)], d])
    return g
