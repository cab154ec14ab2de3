// g2o_io.cpp -- the .g2o text format (include/g2o_io.h) for the device path's
// types: OptimizableGraph::load / save (g2o/core/optimizable_graph.cpp:344-610)
// and the types' read() / write(). Host code only; the loaded graph is handed
// to g2oc_upload as a g2oc_graph view.
#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/g2o_io.h"

namespace g2oc {
void set_error(const char* fmt, ...);
}
using g2oc::set_error;

namespace {

enum Kind : int8_t { kNone = 0, kSE2 = 1, kSE3 = 2, kExpmap = 3, kXYZ = 4 };
enum EKind : int8_t { eSE2 = G2OC_EDGE_SE2, eSE3 = G2OC_EDGE_SE3, eProj = G2OC_EDGE_PROJECT_XYZ2UV,
                      eSE3Exp = G2OC_EDGE_SE3_EXPMAP };

const char* const kVertexTag[5] = {"", "VERTEX_SE2", "VERTEX_SE3:QUAT", "VERTEX_SE3:EXPMAP", "VERTEX_TRACKXYZ"};
// indexed by G2OC_EDGE_*; EdgeSE3ProjectXYZ has no file form with its intrinsics
const char* const kEdgeTag[6] = {"", "EDGE_SE2", "EDGE_SE3:QUAT", "EDGE_PROJECT_XYZ2UV:EXPMAP", "", "EDGE_SE3:EXPMAP"};
const char* const kCameraTag = "PARAMS_CAMERAPARAMETERS";

// estimate doubles per vertex kind in the C-ABI layout
int est_dim(int k) { return k == kSE2 ? 3 : k == kSE3 ? 12 : k == kExpmap ? 7 : 3; }
int vertex_dim(int k) { return k == kSE2 || k == kXYZ ? 3 : 6; }
int meas_dim(int e) { return e == eSE2 ? 3 : e == eSE3 ? 12 : e == eSE3Exp ? 7 : 2; }
int err_dim(int e) { return e == eSE2 ? 3 : (e == eSE3 || e == eSE3Exp) ? 6 : 2; }

struct Vtx {
  int32_t id;
  int8_t kind;
  uint8_t fixed;
  int64_t off;   // into vdata
  int32_t view;  // index in the graph view (poses or points), -1 if not in it
};

struct Edg {
  int8_t kind;
  int32_t v0, v1;  // vertex record indices
  int32_t param;   // CameraParameters id (projection edges), else -1
  int64_t off;     // into edata: measurement then D*D information
  double delta;    // Huber delta, <= 0: none
};

struct Cam {
  double f, cx, cy, baseline;
};

// ---------------------------------------------------------------- rotations
// Unit-quaternion rotation matrix, row-major (Eigen QuaternionBase::toRotationMatrix,
// used by fromVectorQT, g2o/types/slam3d/isometry3d_mappings.cpp:137-142).
void quat_to_rot(double x, double y, double z, double w, double R[9]) {
  const double tx = 2 * x, ty = 2 * y, tz = 2 * z;
  const double twx = tx * w, twy = ty * w, twz = tz * w;
  const double txx = tx * x, txy = ty * x, txz = tz * x;
  const double tyy = ty * y, tyz = tz * y, tzz = tz * z;
  R[0] = 1 - (tyy + tzz); R[1] = txy - twz;       R[2] = txz + twy;
  R[3] = txy + twz;       R[4] = 1 - (txx + tzz); R[5] = tyz - twx;
  R[6] = txz - twy;       R[7] = tyz + twx;       R[8] = 1 - (txx + tyy);
}

// Rotation matrix -> quaternion (x, y, z, w) by Shepperd's method with the
// largest-diagonal branch (the conversion Quaternion(Matrix3) performs).
void rot_to_quat(const double R[9], double q[4]) {
  double t = R[0] + R[4] + R[8];
  if (t > 0) {
    t = std::sqrt(t + 1.0);
    q[3] = 0.5 * t;
    t = 0.5 / t;
    q[0] = (R[7] - R[5]) * t;
    q[1] = (R[2] - R[6]) * t;
    q[2] = (R[3] - R[1]) * t;
  } else {
    int i = 0;
    if (R[4] > R[0]) i = 1;
    if (R[8] > R[i * 4]) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    t = std::sqrt(R[i * 4] - R[j * 4] - R[k * 4] + 1.0);
    q[i] = 0.5 * t;
    t = 0.5 / t;
    q[3] = (R[k * 3 + j] - R[j * 3 + k]) * t;
    q[j] = (R[j * 3 + i] + R[i * 3 + j]) * t;
    q[k] = (R[k * 3 + i] + R[i * 3 + k]) * t;
  }
}

// Quaternion normalize (divide by the norm when it is positive).
void quat_normalize(double q[4]) {
  const double n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
  if (n2 > 0) {
    const double n = std::sqrt(n2);
    for (int i = 0; i < 4; ++i) q[i] /= n;
  }
}

// Isometry (R row-major, t) -> (t, q normalized): toVectorQT
// (g2o/types/slam3d/isometry3d_mappings.cpp:111-121).
void iso_to_qt(const double* iso12, double v[7]) {
  double q[4];
  rot_to_quat(iso12, q);
  quat_normalize(q);
  v[0] = iso12[9]; v[1] = iso12[10]; v[2] = iso12[11];
  v[3] = q[0]; v[4] = q[1]; v[5] = q[2]; v[6] = q[3];
}

// q * v for a quaternion (x, y, z, w): v + 2w (u x v) + u x 2(u x v).
void quat_rotate(const double q[4], const double v[3], double o[3]) {
  double uv[3] = {q[1] * v[2] - q[2] * v[1], q[2] * v[0] - q[0] * v[2], q[0] * v[1] - q[1] * v[0]};
  uv[0] += uv[0]; uv[1] += uv[1]; uv[2] += uv[2];
  o[0] = v[0] + q[3] * uv[0] + (q[1] * uv[2] - q[2] * uv[1]);
  o[1] = v[1] + q[3] * uv[1] + (q[2] * uv[0] - q[0] * uv[2]);
  o[2] = v[2] + q[3] * uv[2] + (q[0] * uv[1] - q[1] * uv[0]);
}

// SE3Quat::inverse (g2o/types/slam3d/se3quat.h:114-119) on (t, q) 7-vectors.
void se3quat_inverse(const double in[7], double out[7]) {
  const double qc[4] = {-in[3], -in[4], -in[5], in[6]};
  const double mt[3] = {in[0] * -1.0, in[1] * -1.0, in[2] * -1.0};
  double t[3];
  quat_rotate(qc, mt, t);
  out[0] = t[0]; out[1] = t[1]; out[2] = t[2];
  out[3] = qc[0]; out[4] = qc[1]; out[5] = qc[2]; out[6] = qc[3];
}

// ---------------------------------------------------------------- tokenizer
inline bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

struct Line {
  const char* p;
  const char* end;
  bool next(const char*& b, const char*& e) {
    while (p < end && is_space(*p)) ++p;
    if (p >= end) return false;
    b = p;
    while (p < end && !is_space(*p)) ++p;
    e = p;
    return true;
  }
  bool num(double& v) {
    const char *b, *e;
    if (!next(b, e)) return false;
    if (*b == '+' && e - b > 1 && b[1] != '-' && b[1] != '+') ++b;
    auto r = std::from_chars(b, e, v, std::chars_format::general);
    return r.ec == std::errc() && r.ptr == e && std::isfinite(v);
  }
  bool integer(int32_t& v) {
    const char *b, *e;
    if (!next(b, e)) return false;
    if (*b == '+' && e - b > 1 && b[1] != '-' && b[1] != '+') ++b;
    auto r = std::from_chars(b, e, v);
    return r.ec == std::errc() && r.ptr == e;
  }
  bool nums(double* v, int n) {
    for (int i = 0; i < n; ++i)
      if (!num(v[i])) return false;
    return true;
  }
  // upper triangle row by row, mirrored (BaseEdge::readInformationMatrix,
  // g2o/core/base_edge.h:173-180)
  bool info(double* I, int D) {
    for (int i = 0; i < D; ++i)
      for (int j = i; j < D; ++j) {
        if (!num(I[i * D + j])) return false;
        I[j * D + i] = I[i * D + j];
      }
    return true;
  }
};

std::string trim(const std::string& s) {
  const size_t b = s.find_first_not_of(" \t\n");
  if (b == std::string::npos) return "";
  const size_t e = s.find_last_not_of(" \t\n");
  return s.substr(b, e - b + 1);
}

bool known_tag(const std::string& t) {
  for (int k = 1; k <= 4; ++k)
    if (t == kVertexTag[k]) return true;
  for (int k = 1; k <= 5; ++k)
    if (kEdgeTag[k][0] && t == kEdgeTag[k]) return true;
  return t == kCameraTag;
}

void put(std::string& s, double v) {
  char buf[40];
  const int n = std::snprintf(buf, sizeof(buf), "%g ", v);
  s.append(buf, n);
}
void put(std::string& s, int v) {
  char buf[16];
  const int n = std::snprintf(buf, sizeof(buf), "%d ", v);
  s.append(buf, n);
}

}  // namespace

struct g2oc_file {
  std::map<int32_t, Cam> params;
  std::vector<Vtx> vtx;
  std::vector<double> vdata;
  std::unordered_map<int32_t, int32_t> by_id;
  std::vector<Edg> edg;
  std::vector<double> edata;
  std::map<std::string, std::string> rename;
  g2oc_file_info info{};
  // graph view
  bool view_valid = false;
  std::vector<int32_t> pose_rec, point_rec;  // vertex record indices in view order
  std::vector<double> pose_est, point_est, meas, infm, delta;
  std::vector<uint8_t> pose_fixed, point_fixed;
  std::vector<int32_t> ev;
  // EDGE_SE3:EXPMAP edges beside projection edges: the graph's pose edge set
  std::vector<int32_t> pev;
  std::vector<double> pmeas, pinfm, pdelta;
  int32_t pose_type = 0, edge_type = 0;
  double focal = 1.0, pp[2] = {0.0, 0.0};

  void problem(int line, const std::string& tag, const char* what) {
    if (info.first_problem_line != 0) return;
    info.first_problem_line = line;
    std::snprintf(info.first_problem, sizeof(info.first_problem), "line %d: %s: %s", line, tag.c_str(), what);
  }

  void set_rename(const char* spec) {
    // OptimizableGraph::setRenamedTypesFromString (optimizable_graph.cpp:619-644)
    if (!spec) return;
    std::string s(spec);
    size_t p = 0;
    while (p <= s.size()) {
      size_t c = s.find(',', p);
      if (c == std::string::npos) c = s.size();
      const std::string item = s.substr(p, c - p);
      p = c + 1;
      const size_t eq = item.find('=');
      if (item.empty() || eq == std::string::npos || item.find('=', eq + 1) != std::string::npos) continue;
      const std::string in = trim(item.substr(0, eq)), to = trim(item.substr(eq + 1));
      if (!known_tag(to)) continue;
      rename[in] = to;
    }
  }

  void parse_line(Line L, int lineno);
  void parse(const char* text, size_t size);
  int build_view();
  std::string write(int mode, const int32_t* ids, int32_t n, int& status) const;
  void write_vertex(std::string& s, const Vtx& v) const;
  void write_edge(std::string& s, const Edg& e) const;
};

void g2oc_file::parse_line(Line L, int lineno) {
  const char *b, *e;
  if (!L.next(b, e)) return;
  if (*b == '#') return;
  std::string tag(b, e);
  if (tag == "FIX") {
    int32_t id;
    while (L.integer(id)) {
      auto it = by_id.find(id);
      if (it != by_id.end()) {
        vtx[it->second].fixed = 1;
      } else {
        info.fix_not_found++;
      }
    }
    return;
  }
  if (!rename.empty()) {
    auto it = rename.find(tag);
    if (it != rename.end()) tag = it->second;
  }
  if (tag == kCameraTag) {
    int32_t id;
    Cam c{1.0, 0.0, 0.0, 0.5};
    double v[3];
    if (!L.integer(id) || !L.nums(v, 3)) {
      info.lines_rejected++;
      problem(lineno, tag, "missing or invalid numbers");
      return;
    }
    double bl;
    Line rest = L;
    if (rest.num(bl)) c.baseline = bl;
    c.f = v[0]; c.cx = v[1]; c.cy = v[2];
    if (!params.emplace(id, c).second) {
      info.lines_rejected++;
      problem(lineno, tag, "parameter id already defined");
      return;
    }
    info.num_parameters++;
    return;
  }
  int vk = kNone, ek = 0;
  for (int k = 1; k <= 4; ++k)
    if (tag == kVertexTag[k]) vk = k;
  for (int k = 1; k <= 5; ++k)
    if (kEdgeTag[k][0] && tag == kEdgeTag[k]) ek = k;
  if (vk != kNone) {
    int32_t id;
    double v[7];
    const int n = (vk == kSE3 || vk == kExpmap) ? 7 : 3;
    if (!L.integer(id) || !L.nums(v, n)) {
      info.lines_rejected++;
      problem(lineno, tag, "missing or invalid numbers");
      return;
    }
    if (id < 0 || by_id.count(id)) {
      // OptimizableGraph::addVertex refuses negative and registered ids
      // (optimizable_graph.cpp:179-206)
      info.lines_rejected++;
      problem(lineno, tag, id < 0 ? "negative vertex id" : "vertex id already registered");
      return;
    }
    Vtx r{id, (int8_t)vk, 0, (int64_t)vdata.size(), -1};
    const size_t o = vdata.size();
    vdata.resize(o + est_dim(vk));
    double* d = vdata.data() + o;
    if (vk == kSE2 || vk == kXYZ) {
      d[0] = v[0]; d[1] = v[1]; d[2] = v[2];
    } else if (vk == kSE3) {
      // VertexSE3::read: fromVectorQT, the quaternion as written (vertex_se3.cpp:46-51)
      quat_to_rot(v[3], v[4], v[5], v[6], d);
      d[9] = v[0]; d[10] = v[1]; d[11] = v[2];
    } else {
      // VertexSE3Expmap::read: SE3Quat(v).inverse() (vertex_se3_expmap.cpp:35-40);
      // the constructor applies normalizeRotation (se3quat.h:81-85, 251-256)
      double q[4] = {v[3], v[4], v[5], v[6]};
      if (q[3] < 0) for (double& c : q) c *= -1;
      quat_normalize(q);
      const double s[7] = {v[0], v[1], v[2], q[0], q[1], q[2], q[3]};
      se3quat_inverse(s, d);
    }
    by_id.emplace(id, (int32_t)vtx.size());
    vtx.push_back(r);
    info.num_vertices++;
    return;
  }
  if (ek != 0) {
    int32_t id0, id1;
    if (!L.integer(id0) || !L.integer(id1)) {
      info.lines_rejected++;
      problem(lineno, tag, "missing or invalid vertex ids");
      return;
    }
    auto i0 = by_id.find(id0), i1 = by_id.find(id1);
    if (i0 == by_id.end() || i1 == by_id.end()) {
      info.lines_rejected++;
      problem(lineno, tag, "unable to find vertices");
      return;
    }
    if (i0->second == i1->second) {
      // HyperGraph::addEdge refuses an edge on one vertex twice (hyper_graph.cpp:98-100)
      info.lines_rejected++;
      problem(lineno, tag, "both ends on one vertex");
      return;
    }
    const int k0 = vtx[i0->second].kind, k1 = vtx[i1->second].kind;
    const bool types_ok = (ek == eSE2 && k0 == kSE2 && k1 == kSE2) || (ek == eSE3 && k0 == kSE3 && k1 == kSE3) ||
                          (ek == eProj && k0 == kXYZ && k1 == kExpmap) ||
                          (ek == eSE3Exp && k0 == kExpmap && k1 == kExpmap);
    if (!types_ok) {
      info.lines_rejected++;
      problem(lineno, tag, "vertex types do not match the edge");
      return;
    }
    int32_t pid = -1;
    if (ek == eProj && !L.integer(pid)) {
      info.lines_rejected++;
      problem(lineno, tag, "missing parameter id");
      return;
    }
    const int D = err_dim(ek), M = meas_dim(ek);
    double m[7];
    double I[36];
    const int nm = ek == eSE2 ? 3 : (ek == eSE3 || ek == eSE3Exp) ? 7 : 2;
    if (!L.nums(m, nm) || !L.info(I, D)) {
      info.lines_rejected++;
      problem(lineno, tag, "missing or invalid numbers");
      return;
    }
    if (ek == eProj && !params.count(pid)) {
      // OptimizableGraph::addEdge -> resolveParameters (optimizable_graph.cpp:232-236)
      info.lines_rejected++;
      problem(lineno, tag, "cannot resolve the parameter");
      return;
    }
    Edg r{(int8_t)ek, i0->second, i1->second, pid, (int64_t)edata.size(), 0.0};
    const size_t o = edata.size();
    edata.resize(o + M + D * D);
    double* d = edata.data() + o;
    if (ek == eSE3) {
      // EdgeSE3::read normalizes the quaternion, then fromVectorQT (edge_se3.cpp:43-53)
      double q[4] = {m[3], m[4], m[5], m[6]};
      quat_normalize(q);
      quat_to_rot(q[0], q[1], q[2], q[3], d);
      d[9] = m[0]; d[10] = m[1]; d[11] = m[2];
    } else if (ek == eSE3Exp) {
      // EdgeSE3Expmap::read: setMeasurement(SE3Quat(meas).inverse()) (edge_se3_expmap.cpp:33-38)
      double q[4] = {m[3], m[4], m[5], m[6]};
      if (q[3] < 0) for (double& cq : q) cq *= -1;
      quat_normalize(q);
      const double s7[7] = {m[0], m[1], m[2], q[0], q[1], q[2], q[3]};
      se3quat_inverse(s7, d);
    } else {
      for (int i = 0; i < M; ++i) d[i] = m[i];
    }
    std::memcpy(d + M, I, sizeof(double) * D * D);
    edg.push_back(r);
    info.num_edges++;
    return;
  }
  if (tag.compare(0, 7, "VERTEX_") == 0 || tag.compare(0, 5, "EDGE_") == 0) {
    info.lines_unsupported++;
    problem(lineno, tag, "type not supported by the device path");
    return;
  }
  info.lines_skipped++;
}

void g2oc_file::parse(const char* text, size_t size) {
  const char* p = text;
  const char* end = text + size;
  int lineno = 0;
  while (p < end) {
    const char* nl = static_cast<const char*>(std::memchr(p, '\n', end - p));
    const char* le = nl ? nl : end;
    ++lineno;
    parse_line(Line{p, le}, lineno);
    p = nl ? nl + 1 : end;
  }
  info.lines = lineno;
  view_valid = false;
}

int g2oc_file::build_view() {
  if (view_valid) return G2OC_OK;
  int et = 0;
  bool with_pose_edges = false;  // projection edges plus EDGE_SE3:EXPMAP: the latter are the pose edge set
  for (const Edg& e : edg) {
    if (et == 0 || et == e.kind) {
      et = e.kind;
    } else if ((et == eProj && e.kind == eSE3Exp) || (et == eSE3Exp && e.kind == eProj)) {
      et = eProj;
      with_pose_edges = true;
    } else {
      set_error("the graph mixes %s and %s edges; the device path takes projection edges with EDGE_SE3:EXPMAP "
                "edges, or one edge type", kEdgeTag[et], kEdgeTag[e.kind]);
      return G2OC_ERR_NOT_SUPPORTED;
    }
  }
  if (et == 0) {
    set_error("the graph has no edge");
    return G2OC_ERR_BAD_GRAPH;
  }
  const int pk = et == eSE2 ? kSE2 : et == eSE3 ? kSE3 : kExpmap;  // projection and SE3Expmap edges: VertexSE3Expmap
  focal = 1.0; pp[0] = pp[1] = 0.0;
  if (et == eProj) {
    int first = 0;
    while (edg[first].kind != eProj) ++first;
    const Cam& c0 = params.at(edg[first].param);
    for (const Edg& e : edg) {
      if (e.kind != eProj) continue;
      const Cam& c = params.at(e.param);
      if (c.f != c0.f || c.cx != c0.cx || c.cy != c0.cy) {
        set_error("projection edges refer to CameraParameters %d and %d, which differ", edg[0].param, e.param);
        return G2OC_ERR_NOT_SUPPORTED;
      }
    }
    focal = c0.f; pp[0] = c0.cx; pp[1] = c0.cy;
  }
  pose_rec.clear();
  point_rec.clear();
  for (int32_t i = 0; i < (int32_t)vtx.size(); ++i) {
    vtx[i].view = -1;
    if (vtx[i].kind == pk) pose_rec.push_back(i);
    else if (et == eProj && vtx[i].kind == kXYZ) point_rec.push_back(i);
  }
  auto by_vid = [&](int32_t a, int32_t b) { return vtx[a].id < vtx[b].id; };
  std::sort(pose_rec.begin(), pose_rec.end(), by_vid);
  std::sort(point_rec.begin(), point_rec.end(), by_vid);
  const int pd = est_dim(pk);
  pose_est.resize(pose_rec.size() * pd);
  pose_fixed.resize(pose_rec.size());
  for (size_t i = 0; i < pose_rec.size(); ++i) {
    Vtx& v = vtx[pose_rec[i]];
    v.view = (int32_t)i;
    std::memcpy(&pose_est[i * pd], &vdata[v.off], sizeof(double) * pd);
    pose_fixed[i] = v.fixed;
  }
  point_est.resize(point_rec.size() * 3);
  point_fixed.resize(point_rec.size());
  for (size_t i = 0; i < point_rec.size(); ++i) {
    Vtx& v = vtx[point_rec[i]];
    v.view = (int32_t)i;
    std::memcpy(&point_est[i * 3], &vdata[v.off], sizeof(double) * 3);
    point_fixed[i] = v.fixed;
  }
  const int M = meas_dim(et), D = err_dim(et);
  size_t E = 0, PE = 0;
  bool robust = false, probust = false;
  for (const Edg& e : edg) {
    if (e.kind == et) {
      ++E;
      robust |= e.delta > 0;
    } else {
      ++PE;
      probust |= e.delta > 0;
    }
  }
  ev.resize(2 * E);
  meas.resize(E * M);
  infm.resize(E * D * D);
  delta.assign(robust ? E : 0, 0.0);
  pev.resize(2 * PE);
  pmeas.resize(PE * 7);
  pinfm.resize(PE * 36);
  pdelta.assign(probust ? PE : 0, 0.0);
  size_t k = 0, q = 0;
  for (const Edg& e : edg) {
    if (e.kind == et) {
      ev[2 * k] = vtx[e.v0].view;
      ev[2 * k + 1] = vtx[e.v1].view;
      std::memcpy(&meas[k * M], &edata[e.off], sizeof(double) * M);
      std::memcpy(&infm[k * D * D], &edata[e.off + M], sizeof(double) * D * D);
      if (robust) delta[k] = e.delta;
      ++k;
    } else {
      pev[2 * q] = vtx[e.v0].view;
      pev[2 * q + 1] = vtx[e.v1].view;
      std::memcpy(&pmeas[q * 7], &edata[e.off], sizeof(double) * 7);
      std::memcpy(&pinfm[q * 36], &edata[e.off + 7], sizeof(double) * 36);
      if (probust) pdelta[q] = e.delta;
      ++q;
    }
  }
  (void)with_pose_edges;
  pose_type = pk == kSE2 ? G2OC_POSE_SE2 : pk == kSE3 ? G2OC_POSE_SE3 : G2OC_POSE_SE3EXPMAP;
  edge_type = et;
  view_valid = true;
  return G2OC_OK;
}

void g2oc_file::write_vertex(std::string& s, const Vtx& v) const {
  // OptimizableGraph::saveVertex (optimizable_graph.cpp:736-751)
  s += kVertexTag[v.kind];
  s += ' ';
  put(s, (int)v.id);
  const double* d = &vdata[v.off];
  if (v.kind == kSE2 || v.kind == kXYZ) {
    for (int i = 0; i < 3; ++i) put(s, d[i]);
  } else if (v.kind == kSE3) {
    double w[7];
    iso_to_qt(d, w);  // VertexSE3::write (vertex_se3.cpp:53-55)
    for (double x : w) put(s, x);
  } else {
    double w[7];
    se3quat_inverse(d, w);  // VertexSE3Expmap::write (vertex_se3_expmap.cpp:42-44)
    for (double x : w) put(s, x);
  }
  s += '\n';
  if (v.fixed) {
    s += "FIX ";
    s += std::to_string(v.id);
    s += '\n';
  }
}

void g2oc_file::write_edge(std::string& s, const Edg& e) const {
  // OptimizableGraph::saveEdge (optimizable_graph.cpp:764-780) and the edges' write()
  s += kEdgeTag[e.kind];
  s += ' ';
  put(s, (int)vtx[e.v0].id);
  put(s, (int)vtx[e.v1].id);
  if (e.kind == eProj) put(s, (int)e.param);
  const double* d = &edata[e.off];
  const int M = meas_dim(e.kind), D = err_dim(e.kind);
  if (e.kind == eSE3) {
    double w[7];
    iso_to_qt(d, w);
    for (double x : w) put(s, x);
  } else if (e.kind == eSE3Exp) {
    double w[7];
    se3quat_inverse(d, w);  // EdgeSE3Expmap::write: measurement().inverse().toVector()
    for (double x : w) put(s, x);
  } else {
    for (int i = 0; i < M; ++i) put(s, d[i]);
  }
  // BaseEdge::writeInformationMatrix (base_edge.h:165-170)
  for (int i = 0; i < D; ++i)
    for (int j = i; j < D; ++j) put(s, d[M + i * D + j]);
  s += '\n';
}

std::string g2oc_file::write(int mode, const int32_t* ids, int32_t n, int& status) const {
  std::string s;
  status = G2OC_OK;
  // ParameterContainer::write, by id (g2o/core/parameter_container.cpp:82-91)
  for (const auto& kv : params) {
    s += kCameraTag;
    s += ' ';
    put(s, (int)kv.first);
    put(s, kv.second.f);
    put(s, kv.second.cx);
    put(s, kv.second.cy);
    put(s, kv.second.baseline);
    s += '\n';
  }
  std::vector<char> vsel(vtx.size(), 0), esel(edg.size(), 0);
  if (mode == G2OC_SAVE_ALL) {
    // save(): the vertices of the edges, by id, then every edge (optimizable_graph.cpp:539-567)
    for (const Edg& e : edg) vsel[e.v0] = vsel[e.v1] = 1;
    std::fill(esel.begin(), esel.end(), 1);
  } else if (mode == G2OC_SAVE_VERTEX_SUBSET) {
    // saveSubset(VertexSet): those vertices, the edges with every vertex among them (:569-594)
    for (int32_t i = 0; i < n; ++i) {
      auto it = by_id.find(ids[i]);
      if (it == by_id.end()) {
        set_error("saveSubset: no vertex with id %d", ids[i]);
        status = G2OC_ERR_INVALID_ARGUMENT;
        return s;
      }
      vsel[it->second] = 1;
    }
    for (size_t k = 0; k < edg.size(); ++k) esel[k] = vsel[edg[k].v0] && vsel[edg[k].v1];
  } else if (mode == G2OC_SAVE_EDGE_SUBSET) {
    // saveSubset(EdgeSet): those edges and their vertices (:596-606)
    for (int32_t i = 0; i < n; ++i) {
      if (ids[i] < 0 || ids[i] >= (int32_t)edg.size()) {
        set_error("saveSubset: no edge with index %d", ids[i]);
        status = G2OC_ERR_INVALID_ARGUMENT;
        return s;
      }
      esel[ids[i]] = 1;
      vsel[edg[ids[i]].v0] = vsel[edg[ids[i]].v1] = 1;
    }
  } else {
    set_error("unknown save mode %d", mode);
    status = G2OC_ERR_INVALID_ARGUMENT;
    return s;
  }
  std::vector<int32_t> order, eorder;
  for (int32_t i = 0; i < (int32_t)vtx.size(); ++i)
    if (vsel[i]) order.push_back(i);
  std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return vtx[a].id < vtx[b].id; });
  for (int32_t k = 0; k < (int32_t)edg.size(); ++k)
    if (esel[k]) eorder.push_back(k);
  // the lines are formatted in parallel chunks and joined in order: the text
  // is the sequential text
  auto emit = [&](const std::vector<int32_t>& items, bool vertices) {
    const int64_t n = (int64_t)items.size();
    const int64_t per = 8192;
    const int64_t nchunks = (n + per - 1) / per;
    std::vector<std::string> parts(nchunks);
#pragma omp parallel for schedule(dynamic)
    for (int64_t ch = 0; ch < nchunks; ++ch) {
      std::string& out = parts[ch];
      for (int64_t i = ch * per; i < std::min(n, (ch + 1) * per); ++i) {
        if (vertices) write_vertex(out, vtx[items[i]]);
        else write_edge(out, edg[items[i]]);
      }
    }
    for (const std::string& part : parts) s += part;
  };
  emit(order, true);
  emit(eorder, false);
  return s;
}

extern "C" {

int g2oc_file_parse(const char* text, size_t size, const char* renamed_types, g2oc_file** out) {
  if (!out || (!text && size)) {
    set_error("g2oc_file_parse: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  g2oc_file* f = new g2oc_file();
  f->set_rename(renamed_types);
  f->parse(text ? text : "", size);
  *out = f;
  return G2OC_OK;
}

int g2oc_file_load(const char* path, const char* renamed_types, g2oc_file** out) {
  if (!path || !out) {
    set_error("g2oc_file_load: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) {
    set_error("unable to open file %s", path);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  std::string text;
  char buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, n);
  const bool bad = std::ferror(fp) != 0;
  std::fclose(fp);
  if (bad) {
    set_error("error reading file %s", path);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  return g2oc_file_parse(text.data(), text.size(), renamed_types, out);
}

int g2oc_file_from_graph(const g2oc_graph* g, const int32_t* pose_ids, const int32_t* point_ids,
                         int32_t camera_param_id, g2oc_file** out) {
  if (!g || !out || g->num_poses < 0 || g->num_points < 0 || g->num_edges < 0 || !g->pose_estimate ||
      (g->num_points && !g->point_estimate) || (g->num_edges && (!g->edge_vertex || !g->measurement ||
                                                                 !g->information))) {
    set_error("g2oc_file_from_graph: invalid argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  int vk, ek = g->edge_type;
  if (g->pose_type == G2OC_POSE_SE2 && ek == G2OC_EDGE_SE2) vk = kSE2;
  else if (g->pose_type == G2OC_POSE_SE3 && ek == G2OC_EDGE_SE3) vk = kSE3;
  else if (g->pose_type == G2OC_POSE_SE3EXPMAP && (ek == G2OC_EDGE_PROJECT_XYZ2UV || ek == G2OC_EDGE_SE3_EXPMAP))
    vk = kExpmap;
  else {
    set_error("g2oc_file_from_graph: pose type %d does not go with edge type %d", g->pose_type, ek);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  g2oc_file* f = new g2oc_file();
  auto add = [&](int32_t id, int kind, const double* est, uint8_t fixed) {
    if (id < 0 || f->by_id.count(id)) return false;
    f->by_id.emplace(id, (int32_t)f->vtx.size());
    f->vtx.push_back(Vtx{id, (int8_t)kind, fixed, (int64_t)f->vdata.size(), -1});
    f->vdata.insert(f->vdata.end(), est, est + est_dim(kind));
    return true;
  };
  std::vector<int32_t> prec(g->num_poses), qrec(g->num_points);
  bool ok = true;
  const int pd = est_dim(vk);
  for (int32_t i = 0; i < g->num_poses && ok; ++i) {
    prec[i] = (int32_t)f->vtx.size();
    ok = add(pose_ids ? pose_ids[i] : i, vk, g->pose_estimate + (size_t)i * pd,
             g->pose_fixed ? (g->pose_fixed[i] != 0) : 0);
  }
  for (int32_t i = 0; i < g->num_points && ok; ++i) {
    qrec[i] = (int32_t)f->vtx.size();
    ok = add(point_ids ? point_ids[i] : g->num_poses + i, kXYZ, g->point_estimate + (size_t)i * 3,
             g->point_fixed ? (g->point_fixed[i] != 0) : 0);
  }
  if (!ok) {
    delete f;
    set_error("g2oc_file_from_graph: negative or repeated vertex id");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (ek == eProj) f->params.emplace(camera_param_id, Cam{g->focal_length, g->principal_point[0],
                                                          g->principal_point[1], 0.5});
  const int M = meas_dim(ek), D = err_dim(ek);
  for (int32_t k = 0; k < g->num_edges; ++k) {
    const int32_t a = g->edge_vertex[2 * k], b = g->edge_vertex[2 * k + 1];
    const bool in_range = ek == eProj ? (a >= 0 && a < g->num_points && b >= 0 && b < g->num_poses)
                                      : (a >= 0 && a < g->num_poses && b >= 0 && b < g->num_poses && a != b);
    if (!in_range) {
      delete f;
      set_error("g2oc_file_from_graph: edge %d has a vertex index out of range", k);
      return G2OC_ERR_INVALID_ARGUMENT;
    }
    Edg e{(int8_t)ek, ek == eProj ? qrec[a] : prec[a], prec[b], ek == eProj ? camera_param_id : -1,
          (int64_t)f->edata.size(), g->robust_delta ? g->robust_delta[k] : 0.0};
    f->edata.insert(f->edata.end(), g->measurement + (size_t)k * M, g->measurement + (size_t)(k + 1) * M);
    f->edata.insert(f->edata.end(), g->information + (size_t)k * D * D, g->information + (size_t)(k + 1) * D * D);
    f->edg.push_back(e);
  }
  if (g->num_pose_edges > 0 && ek == eProj) {  // the pose edge set as EDGE_SE3:EXPMAP records
    if (!g->pose_edge_vertex || !g->pose_edge_measurement || !g->pose_edge_information) {
      delete f;
      set_error("g2oc_file_from_graph: pose edge array is NULL");
      return G2OC_ERR_INVALID_ARGUMENT;
    }
    for (int32_t k = 0; k < g->num_pose_edges; ++k) {
      const int32_t a = g->pose_edge_vertex[2 * k], b = g->pose_edge_vertex[2 * k + 1];
      if (a < 0 || a >= g->num_poses || b < 0 || b >= g->num_poses || a == b) {
        delete f;
        set_error("g2oc_file_from_graph: pose edge %d has a vertex index out of range", k);
        return G2OC_ERR_INVALID_ARGUMENT;
      }
      Edg e{(int8_t)eSE3Exp, prec[a], prec[b], -1, (int64_t)f->edata.size(),
            g->pose_edge_robust_delta ? g->pose_edge_robust_delta[k] : 0.0};
      f->edata.insert(f->edata.end(), g->pose_edge_measurement + (size_t)k * 7,
                      g->pose_edge_measurement + (size_t)(k + 1) * 7);
      f->edata.insert(f->edata.end(), g->pose_edge_information + (size_t)k * 36,
                      g->pose_edge_information + (size_t)(k + 1) * 36);
      f->edg.push_back(e);
    }
  }
  f->info.num_vertices = (int32_t)f->vtx.size();
  f->info.num_edges = (int32_t)f->edg.size();
  f->info.num_parameters = (int32_t)f->params.size();
  *out = f;
  return G2OC_OK;
}

void g2oc_file_free(g2oc_file* f) { delete f; }

int g2oc_file_get_info(const g2oc_file* f, g2oc_file_info* info) {
  if (!f || !info) {
    set_error("g2oc_file_get_info: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *info = f->info;
  int32_t nf = 0;
  for (const Vtx& v : f->vtx) nf += v.fixed;
  info->num_fixed = nf;
  return G2OC_OK;
}

int g2oc_file_graph(g2oc_file* f, g2oc_graph* out) {
  if (!f || !out) {
    set_error("g2oc_file_graph: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const int st = f->build_view();
  if (st != G2OC_OK) return st;
  g2oc_graph g;
  std::memset(&g, 0, sizeof(g));
  g.pose_type = f->pose_type;
  g.num_poses = (int32_t)f->pose_rec.size();
  g.pose_estimate = f->pose_est.data();
  g.pose_fixed = f->pose_fixed.data();
  g.num_points = (int32_t)f->point_rec.size();
  g.point_estimate = g.num_points ? f->point_est.data() : nullptr;
  g.point_fixed = g.num_points ? f->point_fixed.data() : nullptr;
  g.edge_type = f->edge_type;
  g.num_edges = (int32_t)(f->ev.size() / 2);
  g.edge_vertex = f->ev.data();
  g.num_pose_edges = (int32_t)(f->pev.size() / 2);
  if (g.num_pose_edges > 0) {
    g.pose_edge_vertex = f->pev.data();
    g.pose_edge_measurement = f->pmeas.data();
    g.pose_edge_information = f->pinfm.data();
    g.pose_edge_robust_delta = f->pdelta.empty() ? nullptr : f->pdelta.data();
  }
  g.measurement = f->meas.data();
  g.information = f->infm.data();
  g.robust_delta = f->delta.empty() ? nullptr : f->delta.data();
  g.focal_length = f->focal;
  g.principal_point[0] = f->pp[0];
  g.principal_point[1] = f->pp[1];
  *out = g;
  return G2OC_OK;
}

int g2oc_file_vertex_ids(g2oc_file* f, int32_t* pose_ids, int32_t* point_ids) {
  if (!f) {
    set_error("g2oc_file_vertex_ids: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const int st = f->build_view();
  if (st != G2OC_OK) return st;
  if (pose_ids)
    for (size_t i = 0; i < f->pose_rec.size(); ++i) pose_ids[i] = f->vtx[f->pose_rec[i]].id;
  if (point_ids)
    for (size_t i = 0; i < f->point_rec.size(); ++i) point_ids[i] = f->vtx[f->point_rec[i]].id;
  return G2OC_OK;
}

int g2oc_file_set_fixed(g2oc_file* f, int32_t id, int32_t fixed) {
  if (!f) {
    set_error("g2oc_file_set_fixed: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  auto it = f->by_id.find(id);
  if (it == f->by_id.end()) {
    set_error("no vertex with id %d", id);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  f->vtx[it->second].fixed = fixed ? 1 : 0;
  f->view_valid = false;
  return G2OC_OK;
}

int g2oc_file_fix_gauge(g2oc_file* f, int32_t* gauge_id) {
  // SparseOptimizer::gaugeFreedom / findGauge (sparse_optimizer.cpp:132-173): the
  // device path's types have no unary (prior) edges, so the gauge is free
  // unless a vertex of the maximum dimension is fixed.
  if (!f || !gauge_id) {
    set_error("g2oc_file_fix_gauge: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  *gauge_id = -1;
  if (f->vtx.empty()) {
    set_error("the graph has no vertex");
    return G2OC_ERR_BAD_GRAPH;
  }
  int maxd = 0;
  for (const Vtx& v : f->vtx) maxd = std::max(maxd, vertex_dim(v.kind));
  int32_t best = -1;
  for (int32_t i = 0; i < (int32_t)f->vtx.size(); ++i) {
    const Vtx& v = f->vtx[i];
    if (vertex_dim(v.kind) != maxd) continue;
    if (v.fixed) return G2OC_OK;
    if (best < 0 || v.id < f->vtx[best].id) best = i;
  }
  f->vtx[best].fixed = 1;
  f->view_valid = false;
  *gauge_id = f->vtx[best].id;
  return G2OC_OK;
}

int g2oc_file_set_robust_huber(g2oc_file* f, double delta, int32_t non_sequential) {
  if (!f) {
    set_error("g2oc_file_set_robust_huber: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  for (Edg& e : f->edg) {
    const bool seq = std::abs((int64_t)f->vtx[e.v0].id - (int64_t)f->vtx[e.v1].id) == 1;
    e.delta = (delta > 0 && !(non_sequential && seq)) ? delta : 0.0;
  }
  f->view_valid = false;
  return G2OC_OK;
}

int g2oc_file_set_estimates(g2oc_file* f, const double* pose_estimate, const double* point_estimate) {
  if (!f || !pose_estimate) {
    set_error("g2oc_file_set_estimates: null argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const int st = f->build_view();
  if (st != G2OC_OK) return st;
  if (!f->point_rec.empty() && !point_estimate) {
    set_error("g2oc_file_set_estimates: the graph has points");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const int pd = f->pose_type == G2OC_POSE_SE2 ? 3 : f->pose_type == G2OC_POSE_SE3 ? 12 : 7;
  for (size_t i = 0; i < f->pose_rec.size(); ++i) {
    const Vtx& v = f->vtx[f->pose_rec[i]];
    std::memcpy(&f->vdata[v.off], pose_estimate + i * pd, sizeof(double) * pd);
    std::memcpy(&f->pose_est[i * pd], pose_estimate + i * pd, sizeof(double) * pd);
  }
  for (size_t i = 0; i < f->point_rec.size(); ++i) {
    const Vtx& v = f->vtx[f->point_rec[i]];
    std::memcpy(&f->vdata[v.off], point_estimate + i * 3, sizeof(double) * 3);
    std::memcpy(&f->point_est[i * 3], point_estimate + i * 3, sizeof(double) * 3);
  }
  return G2OC_OK;
}

int g2oc_file_save(const g2oc_file* f, const char* path, int32_t mode, const int32_t* ids, int32_t num_ids) {
  if (!f || !path || (num_ids > 0 && !ids) || num_ids < 0) {
    set_error("g2oc_file_save: invalid argument");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  int st;
  const std::string s = f->write(mode, ids, num_ids, st);
  if (st != G2OC_OK) return st;
  FILE* fp = std::fopen(path, "wb");
  if (!fp) {
    set_error("unable to open %s for writing", path);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  const bool ok = std::fwrite(s.data(), 1, s.size(), fp) == s.size();
  const bool closed = std::fclose(fp) == 0;
  if (!ok || !closed) {
    set_error("error writing %s", path);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  return G2OC_OK;
}

}  // extern "C"
