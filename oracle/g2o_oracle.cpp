// g2o_oracle.cpp -- TEST INFRASTRUCTURE ONLY (checker and CPU baseline).
//
// FP64 CPU restatement of g2o's GN/LM iteration over a BlockSolver, written
// from the reference's published algorithm without Eigen. Each function cites
// the reference file:line it follows (paths relative to the g2o tree). The
// product library never links this file; it is built by oracle/Makefile into
// oracle/liboracle.so and used by tests/, bench.py (CPU baseline) and
// __graft_entry__.smoke().
#include "g2o_oracle.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <unordered_map>
#include <utility>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

double now_s() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// ---------------------------------------------------------------- small math
// All matrices are dense row-major.

inline double normalize_theta(double theta) {
  // g2o/stuff/misc.h:66-70
  const double pi = 3.14159265358979323846;
  const double r = std::fmod(theta + pi, 2.0 * pi);
  if (r <= 0.0) return r + pi;
  return r - pi;
}

struct Quat {
  double x, y, z, w;
};

inline void quat_to_rot(const Quat& q, double R[9]) {
  // unit-quaternion rotation matrix (Eigen QuaternionBase::toRotationMatrix)
  const double tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z;
  const double twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
  const double txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
  const double tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
  R[0] = 1 - (tyy + tzz); R[1] = txy - twz;       R[2] = txz + twy;
  R[3] = txy + twz;       R[4] = 1 - (txx + tzz); R[5] = tyz - twx;
  R[6] = txz - twy;       R[7] = tyz + twx;       R[8] = 1 - (txx + tyy);
}

inline Quat rot_to_quat(const double R[9]) {
  // Shepperd's method with the largest-diagonal branch (Eigen quaternion_assign_impl)
  Quat q;
  double t = R[0] + R[4] + R[8];
  if (t > 0) {
    t = std::sqrt(t + 1.0);
    q.w = 0.5 * t;
    t = 0.5 / t;
    q.x = (R[7] - R[5]) * t;
    q.y = (R[2] - R[6]) * t;
    q.z = (R[3] - R[1]) * t;
  } else {
    int i = 0;
    if (R[4] > R[0]) i = 1;
    if (R[8] > R[i * 4]) i = 2;
    int j = (i + 1) % 3, k = (j + 1) % 3;
    double c[3];
    t = std::sqrt(R[i * 4] - R[j * 4] - R[k * 4] + 1.0);
    c[i] = 0.5 * t;
    t = 0.5 / t;
    q.w = (R[k * 3 + j] - R[j * 3 + k]) * t;
    c[j] = (R[j * 3 + i] + R[i * 3 + j]) * t;
    c[k] = (R[k * 3 + i] + R[i * 3 + k]) * t;
    q.x = c[0]; q.y = c[1]; q.z = c[2];
  }
  return q;
}

inline Quat quat_mul(const Quat& a, const Quat& b) {
  Quat r;
  r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  r.y = a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z;
  r.z = a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x;
  return r;
}

inline void quat_rotate(const Quat& q, const double v[3], double out[3]) {
  // v + 2w(u x v) + 2 u x (u x v)
  double uv[3] = {q.y * v[2] - q.z * v[1], q.z * v[0] - q.x * v[2], q.x * v[1] - q.y * v[0]};
  uv[0] += uv[0]; uv[1] += uv[1]; uv[2] += uv[2];
  out[0] = v[0] + q.w * uv[0] + (q.y * uv[2] - q.z * uv[1]);
  out[1] = v[1] + q.w * uv[1] + (q.z * uv[0] - q.x * uv[2]);
  out[2] = v[2] + q.w * uv[2] + (q.x * uv[1] - q.y * uv[0]);
}

inline void quat_normalize_positive_w(Quat& q) {
  // SE3Quat::normalizeRotation (g2o/types/slam3d/se3quat.h:251-256)
  if (q.w < 0) { q.x = -q.x; q.y = -q.y; q.z = -q.z; q.w = -q.w; }
  const double n = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x /= n; q.y /= n; q.z /= n; q.w /= n;
}

inline void matmul3(const double A[9], const double B[9], double C[9]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      C[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}

inline void matvec3(const double A[9], const double v[3], double o[3]) {
  for (int i = 0; i < 3; ++i) o[i] = A[i * 3] * v[0] + A[i * 3 + 1] * v[1] + A[i * 3 + 2] * v[2];
}

// SE3Quat (q, t) as 7 doubles: t xyz, q xyzw (SE3Quat::toVector, se3quat.h:117-127)
struct SE3Q {
  Quat q;
  double t[3];
};

inline SE3Q se3q_load(const double* v) {
  SE3Q s;
  s.t[0] = v[0]; s.t[1] = v[1]; s.t[2] = v[2];
  s.q = {v[3], v[4], v[5], v[6]};
  return s;
}
inline void se3q_store(const SE3Q& s, double* v) {
  v[0] = s.t[0]; v[1] = s.t[1]; v[2] = s.t[2];
  v[3] = s.q.x; v[4] = s.q.y; v[5] = s.q.z; v[6] = s.q.w;
}

SE3Q se3q_exp(const double u[6]) {
  // SE3Quat::exp (g2o/types/slam3d/se3quat.h:202-230): u = (omega, upsilon)
  const double w0 = u[0], w1 = u[1], w2 = u[2];
  const double theta = std::sqrt(w0 * w0 + w1 * w1 + w2 * w2);
  const double O[9] = {0, -w2, w1, w2, 0, -w0, -w1, w0, 0};
  double O2[9];
  matmul3(O, O, O2);
  double R[9], V[9];
  if (theta < 0.00001) {
    // R = I + O + 0.5 O2 ; V = I + 0.5 O + 1/6 O2
    for (int i = 0; i < 9; ++i) {
      R[i] = O[i] + 0.5 * O2[i];
      V[i] = 0.5 * O[i] + (1.0 / 6.0) * O2[i];
    }
  } else {
    const double s = std::sin(theta), co = std::cos(theta);
    const double A = s / theta, B = (1 - co) / (theta * theta), C = (theta - s) / std::pow(theta, 3);
    for (int i = 0; i < 9; ++i) {
      R[i] = A * O[i] + B * O2[i];
      V[i] = B * O[i] + C * O2[i];
    }
  }
  R[0] += 1; R[4] += 1; R[8] += 1;
  V[0] += 1; V[4] += 1; V[8] += 1;
  SE3Q r;
  r.q = rot_to_quat(R);
  matvec3(V, u + 3, r.t);
  quat_normalize_positive_w(r.q);
  return r;
}

inline SE3Q se3q_mul(const SE3Q& a, const SE3Q& b) {
  // SE3Quat::operator* (se3quat.h:97-103)
  SE3Q r;
  double rt[3];
  quat_rotate(a.q, b.t, rt);
  r.t[0] = a.t[0] + rt[0]; r.t[1] = a.t[1] + rt[1]; r.t[2] = a.t[2] + rt[2];
  r.q = quat_mul(a.q, b.q);
  quat_normalize_positive_w(r.q);
  return r;
}

inline SE3Q se3q_inv(const SE3Q& a) {
  // SE3Quat::inverse (se3quat.h:114-119)
  SE3Q r;
  r.q = {-a.q.x, -a.q.y, -a.q.z, a.q.w};
  const double mt[3] = {-a.t[0], -a.t[1], -a.t[2]};
  quat_rotate(r.q, mt, r.t);
  return r;
}

void se3q_log(const SE3Q& a, double out[6]) {
  // SE3Quat::log (se3quat.h:165-199), deltaR / skew (se3_ops.hpp:27-45)
  double R[9];
  quat_to_rot(a.q, R);
  const double d = 0.5 * (R[0] + R[4] + R[8] - 1);
  const double dR[3] = {R[7] - R[5], R[2] - R[6], R[3] - R[1]};
  double w[3], Vi[9];
  double O[9], O2[9];
  if (std::fabs(d) > 0.99999) {
    for (int i = 0; i < 3; ++i) w[i] = 0.5 * dR[i];
    const double Om[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    std::memcpy(O, Om, sizeof(O));
    matmul3(O, O, O2);
    for (int i = 0; i < 9; ++i) Vi[i] = -0.5 * O[i] + (1. / 12.) * O2[i];
  } else {
    const double theta = std::acos(d);
    for (int i = 0; i < 3; ++i) w[i] = theta / (2 * std::sqrt(1 - d * d)) * dR[i];
    const double Om[9] = {0, -w[2], w[1], w[2], 0, -w[0], -w[1], w[0], 0};
    std::memcpy(O, Om, sizeof(O));
    matmul3(O, O, O2);
    const double k = (1 - theta / (2 * std::tan(theta / 2))) / (theta * theta);
    for (int i = 0; i < 9; ++i) Vi[i] = -0.5 * O[i] + k * O2[i];
  }
  Vi[0] += 1; Vi[4] += 1; Vi[8] += 1;
  out[0] = w[0]; out[1] = w[1]; out[2] = w[2];
  matvec3(Vi, a.t, out + 3);
}

void se3q_adj(const SE3Q& a, double sign, double A[36]) {
  // SE3Quat::adj (se3quat.h:232-240)
  double R[9], SR[9];
  quat_to_rot(a.q, R);
  const double S[9] = {0, -a.t[2], a.t[1], a.t[2], 0, -a.t[0], -a.t[1], a.t[0], 0};
  matmul3(S, R, SR);
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      A[r * 6 + c] = sign * R[r * 3 + c];
      A[r * 6 + 3 + c] = 0;
      A[(3 + r) * 6 + c] = sign * SR[r * 3 + c];
      A[(3 + r) * 6 + 3 + c] = sign * R[r * 3 + c];
    }
}

// EdgeSE3Expmap (g2o/types/sba/edge_se3_expmap.cpp:45-72): vertex0 = i,
// vertex1 = j, measurement C: e = log(Tj^-1 C Ti), J_i = adj(Tj^-1 C),
// J_j = -adj(Ti^-1 C^-1)
void se3exp_error(const double* xi, const double* xj, const double* c7, double e[6]) {
  const SE3Q Ti = se3q_load(xi), Tj = se3q_load(xj), C = se3q_load(c7);
  se3q_log(se3q_mul(se3q_mul(se3q_inv(Tj), C), Ti), e);
}
void se3exp_jacobians(const double* xi, const double* xj, const double* c7, double Ji[36], double Jj[36]) {
  const SE3Q Ti = se3q_load(xi), Tj = se3q_load(xj), C = se3q_load(c7);
  se3q_adj(se3q_mul(se3q_inv(Tj), C), 1.0, Ji);
  se3q_adj(se3q_mul(se3q_inv(Ti), se3q_inv(C)), -1.0, Jj);
}

// Isometry3 as R (row-major 9) and t (3): 12 doubles
struct Iso3 {
  double R[9];
  double t[3];
};
inline Iso3 iso_load(const double* v) {
  Iso3 s;
  std::memcpy(s.R, v, 9 * sizeof(double));
  std::memcpy(s.t, v + 9, 3 * sizeof(double));
  return s;
}
inline void iso_store(const Iso3& s, double* v) {
  std::memcpy(v, s.R, 9 * sizeof(double));
  std::memcpy(v + 9, s.t, 3 * sizeof(double));
}
inline Iso3 iso_mul(const Iso3& a, const Iso3& b) {
  Iso3 r;
  matmul3(a.R, b.R, r.R);
  matvec3(a.R, b.t, r.t);
  r.t[0] += a.t[0]; r.t[1] += a.t[1]; r.t[2] += a.t[2];
  return r;
}
inline Iso3 iso_inv(const Iso3& a) {
  Iso3 r;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r.R[i * 3 + j] = a.R[j * 3 + i];
  double tt[3];
  matvec3(r.R, a.t, tt);
  r.t[0] = -tt[0]; r.t[1] = -tt[1]; r.t[2] = -tt[2];
  return r;
}

inline void to_compact_quat(const double R[9], double out[3]) {
  // toCompactQuaternion (g2o/types/slam3d/isometry3d_mappings.cpp:80-85, normalize :40-46)
  Quat q = rot_to_quat(R);
  const double n = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x /= n; q.y /= n; q.z /= n; q.w /= n;
  if (q.w < 0) { q.x = -q.x; q.y = -q.y; q.z = -q.z; }
  out[0] = q.x; out[1] = q.y; out[2] = q.z;
}

inline void from_compact_quat(const double v[3], double R[9]) {
  // fromCompactQuaternion (isometry3d_mappings.cpp:87-94)
  double w = 1 - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (w < 0) {
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  Quat q{v[0], v[1], v[2], std::sqrt(w)};
  quat_to_rot(q, R);
}

// dq/dR of the compact quaternion, with the branch of the rotation->quaternion
// conversion (g2o/types/slam3d/dquat2mat.cpp:36-94). Derived here from the
// closed forms of the four Shepperd branches; column index = c*3 + r (R
// column-major), as the reference's Matrix<3,9> layout.
void compute_dq_dR(const double R[9], double D[27]) {
  auto at = [&](int r, int c) { return R[r * 3 + c]; };
  auto idx = [](int r, int c) { return c * 3 + r; };
  for (int i = 0; i < 27; ++i) D[i] = 0;
  auto set = [&](int qi, int r, int c, double v) { D[qi * 9 + idx(r, c)] += v; };
  const double r00 = at(0, 0), r11 = at(1, 1), r22 = at(2, 2);
  const double tr = r00 + r11 + r22;
  double sign = 1.0;
  if (tr > 0) {
    const double qw = 0.5 * std::sqrt(tr + 1.0);
    const double i4 = 0.25 / qw, i32 = 1.0 / (32.0 * qw * qw * qw);
    const double nx = at(2, 1) - at(1, 2), ny = at(0, 2) - at(2, 0), nz = at(1, 0) - at(0, 1);
    for (int d = 0; d < 3; ++d) {
      set(0, d, d, -nx * i32);
      set(1, d, d, -ny * i32);
      set(2, d, d, -nz * i32);
    }
    set(0, 2, 1, i4); set(0, 1, 2, -i4);
    set(1, 0, 2, i4); set(1, 2, 0, -i4);
    set(2, 1, 0, i4); set(2, 0, 1, -i4);
  } else {
    int i;
    if ((r00 > r11) && (r00 > r22)) i = 0;
    else if (r11 > r22) i = 1;
    else i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    const double s = 0.5 * std::sqrt(1.0 + at(i, i) - at(j, j) - at(k, k));
    const double i4 = 0.25 / s, i8 = 0.125 / s, i32 = 1.0 / (32.0 * s * s * s);
    const double qw = (at(k, j) - at(j, k)) * i4;
    // q_i = s
    set(i, i, i, i8); set(i, j, j, -i8); set(i, k, k, -i8);
    // q_j = (R_ji + R_ij)/(4s), q_k = (R_ki + R_ik)/(4s)
    const double nj = at(j, i) + at(i, j), nk = at(k, i) + at(i, k);
    set(j, j, i, i4); set(j, i, j, i4);
    set(j, i, i, -nj * i32); set(j, j, j, nj * i32); set(j, k, k, nj * i32);
    set(k, k, i, i4); set(k, i, k, i4);
    set(k, i, i, -nk * i32); set(k, j, j, nk * i32); set(k, k, k, nk * i32);
    if (qw <= 0) sign = -1.0;
  }
  if (sign < 0)
    for (int t = 0; t < 27; ++t) D[t] = -D[t];
}

void huber(double e, double delta, double rho[3]) {
  // RobustKernelHuber::robustify (g2o/core/robust_kernel_impl.cpp:60-74)
  const double dsqr = delta * delta;
  if (e <= dsqr) {
    rho[0] = e; rho[1] = 1.; rho[2] = 0.;
  } else {
    const double sqrte = std::sqrt(e);
    rho[0] = 2 * sqrte * delta - dsqr;
    rho[1] = delta / sqrte;
    rho[2] = -0.5 * rho[1] / e;
  }
}

// small dense inverse: 3x3 by cofactors, others Gauss-Jordan with partial pivoting
bool inverse_small(const double* A, int n, double* out) {
  if (n == 3) {
    const double c00 = A[4] * A[8] - A[5] * A[7];
    const double c01 = A[5] * A[6] - A[3] * A[8];
    const double c02 = A[3] * A[7] - A[4] * A[6];
    const double det = A[0] * c00 + A[1] * c01 + A[2] * c02;
    const double id = 1.0 / det;
    out[0] = c00 * id; out[3] = c01 * id; out[6] = c02 * id;
    out[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    out[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    out[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    out[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    out[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    out[8] = (A[0] * A[4] - A[1] * A[3]) * id;
    return std::isfinite(id);
  }
  double M[81], I[81];
  for (int i = 0; i < n * n; ++i) M[i] = A[i];
  for (int i = 0; i < n * n; ++i) I[i] = (i / n == i % n) ? 1.0 : 0.0;
  for (int c = 0; c < n; ++c) {
    int p = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(M[r * n + c]) > std::fabs(M[p * n + c])) p = r;
    if (M[p * n + c] == 0.0) return false;
    if (p != c)
      for (int k = 0; k < n; ++k) {
        std::swap(M[p * n + k], M[c * n + k]);
        std::swap(I[p * n + k], I[c * n + k]);
      }
    const double iv = 1.0 / M[c * n + c];
    for (int k = 0; k < n; ++k) { M[c * n + k] *= iv; I[c * n + k] *= iv; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = M[r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; ++k) { M[r * n + k] -= f * M[c * n + k]; I[r * n + k] -= f * I[c * n + k]; }
    }
  }
  for (int i = 0; i < n * n; ++i) out[i] = I[i];
  return true;
}

// ---------------------------------------------------------- edge functions

int edge_dim(int et) {
  return (et == G2OC_EDGE_SE2 || et == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ) ? 3
         : (et == G2OC_EDGE_SE3 || et == G2OC_EDGE_SE3_EXPMAP)          ? 6
                                                                          : 2;
}
int meas_dim(int et) {
  return (et == G2OC_EDGE_SE2 || et == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ) ? 3
         : et == G2OC_EDGE_SE3                                           ? 12
         : et == G2OC_EDGE_SE3_EXPMAP                                    ? 7
                                                                         : 2;
}
int pose_dim(int pt) { return pt == G2OC_POSE_SE2 ? 3 : pt == G2OC_POSE_BAL_CAMERA ? 9 : 6; }
int pose_est_dim(int pt) {
  return pt == G2OC_POSE_SE2 ? 3 : pt == G2OC_POSE_SE3 ? 12 : pt == G2OC_POSE_BAL_CAMERA ? 9 : 7;
}

// Forward-mode automatic differentiation, the method of g2o's AutoDiff
// (g2o/core/auto_differentiation.h:52-240 over the dual numbers of
// g2o/autodiff/jet.h): every value carries its N partial derivatives, carried
// through + - * / sqrt sin cos by the chain rule. Only what the BAL
// observation uses is defined.
template <int N>
struct Jet {
  double a = 0.0;
  double v[N] = {};
  Jet() = default;
  explicit Jet(double x) : a(x) {}
  Jet(double x, int k) : a(x) { v[k] = 1.0; }
};
template <int N> Jet<N> operator+(const Jet<N>& x, const Jet<N>& y) {
  Jet<N> r(x.a + y.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.v[i] + y.v[i];
  return r;
}
template <int N> Jet<N> operator-(const Jet<N>& x, const Jet<N>& y) {
  Jet<N> r(x.a - y.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.v[i] - y.v[i];
  return r;
}
template <int N> Jet<N> operator-(const Jet<N>& x) {
  Jet<N> r(-x.a);
  for (int i = 0; i < N; ++i) r.v[i] = -x.v[i];
  return r;
}
template <int N> Jet<N> operator*(const Jet<N>& x, const Jet<N>& y) {
  Jet<N> r(x.a * y.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.a * y.v[i] + x.v[i] * y.a;
  return r;
}
template <int N> Jet<N> operator/(const Jet<N>& x, const Jet<N>& y) {
  // (x / y)' = (x' - (x / y) y') / y
  Jet<N> r(x.a / y.a);
  const double inv = 1.0 / y.a;
  for (int i = 0; i < N; ++i) r.v[i] = (x.v[i] - r.a * y.v[i]) * inv;
  return r;
}
template <int N> Jet<N> jsqrt(const Jet<N>& x) {
  Jet<N> r(std::sqrt(x.a));
  const double h = 1.0 / (2.0 * r.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.v[i] * h;
  return r;
}
template <int N> Jet<N> jcos(const Jet<N>& x) {
  Jet<N> r(std::cos(x.a));
  const double d = -std::sin(x.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.v[i] * d;
  return r;
}
template <int N> Jet<N> jsin(const Jet<N>& x) {
  Jet<N> r(std::sin(x.a));
  const double d = std::cos(x.a);
  for (int i = 0; i < N; ++i) r.v[i] = x.v[i] * d;
  return r;
}
inline double jsqrt(double x) { return std::sqrt(x); }
inline double jcos(double x) { return std::cos(x); }
inline double jsin(double x) { return std::sin(x); }
inline double jval(double x) { return x; }
template <int N> double jval(const Jet<N>& x) { return x.a; }

// EdgeObservationBAL::operator() (g2o/examples/bal/bal_example.cpp:160-200):
// Rodrigues rotation of the point by the angle-axis camera(0:3) (first-order
// form X + w x X when |w| == 0), translation camera(3:6), perspective
// division p = -P(0:2) / P(2), radial distortion r(p) = 1 + k1 |p|^2 +
// k2 |p|^4, prediction f r(p) p; error = prediction - measurement. The
// operations and their order follow the reference's expression.
template <typename T>
void bal_error_t(const T* cam, const T* X, const double* z, T e[2]) {
  const T theta2 = cam[0] * cam[0] + cam[1] * cam[1] + cam[2] * cam[2];
  T P[3];
  if (jval(theta2) > 0.0) {
    const T theta = jsqrt(theta2);
    const T v[3] = {cam[0] / theta, cam[1] / theta, cam[2] / theta};
    const T cth = jcos(theta), sth = jsin(theta);
    const T vXp[3] = {v[1] * X[2] - v[2] * X[1], v[2] * X[0] - v[0] * X[2], v[0] * X[1] - v[1] * X[0]};
    const T vDotp = v[0] * X[0] + v[1] * X[1] + v[2] * X[2];
    const T oneMinusCth = T(1.0) - cth;
    for (int i = 0; i < 3; ++i) P[i] = X[i] * cth + vXp[i] * sth + v[i] * vDotp * oneMinusCth;
  } else {
    P[0] = X[0] + (cam[1] * X[2] - cam[2] * X[1]);
    P[1] = X[1] + (cam[2] * X[0] - cam[0] * X[2]);
    P[2] = X[2] + (cam[0] * X[1] - cam[1] * X[0]);
  }
  for (int i = 0; i < 3; ++i) P[i] = P[i] + cam[3 + i];
  const T p0 = -P[0] / P[2], p1 = -P[1] / P[2];
  const T r2 = p0 * p0 + p1 * p1;
  const T rp = T(1.0) + cam[7] * r2 + cam[8] * r2 * r2;
  const T fr = cam[6] * rp;
  e[0] = fr * p0 - T(z[0]);
  e[1] = fr * p1 - T(z[1]);
}

void bal_error(const double* cam9, const double* X, const double* z, double e[2]) {
  bal_error_t<double>(cam9, X, z, e);
}

// the Jacobians by forward-mode differentiation of bal_error_t with respect
// to the 9 camera and 3 point estimate entries (AutoDifferentiation::linearize:
// additive vertices, so d e / d estimate): Jp 2x3, Jc 2x9, row-major
void bal_jacobians(const double* cam9, const double* X, const double* z, double Jp[6], double Jc[18]) {
  using J = Jet<12>;
  J c[9], x[3], e[2];
  for (int i = 0; i < 9; ++i) c[i] = J(cam9[i], i);
  for (int i = 0; i < 3; ++i) x[i] = J(X[i], 9 + i);
  bal_error_t<J>(c, x, z, e);
  for (int r = 0; r < 2; ++r) {
    for (int i = 0; i < 9; ++i) Jc[r * 9 + i] = e[r].v[i];
    for (int i = 0; i < 3; ++i) Jp[r * 3 + i] = e[r].v[9 + i];
  }
}

// EdgeStereoSE3ProjectXYZ (g2o/types/sba/edge_project_stereo_xyz.h:52-57,
// edge_project_stereo_xyz.cpp:34-43 and 58-106), vertex0 = point, vertex1 =
// camera. cam_project takes bf as a float reference, so the right image
// coordinate uses bf rounded to single precision; invz = 1.0f / z is a double
// division. The Jacobians keep bf in double precision.
void stereo_error(const double* cam7, const double* X, const double* z, double fx, double fy, double cx, double cy,
                  double bf, double e[3]);
void stereo_jacobians(const double* cam7, const double* X, double fx, double fy, double bf, double Jp[9],
                      double Jc[18]);

struct SE2v {
  double x, y, th;
};
inline SE2v se2_inv(const SE2v& a) {
  // SE2::inverse (g2o/types/slam2d/se2.h:80-90)
  SE2v r;
  r.th = normalize_theta(-a.th);
  const double c = std::cos(r.th), s = std::sin(r.th);
  r.x = c * (-a.x) - s * (-a.y);
  r.y = s * (-a.x) + c * (-a.y);
  return r;
}
inline SE2v se2_mul(const SE2v& a, const SE2v& b) {
  // SE2::operator*= (se2.h:72-77)
  const double c = std::cos(a.th), s = std::sin(a.th);
  SE2v r;
  r.x = a.x + c * b.x - s * b.y;
  r.y = a.y + s * b.x + c * b.y;
  r.th = normalize_theta(a.th + b.th);
  return r;
}

// EdgeProjectXYZ2UV (g2o/types/sba/edge_project_xyz2uv.cpp:50-97), vertex0 =
// point, vertex1 = camera; CameraParameters::cam_map (parameter_cameraparameters.cpp:59-65),
// fx = fy = focal_length. EdgeSE3ProjectXYZ (g2o/types/sba/edge_project_xyz.cpp:43-100)
// is the same with its own fx, fy, cx, cy.
void ba_error(const double* cam7, const double* X, const double* z, double fx, double fy, double cx, double cy,
              double e[2]) {
  SE3Q T = se3q_load(cam7);
  double Xc[3];
  quat_rotate(T.q, X, Xc);
  Xc[0] += T.t[0]; Xc[1] += T.t[1]; Xc[2] += T.t[2];
  const double u = Xc[0] / Xc[2] * fx + cx;
  const double v = Xc[1] / Xc[2] * fy + cy;
  e[0] = z[0] - u;
  e[1] = z[1] - v;
}

void stereo_error(const double* cam7, const double* X, const double* z, double fx, double fy, double cx, double cy,
                  double bf, double e[3]) {
  SE3Q T = se3q_load(cam7);
  double Xc[3];
  quat_rotate(T.q, X, Xc);
  Xc[0] += T.t[0]; Xc[1] += T.t[1]; Xc[2] += T.t[2];
  const double invz = 1.0 / Xc[2];
  const double u = Xc[0] * invz * fx + cx;
  const double v = Xc[1] * invz * fy + cy;
  const double ur = u - (double)(float)bf * invz;
  e[0] = z[0] - u;
  e[1] = z[1] - v;
  e[2] = z[2] - ur;
}

void stereo_jacobians(const double* cam7, const double* X, double fx, double fy, double bf, double Jp[9],
                      double Jc[18]) {
  SE3Q T = se3q_load(cam7);
  double Xc[3];
  quat_rotate(T.q, X, Xc);
  Xc[0] += T.t[0]; Xc[1] += T.t[1]; Xc[2] += T.t[2];
  const double x = Xc[0], y = Xc[1], z = Xc[2], z2 = z * z;
  double R[9];
  quat_to_rot(T.q, R);
  for (int c = 0; c < 3; ++c) {
    Jp[c] = -fx * R[c] / z + fx * x * R[6 + c] / z2;
    Jp[3 + c] = -fy * R[3 + c] / z + fy * y * R[6 + c] / z2;
    Jp[6 + c] = Jp[c] - bf * R[6 + c] / z2;
  }
  Jc[0] = x * y / z2 * fx;
  Jc[1] = -(1 + (x * x / z2)) * fx;
  Jc[2] = y / z * fx;
  Jc[3] = -1. / z * fx;
  Jc[4] = 0;
  Jc[5] = x / z2 * fx;
  Jc[6] = (1 + y * y / z2) * fy;
  Jc[7] = -x * y / z2 * fy;
  Jc[8] = -x / z * fy;
  Jc[9] = 0;
  Jc[10] = -1. / z * fy;
  Jc[11] = y / z2 * fy;
  Jc[12] = Jc[0] - bf * y / z2;
  Jc[13] = Jc[1] + bf * x / z2;
  Jc[14] = Jc[2];
  Jc[15] = Jc[3];
  Jc[16] = 0;
  Jc[17] = Jc[5] - bf / z2;
}

void ba_jacobians(const double* cam7, const double* X, double fx, double fy, double Jp[6], double Jc[12]) {
  SE3Q T = se3q_load(cam7);
  double Xc[3];
  quat_rotate(T.q, X, Xc);
  Xc[0] += T.t[0]; Xc[1] += T.t[1]; Xc[2] += T.t[2];
  const double x = Xc[0], y = Xc[1], z = Xc[2], z2 = z * z;
  double R[9];
  quat_to_rot(T.q, R);
  const double tmp[6] = {fx, 0, -x / z * fx, 0, fy, -y / z * fy};
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 3; ++c)
      Jp[r * 3 + c] = -1. / z * (tmp[r * 3] * R[c] + tmp[r * 3 + 1] * R[3 + c] + tmp[r * 3 + 2] * R[6 + c]);
  Jc[0] = x * y / z2 * fx;
  Jc[1] = -(1 + (x * x / z2)) * fx;
  Jc[2] = y / z * fx;
  Jc[3] = -1. / z * fx;
  Jc[4] = 0;
  Jc[5] = x / z2 * fx;
  Jc[6] = (1 + y * y / z2) * fy;
  Jc[7] = -x * y / z2 * fy;
  Jc[8] = -x / z * fy;
  Jc[9] = 0;
  Jc[10] = -1. / z * fy;
  Jc[11] = y / z2 * fy;
}

// EdgeSE2 (g2o/types/slam2d/edge_se2.h:46-59, edge_se2.cpp:63-83)
void se2_error(const double* xi, const double* xj, const double* meas, double e[3]) {
  SE2v Zinv = se2_inv({meas[0], meas[1], meas[2]});
  SE2v Xi{xi[0], xi[1], xi[2]}, Xj{xj[0], xj[1], xj[2]};
  SE2v d = se2_mul(Zinv, se2_mul(se2_inv(Xi), Xj));
  e[0] = d.x; e[1] = d.y; e[2] = d.th;
}

void se2_jacobians(const double* xi, const double* xj, const double* meas, double Ji[9], double Jj[9]) {
  const double thetai = xi[2];
  const double dx = xj[0] - xi[0], dy = xj[1] - xi[1];
  const double si = std::sin(thetai), ci = std::cos(thetai);
  const double A[9] = {-ci, -si, -si * dx + ci * dy, si, -ci, -ci * dx - si * dy, 0, 0, -1};
  const double B[9] = {ci, si, 0, -si, ci, 0, 0, 0, 1};
  SE2v Zinv = se2_inv({meas[0], meas[1], meas[2]});
  const double c = std::cos(Zinv.th), s = std::sin(Zinv.th);
  const double Z[9] = {c, -s, 0, s, c, 0, 0, 0, 1};
  matmul3(Z, A, Ji);
  matmul3(Z, B, Jj);
}

// EdgeSE3 (g2o/types/slam3d/edge_se3.cpp:60-88) and computeEdgeSE3Gradient
// (g2o/types/slam3d/isometry3d_gradients.h:205-279)
void se3_error(const double* xi, const double* xj, const double* meas, double e[6]) {
  Iso3 Zinv = iso_inv(iso_load(meas));
  Iso3 d = iso_mul(iso_mul(Zinv, iso_inv(iso_load(xi))), iso_load(xj));
  e[0] = d.t[0]; e[1] = d.t[1]; e[2] = d.t[2];
  to_compact_quat(d.R, e + 3);
}

void se3_jacobians(const double* xi, const double* xj, const double* meas, double Ji[36], double Jj[36]) {
  const Iso3 A = iso_inv(iso_load(meas));
  const Iso3 B = iso_mul(iso_inv(iso_load(xi)), iso_load(xj));
  const Iso3 E = iso_mul(A, B);
  const double* Re = E.R;
  const double* Ra = A.R;
  const double* Rb = B.R;
  const double* tb = B.t;
  double dq[27];
  compute_dq_dR(Re, dq);
  for (int i = 0; i < 36; ++i) { Ji[i] = 0; Jj[i] = 0; }
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      Ji[r * 6 + c] = -Ra[r * 3 + c];
      Jj[r * 6 + c] = Re[r * 3 + c];
    }
  {
    // skewT(tb) with the reference's factor 2
    const double x = 2 * tb[0], y = 2 * tb[1], z = 2 * tb[2];
    const double S[9] = {0., -z, y, z, 0, -x, -y, x, 0};
    double RS[9];
    matmul3(Ra, S, RS);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) Ji[r * 6 + 3 + c] = RS[r * 3 + c];
  }
  auto apply = [&](const double Sx[9], const double Sy[9], const double Sz[9], const double* Rl, double* J) {
    // J(3:6,3:6) = dq_dR * [vec(Rl*Sx) vec(Rl*Sy) vec(Rl*Sz)] with column-major vec
    double M[3][9];
    const double* S3[3] = {Sx, Sy, Sz};
    for (int k = 0; k < 3; ++k) {
      double P[9];
      matmul3(Rl, S3[k], P);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) M[k][c * 3 + r] = P[r * 3 + c];
    }
    for (int qi = 0; qi < 3; ++qi)
      for (int k = 0; k < 3; ++k) {
        double s = 0;
        for (int t = 0; t < 9; ++t) s += dq[qi * 9 + t] * M[k][t];
        J[(3 + qi) * 6 + 3 + k] = s;
      }
  };
  {
    // skewT(Sxt, Syt, Szt, Rb), factor 2
    double r[9];
    for (int i = 0; i < 9; ++i) r[i] = 2 * Rb[i];
    const double Sx[9] = {0, 0, 0, r[6], r[7], r[8], -r[3], -r[4], -r[5]};
    const double Sy[9] = {-r[6], -r[7], -r[8], 0, 0, 0, r[0], r[1], r[2]};
    const double Sz[9] = {r[3], r[4], r[5], -r[0], -r[1], -r[2], 0, 0, 0};
    apply(Sx, Sy, Sz, Ra, Ji);
  }
  {
    // skew(Sx, Sy, Sz, I), factor 2
    const double Sx[9] = {0, 0, 0, 0, 0, -2, 0, 2, 0};
    const double Sy[9] = {0, 0, 2, 0, 0, 0, -2, 0, 0};
    const double Sz[9] = {0, -2, 0, 2, 0, 0, 0, 0, 0};
    apply(Sx, Sy, Sz, Re, Jj);
  }
}

// -------------------------------------------------- block symmetric matrix
// Upper-triangular blocks listed column-major (the order of
// SparseBlockMatrix::blockCols()); each column's diagonal block comes last.
struct BlockSym {
  int nb = 0;
  std::vector<int> off;      // nb + 1 scalar offsets
  std::vector<int> col_ptr;  // nb + 1
  std::vector<int> row;      // nnzb
  std::vector<size_t> val_off;
  const double* val = nullptr;
  int dim(int i) const { return off[i + 1] - off[i]; }
  int n() const { return off[nb]; }
};

// LinearSolverPCG::solve/mult/multDiag (g2o/solvers/pcg/linear_solver_pcg.hpp:87-205)
struct PCGState {
  double residual = -1.0;
};

int g_threads = 1;

bool pcg_solve(const BlockSym& A, const double* b, double* x, const g2oc_params& prm, PCGState& st,
               int* iters_out) {
  const int n = A.n();
  std::vector<std::vector<double>> J(A.nb);
  std::vector<const double*> diag(A.nb);
  for (int c = 0; c < A.nb; ++c) {
    const int last = A.col_ptr[c + 1] - 1;
    diag[c] = A.val + A.val_off[last];
    const int d = A.dim(c);
    J[c].resize(d * d);
    inverse_small(diag[c], d, J[c].data());
  }
  auto multDiag = [&](const std::vector<double>& src, std::vector<double>& dst, bool useJ) {
    for (int c = 0; c < A.nb; ++c) {
      const int d = A.dim(c), o = A.off[c];
      const double* M = useJ ? J[c].data() : diag[c];
      for (int i = 0; i < d; ++i) {
        double s = 0;
        for (int k = 0; k < d; ++k) s += M[i * d + k] * src[o + k];
        dst[o + i] = s;
      }
    }
  };
  auto mult = [&](const std::vector<double>& src, std::vector<double>& dst) {
    multDiag(src, dst, false);
    for (int c = 0; c < A.nb; ++c) {
      const int dc = A.dim(c), oc = A.off[c];
      for (int p = A.col_ptr[c]; p < A.col_ptr[c + 1] - 1; ++p) {
        const int r = A.row[p], dr = A.dim(r), orr = A.off[r];
        const double* M = A.val + A.val_off[p];
        for (int i = 0; i < dr; ++i) {
          double s = 0;
          for (int k = 0; k < dc; ++k) s += M[i * dc + k] * src[oc + k];
          dst[orr + i] += s;
        }
        for (int k = 0; k < dc; ++k) {
          double s = 0;
          for (int i = 0; i < dr; ++i) s += M[i * dc + k] * src[orr + i];
          dst[oc + k] += s;
        }
      }
    }
  };
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& b2) {
    double s = 0;
    for (int i = 0; i < n; ++i) s += a[i] * b2[i];
    return s;
  };
  std::vector<double> xv(n, 0.0), r(b, b + n), d(n, 0.0), q(n, 0.0), s(n, 0.0);
  multDiag(r, d, true);
  double dn = dot(r, d);
  double d0 = prm.pcg_tolerance * dn;
  if (prm.pcg_absolute_tolerance) {
    if (st.residual > 0.0 && st.residual > d0) d0 = st.residual;
  }
  const int maxIter = prm.pcg_max_iterations < 0 ? n : prm.pcg_max_iterations;
  int it;
  for (it = 0; it < maxIter; ++it) {
    if (dn <= d0) break;
    mult(d, q);
    const double a = dn / dot(d, q);
    for (int i = 0; i < n; ++i) xv[i] += a * d[i];
    for (int i = 0; i < n; ++i) r[i] -= a * q[i];
    multDiag(r, s, true);
    const double dold = dn;
    dn = dot(r, s);
    const double ba = dn / dold;
    for (int i = 0; i < n; ++i) d[i] = s[i] + ba * d[i];
  }
  st.residual = 0.5 * dn;
  std::memcpy(x, xv.data(), n * sizeof(double));
  if (iters_out) *iters_out = it;
  return true;
}

// Sparse block Cholesky (the role of LinearSolverEigen's SimplicialLLT with
// an AMD block ordering, g2o/solvers/eigen/linear_solver_eigen.h:94-191):
// minimum-degree block ordering by the elimination game, then a right-looking
// block LL^T. Any exact FP64 factorization of an SPD matrix gives the same
// solution up to rounding.
bool cholesky_solve(const BlockSym& A, const double* b, double* x) {
  const int nb = A.nb;
  auto key = [nb](int u, int v) -> uint64_t {
    if (u > v) std::swap(u, v);
    return (uint64_t)u * (uint64_t)nb + (uint64_t)v;
  };
  // blocks keyed by (min node, max node), stored as rows=min node
  std::unordered_map<uint64_t, std::vector<double>> B;
  B.reserve(A.row.size() * 2);
  std::vector<std::vector<int>> adj(nb);
  for (int c = 0; c < nb; ++c)
    for (int p = A.col_ptr[c]; p < A.col_ptr[c + 1]; ++p) {
      const int r = A.row[p];
      const double* M = A.val + A.val_off[p];
      B[key(r, c)].assign(M, M + A.dim(r) * A.dim(c));
      if (r != c) { adj[r].push_back(c); adj[c].push_back(r); }
    }
  std::vector<std::set<int>> g(nb);
  for (int i = 0; i < nb; ++i) g[i].insert(adj[i].begin(), adj[i].end());
  std::vector<char> done(nb, 0);
  std::vector<int> order;
  order.reserve(nb);
  std::vector<std::vector<int>> lcol(nb);
  for (int step = 0; step < nb; ++step) {
    int best = -1;
    size_t bd = SIZE_MAX;
    for (int i = 0; i < nb; ++i)
      if (!done[i] && g[i].size() < bd) { bd = g[i].size(); best = i; }
    const int k = best;
    done[k] = 1;
    order.push_back(k);
    std::vector<int> nb_k(g[k].begin(), g[k].end());
    lcol[k] = nb_k;
    for (int u : nb_k) g[u].erase(k);
    for (size_t a = 0; a < nb_k.size(); ++a)
      for (size_t c = a + 1; c < nb_k.size(); ++c) {
        const int u = nb_k[a], v = nb_k[c];
        if (g[u].insert(v).second) {
          g[v].insert(u);
          B[key(u, v)].assign(A.dim(std::min(u, v)) * A.dim(std::max(u, v)), 0.0);
        }
      }
    g[k].clear();
  }
  // accessor for block (u,v) as a dim(u) x dim(v) matrix
  auto get = [&](int u, int v, std::vector<double>& out) {
    const std::vector<double>& M = B[key(u, v)];
    const int du = A.dim(u), dv = A.dim(v);
    out.resize(du * dv);
    if (u <= v) std::memcpy(out.data(), M.data(), du * dv * sizeof(double));
    else
      for (int i = 0; i < du; ++i)
        for (int j = 0; j < dv; ++j) out[i * dv + j] = M[j * du + i];
  };
  auto sub = [&](int u, int v, const std::vector<double>& D) {  // B(u,v) -= D (du x dv)
    std::vector<double>& M = B[key(u, v)];
    const int du = A.dim(u), dv = A.dim(v);
    if (u <= v)
      for (int i = 0; i < du * dv; ++i) M[i] -= D[i];
    else
      for (int i = 0; i < du; ++i)
        for (int j = 0; j < dv; ++j) M[j * du + i] -= D[i * dv + j];
  };
  std::vector<std::vector<double>> Lkk(nb);
  std::unordered_map<uint64_t, std::vector<double>> L;  // L(u,k) for u in lcol[k], dim(u) x dim(k)
  std::vector<double> tmp, tmp2;
  for (int k : order) {
    const int dk = A.dim(k);
    get(k, k, tmp);
    std::vector<double>& Lk = Lkk[k];
    Lk.assign(dk * dk, 0.0);
    for (int j = 0; j < dk; ++j) {
      double s = tmp[j * dk + j];
      for (int t = 0; t < j; ++t) s -= Lk[j * dk + t] * Lk[j * dk + t];
      if (!(s > 0.0)) return false;
      Lk[j * dk + j] = std::sqrt(s);
      for (int i = j + 1; i < dk; ++i) {
        double v = tmp[i * dk + j];
        for (int t = 0; t < j; ++t) v -= Lk[i * dk + t] * Lk[j * dk + t];
        Lk[i * dk + j] = v / Lk[j * dk + j];
      }
    }
    for (int u : lcol[k]) {
      const int du = A.dim(u);
      get(u, k, tmp);  // du x dk ; L_uk = B_uk * Lkk^-T  => solve L_uk Lkk^T = B_uk
      std::vector<double>& Luk = L[(uint64_t)u * nb + k];
      Luk.assign(du * dk, 0.0);
      for (int i = 0; i < du; ++i)
        for (int j = 0; j < dk; ++j) {
          double v = tmp[i * dk + j];
          for (int t = 0; t < j; ++t) v -= Luk[i * dk + t] * Lk[j * dk + t];
          Luk[i * dk + j] = v / Lk[j * dk + j];
        }
    }
    const std::vector<int>& nbk = lcol[k];
    for (size_t a = 0; a < nbk.size(); ++a)
      for (size_t c = a; c < nbk.size(); ++c) {
        const int u = nbk[a], v = nbk[c];
        const std::vector<double>& Lu = L[(uint64_t)u * nb + k];
        const std::vector<double>& Lv = L[(uint64_t)v * nb + k];
        const int du = A.dim(u), dv = A.dim(v);
        tmp2.assign(du * dv, 0.0);
        for (int i = 0; i < du; ++i)
          for (int j = 0; j < dv; ++j) {
            double s = 0;
            for (int t = 0; t < dk; ++t) s += Lu[i * dk + t] * Lv[j * dk + t];
            tmp2[i * dv + j] = s;
          }
        sub(u, v, tmp2);
      }
  }
  std::vector<double> y(b, b + A.n());
  for (int k : order) {
    const int dk = A.dim(k), ok = A.off[k];
    const std::vector<double>& Lk = Lkk[k];
    for (int i = 0; i < dk; ++i) {
      double v = y[ok + i];
      for (int t = 0; t < i; ++t) v -= Lk[i * dk + t] * y[ok + t];
      y[ok + i] = v / Lk[i * dk + i];
    }
    for (int u : lcol[k]) {
      const std::vector<double>& Luk = L[(uint64_t)u * nb + k];
      const int du = A.dim(u), ou = A.off[u];
      for (int i = 0; i < du; ++i) {
        double s = 0;
        for (int t = 0; t < dk; ++t) s += Luk[i * dk + t] * y[ok + t];
        y[ou + i] -= s;
      }
    }
  }
  for (int idx = nb - 1; idx >= 0; --idx) {
    const int k = order[idx];
    const int dk = A.dim(k), ok = A.off[k];
    for (int u : lcol[k]) {
      const std::vector<double>& Luk = L[(uint64_t)u * nb + k];
      const int du = A.dim(u), ou = A.off[u];
      for (int t = 0; t < dk; ++t) {
        double s = 0;
        for (int i = 0; i < du; ++i) s += Luk[i * dk + t] * y[ou + i];
        y[ok + t] -= s;
      }
    }
    const std::vector<double>& Lk = Lkk[k];
    for (int i = dk - 1; i >= 0; --i) {
      double v = y[ok + i];
      for (int t = i + 1; t < dk; ++t) v -= Lk[t * dk + i] * y[ok + t];
      y[ok + i] = v / Lk[i * dk + i];
    }
  }
  for (int i = 0; i < A.n(); ++i) {
    if (!std::isfinite(y[i])) return false;
    x[i] = y[i];
  }
  return true;
}

}  // namespace

// ================================================================= problem

struct orc_problem {
  // graph
  int pose_type = 0, edge_type = 0, C = 0, P = 0, E = 0;
  int pd = 0, ped = 0, D = 0, md = 0;
  std::vector<double> pose, point;
  std::vector<uint8_t> pose_fixed, point_fixed;
  std::vector<int> ev;
  std::vector<double> meas, info, delta;
  double fx = 1, fy = 1, cx = 0, cy = 0, bf = 0;
  bool ba = false;  // EdgeProjectXYZ2UV or EdgeSE3ProjectXYZ
  // the pose edge set: EdgeSE3Expmap between the cameras of a projection-edge graph
  int PE = 0;
  std::vector<int> pev;                      // PE * 2 camera indices
  std::vector<double> pmeas, pinfo, pdelta;  // 7, 36, 1 per edge
  std::vector<int> pact;                     // active pose edges
  std::vector<int> pe_diag0, pe_diag1, pe_off;
  std::vector<char> pe_trans;
  std::vector<double> perr;                  // per active pose edge, 6
  std::vector<int> oplus_count;  // VertexSE3 orthogonalization counter
  // active sets and index mapping (sparse_optimizer.cpp:175-287)
  std::vector<int> act;  // active edge ids
  std::vector<int> pose_h, point_l;
  int Cf = 0, Pf = 0;
  bool schur = false;
  // patterns
  std::vector<std::pair<int, int>> hpp_rc, hpl_rc, schur_rc;  // (row, col)
  std::vector<int> e_hpp_diag0, e_hpp_diag1, e_hpp_off, e_hpl;
  std::vector<char> e_off_transposed;
  std::vector<int> hpl_col_ptr;  // per landmark: range into hpl blocks (sorted by pose row)
  std::vector<int> hpp_diag_idx, schur_diag_idx, hpp_in_schur;
  std::unordered_map<uint64_t, int> schur_map;
  // values
  std::vector<double> hpp, hll, hpl, b;
  std::vector<double> diag_backup_pose, diag_backup_point;
  std::vector<double> err;  // per active edge, D
  // solve
  std::vector<double> x, S, bschur, coeff, dinv;
  g2oc_params prm;
  PCGState pcg;
  double lambda = -1, ni = 2;
  int pcg_iters_last = 0;
  // OptimizationAlgorithmDogleg's members
  double dl_delta = 0, dl_lambda = 0;
  bool dl_was_pd = true;
  int dl_step = 0;
  // backup for LM push/pop
  std::vector<double> pose_bak, point_bak;
  bool system_built = false;
};

namespace {

inline double* pose_ptr(orc_problem* p, int i) { return p->pose.data() + (size_t)i * p->ped; }
inline double* point_ptr(orc_problem* p, int i) { return p->point.data() + (size_t)i * 3; }

void compute_edge_error(orc_problem* p, int e, double* out) {
  const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
  const double* m = p->meas.data() + (size_t)e * p->md;
  if (p->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ)
    stereo_error(pose_ptr(p, v1), point_ptr(p, v0), m, p->fx, p->fy, p->cx, p->cy, p->bf, out);
  else if (p->edge_type == G2OC_EDGE_BAL_OBSERVATION)
    bal_error(pose_ptr(p, v1), point_ptr(p, v0), m, out);
  else if (p->ba)
    ba_error(pose_ptr(p, v1), point_ptr(p, v0), m, p->fx, p->fy, p->cx, p->cy, out);
  else if (p->edge_type == G2OC_EDGE_SE2)
    se2_error(pose_ptr(p, v0), pose_ptr(p, v1), m, out);
  else
    p->edge_type == G2OC_EDGE_SE3_EXPMAP ? se3exp_error(pose_ptr(p, v0), pose_ptr(p, v1), m, out)
                                         : se3_error(pose_ptr(p, v0), pose_ptr(p, v1), m, out);
}

void compute_edge_jac(orc_problem* p, int e, double* J0, double* J1) {
  const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
  const double* m = p->meas.data() + (size_t)e * p->md;
  if (p->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ)
    stereo_jacobians(pose_ptr(p, v1), point_ptr(p, v0), p->fx, p->fy, p->bf, J0, J1);
  else if (p->edge_type == G2OC_EDGE_BAL_OBSERVATION)
    bal_jacobians(pose_ptr(p, v1), point_ptr(p, v0), m, J0, J1);
  else if (p->ba)
    ba_jacobians(pose_ptr(p, v1), point_ptr(p, v0), p->fx, p->fy, J0, J1);
  else if (p->edge_type == G2OC_EDGE_SE2)
    se2_jacobians(pose_ptr(p, v0), pose_ptr(p, v1), m, J0, J1);
  else
    p->edge_type == G2OC_EDGE_SE3_EXPMAP ? se3exp_jacobians(pose_ptr(p, v0), pose_ptr(p, v1), m, J0, J1)
                                         : se3_jacobians(pose_ptr(p, v0), pose_ptr(p, v1), m, J0, J1);
}

double edge_chi2(const orc_problem* p, int e, const double* er) {
  // BaseEdge::chi2 (g2o/core/base_edge.h:99)
  const int D = p->D;
  const double* Om = p->info.data() + (size_t)e * D * D;
  double s = 0;
  for (int i = 0; i < D; ++i) {
    double t = 0;
    for (int j = 0; j < D; ++j) t += Om[i * D + j] * er[j];
    s += er[i] * t;
  }
  return s;
}

double pose_edge_chi2(const orc_problem* p, int e, const double* er) {
  const double* Om = p->pinfo.data() + (size_t)e * 36;
  double s = 0;
  for (int i = 0; i < 6; ++i) {
    double t = 0;
    for (int j = 0; j < 6; ++j) t += Om[i * 6 + j] * er[j];
    s += er[i] * t;
  }
  return s;
}

void compute_active_errors(orc_problem* p) {
  // SparseOptimizer::computeActiveErrors (sparse_optimizer.cpp:78-105)
  const int n = (int)p->act.size();
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int k = 0; k < n; ++k) compute_edge_error(p, p->act[k], p->err.data() + (size_t)k * p->D);
  // EdgeSE3Expmap::computeError (g2o/types/sba/edge_se3_expmap.cpp:48-54)
  for (size_t k = 0; k < p->pact.size(); ++k) {
    const int e = p->pact[k];
    se3exp_error(pose_ptr(p, p->pev[2 * e]), pose_ptr(p, p->pev[2 * e + 1]), p->pmeas.data() + (size_t)e * 7,
                 p->perr.data() + k * 6);
  }
}

void active_chi2(orc_problem* p, double* chi2, double* robust) {
  // activeChi2 / activeRobustChi2 (sparse_optimizer.cpp:107-130)
  double c = 0, r = 0;
  for (size_t k = 0; k < p->act.size(); ++k) {
    const int e = p->act[k];
    const double v = edge_chi2(p, e, p->err.data() + k * p->D);
    c += v;
    if (!p->delta.empty() && p->delta[e] > 0) {
      double rho[3];
      huber(v, p->delta[e], rho);
      r += rho[0];
    } else {
      r += v;
    }
  }
  for (size_t k = 0; k < p->pact.size(); ++k) {
    const int e = p->pact[k];
    const double v = pose_edge_chi2(p, e, p->perr.data() + k * 6);
    c += v;
    if (!p->pdelta.empty() && p->pdelta[e] > 0) {
      double rho[3];
      huber(v, p->pdelta[e], rho);
      r += rho[0];
    } else {
      r += v;
    }
  }
  if (chi2) *chi2 = c;
  if (robust) *robust = r;
}


int build_structure(orc_problem* p) {
  // active edges: all vertices present, not all fixed (sparse_optimizer.cpp:233-258)
  const bool ba = p->ba;
  std::vector<char> pa(p->C, 0), qa(p->P, 0);
  p->act.clear();
  for (int e = 0; e < p->E; ++e) {
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    bool f0, f1;
    if (ba) {
      f0 = p->point_fixed[v0];
      f1 = p->pose_fixed[v1];
    } else {
      f0 = p->pose_fixed[v0];
      f1 = p->pose_fixed[v1];
    }
    if (f0 && f1) continue;
    p->act.push_back(e);
    if (ba) { qa[v0] = 1; pa[v1] = 1; }
    else { pa[v0] = 1; pa[v1] = 1; }
  }
  p->pact.clear();
  for (int e = 0; e < p->PE; ++e) {
    const int v0 = p->pev[2 * e], v1 = p->pev[2 * e + 1];
    if (p->pose_fixed[v0] && p->pose_fixed[v1]) continue;
    p->pact.push_back(e);
    pa[v0] = 1;
    pa[v1] = 1;
  }
  if (p->act.empty()) return G2OC_ERR_BAD_GRAPH;
  // buildIndexMapping (sparse_optimizer.cpp:175-200): free non-marginalized, then marginalized
  p->pose_h.assign(p->C, -1);
  p->point_l.assign(p->P, -1);
  p->Cf = 0;
  for (int i = 0; i < p->C; ++i)
    if (pa[i] && !p->pose_fixed[i]) p->pose_h[i] = p->Cf++;
  p->Pf = 0;
  for (int i = 0; i < p->P; ++i)
    if (qa[i] && !p->point_fixed[i]) p->point_l[i] = p->Pf++;
  p->schur = ba && p->Pf > 0;
  if (p->Cf == 0 && p->Pf == 0) return G2OC_ERR_BAD_GRAPH;
  // BlockSolver::buildStructure (block_solver.hpp:110-269)
  std::set<std::pair<int, int>> hpp_set;  // (col, row)
  for (int i = 0; i < p->Cf; ++i) hpp_set.insert({i, i});
  std::set<std::pair<int, int>> hpl_set;  // (landmark col, pose row)
  for (int e : p->act) {
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    if (ba) {
      const int l = p->point_l[v0], c = p->pose_h[v1];
      if (l >= 0 && c >= 0) hpl_set.insert({l, c});
    } else {
      int a = p->pose_h[v0], c = p->pose_h[v1];
      if (a >= 0 && c >= 0) {
        if (a > c) std::swap(a, c);
        hpp_set.insert({c, a});
      }
    }
  }
  for (int e : p->pact) {
    int a = p->pose_h[p->pev[2 * e]], c = p->pose_h[p->pev[2 * e + 1]];
    if (a >= 0 && c >= 0) {
      if (a > c) std::swap(a, c);
      hpp_set.insert({c, a});
    }
  }
  p->hpp_rc.clear();
  std::map<std::pair<int, int>, int> hpp_idx;
  for (auto& cr : hpp_set) {
    hpp_idx[{cr.second, cr.first}] = (int)p->hpp_rc.size();
    p->hpp_rc.push_back({cr.second, cr.first});
  }
  p->hpp_diag_idx.assign(p->Cf, -1);
  for (int i = 0; i < p->Cf; ++i) p->hpp_diag_idx[i] = hpp_idx[{i, i}];
  p->hpl_rc.clear();
  std::map<std::pair<int, int>, int> hpl_idx;  // (pose, landmark)
  p->hpl_col_ptr.assign(p->Pf + 1, 0);
  for (auto& lc : hpl_set) {
    hpl_idx[{lc.second, lc.first}] = (int)p->hpl_rc.size();
    p->hpl_rc.push_back({lc.second, lc.first});
    p->hpl_col_ptr[lc.first + 1]++;
  }
  for (int l = 0; l < p->Pf; ++l) p->hpl_col_ptr[l + 1] += p->hpl_col_ptr[l];
  const int na = (int)p->act.size();
  p->e_hpp_diag0.assign(na, -1);
  p->e_hpp_diag1.assign(na, -1);
  p->e_hpp_off.assign(na, -1);
  p->e_hpl.assign(na, -1);
  p->e_off_transposed.assign(na, 0);
  for (int k = 0; k < na; ++k) {
    const int e = p->act[k];
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    if (ba) {
      const int l = p->point_l[v0], c = p->pose_h[v1];
      if (c >= 0) p->e_hpp_diag1[k] = p->hpp_diag_idx[c];
      if (l >= 0 && c >= 0) p->e_hpl[k] = hpl_idx[{c, l}];
    } else {
      const int a = p->pose_h[v0], c = p->pose_h[v1];
      if (a >= 0) p->e_hpp_diag0[k] = p->hpp_diag_idx[a];
      if (c >= 0) p->e_hpp_diag1[k] = p->hpp_diag_idx[c];
      if (a >= 0 && c >= 0) {
        p->e_off_transposed[k] = a > c;
        p->e_hpp_off[k] = hpp_idx[{std::min(a, c), std::max(a, c)}];
      }
    }
  }
  const int npa = (int)p->pact.size();
  p->pe_diag0.assign(npa, -1);
  p->pe_diag1.assign(npa, -1);
  p->pe_off.assign(npa, -1);
  p->pe_trans.assign(npa, 0);
  for (int k = 0; k < npa; ++k) {
    const int e = p->pact[k];
    const int a = p->pose_h[p->pev[2 * e]], c = p->pose_h[p->pev[2 * e + 1]];
    if (a >= 0) p->pe_diag0[k] = p->hpp_diag_idx[a];
    if (c >= 0) p->pe_diag1[k] = p->hpp_diag_idx[c];
    if (a >= 0 && c >= 0) {
      p->pe_trans[k] = a > c;
      p->pe_off[k] = hpp_idx[{std::min(a, c), std::max(a, c)}];
    }
  }
  p->perr.assign((size_t)npa * 6, 0.0);
  // Schur pattern = Hpp pattern + co-observing pose pairs (block_solver.hpp:229-266)
  p->schur_rc.clear();
  p->schur_map.clear();
  if (p->schur) {
    std::vector<std::pair<int, int>> cr;  // (col, row)
    cr.reserve(hpp_set.size() + p->hpl_rc.size() * 4);
    for (auto& x : hpp_set) cr.push_back(x);
    for (int l = 0; l < p->Pf; ++l)
      for (int a = p->hpl_col_ptr[l]; a < p->hpl_col_ptr[l + 1]; ++a)
        for (int c = a; c < p->hpl_col_ptr[l + 1]; ++c)
          cr.push_back({p->hpl_rc[c].first, p->hpl_rc[a].first});
    std::sort(cr.begin(), cr.end());
    cr.erase(std::unique(cr.begin(), cr.end()), cr.end());
    for (auto& x : cr) {
      p->schur_map[(uint64_t)x.second * p->Cf + x.first] = (int)p->schur_rc.size();
      p->schur_rc.push_back({x.second, x.first});
    }
    p->schur_diag_idx.assign(p->Cf, -1);
    for (int i = 0; i < p->Cf; ++i) p->schur_diag_idx[i] = p->schur_map[(uint64_t)i * p->Cf + i];
    p->hpp_in_schur.assign(p->hpp_rc.size(), -1);
    for (size_t i = 0; i < p->hpp_rc.size(); ++i)
      p->hpp_in_schur[i] = p->schur_map[(uint64_t)p->hpp_rc[i].first * p->Cf + p->hpp_rc[i].second];
  }
  const int pd = p->pd;
  p->hpp.assign(p->hpp_rc.size() * pd * pd, 0.0);
  p->hll.assign((size_t)p->Pf * 9, 0.0);
  p->hpl.assign(p->hpl_rc.size() * pd * 3, 0.0);
  p->b.assign((size_t)p->Cf * pd + (size_t)p->Pf * 3, 0.0);
  p->x.assign(p->b.size(), 0.0);
  p->err.assign((size_t)na * p->D, 0.0);
  p->system_built = false;
  return G2OC_OK;
}

// robust weighting of one edge: omega' = rho' * Omega, weighted error = -rho' Omega e
// (BaseFixedSizedEdge::constructQuadraticForm, g2o/core/base_fixed_sized_edge.hpp:48-63;
//  robustInformation keeps rho' only, g2o/core/base_edge.h:156-162)
void robust_weights(const orc_problem* p, int e, const double* er, double* Om, double* we) {
  const int D = p->D;
  const double* I = p->info.data() + (size_t)e * D * D;
  double w = 1.0;
  if (!p->delta.empty() && p->delta[e] > 0) {
    double rho[3];
    huber(edge_chi2(p, e, er), p->delta[e], rho);
    w = rho[1];
  }
  for (int i = 0; i < D; ++i) {
    double t = 0;
    for (int j = 0; j < D; ++j) t += I[i * D + j] * er[j];
    we[i] = -t * w;
  }
  for (int i = 0; i < D * D; ++i) Om[i] = w * I[i];
}

// At (da x D), Om (D x D), B (D x db): out(da x db) += A^T Om B
void add_AtOB(const double* A, int da, const double* Om, const double* B, int db, int D, double* out,
              bool transposed_store) {
  double AtO[6 * 6];
  for (int i = 0; i < da; ++i)
    for (int j = 0; j < D; ++j) {
      double s = 0;
      for (int k = 0; k < D; ++k) s += A[k * da + i] * Om[k * D + j];
      AtO[i * D + j] = s;
    }
  for (int i = 0; i < da; ++i)
    for (int j = 0; j < db; ++j) {
      double s = 0;
      for (int k = 0; k < D; ++k) s += AtO[i * D + k] * B[k * db + j];
      if (transposed_store) out[j * da + i] += s;
      else out[i * db + j] += s;
    }
}

void add_Atw(const double* A, int da, const double* we, int D, double* out) {
  for (int i = 0; i < da; ++i) {
    double s = 0;
    for (int k = 0; k < D; ++k) s += A[k * da + i] * we[k];
    out[i] += s;
  }
}

void build_system(orc_problem* p) {
  // BlockSolver::buildSystem (block_solver.hpp:492-565)
  std::fill(p->hpp.begin(), p->hpp.end(), 0.0);
  std::fill(p->hll.begin(), p->hll.end(), 0.0);
  std::fill(p->hpl.begin(), p->hpl.end(), 0.0);
  std::fill(p->b.begin(), p->b.end(), 0.0);
  const int na = (int)p->act.size();
  const int D = p->D, pd = p->pd;
  const bool ba = p->ba;
  const int d0 = ba ? 3 : pd, d1 = pd;
  // linearize in parallel into per-edge buffers, then scatter in edge order
  std::vector<double> J0((size_t)na * D * d0), J1((size_t)na * D * d1);
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int k = 0; k < na; ++k)
    compute_edge_jac(p, p->act[k], J0.data() + (size_t)k * D * d0, J1.data() + (size_t)k * D * d1);
  const size_t psize = (size_t)p->Cf * pd;
  for (int k = 0; k < na; ++k) {
    const int e = p->act[k];
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    double Om[36], we[6];
    robust_weights(p, e, p->err.data() + (size_t)k * D, Om, we);
    const double* A0 = J0.data() + (size_t)k * D * d0;
    const double* A1 = J1.data() + (size_t)k * D * d1;
    // vertex 0
    bool free0, free1;
    double *H00 = nullptr, *b0 = nullptr, *H11 = nullptr, *b1 = nullptr;
    if (ba) {
      const int l = p->point_l[v0], c = p->pose_h[v1];
      free0 = l >= 0;
      free1 = c >= 0;
      if (free0) { H00 = p->hll.data() + (size_t)l * 9; b0 = p->b.data() + psize + (size_t)l * 3; }
      if (free1) { H11 = p->hpp.data() + (size_t)p->e_hpp_diag1[k] * pd * pd; b1 = p->b.data() + (size_t)c * pd; }
    } else {
      const int a = p->pose_h[v0], c = p->pose_h[v1];
      free0 = a >= 0;
      free1 = c >= 0;
      if (free0) { H00 = p->hpp.data() + (size_t)p->e_hpp_diag0[k] * pd * pd; b0 = p->b.data() + (size_t)a * pd; }
      if (free1) { H11 = p->hpp.data() + (size_t)p->e_hpp_diag1[k] * pd * pd; b1 = p->b.data() + (size_t)c * pd; }
    }
    if (free0) {
      add_Atw(A0, d0, we, D, b0);
      add_AtOB(A0, d0, Om, A0, d0, D, H00, false);
      if (free1) {
        if (ba) {
          add_AtOB(A0, d0, Om, A1, d1, D, p->hpl.data() + (size_t)p->e_hpl[k] * pd * 3, true);
        } else {
          add_AtOB(A0, d0, Om, A1, d1, D, p->hpp.data() + (size_t)p->e_hpp_off[k] * pd * pd,
                   p->e_off_transposed[k]);
        }
      }
    }
    if (free1) {
      add_Atw(A1, d1, we, D, b1);
      add_AtOB(A1, d1, Om, A1, d1, D, H11, false);
    }
  }
  // the pose edges (EdgeSE3Expmap::linearizeOplus, edge_se3_expmap.cpp:56-68),
  // as the generic binary-edge branch above
  for (size_t k = 0; k < p->pact.size(); ++k) {
    const int e = p->pact[k];
    const int v0 = p->pev[2 * e], v1 = p->pev[2 * e + 1];
    double J0[36], J1[36];
    se3exp_jacobians(pose_ptr(p, v0), pose_ptr(p, v1), p->pmeas.data() + (size_t)e * 7, J0, J1);
    const double* er = p->perr.data() + k * 6;
    const double* I = p->pinfo.data() + (size_t)e * 36;
    double w = 1.0;
    if (!p->pdelta.empty() && p->pdelta[e] > 0) {
      double rho[3];
      huber(pose_edge_chi2(p, e, er), p->pdelta[e], rho);
      w = rho[1];
    }
    double Om[36], we[6];
    for (int i = 0; i < 6; ++i) {
      double t = 0;
      for (int j = 0; j < 6; ++j) t += I[i * 6 + j] * er[j];
      we[i] = -t * w;
    }
    for (int i = 0; i < 36; ++i) Om[i] = w * I[i];
    const int a = p->pose_h[v0], c = p->pose_h[v1];
    if (a >= 0) {
      add_Atw(J0, 6, we, 6, p->b.data() + (size_t)a * 6);
      add_AtOB(J0, 6, Om, J0, 6, 6, p->hpp.data() + (size_t)p->pe_diag0[k] * 36, false);
      if (c >= 0) add_AtOB(J0, 6, Om, J1, 6, 6, p->hpp.data() + (size_t)p->pe_off[k] * 36, p->pe_trans[k]);
    }
    if (c >= 0) {
      add_Atw(J1, 6, we, 6, p->b.data() + (size_t)c * 6);
      add_AtOB(J1, 6, Om, J1, 6, 6, p->hpp.data() + (size_t)p->pe_diag1[k] * 36, false);
    }
  }
  p->system_built = true;
}

void set_lambda(orc_problem* p, double lambda) {
  // BlockSolver::setLambda (block_solver.hpp:567-590), with backup
  const int pd = p->pd;
  p->diag_backup_pose.resize((size_t)p->Cf * pd);
  p->diag_backup_point.resize((size_t)p->Pf * 3);
  for (int i = 0; i < p->Cf; ++i) {
    double* B = p->hpp.data() + (size_t)p->hpp_diag_idx[i] * pd * pd;
    for (int d = 0; d < pd; ++d) {
      p->diag_backup_pose[(size_t)i * pd + d] = B[d * pd + d];
      B[d * pd + d] += lambda;
    }
  }
  for (int i = 0; i < p->Pf; ++i) {
    double* B = p->hll.data() + (size_t)i * 9;
    for (int d = 0; d < 3; ++d) {
      p->diag_backup_point[(size_t)i * 3 + d] = B[d * 4];
      B[d * 4] += lambda;
    }
  }
}

void restore_diagonal(orc_problem* p) {
  // BlockSolver::restoreDiagonal (block_solver.hpp:592-606)
  const int pd = p->pd;
  for (int i = 0; i < p->Cf; ++i) {
    double* B = p->hpp.data() + (size_t)p->hpp_diag_idx[i] * pd * pd;
    for (int d = 0; d < pd; ++d) B[d * pd + d] = p->diag_backup_pose[(size_t)i * pd + d];
  }
  for (int i = 0; i < p->Pf; ++i) {
    double* B = p->hll.data() + (size_t)i * 9;
    for (int d = 0; d < 3; ++d) B[d * 4] = p->diag_backup_point[(size_t)i * 3 + d];
  }
}

BlockSym make_blocksym(int nb, int bd, const std::vector<std::pair<int, int>>& rc, const double* val) {
  BlockSym A;
  A.nb = nb;
  A.off.resize(nb + 1);
  for (int i = 0; i <= nb; ++i) A.off[i] = i * bd;
  A.col_ptr.assign(nb + 1, 0);
  A.row.resize(rc.size());
  A.val_off.resize(rc.size());
  for (size_t k = 0; k < rc.size(); ++k) {
    A.col_ptr[rc[k].second + 1]++;
    A.row[k] = rc[k].first;
    A.val_off[k] = k * bd * bd;
  }
  for (int i = 0; i < nb; ++i) A.col_ptr[i + 1] += A.col_ptr[i];
  A.val = val;
  return A;
}

void schur_complement(orc_problem* p) {
  // Schur part of BlockSolver::solve (block_solver.hpp:346-433)
  const int pd = p->pd;
  const size_t psize = (size_t)p->Cf * pd;
  p->S.assign(p->schur_rc.size() * pd * pd, 0.0);
  for (size_t i = 0; i < p->hpp_rc.size(); ++i)
    std::memcpy(p->S.data() + (size_t)p->hpp_in_schur[i] * pd * pd, p->hpp.data() + i * pd * pd,
                pd * pd * sizeof(double));
  p->coeff.assign(psize, 0.0);
  p->dinv.assign((size_t)p->Pf * 9, 0.0);
  const int Pf = p->Pf;
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int l = 0; l < Pf; ++l) inverse_small(p->hll.data() + (size_t)l * 9, 3, p->dinv.data() + (size_t)l * 9);
  for (int l = 0; l < p->Pf; ++l) {
    const double* Dinv = p->dinv.data() + (size_t)l * 9;
    const double* bl = p->b.data() + psize + (size_t)l * 3;
    double db[3];
    matvec3(Dinv, bl, db);
    for (int a = p->hpl_col_ptr[l]; a < p->hpl_col_ptr[l + 1]; ++a) {
      const int i1 = p->hpl_rc[a].first;
      const double* Bi = p->hpl.data() + (size_t)a * pd * 3;
      double BD[27];
      for (int r = 0; r < pd; ++r)
        for (int c = 0; c < 3; ++c)
          BD[r * 3 + c] = Bi[r * 3] * Dinv[c] + Bi[r * 3 + 1] * Dinv[3 + c] + Bi[r * 3 + 2] * Dinv[6 + c];
      double* cf = p->coeff.data() + (size_t)i1 * pd;
      for (int r = 0; r < pd; ++r) cf[r] += Bi[r * 3] * db[0] + Bi[r * 3 + 1] * db[1] + Bi[r * 3 + 2] * db[2];
      for (int c2 = a; c2 < p->hpl_col_ptr[l + 1]; ++c2) {
        const int i2 = p->hpl_rc[c2].first;
        const double* Bj = p->hpl.data() + (size_t)c2 * pd * 3;
        double* Sb = p->S.data() + (size_t)p->schur_map[(uint64_t)i1 * p->Cf + i2] * pd * pd;
        for (int r = 0; r < pd; ++r)
          for (int c = 0; c < pd; ++c)
            Sb[r * pd + c] -= BD[r * 3] * Bj[c * 3] + BD[r * 3 + 1] * Bj[c * 3 + 1] + BD[r * 3 + 2] * Bj[c * 3 + 2];
      }
    }
  }
  p->bschur.resize(psize);
  for (size_t i = 0; i < psize; ++i) p->bschur[i] = p->b[i] - p->coeff[i];
}

bool linear_solve(orc_problem* p, const BlockSym& A, const double* rhs, double* out) {
  if (p->prm.linear_solver == G2OC_LINEAR_CHOLESKY) {
    p->pcg_iters_last = 0;
    return cholesky_solve(A, rhs, out);
  }
  int it = 0;
  bool ok = pcg_solve(A, rhs, out, p->prm, p->pcg, &it);
  p->pcg_iters_last = it;
  return ok;
}

bool block_solver_solve(orc_problem* p, double* t_schur, double* t_linear) {
  // BlockSolver::solve (block_solver.hpp:331-477)
  const int pd = p->pd;
  const size_t psize = (size_t)p->Cf * pd;
  std::fill(p->x.begin(), p->x.end(), 0.0);
  if (!p->schur) {
    double t = now_s();
    BlockSym A = make_blocksym(p->Cf, pd, p->hpp_rc, p->hpp.data());
    bool ok = p->Cf > 0 ? linear_solve(p, A, p->b.data(), p->x.data()) : true;
    if (t_linear) *t_linear = now_s() - t;
    return ok;
  }
  double t = now_s();
  schur_complement(p);
  if (t_schur) *t_schur = now_s() - t;
  t = now_s();
  bool ok = true;
  if (p->Cf > 0) {
    BlockSym A = make_blocksym(p->Cf, pd, p->schur_rc, p->S.data());
    ok = linear_solve(p, A, p->bschur.data(), p->x.data());
  }
  if (t_linear) *t_linear = now_s() - t;
  if (!ok) return false;
  // back-substitution: xl = Dinv (bl - Hpl^T xp)
  const int Pf = p->Pf;
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int l = 0; l < Pf; ++l) {
    double cl[3];
    const double* bl = p->b.data() + psize + (size_t)l * 3;
    cl[0] = bl[0]; cl[1] = bl[1]; cl[2] = bl[2];
    for (int a = p->hpl_col_ptr[l]; a < p->hpl_col_ptr[l + 1]; ++a) {
      const int i1 = p->hpl_rc[a].first;
      const double* Bi = p->hpl.data() + (size_t)a * pd * 3;
      const double* xp = p->x.data() + (size_t)i1 * pd;
      for (int c = 0; c < 3; ++c) {
        double s = 0;
        for (int r = 0; r < pd; ++r) s += Bi[r * 3 + c] * (-xp[r]);
        cl[c] += s;
      }
    }
    matvec3(p->dinv.data() + (size_t)l * 9, cl, p->x.data() + psize + (size_t)l * 3);
  }
  return true;
}

void vertex_oplus_pose(orc_problem* p, int i, const double* u) {
  double* est = pose_ptr(p, i);
  if (p->pose_type == G2OC_POSE_BAL_CAMERA) {
    // VertexCameraBAL::oplusImpl (g2o/examples/bal/bal_example.cpp:88-91)
    for (int k = 0; k < 9; ++k) est[k] += u[k];
  } else if (p->pose_type == G2OC_POSE_SE3EXPMAP) {
    // VertexSE3Expmap::oplusImpl (g2o/types/sba/vertex_se3_expmap.cpp:48-51)
    SE3Q T = se3q_load(est);
    se3q_store(se3q_mul(se3q_exp(u), T), est);
  } else if (p->pose_type == G2OC_POSE_SE2) {
    // VertexSE2::oplusImpl (g2o/types/slam2d/vertex_se2.h:48-54)
    est[0] += u[0];
    est[1] += u[1];
    est[2] = normalize_theta(est[2] + u[2]);
  } else {
    // VertexSE3::oplusImpl (g2o/types/slam3d/vertex_se3.h:99-108)
    Iso3 X = iso_load(est);
    Iso3 inc;
    from_compact_quat(u + 3, inc.R);
    inc.t[0] = u[0]; inc.t[1] = u[1]; inc.t[2] = u[2];
    Iso3 Y = iso_mul(X, inc);
    if (++p->oplus_count[i] > 1000) {
      p->oplus_count[i] = 0;
      // approximateNearestOrthogonalMatrix (isometry3d_mappings.h:81-85)
      double E[9];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          E[r * 3 + c] = Y.R[r] * Y.R[c] + Y.R[3 + r] * Y.R[3 + c] + Y.R[6 + r] * Y.R[6 + c] - (r == c ? 1.0 : 0.0);
      double RE[9];
      matmul3(Y.R, E, RE);
      for (int k = 0; k < 9; ++k) Y.R[k] -= 0.5 * RE[k];
    }
    iso_store(Y, est);
  }
}

void update(orc_problem* p, const double* x) {
  // SparseOptimizer::update (sparse_optimizer.cpp:457-468): walk _ivMap
  const int pd = p->pd;
  for (int i = 0; i < p->C; ++i)
    if (p->pose_h[i] >= 0) vertex_oplus_pose(p, i, x + (size_t)p->pose_h[i] * pd);
  const size_t psize = (size_t)p->Cf * pd;
  for (int i = 0; i < p->P; ++i)
    if (p->point_l[i] >= 0) {
      const double* u = x + psize + (size_t)p->point_l[i] * 3;
      double* e = point_ptr(p, i);
      e[0] += u[0]; e[1] += u[1]; e[2] += u[2];
    }
}

void push(orc_problem* p) { p->pose_bak = p->pose; p->point_bak = p->point; }
void pop(orc_problem* p) { p->pose = p->pose_bak; p->point = p->point_bak; }

double compute_lambda_init(orc_problem* p) {
  // computeLambdaInit (optimization_algorithm_levenberg.cpp:155-167)
  if (p->prm.initial_lambda > 0) return p->prm.initial_lambda;
  double m = 0;
  const int pd = p->pd;
  for (int i = 0; i < p->Cf; ++i) {
    const double* B = p->hpp.data() + (size_t)p->hpp_diag_idx[i] * pd * pd;
    for (int d = 0; d < pd; ++d) m = std::max(std::fabs(B[d * pd + d]), m);
  }
  for (int i = 0; i < p->Pf; ++i)
    for (int d = 0; d < 3; ++d) m = std::max(std::fabs(p->hll[(size_t)i * 9 + d * 4]), m);
  return p->prm.tau * m;
}

double compute_scale(orc_problem* p) {
  // computeScale (optimization_algorithm_levenberg.cpp:169-176)
  double s = 0;
  for (size_t j = 0; j < p->x.size(); ++j) s += p->x[j] * (p->lambda * p->x[j] + p->b[j]);
  return s;
}

int lm_solve(orc_problem* p, int iteration, g2oc_iteration_stats* st) {
  // OptimizationAlgorithmLevenberg::solve (optimization_algorithm_levenberg.cpp:60-153)
  double t = now_s();
  compute_active_errors(p);
  if (st) st->time_residuals = now_s() - t;
  t = now_s();
  double currentChi;
  active_chi2(p, nullptr, &currentChi);
  build_system(p);
  if (st) st->time_quadratic_form = now_s() - t;
  if (iteration == 0) {
    p->lambda = compute_lambda_init(p);
    p->ni = 2;
  }
  double rho = 0;
  int qmax = 0;
  const int maxTrials = p->prm.max_trials_after_failure;
  do {
    push(p);
    t = now_s();
    set_lambda(p, p->lambda);
    double ts = 0, tl = 0;
    bool ok2 = block_solver_solve(p, &ts, &tl);
    if (st) {
      st->time_schur_complement += ts;
      st->time_linear_solver += tl;
      st->iterations_linear_solver += p->pcg_iters_last;
      st->levenberg_iterations++;
    }
    t = now_s();
    update(p, p->x.data());
    if (st) st->time_update += now_s() - t;
    restore_diagonal(p);
    compute_active_errors(p);
    double tempChi;
    active_chi2(p, nullptr, &tempChi);
    if (!ok2) tempChi = std::numeric_limits<double>::max();
    rho = currentChi - tempChi;
    double scale = ok2 ? compute_scale(p) + 1e-3 : 1;
    rho /= scale;
    if (rho > 0 && std::isfinite(tempChi) && ok2) {
      double alpha = 1. - std::pow((2 * rho - 1), 3);
      alpha = std::min(alpha, 2. / 3.);
      const double scaleFactor = std::max(1. / 3., alpha);
      p->lambda *= scaleFactor;
      p->ni = 2;
      currentChi = tempChi;
    } else {
      p->lambda *= p->ni;
      p->ni *= 2;
      pop(p);
      if (!std::isfinite(p->lambda)) break;
    }
    qmax++;
  } while (rho < 0 && qmax < maxTrials);
  if (qmax == maxTrials || rho == 0 || !std::isfinite(p->lambda)) return G2OC_RESULT_TERMINATE;
  return G2OC_RESULT_OK;
}

void multiply_hessian(orc_problem* p, const double* src, double* dest) {
  // BlockSolver::multiplyHessian (g2o/core/block_solver.h:96):
  // _Hpp->multiplySymmetricUpperTriangle, the pose part only
  const int pd = p->pd;
  std::fill(dest, dest + p->x.size(), 0.0);
  for (size_t k = 0; k < p->hpp_rc.size(); ++k) {
    const int r = p->hpp_rc[k].first, c = p->hpp_rc[k].second;
    const double* B = p->hpp.data() + k * pd * pd;
    for (int i = 0; i < pd; ++i)
      for (int j = 0; j < pd; ++j) dest[(size_t)r * pd + i] += B[i * pd + j] * src[(size_t)c * pd + j];
    if (r != c)
      for (int i = 0; i < pd; ++i)
        for (int j = 0; j < pd; ++j) dest[(size_t)c * pd + j] += B[i * pd + j] * src[(size_t)r * pd + i];
  }
}

double vdot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
  return s;
}

int dl_solve(orc_problem* p, int iteration, g2oc_iteration_stats* st) {
  // OptimizationAlgorithmDogleg::solve (g2o/core/optimization_algorithm_dogleg.cpp:62-180)
  const size_t n = p->x.size();
  if (iteration == 0) {
    p->dl_delta = p->prm.initial_delta;
    p->dl_lambda = p->prm.initial_lambda > 0 ? p->prm.initial_lambda : 1e-7;
    p->dl_was_pd = true;
  }
  compute_active_errors(p);
  double currentChi;
  active_chi2(p, nullptr, &currentChi);
  build_system(p);
  const std::vector<double>& b = p->b;
  std::vector<double> aux(n), hsd(n), hdl(n), hgn;
  multiply_hessian(p, b.data(), aux.data());
  const double bNormSquared = vdot(b, b);
  const double alpha = bNormSquared / vdot(aux, b);
  for (size_t i = 0; i < n; ++i) hsd[i] = alpha * b[i];
  const double hsdSqr = vdot(hsd, hsd);
  const double hsdNorm = std::sqrt(hsdSqr);
  double hgnNorm = -1;
  bool solvedGaussNewton = false, goodStep = false;
  int numTries = 0;
  const int maxTrials = p->prm.max_trials_after_failure;
  do {
    ++numTries;
    if (!solvedGaussNewton) {
      const double minLambda = 1e-12, maxLambda = 1e3;
      solvedGaussNewton = true;
      bool solverOk = false;
      while (!solverOk) {
        if (!p->dl_was_pd) set_lambda(p, p->dl_lambda);
        double ts = 0, tl = 0;
        solverOk = block_solver_solve(p, &ts, &tl);
        if (st) {
          st->time_schur_complement += ts;
          st->time_linear_solver += tl;
          st->iterations_linear_solver += p->pcg_iters_last;
        }
        if (!p->dl_was_pd) restore_diagonal(p);
        p->dl_was_pd = p->dl_was_pd && solverOk;
        if (!p->dl_was_pd) {
          if (solverOk) {
            p->dl_lambda = std::max(minLambda, p->dl_lambda / (0.5 * p->prm.lambda_factor));
          } else {
            p->dl_lambda *= p->prm.lambda_factor;
            if (p->dl_lambda > maxLambda) {
              p->dl_lambda = maxLambda;
              return G2OC_RESULT_FAIL;
            }
          }
        }
      }
      hgn = p->x;
      hgnNorm = std::sqrt(vdot(hgn, hgn));
    }
    const double delta = p->dl_delta;
    if (hgnNorm < delta) {
      hdl = hgn;
      p->dl_step = 2;
    } else if (hsdNorm > delta) {
      for (size_t i = 0; i < n; ++i) hdl[i] = delta / hsdNorm * hsd[i];
      p->dl_step = 1;
    } else {
      for (size_t i = 0; i < n; ++i) aux[i] = hgn[i] - hsd[i];
      const double c = vdot(hsd, aux);
      const double bmaSquaredNorm = vdot(aux, aux);
      double beta;
      if (c <= 0.)
        beta = (-c + std::sqrt(c * c + bmaSquaredNorm * (delta * delta - hsdSqr))) / bmaSquaredNorm;
      else
        beta = (delta * delta - hsdSqr) / (c + std::sqrt(c * c + bmaSquaredNorm * (delta * delta - hsdSqr)));
      for (size_t i = 0; i < n; ++i) hdl[i] = hsd[i] + beta * aux[i];
      p->dl_step = 3;
    }
    multiply_hessian(p, hdl.data(), aux.data());
    double linearGain = -1 * vdot(aux, hdl) + 2 * vdot(b, hdl);
    push(p);
    update(p, hdl.data());
    compute_active_errors(p);
    double newChi;
    active_chi2(p, nullptr, &newChi);
    const double nonLinearGain = currentChi - newChi;
    if (std::fabs(linearGain) < 1e-12) linearGain = 1e-12;
    const double rho = nonLinearGain / linearGain;
    if (rho > 0) goodStep = true;
    else pop(p);
    if (rho > 0.75) p->dl_delta = std::max(p->dl_delta, 3 * std::sqrt(vdot(hdl, hdl)));
    else if (rho < 0.25) p->dl_delta *= 0.5;
  } while (!goodStep && numTries < maxTrials);
  if (st) st->levenberg_iterations = numTries;
  if (numTries == maxTrials || !goodStep) return G2OC_RESULT_TERMINATE;
  return G2OC_RESULT_OK;
}

double so_point_chi2(orc_problem* p, const std::vector<int>& edges) {
  double s = 0;
  for (int e : edges) {
    double er[2];
    compute_edge_error(p, e, er);
    const double c = edge_chi2(p, e, er);
    if (!p->delta.empty() && p->delta[e] > 0) {
      double rho[3];
      huber(c, p->delta[e], rho);
      s += rho[0];
    } else {
      s += c;
    }
  }
  return s;
}

int so_calc(orc_problem* p, int num_iters, int num_max_trials) {
  // StructureOnlySolver<3>::calc (g2o/solvers/structure_only/structure_only_solver.h:66-215)
  // over the free landmarks, each with its edges ordered by camera
  std::vector<std::vector<int>> track(p->P);
  for (int e : p->act) track[p->ev[2 * e]].push_back(e);
  for (auto& t : track)
    std::stable_sort(t.begin(), t.end(), [&](int a, int b) { return p->ev[2 * a + 1] < p->ev[2 * b + 1]; });
  for (int i = 0; i < p->P; ++i) {
    if (p->point_l[i] < 0) continue;  // fixed or inactive
    const std::vector<int>& tr = track[i];
    double* X = point_ptr(p, i);
    double chi2 = so_point_chi2(p, tr);
    double mu = 0.01, nu = 2;
    bool stop = false;
    for (int ig = 0; ig < num_iters; ++ig) {
      double H[9] = {0}, b[3] = {0};
      for (int e : tr) {
        double er[2], Jp[6], Jc[18];
        compute_edge_error(p, e, er);
        compute_edge_jac(p, e, Jp, Jc);
        const double* Om = p->info.data() + (size_t)e * 4;
        double w = 1;
        if (!p->delta.empty() && p->delta[e] > 0) {
          double rho[3];
          huber(edge_chi2(p, e, er), p->delta[e], rho);
          w = rho[1];
        }
        // constructQuadraticForm with robustInformation (base_fixed_sized_edge.hpp:48-63)
        const double r0 = -(Om[0] * er[0] + Om[1] * er[1]) * w, r1 = -(Om[2] * er[0] + Om[3] * er[1]) * w;
        for (int a = 0; a < 3; ++a) {
          b[a] += Jp[a] * r0 + Jp[3 + a] * r1;
          for (int c = 0; c < 3; ++c)
            H[a * 3 + c] += w * (Jp[a] * (Om[0] * Jp[c] + Om[1] * Jp[3 + c]) + Jp[3 + a] * (Om[2] * Jp[c] + Om[3] * Jp[3 + c]));
        }
      }
      if (std::sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) < 0.001) break;
      int trial = 0;
      do {
        // (H + mu I) delta = b by an LDL^T factorization (Eigen::LDLT in g2o;
        // isPositive: every pivot positive)
        const double d0 = H[0] + mu;
        const double l10 = H[1] / d0, l20 = H[2] / d0;
        const double d1 = H[4] + mu - l10 * l10 * d0;
        const double l21 = (H[5] - l20 * l10 * d0) / d1;
        const double d2 = H[8] + mu - l20 * l20 * d0 - l21 * l21 * d1;
        const bool positive = d0 > 0 && d1 > 0 && d2 > 0;
        bool good = false;
        if (positive) {
          const double y0 = b[0], y1 = b[1] - l10 * y0, y2 = b[2] - l20 * y0 - l21 * y1;
          double dp[3];
          dp[2] = y2 / d2;
          dp[1] = y1 / d1 - l21 * dp[2];
          dp[0] = y0 / d0 - l10 * dp[1] - l20 * dp[2];
          const double old[3] = {X[0], X[1], X[2]};
          X[0] += dp[0]; X[1] += dp[1]; X[2] += dp[2];
          const double newChi2 = so_point_chi2(p, tr);
          if (chi2 - newChi2 > 0 && std::isfinite(newChi2)) {
            good = true;
            chi2 = newChi2;
          } else {
            X[0] = old[0]; X[1] = old[1]; X[2] = old[2];
          }
        }
        if (good) {
          mu *= 1. / 3.;
          nu = 2.;
          break;
        }
        mu *= nu;
        nu *= 2.;
        if (++trial >= num_max_trials) stop = true;
      } while (!stop);
      if (stop) break;
    }
  }
  return G2OC_RESULT_OK;
}

int gn_solve(orc_problem* p, int iteration, g2oc_iteration_stats* st) {
  // OptimizationAlgorithmGaussNewton::solve (optimization_algorithm_gauss_newton.cpp:48-93)
  (void)iteration;
  double t = now_s();
  compute_active_errors(p);
  if (st) st->time_residuals = now_s() - t;
  t = now_s();
  build_system(p);
  if (st) st->time_quadratic_form = now_s() - t;
  double ts = 0, tl = 0;
  bool ok = block_solver_solve(p, &ts, &tl);
  if (st) {
    st->time_schur_complement = ts;
    st->time_linear_solver = tl;
    st->iterations_linear_solver = p->pcg_iters_last;
  }
  t = now_s();
  update(p, p->x.data());
  if (st) st->time_update = now_s() - t;
  return ok ? G2OC_RESULT_OK : G2OC_RESULT_FAIL;
}

}  // namespace

// ================================================================ C entry

extern "C" {

void orc_huber(double e2, double delta, double* rho3) { huber(e2, delta, rho3); }

void orc_compute_dq_dR(const double* R, double* out) { compute_dq_dR(R, out); }

void orc_rot_to_quat(const double* R, double* q) {
  Quat r = rot_to_quat(R);
  q[0] = r.x; q[1] = r.y; q[2] = r.z; q[3] = r.w;
}

void orc_se3quat_exp(const double* u, double* out7) { se3q_store(se3q_exp(u), out7); }

double orc_normalize_theta(double t) { return normalize_theta(t); }

int orc_set_threads(int n) {
  g_threads = n < 1 ? 1 : n;
  return G2OC_OK;
}

int orc_create(const g2oc_graph* g, orc_problem** out) {
  if (!g || !out) return G2OC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const bool bal = g->edge_type == G2OC_EDGE_BAL_OBSERVATION;
  const bool ba = g->edge_type == G2OC_EDGE_PROJECT_XYZ2UV || g->edge_type == G2OC_EDGE_SE3_PROJECT_XYZ ||
                  g->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ || bal;
  if (g->pose_type < 1 || g->pose_type > 4 || g->edge_type < 1 || g->edge_type > 7) return G2OC_ERR_BAD_GRAPH;
  if ((g->edge_type == G2OC_EDGE_SE2) != (g->pose_type == G2OC_POSE_SE2)) return G2OC_ERR_BAD_GRAPH;
  if ((g->edge_type == G2OC_EDGE_SE3) != (g->pose_type == G2OC_POSE_SE3)) return G2OC_ERR_BAD_GRAPH;
  if (bal != (g->pose_type == G2OC_POSE_BAL_CAMERA)) return G2OC_ERR_BAD_GRAPH;
  if (((ba && !bal) || g->edge_type == G2OC_EDGE_SE3_EXPMAP) != (g->pose_type == G2OC_POSE_SE3EXPMAP))
    return G2OC_ERR_BAD_GRAPH;
  if (g->num_poses < 0 || g->num_points < 0 || g->num_edges <= 0) return G2OC_ERR_BAD_GRAPH;
  if (!g->pose_estimate || !g->edge_vertex || !g->measurement || !g->information) return G2OC_ERR_INVALID_ARGUMENT;
  if (ba && g->num_points > 0 && !g->point_estimate) return G2OC_ERR_INVALID_ARGUMENT;
  orc_problem* p = new orc_problem();
  p->pose_type = g->pose_type;
  p->edge_type = g->edge_type;
  p->C = g->num_poses;
  p->P = ba ? g->num_points : 0;
  p->E = g->num_edges;
  p->pd = pose_dim(p->pose_type);
  p->ped = pose_est_dim(p->pose_type);
  p->D = edge_dim(p->edge_type);
  p->md = meas_dim(p->edge_type);
  p->pose.assign(g->pose_estimate, g->pose_estimate + (size_t)p->C * p->ped);
  if (p->P) p->point.assign(g->point_estimate, g->point_estimate + (size_t)p->P * 3);
  p->pose_fixed.assign(p->C, 0);
  if (g->pose_fixed) std::memcpy(p->pose_fixed.data(), g->pose_fixed, p->C);
  p->point_fixed.assign(p->P, 0);
  if (g->point_fixed && p->P) std::memcpy(p->point_fixed.data(), g->point_fixed, p->P);
  p->ev.assign(g->edge_vertex, g->edge_vertex + 2 * (size_t)p->E);
  for (int e = 0; e < p->E; ++e) {
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    const int n0 = ba ? p->P : p->C;
    if (v0 < 0 || v0 >= n0 || v1 < 0 || v1 >= p->C || (!ba && v0 == v1)) {
      delete p;
      return G2OC_ERR_BAD_GRAPH;
    }
  }
  if (g->num_pose_edges > 0) {
    // the pose edge set: EdgeSE3Expmap between the cameras of an SE3 projection graph
    if (!ba || bal || p->pose_type != G2OC_POSE_SE3EXPMAP || !g->pose_edge_vertex || !g->pose_edge_measurement ||
        !g->pose_edge_information) {
      delete p;
      return G2OC_ERR_BAD_GRAPH;
    }
    p->PE = g->num_pose_edges;
    p->pev.assign(g->pose_edge_vertex, g->pose_edge_vertex + 2 * (size_t)p->PE);
    for (int e = 0; e < p->PE; ++e) {
      const int v0 = p->pev[2 * e], v1 = p->pev[2 * e + 1];
      if (v0 < 0 || v0 >= p->C || v1 < 0 || v1 >= p->C || v0 == v1) {
        delete p;
        return G2OC_ERR_BAD_GRAPH;
      }
    }
    p->pmeas.assign(g->pose_edge_measurement, g->pose_edge_measurement + (size_t)p->PE * 7);
    p->pinfo.assign(g->pose_edge_information, g->pose_edge_information + (size_t)p->PE * 36);
    if (g->pose_edge_robust_delta) p->pdelta.assign(g->pose_edge_robust_delta, g->pose_edge_robust_delta + p->PE);
  }
  p->meas.assign(g->measurement, g->measurement + (size_t)p->E * p->md);
  p->info.assign(g->information, g->information + (size_t)p->E * p->D * p->D);
  if (g->robust_delta) p->delta.assign(g->robust_delta, g->robust_delta + p->E);
  p->ba = ba;
  p->fx = g->focal_length;
  p->fy = (g->edge_type == G2OC_EDGE_SE3_PROJECT_XYZ || g->edge_type == G2OC_EDGE_STEREO_SE3_PROJECT_XYZ)
              ? g->focal_length_y
              : g->focal_length;
  p->bf = g->stereo_bf;
  p->cx = g->principal_point[0];
  p->cy = g->principal_point[1];
  p->oplus_count.assign(p->C, 0);
  orc_default_params(&p->prm);
  int st = build_structure(p);
  if (st != G2OC_OK) {
    delete p;
    return st;
  }
  *out = p;
  return G2OC_OK;
}

void orc_destroy(orc_problem* p) { delete p; }

int orc_set_params(orc_problem* p, const g2oc_params* prm) {
  if (!p || !prm) return G2OC_ERR_INVALID_ARGUMENT;
  p->prm = *prm;
  return G2OC_OK;
}

int orc_get_hessian_info(orc_problem* p, g2oc_hessian_info* info) {
  if (!p || !info) return G2OC_ERR_INVALID_ARGUMENT;
  info->num_free_poses = p->Cf;
  info->num_free_points = p->Pf;
  info->pose_dim = p->pd;
  info->point_dim = p->P ? 3 : 0;
  info->hpp_nnzb = (int)p->hpp_rc.size();
  info->hpl_nnzb = (int)p->hpl_rc.size();
  info->schur_nnzb = (int)p->schur_rc.size();
  info->num_active_edges = (int)p->act.size();
  info->vector_size = (int64_t)p->b.size();
  // co-observing Hpl block pairs (a < b) of the off-diagonal Schur blocks
  int64_t np = 0;
  for (int l = 0; l < p->Pf; ++l) {
    const int64_t m = p->hpl_col_ptr[l + 1] - p->hpl_col_ptr[l];
    np += m * (m - 1) / 2;
  }
  info->schur_pairs = np;
  info->num_active_pose_edges = (int)p->pact.size();
  return G2OC_OK;
}

int orc_set_estimates(orc_problem* p, const double* pose, const double* point) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (pose) std::memcpy(p->pose.data(), pose, p->pose.size() * sizeof(double));
  if (point && p->P) std::memcpy(p->point.data(), point, p->point.size() * sizeof(double));
  return G2OC_OK;
}

int orc_download(orc_problem* p, double* pose, double* point) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (pose) std::memcpy(pose, p->pose.data(), p->pose.size() * sizeof(double));
  if (point && p->P) std::memcpy(point, p->point.data(), p->point.size() * sizeof(double));
  return G2OC_OK;
}

int orc_chi2(orc_problem* p, double* chi2, double* robust) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  compute_active_errors(p);
  active_chi2(p, chi2, robust);
  return G2OC_OK;
}

int orc_errors(orc_problem* p, double* out) {
  if (!p || !out) return G2OC_ERR_INVALID_ARGUMENT;
  compute_active_errors(p);
  std::memcpy(out, p->err.data(), p->err.size() * sizeof(double));
  if (!p->perr.empty()) std::memcpy(out + p->err.size(), p->perr.data(), p->perr.size() * sizeof(double));
  return G2OC_OK;
}

int orc_jacobians(orc_problem* p, double* j0, double* j1) {
  if (!p || !j0 || !j1) return G2OC_ERR_INVALID_ARGUMENT;
  const bool ba = p->ba;
  const int d0 = ba ? 3 : p->pd, d1 = p->pd, D = p->D;
  for (size_t k = 0; k < p->act.size(); ++k)
    compute_edge_jac(p, p->act[k], j0 + k * D * d0, j1 + k * D * d1);
  return G2OC_OK;
}

int orc_numeric_jacobians(orc_problem* p, double* j0, double* j1) {
  if (!p || !j0 || !j1) return G2OC_ERR_INVALID_ARGUMENT;
  const bool ba = p->ba;
  const int d0 = ba ? 3 : p->pd, d1 = p->pd, D = p->D;
  const double delta = 1e-9, scalar = 1 / (2 * delta);
  for (size_t k = 0; k < p->act.size(); ++k) {
    const int e = p->act[k];
    const int v0 = p->ev[2 * e], v1 = p->ev[2 * e + 1];
    for (int which = 0; which < 2; ++which) {
      const int dim = which == 0 ? d0 : d1;
      double* J = which == 0 ? j0 + k * D * d0 : j1 + k * D * d1;
      double* est;
      size_t n;
      if (which == 0 && ba) { est = point_ptr(p, v0); n = 3; }
      else { est = pose_ptr(p, which == 0 ? v0 : v1); n = p->ped; }
      const int pi = which == 0 ? v0 : v1;
      std::vector<double> bak(est, est + n);
      for (int d = 0; d < dim; ++d) {
        double u[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        double ep[6], em[6];
        const int cnt = (!ba || which == 1) ? p->oplus_count[pi] : 0;
        u[d] = delta;
        if (which == 0 && ba) { est[0] += u[0]; est[1] += u[1]; est[2] += u[2]; }
        else vertex_oplus_pose(p, pi, u);
        compute_edge_error(p, e, ep);
        std::memcpy(est, bak.data(), n * sizeof(double));
        u[d] = -delta;
        if (which == 0 && ba) { est[0] += u[0]; est[1] += u[1]; est[2] += u[2]; }
        else vertex_oplus_pose(p, pi, u);
        compute_edge_error(p, e, em);
        std::memcpy(est, bak.data(), n * sizeof(double));
        if (!ba || which == 1) p->oplus_count[pi] = cnt;
        for (int r = 0; r < D; ++r) J[r * dim + d] = scalar * (ep[r] - em[r]);
      }
    }
  }
  return G2OC_OK;
}

int orc_build_system(orc_problem* p) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  compute_active_errors(p);
  build_system(p);
  return G2OC_OK;
}

int orc_get_pattern(orc_problem* p, int32_t* hpp_rc, int32_t* hpl_rc, int32_t* schur_rc) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (hpp_rc)
    for (size_t i = 0; i < p->hpp_rc.size(); ++i) { hpp_rc[2 * i] = p->hpp_rc[i].first; hpp_rc[2 * i + 1] = p->hpp_rc[i].second; }
  if (hpl_rc)
    for (size_t i = 0; i < p->hpl_rc.size(); ++i) { hpl_rc[2 * i] = p->hpl_rc[i].first; hpl_rc[2 * i + 1] = p->hpl_rc[i].second; }
  if (schur_rc)
    for (size_t i = 0; i < p->schur_rc.size(); ++i) { schur_rc[2 * i] = p->schur_rc[i].first; schur_rc[2 * i + 1] = p->schur_rc[i].second; }
  return G2OC_OK;
}

int orc_get_hessian(orc_problem* p, double* hpp, double* hll, double* hpl, double* b) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (!p->system_built) return G2OC_ERR_STATE;
  if (hpp) std::memcpy(hpp, p->hpp.data(), p->hpp.size() * sizeof(double));
  if (hll) std::memcpy(hll, p->hll.data(), p->hll.size() * sizeof(double));
  if (hpl) std::memcpy(hpl, p->hpl.data(), p->hpl.size() * sizeof(double));
  if (b) std::memcpy(b, p->b.data(), p->b.size() * sizeof(double));
  return G2OC_OK;
}

int orc_schur(orc_problem* p, double lambda, double* S, double* bs) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (!p->system_built) return G2OC_ERR_STATE;
  if (!p->schur) return G2OC_ERR_NOT_SUPPORTED;
  set_lambda(p, lambda);
  schur_complement(p);
  restore_diagonal(p);
  if (S) std::memcpy(S, p->S.data(), p->S.size() * sizeof(double));
  if (bs) std::memcpy(bs, p->bschur.data(), p->bschur.size() * sizeof(double));
  return G2OC_OK;
}

int orc_update(orc_problem* p, const double* x) {
  // SparseOptimizer::update (sparse_optimizer.cpp:457-468) with a caller step
  // in Hessian order: the host side of an algorithm that drives a Solver
  if (!p || !x) return G2OC_ERR_INVALID_ARGUMENT;
  update(p, x);
  return G2OC_OK;
}

int orc_solve(orc_problem* p, double lambda, double* x, int32_t* iters) {
  if (!p) return G2OC_ERR_INVALID_ARGUMENT;
  if (!p->system_built) return G2OC_ERR_STATE;
  set_lambda(p, lambda);
  bool ok = block_solver_solve(p, nullptr, nullptr);
  restore_diagonal(p);
  if (iters) *iters = p->pcg_iters_last;
  if (x) std::memcpy(x, p->x.data(), p->x.size() * sizeof(double));
  return ok ? G2OC_OK : G2OC_ERR_NOT_PD;
}

int orc_optimize(orc_problem* p, int iterations, g2oc_iteration_stats* stats, int* done) {
  // SparseOptimizer::optimize (sparse_optimizer.cpp:393-455)
  if (!p || iterations < 0) return G2OC_ERR_INVALID_ARGUMENT;
  p->pcg.residual = -1.0;  // LinearSolverPCG::init via BlockSolver::init
  int result = G2OC_RESULT_OK;
  int it = 0;
  for (int i = 0; i < iterations && result == G2OC_RESULT_OK; ++i) {
    g2oc_iteration_stats local;
    std::memset(&local, 0, sizeof(local));
    double t = now_s();
    if (p->prm.algorithm == G2OC_ALGO_LEVENBERG) result = lm_solve(p, i, &local);
    else if (p->prm.algorithm == G2OC_ALGO_DOGLEG) result = dl_solve(p, i, &local);
    else if (p->prm.algorithm == G2OC_ALGO_STRUCTURE_ONLY) result = so_calc(p, 1, p->prm.max_trials_after_failure);
    else result = gn_solve(p, i, &local);
    local.iteration = i;
    local.result = result;
    local.lambda = p->lambda;
    if (p->prm.algorithm == G2OC_ALGO_DOGLEG) {
      local.lambda = p->dl_was_pd ? 0.0 : p->dl_lambda;
      local.trust_radius = p->dl_delta;
      local.dogleg_step = p->dl_step;
    }
    compute_active_errors(p);
    active_chi2(p, nullptr, &local.chi2);
    local.time_iteration = now_s() - t;
    if (stats) stats[i] = local;
    ++it;
  }
  if (done) *done = (result == G2OC_RESULT_FAIL) ? 0 : it;
  return G2OC_OK;
}

int orc_solve_block_system(int32_t linear_solver, const g2oc_params* params, int32_t nb,
                           const int32_t* block_offsets, int32_t nnzb, const int32_t* block_rc,
                           const double* values, const double* b, double* x, int32_t* iterations) {
  if (nb <= 0 || !block_offsets || nnzb <= 0 || !block_rc || !values || !b || !x) return G2OC_ERR_INVALID_ARGUMENT;
  BlockSym A;
  A.nb = nb;
  A.off.assign(block_offsets, block_offsets + nb + 1);
  A.col_ptr.assign(nb + 1, 0);
  A.row.resize(nnzb);
  A.val_off.resize(nnzb);
  size_t off = 0;
  for (int k = 0; k < nnzb; ++k) {
    const int r = block_rc[2 * k], c = block_rc[2 * k + 1];
    if (r < 0 || c < 0 || r >= nb || c >= nb || r > c) return G2OC_ERR_INVALID_ARGUMENT;
    if (k > 0) {
      const int pr = block_rc[2 * k - 2], pc = block_rc[2 * k - 1];
      if (pc > c || (pc == c && pr >= r)) return G2OC_ERR_INVALID_ARGUMENT;
    }
    A.col_ptr[c + 1]++;
    A.row[k] = r;
    A.val_off[k] = off;
    off += (size_t)A.dim(r) * A.dim(c);
  }
  for (int i = 0; i < nb; ++i) A.col_ptr[i + 1] += A.col_ptr[i];
  for (int c = 0; c < nb; ++c)
    if (A.col_ptr[c + 1] == A.col_ptr[c] || A.row[A.col_ptr[c + 1] - 1] != c) return G2OC_ERR_INVALID_ARGUMENT;
  A.val = values;
  g2oc_params prm;
  if (params) prm = *params;
  else orc_default_params(&prm);
  if (linear_solver == G2OC_LINEAR_CHOLESKY) {
    if (iterations) *iterations = 0;
    return cholesky_solve(A, b, x) ? G2OC_OK : G2OC_ERR_NOT_PD;
  }
  PCGState st;
  int it = 0;
  pcg_solve(A, b, x, prm, st, &it);
  if (iterations) *iterations = it;
  return G2OC_OK;
}

// The oracle carries its own copy of the parameter defaults so it does not
// link the product library.
void orc_default_params(g2oc_params* p) {
  p->algorithm = G2OC_ALGO_LEVENBERG;
  p->linear_solver = G2OC_LINEAR_PCG;
  p->precision = G2OC_PREC_FP64;
  p->pcg_max_iterations = -1;
  p->pcg_tolerance = 1e-6;
  p->pcg_absolute_tolerance = 1;
  p->max_trials_after_failure = 10;
  p->initial_lambda = 0.0;
  p->tau = 1e-5;
  p->refine_max_iterations = 2;
  p->refine_tolerance = 1e-10;
  p->initial_delta = 1e4;  // OptimizationAlgorithmDogleg "initialDelta"
  p->lambda_factor = 10.;  // "lambdaFactor"
}

}  // extern "C"
