// g2o_math.cuh -- device/host math for the hot-path types, templated on the
// arithmetic type T (double for the FP64 path, float for the FP32 Jacobian /
// Hessian part of the mixed path). Every function cites the g2o source it
// restates (paths relative to the g2o tree). Matrices are dense row-major.
#pragma once

#include <cmath>
#include <cuda_runtime.h>

#define G2OC_HD __host__ __device__ __forceinline__

namespace g2oc {

template <typename T>
struct Q4 {
  T x, y, z, w;
};

template <typename T>
G2OC_HD T normalize_theta(T theta) {
  // g2o/stuff/misc.h:66-70
  const T pi = T(3.14159265358979323846);
  const T r = fmod(theta + pi, T(2) * pi);
  if (r <= T(0)) return r + pi;
  return r - pi;
}

template <typename T>
G2OC_HD void quat_to_rot(const Q4<T>& q, T R[9]) {
  // unit quaternion -> rotation matrix (Eigen QuaternionBase::toRotationMatrix)
  const T tx = 2 * q.x, ty = 2 * q.y, tz = 2 * q.z;
  const T twx = tx * q.w, twy = ty * q.w, twz = tz * q.w;
  const T txx = tx * q.x, txy = ty * q.x, txz = tz * q.x;
  const T tyy = ty * q.y, tyz = tz * q.y, tzz = tz * q.z;
  R[0] = T(1) - (tyy + tzz); R[1] = txy - twz;          R[2] = txz + twy;
  R[3] = txy + twz;          R[4] = T(1) - (txx + tzz); R[5] = tyz - twx;
  R[6] = txz - twy;          R[7] = tyz + twx;          R[8] = T(1) - (txx + tyy);
}

template <typename T>
G2OC_HD Q4<T> rot_to_quat(const T R[9]) {
  // Shepperd's method, largest-diagonal branch (Eigen quaternion_assign_impl)
  Q4<T> q;
  T t = R[0] + R[4] + R[8];
  if (t > T(0)) {
    t = sqrt(t + T(1));
    q.w = T(0.5) * t;
    t = T(0.5) / t;
    q.x = (R[7] - R[5]) * t;
    q.y = (R[2] - R[6]) * t;
    q.z = (R[3] - R[1]) * t;
  } else {
    int i = 0;
    if (R[4] > R[0]) i = 1;
    if (R[8] > R[i * 4]) i = 2;
    const int j = (i + 1) % 3, k = (j + 1) % 3;
    T c[3];
    t = sqrt(R[i * 4] - R[j * 4] - R[k * 4] + T(1));
    c[i] = T(0.5) * t;
    t = T(0.5) / t;
    q.w = (R[k * 3 + j] - R[j * 3 + k]) * t;
    c[j] = (R[j * 3 + i] + R[i * 3 + j]) * t;
    c[k] = (R[k * 3 + i] + R[i * 3 + k]) * t;
    q.x = c[0]; q.y = c[1]; q.z = c[2];
  }
  return q;
}

template <typename T>
G2OC_HD Q4<T> quat_mul(const Q4<T>& a, const Q4<T>& b) {
  Q4<T> r;
  r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  r.y = a.w * b.y + a.y * b.w + a.z * b.x - a.x * b.z;
  r.z = a.w * b.z + a.z * b.w + a.x * b.y - a.y * b.x;
  return r;
}

template <typename T>
G2OC_HD void quat_rotate(const Q4<T>& q, const T v[3], T o[3]) {
  // v + 2w (u x v) + 2 u x (u x v)
  T uv0 = q.y * v[2] - q.z * v[1], uv1 = q.z * v[0] - q.x * v[2], uv2 = q.x * v[1] - q.y * v[0];
  uv0 += uv0; uv1 += uv1; uv2 += uv2;
  o[0] = v[0] + q.w * uv0 + (q.y * uv2 - q.z * uv1);
  o[1] = v[1] + q.w * uv1 + (q.z * uv0 - q.x * uv2);
  o[2] = v[2] + q.w * uv2 + (q.x * uv1 - q.y * uv0);
}

template <typename T>
G2OC_HD void quat_normalize_positive_w(Q4<T>& q) {
  // SE3Quat::normalizeRotation (g2o/types/slam3d/se3quat.h:251-256)
  if (q.w < T(0)) { q.x = -q.x; q.y = -q.y; q.z = -q.z; q.w = -q.w; }
  const T n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x /= n; q.y /= n; q.z /= n; q.w /= n;
}

template <typename T>
G2OC_HD void matmul3(const T* A, const T* B, T* C) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) C[i * 3 + j] = A[i * 3] * B[j] + A[i * 3 + 1] * B[3 + j] + A[i * 3 + 2] * B[6 + j];
}

template <typename T>
G2OC_HD void matvec3(const T* A, const T* v, T* o) {
#pragma unroll
  for (int i = 0; i < 3; ++i) o[i] = A[i * 3] * v[0] + A[i * 3 + 1] * v[1] + A[i * 3 + 2] * v[2];
}

// SE3Quat as (q, t)
template <typename T>
struct SE3Q {
  Q4<T> q;
  T t[3];
};

template <typename T>
G2OC_HD SE3Q<T> se3q_exp(const T u[6]) {
  // SE3Quat::exp (g2o/types/slam3d/se3quat.h:202-230), u = (omega, upsilon)
  const T w0 = u[0], w1 = u[1], w2 = u[2];
  const T theta = sqrt(w0 * w0 + w1 * w1 + w2 * w2);
  const T O[9] = {T(0), -w2, w1, w2, T(0), -w0, -w1, w0, T(0)};
  T O2[9];
  matmul3(O, O, O2);
  T R[9], V[9];
  if (theta < T(0.00001)) {
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      R[i] = O[i] + T(0.5) * O2[i];
      V[i] = T(0.5) * O[i] + (T(1) / T(6)) * O2[i];
    }
  } else {
    const T s = sin(theta), c = cos(theta);
    const T A = s / theta, B = (T(1) - c) / (theta * theta), C = (theta - s) / (theta * theta * theta);
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      R[i] = A * O[i] + B * O2[i];
      V[i] = B * O[i] + C * O2[i];
    }
  }
  R[0] += T(1); R[4] += T(1); R[8] += T(1);
  V[0] += T(1); V[4] += T(1); V[8] += T(1);
  SE3Q<T> r;
  r.q = rot_to_quat(R);
  matvec3(V, u + 3, r.t);
  quat_normalize_positive_w(r.q);
  return r;
}

template <typename T>
G2OC_HD SE3Q<T> se3q_mul(const SE3Q<T>& a, const SE3Q<T>& b) {
  // SE3Quat::operator* (se3quat.h:97-103)
  SE3Q<T> r;
  T rt[3];
  quat_rotate(a.q, b.t, rt);
  r.t[0] = a.t[0] + rt[0]; r.t[1] = a.t[1] + rt[1]; r.t[2] = a.t[2] + rt[2];
  r.q = quat_mul(a.q, b.q);
  quat_normalize_positive_w(r.q);
  return r;
}

// SE3Quat in the C-ABI's 7-vector (t, q: SE3Quat::toVector) and back
template <typename T>
G2OC_HD SE3Q<T> se3q_from7(const T* v) {
  SE3Q<T> s;
  s.t[0] = v[0]; s.t[1] = v[1]; s.t[2] = v[2];
  s.q = Q4<T>{v[3], v[4], v[5], v[6]};
  return s;
}
template <typename T>
G2OC_HD void se3q_to7(const SE3Q<T>& s, T* v) {
  v[0] = s.t[0]; v[1] = s.t[1]; v[2] = s.t[2];
  v[3] = s.q.x; v[4] = s.q.y; v[5] = s.q.z; v[6] = s.q.w;
}

template <typename T>
G2OC_HD SE3Q<T> se3q_inverse(const SE3Q<T>& a) {
  // SE3Quat::inverse (se3quat.h:114-119): conjugate, t' = q' (-t); no renormalization
  SE3Q<T> r;
  r.q = Q4<T>{-a.q.x, -a.q.y, -a.q.z, a.q.w};
  const T mt[3] = {a.t[0] * T(-1), a.t[1] * T(-1), a.t[2] * T(-1)};
  quat_rotate(r.q, mt, r.t);
  return r;
}

template <typename T>
G2OC_HD void se3q_log(const SE3Q<T>& a, T out[6]) {
  // SE3Quat::log (se3quat.h:165-199) with deltaR and skew (se3_ops.hpp:27-45)
  T R[9];
  quat_to_rot(a.q, R);
  const T d = T(0.5) * (R[0] + R[4] + R[8] - T(1));
  const T dR[3] = {R[7] - R[5], R[2] - R[6], R[3] - R[1]};
  T w[3], k1, k2;
  if (fabs(d) > T(0.99999)) {
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = T(0.5) * dR[i];
    k2 = T(1) / T(12);
  } else {
    const T theta = acos(d);
    const T f = theta / (T(2) * sqrt(T(1) - d * d));
#pragma unroll
    for (int i = 0; i < 3; ++i) w[i] = f * dR[i];
    k2 = (T(1) - theta / (T(2) * tan(theta / T(2)))) / (theta * theta);
  }
  k1 = T(-0.5);
  const T O[9] = {T(0), -w[2], w[1], w[2], T(0), -w[0], -w[1], w[0], T(0)};
  T O2[9], Vi[9];
  matmul3(O, O, O2);
#pragma unroll
  for (int i = 0; i < 9; ++i) Vi[i] = k1 * O[i] + k2 * O2[i];
  Vi[0] += T(1); Vi[4] += T(1); Vi[8] += T(1);
  out[0] = w[0]; out[1] = w[1]; out[2] = w[2];
  matvec3(Vi, a.t, out + 3);
}

template <typename T>
G2OC_HD void se3q_adj(const SE3Q<T>& a, T sign, T A[36]) {
  // sign * SE3Quat::adj (se3quat.h:232-240): [[R, 0], [skew(t) R, R]], row-major
  T R[9], S[9], SR[9];
  quat_to_rot(a.q, R);
  const T* t = a.t;
  S[0] = T(0); S[1] = -t[2]; S[2] = t[1];
  S[3] = t[2]; S[4] = T(0); S[5] = -t[0];
  S[6] = -t[1]; S[7] = t[0]; S[8] = T(0);
  matmul3(S, R, SR);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      A[r * 6 + c] = sign * R[r * 3 + c];
      A[r * 6 + 3 + c] = T(0) * sign;
      A[(3 + r) * 6 + c] = sign * SR[r * 3 + c];
      A[(3 + r) * 6 + 3 + c] = sign * R[r * 3 + c];
    }
}

// EdgeSE3Expmap (g2o/types/sba/edge_se3_expmap.cpp:45-72) on 7-vector
// estimates, C the measurement: e = log(Tj^-1 C Ti);
// J_i = adj(Tj^-1 C), J_j = -adj(Ti^-1 C^-1)
template <typename T>
G2OC_HD void se3exp_error(const T* xi, const T* xj, const T* c7, T e[6]) {
  const SE3Q<T> Ti = se3q_from7(xi), Tj = se3q_from7(xj), C = se3q_from7(c7);
  se3q_log(se3q_mul(se3q_mul(se3q_inverse(Tj), C), Ti), e);
}
template <typename T>
G2OC_HD void se3exp_jacobians(const T* xi, const T* xj, const T* c7, T Ji[36], T Jj[36]) {
  const SE3Q<T> Ti = se3q_from7(xi), Tj = se3q_from7(xj), C = se3q_from7(c7);
  se3q_adj(se3q_mul(se3q_inverse(Tj), C), T(1), Ji);
  se3q_adj(se3q_mul(se3q_inverse(Ti), se3q_inverse(C)), T(-1), Jj);
}

template <typename T>
G2OC_HD void huber(T e, T delta, T rho[3]) {
  // RobustKernelHuber::robustify (g2o/core/robust_kernel_impl.cpp:60-74)
  const T dsqr = delta * delta;
  if (e <= dsqr) {
    rho[0] = e; rho[1] = T(1); rho[2] = T(0);
  } else {
    const T sqrte = sqrt(e);
    rho[0] = T(2) * sqrte * delta - dsqr;
    rho[1] = delta / sqrte;
    rho[2] = T(-0.5) * rho[1] / e;
  }
}

// ----------------------------------------------------------------- BA edge
// EdgeProjectXYZ2UV (g2o/types/sba/edge_project_xyz2uv.cpp:50-97); vertex0 =
// VertexPointXYZ, vertex1 = VertexSE3Expmap; cam_map
// (g2o/types/sba/parameter_cameraparameters.cpp:59-65). Camera stored as
// (qx, qy, qz, qw, tx, ty, tz).

template <typename T>
G2OC_HD void ba_transform(const T* cam, const T* X, T Xc[3]) {
  Q4<T> q{cam[0], cam[1], cam[2], cam[3]};
  quat_rotate(q, X, Xc);
  Xc[0] += cam[4]; Xc[1] += cam[5]; Xc[2] += cam[6];
}

template <typename T>
G2OC_HD void ba_error(const T* cam, const T* X, const T* z, T f, T cx, T cy, T e[2]) {
  T Xc[3];
  ba_transform(cam, X, Xc);
  e[0] = z[0] - (Xc[0] / Xc[2] * f + cx);
  e[1] = z[1] - (Xc[1] / Xc[2] * f + cy);
}

// Jp (2x3) and Jc (2x6, columns omega then upsilon)
template <typename T>
G2OC_HD void ba_jacobians_from_xc(const T* cam, const T Xc[3], T fx, T fy, T Jp[6], T Jc[12]) {
  // fx = fy = CameraParameters::focal_length for EdgeProjectXYZ2UV; the
  // members fx, fy of EdgeSE3ProjectXYZ (g2o/types/sba/edge_project_xyz.cpp:59-93)
  const T x = Xc[0], y = Xc[1], z = Xc[2], z2 = z * z;
  T R[9];
  quat_to_rot(Q4<T>{cam[0], cam[1], cam[2], cam[3]}, R);
  const T a02 = -x / z * fx, a12 = -y / z * fy;
  const T iz = T(-1) / z;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Jp[c] = iz * (fx * R[c] + a02 * R[6 + c]);
    Jp[3 + c] = iz * (fy * R[3 + c] + a12 * R[6 + c]);
  }
  Jc[0] = x * y / z2 * fx;
  Jc[1] = -(T(1) + (x * x / z2)) * fx;
  Jc[2] = y / z * fx;
  Jc[3] = T(-1) / z * fx;
  Jc[4] = T(0);
  Jc[5] = x / z2 * fx;
  Jc[6] = (T(1) + y * y / z2) * fy;
  Jc[7] = -x * y / z2 * fy;
  Jc[8] = -x / z * fy;
  Jc[9] = T(0);
  Jc[10] = T(-1) / z * fy;
  Jc[11] = y / z2 * fy;
}

// --------------------------------------------------------------- SE2 edge
// EdgeSE2 (g2o/types/slam2d/edge_se2.h:46-59, edge_se2.cpp:63-83), SE2 ops
// (g2o/types/slam2d/se2.h:72-90)
template <typename T>
G2OC_HD void se2_inv(const T* a, T* r) {
  r[2] = normalize_theta(-a[2]);
  const T c = cos(r[2]), s = sin(r[2]);
  r[0] = c * (-a[0]) - s * (-a[1]);
  r[1] = s * (-a[0]) + c * (-a[1]);
}

template <typename T>
G2OC_HD void se2_mul(const T* a, const T* b, T* r) {
  const T c = cos(a[2]), s = sin(a[2]);
  r[0] = a[0] + c * b[0] - s * b[1];
  r[1] = a[1] + s * b[0] + c * b[1];
  r[2] = normalize_theta(a[2] + b[2]);
}

template <typename T>
G2OC_HD void se2_error(const T* xi, const T* xj, const T* zinv, T e[3]) {
  T ii[3], d[3];
  se2_inv(xi, ii);
  se2_mul(ii, xj, d);
  se2_mul(zinv, d, e);
}

template <typename T>
G2OC_HD void se2_jacobians(const T* xi, const T* xj, const T* zinv, T Ji[9], T Jj[9]) {
  const T thetai = xi[2];
  const T dx = xj[0] - xi[0], dy = xj[1] - xi[1];
  const T si = sin(thetai), ci = cos(thetai);
  const T A[9] = {-ci, -si, -si * dx + ci * dy, si, -ci, -ci * dx - si * dy, T(0), T(0), T(-1)};
  const T B[9] = {ci, si, T(0), -si, ci, T(0), T(0), T(0), T(1)};
  const T c = cos(zinv[2]), s = sin(zinv[2]);
  const T Z[9] = {c, -s, T(0), s, c, T(0), T(0), T(0), T(1)};
  matmul3(Z, A, Ji);
  matmul3(Z, B, Jj);
}

// --------------------------------------------------------------- SE3 edge
// Isometry3 stored as R (row-major 9) then t (3).
template <typename T>
G2OC_HD void iso_mul(const T* a, const T* b, T* r) {
  matmul3(a, b, r);
  matvec3(a, b + 9, r + 9);
  r[9] += a[9]; r[10] += a[10]; r[11] += a[11];
}

template <typename T>
G2OC_HD void iso_inv(const T* a, T* r) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r[i * 3 + j] = a[j * 3 + i];
  T tt[3];
  matvec3(r, a + 9, tt);
  r[9] = -tt[0]; r[10] = -tt[1]; r[11] = -tt[2];
}

template <typename T>
G2OC_HD void to_compact_quat(const T* R, T out[3]) {
  // toCompactQuaternion (g2o/types/slam3d/isometry3d_mappings.cpp:80-85, normalize :40-46)
  Q4<T> q = rot_to_quat(R);
  const T n = sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
  q.x /= n; q.y /= n; q.z /= n; q.w /= n;
  if (q.w < T(0)) { q.x = -q.x; q.y = -q.y; q.z = -q.z; }
  out[0] = q.x; out[1] = q.y; out[2] = q.z;
}

template <typename T>
G2OC_HD void from_compact_quat(const T* v, T* R) {
  // fromCompactQuaternion (isometry3d_mappings.cpp:87-94)
  const T w = T(1) - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  if (w < T(0)) {
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = (i % 4 == 0) ? T(1) : T(0);
    return;
  }
  quat_to_rot(Q4<T>{v[0], v[1], v[2], sqrt(w)}, R);
}

template <typename T>
G2OC_HD void se3_error(const T* xi, const T* xj, const T* zinv, T e[6]) {
  // EdgeSE3::computeError (g2o/types/slam3d/edge_se3.cpp:60-66)
  T a[12], ii[12], d[12];
  iso_inv(xi, ii);
  iso_mul(zinv, ii, a);
  iso_mul(a, xj, d);
  e[0] = d[9]; e[1] = d[10]; e[2] = d[11];
  to_compact_quat(d, e + 3);
}

// dq/dR of the compact quaternion for the Shepperd branch of R
// (g2o/types/slam3d/dquat2mat.cpp:36-94), derived from the branch closed
// forms; D[q*9 + c*3 + r] = d q / d R(r, c).
template <typename T>
G2OC_HD void compute_dq_dR(const T* R, T D[27]) {
#pragma unroll
  for (int i = 0; i < 27; ++i) D[i] = T(0);
  const T r00 = R[0], r11 = R[4], r22 = R[8];
  const T tr = r00 + r11 + r22;
  if (tr > T(0)) {
    const T qw = T(0.5) * sqrt(tr + T(1));
    const T i4 = T(0.25) / qw, i32 = T(1) / (T(32) * qw * qw * qw);
    const T nx = R[7] - R[5], ny = R[2] - R[6], nz = R[3] - R[1];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      D[0 * 9 + d * 4] = -nx * i32;
      D[1 * 9 + d * 4] = -ny * i32;
      D[2 * 9 + d * 4] = -nz * i32;
    }
    // index c*3 + r
    D[0 * 9 + 1 * 3 + 2] += i4;  D[0 * 9 + 2 * 3 + 1] -= i4;  // qx: +R21 -R12
    D[1 * 9 + 2 * 3 + 0] += i4;  D[1 * 9 + 0 * 3 + 2] -= i4;  // qy: +R02 -R20
    D[2 * 9 + 0 * 3 + 1] += i4;  D[2 * 9 + 1 * 3 + 0] -= i4;  // qz: +R10 -R01
    return;
  }
  int i;
  if ((r00 > r11) && (r00 > r22)) i = 0;
  else if (r11 > r22) i = 1;
  else i = 2;
  const int j = (i + 1) % 3, k = (j + 1) % 3;
  auto at = [&](int r, int c) { return R[r * 3 + c]; };
  auto ix = [](int r, int c) { return c * 3 + r; };
  const T s = T(0.5) * sqrt(T(1) + at(i, i) - at(j, j) - at(k, k));
  const T i4 = T(0.25) / s, i8 = T(0.125) / s, i32 = T(1) / (T(32) * s * s * s);
  const T qw = (at(k, j) - at(j, k)) * i4;
  D[i * 9 + ix(i, i)] += i8; D[i * 9 + ix(j, j)] -= i8; D[i * 9 + ix(k, k)] -= i8;
  const T nj = at(j, i) + at(i, j), nk = at(k, i) + at(i, k);
  D[j * 9 + ix(j, i)] += i4; D[j * 9 + ix(i, j)] += i4;
  D[j * 9 + ix(i, i)] -= nj * i32; D[j * 9 + ix(j, j)] += nj * i32; D[j * 9 + ix(k, k)] += nj * i32;
  D[k * 9 + ix(k, i)] += i4; D[k * 9 + ix(i, k)] += i4;
  D[k * 9 + ix(i, i)] -= nk * i32; D[k * 9 + ix(j, j)] += nk * i32; D[k * 9 + ix(k, k)] += nk * i32;
  if (qw <= T(0)) {
#pragma unroll
    for (int t = 0; t < 27; ++t) D[t] = -D[t];
  }
}

// computeEdgeSE3Gradient (g2o/types/slam3d/isometry3d_gradients.h:205-279)
template <typename T>
G2OC_HD void se3_jacobians(const T* xi, const T* xj, const T* zinv, T Ji[36], T Jj[36]) {
  T ii[12], B[12], E[12];
  iso_inv(xi, ii);
  iso_mul(ii, xj, B);
  iso_mul(zinv, B, E);
  const T* Re = E;
  const T* Ra = zinv;
  const T* Rb = B;
  const T* tb = B + 9;
  T dq[27];
  compute_dq_dR(Re, dq);
#pragma unroll
  for (int i = 0; i < 36; ++i) { Ji[i] = T(0); Jj[i] = T(0); }
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      Ji[r * 6 + c] = -Ra[r * 3 + c];
      Jj[r * 6 + c] = Re[r * 3 + c];
    }
  {
    const T x = 2 * tb[0], y = 2 * tb[1], z = 2 * tb[2];
    const T S[9] = {T(0), -z, y, z, T(0), -x, -y, x, T(0)};
    T RS[9];
    matmul3(Ra, S, RS);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) Ji[r * 6 + 3 + c] = RS[r * 3 + c];
  }
  auto apply = [&](const T* Sx, const T* Sy, const T* Sz, const T* Rl, T* J) {
    const T* S3[3] = {Sx, Sy, Sz};
#pragma unroll
    for (int kk = 0; kk < 3; ++kk) {
      T P[9];
      matmul3(Rl, S3[kk], P);
#pragma unroll
      for (int qi = 0; qi < 3; ++qi) {
        T s = T(0);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) s += dq[qi * 9 + c * 3 + r] * P[r * 3 + c];
        J[(3 + qi) * 6 + 3 + kk] = s;
      }
    }
  };
  {
    T r[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) r[i] = 2 * Rb[i];
    const T Sx[9] = {T(0), T(0), T(0), r[6], r[7], r[8], -r[3], -r[4], -r[5]};
    const T Sy[9] = {-r[6], -r[7], -r[8], T(0), T(0), T(0), r[0], r[1], r[2]};
    const T Sz[9] = {r[3], r[4], r[5], -r[0], -r[1], -r[2], T(0), T(0), T(0)};
    apply(Sx, Sy, Sz, Ra, Ji);
  }
  {
    const T Sx[9] = {T(0), T(0), T(0), T(0), T(0), T(-2), T(0), T(2), T(0)};
    const T Sy[9] = {T(0), T(0), T(2), T(0), T(0), T(0), T(-2), T(0), T(0)};
    const T Sz[9] = {T(0), T(-2), T(0), T(2), T(0), T(0), T(0), T(0), T(0)};
    apply(Sx, Sy, Sz, Re, Jj);
  }
}

// small symmetric 3x3 inverse by cofactors (the reference uses Eigen's 3x3
// inverse for H_ll, g2o/core/block_solver.hpp:371)
template <typename T>
G2OC_HD bool inverse3(const T* A, T* out) {
  const T c00 = A[4] * A[8] - A[5] * A[7];
  const T c01 = A[5] * A[6] - A[3] * A[8];
  const T c02 = A[3] * A[7] - A[4] * A[6];
  const T det = A[0] * c00 + A[1] * c01 + A[2] * c02;
  const T id = T(1) / det;
  out[0] = c00 * id; out[3] = c01 * id; out[6] = c02 * id;
  out[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  out[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  out[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  out[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  out[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  out[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  return isfinite(id);
}

// n x n inverse (n <= 6) by Gauss-Jordan with partial pivoting
template <typename T, int N>
G2OC_HD bool inverse_gj(const T* A, T* out) {
  T M[N * N], I[N * N];
#pragma unroll
  for (int i = 0; i < N * N; ++i) { M[i] = A[i]; I[i] = (i / N == i % N) ? T(1) : T(0); }
  for (int c = 0; c < N; ++c) {
    int p = c;
    for (int r = c + 1; r < N; ++r)
      if (fabs(M[r * N + c]) > fabs(M[p * N + c])) p = r;
    if (M[p * N + c] == T(0)) return false;
    if (p != c)
      for (int k = 0; k < N; ++k) {
        T t = M[p * N + k]; M[p * N + k] = M[c * N + k]; M[c * N + k] = t;
        t = I[p * N + k]; I[p * N + k] = I[c * N + k]; I[c * N + k] = t;
      }
    const T iv = T(1) / M[c * N + c];
    for (int k = 0; k < N; ++k) { M[c * N + k] *= iv; I[c * N + k] *= iv; }
    for (int r = 0; r < N; ++r) {
      if (r == c) continue;
      const T f = M[r * N + c];
      for (int k = 0; k < N; ++k) { M[r * N + k] -= f * M[c * N + k]; I[r * N + k] -= f * I[c * N + k]; }
    }
  }
#pragma unroll
  for (int i = 0; i < N * N; ++i) out[i] = I[i];
  return true;
}

}  // namespace g2oc
